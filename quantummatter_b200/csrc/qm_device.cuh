// qm_device.cuh -- device-side helpers shared by the kernels of libqmb200.so.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace qm {

// Interleaved complex element of a state: double2 (complex128) or float2 (complex64).
template <typename T> struct Vec2;
template <> struct Vec2<double> { using type = double2; };
template <> struct Vec2<float> { using type = float2; };

template <typename T> struct Cx { T re, im; };

template <typename T>
__device__ __forceinline__ Cx<T> load_amp(const typename Vec2<T>::type* p, uint64_t i) {
    typename Vec2<T>::type v = p[i];
    return Cx<T>{v.x, v.y};
}
template <typename T>
__device__ __forceinline__ void store_amp(typename Vec2<T>::type* p, uint64_t i, Cx<T> v) {
    typename Vec2<T>::type o;
    o.x = v.re;
    o.y = v.im;
    p[i] = o;
}

// (a) * (x) for complex a, x.
template <typename T>
__device__ __forceinline__ Cx<T> cmul(T ar, T ai, Cx<T> x) {
    return Cx<T>{ar * x.re - ai * x.im, ar * x.im + ai * x.re};
}
// a*x + b*y
template <typename T>
__device__ __forceinline__ Cx<T> cmac2(T ar, T ai, Cx<T> x, T br, T bi, Cx<T> y) {
    Cx<T> o;
    o.re = ar * x.re - ai * x.im + br * y.re - bi * y.im;
    o.im = ar * x.im + ai * x.re + br * y.im + bi * y.re;
    return o;
}

// Inserts a zero bit at position `pos` of x: the pair enumeration of
// CudaStateVectorKernel.cs:41-43 (low = pair & (bit-1); first = ((pair-low)<<1)|low).
__device__ __forceinline__ uint32_t insert_zero(uint32_t x, int pos) {
    uint32_t low = x & ((1u << pos) - 1u);
    return ((x - low) << 1) | low;
}

// Scatters the low bits of `value` onto the set bits of `mask` (bit deposit).
__device__ __forceinline__ uint32_t deposit(uint32_t value, uint32_t mask) {
    uint32_t out = 0;
    while (mask) {
        uint32_t low = mask & (0u - mask);
        if (value & 1u) out |= low;
        value >>= 1;
        mask ^= low;
    }
    return out;
}

// One tensor-map box (cp.async.bulk.tensor) between global and shared memory: `map` is the address
// of a __grid_constant__ CUtensorMap, `rank` its dimensions (1..5), c the box coordinates.  The load
// completes on the mbarrier at shared address `bar`; the store joins the thread's bulk group.
__device__ __forceinline__ void tma_box_load(const void* map, int rank, uint32_t dst, uint32_t bar, const int32_t* c) {
    const uint64_t m = reinterpret_cast<uint64_t>(map);
    switch (rank) {
    case 1:
        asm volatile("cp.async.bulk.tensor.1d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2}], [%3];"
                     ::"r"(dst), "l"(m), "r"(c[0]), "r"(bar) : "memory");
        break;
    case 2:
        asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
                     ::"r"(dst), "l"(m), "r"(c[0]), "r"(c[1]), "r"(bar) : "memory");
        break;
    case 3:
        asm volatile("cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
                     ::"r"(dst), "l"(m), "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(bar) : "memory");
        break;
    case 4:
        asm volatile("cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];"
                     ::"r"(dst), "l"(m), "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(c[3]), "r"(bar) : "memory");
        break;
    default:
        asm volatile("cp.async.bulk.tensor.5d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5, %6}], [%7];"
                     ::"r"(dst), "l"(m), "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(c[3]), "r"(c[4]), "r"(bar) : "memory");
        break;
    }
}

__device__ __forceinline__ void tma_box_store(const void* map, int rank, uint32_t src, const int32_t* c) {
    const uint64_t m = reinterpret_cast<uint64_t>(map);
    switch (rank) {
    case 1:
        asm volatile("cp.async.bulk.tensor.1d.global.shared::cta.bulk_group [%0, {%1}], [%2];" ::"l"(m), "r"(c[0]), "r"(src)
                     : "memory");
        break;
    case 2:
        asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%1, %2}], [%3];" ::"l"(m), "r"(c[0]),
                     "r"(c[1]), "r"(src) : "memory");
        break;
    case 3:
        asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%1, %2, %3}], [%4];" ::"l"(m), "r"(c[0]),
                     "r"(c[1]), "r"(c[2]), "r"(src) : "memory");
        break;
    case 4:
        asm volatile("cp.async.bulk.tensor.4d.global.shared::cta.bulk_group [%0, {%1, %2, %3, %4}], [%5];" ::"l"(m),
                     "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(c[3]), "r"(src) : "memory");
        break;
    default:
        asm volatile("cp.async.bulk.tensor.5d.global.shared::cta.bulk_group [%0, {%1, %2, %3, %4, %5}], [%6];" ::"l"(m),
                     "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(c[3]), "r"(c[4]), "r"(src) : "memory");
        break;
    }
}

// Box coordinates of a work item whose outer index bits are `base`: 0 on tile dimensions, the
// item's bits on the others.
// Box coordinates of tile `item`: the tile's outer index bits, in increasing order, are the
// concatenated coordinates of the box-size-1 dimensions (tile dimensions start at 0).
__device__ __forceinline__ void tma_item_coords(int rank, const int32_t* len, const int32_t* tile, uint32_t item,
                                                int32_t* c) {
    int shift = 0;
#pragma unroll
    for (int d = 0; d < 5; ++d) {
        const bool outer = d < rank && !tile[d];
        const uint32_t mask = len[d] >= 32 ? 0xffffffffu : (1u << len[d]) - 1u;
        c[d] = (outer && shift < 32) ? (int32_t)((item >> shift) & mask) : 0;
        if (outer) shift += len[d];
    }
}

// Brings a __grid_constant__ tensor map into the descriptor cache ahead of its first use.
__device__ __forceinline__ void tma_prefetch(const void* map) {
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

// Compensated FP64 accumulation (Neumaier): sum + comp carries the exact running total
// to within one rounding of the largest partial.
struct KSum {
    double s, c;
    __device__ __forceinline__ void add(double v) {
        double t = s + v;
        c += fabs(s) >= fabs(v) ? (s - t) + v : (v - t) + s;
        s = t;
    }
    __device__ __forceinline__ void merge(const KSum& o) {
        add(o.s);
        c += o.c;
    }
    __device__ __forceinline__ double value() const { return s + c; }
};

__device__ __forceinline__ KSum shfl_down_ksum(KSum v, int delta) {
    KSum o;
    o.s = __shfl_down_sync(0xffffffffu, v.s, delta);
    o.c = __shfl_down_sync(0xffffffffu, v.c, delta);
    return o;
}

// Reduces one KSum per thread of the block to thread 0 (deterministic tree order).
// `shared` needs blockDim.x/32 entries.
__device__ __forceinline__ KSum block_reduce_ksum(KSum v, KSum* shared) {
    for (int d = 16; d > 0; d >>= 1) v.merge(shfl_down_ksum(v, d));
    int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __syncthreads();
    if (lane == 0) shared[warp] = v;
    __syncthreads();
    int warps = (blockDim.x + 31) >> 5;
    if (warp == 0) {
        v = lane < warps ? shared[lane] : KSum{0.0, 0.0};
        for (int d = 16; d > 0; d >>= 1) v.merge(shfl_down_ksum(v, d));
    }
    return v;
}

}  // namespace qm
