// qm_dense.cu -- kernels of the dense fused gates (fusion widths 2..6, planned by qm_dense.cpp).
//
// A fused gate on m <= 6 qubits Q is a dense 2^m x 2^m unitary U applied to every column of the
// state: out(a, c) = sum_b U(a, b) in(b, c), where b, a enumerate the Q bits and c the others.
// A CTA tile holds 2^m rows and 2^c columns (m + c = 12, 4096 amplitudes): the columns are the
// lowest c index bits outside Q, so global memory is read in runs.
//
// Staging: the tile travels between HBM and shared memory by bulk copies (cp.async.bulk, the TMA
// unit's untiled form) that complete on an mbarrier, in a ring of 2-4 buffers: while the CTA
// computes one tile, the next ones load, and the previous one is written back by bulk stores from
// the same buffer.  Each copy moves one run of global index bits [0, r), chosen so that inside a
// run every column bit lies below every Q bit; runs of 128 bytes or more are spaced 16 bytes apart
// in shared memory, so the column accesses of a warp hit distinct banks.
//
// Arithmetic: each of the 256 threads owns a 4 x 4 block of (row, column) outputs (2 x 8 for
// m = 1) and walks b over the 2^m rows of the tile: four complex FMAs per output and step, with
// U(a, b) for consecutive a read as one row of the transposed unitary (a broadcast within the
// warp's rows).  Complex128 states compute in FP64, complex64 states in FP32.
//
// Every wait on an mbarrier is bounded (about a second of clock cycles); a wait that runs out
// records QM_E_TIMEOUT in the launch's status word and the CTA waits, again bounded, for its own
// copies in flight before it returns.
#include <cuda.h>
#include <cuda_runtime.h>

#include <atomic>

#include <algorithm>
#include <cstdlib>
#include <mutex>

#include "qm_device.cuh"
#include "qm_internal.h"

namespace qm {

namespace {

constexpr int kDenseThreads = 256;
constexpr int kDenseTileBits = 12;
constexpr int kDenseMaxBufs = 4;
constexpr long long kWaitCycles = 2000000000ll;  // about one second at the B200's clocks
constexpr int kDenseSmemMax = 226 * 1024;        // dynamic shared memory; the static part stays below 1 KiB

constexpr int kTmaMaxRank = 5;

struct DenseLaunch {
    // Tensor-map path: the tile is one box of a tensor map over the state whose dimensions are the
    // runs of tile and outer index bits from bit 0 up (tile runs: full extent in the box; outer
    // runs: extent 1, coordinate from the work item); one cp.async.bulk.tensor moves the tile.
    CUtensorMap tmap;
    int32_t tma_rank;         // 0: bulk copies of runs instead
    int32_t tma_lo[kTmaMaxRank], tma_len[kTmaMaxRank], tma_tile[kTmaMaxRank];
    const double2* matrix;    // transposed unitary: row b holds U(a, b) for a = 0 .. 2^m-1
    int32_t* status;          // QM_E_TIMEOUT after a wait that ran out
    uint64_t items;           // tiles
    uint32_t outer_mask;      // global bits enumerated by the tile index
    uint32_t copy_mask;       // tile bits above the run, enumerated by the copy index
    int32_t q_bits[kDenseMaxQubits];
    int32_t l_bits[kDenseTileBits];
    int32_t m;                // fused qubits
    int32_t cols_bits;        // c: column bits of the tile
    int32_t run_bits;         // r: the layout's runs are global bits [0, r)
    int32_t copies;           // 2^(12 - r) runs per tile
    int32_t stride;           // elements between consecutive runs in shared memory
    // The bulk copies: runs of global bits [0, xfer_bits), one per value of the tile bits in
    // xfer_mask, xfer_stride elements apart.  Unpadded layouts (runs under 128 bytes) are the tile's
    // natural index order, so their copies take the longest natural runs instead.
    uint32_t xfer_mask;
    int32_t xfer_bits, xfers, xfer_stride, xfer_pad;
    int32_t nbuf;             // buffers in the ring
    int32_t buf_elems;        // elements per buffer
    int32_t buf_offset;       // byte offset of the first buffer in dynamic shared memory
    int32_t pad;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return done != 0;
}

// Waits for the phase with the given parity to complete; false after about a second.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
    if (mbar_try_wait(bar, parity)) return true;
    const long long start = clock64();
    while (!mbar_try_wait(bar, parity))
        if (clock64() - start > kWaitCycles) return false;
    return true;
}

__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void bulk_store(void* dst, const void* src, uint32_t bytes) {
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst), "r"(smem_u32(src)),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

template <typename V>
__device__ __forceinline__ void issue_tile_load(const DenseLaunch& P, const V* s, V* buf, uint64_t* bar,
                                                uint64_t item, int lane) {
    if (P.tma_rank) {
        if (lane == 0) {
            int32_t c[kTmaMaxRank];
            tma_item_coords(P.tma_rank, P.tma_len, P.tma_tile, (uint32_t)item, c);
            mbar_arrive_expect_tx(bar, (uint32_t)sizeof(V) << (P.cols_bits + P.m));
            tma_box_load(&P.tmap, P.tma_rank, smem_u32(buf), smem_u32(bar), c);
        }
        return;
    }
    const uint32_t base = deposit((uint32_t)item, P.outer_mask);
    const uint32_t run_bytes = (uint32_t)sizeof(V) << P.xfer_bits;
    if (lane == 0) mbar_arrive_expect_tx(bar, run_bytes * (uint32_t)P.xfers);
    __syncwarp();
    for (int x = lane; x < P.xfers; x += 32)
        bulk_load(buf + (size_t)x * P.xfer_stride, s + (base | deposit((uint32_t)x, P.xfer_mask)), run_bytes, bar);
}

template <typename V>
__device__ __forceinline__ void issue_tile_store(const DenseLaunch& P, V* s, const V* buf, uint64_t item, int lane) {
    if (P.tma_rank) {
        if (lane == 0) {
            int32_t c[kTmaMaxRank];
            tma_item_coords(P.tma_rank, P.tma_len, P.tma_tile, (uint32_t)item, c);
            tma_box_store(&P.tmap, P.tma_rank, smem_u32(buf), c);
            bulk_commit();
        }
        return;
    }
    const uint32_t base = deposit((uint32_t)item, P.outer_mask);
    const uint32_t run_bytes = (uint32_t)sizeof(V) << P.xfer_bits;
    for (int x = lane; x < P.xfers; x += 32)
        bulk_store(s + (base | deposit((uint32_t)x, P.xfer_mask)), buf + (size_t)x * P.xfer_stride, run_bytes);
    bulk_commit();
}

// shared-memory element offset of global bit g inside a tile
__device__ __forceinline__ int tile_weight(const DenseLaunch& P, int g) {
    if (g < P.run_bits) return 1 << g;
    return P.stride << __popc(P.copy_mask & ((1u << g) - 1u));
}

template <typename T, int M>
__global__ void __launch_bounds__(kDenseThreads, 1)
    k_dense(typename Vec2<T>::type* __restrict__ s, const __grid_constant__ DenseLaunch P) {
    using V = typename Vec2<T>::type;
    constexpr int D = 1 << M;
    constexpr int RA = D < 4 ? D : 4;  // rows per thread
    constexpr int RC = 16 / RA;        // columns per thread
    constexpr int RG = D / RA;         // row groups
    extern __shared__ __align__(128) unsigned char smem[];
    V* U = reinterpret_cast<V*>(smem);                                   // [b][a]
    int* wq = reinterpret_cast<int*>(smem + sizeof(V) * D * D);          // [b]
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + sizeof(V) * D * D + sizeof(int) * 64);
    V* bufs = reinterpret_cast<V*>(smem + P.buf_offset);
    __shared__ int abort_flag;

    const int t = threadIdx.x, lane = t & 31;
    const int nt = blockDim.x;
    const int CG = nt / RG;  // column groups
    const int cg = t % CG, rg = t / CG;

    for (int i = t; i < D * D; i += nt) {
        const double2 u = P.matrix[i];
        V v;
        v.x = (T)u.x;
        v.y = (T)u.y;
        U[i] = v;
    }
    for (int b = t; b < D; b += nt) {
        int w = 0;
        for (int i = 0; i < M; ++i)
            if ((b >> i) & 1) w += tile_weight(P, P.q_bits[i]);
        wq[b] = w;
    }
    int wbit[M];
#pragma unroll
    for (int q = 0; q < M; ++q) wbit[q] = tile_weight(P, P.q_bits[q]);
    int wl[RC];
#pragma unroll
    for (int i = 0; i < RC; ++i) {
        const int j = cg + CG * i;
        int w = 0;
        for (int k = 0; k < P.cols_bits; ++k)
            if ((j >> k) & 1) w += tile_weight(P, P.l_bits[k]);
        wl[i] = w;
    }
    if (t == 0) {
        if (P.tma_rank) tma_prefetch(&P.tmap);
        for (int b = 0; b < P.nbuf; ++b) mbar_init(&bar[b], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        abort_flag = 0;
    }
    __syncthreads();

    const uint64_t step = gridDim.x;
    if (t < 32) {
        for (int k = 0; k < P.nbuf - 1; ++k) {
            const uint64_t it = blockIdx.x + k * step;
            if (it < P.items) issue_tile_load<V>(P, s, bufs + (size_t)k * P.buf_elems, &bar[k], it, lane);
        }
    }

    int i = 0;
    uint64_t it = blockIdx.x;
    for (; it < P.items; it += step, ++i) {
        const int cur = i % P.nbuf;
        if (t < 32) {
            const uint64_t nxt = it + (uint64_t)(P.nbuf - 1) * step;
            if (nxt < P.items) {
                const int nb = (i + P.nbuf - 1) % P.nbuf;
                bulk_wait_read();  // this lane's stores out of that buffer have read it
                fence_proxy_async();
                __syncwarp();
                issue_tile_load<V>(P, s, bufs + (size_t)nb * P.buf_elems, &bar[nb], nxt, lane);
            }
        }
        if (!mbar_wait_bounded(&bar[cur], (uint32_t)(i / P.nbuf) & 1u)) abort_flag = 1;
        __syncthreads();
        if (abort_flag) break;
        V* tile = bufs + (size_t)cur * P.buf_elems;

        T ar[RA][RC], ai[RA][RC];
#pragma unroll
        for (int r = 0; r < RA; ++r)
#pragma unroll
            for (int c = 0; c < RC; ++c) ar[r][c] = ai[r][c] = (T)0;
        const V* col[RC];
#pragma unroll
        for (int c = 0; c < RC; ++c) col[c] = tile + wl[c];
#pragma unroll
        for (int b = 0; b < D; ++b) {
            // row b's offset: the sum of its fused bits' weights (b is a constant after unrolling)
            int off = 0;
#pragma unroll
            for (int q = 0; q < M; ++q)
                if ((b >> q) & 1) off += wbit[q];
            V x[RC], u[RA];
#pragma unroll
            for (int c = 0; c < RC; ++c) x[c] = col[c][off];
#pragma unroll
            for (int r = 0; r < RA; ++r) u[r] = U[b * D + rg * RA + r];
#pragma unroll
            for (int r = 0; r < RA; ++r)
#pragma unroll
                for (int c = 0; c < RC; ++c) {
                    ar[r][c] = fma(u[r].x, x[c].x, ar[r][c]);
                    ar[r][c] = fma(-u[r].y, x[c].y, ar[r][c]);
                    ai[r][c] = fma(u[r].x, x[c].y, ai[r][c]);
                    ai[r][c] = fma(u[r].y, x[c].x, ai[r][c]);
                }
        }
        __syncthreads();  // every thread has read the tile
#pragma unroll
        for (int r = 0; r < RA; ++r) {
            const int off = wq[rg * RA + r];
#pragma unroll
            for (int c = 0; c < RC; ++c) {
                V o;
                o.x = ar[r][c];
                o.y = ai[r][c];
                tile[off + wl[c]] = o;
            }
        }
        fence_proxy_async();  // the bulk stores (async proxy) read what these threads wrote
        __syncthreads();
        if (t < 32) issue_tile_store<V>(P, s, tile, it, lane);
    }
    if (abort_flag) {
        if (t == 0) atomicExch(P.status, (int32_t)QM_E_TIMEOUT);
        // loads already issued for the tiles after the one that timed out
        if (t == 0)
            for (int k = 1; k < P.nbuf; ++k) {
                const uint64_t later = it + (uint64_t)k * step;
                if (later < P.items) mbar_wait_bounded(&bar[(i + k) % P.nbuf], (uint32_t)((i + k) / P.nbuf) & 1u);
            }
    }
    if (t < 32) bulk_wait_all();
}

// States of fewer than 9 qubits: one CTA holds the whole state in shared memory.
template <typename T>
__global__ void __launch_bounds__(256) k_dense_small(typename Vec2<T>::type* __restrict__ s, const double2* matrix,
                                                      uint32_t qmask, int m, int qubits) {
    using V = typename Vec2<T>::type;
    __shared__ V in[256];
    const uint32_t n = 1u << qubits, dim = 1u << m;
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) in[i] = s[i];
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
        const uint32_t rest = i & ~qmask;
        uint32_t a = 0;
        for (int k = 0, bit = 0; k < 32; ++k)
            if (qmask & (1u << k)) {
                if (i & (1u << k)) a |= 1u << bit;
                ++bit;
            }
        T re = 0, im = 0;
        for (uint32_t b = 0; b < dim; ++b) {
            const double2 u = matrix[(size_t)b * dim + a];
            const V x = in[rest | deposit(b, qmask)];
            re = fma((T)u.x, x.x, re);
            re = fma(-(T)u.y, x.y, re);
            im = fma((T)u.x, x.y, im);
            im = fma((T)u.y, x.x, im);
        }
        V o;
        o.x = re;
        o.y = im;
        s[i] = o;
    }
}

template <typename T, int M>
cudaError_t launch_dense_m(void* amps, const DenseLaunch& P, int grid, int threads, size_t smem, cudaStream_t st) {
    static std::once_flag once;
    static cudaError_t attr = cudaSuccess;
    std::call_once(once, [] {
        attr = cudaFuncSetAttribute(k_dense<T, M>, cudaFuncAttributeMaxDynamicSharedMemorySize, kDenseSmemMax);
    });
    if (attr != cudaSuccess) return attr;
    k_dense<T, M><<<grid, threads, smem, st>>>(reinterpret_cast<typename Vec2<T>::type*>(amps), P);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_dense_t(void* amps, int m, const DenseLaunch& P, int grid, int threads, size_t smem,
                           cudaStream_t st) {
    switch (m) {
    case 1: return launch_dense_m<T, 1>(amps, P, grid, threads, smem, st);
    case 2: return launch_dense_m<T, 2>(amps, P, grid, threads, smem, st);
    case 3: return launch_dense_m<T, 3>(amps, P, grid, threads, smem, st);
    case 4: return launch_dense_m<T, 4>(amps, P, grid, threads, smem, st);
    case 5: return launch_dense_m<T, 5>(amps, P, grid, threads, smem, st);
    case 6: return launch_dense_m<T, 6>(amps, P, grid, threads, smem, st);
    default: return cudaErrorInvalidValue;
    }
}

using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// cuTensorMapEncodeTiled from the driver, through the runtime (the library does not link libcuda)
EncodeTiled tensor_map_encoder() {
    static const EncodeTiled fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return (EncodeTiled) nullptr;
        return reinterpret_cast<EncodeTiled>(p);
    }();
    return fn;
}

}  // namespace

bool dense_tma_enabled() {
    static const bool on = [] {
        const char* e = std::getenv("QM_DENSE_TMA");
        return !(e && e[0] == '0');
    }();
    return on;
}

bool tile_map_dims(uint32_t tile_mask, int qubits, int32_t* lo, int32_t* len, int32_t* tile, int32_t* rank) {
    // runs of tile / outer bits from bit 0 up; a tile run is split into boxes of at most 2^7
    // elements for the innermost dimension (256 scalars) and 2^8 otherwise
    int r = 0, b = 0;
    while (b < qubits) {
        const bool in = (tile_mask >> b) & 1u;
        int n = 0;
        while (b + n < qubits && (((tile_mask >> (b + n)) & 1u) != 0) == in) ++n;
        int at = b;
        while (n > 0) {
            const int cap = in ? (r == 0 ? 7 : 8) : 32;
            const int l = std::min(n, cap);
            if (r == kDenseTmaMaxRank) return false;
            lo[r] = at;
            len[r] = l;
            tile[r] = in ? 1 : 0;
            ++r;
            at += l;
            n -= l;
        }
        b = at;
    }
    *rank = r;
    return r > 0 && tile[0] == 1;
}

bool encode_tile_map(CUtensorMap* map, void* amps, int precision, int rank, const int32_t* lo, const int32_t* len,
                     const int32_t* tile) {
    auto encode = tensor_map_encoder();
    if (!encode || rank < 1 || rank > kDenseTmaMaxRank) return false;
    cuuint64_t dims[kDenseTmaMaxRank], strides[kDenseTmaMaxRank];
    cuuint32_t box[kDenseTmaMaxRank], estr[kDenseTmaMaxRank];
    const int elem = precision == QM_FP32 ? 8 : 16;
    for (int d = 0; d < rank; ++d) {
        dims[d] = (cuuint64_t)1 << len[d];
        box[d] = tile[d] ? (cuuint32_t)1 << len[d] : 1u;
        estr[d] = 1;
        if (d > 0) strides[d - 1] = (cuuint64_t)elem << lo[d];
    }
    dims[0] *= 2;  // the innermost dimension counts scalars: (re, im) pairs
    box[0] *= 2;
    return encode(map, precision == QM_FP32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64,
                  (cuuint32_t)rank, amps, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                  CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

bool dense_geometry(int qubits, int precision, const DenseOp& op, DenseGeometry& g) {
    const int m = op.m;
    if (m < 1 || m > kDenseMaxQubits || qubits < 9) return false;
    const int elem = precision == QM_FP32 ? 8 : 16;
    uint32_t qmask = 0;
    for (int i = 0; i < m; ++i) qmask |= 1u << op.q[i];
    const int tb = std::min(kDenseTileBits, qubits);
    const int c = tb - m;
    uint32_t lmask = 0;
    int nl = 0;
    for (int b = 0; b < qubits && nl < c; ++b)
        if (!(qmask & (1u << b))) {
            lmask |= 1u << b;
            g.l_bits[nl++] = b;
        }
    // run: global bits [0, r) inside the tile, every column bit below every Q bit
    int r = 0;
    bool seen_q = false;
    while (r < qubits && ((qmask | lmask) >> r & 1u)) {
        const bool is_q = (qmask >> r) & 1u;
        if (!is_q && seen_q) break;
        seen_q = seen_q || is_q;
        ++r;
    }
    g.qmask = qmask;
    g.lmask = lmask;
    g.cols_bits = c;
    g.run_bits = r;
    g.copy_mask = (qmask | lmask) & ~((1u << r) - 1u);
    g.copies = 1 << (tb - r);
    const int run_bytes = elem << r;
    // A tensor-map box is the unpadded natural order, whose column accesses are free of bank
    // conflicts when the lowest index bits (a wavefront's worth: 8 complex128, 16 complex64) are
    // column bits; otherwise only 1- and 2-qubit gates (too little arithmetic to mind) take it.
    g.tma_rank = 0;
    {
        const int low = precision == QM_FP32 ? 4 : 3;
        const bool contiguous_columns = (lmask & ((1u << low) - 1u)) == ((1u << low) - 1u);
        int32_t rank = 0;
        if (dense_tma_enabled() && (contiguous_columns || m <= 2) &&
            tile_map_dims(qmask | lmask, qubits, g.tma_lo, g.tma_len, g.tma_tile, &rank))
            g.tma_rank = rank;
    }
    // padding keeps column accesses free of bank conflicts, but a tensor-map box is unpadded
    const int pad = (run_bytes >= 128 && g.tma_rank == 0) ? 16 / elem : 0;
    g.stride = (1 << r) + pad;
    // copies: the layout's runs when padded, else the longest natural runs of the tile
    int rn = r;
    if (pad == 0)
        while (rn < qubits && rn < 31 && ((qmask | lmask) >> rn & 1u)) ++rn;
    g.xfer_bits = rn;
    g.xfer_mask = (qmask | lmask) & ~((1u << rn) - 1u);
    g.xfers = 1 << (tb - rn);
    g.xfer_stride = pad == 0 ? (1 << rn) : g.stride;
    const int buf_bytes = ((g.copies * g.stride * elem + 127) / 128) * 128;
    g.buf_elems = buf_bytes / elem;
    const int header = ((elem * (1 << m) * (1 << m) + 4 * 64 + 8 * kDenseMaxBufs + 127) / 128) * 128;
    const int budget = kDenseSmemMax;
    g.nbuf = std::min(kDenseMaxBufs, (budget - header) / buf_bytes);
    if (g.nbuf < 2) return false;
    g.buf_offset = header;
    g.smem = (size_t)header + (size_t)g.nbuf * buf_bytes;
    g.outer_mask = ((qubits >= 32 ? 0xffffffffu : (1u << qubits) - 1u)) & ~(qmask | lmask);
    g.items = uint64_t(1) << (qubits - tb);
    return true;
}

std::atomic<int64_t> g_dense_launches{0}, g_dense_tc_launches{0};

cudaError_t launch_dense(void* amps, int qubits, int precision, const DenseOp& op, const double2* matrix,
                         int32_t* status, int sm_count, cudaStream_t st) {
    uint32_t qmask = 0;
    for (int i = 0; i < op.m; ++i) qmask |= 1u << op.q[i];
    if (qubits < 9) {
        g_dense_launches.fetch_add(1, std::memory_order_relaxed);
        if (precision == QM_FP32)
            k_dense_small<float><<<1, 256, 0, st>>>(reinterpret_cast<float2*>(amps), matrix, qmask, op.m, qubits);
        else
            k_dense_small<double><<<1, 256, 0, st>>>(reinterpret_cast<double2*>(amps), matrix, qmask, op.m, qubits);
        return cudaGetLastError();
    }
    DenseGeometry g;
    if (!dense_geometry(qubits, precision, op, g)) return cudaErrorInvalidValue;
    DenseLaunch P{};
    P.matrix = matrix;
    P.status = status;
    P.items = g.items;
    P.outer_mask = g.outer_mask;
    P.copy_mask = g.copy_mask;
    for (int i = 0; i < op.m; ++i) P.q_bits[i] = op.q[i];
    for (int i = 0; i < g.cols_bits; ++i) P.l_bits[i] = g.l_bits[i];
    P.cols_bits = g.cols_bits;
    P.run_bits = g.run_bits;
    P.copies = g.copies;
    P.stride = g.stride;
    P.xfer_mask = g.xfer_mask;
    P.xfer_bits = g.xfer_bits;
    P.xfers = g.xfers;
    P.xfer_stride = g.xfer_stride;
    P.m = op.m;
    P.tma_rank = 0;
    if (g.tma_rank) {
        if (encode_tile_map(&P.tmap, amps, precision, g.tma_rank, g.tma_lo, g.tma_len, g.tma_tile)) {
            P.tma_rank = g.tma_rank;
            for (int d = 0; d < g.tma_rank; ++d) {
                P.tma_lo[d] = g.tma_lo[d];
                P.tma_len[d] = g.tma_len[d];
                P.tma_tile[d] = g.tma_tile[d];
            }
        }
        if (!P.tma_rank) {
            // no encoder: the unpadded layout's natural runs through bulk copies
            P.xfer_bits = g.run_bits;
            P.xfer_mask = g.copy_mask;
            P.xfers = g.copies;
            P.xfer_stride = g.stride;
            int rn = g.run_bits;
            while (rn < qubits && ((g.qmask | g.lmask) >> rn & 1u)) ++rn;
            P.xfer_bits = rn;
            P.xfer_mask = (g.qmask | g.lmask) & ~((1u << rn) - 1u);
            P.xfers = 1 << (g.cols_bits + op.m - rn);
            P.xfer_stride = 1 << rn;
        }
    }
    P.nbuf = g.nbuf;
    P.buf_elems = g.buf_elems;
    P.buf_offset = g.buf_offset;
    const int grid = (int)std::min<uint64_t>(g.items, (uint64_t)std::max(1, sm_count));
    g_dense_launches.fetch_add(1, std::memory_order_relaxed);
    // 16 outputs per thread: 256 threads for a 4096-amplitude tile, 32 for the 512 of a 9-qubit state
    const int threads = 1 << (g.cols_bits + op.m - 4);
    if (precision == QM_FP32) return launch_dense_t<float>(amps, op.m, P, grid, threads, g.smem, st);
    return launch_dense_t<double>(amps, op.m, P, grid, threads, g.smem, st);
}

}  // namespace qm

// Launch counts of the dense fused-gate kernels since the library was loaded: all of them, and
// those that ran on the tensor cores.
extern "C" int32_t qm_dense_info(int64_t* launches, int64_t* tensor_core_launches) {
    if (launches) *launches = qm::g_dense_launches.load() + qm::g_dense_tc_launches.load();
    if (tensor_core_launches) *tensor_core_launches = qm::g_dense_tc_launches.load();
    return QM_OK;
}
