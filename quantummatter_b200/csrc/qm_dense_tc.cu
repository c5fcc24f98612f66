// qm_dense_tc.cu -- dense 6-qubit fused gates on complex64 states through the tensor cores.
//
// A fused gate on 6 qubits costs 64 complex multiply-adds per amplitude, 512 FP32 flops: more
// than the FP32 pipes deliver at the HBM rate, so these gates (and 5-qubit gates, widened to 6
// qubits by the planner) run here as real GEMMs on tcgen05:
//
//   D[128 x N] = A[128 x 64] * B[64 x N]
//   A row 2a + p, column b:  p = 0: Re U(a, b),  p = 1: Im U(a, b)
//   B row b, column 2j + c:  c = 0: Re in(b, j),  c = 1: Im in(b, j)
//   out(a, j) = (D[2a][2j] - D[2a+1][2j+1]) + i (D[2a][2j+1] + D[2a+1][2j])
//
// FP32 accuracy from TF32 operands: each operand is split into a TF32 head and an FP32 tail
// (x = hi + lo exactly, hi with the low 13 mantissa bits cleared) and D accumulates in FP32 the
// three products hi*hi + hi*lo + lo*hi (the 3xTF32 scheme).  A's split is done once on the host.
//
// Per CTA (one per SM), for a ring of tiles of 64 rows x 32 columns (2048 amplitudes, 16 KiB):
//   - bulk copies (cp.async.bulk, mbarrier completion) stage each tile into one of four buffers,
//     three tiles ahead of the one being converted;
//   - all 256 threads split the tile into B_hi / B_lo in the canonical K-major layout of the
//     MMA (two B buffers, so tile i converts while tile i-1's MMAs run);
//   - one thread issues the 24 MMAs of the tile (8 K-steps x 3 products, M = 128, N = 64, K = 8)
//     into one of two TMEM accumulators and commits them to an mbarrier;
//   - the previous tile's accumulator is read back with tcgen05.ld, the real/imaginary rows are
//     combined across lane pairs, written over that tile's staging buffer and bulk-stored.
// Every mbarrier wait is bounded; after one runs out the CTA records QM_E_TIMEOUT, waits (bounded)
// for its MMAs and copies in flight, frees its TMEM and returns.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>

#include "qm_device.cuh"
#include "qm_internal.h"

namespace qm {

namespace {

constexpr int kTcThreads = 256;
constexpr int kTcTileBits = 11;      // 64 rows x 32 columns
constexpr int kTcCols = 32;          // complex columns per tile
constexpr int kTcN = 2 * kTcCols;    // real columns of B and D
constexpr int kTcStages = 4;         // staging buffers
constexpr int kTmemCols = 2 * kTcN;  // two accumulators
constexpr long long kTcWaitCycles = 2000000000ll;
constexpr size_t kTcSmemMax = 220 * 1024;

// shared-memory layout (bytes)
constexpr int kAHalf = 128 * 64 * 4;           // one 128 x 64 TF32 operand image: 32 KiB
// B, K-major without swizzle: core matrices of 8 real columns (n) x 4 rows (k, 16 bytes); the 16
// k-groups of a column group 144 bytes apart (16 more than dense, so the conversion's stores of
// k and k + 4 land in different banks), column groups 2304 bytes apart
constexpr int kBLbo = 144;
constexpr int kBSbo = 16 * kBLbo;              // 2304
constexpr int kBHalf = (kTcN / 8) * kBSbo;     // one 64 x 64 B image: 18432 B
constexpr int kOffA = 0;                       // A_hi, A_lo
constexpr int kOffB = 2 * kAHalf;              // [2 buffers][hi, lo]
constexpr int kOffStage = kOffB + 4 * kBHalf;  // staging ring, stage_bytes each

struct TcLaunch {
    const float* a_image;    // A_hi then A_lo, already in the MMA's K-major layout (64 KiB)
    int32_t* status;
    uint64_t items;
    uint32_t outer_mask, copy_mask;
    int32_t q_bits[6];
    int32_t l_bits[kTcTileBits];
    int32_t cols_bits, run_bits, copies, stride, stage_elems, pad;
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
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
    if (mbar_try_wait(bar, parity)) return true;
    const long long start = clock64();
    while (!mbar_try_wait(bar, parity))
        if (clock64() - start > kTcWaitCycles) return false;
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
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Shared-memory matrix descriptor, no swizzle: start, leading (K-direction) and stride
// (M/N-direction) byte offsets of the 8 x 16-byte core matrices, descriptor version 1.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3fffu);
    d |= (uint64_t)((lbo >> 4) & 0x3fffu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3fffu) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

// Instruction descriptor of kind::tf32: FP32 accumulator, TF32 A and B both K-major (an MN-major
// TF32 operand without swizzle reads as zeros on B200), M = 128, N = kTcN.
constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(kTcN >> 3) << 17) |
                            ((uint32_t)(128 >> 4) << 24);

__device__ __forceinline__ void mma_tf32(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.u32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(kIdesc), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ int tile_weight(const TcLaunch& P, int g) {
    if (g < P.run_bits) return 1 << g;
    return P.stride << __popc(P.copy_mask & ((1u << g) - 1u));
}

__device__ __forceinline__ void issue_load(const TcLaunch& P, const float2* s, float2* buf, uint64_t* bar,
                                           uint64_t item, int lane) {
    const uint32_t base = deposit((uint32_t)item, P.outer_mask);
    const uint32_t run_bytes = 8u << P.run_bits;
    if (lane == 0) mbar_arrive_expect_tx(bar, run_bytes * (uint32_t)P.copies);
    __syncwarp();
    for (int x = lane; x < P.copies; x += 32)
        bulk_load(buf + (size_t)x * P.stride, s + (base | deposit((uint32_t)x, P.copy_mask)), run_bytes, bar);
}

__device__ __forceinline__ void issue_store(const TcLaunch& P, float2* s, const float2* buf, uint64_t item, int lane) {
    const uint32_t base = deposit((uint32_t)item, P.outer_mask);
    const uint32_t run_bytes = 8u << P.run_bits;
    for (int x = lane; x < P.copies; x += 32)
        bulk_store(s + (base | deposit((uint32_t)x, P.copy_mask)), buf + (size_t)x * P.stride, run_bytes);
    bulk_commit();
}

__device__ __forceinline__ float tf32_head(float x) { return __uint_as_float(__float_as_uint(x) & 0xffffe000u); }

__global__ void __launch_bounds__(kTcThreads, 1) k_dense_tc(float2* __restrict__ s, const __grid_constant__ TcLaunch P) {
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ uint64_t bar_load[kTcStages];
    __shared__ uint64_t bar_mma[2];
    __shared__ uint64_t bar_a;
    __shared__ uint32_t tmem_base;
    __shared__ int wq[64];
    __shared__ int abort_flag;

    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    float* a_img = reinterpret_cast<float*>(smem + kOffA);
    unsigned char* b_img = smem + kOffB;
    float2* stage = reinterpret_cast<float2*>(smem + kOffStage);

    for (int b = t; b < 64; b += kTcThreads) {
        int w = 0;
        for (int i = 0; i < 6; ++i)
            if ((b >> i) & 1) w += tile_weight(P, P.q_bits[i]);
        wq[b] = w;
    }
    // conversion: thread t takes elements e = t + 256 * k (k < 8): b % 8 = e & 7, j = (e >> 3) & 31,
    // b / 8 = e >> 8
    int wl_conv = 0;
    {
        const int j = (t >> 3) & 31;
        for (int k = 0; k < P.cols_bits; ++k)
            if ((j >> k) & 1) wl_conv += tile_weight(P, P.l_bits[k]);
    }
    if (t == 0) {
        for (int i = 0; i < kTcStages; ++i) mbar_init(&bar_load[i], 1);
        mbar_init(&bar_mma[0], 1);
        mbar_init(&bar_mma[1], 1);
        mbar_init(&bar_a, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        abort_flag = 0;
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                     "r"((uint32_t)kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_base;

    const uint64_t step = gridDim.x;
    uint64_t tiles = 0;
    if ((uint64_t)blockIdx.x < P.items) tiles = (P.items - 1 - blockIdx.x) / step + 1;

    if (warp == 0) {
        if (lane == 0) {
            mbar_arrive_expect_tx(&bar_a, 2u * kAHalf);
            bulk_load(a_img, P.a_image, 2u * kAHalf, &bar_a);
        }
        for (int k = 0; k < kTcStages - 1; ++k)
            if ((uint64_t)k < tiles)
                issue_load(P, s, stage + (size_t)k * P.stage_elems, &bar_load[k], blockIdx.x + k * step, lane);
    }
    if (!mbar_wait_bounded(&bar_a, 0)) abort_flag = 1;

    const uint32_t a_base = smem_u32(a_img);
    const uint32_t b_base = smem_u32(b_img);
    uint64_t i = 0;
    for (; i <= tiles; ++i) {
        const int cur = (int)(i % kTcStages);
        const int bb = (int)(i & 1);
        if (i < tiles) {
            // 1. the tile has landed; 2. the MMAs that read this B buffer two tiles ago are done
            bool ok = mbar_wait_bounded(&bar_load[cur], (uint32_t)(i / kTcStages) & 1u);
            if (ok && i >= 2) ok = mbar_wait_bounded(&bar_mma[bb], (uint32_t)((i - 2) >> 1) & 1u);
            if (!ok) abort_flag = 1;
        }
        __syncthreads();
        if (abort_flag) break;
        if (i < tiles) {
            // 3. split into the MMA's B layout: (k = b, n = 2j + c) at (n%8)*16 + (n/8)*SBO + (b%4)*4 + (b/4)*LBO
            const float2* tile = stage + (size_t)cur * P.stage_elems;
            unsigned char* bhi = b_img + (size_t)bb * 2 * kBHalf;
            unsigned char* blo = bhi + kBHalf;
            const int j = (t >> 3) & 31;
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const int b = (t & 7) | (k << 3);
                const float2 x = tile[wq[b] + wl_conv];
                float2 hi, lo;
                hi.x = tf32_head(x.x);
                hi.y = tf32_head(x.y);
                lo.x = x.x - hi.x;
                lo.y = x.y - hi.y;
                const int n = 2 * j;  // real part in column n, imaginary part in column n + 1 (16 bytes on)
                const int off = (n & 7) * 16 + (n >> 3) * kBSbo + (b & 3) * 4 + (b >> 2) * kBLbo;
                *reinterpret_cast<float*>(bhi + off) = hi.x;
                *reinterpret_cast<float*>(bhi + off + 16) = hi.y;
                *reinterpret_cast<float*>(blo + off) = lo.x;
                *reinterpret_cast<float*>(blo + off + 16) = lo.y;
            }
            fence_proxy_async();
        }
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
        if (i < tiles && t == 0) {
            // 4. the tile's 24 MMAs into accumulator bb
            const uint32_t d = tmem + (uint32_t)(bb * kTcN);
            const uint32_t bhi = b_base + (uint32_t)(bb * 2 * kBHalf), blo = bhi + kBHalf;
#pragma unroll
            for (int ks = 0; ks < 8; ++ks) {
                const uint64_t ahi_d = smem_desc(a_base + ks * 256, 128, 2048);
                const uint64_t alo_d = smem_desc(a_base + kAHalf + ks * 256, 128, 2048);
                const uint64_t bhi_d = smem_desc(bhi + ks * 2 * kBLbo, kBLbo, kBSbo);
                const uint64_t blo_d = smem_desc(blo + ks * 2 * kBLbo, kBLbo, kBSbo);
                mma_tf32(d, ahi_d, bhi_d, ks > 0 ? 1u : 0u);
                mma_tf32(d, ahi_d, blo_d, 1u);
                mma_tf32(d, alo_d, bhi_d, 1u);
            }
            mma_commit(&bar_mma[bb]);
        }
        if (i >= 1) {
            // 5. epilogue of the previous tile
            const uint64_t pi = i - 1;
            const int pb = (int)(pi & 1);
            const int pst = (int)(pi % kTcStages);
            if (!mbar_wait_bounded(&bar_mma[pb], (uint32_t)(pi >> 1) & 1u)) abort_flag = 1;
            tc_fence_after();
            __syncwarp();
            float v[32];
            const uint32_t col = (uint32_t)(pb * kTcN + (warp >> 2) * 32);
            tmem_ld32(tmem + ((uint32_t)((warp & 3) * 32) << 16) + col, v);
            // row r = 2a + p; columns n = 2j + c for j in [jc, jc + 16)
            const int r = (warp & 3) * 32 + lane, a = r >> 1, p = r & 1;
            const int jc = (warp >> 2) * 16;
            float2* out = stage + (size_t)pst * P.stage_elems;
            // p = 0 finishes j = jc .. jc+7, p = 1 finishes j = jc+8 .. jc+15
            float other_re[8], other_im[8];
#pragma unroll
            for (int jj = 0; jj < 8; ++jj) {
                const float send_re = p ? v[2 * jj] : v[2 * (jj + 8)];
                const float send_im = p ? v[2 * jj + 1] : v[2 * (jj + 8) + 1];
                other_re[jj] = __shfl_xor_sync(0xffffffffu, send_re, 1);
                other_im[jj] = __shfl_xor_sync(0xffffffffu, send_im, 1);
            }
            tc_fence_before();
#pragma unroll
            for (int jj = 0; jj < 8; ++jj) {
                const int jl = p ? jj + 8 : jj;  // local column within this warp's 16
                // own row: D(2a+p, 2j), D(2a+p, 2j+1); partner row: other_*
                const float mre = p ? v[2 * (jj + 8)] : v[2 * jj];
                const float mim = p ? v[2 * (jj + 8) + 1] : v[2 * jj + 1];
                float2 o;
                if (p == 0) {  // own = Re U row: out = (mre - other_im) + i (mim + other_re)
                    o.x = mre - other_im[jj];
                    o.y = mim + other_re[jj];
                } else {       // own = Im U row, other = Re U row
                    o.x = other_re[jj] - mim;
                    o.y = other_im[jj] + mre;
                }
                const int jg = jc + jl;
                int w = 0;
                for (int k = 0; k < P.cols_bits; ++k)
                    if ((jg >> k) & 1) w += tile_weight(P, P.l_bits[k]);
                out[wq[a] + w] = o;
            }
            fence_proxy_async();
        }
        __syncthreads();
        if (warp == 0) {
            if (i >= 1) issue_store(P, s, stage + (size_t)((i - 1) % kTcStages) * P.stage_elems,
                                    blockIdx.x + (i - 1) * step, lane);
            // 6. refill: tile i + stages - 1 goes into the buffer just stored from
            const uint64_t nxt = i + kTcStages - 1;
            if (nxt < tiles) {
                bulk_wait_read();
                fence_proxy_async();
                __syncwarp();
                issue_load(P, s, stage + (size_t)(nxt % kTcStages) * P.stage_elems, &bar_load[nxt % kTcStages],
                           blockIdx.x + nxt * step, lane);
            }
        }
    }
    if (abort_flag) {
        if (t == 0) {
            atomicExch(P.status, (int32_t)QM_E_TIMEOUT);
            // MMAs and loads already issued
            for (uint64_t k = (i >= 1 ? i - 1 : 0); k < i + 1 && k < tiles; ++k)
                mbar_wait_bounded(&bar_mma[k & 1], (uint32_t)(k >> 1) & 1u);
            for (uint64_t k = i + 1; k < i + kTcStages && k < tiles; ++k)
                mbar_wait_bounded(&bar_load[k % kTcStages], (uint32_t)(k / kTcStages) & 1u);
        }
    }
    if (warp == 0) bulk_wait_all();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)kTmemCols)
                     : "memory");
}

}  // namespace

// A's image for the MMA: rows 2a + p (p = 0 real, 1 imaginary part of U(a, b)), 64 columns b, as
// TF32 head and FP32 tail, in the canonical K-major layout without swizzle (core matrices of 8
// rows x 4 columns, 16 per row group).  `ut` is the transposed unitary (row b holds U(., b)).
void dense_tc_image(const double* ut, std::vector<float>& image) {
    image.assign(2 * 128 * 64, 0.0f);
    auto head = [](float x) {
        uint32_t u;
        std::memcpy(&u, &x, 4);
        u &= 0xffffe000u;
        float h;
        std::memcpy(&h, &u, 4);
        return h;
    };
    for (int row = 0; row < 128; ++row)
        for (int b = 0; b < 64; ++b) {
            const int a = row >> 1, p = row & 1;
            const double u = ut[2 * (b * 64 + a) + p];
            const float f = (float)u;
            const float h = head(f);
            const float l = (float)(u - (double)h);
            const size_t off = (size_t)(row >> 3) * 512 + (size_t)(b >> 2) * 32 + (size_t)(row & 7) * 4 + (b & 3);
            image[off] = h;
            image[128 * 64 + off] = l;
        }
}

bool dense_tc_supported(int qubits, int precision, const DenseOp& op) {
    return precision == QM_FP32 && op.m == 6 && qubits >= kTcTileBits && dense_tc_enabled();
}

bool dense_tc_enabled() {
    static const bool on = [] {
        const char* e = std::getenv("QM_DENSE_TC");
        return e && e[0] == '1';
    }();
    return on;
}

cudaError_t launch_dense_tc(void* amps, int qubits, const DenseOp& op, const float* a_image, int32_t* status,
                            int sm_count, cudaStream_t st) {
    static std::once_flag once;
    static cudaError_t attr = cudaSuccess;
    uint32_t qmask = 0;
    for (int i = 0; i < 6; ++i) qmask |= 1u << op.q[i];
    TcLaunch P{};
    P.a_image = a_image;
    P.status = status;
    const int c = kTcTileBits - 6;
    uint32_t lmask = 0;
    int nl = 0;
    for (int b = 0; b < qubits && nl < c; ++b)
        if (!(qmask & (1u << b))) {
            lmask |= 1u << b;
            P.l_bits[nl++] = b;
        }
    int r = 0;
    bool seen_q = false;
    while (r < qubits && ((qmask | lmask) >> r & 1u)) {
        const bool is_q = (qmask >> r) & 1u;
        if (!is_q && seen_q) break;
        seen_q = seen_q || is_q;
        ++r;
    }
    for (int i = 0; i < 6; ++i) P.q_bits[i] = op.q[i];
    P.cols_bits = c;
    P.run_bits = r;
    P.copy_mask = (qmask | lmask) & ~((1u << r) - 1u);
    P.copies = 1 << (kTcTileBits - r);
    const int run_bytes = 8 << r;
    P.stride = (1 << r) + (run_bytes >= 128 ? 2 : 0);
    P.stage_elems = ((P.copies * P.stride * 8 + 127) / 128) * 16;
    P.outer_mask = ((1u << qubits) - 1u) & ~(qmask | lmask);
    P.items = uint64_t(1) << (qubits - kTcTileBits);
    const size_t smem = (size_t)kOffStage + (size_t)kTcStages * P.stage_elems * 8;
    if (smem > kTcSmemMax) return cudaErrorInvalidValue;
    std::call_once(once, [] {
        attr = cudaFuncSetAttribute(k_dense_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTcSmemMax);
    });
    if (attr != cudaSuccess) return attr;
    const int grid = (int)std::min<uint64_t>(P.items, (uint64_t)std::max(1, sm_count));
    k_dense_tc<<<grid, kTcThreads, smem, st>>>(reinterpret_cast<float2*>(amps), P);
    return cudaGetLastError();
}

}  // namespace qm
