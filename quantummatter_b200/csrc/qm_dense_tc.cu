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
//   - one tensor-map box (cp.async.bulk.tensor, natural index order) or bulk copies of runs
//     (cp.async.bulk) stage each tile into one of four buffers, three tiles ahead of the one being
//     converted, with mbarrier completion;
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

constexpr int kTcConsumers = 512;                 // 16 warps: conversion and epilogue
constexpr int kTcProducerWarp = kTcConsumers / 32;  // tile loads and stores
constexpr int kTcMmaWarp = kTcProducerWarp + 1;     // TMEM allocation, A into TMEM order, MMAs
constexpr int kTcThreads = kTcConsumers + 64;
constexpr int kTcTileBits = 11;      // 64 rows x 32 columns
constexpr int kTcCols = 32;          // complex columns per tile
constexpr int kTcN = 2 * kTcCols;    // real columns of B and D
constexpr int kTcMaxStages = 5;      // staging buffers (4 where five do not fit)
constexpr int kTmemCols = 4 * kTcN;  // two accumulators, then A_hi and A_lo (64 columns each)
constexpr int kTmemA = 2 * kTcN;     // first column of A_hi
constexpr long long kTcWaitCycles = 2000000000ll;
constexpr size_t kTcSmemMax = 226 * 1024;

// shared-memory layout (bytes)
constexpr int kAHalf = 128 * 64 * 4;           // one 128 x 64 TF32 operand image: 32 KiB
// B, K-major without swizzle: core matrices of 8 real columns (n) x 4 rows (k, 16 bytes); the 16
// k-groups of a column group 144 bytes apart (16 more than dense, so the conversion's stores of
// k and k + 4 land in different banks), column groups 2320 bytes apart
constexpr int kBLbo = 144;
constexpr int kBSbo = 16 * kBLbo + 16;         // 2320: column groups skewed by 16 bytes as well
constexpr int kBHalf = (kTcN / 8) * kBSbo;     // one 64 x 64 B image: 18560 B
constexpr int kOffA = 0;                       // A_hi, A_lo
constexpr int kOffB = 2 * kAHalf;              // [2 buffers][hi, lo]
constexpr int kOffStage = kOffB + 4 * kBHalf;  // staging ring, stage_bytes each

struct TcLaunch {
    CUtensorMap tmap;        // the tile as one box (tma_rank > 0), else bulk copies of runs
    int32_t tma_rank, tma_lo[5], tma_len[5], tma_tile[5];
    const float* a_image;    // A_hi then A_lo, already in the MMA's K-major layout (64 KiB)
    int32_t* status;
    uint64_t items;
    uint32_t outer_mask, copy_mask;
    int32_t q_bits[6];
    int32_t l_bits[kTcTileBits];
    int32_t cols_bits, run_bits, copies, stride, stage_elems, stages;
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
// all bulk groups but the newest have finished reading their shared-memory sources
__device__ __forceinline__ void bulk_wait_read_older() { asm volatile("cp.async.bulk.wait_group.read 1;" ::: "memory"); }
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

// D (TMEM) += A (TMEM: row m in lane m, K along columns) * B (shared memory descriptor)
__device__ __forceinline__ void mma_tf32_ts(uint32_t d_tmem, uint32_t a_tmem, uint64_t b, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.u32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, p;\n\t}" ::"r"(d_tmem),
        "r"(a_tmem), "l"(b), "r"(kIdesc), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void tmem_st32(uint32_t taddr, const float (&v)[32]) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31, %32};" ::"r"(taddr),
        "f"(v[0]), "f"(v[1]), "f"(v[2]), "f"(v[3]), "f"(v[4]), "f"(v[5]), "f"(v[6]), "f"(v[7]), "f"(v[8]), "f"(v[9]),
        "f"(v[10]), "f"(v[11]), "f"(v[12]), "f"(v[13]), "f"(v[14]), "f"(v[15]), "f"(v[16]), "f"(v[17]), "f"(v[18]),
        "f"(v[19]), "f"(v[20]), "f"(v[21]), "f"(v[22]), "f"(v[23]), "f"(v[24]), "f"(v[25]), "f"(v[26]), "f"(v[27]),
        "f"(v[28]), "f"(v[29]), "f"(v[30]), "f"(v[31])
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ int tile_weight(const TcLaunch& P, int g) {
    if (g < P.run_bits) return 1 << g;
    return P.stride << __popc(P.copy_mask & ((1u << g) - 1u));
}
// staged-tile offsets (amplitudes) of row b (fused-qubit index) and column j
__device__ __forceinline__ int row_offset(const TcLaunch& P, int b) {
    int w = 0;
    for (int i = 0; i < 6; ++i)
        if ((b >> i) & 1) w += tile_weight(P, P.q_bits[i]);
    return w;
}
__device__ __forceinline__ int col_offset(const TcLaunch& P, int j) {
    int w = 0;
    for (int k = 0; k < P.cols_bits; ++k)
        if ((j >> k) & 1) w += tile_weight(P, P.l_bits[k]);
    return w;
}
// byte offset of (row b, complex column j) in a B image: real part in column n = 2j, imaginary
// part 16 bytes on (column n + 1 of the same core matrix)
__device__ __forceinline__ int b_image_offset(int b, int j) {
    const int n = 2 * j;
    return (n & 7) * 16 + (n >> 3) * kBSbo + (b & 3) * 4 + (b >> 2) * kBLbo;
}

__device__ __forceinline__ void issue_load(const TcLaunch& P, const float2* s, float2* buf, uint64_t* bar,
                                           uint64_t item, int lane) {
    if (P.tma_rank) {
        if (lane == 0) {
            int32_t c[5];
            tma_item_coords(P.tma_rank, P.tma_len, P.tma_tile, (uint32_t)item, c);
            mbar_arrive_expect_tx(bar, 8u << kTcTileBits);
            tma_box_load(&P.tmap, P.tma_rank, smem_u32(buf), smem_u32(bar), c);
        }
        return;
    }
    const uint32_t base = deposit((uint32_t)item, P.outer_mask);
    const uint32_t run_bytes = 8u << P.run_bits;
    if (lane == 0) mbar_arrive_expect_tx(bar, run_bytes * (uint32_t)P.copies);
    __syncwarp();
    for (int x = lane; x < P.copies; x += 32)
        bulk_load(buf + (size_t)x * P.stride, s + (base | deposit((uint32_t)x, P.copy_mask)), run_bytes, bar);
}

__device__ __forceinline__ void issue_store(const TcLaunch& P, float2* s, const float2* buf, uint64_t item, int lane) {
    if (P.tma_rank) {
        if (lane == 0) {
            int32_t c[5];
            tma_item_coords(P.tma_rank, P.tma_len, P.tma_tile, (uint32_t)item, c);
            tma_box_store(&P.tmap, P.tma_rank, smem_u32(buf), c);
            bulk_commit();
        }
        return;
    }
    const uint32_t base = deposit((uint32_t)item, P.outer_mask);
    const uint32_t run_bytes = 8u << P.run_bits;
    for (int x = lane; x < P.copies; x += 32)
        bulk_store(s + (base | deposit((uint32_t)x, P.copy_mask)), buf + (size_t)x * P.stride, run_bytes);
    bulk_commit();
}

__device__ __forceinline__ float tf32_head(float x) { return __uint_as_float(__float_as_uint(x) & 0xffffe000u); }

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// kConvJ: column bit 0 is index bit 0 (the staged tile is contiguous along columns), which picks
// the conversion's lane mapping and rotates the epilogue's stores (see below).
//
// Roles, synchronised by mbarriers only (no block-wide barrier inside the tile loop):
//   producer warp: tile i into buffer i % S (full[b]), S - 1 tiles ahead; stores tile i once its
//     epilogue is written (done[b]) and reloads the buffer stored before it;
//   MMA warp: after conv[bb] (tile i in B buffer bb) and accf[bb] (the epilogue of tile i - 2 has
//     read accumulator bb), the tile's 24 MMAs, committed to mma[bb];
//   16 consumer warps: convert tile i into B buffer i % 2 once mma[bb] shows tile i - 2's MMAs
//     done, then the epilogue of tile i - 1 over its own staging buffer.
template <bool kConvJ>
__global__ void __launch_bounds__(kTcThreads, 1) k_dense_tc(float2* __restrict__ s, const __grid_constant__ TcLaunch P) {
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ uint64_t full[kTcMaxStages], done[kTcMaxStages];
    __shared__ uint64_t conv[2], accf[2], mma[2];
    __shared__ uint64_t bar_a;
    __shared__ uint32_t tmem_base;
    __shared__ volatile int abort_flag;

    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const uint32_t S = (uint32_t)P.stages;
    float* a_img = reinterpret_cast<float*>(smem + kOffA);
    unsigned char* b_img = smem + kOffB;
    float2* stage = reinterpret_cast<float2*>(smem + kOffStage);

    if (t == 0) {
        if (P.tma_rank) tma_prefetch(&P.tmap);
        for (uint32_t k = 0; k < S; ++k) {
            mbar_init(&full[k], 1);
            mbar_init(&done[k], kTcConsumers);
        }
        for (int k = 0; k < 2; ++k) {
            mbar_init(&conv[k], kTcConsumers);
            mbar_init(&accf[k], kTcConsumers);
            mbar_init(&mma[k], 1);
        }
        mbar_init(&bar_a, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        abort_flag = 0;
    }
    if (warp == kTcMmaWarp) {
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
    uint32_t tiles = 0;
    if ((uint64_t)blockIdx.x < P.items) tiles = (uint32_t)((P.items - 1 - blockIdx.x) / step + 1);

    if (warp == kTcProducerWarp) {
        if (lane == 0) {
            mbar_arrive_expect_tx(&bar_a, 2u * kAHalf);
            bulk_load(a_img, P.a_image, 2u * kAHalf, &bar_a);
        }
        uint32_t issued = 0;
        for (; issued + 1 < S && issued < tiles; ++issued)
            issue_load(P, s, stage + (size_t)issued * P.stage_elems, &full[issued], blockIdx.x + issued * step, lane);
        uint32_t b = 0, lap = 0;
        for (uint32_t j = 0; j < tiles; ++j) {
            // lane 0 waits and decides for the warp: 0 go on, 1 another role stopped, 2 timed out
            int st = 0;
            if (lane == 0) st = abort_flag ? 1 : (mbar_wait_bounded(&done[b], lap & 1u) ? 0 : 2);
            st = __shfl_sync(0xffffffffu, st, 0);
            if (st) {
                if (st == 2 && lane == 0) abort_flag = 1;
                break;
            }
            issue_store(P, s, stage + (size_t)b * P.stage_elems, blockIdx.x + (uint64_t)j * step, lane);
            const uint32_t n = j + S - 1;
            if (n < tiles) {
                // the buffer of tile j - 1: all stores but the newest have read their buffers
                const uint32_t nb = b == 0 ? S - 1 : b - 1;
                bulk_wait_read_older();
                fence_proxy_async();
                __syncwarp();
                issue_load(P, s, stage + (size_t)nb * P.stage_elems, &full[nb], blockIdx.x + (uint64_t)n * step, lane);
                ++issued;
            }
            if (++b == S) {
                b = 0;
                ++lap;
            }
        }
        // no load may still be writing shared memory when the block exits
        for (uint32_t k = issued > S ? issued - S : 0; k < issued; ++k)
            mbar_wait_bounded(&full[k % S], (k / S) & 1u);
        bulk_wait_all();
    } else if (warp == kTcMmaWarp) {
        if (lane == 0) {
            uint32_t issued = 0;
            for (uint32_t i = 0; i < tiles; ++i) {
                const int bb = (int)(i & 1);
                bool ok = !abort_flag && mbar_wait_bounded(&conv[bb], (i >> 1) & 1u);
                if (ok && i >= 2) ok = mbar_wait_bounded(&accf[bb], ((i - 2) >> 1) & 1u);
                if (!ok) {
                    abort_flag = 1;
                    break;
                }
                tc_fence_after();
                const uint32_t d = tmem + (uint32_t)(bb * kTcN);
                const uint32_t bhi = smem_u32(b_img) + (uint32_t)(bb * 2 * kBHalf), blo = bhi + kBHalf;
#pragma unroll
                for (int ks = 0; ks < 8; ++ks) {
                    const uint32_t ahi = tmem + (uint32_t)(kTmemA + 8 * ks), alo = ahi + 64u;
                    const uint64_t bhi_d = smem_desc(bhi + ks * 2 * kBLbo, kBLbo, kBSbo);
                    const uint64_t blo_d = smem_desc(blo + ks * 2 * kBLbo, kBLbo, kBSbo);
                    mma_tf32_ts(d, ahi, bhi_d, ks > 0 ? 1u : 0u);
                    mma_tf32_ts(d, ahi, blo_d, 1u);
                    mma_tf32_ts(d, alo, bhi_d, 1u);
                }
                mma_commit(&mma[bb]);
                ++issued;
            }
            // the MMAs still running when the loop ended early
            for (uint32_t k = issued > 2 ? issued - 2 : 0; k < issued; ++k)
                mbar_wait_bounded(&mma[k & 1], (k >> 1) & 1u);
        }
        __syncwarp();
    } else {
        // Conversion: 4 elements per thread, element k at row b, column j_k = j_0 + 8k.  kConvJ: a
        // warp takes 8 consecutive columns of 4 consecutive rows (j_0 = lane % 8, b = lane / 8 +
        // 4 warp), so that its B-image stores of one core-matrix row fill all 32 banks; otherwise
        // 32 consecutive rows of one column (b = lane + 32 (warp % 2), j_0 = warp / 2).  In both
        // the B-image offset of element k is that of element 0 plus k * 2 SBO.
        const int cb = kConvJ ? (lane >> 3) + 4 * warp : lane + 32 * (warp & 1);
        const int cj = kConvJ ? (lane & 7) : (warp >> 1);
        int conv_src[4];
        {
            const int rb = row_offset(P, cb);
#pragma unroll
            for (int k = 0; k < 4; ++k) conv_src[k] = rb + col_offset(P, cj + 8 * k);
        }
        const int conv_dst = b_image_offset(cb, cj);

        // Epilogue: warp w reads TMEM lanes 32 (w % 4) .. + 31 (rows r = 2a + p) and real columns
        // 16 (w / 4) .. + 15, i.e. complex columns j = 8 (w / 4) + jj, jj < 8; the row pair
        // (2a, 2a + 1) sits in adjacent lanes, p = 0 finishes jj = 0..3 and p = 1 jj = 4..7.  Where
        // rows are multiples of 32 amplitudes apart (kConvJ layouts), every row of a warp would
        // store the same column at once, all in one bank: step s stores column (s + a) % 4 instead.
        const int er = (warp & 3) * 32 + lane, ea = er >> 1, ep = er & 1;
        int out_off[4];
        {
            const int base = row_offset(P, ea) + col_offset(P, 8 * (warp >> 2) + 4 * ep);
#pragma unroll
            for (int q = 0; q < 4; ++q) out_off[q] = base + col_offset(P, kConvJ ? ((q + ea) & 3) : q);
        }
        const uint32_t lane_base = (uint32_t)((warp & 3) * 32) << 16;

        // A (the unitary's TF32 head and tail) into TMEM order: warps 0..7, row m = 32 (w % 4) +
        // lane, head (w < 4) or tail, 64 K columns from the K-major shared-memory image
        if (warp < 8) {
            if (!__all_sync(0xffffffffu, mbar_wait_bounded(&bar_a, 0))) abort_flag = 1;
            const float* img = a_img + (warp >> 2) * (kAHalf / 4);
            const int m = er;
#pragma unroll
            for (int c = 0; c < 2; ++c) {
                float v[32];
#pragma unroll
                for (int kk = 0; kk < 32; ++kk) {
                    const int k = 32 * c + kk;
                    v[kk] = img[(m >> 3) * 512 + (k >> 2) * 32 + (m & 7) * 4 + (k & 3)];
                }
                tmem_st32(tmem + lane_base + (uint32_t)(kTmemA + 64 * (warp >> 2) + 32 * c), v);
            }
            asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
        }

        uint32_t cur = 0, prev = S - 1, lap = 0;  // cur = i % S, prev = (i - 1) % S, lap = i / S
        // every stop below is decided for the whole warp (the TMEM loads and shuffles need all lanes)
        for (uint32_t i = 0; i <= tiles; ++i) {
            if (__any_sync(0xffffffffu, abort_flag != 0)) break;
            if (i < tiles) {
                const int bb = (int)(i & 1);
                // the tile has landed, and the MMAs that read B buffer bb (tile i - 2) are done
                bool ok = mbar_wait_bounded(&full[cur], lap & 1u);
                if (ok && i >= 2) ok = mbar_wait_bounded(&mma[bb], ((i - 2) >> 1) & 1u);
                if (!__all_sync(0xffffffffu, ok)) {
                    abort_flag = 1;
                    break;
                }
                const float2* tile = stage + (size_t)cur * P.stage_elems;
                unsigned char* bhi = b_img + (size_t)bb * 2 * kBHalf + conv_dst;
                unsigned char* blo = bhi + kBHalf;
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const float2 x = tile[conv_src[k]];
                    float2 hi, lo;
                    hi.x = tf32_head(x.x);
                    hi.y = tf32_head(x.y);
                    lo.x = x.x - hi.x;
                    lo.y = x.y - hi.y;
                    *reinterpret_cast<float*>(bhi + k * 2 * kBSbo) = hi.x;
                    *reinterpret_cast<float*>(bhi + k * 2 * kBSbo + 16) = hi.y;
                    *reinterpret_cast<float*>(blo + k * 2 * kBSbo) = lo.x;
                    *reinterpret_cast<float*>(blo + k * 2 * kBSbo + 16) = lo.y;
                }
                fence_proxy_async();
                tc_fence_before();
                mbar_arrive(&conv[bb]);
            }
            if (i >= 1) {
                const uint32_t pi = i - 1;
                const int pb = (int)(pi & 1);
                if (!__all_sync(0xffffffffu, mbar_wait_bounded(&mma[pb], (pi >> 1) & 1u))) {
                    abort_flag = 1;
                    break;
                }
                tc_fence_after();
                __syncwarp();
                float v[16];
                tmem_ld16(tmem + lane_base + (uint32_t)(pb * kTcN + (warp >> 2) * 16), v);
                tc_fence_before();
                mbar_arrive(&accf[pb]);
                // v[2 jj], v[2 jj + 1] = D(r, 2 j), D(r, 2 j + 1); the partner row's values for
                // the columns this lane finishes come over a shuffle
                float other_re[4], other_im[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const float send_re = ep ? v[2 * q] : v[2 * (q + 4)];
                    const float send_im = ep ? v[2 * q + 1] : v[2 * (q + 4) + 1];
                    other_re[q] = __shfl_xor_sync(0xffffffffu, send_re, 1);
                    other_im[q] = __shfl_xor_sync(0xffffffffu, send_im, 1);
                }
                float2 o[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const float mre = ep ? v[2 * (q + 4)] : v[2 * q];
                    const float mim = ep ? v[2 * (q + 4) + 1] : v[2 * q + 1];
                    if (ep == 0) {  // own = Re U row: out = (mre - other_im) + i (mim + other_re)
                        o[q].x = mre - other_im[q];
                        o[q].y = mim + other_re[q];
                    } else {        // own = Im U row, other = Re U row
                        o[q].x = other_re[q] - mim;
                        o[q].y = other_im[q] + mre;
                    }
                }
                if (kConvJ) {  // o[s] <- o[(s + a) % 4]
                    if (ea & 1) {
                        const float2 x0 = o[0];
                        o[0] = o[1];
                        o[1] = o[2];
                        o[2] = o[3];
                        o[3] = x0;
                    }
                    if (ea & 2) {
                        const float2 x0 = o[0], x1 = o[1];
                        o[0] = o[2];
                        o[1] = o[3];
                        o[2] = x0;
                        o[3] = x1;
                    }
                }
                float2* out = stage + (size_t)prev * P.stage_elems;
#pragma unroll
                for (int q = 0; q < 4; ++q) out[out_off[q]] = o[q];
                fence_proxy_async();
                mbar_arrive(&done[prev]);
            }
            prev = cur;
            if (++cur == S) {
                cur = 0;
                ++lap;
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (abort_flag && t == 0) atomicExch(P.status, (int32_t)QM_E_TIMEOUT);
    if (warp == kTcMmaWarp)
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

// On unless QM_DENSE_TC=0; read at every plan, so a process can plan with and without the tensor
// cores.  Measured on the 30-qubit brick (complex64): dense fused gates of <= 5 qubits 1237 against
// 1693 ms per step, of <= 6 qubits 1760 against 2601 ms, with the largest amplitude error against
// complex128 1.4e-8 against 3e-10 (3xTF32 keeps about 21 significant bits per product).
bool dense_tc_enabled() {
    const char* e = std::getenv("QM_DENSE_TC");
    return !(e && e[0] == '0');
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
    // one tensor-map box per tile where the tile's bit runs fit five dimensions: the staged tile
    // is then in natural index order (unpadded), and so are its runs for bulk copies without an
    // encoder; otherwise padded runs in which every column bit lies below every fused bit
    int32_t rank = 0;
    const bool natural = dense_tma_enabled() && (qmask | lmask) & 1u &&
                         tile_map_dims(qmask | lmask, qubits, P.tma_lo, P.tma_len, P.tma_tile, &rank);
    if (natural) {
        r = 0;
        while (r < qubits && ((qmask | lmask) >> r & 1u)) ++r;
        if (encode_tile_map(&P.tmap, amps, QM_FP32, rank, P.tma_lo, P.tma_len, P.tma_tile)) P.tma_rank = rank;
    }
    P.run_bits = r;
    P.copy_mask = (qmask | lmask) & ~((1u << r) - 1u);
    P.copies = 1 << (kTcTileBits - r);
    const int run_bytes = 8 << r;
    P.stride = (1 << r) + (run_bytes >= 128 && !natural ? 2 : 0);
    P.stage_elems = ((P.copies * P.stride * 8 + 127) / 128) * 16;
    P.outer_mask = ((1u << qubits) - 1u) & ~(qmask | lmask);
    P.items = uint64_t(1) << (qubits - kTcTileBits);
    const size_t stage_bytes = (size_t)P.stage_elems * 8;
    P.stages = kOffStage + kTcMaxStages * stage_bytes <= kTcSmemMax ? kTcMaxStages : kTcMaxStages - 1;
    const size_t smem = (size_t)kOffStage + (size_t)P.stages * stage_bytes;
    if (smem > kTcSmemMax) return cudaErrorInvalidValue;
    std::call_once(once, [] {
        attr = cudaFuncSetAttribute(k_dense_tc<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTcSmemMax);
        if (attr == cudaSuccess)
            attr = cudaFuncSetAttribute(k_dense_tc<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTcSmemMax);
    });
    if (attr != cudaSuccess) return attr;
    const int grid = (int)std::min<uint64_t>(P.items, (uint64_t)std::max(1, sm_count));
    g_dense_tc_launches.fetch_add(1, std::memory_order_relaxed);
    if (lmask & 1u)
        k_dense_tc<true><<<grid, kTcThreads, smem, st>>>(reinterpret_cast<float2*>(amps), P);
    else
        k_dense_tc<false><<<grid, kTcThreads, smem, st>>>(reinterpret_cast<float2*>(amps), P);
    return cudaGetLastError();
}

}  // namespace qm
