// qm_expect.cu -- tiled Pauli-sum expectation for batches of states (sm_100a).
//
// StateVector.ExpectationValue (StateVector.Observations.cs:107-141) evaluates one term per
// pass over the state.  Here a CTA stages a block of 2^K amplitudes in shared memory (the
// block's qubits are a "tile": the lowest qubits plus a window chosen so that the flip masks
// of the assigned terms lie inside it) and evaluates every assigned term against it:
// conj(psi[j ^ F]) psi[j] with the Y phase and the Z-sign parity of the global index, in
// FP64.  A Hamiltonian whose flip masks fit in a few windows costs a few reads of the state
// instead of one per term.  Sums are deterministic: thread, warp tree, fixed warp order, and
// a fixed-order column sum over CTAs.
#include <cuda_runtime.h>

#include <algorithm>

#include "qm_device.cuh"
#include "qm_internal.h"

namespace qm {

namespace {

constexpr int R = kRegBits;
constexpr int NR = 1 << R;

template <int MAXT>
struct TileLaunch {
    uint32_t outer_mask;      // qubits outside the tile
    uint32_t thread_mask;     // global bits carried by the thread index (local bits 0..K-R-1)
    uint32_t reg_g[R];        // global bits of the register index (local bits K-R..K-1)
    int32_t terms;
    int32_t with_mass;
    int32_t columns;          // row width of the partial table
    int32_t mass_column;
    int32_t row_offset;       // first partial row of this tile pass
    int32_t rows_per_state;
    uint64_t state_stride;
    double* partials;         // [states][rows_per_state][columns]
    TileTerm t[MAXT];
};

__device__ __forceinline__ double warp_sum(double v) {
    for (int d = 16; d > 0; d >>= 1) v += __shfl_down_sync(0xffffffffu, v, d);
    return v;
}

template <typename T, int K, int MAXT>
__global__ void __launch_bounds__(1 << (K - R), 512 / (1 << (K - R)))
    k_expect_tile(const typename Vec2<T>::type* __restrict__ s, const __grid_constant__ TileLaunch<MAXT> P) {
    using V = typename Vec2<T>::type;
    constexpr int NT = 1 << (K - R);
    constexpr int WARPS = NT / 32;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V* tile = reinterpret_cast<V*>(smem_raw);
    double* red = reinterpret_cast<double*>(smem_raw + (sizeof(V) << K));  // [WARPS][terms + 1]
    const uint32_t t = threadIdx.x;
    const int warp = t >> 5, lane = t & 31;
    s += (size_t)blockIdx.y * P.state_stride;
    const uint32_t outer = deposit(blockIdx.x, P.outer_mask);
    const uint32_t g0 = outer | deposit(t, P.thread_mask);

    // stage the block; each thread later re-reads its own amplitudes from shared memory
    // (keeping them in registers would cap occupancy at one CTA per SM)
    uint32_t g[NR];
#pragma unroll
    for (int i = 0; i < NR; ++i) {
        uint32_t gi = g0;
#pragma unroll
        for (int m = 0; m < R; ++m)
            if ((i >> m) & 1) gi |= P.reg_g[m];
        g[i] = gi;
        tile[t | ((uint32_t)i << (K - R))] = s[gi];
    }
    __syncthreads();

    // Terms arrive sorted by flip mask, the diagonal ones (flip 0) first.  Three or more
    // diagonal terms are evaluated together through a Walsh-Hadamard transform of the tile's
    // Born probabilities (below); the rest in groups of up to kGroup consecutive terms with the
    // same mask, which share one partner load and one overlap per amplitude.
    int ndiag = 0;
    while (ndiag < P.terms && P.t[ndiag].flip_local == 0) ++ndiag;
    const bool wht = ndiag >= 3;
    constexpr int kGroup = 4;
    for (int k = wht ? ndiag : 0; k < P.terms;) {
        const uint32_t flip = P.t[k].flip_local;
        int cnt = 1;
        while (cnt < kGroup && k + cnt < P.terms && P.t[k + cnt].flip_local == flip) ++cnt;
        uint32_t sign[kGroup];
        int phase[kGroup];
#pragma unroll
        for (int u = 0; u < kGroup; ++u) {
            sign[u] = u < cnt ? P.t[k + u].sign : 0u;
            phase[u] = u < cnt ? P.t[k + u].phase : 0;
        }
        // A Hermitian term (phase parity = parity of its Y count, as Pauli strings have) takes the
        // same real part from index j and its partner j ^ F, so only the indices whose highest
        // flip bit is 0 are summed, and doubled.  Each term's Z signs come from its sign mask over
        // the tile's local bits plus one parity of the bits outside the tile; its phase is two
        // flags.  Products and sums are FP64 for both precisions (exact products of complex64).
        uint32_t sgl[kGroup], sbase[kGroup];
        bool use_im[kGroup];
        bool paired = flip != 0;
#pragma unroll
        for (int u = 0; u < kGroup; ++u) {
            sgl[u] = 0u;
            sbase[u] = 0u;
            use_im[u] = false;
            if (u < cnt) {
                const uint32_t sg = P.t[k + u].sign;
                uint32_t loc = 0, tm = P.thread_mask;
                for (int b = 0; tm; ++b) {
                    const uint32_t lowb = tm & (0u - tm);
                    if (sg & lowb) loc |= 1u << b;
                    tm ^= lowb;
                }
#pragma unroll
                for (int m = 0; m < R; ++m)
                    if (sg & P.reg_g[m]) loc |= 1u << (K - R + m);
                const int ph = P.t[k + u].phase;
                sgl[u] = loc;
                use_im[u] = (ph & 1) != 0;
                sbase[u] = ((ph == 1 || ph == 2) ? 1u : 0u) ^ ((uint32_t)__popc(sg & outer) & 1u);
                if (((__popc(flip & loc) ^ ph) & 1) != 0) paired = false;
            }
        }
        if (paired) {
            const uint32_t pivot = 1u << (31 - __clz(flip));
            const uint32_t below = pivot - 1u;
            double hacc[kGroup] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
            for (int r = 0; r < NR / 2; ++r) {
                const uint32_t h = t + (uint32_t)NT * r;
                const uint32_t j = (h & below) | ((h & ~below) << 1);
                const V a = tile[j], b = tile[j ^ flip];
                const double ar = a.x, ai = a.y, br = b.x, bi = b.y;
                const double ore = br * ar + bi * ai, oim = br * ai - bi * ar;
#pragma unroll
                for (int u = 0; u < kGroup; ++u) {
                    if (u >= cnt) break;
                    const double c = use_im[u] ? oim : ore;
                    hacc[u] += ((__popc(j & sgl[u]) ^ sbase[u]) & 1u) ? -c : c;
                }
            }
#pragma unroll
            for (int u = 0; u < kGroup; ++u) {
                if (u >= cnt) break;
                const double v = warp_sum(2.0 * hacc[u]);
                if (lane == 0) red[warp * (P.terms + 1) + k + u] = v;
            }
            k += cnt;
            continue;
        }
        double acc[kGroup] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
        for (int i = 0; i < NR; ++i) {
            const V own = tile[t | ((uint32_t)i << (K - R))];
            const double ar = own.x, ai = own.y;
            double ore, oim;
            if (flip == 0) {
                ore = ar * ar + ai * ai;
                oim = 0.0;
            } else {
                const V b = tile[(t | ((uint32_t)i << (K - R))) ^ flip];
                const double br = b.x, bi = b.y;
                ore = br * ar + bi * ai;
                oim = br * ai - bi * ar;
            }
#pragma unroll
            for (int u = 0; u < kGroup; ++u) {
                if (u >= cnt) break;
                double c;
                switch (phase[u]) {
                case 0: c = ore; break;
                case 1: c = -oim; break;
                case 2: c = -ore; break;
                default: c = oim; break;
                }
                acc[u] += (__popc(g[i] & sign[u]) & 1) ? -c : c;
            }
        }
#pragma unroll
        for (int u = 0; u < kGroup; ++u) {
            if (u >= cnt) break;
            const double v = warp_sum(acc[u]);
            if (lane == 0) red[warp * (P.terms + 1) + k + u] = v;
        }
        k += cnt;
    }
    if (P.with_mass) {
        double acc = 0.0;
#pragma unroll
        for (int i = 0; i < NR; ++i) {
            const V own = tile[t | ((uint32_t)i << (K - R))];
            acc += (double)own.x * own.x + (double)own.y * own.y;
        }
        acc = warp_sum(acc);
        if (lane == 0) red[warp * (P.terms + 1) + P.terms] = acc;
    }
    // Walsh-Hadamard transform over the tile's local bits: W[S] = sum_j |psi_j|^2 (-1)^popc(j & S),
    // so a diagonal term with local sign mask S is W[S] times the sign of its bits outside the
    // tile.  Register bits in registers, lane bits through shuffles, warp bits through shared
    // memory (the tile, no longer needed), all in a fixed order.
    double* wbuf = reinterpret_cast<double*>(smem_raw);
    if (wht) {
        double w[NR];
#pragma unroll
        for (int i = 0; i < NR; ++i) {
            const V a = tile[t | ((uint32_t)i << (K - R))];
            w[i] = (double)a.x * a.x + (double)a.y * a.y;
        }
#pragma unroll
        for (int m = 0; m < R; ++m)
#pragma unroll
            for (int i = 0; i < NR; ++i)
                if (!((i >> m) & 1)) {
                    const double x = w[i], y = w[i | (1 << m)];
                    w[i] = x + y;
                    w[i | (1 << m)] = x - y;
                }
#pragma unroll
        for (int m = 0; m < 5; ++m)
#pragma unroll
            for (int i = 0; i < NR; ++i) {
                const double y = __shfl_xor_sync(0xffffffffu, w[i], 1 << m);
                w[i] = ((lane >> m) & 1) ? y - w[i] : w[i] + y;
            }
        __syncthreads();  // every read of the tile is done
#pragma unroll
        for (int i = 0; i < NR; ++i) wbuf[t | ((uint32_t)i << (K - R))] = w[i];
#pragma unroll
        for (int m = 5; m < K - R; ++m) {
            __syncthreads();
#pragma unroll
            for (int i = 0; i < NR; ++i) {
                const uint32_t j = t | ((uint32_t)i << (K - R));
                const double x = wbuf[j], y = wbuf[j ^ (1u << m)];
                w[i] = ((j >> m) & 1u) ? y - x : x + y;
            }
            __syncthreads();
#pragma unroll
            for (int i = 0; i < NR; ++i) wbuf[t | ((uint32_t)i << (K - R))] = w[i];
        }
    }
    __syncthreads();
    const size_t row = (size_t)blockIdx.y * P.rows_per_state + P.row_offset + blockIdx.x;
    for (int k = t; k < P.terms + (P.with_mass ? 1 : 0); k += NT) {
        double sum = 0.0;
        if (wht && k < ndiag) {
            const uint32_t sg = P.t[k].sign;
            uint32_t loc = 0, tm = P.thread_mask;
            for (int b = 0; tm; ++b) {
                const uint32_t low = tm & (0u - tm);
                if (sg & low) loc |= 1u << b;
                tm ^= low;
            }
#pragma unroll
            for (int m = 0; m < R; ++m)
                if (sg & P.reg_g[m]) loc |= 1u << (K - R + m);
            sum = wbuf[loc];
            if (__popc(sg & outer) & 1) sum = -sum;
            P.partials[row * P.columns + P.t[k].column] = sum;
            continue;
        }
        for (int w = 0; w < WARPS; ++w) sum += red[w * (P.terms + 1) + k];
        const int col = k < P.terms ? P.t[k].column : P.mass_column;
        P.partials[row * P.columns + col] = sum;
    }
}

template <typename T, int K, int MAXT>
cudaError_t launch_tile_k(const void* amps, int qubits, const TilePass& tp, const TileTerm* terms, int states,
                          uint64_t state_stride, double* partials, int columns, int rows_per_state, int mass_column,
                          cudaStream_t st) {
    using V = typename Vec2<T>::type;
    TileLaunch<MAXT> L;
    const uint32_t all = (1u << qubits) - 1u;
    L.outer_mask = all & ~tp.block_mask;
    L.thread_mask = 0;
    for (int b = 0; b < K - R; ++b) L.thread_mask |= 1u << tp.q[b];
    for (int m = 0; m < R; ++m) L.reg_g[m] = 1u << tp.q[K - R + m];
    L.terms = tp.term_count;
    L.with_mass = tp.with_mass;
    L.columns = columns;
    L.mass_column = mass_column;
    L.row_offset = tp.row_offset;
    L.rows_per_state = rows_per_state;
    L.state_stride = state_stride;
    L.partials = partials;
    for (int i = 0; i < tp.term_count; ++i) L.t[i] = terms[tp.term_begin + i];
    const size_t smem = (sizeof(V) << K) + sizeof(double) * (size_t)((1 << (K - R)) / 32) * (tp.term_count + 1);
    static const cudaError_t configured =  // once per process, thread-safe
        cudaFuncSetAttribute(k_expect_tile<T, K, MAXT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)((sizeof(V) << K) + sizeof(double) * ((1 << (K - R)) / 32) * (MAXT + 1)));
    if (configured != cudaSuccess) return configured;
    dim3 grid(1u << (qubits - K), (unsigned)states);
    k_expect_tile<T, K, MAXT><<<grid, 1 << (K - R), smem, st>>>(reinterpret_cast<const V*>(amps), L);
    return cudaGetLastError();
}

template <typename T, int K>
cudaError_t launch_tile_sized(const void* amps, int qubits, const TilePass& tp, const TileTerm* terms, int states,
                              uint64_t stride, double* partials, int columns, int rows, int mass_column,
                              cudaStream_t st) {
    if (tp.term_count <= 32)
        return launch_tile_k<T, K, 32>(amps, qubits, tp, terms, states, stride, partials, columns, rows, mass_column, st);
    return launch_tile_k<T, K, kTileMaxTerms>(amps, qubits, tp, terms, states, stride, partials, columns, rows,
                                              mass_column, st);
}

// Column sums per state of a [states][rows][columns] table: one warp per (state, column).
__global__ void k_finish_batched(const double* __restrict__ partials, int rows, int columns, double* out) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= columns) return;
    const size_t base = (size_t)blockIdx.y * rows * columns;
    KSum acc{0, 0};
    for (int r = lane; r < rows; r += 32) acc.add(partials[base + (size_t)r * columns + warp]);
    for (int d = 16; d > 0; d >>= 1) acc.merge(shfl_down_ksum(acc, d));
    if (lane == 0) out[(size_t)blockIdx.y * columns + warp] = acc.value();
}

template <typename T>
__global__ void k_reset_batched(typename Vec2<T>::type* s, uint64_t per_state, uint64_t total) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (; i < total; i += stride) {
        typename Vec2<T>::type v;
        v.x = (i % per_state) == 0 ? (T)1 : (T)0;
        v.y = (T)0;
        s[i] = v;
    }
}

}  // namespace

int tile_block_qubits(int qubits, int precision) {
    int k = precision == QM_FP32 ? 12 : 11;  // leaves room for the per-warp term sums in shared memory
    return k < qubits ? k : qubits;
}

cudaError_t launch_expect_tile(const void* amps, int qubits, int precision, const TilePass& tp, const TileTerm* terms,
                               int states, uint64_t state_stride, double* partials, int columns, int rows_per_state,
                               int mass_column, cudaStream_t st) {
    if (tp.term_count > kTileMaxTerms || tp.term_count < 0 || states < 1 || states > 65535)
        return cudaErrorInvalidValue;
#define QM_TILE_CASE(TT, KK)                                                                                   \
    case KK:                                                                                                   \
        return launch_tile_sized<TT, KK>(amps, qubits, tp, terms, states, state_stride, partials, columns,    \
                                         rows_per_state, mass_column, st);
    if (precision == QM_FP32) {
        switch (tp.k) {
            QM_TILE_CASE(float, 9) QM_TILE_CASE(float, 10) QM_TILE_CASE(float, 11) QM_TILE_CASE(float, 12)
        default: return cudaErrorInvalidValue;
        }
    }
    switch (tp.k) {
        QM_TILE_CASE(double, 9) QM_TILE_CASE(double, 10) QM_TILE_CASE(double, 11)
    default: return cudaErrorInvalidValue;
    }
#undef QM_TILE_CASE
}

cudaError_t launch_finish_batched(const double* partials, int states, int rows, int columns, double* out,
                                  cudaStream_t st) {
    const int threads = 128;
    dim3 grid((columns * 32 + threads - 1) / threads, states);
    k_finish_batched<<<grid, threads, 0, st>>>(partials, rows, columns, out);
    return cudaGetLastError();
}

cudaError_t launch_reset_batched(void* amps, int qubits, int precision, int states, cudaStream_t st) {
    const uint64_t per = 1ull << qubits, total = per * (uint64_t)states;
    const uint64_t blocks = std::min<uint64_t>((total + 255) / 256, 148ull * 32);
    if (precision == QM_FP32) k_reset_batched<float><<<(unsigned)blocks, 256, 0, st>>>((float2*)amps, per, total);
    else k_reset_batched<double><<<(unsigned)blocks, 256, 0, st>>>((double2*)amps, per, total);
    return cudaGetLastError();
}

}  // namespace qm
