// qm_kernels.cu -- per-gate, noise, reduction and sampling kernels of libqmb200.so
// (sm_100a).  The fused multi-gate pass kernel lives in qm_fused.cu.
//
// All kernels here are streaming passes bounded by HBM bandwidth: every amplitude is
// read and written at most once per launch with 16-byte (complex128) or 8-byte
// (complex64) accesses that are contiguous across a warp whenever the gate's target
// is not among the lowest qubits.
#include <cuda_runtime.h>

#include <algorithm>

#include "qm_device.cuh"
#include "qm_internal.h"

namespace qm {

namespace {

constexpr int kThreads = 256;
constexpr int kItems = 2;  // independent pairs per thread (memory-level parallelism)

// Enumeration of the active pairs of one gate: the item index gets zero bits inserted at
// the target and every control position (ascending), then the controls are set.  Only
// pairs whose control bits are all one are visited, so controlled gates read and write
// only the amplitudes they change (CudaStateVectorKernel.cs:41-48 visits every pair and
// filters).
struct GateLaunch {
    uint32_t count;
    int32_t npos;
    int32_t pos[32];
    uint32_t set_mask;
    uint32_t target_bit;
    uint32_t swap_bit;
    int32_t a_is_one, d_is_one;
    double a[2], b[2], c[2], d[2];
};

__device__ __forceinline__ uint32_t first_of(const GateLaunch& L, uint32_t item) {
    uint32_t x = item;
    for (int i = 0; i < L.npos; ++i) x = insert_zero(x, L.pos[i]);
    return x | L.set_mask;
}

template <typename T, int KIND>
__global__ void __launch_bounds__(kThreads) k_gate(typename Vec2<T>::type* __restrict__ s, const GateLaunch L) {
    uint32_t base = (blockIdx.x * kThreads + threadIdx.x) * kItems;
    uint32_t firsts[kItems], seconds[kItems];
    bool live[kItems];
#pragma unroll
    for (int u = 0; u < kItems; ++u) {
        uint32_t item = base + u;
        live[u] = item < L.count;
        uint32_t f = first_of(L, live[u] ? item : 0);
        uint32_t g = f | L.target_bit;
        if (KIND == QM_KERNEL_SWAP) g = (f ^ L.swap_bit) | L.target_bit;
        firsts[u] = f;
        seconds[u] = g;
    }
    if (KIND == QM_KERNEL_DIAGONAL) {
        T ar = (T)L.a[0], ai = (T)L.a[1], dr = (T)L.d[0], di = (T)L.d[1];
        Cx<T> x[kItems], y[kItems];
#pragma unroll
        for (int u = 0; u < kItems; ++u) {
            if (!live[u]) continue;
            if (!L.a_is_one) x[u] = load_amp<T>(s, firsts[u]);
            if (!L.d_is_one) y[u] = load_amp<T>(s, seconds[u]);
        }
#pragma unroll
        for (int u = 0; u < kItems; ++u) {
            if (!live[u]) continue;
            if (!L.a_is_one) store_amp<T>(s, firsts[u], cmul<T>(ar, ai, x[u]));
            if (!L.d_is_one) store_amp<T>(s, seconds[u], cmul<T>(dr, di, y[u]));
        }
        return;
    }
    Cx<T> x[kItems], y[kItems];
#pragma unroll
    for (int u = 0; u < kItems; ++u) {
        if (!live[u]) continue;
        x[u] = load_amp<T>(s, firsts[u]);
        y[u] = load_amp<T>(s, seconds[u]);
    }
#pragma unroll
    for (int u = 0; u < kItems; ++u) {
        if (!live[u]) continue;
        Cx<T> o0, o1;
        if (KIND == QM_KERNEL_EXCHANGE || KIND == QM_KERNEL_SWAP) {
            o0 = y[u];
            o1 = x[u];
        } else if (KIND == QM_KERNEL_HADAMARD) {
            T h = (T)L.a[0];
            o0 = Cx<T>{h * x[u].re + h * y[u].re, h * x[u].im + h * y[u].im};
            o1 = Cx<T>{h * x[u].re - h * y[u].re, h * x[u].im - h * y[u].im};
        } else {
            o0 = cmac2<T>((T)L.a[0], (T)L.a[1], x[u], (T)L.b[0], (T)L.b[1], y[u]);
            o1 = cmac2<T>((T)L.c[0], (T)L.c[1], x[u], (T)L.d[0], (T)L.d[1], y[u]);
        }
        store_amp<T>(s, firsts[u], o0);
        store_amp<T>(s, seconds[u], o1);
    }
}

template <typename T>
cudaError_t launch_gate_t(void* amps, int qubits, const DevGate& g, cudaStream_t st) {
    GateLaunch L;
    uint32_t positions = g.target_bit | g.control_mask | g.swap_bit;
    L.npos = 0;
    for (int b = 0; b < 32; ++b)
        if (positions & (1u << b)) L.pos[L.npos++] = b;
    if (L.npos > qubits) return cudaErrorInvalidValue;
    L.count = (uint32_t)((1ull << qubits) >> L.npos);
    L.set_mask = g.control_mask | g.swap_bit;
    L.target_bit = g.target_bit;
    L.swap_bit = g.swap_bit;
    L.a_is_one = g.a_is_one;
    L.d_is_one = g.d_is_one;
    for (int i = 0; i < 2; ++i) {
        L.a[i] = g.a[i]; L.b[i] = g.b[i]; L.c[i] = g.c[i]; L.d[i] = g.d[i];
    }
    if (L.count == 0) return cudaSuccess;
    uint32_t per_block = kThreads * kItems;
    dim3 grid((L.count + per_block - 1) / per_block);
    auto* s = reinterpret_cast<typename Vec2<T>::type*>(amps);
    switch (g.kernel) {
    case QM_KERNEL_MATRIX: k_gate<T, QM_KERNEL_MATRIX><<<grid, kThreads, 0, st>>>(s, L); break;
    case QM_KERNEL_HADAMARD: k_gate<T, QM_KERNEL_HADAMARD><<<grid, kThreads, 0, st>>>(s, L); break;
    case QM_KERNEL_EXCHANGE: k_gate<T, QM_KERNEL_EXCHANGE><<<grid, kThreads, 0, st>>>(s, L); break;
    case QM_KERNEL_DIAGONAL:
        if (g.a_is_one && g.d_is_one) return cudaSuccess;
        k_gate<T, QM_KERNEL_DIAGONAL><<<grid, kThreads, 0, st>>>(s, L);
        break;
    case QM_KERNEL_SWAP: k_gate<T, QM_KERNEL_SWAP><<<grid, kThreads, 0, st>>>(s, L); break;
    default: return cudaSuccess;  // identity
    }
    return cudaGetLastError();
}

// ---------------------------------------------------------------- state utilities

template <typename T>
__global__ void k_reset(typename Vec2<T>::type* s, uint64_t n) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (; i < n; i += stride) store_amp<T>(s, i, Cx<T>{i == 0 ? (T)1 : (T)0, (T)0});
}

__global__ void k_f64_to_f32(float2* dst, const double2* src, uint64_t n) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (; i < n; i += stride) {
        double2 v = src[i];
        dst[i] = make_float2((float)v.x, (float)v.y);
    }
}

__global__ void k_f32_to_f64(double2* dst, const float2* src, uint64_t n) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (; i < n; i += stride) {
        float2 v = src[i];
        dst[i] = make_double2((double)v.x, (double)v.y);
    }
}

int stream_blocks(uint64_t n) {
    uint64_t b = (n + kThreads - 1) / kThreads;
    return (int)std::min<uint64_t>(b, 148ull * 16);
}

// ---------------------------------------------------------------- noise

// Masses of target-zero and target-one amplitudes (CpuNoiseChannelBackend.cs:88-106):
// compensated FP64 per thread, deterministic block tree; one (zero, one) pair of
// compensated partials per block.
template <typename T>
__global__ void __launch_bounds__(kThreads) k_masses(const typename Vec2<T>::type* __restrict__ s, uint32_t pairs,
                                                     int target, double* out) {
    __shared__ KSum red[kThreads / 32];
    KSum z{0, 0}, o{0, 0};
    uint32_t bit = 1u << target;
    for (uint32_t p = blockIdx.x * kThreads + threadIdx.x; p < pairs; p += gridDim.x * kThreads) {
        uint32_t f = insert_zero(p, target);
        Cx<T> x = load_amp<T>(s, f), y = load_amp<T>(s, f | bit);
        double xr = x.re, xi = x.im, yr = y.re, yi = y.im;
        z.add(xr * xr + xi * xi);
        o.add(yr * yr + yi * yi);
    }
    KSum zt = block_reduce_ksum(z, red);
    KSum ot = block_reduce_ksum(o, red);
    if (threadIdx.x == 0) {
        out[4 * blockIdx.x + 0] = zt.s;
        out[4 * blockIdx.x + 1] = zt.c;
        out[4 * blockIdx.x + 2] = ot.s;
        out[4 * blockIdx.x + 3] = ot.c;
    }
}

// Pauli branch (CpuNoiseChannelBackend.cs:59-80): X swaps, Y swaps with phases
// (psi0' = -i psi1, psi1' = i psi0), Z negates the target-one half.
template <typename T>
__global__ void __launch_bounds__(kThreads) k_pauli(typename Vec2<T>::type* __restrict__ s, uint32_t pairs, int target,
                                                    int pauli) {
    uint32_t bit = 1u << target;
    for (uint32_t p = blockIdx.x * kThreads + threadIdx.x; p < pairs; p += gridDim.x * kThreads) {
        uint32_t f = insert_zero(p, target);
        if (pauli == 3) {
            Cx<T> y = load_amp<T>(s, f | bit);
            store_amp<T>(s, f | bit, Cx<T>{-y.re, -y.im});
            continue;
        }
        Cx<T> x = load_amp<T>(s, f), y = load_amp<T>(s, f | bit);
        if (pauli == 1) {
            store_amp<T>(s, f, y);
            store_amp<T>(s, f | bit, x);
        } else {
            store_amp<T>(s, f, Cx<T>{y.im, -y.re});
            store_amp<T>(s, f | bit, Cx<T>{-x.im, x.re});
        }
    }
}

// Damping branch (CpuNoiseChannelBackend.cs:118-142).  Scales arrive in FP64 and are
// applied in the state's precision.
template <typename T>
__global__ void __launch_bounds__(kThreads) k_damping(typename Vec2<T>::type* __restrict__ s, uint32_t pairs,
                                                      int target, int jump, double scale, double jump_scale,
                                                      double stay_scale) {
    uint32_t bit = 1u << target;
    for (uint32_t p = blockIdx.x * kThreads + threadIdx.x; p < pairs; p += gridDim.x * kThreads) {
        uint32_t f = insert_zero(p, target);
        Cx<T> y = load_amp<T>(s, f | bit);
        if (jump) {
            store_amp<T>(s, f, Cx<T>{(T)(jump_scale * (double)y.re), (T)(jump_scale * (double)y.im)});
            store_amp<T>(s, f | bit, Cx<T>{(T)0, (T)0});
        } else {
            Cx<T> x = load_amp<T>(s, f);
            store_amp<T>(s, f, Cx<T>{(T)((double)x.re * scale), (T)((double)x.im * scale)});
            store_amp<T>(s, f | bit, Cx<T>{(T)((double)y.re * stay_scale), (T)((double)y.im * stay_scale)});
        }
    }
}

// ---------------------------------------------------------------- observables

// One pass per distinct flip mask F.  Each pair {j, j^F} is read once; every term of the
// group (same F) gets conj(psi[j^F]) psi[j] times its Y phase and Z sign for both members
// (StateVector.Observations.cs:115-132).  With F == 0 each amplitude is its own partner.
// The Born mass rides along in the F == 0 pass as an extra column.
constexpr int kGroupMax = 8;
struct GroupLaunch {
    uint32_t flip;
    int32_t low;          // lowest set bit of flip (pair enumeration); -1 when flip == 0
    int32_t terms;        // <= kGroupMax
    int32_t with_mass;
    uint32_t sign[kGroupMax];
    int32_t phase[kGroupMax];  // y_count & 3
    int32_t column[kGroupMax]; // output column of each term
    int32_t mass_column;
    int32_t columns;           // row width of the partial table
};

template <typename T>
__global__ void __launch_bounds__(kThreads) k_pauli_group(const typename Vec2<T>::type* __restrict__ s, uint32_t items,
                                                          const GroupLaunch L, double* partials) {
    __shared__ KSum red[kThreads / 32];
    KSum acc[kGroupMax + 1];
#pragma unroll
    for (int t = 0; t <= kGroupMax; ++t) acc[t] = KSum{0, 0};
    for (uint32_t it = blockIdx.x * kThreads + threadIdx.x; it < items; it += gridDim.x * kThreads) {
        if (L.low < 0) {
            Cx<T> v = load_amp<T>(s, it);
            double p = (double)v.re * (double)v.re + (double)v.im * (double)v.im;
#pragma unroll
            for (int t = 0; t < kGroupMax; ++t) {
                if (t >= L.terms) break;
                // overlap = |psi|^2 (real); phase classes 1 and 3 take its zero imaginary part
                double c = (L.phase[t] & 1) ? 0.0 : (L.phase[t] == 2 ? -p : p);
                acc[t].add((__popc(it & L.sign[t]) & 1) ? -c : c);
            }
            if (L.with_mass) acc[kGroupMax].add(p);
        } else {
            uint32_t j = insert_zero(it, L.low);
            uint32_t k = j ^ L.flip;
            Cx<T> a = load_amp<T>(s, j), b = load_amp<T>(s, k);
            double ar = a.re, ai = a.im, br = b.re, bi = b.im;
            // conj(psi_k) psi_j; the partner's overlap is its conjugate
            double ore = br * ar + bi * ai;
            double oim = br * ai - bi * ar;
#pragma unroll
            for (int t = 0; t < kGroupMax; ++t) {
                if (t >= L.terms) break;
                double cj, ck;
                switch (L.phase[t]) {
                case 0: cj = ore; ck = ore; break;
                case 1: cj = -oim; ck = oim; break;
                case 2: cj = -ore; ck = -ore; break;
                default: cj = oim; ck = -oim; break;
                }
                if (__popc(j & L.sign[t]) & 1) cj = -cj;
                if (__popc(k & L.sign[t]) & 1) ck = -ck;
                acc[t].add(cj + ck);
            }
            if (L.with_mass) acc[kGroupMax].add(ar * ar + ai * ai + br * br + bi * bi);
        }
    }
    for (int t = 0; t < L.terms; ++t) {
        KSum r = block_reduce_ksum(acc[t], red);
        if (threadIdx.x == 0) partials[(size_t)blockIdx.x * L.columns + L.column[t]] = r.value();
    }
    if (L.with_mass) {
        KSum r = block_reduce_ksum(acc[kGroupMax], red);
        if (threadIdx.x == 0) partials[(size_t)blockIdx.x * L.columns + L.mass_column] = r.value();
    }
}

// Column sums of a [rows][columns] table in fixed order: one warp per column.
__global__ void k_finish_sums(const double* __restrict__ partials, int rows, int columns, double* out) {
    int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    if (warp >= columns) return;
    KSum acc{0, 0};
    for (int r = lane; r < rows; r += 32) acc.add(partials[(size_t)r * columns + warp]);
    for (int d = 16; d > 0; d >>= 1) acc.merge(shfl_down_ksum(acc, d));
    if (lane == 0) out[warp] = acc.value();
}

// ---------------------------------------------------------------- sampling

// Probability mass of each contiguous chunk and the last supported index in it.
template <typename T>
__global__ void __launch_bounds__(kThreads) k_block_probs(const typename Vec2<T>::type* __restrict__ s, uint32_t chunk,
                                                          double* sums, int64_t* last) {
    __shared__ KSum red[kThreads / 32];
    __shared__ int64_t lastw[kThreads / 32];
    uint32_t begin = blockIdx.x * chunk;
    KSum acc{0, 0};
    int64_t my_last = -1;
    for (uint32_t i = threadIdx.x; i < chunk; i += kThreads) {
        Cx<T> v = load_amp<T>(s, begin + i);
        double p = (double)v.re * (double)v.re + (double)v.im * (double)v.im;
        acc.add(p);
        if (p > 0) my_last = begin + i;
    }
    for (int d = 16; d > 0; d >>= 1) {
        int64_t o = __shfl_down_sync(0xffffffffu, my_last, d);
        my_last = o > my_last ? o : my_last;
    }
    if ((threadIdx.x & 31) == 0) lastw[threadIdx.x >> 5] = my_last;
    KSum r = block_reduce_ksum(acc, red);
    if (threadIdx.x == 0) {
        int64_t m = -1;
        for (int w = 0; w < kThreads / 32; ++w) m = lastw[w] > m ? lastw[w] : m;
        sums[blockIdx.x] = r.value();
        last[blockIdx.x] = m;
    }
}

// One warp per shot: locate the chunk from the FP64 chunk prefix, then scan it with a warp
// prefix sum to the first index whose cumulative mass exceeds the target (the strict upper
// bound of StateVectorSimulator.cs:72-88).  If rounding carries the target past a chunk,
// the scan continues into the following chunks.  out[shot] = index, or -1 when the target
// lies beyond the final cumulative mass (the caller then takes the last supported index).
// out[shots + shot] = 1 when the target lies within `margin` of the cumulative mass at the
// chosen boundary.
template <typename T>
__global__ void k_search(const typename Vec2<T>::type* __restrict__ s, const double* __restrict__ prefix, int blocks,
                         uint32_t chunk, const double* __restrict__ targets, int shots, double margin,
                         int64_t* out) {
    int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    if (warp >= shots) return;
    double t = targets[warp];
    // last chunk whose starting prefix is <= t
    int lo = 0, hi = blocks;  // prefix has blocks+1 entries
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (prefix[mid + 1] <= t) lo = mid + 1; else hi = mid;
    }
    int64_t found = -1;
    int ambiguous = 0;
    for (int b = lo; b < blocks && found < 0; ++b) {
        double running = prefix[b];
        uint32_t begin = (uint32_t)b * chunk;
        for (uint32_t off = 0; off < chunk; off += 32) {
            double p = 0.0;
            if (off + lane < chunk) {
                Cx<T> v = load_amp<T>(s, begin + off + lane);
                p = (double)v.re * (double)v.re + (double)v.im * (double)v.im;
            }
            double inc = p;
            for (int d = 1; d < 32; d <<= 1) {
                double o = __shfl_up_sync(0xffffffffu, inc, d);
                if (lane >= d) inc += o;
            }
            double cum = running + inc;
            unsigned hit = __ballot_sync(0xffffffffu, cum > t);
            if (hit) {
                int l = __ffs(hit) - 1;
                double at = __shfl_sync(0xffffffffu, cum, l);
                double before = __shfl_sync(0xffffffffu, cum - p, l);
                found = begin + off + l;
                // the reference's CDF could still be <= t here (it would pick a later index),
                // or could already exceed t one supported index earlier; with no mass before
                // this index there is no earlier outcome to pick
                ambiguous = (at - t <= margin) || (before > 0 && t - before <= margin);
                break;
            }
            running = __shfl_sync(0xffffffffu, cum, 31);
        }
    }
    if (lane == 0) {
        out[warp] = found;
        out[shots + warp] = ambiguous || (found < 0);
    }
}

// Born masses of the amplitudes whose masked bits equal `pattern` and of all amplitudes
// (StateVector.MarginalProbability and Measure's branch mass, StateVector.Observations.cs:10-88):
// compensated FP64 per thread, deterministic block tree, (selected, total) per block.
template <typename T>
__global__ void __launch_bounds__(kThreads) k_pattern_masses(const typename Vec2<T>::type* __restrict__ s, uint64_t n,
                                                             uint64_t mask, uint64_t pattern, double* out) {
    __shared__ KSum red[kThreads / 32];
    KSum sel{0, 0}, tot{0, 0};
    for (uint64_t i = (uint64_t)blockIdx.x * kThreads + threadIdx.x; i < n; i += (uint64_t)gridDim.x * kThreads) {
        const Cx<T> x = load_amp<T>(s, i);
        const double xr = x.re, xi = x.im;
        const double p = xr * xr + xi * xi;
        tot.add(p);
        if ((i & mask) == pattern) sel.add(p);
    }
    KSum st = block_reduce_ksum(sel, red);
    KSum tt = block_reduce_ksum(tot, red);
    if (threadIdx.x == 0) {
        out[4 * blockIdx.x + 0] = st.s;
        out[4 * blockIdx.x + 1] = st.c;
        out[4 * blockIdx.x + 2] = tt.s;
        out[4 * blockIdx.x + 3] = tt.c;
    }
}

// Measure's projection (StateVector.Observations.cs:86-93): the matching branch divided by the
// square root of its mass, every other amplitude zero.
template <typename T>
__global__ void k_project(typename Vec2<T>::type* s, uint64_t n, uint64_t mask, uint64_t pattern, double norm) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        Cx<T> x = load_amp<T>(s, i);
        if ((i & mask) == pattern) {
            x.re = (T)((double)x.re / norm);
            x.im = (T)((double)x.im / norm);
        } else {
            x.re = (T)0;
            x.im = (T)0;
        }
        store_amp<T>(s, i, x);
    }
}

template <typename T>
__global__ void k_collapse(typename Vec2<T>::type* s, uint64_t n, uint64_t outcome) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (; i < n; i += stride) store_amp<T>(s, i, Cx<T>{i == outcome ? (T)1 : (T)0, (T)0});
}

}  // namespace

// ---------------------------------------------------------------- launchers

cudaError_t launch_gate(void* amps, int qubits, int precision, const DevGate& g, cudaStream_t s) {
    return precision == QM_FP32 ? launch_gate_t<float>(amps, qubits, g, s) : launch_gate_t<double>(amps, qubits, g, s);
}

cudaError_t launch_reset(void* amps, int qubits, int precision, cudaStream_t st) {
    uint64_t n = 1ull << qubits;
    if (precision == QM_FP32) k_reset<float><<<stream_blocks(n), kThreads, 0, st>>>((float2*)amps, n);
    else k_reset<double><<<stream_blocks(n), kThreads, 0, st>>>((double2*)amps, n);
    return cudaGetLastError();
}

cudaError_t launch_convert_from_f64(void* dst, const double* src, int64_t n, cudaStream_t st) {
    k_f64_to_f32<<<stream_blocks((uint64_t)n), kThreads, 0, st>>>((float2*)dst, (const double2*)src, (uint64_t)n);
    return cudaGetLastError();
}

cudaError_t launch_convert_to_f64(double* dst, const void* src, int64_t n, cudaStream_t st) {
    k_f32_to_f64<<<stream_blocks((uint64_t)n), kThreads, 0, st>>>((double2*)dst, (const float2*)src, (uint64_t)n);
    return cudaGetLastError();
}

static int reduce_blocks(uint64_t items) {
    uint64_t b = (items + kThreads * 8 - 1) / (kThreads * 8);
    return (int)std::max<uint64_t>(1, std::min<uint64_t>(b, (uint64_t)kReduceBlocksMax));
}

cudaError_t launch_masses(const void* amps, int qubits, int precision, int target, double* scratch, int* blocks_out,
                          cudaStream_t st) {
    uint32_t pairs = (uint32_t)((1ull << qubits) >> 1);
    int blocks = reduce_blocks(pairs);
    *blocks_out = blocks;
    if (precision == QM_FP32) k_masses<float><<<blocks, kThreads, 0, st>>>((const float2*)amps, pairs, target, scratch);
    else k_masses<double><<<blocks, kThreads, 0, st>>>((const double2*)amps, pairs, target, scratch);
    return cudaGetLastError();
}

cudaError_t launch_pauli(void* amps, int qubits, int precision, int target, int pauli, cudaStream_t st) {
    uint32_t pairs = (uint32_t)((1ull << qubits) >> 1);
    int blocks = stream_blocks(pairs);
    if (precision == QM_FP32) k_pauli<float><<<blocks, kThreads, 0, st>>>((float2*)amps, pairs, target, pauli);
    else k_pauli<double><<<blocks, kThreads, 0, st>>>((double2*)amps, pairs, target, pauli);
    return cudaGetLastError();
}

cudaError_t launch_damping(void* amps, int qubits, int precision, int target, int jump, double scale,
                           double jump_scale, double stay_scale, cudaStream_t st) {
    uint32_t pairs = (uint32_t)((1ull << qubits) >> 1);
    int blocks = stream_blocks(pairs);
    if (precision == QM_FP32)
        k_damping<float><<<blocks, kThreads, 0, st>>>((float2*)amps, pairs, target, jump, scale, jump_scale, stay_scale);
    else
        k_damping<double><<<blocks, kThreads, 0, st>>>((double2*)amps, pairs, target, jump, scale, jump_scale, stay_scale);
    return cudaGetLastError();
}

// Groups terms by flip mask and runs one pass per group (chunks of kGroupMax terms).
// Partials table: [blocks][terms + 1]; the last column is the Born mass.
cudaError_t launch_expectation(const void* amps, int qubits, int precision, const DevPauli* terms, int count,
                               double* scratch, int* blocks_out, cudaStream_t st) {
    uint64_t n = 1ull << qubits;
    int columns = count + 1;
    int blocks = reduce_blocks(n);
    *blocks_out = blocks;
    std::vector<int> order(count);
    for (int i = 0; i < count; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return terms[x].flip < terms[y].flip; });
    bool mass_done = false;
    size_t i = 0;
    auto run = [&](GroupLaunch& L) -> cudaError_t {
        L.columns = columns;
        L.mass_column = count;
        uint32_t items = L.low < 0 ? (uint32_t)n : (uint32_t)(n >> 1);
        if (precision == QM_FP32)
            k_pauli_group<float><<<blocks, kThreads, 0, st>>>((const float2*)amps, items, L, scratch);
        else
            k_pauli_group<double><<<blocks, kThreads, 0, st>>>((const double2*)amps, items, L, scratch);
        return cudaGetLastError();
    };
    while (i < order.size()) {
        uint32_t flip = terms[order[i]].flip;
        GroupLaunch L{};
        L.flip = flip;
        L.low = flip ? __builtin_ctz(flip) : -1;
        L.terms = 0;
        while (i < order.size() && terms[order[i]].flip == flip && L.terms < kGroupMax) {
            int t = order[i++];
            L.sign[L.terms] = terms[t].sign;
            L.phase[L.terms] = terms[t].phase & 3;
            L.column[L.terms] = t;
            ++L.terms;
        }
        L.with_mass = !mass_done;
        mass_done = true;
        cudaError_t e = run(L);
        if (e != cudaSuccess) return e;
    }
    if (!mass_done) {
        GroupLaunch L{};
        L.flip = 0;
        L.low = -1;
        L.terms = 0;
        L.with_mass = 1;
        cudaError_t e = run(L);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

int expectation_blocks(int qubits) { return reduce_blocks(1ull << qubits); }

cudaError_t launch_pauli_group(const void* amps, int qubits, int precision, uint32_t flip, int terms,
                               const uint32_t* sign, const int32_t* phase, const int32_t* column, int with_mass,
                               int mass_column, int columns, double* partials, cudaStream_t st) {
    if (terms < 0 || terms > kGroupMax) return cudaErrorInvalidValue;
    const uint64_t n = 1ull << qubits;
    GroupLaunch L{};
    L.flip = flip;
    L.low = flip ? __builtin_ctz(flip) : -1;
    L.terms = terms;
    L.with_mass = with_mass;
    for (int t = 0; t < terms; ++t) {
        L.sign[t] = sign[t];
        L.phase[t] = phase[t] & 3;
        L.column[t] = column[t];
    }
    L.columns = columns;
    L.mass_column = mass_column;
    const uint32_t items = L.low < 0 ? (uint32_t)n : (uint32_t)(n >> 1);
    const int blocks = reduce_blocks(n);
    if (precision == QM_FP32)
        k_pauli_group<float><<<blocks, kThreads, 0, st>>>((const float2*)amps, items, L, partials);
    else
        k_pauli_group<double><<<blocks, kThreads, 0, st>>>((const double2*)amps, items, L, partials);
    return cudaGetLastError();
}

cudaError_t launch_finish_sums(const double* partials, int rows, int columns, double* out, cudaStream_t st) {
    int threads = 128;
    int blocks = (columns * 32 + threads - 1) / threads;
    k_finish_sums<<<blocks, threads, 0, st>>>(partials, rows, columns, out);
    return cudaGetLastError();
}

cudaError_t launch_block_probs(const void* amps, int qubits, int precision, double* sums, int64_t* last,
                               int* blocks_out, int* chunk_out, cudaStream_t st) {
    uint64_t n = 1ull << qubits;
    uint64_t chunk = std::max<uint64_t>(1024, n / (148 * 8));
    // chunks are powers of two that divide n
    uint64_t c = 1;
    while (c < chunk) c <<= 1;
    if (c > n) c = n;
    int blocks = (int)(n / c);
    *blocks_out = blocks;
    *chunk_out = (int)c;
    if (precision == QM_FP32)
        k_block_probs<float><<<blocks, kThreads, 0, st>>>((const float2*)amps, (uint32_t)c, sums, last);
    else
        k_block_probs<double><<<blocks, kThreads, 0, st>>>((const double2*)amps, (uint32_t)c, sums, last);
    return cudaGetLastError();
}

cudaError_t launch_search(const void* amps, int qubits, int precision, const double* prefix, int blocks, int chunk,
                          const double* targets, int shots, double margin, int64_t* out, cudaStream_t st) {
    (void)qubits;
    int threads = 128;
    int grid = (shots * 32 + threads - 1) / threads;
    if (precision == QM_FP32)
        k_search<float><<<grid, threads, 0, st>>>((const float2*)amps, prefix, blocks, (uint32_t)chunk, targets, shots,
                                                  margin, out);
    else
        k_search<double><<<grid, threads, 0, st>>>((const double2*)amps, prefix, blocks, (uint32_t)chunk, targets, shots,
                                                   margin, out);
    return cudaGetLastError();
}

cudaError_t launch_pattern_masses(const void* amps, int qubits, int precision, uint64_t mask, uint64_t pattern,
                                  double* scratch, int* blocks_out, cudaStream_t st) {
    const uint64_t n = 1ull << qubits;
    const int blocks = reduce_blocks(n);
    *blocks_out = blocks;
    if (precision == QM_FP32)
        k_pattern_masses<float><<<blocks, kThreads, 0, st>>>((const float2*)amps, n, mask, pattern, scratch);
    else
        k_pattern_masses<double><<<blocks, kThreads, 0, st>>>((const double2*)amps, n, mask, pattern, scratch);
    return cudaGetLastError();
}

cudaError_t launch_project(void* amps, int qubits, int precision, uint64_t mask, uint64_t pattern, double norm,
                           cudaStream_t st) {
    const uint64_t n = 1ull << qubits;
    if (precision == QM_FP32)
        k_project<float><<<stream_blocks(n), kThreads, 0, st>>>((float2*)amps, n, mask, pattern, norm);
    else
        k_project<double><<<stream_blocks(n), kThreads, 0, st>>>((double2*)amps, n, mask, pattern, norm);
    return cudaGetLastError();
}

cudaError_t launch_collapse(void* amps, int qubits, int precision, int64_t outcome, cudaStream_t st) {
    uint64_t n = 1ull << qubits;
    if (precision == QM_FP32) k_collapse<float><<<stream_blocks(n), kThreads, 0, st>>>((float2*)amps, n, (uint64_t)outcome);
    else k_collapse<double><<<stream_blocks(n), kThreads, 0, st>>>((double2*)amps, n, (uint64_t)outcome);
    return cudaGetLastError();
}

}  // namespace qm
