// qm_noise.cu -- device side of the batched noise-trajectory runner of libqmb200.so.
//
// CpuNoiseChannelBackend (src/QuantumMatter.Infrastructure/CpuNoiseChannelBackend.cs:10-145)
// decides each channel placement of one trajectory on the host: a Pauli branch from one draw,
// a damping branch from the Kahan masses of the target's zero and one halves and one draw,
// then a full pass over the state.  Here many trajectories run as the states of one batch and
// every decision is taken on the device, in program order per trajectory:
//   - each trajectory carries a Pauli frame (X^fx Z^fz): a selected Pauli error only updates
//     the frame, so Pauli channels cost no pass at all; gates and Kraus operators run
//     conjugated by the frame (F U F, an exact permutation and sign change of U's entries);
//   - k_group_hist reads the states once for a whole run of consecutive dampings and writes the
//     joint Born masses over their qubits (at most 8 of them, 256 bins) per state;
//   - k_decide (one warp per trajectory) walks the trajectory's steps: consumes its draws, takes
//     the Pauli and damping decisions with the reference's thresholds, tracks how each damping
//     reshapes the joint masses for the next one, updates the frame, and writes each
//     conjugated gate or Kraus operator into the coefficient table read by the next fused pass;
//   - k_welford accumulates the per-index Born probabilities of finished trajectories in
//     trajectory order (NoisyStateVectorSimulator.EstimateProbabilities, :64-106).
// All sums run in FP64 in a fixed order, so results do not depend on scheduling or batching.
#include <cuda_runtime.h>

#include <cmath>

#include "qm_internal.h"

namespace qm {

namespace {

__device__ __forceinline__ double prob(const float2* s, uint64_t i) {
    const float2 v = s[i];
    const double re = v.x, im = v.y;
    return re * re + im * im;  // exact products of floats, one rounding
}
__device__ __forceinline__ double prob(const double2* s, uint64_t i) {
    const double2 v = s[i];
    return v.x * v.x + v.y * v.y;
}

constexpr int kHistThreads = 256;
constexpr int kHistWarps = kHistThreads / 32;
constexpr int kHistUnroll = 8;

struct HistArgs {
    uint64_t state_len;    // amplitudes per state (stride)
    uint64_t per_warp;     // amplitudes per warp, a multiple of 32
    int32_t ctas;          // CTAs per state
    int32_t bins;
    uint32_t glow;         // group bits among the five lane bits of an index
    int32_t nbits;
    int8_t pos[kGroupMaxBits];  // group qubits, ascending: qubit pos[j] is bin bit j
};

__device__ __forceinline__ uint32_t bin_of(uint64_t index, const HistArgs& h) {
    uint32_t b = 0;
    for (int j = 0; j < h.nbits; ++j) b |= (uint32_t)((index >> h.pos[j]) & 1u) << j;
    return b;
}

// Each warp reads runs of 32 consecutive amplitudes.  A butterfly over the lane bits that are
// not group bits leaves every lane with the sum of its bin within the run; the lanes whose
// non-group lane bits are zero add it to the warp's own bin row (distinct bins, no conflicts,
// fixed order).  The CTA then sums its warp rows in order.  Bins are in stored coordinates.
template <typename V>
__global__ void __launch_bounds__(kHistThreads) k_group_hist(const V* __restrict__ amps, const HistArgs h,
                                                             double* __restrict__ partials) {
    __shared__ double acc[kHistWarps][kGroupMaxBins];
    for (int i = threadIdx.x; i < kHistWarps * kGroupMaxBins; i += kHistThreads) (&acc[0][0])[i] = 0.0;
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int state = blockIdx.x / h.ctas;
    const int cta = blockIdx.x - state * h.ctas;
    const V* s = amps + (uint64_t)state * h.state_len;
    const uint64_t wbegin = ((uint64_t)cta * kHistWarps + warp) * h.per_warp;
    const bool writer = ((uint32_t)lane & ~h.glow) == 0;
    for (uint64_t c = 0; c < h.per_warp; c += 32 * kHistUnroll) {
        double p[kHistUnroll];
#pragma unroll
        for (int u = 0; u < kHistUnroll; ++u)
            p[u] = (c + 32 * u < h.per_warp) ? prob(s, wbegin + c + 32 * u + lane) : 0.0;
#pragma unroll
        for (int u = 0; u < kHistUnroll; ++u) {
            if (c + 32 * u >= h.per_warp) break;  // uniform across the warp
            double v = p[u];
#pragma unroll
            for (int m = 0; m < 5; ++m)
                if (!((h.glow >> m) & 1u)) v += __shfl_xor_sync(0xffffffffu, v, 1 << m);
            if (writer) acc[warp][bin_of(wbegin + c + 32 * u + lane, h)] += v;
        }
    }
    __syncthreads();
    double* out = partials + ((uint64_t)state * h.ctas + cta) * h.bins;
    for (int b = threadIdx.x; b < h.bins; b += kHistThreads) {
        double sum = 0.0;
        for (int w = 0; w < kHistWarps; ++w) sum += acc[w][b];
        out[b] = sum;
    }
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int m = 16; m >= 1; m >>= 1) v += __shfl_xor_sync(0xffffffffu, v, m);
    return v;  // the xor butterfly leaves the same bits in every lane
}

// F U F for the frame's Pauli X^ax Z^az on U's qubit: X U X swaps rows and columns, Z U Z
// negates the off-diagonal entries.
__device__ __forceinline__ void conjugate(double (&m)[8], uint32_t ax, uint32_t az) {
    if (ax) {
        double t0 = m[0], t1 = m[1];
        m[0] = m[6]; m[1] = m[7]; m[6] = t0; m[7] = t1;
        t0 = m[2]; t1 = m[3];
        m[2] = m[4]; m[3] = m[5]; m[4] = t0; m[5] = t1;
    }
    if (az) {
        m[2] = -m[2]; m[3] = -m[3]; m[4] = -m[4]; m[5] = -m[5];
    }
}

__device__ __forceinline__ uint32_t swap_bits(uint32_t v, uint32_t a, uint32_t b) {
    const uint32_t x = ((v >> a) ^ (v >> b)) & 1u;
    return v ^ ((x << a) | (x << b));
}

constexpr int kDecideWarps = 4;

__global__ void __launch_bounds__(32 * kDecideWarps) k_decide(const DecideArgs a, int states) {
    __shared__ double hist_all[kDecideWarps][kGroupMaxBins];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int state = blockIdx.x * kDecideWarps + warp;
    if (state >= states) return;  // whole warps leave together
    double* hs = hist_all[warp];
    int status = a.status[state];
    if (status != QM_OK) return;
    if (a.partials) {
        const double* part = a.partials + (uint64_t)state * a.ctas * a.bins;
        for (int b = lane; b < a.bins; b += 32) {
            double sum = 0.0;
            for (int c = 0; c < a.ctas; ++c) sum += part[(uint64_t)c * a.bins + b];
            hs[b] = sum;
        }
        __syncwarp();
    }
    uint32_t fx = a.frame_x[state], fz = a.frame_z[state];
    int counter = a.counters[state];
    int amb = 0;
    const double* draws = a.draws + (uint64_t)state * a.draw_stride;
    double* row = a.table + (uint64_t)state * a.table_stride;
    for (int d = 0; d < a.count; ++d) {
        const Decision& D = a.decisions[d];
        const int kind = D.kind;
        const uint32_t qa = 1u << D.a;
        double co[8] = {1.0, 0.0, 0.0, 0.0, 0.0, 0.0, 1.0, 0.0};
        int branch = -1;
        switch (kind) {
        case STEP_PAULI_BIT_FLIP:
        case STEP_PAULI_PHASE_FLIP:
        case STEP_PAULI_DEPOLARIZING: {
            // CpuNoiseChannelBackend.Apply Pauli selection (:40-52); the error joins the frame
            if (counter >= a.draw_stride) {
                status = QM_E_RANGE;
                break;
            }
            const double u = draws[counter++];
            int pauli;
            if (kind == STEP_PAULI_DEPOLARIZING) {
                const double quarter = D.p / 4;
                pauli = u < quarter ? 1 : u < 2 * quarter ? 2 : u < 3 * quarter ? 3 : 0;
            } else {
                pauli = u < D.p ? (kind == STEP_PAULI_BIT_FLIP ? 1 : 3) : 0;
            }
            if (pauli == 1 || pauli == 2) fx ^= qa;
            if (pauli == 2 || pauli == 3) fz ^= qa;
            branch = pauli;
            break;
        }
        case STEP_DAMPING: {
            // CpuNoiseChannelBackend.ApplyDamping (:85-145) on the tracked joint masses.  The
            // histogram is in stored coordinates; the true state's bit is the stored one ^ ax.
            const uint32_t bit = 1u << D.bit;
            const uint32_t ax = (fx >> D.a) & 1u, az = (fz >> D.a) & 1u;
            double m0 = 0.0, m1 = 0.0;
            for (int b = lane; b < a.bins; b += 32) {
                if ((((uint32_t)b >> D.bit) & 1u) ^ ax) m1 += hs[b];
                else m0 += hs[b];
            }
            m0 = warp_sum(m0);
            m1 = warp_sum(m1);
            const double jump_mass = D.p * m1;
            const double stay_mass = m0 + (1 - D.p) * m1;
            const double total = jump_mass + stay_mass;
            if (!isfinite(total) || total <= 0) {
                status = QM_E_MASS;
                break;
            }
            bool jump;
            if (jump_mass > 0 && stay_mass != 0) {
                if (counter >= a.draw_stride) {
                    status = QM_E_RANGE;
                    break;
                }
                const double u = draws[counter++];
                const double ratio = jump_mass / total;
                jump = u < ratio;
                if (fabs(u - ratio) <= a.margin * ratio) ++amb;
            } else {
                jump = jump_mass > 0;
            }
            const double scale = 1 / sqrt(jump ? jump_mass : stay_mass);
            // stored bins whose true bit is one
            const uint32_t one = ax ? 0u : bit;
            __syncwarp();
            if (jump) {
                const double js = sqrt(D.p) * scale;
                co[0] = 0.0;
                co[2] = js;
                co[6] = 0.0;
                const double w = js * js;
                for (int b = lane; b < a.bins; b += 32)
                    if (((uint32_t)b & bit) != one) hs[b] = w * hs[b ^ bit];
                __syncwarp();
                for (int b = lane; b < a.bins; b += 32)
                    if (((uint32_t)b & bit) == one) hs[b] = 0.0;
            } else {
                const double ss = sqrt(1 - D.p) * scale;
                co[0] = scale;
                co[6] = ss;
                const double w0 = scale * scale, w1 = ss * ss;
                for (int b = lane; b < a.bins; b += 32) hs[b] *= (((uint32_t)b & bit) == one) ? w1 : w0;
            }
            __syncwarp();
            conjugate(co, ax, az);
            branch = jump ? 1 : 0;
            break;
        }
        case STEP_FRAME_X: fx ^= qa; break;
        case STEP_FRAME_Y: fx ^= qa; fz ^= qa; break;
        case STEP_FRAME_Z: fz ^= qa; break;
        case STEP_FRAME_H: {
            const uint32_t x = fx & qa, z = fz & qa;
            fx = (fx & ~qa) | z;
            fz = (fz & ~qa) | x;
            break;
        }
        case STEP_FRAME_S: fz ^= fx & qa; break;
        case STEP_FRAME_CNOT: {
            const uint32_t qb = 1u << D.b;  // control
            if (fx & qb) fx ^= qa;
            if (fz & qa) fz ^= qb;
            break;
        }
        case STEP_FRAME_CZ: {
            const uint32_t qb = 1u << D.b;
            const uint32_t xa = fx & qa, xb = fx & qb;
            if (xa) fz ^= qb;
            if (xb) fz ^= qa;
            break;
        }
        case STEP_FRAME_SWAP:
            fx = swap_bits(fx, (uint32_t)D.a, (uint32_t)D.b);
            fz = swap_bits(fz, (uint32_t)D.a, (uint32_t)D.b);
            break;
        case STEP_CONJ:
#pragma unroll
            for (int k = 0; k < 8; ++k) co[k] = D.coef[k];
            conjugate(co, (fx >> D.a) & 1u, (fz >> D.a) & 1u);
            break;
        case STEP_FLUSH_X:
            if (fx & qa) {
                co[0] = 0.0; co[2] = 1.0; co[4] = 1.0; co[6] = 0.0;
                fx ^= qa;
            }
            break;
        default: break;
        }
        if (status != QM_OK) break;
        if (D.slot >= 0 && lane < 8) row[8 * (uint64_t)D.slot + lane] = co[lane];
        if (D.channel >= 0 && lane == 0 && a.branches)
            a.branches[(uint64_t)state * a.channels + D.channel] = (int8_t)branch;
    }
    if (lane == 0) {
        a.counters[state] = counter;
        a.status[state] = status;
        a.ambiguous[state] += amb;
        a.frame_x[state] = fx;
        a.frame_z[state] = fz;
    }
}

template <typename V>
__global__ void k_welford(const V* __restrict__ amps, int states, uint64_t stride, int64_t len,
                          const double* __restrict__ masses, const uint32_t* __restrict__ frame_x, int64_t first,
                          double* __restrict__ mean, double* __restrict__ m2) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < len; i += (int64_t)gridDim.x * blockDim.x) {
        double mu = mean[i], acc = m2[i];
        for (int b = 0; b < states; ++b) {
            const double p = prob(amps + (uint64_t)b * stride, (uint64_t)i ^ frame_x[b]) / masses[b];
            const double delta = p - mu;
            mu += delta / (double)(first + b + 1);
            acc += delta * (p - mu);
        }
        mean[i] = mu;
        m2[i] = acc;
    }
}

__global__ void k_welford_finish(double* m2, int64_t len, double divisor) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < len; i += (int64_t)gridDim.x * blockDim.x)
        m2[i] = sqrt(fmax(0.0, m2[i]) / divisor);
}

// Each pair (i, i ^ f) with i < i ^ f is swapped by the thread that owns i.
template <typename V>
__global__ void k_frame_flip(V* __restrict__ amps, int qubits, int states, const uint32_t* __restrict__ frame_x) {
    const uint64_t len = 1ull << qubits;
    const uint64_t total = len * (uint64_t)states;
    for (uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; g < total; g += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t b = g >> qubits, i = g & (len - 1);
        const uint64_t j = i ^ frame_x[b];
        if (j > i) {
            V* s = amps + b * len;
            const V t = s[i];
            s[i] = s[j];
            s[j] = t;
        }
    }
}

int grid_for(int64_t n, int threads) {
    const int64_t blocks = (n + threads - 1) / threads;
    return (int)(blocks < 148 * 16 ? (blocks < 1 ? 1 : blocks) : 148 * 16);
}

}  // namespace

int histogram_ctas(int qubits) {
    // 2^16 amplitudes per CTA: a function of the state size alone, so a trajectory's sums do
    // not depend on how many other trajectories share its batch
    return qubits > 16 ? 1 << (qubits - 16) : 1;
}

cudaError_t launch_group_histogram(const void* amps, int qubits, int precision, int states, uint32_t group_mask,
                                   double* partials, cudaStream_t st) {
    HistArgs h{};
    h.state_len = 1ull << qubits;
    h.ctas = histogram_ctas(qubits);
    h.per_warp = h.state_len / ((uint64_t)h.ctas * kHistWarps);
    if (h.per_warp < 32 || h.per_warp % 32) return cudaErrorInvalidValue;
    h.nbits = 0;
    for (int q = 0; q < qubits; ++q)
        if (group_mask & (1u << q)) {
            if (h.nbits == kGroupMaxBits) return cudaErrorInvalidValue;
            h.pos[h.nbits++] = (int8_t)q;
        }
    h.bins = 1 << h.nbits;
    h.glow = group_mask & 31u;
    const unsigned grid = (unsigned)((int64_t)states * h.ctas);
    if (precision == QM_FP32)
        k_group_hist<float2><<<grid, kHistThreads, 0, st>>>(static_cast<const float2*>(amps), h, partials);
    else
        k_group_hist<double2><<<grid, kHistThreads, 0, st>>>(static_cast<const double2*>(amps), h, partials);
    return cudaGetLastError();
}

cudaError_t launch_decide(const DecideArgs& a, int states, cudaStream_t st) {
    if (a.count == 0) return cudaSuccess;
    if (a.bins > kGroupMaxBins) return cudaErrorInvalidValue;
    const unsigned grid = (unsigned)((states + kDecideWarps - 1) / kDecideWarps);
    k_decide<<<grid, 32 * kDecideWarps, 0, st>>>(a, states);
    return cudaGetLastError();
}

cudaError_t launch_welford(const void* amps, int precision, int states, uint64_t state_stride, int64_t len,
                           const double* masses, const uint32_t* frame_x, int64_t first, double* mean, double* m2,
                           cudaStream_t st) {
    const int grid = grid_for(len, 256);
    if (precision == QM_FP32)
        k_welford<float2><<<grid, 256, 0, st>>>(static_cast<const float2*>(amps), states, state_stride, len, masses,
                                                frame_x, first, mean, m2);
    else
        k_welford<double2><<<grid, 256, 0, st>>>(static_cast<const double2*>(amps), states, state_stride, len, masses,
                                                 frame_x, first, mean, m2);
    return cudaGetLastError();
}

cudaError_t launch_welford_finish(double* m2, int64_t len, int64_t trajectories, cudaStream_t st) {
    k_welford_finish<<<grid_for(len, 256), 256, 0, st>>>(m2, len, (double)trajectories * (double)(trajectories - 1));
    return cudaGetLastError();
}

cudaError_t launch_frame_flip(void* amps, int qubits, int precision, int states, const uint32_t* frame_x,
                              cudaStream_t st) {
    const int grid = grid_for((int64_t)states << qubits, 256);
    if (precision == QM_FP32)
        k_frame_flip<float2><<<grid, 256, 0, st>>>(static_cast<float2*>(amps), qubits, states, frame_x);
    else
        k_frame_flip<double2><<<grid, 256, 0, st>>>(static_cast<double2*>(amps), qubits, states, frame_x);
    return cudaGetLastError();
}

}  // namespace qm
