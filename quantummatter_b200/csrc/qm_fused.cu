// qm_fused.cu -- the fused multi-gate pass kernel of libqmb200.so (sm_100a).
//
// One launch applies a whole planned run of gates (a "pass") in one read and one write
// of the state.  A CTA owns a block of 2^K amplitudes: the block's local index bits are
// the pass's block qubits (ascending; the lowest qubits are always among them, so global
// accesses come in contiguous 128-byte runs), the remaining qubits are fixed by the CTA
// index.  Each thread holds 2^R = 16 amplitudes in registers.  The planner splits the
// pass into stages; in a stage R local bits are register bits and every gate either
// targets a register bit (2x2 matrix, X, SWAP applied on registers) or is diagonal (any
// qubit, applied by index test).  Controls may sit on any qubit: inside the block they
// are a per-amplitude predicate, outside it they are uniform per CTA.  Between stages
// the block is exchanged through shared memory with an XOR swizzle on the 128-byte rows.
//
// The arithmetic per gate is the pair update of CudaStateVectorKernel.cs:63-75
// (a*x + b*y, c*x + d*y) in the state's precision with fused multiply-adds.
#include <cuda_runtime.h>

#include "qm_device.cuh"
#include "qm_internal.h"

namespace qm {

namespace {

constexpr int R = kRegBits;
constexpr int NR = 1 << R;

struct FusedLaunch {
    uint32_t outer_mask;  // qubits outside the block
    int32_t op_begin, op_count;
    int32_t q[kMaxBlockQubits];
};

// Shared-memory slot of local index j: the low row bits are XORed with a fold of the
// higher bits, so that the 8 (complex128) or 16 (complex64) lanes of one shared-memory
// phase land in distinct banks for the usual stage layouts.
template <typename T>
__device__ __forceinline__ uint32_t swz(uint32_t j) {
    if (sizeof(T) == 8) {
        uint32_t h = j >> 3;
        return j ^ ((h ^ (h >> 3) ^ (h >> 6) ^ (h >> 9)) & 7u);
    } else {
        uint32_t h = j >> 4;
        return j ^ ((h ^ (h >> 4) ^ (h >> 8)) & 15u);
    }
}

struct Layout {
    uint32_t base;     // local index of register 0
    uint32_t pm[R];    // local masks of the register bits
    __device__ __forceinline__ uint32_t local(int i) const {
        uint32_t j = base;
#pragma unroll
        for (int m = 0; m < R; ++m)
            if ((i >> m) & 1) j |= pm[m];
        return j;
    }
};

template <typename T, int M>
__device__ __forceinline__ void op_matrix(Cx<T> (&a)[NR], const FusedOp& op, const Layout& L, bool real) {
    const T ar = (T)op.coef[0], ai = (T)op.coef[1], br = (T)op.coef[2], bi = (T)op.coef[3];
    const T cr = (T)op.coef[4], ci = (T)op.coef[5], dr = (T)op.coef[6], di = (T)op.coef[7];
    const uint32_t cm = op.cmask_local;
#pragma unroll
    for (int i = 0; i < NR; ++i) {
        if ((i >> M) & 1) continue;
        const int k = i | (1 << M);
        if (cm != 0 && (L.local(i) & cm) != cm) continue;
        Cx<T> x = a[i], y = a[k];
        if (real) {
            a[i] = Cx<T>{ar * x.re + br * y.re, ar * x.im + br * y.im};
            a[k] = Cx<T>{cr * x.re + dr * y.re, cr * x.im + dr * y.im};
        } else {
            a[i] = cmac2<T>(ar, ai, x, br, bi, y);
            a[k] = cmac2<T>(cr, ci, x, dr, di, y);
        }
    }
}

template <typename T, int M>
__device__ __forceinline__ void op_exchange(Cx<T> (&a)[NR], const FusedOp& op, const Layout& L) {
    const uint32_t cm = op.cmask_local;
#pragma unroll
    for (int i = 0; i < NR; ++i) {
        if ((i >> M) & 1) continue;
        const int k = i | (1 << M);
        if (cm != 0 && (L.local(i) & cm) != cm) continue;
        Cx<T> x = a[i];
        a[i] = a[k];
        a[k] = x;
    }
}

// SWAP of register bits M1 and M2: exchanges the (M1=1, M2=0) and (M1=0, M2=1) members.
template <typename T, int M1, int M2>
__device__ __forceinline__ void op_swap(Cx<T> (&a)[NR], const FusedOp& op, const Layout& L) {
    const uint32_t cm = op.cmask_local;
#pragma unroll
    for (int i = 0; i < NR; ++i) {
        if (!((i >> M1) & 1) || ((i >> M2) & 1)) continue;
        const int k = i ^ (1 << M1) ^ (1 << M2);
        if (cm != 0 && (L.local(i) & cm) != cm) continue;
        Cx<T> x = a[i];
        a[i] = a[k];
        a[k] = x;
    }
}

template <typename T>
__device__ __forceinline__ void op_swap_any(Cx<T> (&a)[NR], const FusedOp& op, const Layout& L) {
#define QM_SWAP_CASE(m1, m2) \
    if (op.reg == m1 && op.reg2 == m2) { op_swap<T, m1, m2>(a, op, L); return; }
    QM_SWAP_CASE(0, 1) QM_SWAP_CASE(0, 2) QM_SWAP_CASE(0, 3) QM_SWAP_CASE(1, 0) QM_SWAP_CASE(1, 2)
    QM_SWAP_CASE(1, 3) QM_SWAP_CASE(2, 0) QM_SWAP_CASE(2, 1) QM_SWAP_CASE(2, 3) QM_SWAP_CASE(3, 0)
    QM_SWAP_CASE(3, 1) QM_SWAP_CASE(3, 2)
#undef QM_SWAP_CASE
}

template <typename T>
__device__ __forceinline__ void op_diag(Cx<T> (&a)[NR], const FusedOp& op, const Layout& L, uint32_t outer) {
    const T ar = (T)op.coef[0], ai = (T)op.coef[1], dr = (T)op.coef[6], di = (T)op.coef[7];
    const bool a_one = op.flags & 1, d_one = op.flags & 2;
    const uint32_t cm = op.cmask_local;
    const int lt = op.local;
    const bool outer_bit = (outer & op.target_outer) != 0;
#pragma unroll
    for (int i = 0; i < NR; ++i) {
        const uint32_t j = L.local(i);
        if (cm != 0 && (j & cm) != cm) continue;
        const bool bit = lt >= 0 ? ((j >> lt) & 1u) != 0 : outer_bit;
        if (bit) {
            if (!d_one) a[i] = cmul<T>(dr, di, a[i]);
        } else if (!a_one) {
            a[i] = cmul<T>(ar, ai, a[i]);
        }
    }
}

template <typename T>
__device__ __forceinline__ void op_negate(Cx<T> (&a)[NR], const FusedOp& op, const Layout& L) {
    const uint32_t cm = op.cmask_local;
#pragma unroll
    for (int i = 0; i < NR; ++i) {
        if ((L.local(i) & cm) != cm) continue;
        a[i].re = -a[i].re;
        a[i].im = -a[i].im;
    }
}

template <typename T, int K>
__global__ void __launch_bounds__(1 << (K - R), (sizeof(T) == 8 && K == 12) ? 2 : 1)
    k_fused(typename Vec2<T>::type* __restrict__ s, const FusedLaunch P, const FusedOp* __restrict__ ops) {
    using V = typename Vec2<T>::type;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V* tile = reinterpret_cast<V*>(smem_raw);
    const uint32_t t = threadIdx.x;
    const uint32_t outer = deposit(blockIdx.x, P.outer_mask);

    // Canonical layout: the register bits are the top R local bits, so consecutive
    // threads read consecutive block-local indices (contiguous global runs).
    uint32_t gthread = outer;
#pragma unroll
    for (int b = 0; b < K - R; ++b)
        if ((t >> b) & 1u) gthread |= 1u << P.q[b];
    uint32_t greg[R];
#pragma unroll
    for (int m = 0; m < R; ++m) greg[m] = 1u << P.q[K - R + m];

    Cx<T> a[NR];
#pragma unroll
    for (int i = 0; i < NR; ++i) {
        uint32_t g = gthread;
#pragma unroll
        for (int m = 0; m < R; ++m)
            if ((i >> m) & 1) g |= greg[m];
        a[i] = load_amp<T>(s, g);
    }

    Layout L;
    L.base = t;
#pragma unroll
    for (int m = 0; m < R; ++m) L.pm[m] = 1u << (K - R + m);

    const int end = P.op_begin + P.op_count;
    for (int o = P.op_begin; o < end; ++o) {
        const FusedOp& op = ops[o];
        const int code = op.code;
        if (code == OP_STAGE) {
            __syncthreads();
#pragma unroll
            for (int i = 0; i < NR; ++i) {
                V v;
                v.x = a[i].re;
                v.y = a[i].im;
                tile[swz<T>(L.local(i))] = v;
            }
            uint32_t regs = 0;
#pragma unroll
            for (int m = 0; m < R; ++m) {
                L.pm[m] = 1u << op.reg_pos[m];
                regs |= L.pm[m];
            }
            L.base = deposit(t, ((1u << K) - 1u) & ~regs);
            __syncthreads();
#pragma unroll
            for (int i = 0; i < NR; ++i) {
                V v = tile[swz<T>(L.local(i))];
                a[i] = Cx<T>{v.x, v.y};
            }
            continue;
        }
        if ((outer & op.cmask_outer) != op.cmask_outer) continue;
        switch (code) {
        case OP_MATRIX:
        case OP_MATRIX_REAL: {
            const bool real = code == OP_MATRIX_REAL;
            switch (op.reg) {
            case 0: op_matrix<T, 0>(a, op, L, real); break;
            case 1: op_matrix<T, 1>(a, op, L, real); break;
            case 2: op_matrix<T, 2>(a, op, L, real); break;
            default: op_matrix<T, 3>(a, op, L, real); break;
            }
            break;
        }
        case OP_EXCHANGE:
            switch (op.reg) {
            case 0: op_exchange<T, 0>(a, op, L); break;
            case 1: op_exchange<T, 1>(a, op, L); break;
            case 2: op_exchange<T, 2>(a, op, L); break;
            default: op_exchange<T, 3>(a, op, L); break;
            }
            break;
        case OP_DIAG: op_diag<T>(a, op, L, outer); break;
        case OP_NEGATE: op_negate<T>(a, op, L); break;
        case OP_SWAP: op_swap_any<T>(a, op, L); break;
        default: break;
        }
    }

    // The planner ends every pass in the canonical layout.
#pragma unroll
    for (int i = 0; i < NR; ++i) {
        uint32_t g = gthread;
#pragma unroll
        for (int m = 0; m < R; ++m)
            if ((i >> m) & 1) g |= greg[m];
        store_amp<T>(s, g, a[i]);
    }
}

template <typename T, int K>
cudaError_t launch_k(void* amps, int qubits, const FusedLaunch& L, const FusedOp* d_ops, cudaStream_t st) {
    using V = typename Vec2<T>::type;
    const size_t smem = sizeof(V) << K;
    static bool configured = false;
    if (!configured) {
        cudaError_t e = cudaFuncSetAttribute(k_fused<T, K>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        configured = true;
    }
    dim3 grid(1u << (qubits - K));
    k_fused<T, K><<<grid, 1 << (K - R), smem, st>>>(reinterpret_cast<V*>(amps), L, d_ops);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_fused(void* amps, int qubits, int precision, const FusedPass& p, const FusedOp* d_ops,
                         cudaStream_t st) {
    FusedLaunch L;
    uint32_t all = qubits >= 32 ? 0xffffffffu : ((1u << qubits) - 1u);
    L.outer_mask = all & ~p.block_mask;
    L.op_begin = p.op_begin;
    L.op_count = p.op_count;
    for (int i = 0; i < kMaxBlockQubits; ++i) L.q[i] = i < p.k ? p.q[i] : 0;
    if (p.k > qubits) return cudaErrorInvalidValue;
    if (precision == QM_FP32) {
        switch (p.k) {
        case 9: return launch_k<float, 9>(amps, qubits, L, d_ops, st);
        case 10: return launch_k<float, 10>(amps, qubits, L, d_ops, st);
        case 11: return launch_k<float, 11>(amps, qubits, L, d_ops, st);
        case 12: return launch_k<float, 12>(amps, qubits, L, d_ops, st);
        case 13: return launch_k<float, 13>(amps, qubits, L, d_ops, st);
        default: return cudaErrorInvalidValue;
        }
    }
    switch (p.k) {
    case 9: return launch_k<double, 9>(amps, qubits, L, d_ops, st);
    case 10: return launch_k<double, 10>(amps, qubits, L, d_ops, st);
    case 11: return launch_k<double, 11>(amps, qubits, L, d_ops, st);
    case 12: return launch_k<double, 12>(amps, qubits, L, d_ops, st);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace qm
