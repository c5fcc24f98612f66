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
// The load and store use the first and last stage layouts directly whenever those keep
// the lowest qubits on thread bits (coalesced), so most passes have no extra exchange.
//
// The op program is a __grid_constant__ kernel parameter: every op field is a uniform
// load from the constant bank, so interpreting the program costs no memory traffic.
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

template <int MAXOPS>
struct FusedLaunch {
    uint32_t outer_mask;        // qubits outside the block
    uint32_t thread_in;         // global mask of the block qubits that are thread bits at load
    uint32_t thread_out;        // ... at store
    int32_t op_count;
    uint32_t reg_in_g[R];       // global bit of each register bit at load
    uint32_t reg_out_g[R];      // ... at store
    int32_t reg_in_l[R];        // local positions of the load layout
    int32_t pad[R];
    // Batches: state b = blockIdx.y lives at s + b * state_stride; ops flagged kOpTable take
    // their coefficients from table + b * table_stride + 8 * op.reserved.
    const double* table;
    uint64_t state_stride;
    uint64_t table_stride;
    FusedOp ops[MAXOPS];
};

struct Coef {
    double v[8];
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

template <typename T, int M, bool REAL, bool CTRL>
__device__ __forceinline__ void op_matrix(Cx<T> (&a)[NR], const FusedOp& op, const Coef& c, const Layout& L) {
    const T ar = (T)c.v[0], br = (T)c.v[2], cr = (T)c.v[4], dr = (T)c.v[6];
    const T ai = REAL ? (T)0 : (T)c.v[1], bi = REAL ? (T)0 : (T)c.v[3];
    const T ci = REAL ? (T)0 : (T)c.v[5], di = REAL ? (T)0 : (T)c.v[7];
    const uint32_t cm = op.cmask_local;
#pragma unroll
    for (int i = 0; i < NR; ++i) {
        if ((i >> M) & 1) continue;
        const int k = i | (1 << M);
        if (CTRL && (L.local(i) & cm) != cm) continue;
        Cx<T> x = a[i], y = a[k];
        if (REAL) {
            a[i] = Cx<T>{ar * x.re + br * y.re, ar * x.im + br * y.im};
            a[k] = Cx<T>{cr * x.re + dr * y.re, cr * x.im + dr * y.im};
        } else {
            a[i] = cmac2<T>(ar, ai, x, br, bi, y);
            a[k] = cmac2<T>(cr, ci, x, dr, di, y);
        }
    }
}

template <typename T, bool REAL, bool CTRL>
__device__ __forceinline__ void op_matrix_any(Cx<T> (&a)[NR], const FusedOp& op, const Coef& c, const Layout& L) {
    switch (op.reg) {
    case 0: op_matrix<T, 0, REAL, CTRL>(a, op, c, L); break;
    case 1: op_matrix<T, 1, REAL, CTRL>(a, op, c, L); break;
#if QM_REG_BITS > 3
    case 2: op_matrix<T, 2, REAL, CTRL>(a, op, c, L); break;
    default: op_matrix<T, 3, REAL, CTRL>(a, op, c, L); break;
#else
    default: op_matrix<T, 2, REAL, CTRL>(a, op, c, L); break;
#endif
    }
}

// X on register bit M where the control lies outside the registers (or there is none):
// a per-amplitude predicate.
template <typename T, int M>
__device__ __forceinline__ void op_exchange(Cx<T> (&a)[NR], const FusedOp& op, const Layout& L) {
    const uint32_t cm = op.cmask_local;
#pragma unroll
    for (int i = 0; i < NR; ++i) {
        if ((i >> M) & 1) continue;
        const int k = i | (1 << M);
        const bool on = (L.local(i) & cm) == cm;
        Cx<T> x = a[i], y = a[k];
        a[i] = on ? y : x;
        a[k] = on ? x : y;
    }
}

// X on register bit M controlled by register bit MC: the swapped pairs are known at compile
// time, so the op is a fixed register permutation (plus a predicate for any other control).
template <typename T, int M, int MC>
__device__ __forceinline__ void op_exchange_rc(Cx<T> (&a)[NR], const FusedOp& op, const Layout& L) {
    const uint32_t cm = op.cmask_local & ~L.pm[MC];
#pragma unroll
    for (int i = 0; i < NR; ++i) {
        if (((i >> M) & 1) || !((i >> MC) & 1)) continue;
        const int k = i | (1 << M);
        Cx<T> x = a[i], y = a[k];
        if (cm == 0) {
            a[i] = y;
            a[k] = x;
        } else {
            const bool on = (L.local(i) & cm) == cm;
            a[i] = on ? y : x;
            a[k] = on ? x : y;
        }
    }
}

template <typename T>
__device__ __forceinline__ void op_exchange_any(Cx<T> (&a)[NR], const FusedOp& op, const Layout& L) {
    if (op.reg2 < 0) {
        switch (op.reg) {
        case 0: op_exchange<T, 0>(a, op, L); break;
        case 1: op_exchange<T, 1>(a, op, L); break;
#if QM_REG_BITS > 3
        case 2: op_exchange<T, 2>(a, op, L); break;
        default: op_exchange<T, 3>(a, op, L); break;
#else
        default: op_exchange<T, 2>(a, op, L); break;
#endif
        }
        return;
    }
#define QM_XC_CASE(m, mc) \
    if (op.reg == m && op.reg2 == mc) { op_exchange_rc<T, m, mc>(a, op, L); return; }
    QM_XC_CASE(0, 1) QM_XC_CASE(0, 2) QM_XC_CASE(1, 0) QM_XC_CASE(1, 2) QM_XC_CASE(2, 0) QM_XC_CASE(2, 1)
#if QM_REG_BITS > 3
    QM_XC_CASE(0, 3) QM_XC_CASE(1, 3) QM_XC_CASE(2, 3) QM_XC_CASE(3, 0) QM_XC_CASE(3, 1) QM_XC_CASE(3, 2)
#endif
#undef QM_XC_CASE
}

// SWAP of register bits M1 and M2: exchanges the (M1=1, M2=0) and (M1=0, M2=1) members.
template <typename T, int M1, int M2>
__device__ __forceinline__ void op_swap(Cx<T> (&a)[NR], const FusedOp& op, const Layout& L) {
    const uint32_t cm = op.cmask_local;
#pragma unroll
    for (int i = 0; i < NR; ++i) {
        if (!((i >> M1) & 1) || ((i >> M2) & 1)) continue;
        const int k = i ^ (1 << M1) ^ (1 << M2);
        const bool on = (L.local(i) & cm) == cm;
        Cx<T> x = a[i], y = a[k];
        a[i] = on ? y : x;
        a[k] = on ? x : y;
    }
}

template <typename T>
__device__ __forceinline__ void op_swap_any(Cx<T> (&a)[NR], const FusedOp& op, const Layout& L) {
    const int lo = op.reg < op.reg2 ? op.reg : op.reg2, hi = op.reg < op.reg2 ? op.reg2 : op.reg;
#define QM_SWAP_CASE(m1, m2) \
    if (lo == m1 && hi == m2) { op_swap<T, m2, m1>(a, op, L); return; }
    QM_SWAP_CASE(0, 1) QM_SWAP_CASE(0, 2) QM_SWAP_CASE(1, 2)
#if QM_REG_BITS > 3
    QM_SWAP_CASE(0, 3) QM_SWAP_CASE(1, 3) QM_SWAP_CASE(2, 3)
#endif
#undef QM_SWAP_CASE
}

// Shared-memory slots of the 2^R registers.  swz() is linear over GF(2) and the base and
// register bits are disjoint, so slot(base | bits) = swz(base) ^ XOR of swz(register bits):
// one XOR per register instead of a full swizzle per amplitude.
template <typename T>
__device__ __forceinline__ void slots(const Layout& L, uint32_t (&s)[NR]) {
    uint32_t sp[R];
#pragma unroll
    for (int m = 0; m < R; ++m) sp[m] = swz<T>(L.pm[m]);
    s[0] = swz<T>(L.base);
#pragma unroll
    for (int i = 1; i < NR; ++i) {
        const int low = (i & 1) ? 0 : (i & 2) ? 1 : (i & 4) ? 2 : 3;
        s[i] = s[i & (i - 1)] ^ sp[low];
    }
}

template <typename T>
__device__ __forceinline__ void op_diag(Cx<T> (&a)[NR], const FusedOp& op, const Coef& c, const Layout& L,
                                        uint32_t outer) {
    const T ar = (T)c.v[0], ai = (T)c.v[1], dr = (T)c.v[6], di = (T)c.v[7];
    const bool a_one = op.flags & 1, d_one = op.flags & 2;
    const uint32_t cm = op.cmask_local;
    const int lt = op.local;
    if (lt < 0) {
        // target outside the block: one phase for the whole CTA
        const bool bit = (outer & op.target_outer) != 0;
        if (bit ? d_one : a_one) return;
        const T pr = bit ? dr : ar, pi = bit ? di : ai;
#pragma unroll
        for (int i = 0; i < NR; ++i) {
            if (cm != 0 && (L.local(i) & cm) != cm) continue;
            a[i] = cmul<T>(pr, pi, a[i]);
        }
        return;
    }
#pragma unroll
    for (int i = 0; i < NR; ++i) {
        const uint32_t j = L.local(i);
        if (cm != 0 && (j & cm) != cm) continue;
        const bool bit = ((j >> lt) & 1u) != 0;
        if (bit ? d_one : a_one) continue;
        a[i] = cmul<T>(bit ? dr : ar, bit ? di : ai, a[i]);
    }
}

template <typename T>
__device__ __forceinline__ void op_negate(Cx<T> (&a)[NR], const FusedOp& op, const Layout& L) {
    const uint32_t cm = op.cmask_local;
#pragma unroll
    for (int i = 0; i < NR; ++i) {
        const bool on = (L.local(i) & cm) == cm;
        a[i].re = on ? -a[i].re : a[i].re;
        a[i].im = on ? -a[i].im : a[i].im;
    }
}

template <typename T, int K, int MAXOPS>
__global__ void __launch_bounds__(1 << (K - R), ((sizeof(T) == 8 && K == 12) || (sizeof(T) == 4 && K == 13)) ? 2 : 1)
    // two CTAs per SM at the default widths: one exchanging with HBM while the other computes
    k_fused(typename Vec2<T>::type* __restrict__ s, const __grid_constant__ FusedLaunch<MAXOPS> P) {
    using V = typename Vec2<T>::type;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V* tile = reinterpret_cast<V*>(smem_raw);
    const uint32_t t = threadIdx.x;
    const uint32_t outer = deposit(blockIdx.x, P.outer_mask);
    s += (size_t)blockIdx.y * P.state_stride;
    const double* table = P.table ? P.table + (size_t)blockIdx.y * P.table_stride : nullptr;

    Cx<T> a[NR];
    {
        const uint32_t g0 = outer | deposit(t, P.thread_in);
#pragma unroll
        for (int i = 0; i < NR; ++i) {
            uint32_t g = g0;
#pragma unroll
            for (int m = 0; m < R; ++m)
                if ((i >> m) & 1) g |= P.reg_in_g[m];
            a[i] = load_amp<T>(s, g);
        }
    }

    Layout L;
    {
        uint32_t regs = 0;
#pragma unroll
        for (int m = 0; m < R; ++m) {
            L.pm[m] = 1u << P.reg_in_l[m];
            regs |= L.pm[m];
        }
        L.base = deposit(t, ((1u << K) - 1u) & ~regs);
    }

    for (int o = 0; o < P.op_count; ++o) {
        const FusedOp& op = P.ops[o];
        const int code = op.code;
        if (code == OP_STAGE) {
            uint32_t sl[NR];
            slots<T>(L, sl);
            __syncthreads();
#pragma unroll
            for (int i = 0; i < NR; ++i) {
                V v;
                v.x = a[i].re;
                v.y = a[i].im;
                tile[sl[i]] = v;
            }
            uint32_t regs = 0;
#pragma unroll
            for (int m = 0; m < R; ++m) {
                L.pm[m] = 1u << op.reg_pos[m];
                regs |= L.pm[m];
            }
            L.base = deposit(t, ((1u << K) - 1u) & ~regs);
            slots<T>(L, sl);
            __syncthreads();
#pragma unroll
            for (int i = 0; i < NR; ++i) {
                V v = tile[sl[i]];
                a[i] = Cx<T>{v.x, v.y};
            }
            continue;
        }
        if ((outer & op.cmask_outer) != op.cmask_outer) continue;
        const bool ctrl = op.cmask_local != 0;
        Coef c;
        if (code == OP_MATRIX || code == OP_MATRIX_REAL || code == OP_DIAG) {
            if (op.flags & kOpTable) {
                const double* src = table + 8 * (size_t)op.reserved;
#pragma unroll
                for (int k = 0; k < 8; ++k) c.v[k] = __ldg(src + k);
            } else {
#pragma unroll
                for (int k = 0; k < 8; ++k) c.v[k] = op.coef[k];
            }
        }
        switch (code) {
        case OP_MATRIX:
            if (ctrl) op_matrix_any<T, false, true>(a, op, c, L);
            else op_matrix_any<T, false, false>(a, op, c, L);
            break;
        case OP_MATRIX_REAL:
            if (ctrl) op_matrix_any<T, true, true>(a, op, c, L);
            else op_matrix_any<T, true, false>(a, op, c, L);
            break;
        case OP_EXCHANGE: op_exchange_any<T>(a, op, L); break;
        case OP_DIAG: op_diag<T>(a, op, c, L, outer); break;
        case OP_NEGATE: op_negate<T>(a, op, L); break;
        case OP_SWAP: op_swap_any<T>(a, op, L); break;
        default: break;
        }
    }

    // the planner ends every pass in the store layout
    const uint32_t g0 = outer | deposit(t, P.thread_out);
#pragma unroll
    for (int i = 0; i < NR; ++i) {
        uint32_t g = g0;
#pragma unroll
        for (int m = 0; m < R; ++m)
            if ((i >> m) & 1) g |= P.reg_out_g[m];
        store_amp<T>(s, g, a[i]);
    }
}

template <typename T, int K, int MAXOPS>
cudaError_t launch_k(void* amps, int qubits, const FusedPass& p, const FusedOp* ops, const FusedBatch* batch,
                     cudaStream_t st) {
    using V = typename Vec2<T>::type;
    FusedLaunch<MAXOPS> L;
    const uint32_t all = (1u << qubits) - 1u;
    L.outer_mask = all & ~p.block_mask;
    uint32_t reg_in_local = 0, reg_out_local = 0;
    for (int m = 0; m < R; ++m) {
        L.reg_in_l[m] = p.reg_in[m];
        L.pad[m] = 0;
        L.reg_in_g[m] = 1u << p.q[p.reg_in[m]];
        L.reg_out_g[m] = 1u << p.q[p.reg_out[m]];
        reg_in_local |= 1u << p.reg_in[m];
        reg_out_local |= 1u << p.reg_out[m];
    }
    L.thread_in = 0;
    L.thread_out = 0;
    for (int b = 0; b < K; ++b) {
        if (!(reg_in_local & (1u << b))) L.thread_in |= 1u << p.q[b];
        if (!(reg_out_local & (1u << b))) L.thread_out |= 1u << p.q[b];
    }
    L.op_count = p.op_count;
    for (int i = 0; i < p.op_count; ++i) L.ops[i] = ops[p.op_begin + i];
    L.table = batch ? batch->table : nullptr;
    L.state_stride = batch ? batch->state_stride : 0;
    L.table_stride = batch ? batch->table_stride : 0;
    const unsigned states = batch ? (unsigned)batch->states : 1u;
    const size_t smem = sizeof(V) << K;
    static bool configured = false;
    if (!configured) {
        cudaError_t e =
            cudaFuncSetAttribute(k_fused<T, K, MAXOPS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        configured = true;
    }
    dim3 grid(1u << (qubits - K), states);
    k_fused<T, K, MAXOPS><<<grid, 1 << (K - R), smem, st>>>(reinterpret_cast<V*>(amps), L);
    return cudaGetLastError();
}

template <typename T, int K>
cudaError_t launch_sized(void* amps, int qubits, const FusedPass& p, const FusedOp* ops, const FusedBatch* batch,
                         cudaStream_t st) {
    if (p.op_count <= kSmallPassOps) return launch_k<T, K, kSmallPassOps>(amps, qubits, p, ops, batch, st);
    return launch_k<T, K, kMaxPassOps>(amps, qubits, p, ops, batch, st);
}

}  // namespace

cudaError_t launch_fused(void* amps, int qubits, int precision, const FusedPass& p, const FusedOp* ops,
                         const FusedBatch* batch, cudaStream_t st) {
    if (p.k > qubits || p.op_count > kMaxPassOps || p.op_count < 0) return cudaErrorInvalidValue;
    if (batch && (batch->states < 1 || batch->states > 65535)) return cudaErrorInvalidValue;
    if (precision == QM_FP32) {
        switch (p.k) {
        case 9: return launch_sized<float, 9>(amps, qubits, p, ops, batch, st);
        case 10: return launch_sized<float, 10>(amps, qubits, p, ops, batch, st);
        case 11: return launch_sized<float, 11>(amps, qubits, p, ops, batch, st);
        case 12: return launch_sized<float, 12>(amps, qubits, p, ops, batch, st);
        case 13: return launch_sized<float, 13>(amps, qubits, p, ops, batch, st);
        default: return cudaErrorInvalidValue;
        }
    }
    switch (p.k) {
    case 9: return launch_sized<double, 9>(amps, qubits, p, ops, batch, st);
    case 10: return launch_sized<double, 10>(amps, qubits, p, ops, batch, st);
    case 11: return launch_sized<double, 11>(amps, qubits, p, ops, batch, st);
    case 12: return launch_sized<double, 12>(amps, qubits, p, ops, batch, st);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace qm
