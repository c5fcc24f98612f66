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
// The kernel is persistent (grid = resident CTAs): each CTA stages the pass program into
// shared memory once and then loops over (state, block) work items, so interpreting the
// program costs uniform shared-memory loads only, and a batch state's coefficient row is
// staged once per state change.
//
// The arithmetic per gate is the pair update of CudaStateVectorKernel.cs:63-75
// (a*x + b*y, c*x + d*y) in the state's precision with fused multiply-adds.
#include <cuda_runtime.h>

#include <algorithm>

#include "qm_device.cuh"
#include "qm_internal.h"

namespace qm {

namespace {

constexpr int R = kRegBits;
constexpr int NR = 1 << R;

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

// Local index of thread t in a stage layout with lanes (OP_STAGE `reserved`): thread ranks 0..n-1
// on the lanes, the others on the remaining non-register local bits in ascending order.
__device__ __forceinline__ uint32_t lane_base(uint32_t t, uint32_t regs, uint32_t code, int K) {
    const int n = (int)(code & 15u);
    uint32_t base = 0, used = regs;
    for (int r = 0; r < n; ++r) {
        const uint32_t b = (code >> (4 + 4 * r)) & 15u;
        base |= ((t >> r) & 1u) << b;
        used |= 1u << b;
    }
    return base | deposit(t >> n, ((1u << K) - 1u) & ~used);
}

// Registers whose index has bit m set, as a 2^R-bit pattern.
__host__ __device__ constexpr uint32_t reg_half(int m) {
    uint32_t p = 0;
    for (int i = 0; i < NR; ++i)
        if ((i >> m) & 1) p |= 1u << i;
    return p;
}

// Bit i is set when register i has every local bit of cm set: the thread bits of cm must all
// be set in this thread's base index, and each register bit of cm keeps half the registers.
__device__ __forceinline__ uint32_t control_pattern(const Layout& L, uint32_t cm) {
    uint32_t regs = 0, pat = (NR == 32) ? 0xffffffffu : ((1u << NR) - 1u);
#pragma unroll
    for (int m = 0; m < R; ++m)
        if (cm & L.pm[m]) {
            regs |= L.pm[m];
            pat &= reg_half(m);
        }
    const uint32_t thread_bits = cm & ~regs;
    return (L.base & thread_bits) == thread_bits ? pat : 0u;
}

template <typename T, int M, bool REAL, bool CTRL>
__device__ __forceinline__ void op_matrix(Cx<T> (&a)[NR], const FusedOp& op, const Coef& c, const Layout& L) {
    const T ar = (T)c.v[0], br = (T)c.v[2], cr = (T)c.v[4], dr = (T)c.v[6];
    const T ai = REAL ? (T)0 : (T)c.v[1], bi = REAL ? (T)0 : (T)c.v[3];
    const T ci = REAL ? (T)0 : (T)c.v[5], di = REAL ? (T)0 : (T)c.v[7];
    const uint32_t pat = CTRL ? control_pattern(L, op.cmask_local) : 0u;
#pragma unroll
    for (int i = 0; i < NR; ++i) {
        if ((i >> M) & 1) continue;
        const int k = i | (1 << M);
        if (CTRL && !((pat >> i) & 1u)) continue;
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

template <typename T, int M>
__device__ __forceinline__ void op_scale(Cx<T> (&a)[NR], T s0, T s1) {
#pragma unroll
    for (int i = 0; i < NR; ++i) {
        const T s = ((i >> M) & 1) ? s1 : s0;
        a[i].re *= s;
        a[i].im *= s;
    }
}

// A noise-branch op (kOpBranch, uncontrolled, target in register bit op.reg).  Its per-state
// coefficients are mostly the identity (no Pauli error) or a real diagonal (a damping without
// a jump, a Z error); the test is uniform across the CTA, which works on one state.
template <typename T>
__device__ __forceinline__ void op_branch(Cx<T> (&a)[NR], const FusedOp& op, const Coef& c, const Layout& L) {
    const bool real = c.v[1] == 0 && c.v[3] == 0 && c.v[5] == 0 && c.v[7] == 0;
    if (!real) {
        op_matrix_any<T, false, false>(a, op, c, L);
        return;
    }
    if (c.v[2] != 0 || c.v[4] != 0) {
        op_matrix_any<T, true, false>(a, op, c, L);
        return;
    }
    if (c.v[0] == 1 && c.v[6] == 1) return;
    const T s0 = (T)c.v[0], s1 = (T)c.v[6];
    switch (op.reg) {
    case 0: op_scale<T, 0>(a, s0, s1); break;
    case 1: op_scale<T, 1>(a, s0, s1); break;
#if QM_REG_BITS > 3
    case 2: op_scale<T, 2>(a, s0, s1); break;
    default: op_scale<T, 3>(a, s0, s1); break;
#else
    default: op_scale<T, 2>(a, s0, s1); break;
#endif
    }
}

// X on register bit M where the control lies outside the registers (or there is none):
// a per-amplitude predicate.
template <typename T, int M>
__device__ __forceinline__ void op_exchange(Cx<T> (&a)[NR], const FusedOp& op, const Layout& L) {
    const uint32_t pat = control_pattern(L, op.cmask_local);
#pragma unroll
    for (int i = 0; i < NR; ++i) {
        if ((i >> M) & 1) continue;
        const int k = i | (1 << M);
        const bool on = (pat >> i) & 1u;
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
    const uint32_t pat = cm ? control_pattern(L, cm) : 0u;
#pragma unroll
    for (int i = 0; i < NR; ++i) {
        if (((i >> M) & 1) || !((i >> MC) & 1)) continue;
        const int k = i | (1 << M);
        Cx<T> x = a[i], y = a[k];
        if (cm == 0) {
            a[i] = y;
            a[k] = x;
        } else {
            const bool on = (pat >> i) & 1u;
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
    const uint32_t pat = control_pattern(L, op.cmask_local);
#pragma unroll
    for (int i = 0; i < NR; ++i) {
        if (!((i >> M1) & 1) || ((i >> M2) & 1)) continue;
        const int k = i ^ (1 << M1) ^ (1 << M2);
        const bool on = (pat >> i) & 1u;
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

// Diagonal whose target bit is a register bit M: the phase of each register is known at
// compile time.
template <typename T, int M>
__device__ __forceinline__ void op_diag_reg(Cx<T> (&a)[NR], const FusedOp& op, const Coef& c, const Layout& L) {
    const T ar = (T)c.v[0], ai = (T)c.v[1], dr = (T)c.v[6], di = (T)c.v[7];
    const bool a_one = op.flags & 1, d_one = op.flags & 2;
    const uint32_t pat = control_pattern(L, op.cmask_local);
#pragma unroll
    for (int i = 0; i < NR; ++i) {
        if (!((pat >> i) & 1u)) continue;
        if ((i >> M) & 1) {
            if (!d_one) a[i] = cmul<T>(dr, di, a[i]);
        } else if (!a_one) {
            a[i] = cmul<T>(ar, ai, a[i]);
        }
    }
}

template <typename T>
__device__ __forceinline__ void op_diag(Cx<T> (&a)[NR], const FusedOp& op, const Coef& c, const Layout& L,
                                        uint32_t outer) {
    const T ar = (T)c.v[0], ai = (T)c.v[1], dr = (T)c.v[6], di = (T)c.v[7];
    const bool a_one = op.flags & 1, d_one = op.flags & 2;
    const uint32_t cm = op.cmask_local;
    const int lt = op.local;
    bool bit;
    if (lt < 0) {
        // target outside the block: one phase for the whole CTA
        bit = (outer & op.target_outer) != 0;
    } else {
#pragma unroll
        for (int m = 0; m < R; ++m) {
            if (L.pm[m] == (1u << lt)) {
                switch (m) {
                case 0: op_diag_reg<T, 0>(a, op, c, L); return;
                case 1: op_diag_reg<T, 1>(a, op, c, L); return;
#if QM_REG_BITS > 3
                case 2: op_diag_reg<T, 2>(a, op, c, L); return;
                default: op_diag_reg<T, 3>(a, op, c, L); return;
#else
                default: op_diag_reg<T, 2>(a, op, c, L); return;
#endif
                }
            }
        }
        // target on a thread bit: one phase for all of this thread's registers
        bit = ((L.base >> lt) & 1u) != 0;
    }
    if (bit ? d_one : a_one) return;
    const T pr = bit ? dr : ar, pi = bit ? di : ai;
    const uint32_t pat = control_pattern(L, cm);
#pragma unroll
    for (int i = 0; i < NR; ++i) {
        if (!((pat >> i) & 1u)) continue;
        a[i] = cmul<T>(pr, pi, a[i]);
    }
}

template <typename T>
__device__ __forceinline__ void op_negate(Cx<T> (&a)[NR], const FusedOp& op, const Layout& L) {
    const uint32_t pat = control_pattern(L, op.cmask_local);
#pragma unroll
    for (int i = 0; i < NR; ++i) {
        const bool on = (pat >> i) & 1u;
        a[i].re = on ? -a[i].re : a[i].re;
        a[i].im = on ? -a[i].im : a[i].im;
    }
}

template <typename T>
__device__ __forceinline__ Cx<T> cmulc(Cx<T> x, Cx<T> y) {
    return Cx<T>{x.re * y.re - x.im * y.im, x.re * y.im + x.im * y.re};
}

// A group of commuting diagonals applied as one phase per register.  Every member's factor
// splits by where its qubits sit: outside the block or on a thread bit it is one value for
// the whole thread (folded into u); on a register bit m it is a pair (zero-phase, one-phase)
// multiplied into (az[m], on[m]); a negate on register bits flips the sign of the registers
// whose index has those bits (a 16-bit pattern).  Then phase[i] = u * prod_m (i_m ? on : az)
// is built as a product tree and applied once.
template <typename T>
__device__ __forceinline__ void op_diag_group(Cx<T> (&a)[NR], const FusedOp* members, int count, const double* table,
                                              const Layout& L, uint32_t outer) {
    Cx<T> u{(T)1, (T)0};
    Cx<T> az[R], on[R];
#pragma unroll
    for (int m = 0; m < R; ++m) {
        az[m] = Cx<T>{(T)1, (T)0};
        on[m] = Cx<T>{(T)1, (T)0};
    }
    uint32_t negate = 0;  // bit i: register i changes sign
    bool phased = false;  // some member is more than a sign
    uint32_t regmask = 0;
#pragma unroll
    for (int m = 0; m < R; ++m) regmask |= L.pm[m];
    for (int k = 0; k < count; ++k) {
        const FusedOp& op = members[k];
        if ((outer & op.cmask_outer) != op.cmask_outer) continue;
        if (op.code == OP_NEGATE) {
            negate ^= control_pattern(L, op.cmask_local);
            continue;
        }
        phased = true;
        // uncontrolled single-qubit diagonal
        const double* src = (op.flags & kOpTable) ? table + 8 * (size_t)op.reserved : op.coef;
        const Cx<T> pa{(T)src[0], (T)src[1]}, pd{(T)src[6], (T)src[7]};
        const int lt = op.local;
        if (lt >= 0 && (regmask & (1u << lt))) {
#pragma unroll
            for (int m = 0; m < R; ++m)
                if (L.pm[m] == (1u << lt)) {
                    az[m] = cmulc<T>(az[m], pa);
                    on[m] = cmulc<T>(on[m], pd);
                }
            continue;
        }
        const bool bit = lt < 0 ? (outer & op.target_outer) != 0 : ((L.base >> lt) & 1u) != 0;
        u = cmulc<T>(u, bit ? pd : pa);
    }
    if (!phased) {  // only CZ / Z members: signs
#pragma unroll
        for (int i = 0; i < NR; ++i) {
            const bool neg = (negate >> i) & 1u;
            a[i].re = neg ? -a[i].re : a[i].re;
            a[i].im = neg ? -a[i].im : a[i].im;
        }
        return;
    }
    // phase[i] = lo[i & low] * hi[i >> LB]: two small product tables instead of a full tree,
    // to keep the live registers low
    constexpr int LB = R / 2, HB = R - LB;
    Cx<T> lo[1 << LB], hi[1 << HB];
    lo[0] = Cx<T>{(T)1, (T)0};
    hi[0] = u;
#pragma unroll
    for (int m = 0; m < LB; ++m)
#pragma unroll
        for (int i = (1 << m) - 1; i >= 0; --i) {
            lo[i | (1 << m)] = cmulc<T>(lo[i], on[m]);
            lo[i] = cmulc<T>(lo[i], az[m]);
        }
#pragma unroll
    for (int m = 0; m < HB; ++m)
#pragma unroll
        for (int i = (1 << m) - 1; i >= 0; --i) {
            hi[i | (1 << m)] = cmulc<T>(hi[i], on[LB + m]);
            hi[i] = cmulc<T>(hi[i], az[LB + m]);
        }
#pragma unroll
    for (int i = 0; i < NR; ++i) {
        const Cx<T> p = cmulc<T>(lo[i & ((1 << LB) - 1)], hi[i >> LB]);
        Cx<T> v = cmulc<T>(p, a[i]);
        const bool neg = (negate >> i) & 1u;
        a[i].re = neg ? -v.re : v.re;
        a[i].im = neg ? -v.im : v.im;
    }
}


// Shared memory: [block of 2^K amplitudes][pass program][coefficient row of the current state]
template <typename T, int K>
__host__ __device__ constexpr size_t tile_bytes() {
    return sizeof(typename Vec2<T>::type) << K;
}
__host__ __device__ constexpr size_t program_bytes(int ops) { return ((size_t)ops * sizeof(FusedOp) + 15) & ~size_t(15); }

// Persistent: each CTA loops over (state, block) work items, so the pass program is staged
// into shared memory once per CTA and a state's coefficient row once per state change.
template <typename T, int K>
__global__ void __launch_bounds__(1 << (K - R), ((sizeof(T) == 8 && K == 12) || (sizeof(T) == 4 && K == 13)) ? 2 : 1)
    k_fused(typename Vec2<T>::type* __restrict__ s0, const __grid_constant__ FusedLaunch P) {
    using V = typename Vec2<T>::type;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V* tile = reinterpret_cast<V*>(smem_raw);
    FusedOp* prog = reinterpret_cast<FusedOp*>(smem_raw + tile_bytes<T, K>());
    double* table = reinterpret_cast<double*>(smem_raw + tile_bytes<T, K>() + program_bytes(P.op_count));
    const uint32_t t = threadIdx.x;
    {
        const uint2* src = reinterpret_cast<const uint2*>(P.ops);
        uint2* dst = reinterpret_cast<uint2*>(prog);
        const int words = P.op_count * (int)(sizeof(FusedOp) / sizeof(uint2));
        for (int i = t; i < words; i += blockDim.x) dst[i] = __ldg(src + i);
    }
    const int64_t total = (int64_t)P.states << P.cta_shift;
    const uint32_t cta_mask = (1u << P.cta_shift) - 1u;
    int current = -1;
    for (int64_t item = blockIdx.x; item < total; item += gridDim.x) {
        const int b = (int)(item >> P.cta_shift);
        const uint32_t cta = (uint32_t)item & cta_mask;
        __syncthreads();  // program staged / previous block's exchanges finished
        if (P.table_slots > 0 && b != current) {
            const double* row = P.table + (size_t)b * P.table_stride;
            for (int i = t; i < 8 * P.table_slots; i += blockDim.x) table[i] = __ldg(row + i);
            __syncthreads();
        }
        current = b;
        typename Vec2<T>::type* __restrict__ s = s0 + (size_t)b * P.state_stride;
        const uint32_t outer = deposit(cta, P.outer_mask);

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
            const FusedOp& op = prog[o];
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
                L.base = op.reserved ? lane_base(t, regs, op.reserved, K) : deposit(t, ((1u << K) - 1u) & ~regs);
                slots<T>(L, sl);
                __syncthreads();
#pragma unroll
                for (int i = 0; i < NR; ++i) {
                    V v = tile[sl[i]];
                    a[i] = Cx<T>{v.x, v.y};
                }
                continue;
            }
            if (code == OP_DIAG_GROUP) {
                const int count = (int)op.reserved;
                op_diag_group<T>(a, prog + o + 1, count, table, L, outer);
                o += count;
                continue;
            }
            if ((outer & op.cmask_outer) != op.cmask_outer) continue;
            const bool ctrl = op.cmask_local != 0;
            Coef c;
            if (code == OP_MATRIX || code == OP_MATRIX_REAL || code == OP_DIAG) {
                const double* src = (op.flags & kOpTable) ? table + 8 * (size_t)op.reserved : op.coef;
                // only the entries the op kind reads
                if (code == OP_MATRIX) {
#pragma unroll
                    for (int k = 0; k < 8; ++k) c.v[k] = src[k];
                } else if (code == OP_MATRIX_REAL) {
#pragma unroll
                    for (int k = 0; k < 8; k += 2) {
                        c.v[k] = src[k];
                        c.v[k + 1] = 0.0;
                    }
                } else {
                    c.v[0] = src[0];
                    c.v[1] = src[1];
                    c.v[6] = src[6];
                    c.v[7] = src[7];
                    c.v[2] = c.v[3] = c.v[4] = c.v[5] = 0.0;
                }
            }
            switch (code) {
            case OP_MATRIX:
                if (op.flags & kOpBranch) op_branch<T>(a, op, c, L);
                else if (ctrl) op_matrix_any<T, false, true>(a, op, c, L);
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

        // the planner ends every pass in the store layout; thread rank r writes index bit out_bit[r]
        uint32_t g0 = outer;
#pragma unroll
        for (int r = 0; r < K - R; ++r) g0 |= ((t >> r) & 1u) << P.out_bit[r];
#pragma unroll
        for (int i = 0; i < NR; ++i) {
            uint32_t g = g0;
#pragma unroll
            for (int m = 0; m < R; ++m)
                if ((i >> m) & 1) g |= P.reg_out_g[m];
            store_amp<T>(s, g, a[i]);
        }
    }
}

template <typename T, int K>
cudaError_t launch_k(void* amps, int qubits, const FusedPass& p, const FusedOp* d_ops, const FusedBatch* batch,
                     cudaStream_t st) {
    using V = typename Vec2<T>::type;
    const FusedLaunch L = fused_launch_params(qubits, p, d_ops, batch);
    const size_t smem = tile_bytes<T, K>() + program_bytes(p.op_count) + sizeof(double) * 8 * (size_t)L.table_slots;
    // device limits and the kernel's shared-memory opt-in, set once per process (thread-safe:
    // several host threads may launch at the same time)
    struct Limits {
        cudaError_t err;
        int optin, sms;
    };
    static const Limits lim = [] {
        Limits l{cudaSuccess, 0, 0};
        int dev = 0;
        l.err = cudaGetDevice(&dev);
        if (l.err == cudaSuccess) l.err = cudaDeviceGetAttribute(&l.optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
        if (l.err == cudaSuccess) l.err = cudaDeviceGetAttribute(&l.sms, cudaDevAttrMultiProcessorCount, dev);
        if (l.err == cudaSuccess)
            l.err = cudaFuncSetAttribute(k_fused<T, K>, cudaFuncAttributeMaxDynamicSharedMemorySize, l.optin);
        return l;
    }();
    if (lim.err != cudaSuccess) return lim.err;
    const int optin = lim.optin, sms = lim.sms;
    if (smem > (size_t)optin) return cudaErrorInvalidValue;  // program or coefficient row too large
    int per_sm = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_fused<T, K>, 1 << (K - R), smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    const int64_t items = (int64_t)L.states << L.cta_shift;
    const int64_t grid = std::min<int64_t>(items, (int64_t)sms * per_sm);
    k_fused<T, K><<<(unsigned)grid, 1 << (K - R), smem, st>>>(reinterpret_cast<V*>(amps), L);
    return cudaGetLastError();
}

}  // namespace

FusedLaunch fused_launch_params(int qubits, const FusedPass& p, const FusedOp* d_ops, const FusedBatch* batch) {
    FusedLaunch L;
    const int K = p.k;
    const uint32_t all = (1u << qubits) - 1u;
    L.outer_mask = all & ~p.block_mask;
    uint32_t reg_in_local = 0, reg_out_local = 0;
    for (int m = 0; m < R; ++m) {
        L.reg_in_l[m] = p.reg_in[m];
        L.reg_in_g[m] = 1u << p.q[p.reg_in[m]];
        L.reg_out_g[m] = 1u << p.q_out[p.reg_out[m]];
        reg_in_local |= 1u << p.reg_in[m];
        reg_out_local |= 1u << p.reg_out[m];
    }
    L.thread_in = 0;
    L.thread_out = 0;
    for (int b = 0; b < K; ++b) {
        if (!(reg_in_local & (1u << b))) L.thread_in |= 1u << p.q[b];
        if (!(reg_out_local & (1u << b))) L.thread_out |= 1u << p.q_out[b];
    }
    for (int r = 0; r < 16; ++r) L.out_bit[r] = r < K - R ? (uint8_t)p.out_bit[r] : 0;
    L.op_count = p.op_count;
    L.ops = d_ops + p.op_begin;
    L.cta_shift = qubits - K;
    L.states = batch ? batch->states : 1;
    const bool tabled = batch && batch->table;
    L.table = tabled ? batch->table + 8 * (size_t)batch->slot_offset : nullptr;
    L.state_stride = batch ? batch->state_stride : 0;
    L.table_stride = batch ? batch->table_stride : 0;
    L.table_slots = !tabled ? 0 : batch->slot_count >= 0 ? batch->slot_count : (int32_t)(batch->table_stride / 8);
    L.pad = 0;
    return L;
}

cudaError_t launch_fused(void* amps, int qubits, int precision, const FusedPass& p, const FusedOp* d_ops,
                         const FusedBatch* batch, cudaStream_t st) {
    if (p.k > qubits || p.op_count > kMaxPassOps || p.op_count < 0 || !d_ops) return cudaErrorInvalidValue;
    if (batch && (batch->states < 1 || batch->states > 65535)) return cudaErrorInvalidValue;
    if (precision == QM_FP32) {
        switch (p.k) {
        case 9: return launch_k<float, 9>(amps, qubits, p, d_ops, batch, st);
        case 10: return launch_k<float, 10>(amps, qubits, p, d_ops, batch, st);
        case 11: return launch_k<float, 11>(amps, qubits, p, d_ops, batch, st);
        case 12: return launch_k<float, 12>(amps, qubits, p, d_ops, batch, st);
        case 13: return launch_k<float, 13>(amps, qubits, p, d_ops, batch, st);
        default: return cudaErrorInvalidValue;
        }
    }
    switch (p.k) {
    case 9: return launch_k<double, 9>(amps, qubits, p, d_ops, batch, st);
    case 10: return launch_k<double, 10>(amps, qubits, p, d_ops, batch, st);
    case 11: return launch_k<double, 11>(amps, qubits, p, d_ops, batch, st);
    case 12: return launch_k<double, 12>(amps, qubits, p, d_ops, batch, st);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace qm
