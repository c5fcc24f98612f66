// qm_jit.cpp -- fused passes compiled for their own op sequence (NVRTC, sm_100a).
//
// k_fused interprets a pass program: for every op it decodes the record, selects the register
// bit through a switch and, for an X or SWAP on register bits, moves the amplitudes between
// registers.  Here a pass's op sequence is turned into straight-line CUDA C++ and compiled once
// with NVRTC for sm_100a.  The generated kernel takes k_fused's launch record and shared-memory
// layout plus a constant parameter block: coefficients come from the staged program, the batch
// table or that block, never from the source, so one compiled kernel serves every pass with
// the same structure and rotation forms.  What the generation fixes at compile time:
//   - the register of every op, and the register pairs it touches;
//   - the control predicates: register bits select pairs at compile time, thread bits become
//     one uniform test per op, bits outside the block one test per work item;
//   - an X, CNOT or SWAP acting on register bits only renames registers: no instruction;
//   - the load, store and shared-memory exchange addresses as constants and bit deposits,
//     including a relabeling pass's store (qubits written to other index bits of the block)
//     and the lane order a stage may set for it;
//   - uncontrolled 2x2 unitaries as scaled rotations between deferred phases (below), with the
//     phases carried from pass to pass of a plan;
//   - from 26 qubits, the copy of the next work item's tile during the current one;
//   - the variants of the batch workloads: a first pass that starts from |0...0>, a last pass
//     whose epilogue writes a damping group's joint masses.
// The tiled expectation of the batched variational evaluator is generated here as well, for its
// term list.  NVRTC is loaded at run time; without it every pass runs on k_fused, the GPU
// interpreter, and every expectation on the generic tiled kernel.
#include <cuda_runtime.h>
#include <dlfcn.h>
#include <nvrtc.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <complex>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <sstream>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "qm_internal.h"

namespace qm {

namespace {

static_assert(sizeof(FusedOp) == 88, "FusedOp layout is mirrored in the generated source");
static_assert(sizeof(FusedLaunch) == 128 && offsetof(FusedLaunch, out_bit) == 112,
              "FusedLaunch layout is mirrored in the generated source");
static_assert(offsetof(FusedLaunch, ops) == 80 && offsetof(FusedLaunch, table) == 88 &&
                  offsetof(FusedLaunch, state_stride) == 96 && offsetof(FusedLaunch, table_stride) == 104,
              "FusedLaunch layout is mirrored in the generated source");
static_assert(offsetof(FusedOp, coef) == 24, "FusedOp layout is mirrored in the generated source");

// ---------------------------------------------------------------- NVRTC, loaded on first use
struct Nvrtc {
    bool ok = false;
    decltype(&nvrtcCreateProgram) create = nullptr;
    decltype(&nvrtcCompileProgram) compile = nullptr;
    decltype(&nvrtcGetCUBINSize) cubin_size = nullptr;
    decltype(&nvrtcGetCUBIN) cubin = nullptr;
    decltype(&nvrtcGetProgramLogSize) log_size = nullptr;
    decltype(&nvrtcGetProgramLog) log = nullptr;
    decltype(&nvrtcDestroyProgram) destroy = nullptr;
};

const Nvrtc& nvrtc() {
    static const Nvrtc lib = [] {
        Nvrtc n;
        const char* env = std::getenv("QM_JIT");
        if (env && std::strcmp(env, "0") == 0) return n;
        void* h = nullptr;
        for (const char* name : {"libnvrtc.so.12", "libnvrtc.so", "/usr/local/cuda/lib64/libnvrtc.so.12"})
            if ((h = dlopen(name, RTLD_NOW | RTLD_LOCAL))) break;
        if (!h) return n;
        n.create = reinterpret_cast<decltype(n.create)>(dlsym(h, "nvrtcCreateProgram"));
        n.compile = reinterpret_cast<decltype(n.compile)>(dlsym(h, "nvrtcCompileProgram"));
        n.cubin_size = reinterpret_cast<decltype(n.cubin_size)>(dlsym(h, "nvrtcGetCUBINSize"));
        n.cubin = reinterpret_cast<decltype(n.cubin)>(dlsym(h, "nvrtcGetCUBIN"));
        n.log_size = reinterpret_cast<decltype(n.log_size)>(dlsym(h, "nvrtcGetProgramLogSize"));
        n.log = reinterpret_cast<decltype(n.log)>(dlsym(h, "nvrtcGetProgramLog"));
        n.destroy = reinterpret_cast<decltype(n.destroy)>(dlsym(h, "nvrtcDestroyProgram"));
        n.ok = n.create && n.compile && n.cubin_size && n.cubin && n.log_size && n.log && n.destroy;
        return n;
    }();
    return lib;
}

// ---------------------------------------------------------------- source generation
constexpr int R = kRegBits;
constexpr int NR = 1 << R;

uint32_t swz_host(uint32_t j, bool fp64) {
    if (fp64) {
        uint32_t h = j >> 3;
        return j ^ ((h ^ (h >> 3) ^ (h >> 6) ^ (h >> 9)) & 7u);
    }
    uint32_t h = j >> 4;
    return j ^ ((h ^ (h >> 4) ^ (h >> 8)) & 15u);
}

std::string hexu(uint32_t v) {
    std::ostringstream o;
    o << "0x" << std::hex << v << "u";
    return o.str();
}

// value's low bits scattered onto the set bits of a constant mask, as shifts of runs
std::string deposit_expr(const char* value, uint32_t mask) {
    std::ostringstream e;
    e << "(0u";
    int src = 0;
    for (int b = 0; b < 32;) {
        if (!((mask >> b) & 1u)) {
            ++b;
            continue;
        }
        int len = 0;
        while (b + len < 32 && ((mask >> (b + len)) & 1u)) ++len;
        const uint32_t ones = len == 32 ? 0xffffffffu : ((1u << len) - 1u);
        e << " | (((" << value << " >> " << src << ") & " << hexu(ones) << ") << " << b << ")";
        src += len;
        b += len;
    }
    e << ")";
    return e.str();
}

// bit r of value moved to bit bits[r] (r < n), as shifts of runs
std::string permute_expr(const char* value, const int8_t* bits, int n) {
    std::ostringstream e;
    e << "(0u";
    for (int r = 0; r < n;) {
        int len = 1;
        while (r + len < n && bits[r + len] == bits[r] + len) ++len;
        const uint32_t ones = (1u << len) - 1u;
        e << " | (((" << value << " >> " << r << ") & " << hexu(ones) << ") << " << (int)bits[r] << ")";
        r += len;
    }
    e << ")";
    return e.str();
}

// ---------------------------------------------------------------- deferred phases
// An uncontrolled 2x2 unitary is applied as
//     U = g diag(1, phi) m R diag(1, lam),  R = [[1, -t], [t, 1]] (|u00| >= |u10|) or [[t, -1], [1, t]],
// with |t| <= 1 and g, phi, lam of unit modulus.  On a register pair (x, y) that is
// w = lam y; x' = x - t w; y' = t x + w (or x' = t x - w; y' = x + t w): 8 flops against 16 for the
// dense product.  The scalar g m and the phase phi are deferred: phi becomes a pending phase
// exp(i theta parity(S)) over a set S of qubits, which the next rotation on a qubit of S takes
// into its lam, which an X or CNOT rewrites (conjugate; S xor {control}), and which the plan's
// last pass multiplies in.  Other passes only rescale by |g m| so magnitudes stay bounded.
using cplx = std::complex<double>;

struct Split {
    bool ok = false;
    bool form_b = false;  // R = [[t, -1], [1, t]]
    double t = 0.0;
    cplx gm{1.0, 0.0};
    cplx lam{1.0, 0.0}, phi{1.0, 0.0};
};

// The split of a 2x2 matrix (a, b, c, d as re/im pairs); ok only when it gives the matrix back
// to within 1e-15 in every entry (a unitary to double precision), so results stay those of the
// dense product to rounding.
Split split_unitary(const double* c) {
    Split s;
    const cplx u00(c[0], c[1]), u01(c[2], c[3]), u10(c[4], c[5]), u11(c[6], c[7]);
    if (c[1] == 0.0 && c[3] == 0.0 && c[5] == 0.0 && c[7] == 0.0 && c[0] == c[6] && c[2] == -c[4]) {
        // a real rotation needs no phases; m keeps its sign
        s.form_b = std::fabs(c[4]) > std::fabs(c[0]);
        const double m = s.form_b ? c[4] : c[0];
        if (m == 0.0) return Split{};
        s.t = (s.form_b ? c[0] : c[4]) / m;
        s.gm = m;
    } else {
        const double a = std::abs(u00), b = std::abs(u10);
        cplx g;
        if (a >= b) {
            if (!(a > 0.0)) return Split{};
            g = u00 / a;
        } else {
            g = a > 0.0 ? (u10 / b) * (-u01 / b) / (u11 / a) : u10 / b;
            const double gn = std::abs(g);
            if (!(gn > 0.0) || !std::isfinite(gn)) return Split{};
            g /= gn;
        }
        if (b > 0.0) {
            s.phi = u10 / (g * b);
            s.lam = -u01 / (g * b);
        } else {
            s.lam = u11 / (g * a);
        }
        s.form_b = b > a;
        const double m = s.form_b ? b : a;
        s.t = (s.form_b ? a : b) / m;
        s.gm = g * m;
    }
    cplx r00, r01, r10, r11;
    if (!s.form_b) {
        r00 = s.gm;
        r01 = -s.gm * s.t * s.lam;
        r10 = s.gm * s.t * s.phi;
        r11 = s.gm * s.phi * s.lam;
    } else {
        r00 = s.gm * s.t;
        r01 = -s.gm * s.lam;
        r10 = s.gm * s.phi;
        r11 = s.gm * s.t * s.phi * s.lam;
    }
    const double err = std::max(std::max(std::abs(r00 - u00), std::abs(r01 - u01)),
                                std::max(std::abs(r10 - u10), std::abs(r11 - u11)));
    s.ok = std::isfinite(err) && std::isfinite(s.t) && err <= 1e-15;
    return s;
}

// A pending phase: exp(i theta) on the amplitudes whose bits in S (local bits and bits outside
// the block, as global bits) have odd parity; v = exp(i theta).
struct Pend {
    uint32_t lmask, omask;
    cplx v;
};

// What a plan's pass hands to the next: pending sets as global qubit masks, and the global phase.
struct Carry {
    std::vector<std::pair<uint32_t, cplx>> pend;
    cplx g{1.0, 0.0};
};

constexpr int kMaxVariantBits = 5;      // pending sets one rotation may depend on at run time
constexpr size_t kMaxAuxValues = 3000;  // constants per pass (kernel parameter space)

// States of at least this many qubits copy the next work item's tile during the current one
// (QM_PIPE_QUBITS overrides the 26; the CPU emulator of the generated kernels uses it to run the
// pipelined forms on small states).
int pipe_min_qubits() {
    const char* e = std::getenv("QM_PIPE_QUBITS");
    const int v = e ? std::atoi(e) : 0;
    return v > 0 ? v : 26;
}

// Complex128 pipelined passes as two teams per block with a compute token (QM_TEAMS=1; off by
// default).  Measured on the 30-qubit brick: 512.5 against 515.2 ms per step with conditional
// register swaps in the passes, 446.0 against 440.5 ms once the CNOTs are folded into H CZ H.
bool teams_enabled() {
    const char* e = std::getenv("QM_TEAMS");
    return e && e[0] == '1';
}

const char* kPrelude = R"SRC(
typedef unsigned int u32;
typedef unsigned long long u64;
struct FusedOp {
    unsigned char code;
    signed char reg, reg2, local;
    signed char reg_pos[4];
    unsigned short cmask_local, flags;
    u32 cmask_outer, target_outer, reserved;
    double coef[8];
};
struct FusedLaunch {
    u32 outer_mask, thread_in, thread_out;
    int op_count;
    u32 reg_in_g[4], reg_out_g[4];
    int reg_in_l[4];
    int cta_shift, states, table_slots, pad;
    const FusedOp* ops;
    const double* table;
    u64 state_stride, table_stride;
    unsigned char out_bit[16];
};
__device__ __forceinline__ u32 qm_deposit(u32 value, u32 mask) {
    u32 out = 0;
    while (mask) {
        const u32 low = mask & (0u - mask);
        if (value & 1u) out |= low;
        value >>= 1;
        mask ^= low;
    }
    return out;
}
#ifndef QM_EMULATED
// tile copies (cp.async, no registers) and the named barriers of two-team blocks
__device__ __forceinline__ void qm_cp16(u32 dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" :: "r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void qm_cp8(u32 dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" :: "r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void qm_cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void qm_cp_wait() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }
__device__ __forceinline__ void qm_bar(u32 id, u32 n) { asm volatile("bar.sync %0, %1;" :: "r"(id), "r"(n) : "memory"); }
__device__ __forceinline__ void qm_arrive(u32 id, u32 n) { asm volatile("bar.arrive %0, %1;" :: "r"(id), "r"(n) : "memory"); }
#endif
)SRC";

struct Gen {
    std::ostringstream os;
    bool fp64;
    int K;
    int phys[NR];
    uint32_t pm[R];  // local masks of the register bits in the current layout
    const char* T;
    // deferred phases (compile-time bookkeeping; values go to the kernel's constant parameter)
    std::vector<double> aux;
    std::vector<Pend> pend;
    cplx G{1.0, 0.0};
    int uid = 0;
    uint32_t lanes = 0;  // lane order of the current layout (OP_STAGE `reserved`; 0: ascending)
    // the block barrier of the exchanges (a team's named barrier in two-team blocks)
    std::string bar = "__syncthreads();\n";

    std::string X(int i) const { return "x" + std::to_string(phys[i]); }
    std::string Y(int i) const { return "y" + std::to_string(phys[i]); }

    uint32_t regmask() const {
        uint32_t r = 0;
        for (int m = 0; m < R; ++m) r |= pm[m];
        return r;
    }
    // register-index bits and thread (local, non-register) bits of a local mask
    void split(uint32_t local, uint32_t& reg_idx, uint32_t& thread_bits) const {
        reg_idx = 0;
        for (int m = 0; m < R; ++m)
            if (local & pm[m]) reg_idx |= 1u << m;
        thread_bits = local & ~regmask();
    }
    int reg_of_local(int lt) const {
        for (int m = 0; m < R; ++m)
            if (pm[m] == (1u << lt)) return m;
        return -1;
    }
    uint32_t const_slot(int i) const {
        uint32_t j = 0;
        for (int m = 0; m < R; ++m)
            if ((i >> m) & 1) j |= pm[m];
        return swz_host(j, fp64);
    }
    void set_layout(const int8_t* pos) {
        for (int m = 0; m < R; ++m) pm[m] = 1u << pos[m];
    }
    // thread t's local index: thread ranks on the lanes first (when the layout has lanes), then
    // on the remaining non-register local bits in ascending order
    std::string base_expr() const {
        uint32_t free = ((1u << K) - 1u) & ~regmask();
        const int n = stage_lane_count(lanes);
        if (n == 0) return deposit_expr("t", free);
        int8_t lb[8];
        for (int r = 0; r < n; ++r) {
            lb[r] = (int8_t)stage_lane(lanes, r);
            free &= ~(1u << lb[r]);
        }
        const std::string rest = "(t >> " + std::to_string(n) + ")";
        return "(" + permute_expr("t", lb, n) + " | " + deposit_expr(rest.c_str(), free) + ")";
    }

    // opens runtime conditions for outer and thread control bits; returns how many to close
    int open_conditions(uint32_t outer_bits, uint32_t thread_bits) {
        int n = 0;
        if (outer_bits) {
            os << "if ((outer & " << hexu(outer_bits) << ") == " << hexu(outer_bits) << ") {\n";
            ++n;
        }
        if (thread_bits) {
            os << "if ((base & " << hexu(thread_bits) << ") == " << hexu(thread_bits) << ") {\n";
            ++n;
        }
        return n;
    }
    void close(int n) {
        for (int i = 0; i < n; ++i) os << "}\n";
    }
    std::string coef_ptr(int o, const FusedOp& op) const {
        if (op.flags & kOpTable) return "(table + " + std::to_string(8 * op.reserved) + ")";
        return "prog[" + std::to_string(o) + "].coef";
    }

    void pairs_matrix(int M, uint32_t rm, bool real) {
        for (int i = 0; i < NR; ++i) {
            if ((i >> M) & 1) continue;
            if (((uint32_t)i & rm) != rm) continue;
            const int k = i | (1 << M);
            os << "{ const " << T << " xr = " << X(i) << ", xi = " << Y(i) << ", yr = " << X(k) << ", yi = " << Y(k)
               << ";\n";
            if (real) {
                os << X(i) << " = ar * xr + br * yr; " << Y(i) << " = ar * xi + br * yi;\n";
                os << X(k) << " = cr * xr + dr * yr; " << Y(k) << " = cr * xi + dr * yi; }\n";
            } else {
                os << X(i) << " = ar * xr - ai * xi + br * yr - bi * yi; " << Y(i)
                   << " = ar * xi + ai * xr + br * yi + bi * yr;\n";
                os << X(k) << " = cr * xr - ci * xi + dr * yr - di * yi; " << Y(k)
                   << " = cr * xi + ci * xr + dr * yi + di * yr; }\n";
            }
        }
    }
    void load_coef(const std::string& c, bool real) {
        os << "const " << T << " ar = (" << T << ")" << c << "[0], br = (" << T << ")" << c << "[2], cr = (" << T
           << ")" << c << "[4], dr = (" << T << ")" << c << "[6];\n";
        if (!real)
            os << "const " << T << " ai = (" << T << ")" << c << "[1], bi = (" << T << ")" << c << "[3], ci = (" << T
               << ")" << c << "[5], di = (" << T << ")" << c << "[7];\n";
    }
    void cmul_reg(int i, const char* pr, const char* pi) {
        os << "{ const " << T << " vr = " << X(i) << ", vi = " << Y(i) << "; " << X(i) << " = " << pr << " * vr - "
           << pi << " * vi; " << Y(i) << " = " << pr << " * vi + " << pi << " * vr; }\n";
    }
    void negate_reg(int i) { os << X(i) << " = -" << X(i) << "; " << Y(i) << " = -" << Y(i) << ";\n"; }

    void swap_pairs(const std::vector<std::pair<int, int>>& prs, bool runtime) {
        if (!runtime) {  // a fixed register permutation: rename
            for (auto& pr : prs) std::swap(phys[pr.first], phys[pr.second]);
            return;
        }
        for (auto& pr : prs)
            os << "{ " << T << " u = " << X(pr.first) << "; " << X(pr.first) << " = " << X(pr.second) << "; "
               << X(pr.second) << " = u; u = " << Y(pr.first) << "; " << Y(pr.first) << " = " << Y(pr.second) << "; "
               << Y(pr.second) << " = u; }\n";
    }

    void stage(const int8_t* pos, uint32_t lane_code) {
        os << "{ const u32 sb = qm_swz(base);\n" << bar;
        for (int i = 0; i < NR; ++i) {
            os << "{ V v; v.x = " << X(i) << "; v.y = " << Y(i) << "; tile[sb ^ " << hexu(const_slot(i)) << "] = v; }\n";
        }
        set_layout(pos);
        lanes = lane_code;
        for (int i = 0; i < NR; ++i) phys[i] = i;
        os << "base = " << base_expr() << ";\n";
        os << "const u32 sn = qm_swz(base);\n" << bar;
        for (int i = 0; i < NR; ++i)
            os << "{ const V v = tile[sn ^ " << hexu(const_slot(i)) << "]; x" << i << " = v.x; y" << i << " = v.y; }\n";
        os << "}\n";
    }

    void diag(int o, const FusedOp& op) {
        uint32_t rm, tb;
        split(op.cmask_local, rm, tb);
        const bool a_one = (op.flags & 1) != 0, d_one = (op.flags & 2) != 0;
        if (a_one && d_one) return;
        const int n = open_conditions(op.cmask_outer, tb);
        const std::string c = coef_ptr(o, op);
        os << "{ const " << T << " ar = (" << T << ")" << c << "[0], ai = (" << T << ")" << c << "[1], dr = (" << T
           << ")" << c << "[6], di = (" << T << ")" << c << "[7];\n";
        const int M = op.local >= 0 ? reg_of_local(op.local) : -1;
        if (M >= 0) {
            for (int i = 0; i < NR; ++i) {
                if (((uint32_t)i & rm) != rm) continue;
                if ((i >> M) & 1) {
                    if (!d_one) cmul_reg(i, "dr", "di");
                } else if (!a_one) {
                    cmul_reg(i, "ar", "ai");
                }
            }
        } else {
            if (op.local >= 0)
                os << "const bool bt = ((base >> " << (int)op.local << ") & 1u) != 0u;\n";
            else
                os << "const bool bt = (outer & " << hexu(op.target_outer) << ") != 0u;\n";
            os << "if (!(bt ? " << (d_one ? "true" : "false") << " : " << (a_one ? "true" : "false") << ")) {\n";
            os << "const " << T << " pr = bt ? dr : ar, pi = bt ? di : ai;\n";
            for (int i = 0; i < NR; ++i)
                if (((uint32_t)i & rm) == rm) cmul_reg(i, "pr", "pi");
            os << "}\n";
        }
        os << "}\n";
        close(n);
    }

    // Z and CZ (a sign on at most two bits) as deferred parity phases: (-1)^a, or
    // (-1)^(a b) = i^a i^b (-i)^(a xor b), where `defer_ok` allows it for op o of the pass.
    std::vector<char> defer_ok;
    bool defer_sign(const FusedOp& op, int o) {
        if (o < 0 || (size_t)o >= defer_ok.size() || !defer_ok[(size_t)o]) return false;
        const int bits = __builtin_popcount(op.cmask_local) + __builtin_popcount(op.cmask_outer);
        if (bits == 1) {
            pend.push_back({op.cmask_local, op.cmask_outer, cplx(-1.0, 0.0)});
        } else if (bits == 2) {
            uint32_t l = op.cmask_local, o = op.cmask_outer;
            Pend a{0u, 0u, cplx(0.0, 1.0)}, b{0u, 0u, cplx(0.0, 1.0)};
            if (l) {
                a.lmask = l & (0u - l);
                l &= l - 1u;
            } else {
                a.omask = o & (0u - o);
                o &= o - 1u;
            }
            if (l) b.lmask = l;
            else b.omask = o;
            pend.push_back(a);
            pend.push_back(b);
            pend.push_back({op.cmask_local, op.cmask_outer, cplx(0.0, -1.0)});
        } else {
            return false;
        }
        normalize();
        return true;
    }

    void negate(const FusedOp& op) {
        uint32_t rm, tb;
        split(op.cmask_local, rm, tb);
        const int n = open_conditions(op.cmask_outer, tb);
        for (int i = 0; i < NR; ++i)
            if (((uint32_t)i & rm) == rm) negate_reg(i);
        close(n);
    }

    void group(int o, const std::vector<FusedOp>& ops, int first, int count) {
        // register-bit phases per member; thread and outer phases folded into u
        bool any_u = false;
        for (int k = 0; k < count; ++k) {
            const FusedOp& m = ops[(size_t)(first + k)];
            if (m.code == OP_DIAG && !(m.local >= 0 && reg_of_local(m.local) >= 0)) any_u = true;
        }
        os << "{\n";
        if (any_u) os << T << " ur = (" << T << ")1, ui = (" << T << ")0;\n";
        for (int k = 0; k < count; ++k) {
            const FusedOp& m = ops[(size_t)(first + k)];
            const int om = o + 1 + k;
            if (m.code == OP_NEGATE) {
                if (!defer_sign(m, om)) negate(m);
                continue;
            }
            const int M = m.local >= 0 ? reg_of_local(m.local) : -1;
            if (M >= 0) {
                diag(om, m);
                continue;
            }
            const int n = open_conditions(m.cmask_outer, 0);
            const std::string c = coef_ptr(om, m);
            if (m.local >= 0)
                os << "{ const bool bt = ((base >> " << (int)m.local << ") & 1u) != 0u;\n";
            else
                os << "{ const bool bt = (outer & " << hexu(m.target_outer) << ") != 0u;\n";
            os << "const " << T << " pr = (" << T << ")(bt ? " << c << "[6] : " << c << "[0]), pi = (" << T
               << ")(bt ? " << c << "[7] : " << c << "[1]);\n";
            os << "const " << T << " nr = ur * pr - ui * pi; ui = ur * pi + ui * pr; ur = nr; }\n";
            close(n);
        }
        if (any_u)
            for (int i = 0; i < NR; ++i) cmul_reg(i, "ur", "ui");
        os << "}\n";
    }

    // ------------------------------------------------ deferred phases
    int slot(double v) {
        aux.push_back(v);
        return (int)aux.size() - 1;
    }
    int slot2(cplx v) {
        aux.push_back(v.real());
        aux.push_back(v.imag());
        return (int)aux.size() - 2;
    }
    static std::string av(int s) { return "A.v[" + std::to_string(s) + "]"; }
    int local_of_reg(int M) const { return __builtin_ctz(pm[M]); }
    uint32_t reg_part(uint32_t lmask) const {
        uint32_t r, t;
        split(lmask, r, t);
        return r;
    }
    // run-time parity (an int expression, 0 or 1) of a set's thread bits and bits outside the
    // block; "" when the set has none
    std::string sel_expr(uint32_t lmask, uint32_t omask) const {
        const uint32_t tb = lmask & ~regmask();
        std::string e;
        if (tb) e = "__popc(base & " + hexu(tb) + ")";
        if (omask) e += std::string(e.empty() ? "" : " + ") + "__popc(outer & " + hexu(omask) + ")";
        return e.empty() ? e : "((" + e + ") & 1)";
    }
    // one entry per set; an empty set has even parity and a phase of 1 is nothing
    void normalize() {
        std::vector<Pend> out;
        for (const Pend& e : pend) {
            bool merged = false;
            for (Pend& o : out)
                if (o.lmask == e.lmask && o.omask == e.omask) {
                    o.v *= e.v;
                    merged = true;
                    break;
                }
            if (!merged) out.push_back(e);
        }
        pend.clear();
        for (const Pend& e : out)
            if ((e.lmask || e.omask) && !(e.v == cplx(1.0, 0.0))) pend.push_back(e);
    }
    bool holds(int q) const {
        for (const Pend& e : pend)
            if ((e.lmask >> q) & 1u) return true;
        return false;
    }
    // distinct sets that remain of the pending sets holding q once q leaves them
    int dep_count(int q) const {
        std::vector<std::pair<uint32_t, uint32_t>> sets;
        for (const Pend& e : pend) {
            if (!((e.lmask >> q) & 1u)) continue;
            const std::pair<uint32_t, uint32_t> r(e.lmask & ~(1u << q), e.omask);
            if ((r.first || r.second) && std::find(sets.begin(), sets.end(), r) == sets.end()) sets.push_back(r);
        }
        return (int)sets.size();
    }
    void cmul_var(const std::string& v, const std::string& pr, const std::string& pi) {
        os << "{ const " << T << " vr = " << v << "r, vi = " << v << "i; " << v << "r = " << pr << " * vr - (" << pi
           << ") * vi; " << v << "i = " << pr << " * vi + (" << pi << ") * vr; }\n";
    }

    // The phase that the amplitudes with local bit q set take from the pending sets holding q,
    // times `extra`; q leaves those sets:
    //     exp(i theta (b_q ^ p)) = [p ? e : 1] * [b_q ? (p ? conj e : e) : 1],  p = parity(S \ {q}).
    // The variants over p are constants; the run-time part of p selects one.  Returns, per
    // register pair (by its low register index), the class (0: one, 1: minus one, 2: variables).
    struct PairPhase {
        int cls = 0;
        std::string re[NR], im[NR];
        // shear form (rotations only): the pair's phase known at compile time as i^quad exp(i a),
        // |a| <= pi/4, applied to y as three shears with tan(a / 2) and sin(a) (names in re / im)
        bool shear[NR] = {};
        int quad[NR] = {};
    };
    // One phase value as i^quad exp(i a), |a| <= pi/4: its shear constants tan(a / 2), sin(a).
    void shear_constants(cplx v, int& quad, int& st, int& ss) {
        double a = std::arg(v);
        const double q = std::nearbyint(a / (M_PI / 2));
        a -= q * (M_PI / 2);
        quad = ((int)q % 4 + 4) % 4;
        st = slot(std::tan(a / 2));
        ss = slot(std::sin(a));
    }
    PairPhase take_phase(int q, cplx extra, bool shears = false) {
        PairPhase P;
        cplx ls = extra;
        std::vector<Pend> dep, keep;
        for (const Pend& e : pend) {
            if (!((e.lmask >> q) & 1u)) {
                keep.push_back(e);
                continue;
            }
            const Pend r{e.lmask & ~(1u << q), e.omask, e.v};
            if (!r.lmask && !r.omask) {
                ls *= e.v;
                continue;
            }
            bool merged = false;
            for (Pend& d : dep)
                if (d.lmask == r.lmask && d.omask == r.omask) {
                    d.v *= r.v;
                    merged = true;
                }
            if (!merged) dep.push_back(r);
            keep.push_back(r);
        }
        pend.swap(keep);
        normalize();
        if (dep.empty()) {
            if (ls == cplx(1.0, 0.0)) return P;
            if (ls == cplx(-1.0, 0.0)) {
                P.cls = 1;
                return P;
            }
            const std::string n = "l" + std::to_string(uid++);
            P.cls = 2;
            if (shears) {
                int quad, st, ss;
                shear_constants(ls, quad, st, ss);
                os << "const " << T << " " << n << "a = " << av(st) << ", " << n << "b = " << av(ss) << ";\n";
                for (int i = 0; i < NR; ++i) {
                    P.re[i] = n + "a";
                    P.im[i] = n + "b";
                    P.shear[i] = true;
                    P.quad[i] = quad;
                }
                return P;
            }
            const int s = slot2(ls);
            os << "const " << T << " " << n << "r = " << av(s) << ", " << n << "i = " << av(s + 1) << ";\n";
            for (int i = 0; i < NR; ++i) {
                P.re[i] = n + "r";
                P.im[i] = n + "i";
            }
            return P;
        }
        const int J = (int)dep.size();
        auto variant = [&](int key) {
            cplx v = ls;
            for (int d = 0; d < J; ++d) v *= ((key >> d) & 1) ? std::conj(dep[d].v) : dep[d].v;
            return v;
        };
        std::string kr;
        for (int d = 0; d < J; ++d) {
            const std::string e = sel_expr(dep[d].lmask, dep[d].omask);
            if (!e.empty()) kr += (kr.empty() ? "(" : " | (") + e + " << " + std::to_string(d) + ")";
        }
        const std::string id = std::to_string(uid++);
        P.cls = 2;
        std::string declared[1 << kMaxVariantBits];
        if (shears && kr.empty()) {  // every pair's variant is fixed by its register bits
            int quads[1 << kMaxVariantBits];
            for (int i = 0; i < NR; ++i) {
                int rk = 0;
                for (int d = 0; d < J; ++d)
                    if (__builtin_popcount((uint32_t)i & reg_part(dep[d].lmask)) & 1) rk |= 1 << d;
                if (declared[rk].empty()) {
                    int st, ss;
                    shear_constants(variant(rk), quads[rk], st, ss);
                    const std::string n = "l" + id + "_" + std::to_string(rk);
                    os << "const " << T << " " << n << "a = " << av(st) << ", " << n << "b = " << av(ss) << ";\n";
                    declared[rk] = n;
                }
                P.re[i] = declared[rk] + "a";
                P.im[i] = declared[rk] + "b";
                P.shear[i] = true;
                P.quad[i] = quads[rk];
            }
            return P;
        }
        // Phases chosen at run time take the shear form too when one quadrant i^quad leaves every
        // variant within 3 pi / 4 of it (shear constants up to tan(3 pi / 8) = 2.41): the table
        // then holds each variant's (tan(a / 2), sin(a)) instead of (re, im).
        int rquad = -1;
        if (shears) {
            double best = 3 * M_PI / 4 + 1e-12;
            for (int qd = 0; qd < 4; ++qd) {
                double worst = 0.0;
                for (int key = 0; key < (1 << J); ++key) {
                    const double a = std::remainder(std::arg(variant(key)) - qd * (M_PI / 2), 2 * M_PI);
                    worst = std::max(worst, std::fabs(a));
                }
                if (worst < best) {
                    best = worst;
                    rquad = qd;
                }
            }
        }
        const int first = (int)aux.size();
        for (int key = 0; key < (1 << J); ++key) {
            if (rquad < 0) {
                slot2(variant(key));
            } else {
                const double a = std::remainder(std::arg(variant(key)) - rquad * (M_PI / 2), 2 * M_PI);
                slot(std::tan(a / 2));
                slot(std::sin(a));
            }
        }
        if (!kr.empty()) os << "const int k" << id << " = " << kr << ";\n";
        const char* c0 = rquad < 0 ? "r" : "a";
        const char* c1 = rquad < 0 ? "i" : "b";
        for (int i = 0; i < NR; ++i) {
            int rk = 0;
            for (int d = 0; d < J; ++d)
                if (__builtin_popcount((uint32_t)i & reg_part(dep[d].lmask)) & 1) rk |= 1 << d;
            if (declared[rk].empty()) {
                const std::string n = "l" + id + "_" + std::to_string(rk);
                const std::string at = kr.empty() ? std::to_string(first + 2 * rk)
                                                  : std::to_string(first) + " + 2 * (k" + id + " ^ " + std::to_string(rk) + ")";
                os << "const " << T << " " << n << c0 << " = A.v[" << at << "], " << n << c1 << " = A.v[" << at
                   << " + 1];\n";
                declared[rk] = n;
            }
            P.re[i] = declared[rk] + c0;
            P.im[i] = declared[rk] + c1;
            if (rquad >= 0) {
                P.shear[i] = true;
                P.quad[i] = rquad;
            }
        }
        return P;
    }
    // Applies the pending phases that hold the qubit of register bit M (before an op on it that
    // does not take them).
    void resolve(int M) {
        const int q = local_of_reg(M);
        if (!holds(q)) return;
        if (dep_count(q) > kMaxVariantBits) {
            flush_all();
            return;
        }
        os << "{\n";
        const PairPhase P = take_phase(q, cplx(1.0, 0.0));
        for (int i = 0; i < NR; ++i) {
            if ((i >> M) & 1) continue;
            const int k = i | (1 << M);
            if (P.cls == 1) negate_reg(k);
            else if (P.cls == 2) cmul_reg(k, P.re[i].c_str(), P.im[i].c_str());
        }
        os << "}\n";
    }
    // Multiplies every amplitude by its pending phase and by G; nothing is pending afterwards.
    //     F(i) = G * prod_j ((par_j(i) ^ sel_j) ? e_j : 1)
    // with par_j the parity of set j's register bits in register index i and sel_j that of its
    // thread and outer bits.  The factors of sets without register bits multiply the thread
    // factor; the others group by register mask m into q_m, and a Gray-code walk over the
    // register indices steps F from one index to the next with one q_m (or its conjugate) per
    // mask holding the flipped bit.
    void flush_all() {
        normalize();
        if (pend.empty() && G == cplx(1.0, 0.0)) return;
        const std::string f = "f" + std::to_string(uid++);
        os << "{\n";
        std::vector<uint32_t> masks;
        std::vector<cplx> qc;
        struct Rt {
            std::string sel;
            cplx v;
            int group;
        };
        std::vector<Rt> rt;
        for (const Pend& e : pend) {
            const uint32_t rm = reg_part(e.lmask);
            int gi = -1;
            if (rm) {
                for (size_t j = 0; j < masks.size(); ++j)
                    if (masks[j] == rm) gi = (int)j;
                if (gi < 0) {
                    masks.push_back(rm);
                    qc.push_back(cplx(1.0, 0.0));
                    gi = (int)masks.size() - 1;
                }
            }
            const std::string sel = sel_expr(e.lmask, e.omask);
            if (sel.empty()) qc[(size_t)gi] *= e.v;
            else rt.push_back({sel, e.v, gi});
        }
        const int gs = slot2(G);
        os << T << " " << f << "r = " << av(gs) << ", " << f << "i = " << av(gs + 1) << ";\n";
        std::vector<std::string> qn(masks.size());
        std::vector<bool> qrun(masks.size(), false);
        for (const Rt& r : rt)
            if (r.group >= 0) qrun[(size_t)r.group] = true;
        for (size_t j = 0; j < masks.size(); ++j) {
            qn[j] = f + "q" + std::to_string(j);
            const int s = slot2(qc[j]);
            os << (qrun[j] ? "" : "const ") << T << " " << qn[j] << "r = " << av(s) << ", " << qn[j]
               << "i = " << av(s + 1) << ";\n";
        }
        for (const Rt& r : rt) {
            const int s = slot2(r.v);
            os << "{ const bool s = " << r.sel << " != 0;\n";
            os << "const " << T << " er = s ? " << av(s) << " : (" << T << ")1, ei = s ? " << av(s + 1) << " : (" << T
               << ")0;\n";
            cmul_var(f, "er", "ei");
            if (r.group >= 0) {
                os << "const " << T << " qr = " << av(s) << ", qi = s ? -" << av(s + 1) << " : " << av(s + 1) << ";\n";
                cmul_var(qn[(size_t)r.group], "qr", "qi");
            }
            os << "}\n";
        }
        cmul_reg(0, (f + "r").c_str(), (f + "i").c_str());
        for (int k = 1; k < NR; ++k) {
            const int prev = (k - 1) ^ ((k - 1) >> 1), cur = k ^ (k >> 1);
            const int b = __builtin_ctz((unsigned)k);
            for (size_t j = 0; j < masks.size(); ++j) {
                if (!((masks[j] >> b) & 1u)) continue;
                // entering odd parity takes q_m, leaving it takes conj(q_m)
                const bool odd = __builtin_popcount((uint32_t)prev & masks[j]) & 1;
                cmul_var(f, qn[j] + "r", (odd ? "-" : "") + qn[j] + "i");
            }
            cmul_reg(cur, (f + "r").c_str(), (f + "i").c_str());
        }
        os << "}\n";
        pend.clear();
        G = cplx(1.0, 0.0);
    }
    // Multiplies by |G| so that magnitudes stay those of the state; G keeps its phase.
    void rescale() {
        const double r = std::abs(G);
        if (r == 1.0) return;
        const int s = slot(r);
        os << "{ const " << T << " r = " << av(s) << ";\n";
        for (int i = 0; i < NR; ++i) os << X(i) << " *= r; " << Y(i) << " *= r;\n";
        os << "}\n";
        G /= r;
    }
    bool rotatable(const FusedOp& op) const {
        return (op.code == OP_MATRIX || op.code == OP_MATRIX_REAL) && !(op.flags & (kOpTable | kOpBranch)) &&
               op.cmask_local == 0 && op.cmask_outer == 0 && aux.size() < kMaxAuxValues;
    }
    // An uncontrolled unitary on register bit M as a scaled rotation between two deferred phases.
    void rotation(const FusedOp& op, const Split& sp) {
        const int M = op.reg, q = local_of_reg(M);
        if (dep_count(q) > kMaxVariantBits) flush_all();
        os << "{\n";
        const PairPhase P = take_phase(q, sp.lam, true);
        const int ts = slot(sp.t);
        os << "const " << T << " t = " << av(ts) << ";\n";
        for (int i = 0; i < NR; ++i) {
            if ((i >> M) & 1) continue;
            const int k = i | (1 << M);
            os << "{ const " << T << " xr = " << X(i) << ", xi = " << Y(i) << ";\n";
            if (P.cls == 0)
                os << "const " << T << " wr = " << X(k) << ", wi = " << Y(k) << ";\n";
            else if (P.cls == 1)
                os << "const " << T << " wr = -" << X(k) << ", wi = -" << Y(k) << ";\n";
            else if (P.shear[i]) {
                // w = i^quad exp(i a) y: (ur, ui) = i^quad y (a renaming, its signs folded into the
                // multiply-adds), then three shears, 3 FMAs against 4 for the complex product
                static const char* const ur_of[4] = {"", "-", "-", ""};
                static const char* const ui_of[4] = {"", "", "-", "-"};
                const int qd = P.quad[i];
                const std::string ur = std::string(ur_of[qd]) + ((qd & 1) ? Y(k) : X(k));
                const std::string ui = std::string(ui_of[qd]) + ((qd & 1) ? X(k) : Y(k));
                os << "const " << T << " pu = " << ur << " - " << P.re[i] << " * " << ui << ";\n";
                os << "const " << T << " wi = " << ui << " + " << P.im[i] << " * pu;\n";
                os << "const " << T << " wr = pu - " << P.re[i] << " * wi;\n";
            } else
                os << "const " << T << " wr = " << P.re[i] << " * " << X(k) << " - " << P.im[i] << " * " << Y(k)
                   << ", wi = " << P.re[i] << " * " << Y(k) << " + " << P.im[i] << " * " << X(k) << ";\n";
            if (!sp.form_b)
                os << X(i) << " = xr - t * wr; " << Y(i) << " = xi - t * wi; " << X(k) << " = t * xr + wr; " << Y(k)
                   << " = t * xi + wi; }\n";
            else
                os << X(i) << " = t * xr - wr; " << Y(i) << " = t * xi - wi; " << X(k) << " = xr + t * wr; " << Y(k)
                   << " = xi + t * wi; }\n";
        }
        os << "}\n";
        if (!(sp.phi == cplx(1.0, 0.0))) pend.push_back({1u << q, 0u, sp.phi});
        normalize();
        G *= sp.gm;
    }

    // A CNOT folded into H CZ H (the H's went into the ops on its target before and after it):
    // CZ(c, t) = exp(i pi c t) deferred as the parity phases i^c, i^t and (-i)^(c xor t).
    void cz(const FusedOp& op) {
        const uint32_t t = 1u << local_of_reg(op.reg);
        pend.push_back({op.cmask_local, op.cmask_outer, cplx(0.0, 1.0)});
        pend.push_back({t, 0u, cplx(0.0, 1.0)});
        pend.push_back({t | op.cmask_local, op.cmask_outer, cplx(0.0, -1.0)});
        normalize();
    }

    void op(int o, const FusedOp& op) {
        uint32_t rm, tb;
        split(op.cmask_local, rm, tb);
        switch (op.code) {
        case OP_MATRIX:
        case OP_MATRIX_REAL: {
            if (rotatable(op)) {
                const Split sp = split_unitary(op.coef);
                if (sp.ok) {
                    rotation(op, sp);
                    break;
                }
            }
            resolve(op.reg);
            const int M = op.reg;
            const int n = open_conditions(op.cmask_outer, tb);
            const std::string c = coef_ptr(o, op);
            os << "{\n";
            if (op.flags & kOpBranch) {
                // noise branch: identity skipped, real diagonal as a scaling
                os << "const double* c = " << c << ";\n";
                os << "if (c[1] != 0.0 || c[3] != 0.0 || c[5] != 0.0 || c[7] != 0.0) {\n";
                load_coef("c", false);
                pairs_matrix(M, rm, false);
                os << "} else if (c[2] != 0.0 || c[4] != 0.0) {\n";
                load_coef("c", true);
                pairs_matrix(M, rm, true);
                os << "} else if (!(c[0] == 1.0 && c[6] == 1.0)) {\n";
                os << "const " << T << " s0 = (" << T << ")c[0], s1 = (" << T << ")c[6];\n";
                for (int i = 0; i < NR; ++i) {
                    const char* s = ((i >> M) & 1) ? "s1" : "s0";
                    os << X(i) << " *= " << s << "; " << Y(i) << " *= " << s << ";\n";
                }
                os << "}\n";
            } else {
                const bool real = op.code == OP_MATRIX_REAL;
                load_coef(c, real);
                pairs_matrix(M, rm, real);
            }
            os << "}\n";
            close(n);
            break;
        }
        case OP_EXCHANGE: {
            const int M = op.reg;
            // X: parity p -> p ^ 1, so exp(i theta p) = e * conj(e)^p; one control c: S ^= {c}
            const int q = local_of_reg(M);
            const int nc = __builtin_popcount(op.cmask_local) + __builtin_popcount(op.cmask_outer);
            if (nc == 0) {
                for (Pend& e : pend)
                    if ((e.lmask >> q) & 1u) {
                        G *= e.v;
                        e.v = std::conj(e.v);
                    }
            } else if (nc == 1) {
                for (Pend& e : pend)
                    if ((e.lmask >> q) & 1u) {
                        e.lmask ^= op.cmask_local;
                        e.omask ^= op.cmask_outer;
                    }
                normalize();
            } else {
                resolve(M);
            }
            std::vector<std::pair<int, int>> prs;
            for (int i = 0; i < NR; ++i)
                if (!((i >> M) & 1) && ((uint32_t)i & rm) == rm) prs.push_back({i, i | (1 << M)});
            const bool runtime = op.cmask_outer != 0 || tb != 0;
            const int n = open_conditions(op.cmask_outer, tb);
            swap_pairs(prs, runtime);
            close(n);
            break;
        }
        case OP_SWAP: {
            const int M1 = op.reg, M2 = op.reg2;
            if (op.cmask_local == 0 && op.cmask_outer == 0) {
                const uint32_t b1 = 1u << local_of_reg(M1), b2 = 1u << local_of_reg(M2);
                for (Pend& e : pend)
                    if (((e.lmask & b1) != 0) != ((e.lmask & b2) != 0)) e.lmask ^= b1 | b2;
                normalize();
            } else {
                resolve(M1);
                resolve(M2);
            }
            std::vector<std::pair<int, int>> prs;
            for (int i = 0; i < NR; ++i)
                if (((i >> M1) & 1) && !((i >> M2) & 1) && ((uint32_t)i & rm) == rm)
                    prs.push_back({i, i ^ (1 << M1) ^ (1 << M2)});
            const bool runtime = op.cmask_outer != 0 || tb != 0;
            const int n = open_conditions(op.cmask_outer, tb);
            swap_pairs(prs, runtime);
            close(n);
            break;
        }
        case OP_DIAG: diag(o, op); break;
        case OP_NEGATE:
            if (!defer_sign(op, o)) negate(op);
            break;
        default: break;
        }
    }
};

// The source of one pass's kernel and the constants it takes (kernel parameter `A`).  The source
// depends on the pass structure and on which form each rotation takes, never on the angles.
// With `carry`, pending phases come in from the previous pass and, unless `last`, go on to the
// next one; without it the pass is self-contained.
struct Generated {
    std::string src;
    std::vector<unsigned char> aux;  // the parameter block: doubles (complex128) or floats
    int tiles = 1;                   // tiles of shared memory (2: pipelined, or one per team)
    int teams = 1;                   // teams of 2^(k - 4) threads per block
    int hist_bins = 0;               // joint-mass epilogue bins (0: none)
    bool zero_start = false;         // the pass writes |0...0> instead of loading the state
};

// CNOT folding (QM_CZ_FOLD=0 turns it off).  A CNOT whose one control is a thread bit or a bit
// outside the block, with its target t in a register, is a conditional register swap: four
// selects per amplitude pair.  Since CNOT = H_t CZ H_t, where the op before it on t and the op
// after it on t (in the plan) are both uncontrolled 2x2 unitaries U_p and U_n, they become
// H U_p and U_n H (still rotations, at the same cost), and the CNOT becomes CZ(c, t), which the
// generator defers as three parity phases (exp(i pi c t) = i^c i^t (-i)^(c xor t)): no
// instruction at the CNOT.  `cz` marks the folded CNOTs and `forced` the ops whose coefficients
// changed: those must run as rotations (their constants travel in the kernel parameter; the
// staged program keeps the original coefficients, which the interpreter runs whole).
bool cz_fold_enabled() {
    const char* e = std::getenv("QM_CZ_FOLD");
    return !(e && e[0] == '0');
}

// The plan's ops with the folds applied: `cz` marks the folded CNOTs, `forced` the ops whose
// coefficients changed.  With `across` (chained plans, whose passes all run compiled) the op
// before or after a CNOT on its target may lie in another pass: qubits are followed through each
// pass's relabeling store (local bit b read from index bit q[b], written to q_out[b]).  Without
// it only folds within one pass are made, so a pass that runs on the interpreter (the original
// ops) never meets a neighbour changed for it.
struct Fold {
    std::vector<FusedOp> ops;
    std::vector<char> cz, forced;
};

// Which Z / CZ ops of a pass become deferred parity phases (QM_CZ_DEFER=0 turns it off): in a
// pass without table ops, a sign on at most two bits whose every local bit next meets, past
// diagonals and within the pass, an uncontrolled complex 2x2 (a rotation whose phase is a
// complex product anyway).  Elsewhere a deferred phase would turn a real rotation into a
// complex one or be resolved by a complex product before a table op: the sign stays a negation.
// Measured on the 30-qubit brick planned with CZs: 407.4 to 402.2 ms per step (FP64), 253.3 to
// 247.6 ms (FP32).
std::vector<char> sign_deferrals(const FusedPass& p, const std::vector<FusedOp>& all, bool tabled) {
    std::vector<char> ok((size_t)p.op_count, 0);
    const char* e = std::getenv("QM_CZ_DEFER");
    if (tabled || (e && e[0] == '0')) return ok;
    // per op: local bits touched, and whether the op is a diagonal (commutes with the phases)
    std::vector<uint32_t> touch((size_t)p.op_count, 0);
    std::vector<char> diagonal((size_t)p.op_count, 0);
    int8_t pos[R];
    for (int m = 0; m < R; ++m) pos[m] = p.reg_in[m];
    for (int o = 0; o < p.op_count; ++o) {
        const FusedOp& op = all[(size_t)(p.op_begin + o)];
        uint32_t t = op.cmask_local;
        switch (op.code) {
        case OP_STAGE:
            for (int m = 0; m < R; ++m) pos[m] = op.reg_pos[m];
            t = 0;
            diagonal[(size_t)o] = 1;
            break;
        case OP_MATRIX:
        case OP_MATRIX_REAL:
        case OP_EXCHANGE: t |= 1u << pos[op.reg]; break;
        case OP_SWAP: t |= (1u << pos[op.reg]) | (1u << pos[op.reg2]); break;
        case OP_DIAG:
            if (op.local >= 0) t |= 1u << op.local;
            diagonal[(size_t)o] = 1;
            break;
        case OP_NEGATE:
        case OP_DIAG_GROUP: diagonal[(size_t)o] = 1; break;
        default: t = ~0u;
        }
        touch[(size_t)o] = t;
    }
    for (int o = 0; o < p.op_count; ++o) {
        const FusedOp& op = all[(size_t)(p.op_begin + o)];
        if (op.code != OP_NEGATE || __builtin_popcount(op.cmask_local) + __builtin_popcount(op.cmask_outer) > 2) continue;
        bool good = op.cmask_local != 0;
        for (uint32_t bits = op.cmask_local; bits && good; bits &= bits - 1u) {
            const uint32_t b = bits & (0u - bits);
            good = false;  // nothing further on the bit in this pass: the sign stays a negation
            for (int j = o + 1; j < p.op_count; ++j) {
                if (!(touch[(size_t)j] & b) || diagonal[(size_t)j]) continue;
                const FusedOp& n = all[(size_t)(p.op_begin + j)];
                good = n.code == OP_MATRIX && n.cmask_local == 0 && n.cmask_outer == 0 &&
                       !(n.flags & (kOpTable | kOpBranch));
                break;
            }
        }
        ok[(size_t)o] = good;
    }
    return ok;
}

Fold fold_plan(const Plan& plan, bool across) {
    Fold f;
    f.ops = plan.ops;
    f.cz.assign(plan.ops.size(), 0);
    f.forced.assign(plan.ops.size(), 0);
    if (!cz_fold_enabled() || plan.qubits > 32) return f;
    // per op: its pass, the logical qubits it touches (~0: unknown, touches all), and for a CNOT
    // candidate its target's logical qubit
    const size_t n = plan.ops.size();
    std::vector<int> pass_of(n, -1), target(n, -1);
    std::vector<uint64_t> touch(n, 0);
    int phys_to_log[32], log_to_phys[32];
    for (int q = 0; q < 32; ++q) phys_to_log[q] = log_to_phys[q] = q;
    auto logical = [&](uint32_t phys_mask) {
        uint64_t m = 0;
        for (int q = 0; q < 32; ++q)
            if ((phys_mask >> q) & 1u) m |= uint64_t(1) << phys_to_log[q];
        return m;
    };
    for (size_t pi = 0; pi < plan.passes.size(); ++pi) {
        const FusedPass& p = plan.passes[pi];
        int8_t pos[R];
        for (int m = 0; m < R; ++m) pos[m] = p.reg_in[m];
        auto local_logical = [&](uint32_t local_mask) {
            uint32_t phys = 0;
            for (int b = 0; b < p.k; ++b)
                if ((local_mask >> b) & 1u) phys |= 1u << p.q[b];
            return logical(phys);
        };
        for (int o = 0; o < p.op_count; ++o) {
            const size_t gi = (size_t)(p.op_begin + o);
            const FusedOp& op = plan.ops[gi];
            pass_of[gi] = (int)pi;
            uint32_t rm = 0;
            for (int m = 0; m < R; ++m) rm |= 1u << pos[m];
            uint32_t loc = op.cmask_local;
            uint64_t t = 0;
            switch (op.code) {
            case OP_STAGE:
                for (int m = 0; m < R; ++m) pos[m] = op.reg_pos[m];
                loc = 0;
                break;
            case OP_MATRIX:
            case OP_MATRIX_REAL:
            case OP_EXCHANGE: loc |= 1u << pos[op.reg]; break;
            case OP_SWAP: loc |= (1u << pos[op.reg]) | (1u << pos[op.reg2]); break;
            case OP_DIAG:
                if (op.local >= 0) loc |= 1u << op.local;
                break;
            case OP_NEGATE:
            case OP_DIAG_GROUP: break;  // a group's members follow as ops of their own
            default: t = ~uint64_t(0);
            }
            if (op.code != OP_STAGE) t |= local_logical(loc) | logical(op.cmask_outer | op.target_outer);
            touch[gi] = t;
            if (op.code == OP_EXCHANGE && __builtin_popcount(op.cmask_local) + __builtin_popcount(op.cmask_outer) == 1 &&
                !(op.cmask_local & rm))
                target[gi] = (int)__builtin_ctzll(local_logical(1u << pos[op.reg]));
        }
        // the store: the logical qubit read from index bit q[b] now sits at q_out[b]
        int moved[32];
        for (int q = 0; q < 32; ++q) moved[q] = phys_to_log[q];
        for (int b = 0; b < p.k; ++b) moved[p.q_out[b]] = phys_to_log[p.q[b]];
        for (int q = 0; q < 32; ++q) {
            phys_to_log[q] = moved[q];
            log_to_phys[moved[q]] = q;
        }
    }
    // ops in plan order (passes are laid out in order in the op array)
    std::vector<size_t> order;
    for (const FusedPass& p : plan.passes)
        for (int o = 0; o < p.op_count; ++o) order.push_back((size_t)(p.op_begin + o));
    const double h = std::sqrt(0.5);
    auto plain = [&](size_t gi) {
        const FusedOp& op = f.ops[gi];
        return (op.code == OP_MATRIX || op.code == OP_MATRIX_REAL) && op.cmask_local == 0 && op.cmask_outer == 0 &&
               !(op.flags & (kOpTable | kOpBranch));
    };
    // the previous and next op touching each candidate's target, in plan order (folding keeps
    // every op's qubits)
    const size_t m = order.size();
    std::vector<long> prev_on(m, -1), next_on(m, -1);
    {
        long last[64];
        std::fill(last, last + 64, -1L);
        for (size_t k = 0; k < m; ++k) {
            const size_t gi = order[k];
            if (target[gi] >= 0) prev_on[k] = last[target[gi]];
            for (int q = 0; q < 64; ++q)
                if ((touch[gi] >> q) & 1u) last[q] = (long)k;
        }
        std::fill(last, last + 64, -1L);
        for (size_t k = m; k-- > 0;) {
            const size_t gi = order[k];
            if (target[gi] >= 0) next_on[k] = last[target[gi]];
            for (int q = 0; q < 64; ++q)
                if ((touch[gi] >> q) & 1u) last[q] = (long)k;
        }
    }
    for (size_t k = 0; k < m; ++k) {
        const size_t gi = order[k];
        if (target[gi] < 0) continue;
        const long before = prev_on[k], after = next_on[k];
        if (before < 0 || after < 0) continue;
        if (!across && (pass_of[order[(size_t)before]] != pass_of[gi] || pass_of[order[(size_t)after]] != pass_of[gi]))
            continue;
        const size_t bi = order[(size_t)before], ai = order[(size_t)after];
        if (!plain(bi) || !plain(ai)) continue;
        // H U (rows mixed) for the op before, U H (columns mixed) for the op after
        double* u = f.ops[bi].coef;
        double* v = f.ops[ai].coef;
        double nu[8], nv[8];
        for (int c = 0; c < 4; ++c) {
            nu[c] = h * (u[c] + u[c + 4]);
            nu[c + 4] = h * (u[c] - u[c + 4]);
        }
        for (int r = 0; r < 2; ++r)
            for (int c = 0; c < 2; ++c) {
                nv[4 * r + c] = h * (v[4 * r + c] + v[4 * r + 2 + c]);
                nv[4 * r + 2 + c] = h * (v[4 * r + c] - v[4 * r + 2 + c]);
            }
        if (!split_unitary(nu).ok || !split_unitary(nv).ok) continue;
        std::copy(nu, nu + 8, u);
        std::copy(nv, nv + 8, v);
        f.cz[gi] = 1;
        f.forced[bi] = f.forced[ai] = 1;
    }
    return f;
}

Generated generate(const FusedPass& p, const std::vector<FusedOp>& plan_ops, const Fold& fold, int qubits, bool fp64,
                   Carry* carry, bool last, uint32_t hist_mask = 0, bool zero_start = false) {
    Gen g;
    g.fp64 = fp64;
    g.K = p.k;
    g.T = fp64 ? "double" : "float";
    for (int i = 0; i < NR; ++i) g.phys[i] = i;
    g.set_layout(p.reg_in);
    if (carry) {
        for (const auto& e : carry->pend) {
            Pend x{0u, e.first & ~p.block_mask, e.second};
            for (int b = 0; b < p.k; ++b)
                if (e.first & (1u << p.q[b])) x.lmask |= 1u << b;
            g.pend.push_back(x);
        }
        g.G = carry->g;
        g.normalize();
    }
    uint32_t thread_in = 0, reg_in_local = 0;
    uint32_t reg_in_g[R], reg_out_g[R];
    for (int m = 0; m < R; ++m) {
        reg_in_local |= 1u << p.reg_in[m];
        reg_in_g[m] = 1u << p.q[p.reg_in[m]];
        reg_out_g[m] = 1u << p.q_out[p.reg_out[m]];
    }
    for (int b = 0; b < p.k; ++b) {
        if (!(reg_in_local & (1u << b))) thread_in |= 1u << p.q[b];
    }
    const int nt = 1 << (p.k - R);
    const size_t tile_bytes = (size_t)(fp64 ? 16 : 8) << p.k;
    const size_t prog_bytes = ((size_t)p.op_count * sizeof(FusedOp) + 15) & ~size_t(15);
    bool tabled = false;
    for (int o = 0; o < p.op_count; ++o)
        if (plan_ops[(size_t)(p.op_begin + o)].flags & kOpTable) tabled = true;
    // The tile pipeline needs a second tile of shared memory.  Complex64 blocks of 12 qubits keep
    // two blocks per SM with it (5.9 against 6.5 ms per 30-qubit brick pass).  A complex128 block
    // would take an SM alone, and one 8-warp block per SM computes too slowly (12.3 against
    // 10.7 ms).  States of fewer than 26 qubits largely stay in L2, where the extra trip through
    // shared memory costs more than it hides, and passes with a batch table lose more from
    // reading it without staging: all of those load straight from global memory.
    // Joint-mass epilogue: work items go in chunks of C consecutive tiles of one state, so that
    // partial row u = state * rows + r always holds the same tiles [r C, (r + 1) C) of its state
    // (rows = 2^(n-16), the layout of launch_group_histogram), whatever the state's place in the
    // batch.  Within a chunk the bins accumulate per warp in shared memory in a fixed order.
    // a relabeling pass (qubits written to other bits, lanes in the store layout) keeps the
    // separate joint-mass kernel: the epilogue reads the bins in the unpermuted, ascending layout
    bool relabels = false;
    for (int b = 0; b < p.k; ++b) relabels |= p.q_out[b] != p.q[b];
    for (int o = p.op_count - 1; o >= 0; --o) {
        const FusedOp& op = plan_ops[(size_t)(p.op_begin + o)];
        if (op.code != OP_STAGE) continue;
        relabels |= op.reserved != 0;  // the last stage sets the store layout
        break;
    }
    const bool hist = hist_mask != 0 && __builtin_popcount(hist_mask) <= kGroupMaxBits && !relabels;
    const int hist_bins = hist ? 1 << __builtin_popcount(hist_mask) : 0;
    const int chunk = hist ? (qubits > 16 ? 1 << (16 - p.k) : 1 << (qubits - p.k)) : 1;
    const int warps = nt / 32;
    const size_t hist_bytes = hist ? sizeof(double) * (size_t)warps * hist_bins : 0;
    const bool large = !tabled && !hist && !zero_start && qubits >= pipe_min_qubits();
    const bool second = large && !fp64 && 2 * tile_bytes + prog_bytes <= (100u << 10);
    // Complex128: the exchange tile itself takes the next item's copy once the pass's last
    // exchange is done, so the copy overlaps the ops after it, the flush and the stores.
    const bool late = large && fp64;
    const bool piped = second || late;
    int last_stage = -1, stages = 0;
    for (int o = 0; o < p.op_count; ++o)
        if (plan_ops[(size_t)(p.op_begin + o)].code == OP_STAGE) {
            last_stage = o;
            ++stages;
        }
    // Two teams per block (complex128 pipelined passes): the block is two teams of nt threads,
    // each with its own tile and work items, synchronised by its own named barrier (1 + team).
    // The teams take turns at the arithmetic: a team runs a compute segment (the ops between two
    // exchanges) only while it holds the token, and hands it over before its next exchange, so
    // one team's FP64 rotations overlap the other's shared-memory exchange and tile copy instead
    // of both teams computing, then both exchanging.  The token is a pair of named barriers of
    // both teams' threads: a team waits on its own (bar.sync) and signals the other's
    // (bar.arrive).  Team 1 signals once up front, and team 0 takes one more token after its last
    // item, so every barrier phase gets exactly its 2 nt arrivals; both teams run the same number
    // of loop iterations and segments (a team without an item passes the token on unused).
    const bool teams = late && teams_enabled() && 2 * nt <= 1024;
    const int segs = stages + 1;
    const std::string acquire = teams ? "qm_bar(tok_in, " + std::to_string(2 * nt) + "u);\n" : "";
    const std::string release = teams ? "qm_arrive(tok_out, " + std::to_string(2 * nt) + "u);\n" : "";
    if (teams) g.bar = "qm_bar(1u + team, " + std::to_string(nt) + "u);\n";
    const int tiles = second || teams ? 2 : 1;
    // Blocks per SM: 128 registers per thread (512 threads per SM; fewer registers would spill
    // the 16 amplitudes) and the shared memory (a pipelined complex128 block of 12 qubits takes
    // an SM alone).
    const int minb =
        teams ? std::max(1, 512 / (2 * nt))
              : std::max(1, std::min(512 / nt, (int)((220u << 10) / (tiles * tile_bytes + prog_bytes + 8192))));
    std::ostringstream& os = g.os;  // the kernel body
    os << "extern __shared__ __align__(16) unsigned char smem_raw[];\n";
    if (teams) {
        os << "const u32 team = threadIdx.x >> " << p.k - R << ";\n";
        os << "V* tile = reinterpret_cast<V*>(smem_raw + team * " << tile_bytes << "u);\n";
    } else {
        os << "V* tile = reinterpret_cast<V*>(smem_raw);\n";
    }
    if (second) os << "V* ptile = reinterpret_cast<V*>(smem_raw + " << tile_bytes << ");\n";
    if (late) os << "V* ptile = tile;\n";
    if (hist) os << "double* hacc = reinterpret_cast<double*>(smem_raw + " << tiles * tile_bytes << ");\n";
    os << "FusedOp* prog = reinterpret_cast<FusedOp*>(smem_raw + " << tiles * tile_bytes + hist_bytes << ");\n";
    os << "double* table = reinterpret_cast<double*>(smem_raw + " << (tiles * tile_bytes + hist_bytes + prog_bytes)
       << ");\n";
    os << (teams ? "const u32 t = threadIdx.x & " + hexu((uint32_t)nt - 1u) + ";\n" : "const u32 t = threadIdx.x;\n");
    os << "{ const uint2* src = reinterpret_cast<const uint2*>(P.ops); uint2* dst = reinterpret_cast<uint2*>(prog);\n"
       << "  for (int i = threadIdx.x; i < " << p.op_count * (int)(sizeof(FusedOp) / 8) << "; i += " << nt * (teams ? 2 : 1)
       << ") dst[i] = __ldg(src + i); }\n";
    if (teams) os << "__syncthreads();\n";  // both teams read the whole program
    os << "const long long total = (long long)P.states << P.cta_shift;\n";
    os << "const u32 cta_mask = (1u << P.cta_shift) - 1u;\n";
    // Tile pipeline: the next work item's tile is copied into `ptile` (cp.async, no registers)
    // while this one computes.  Thread t copies local indices t + nt*r, r < 16: consecutive
    // threads take consecutive amplitudes, so the copies come in the block's 128-byte runs.
    if (piped) {
        uint32_t lo = 0;
        for (int b = 0; b < p.k - R; ++b) lo |= 1u << p.q[b];
        os << "const u32 pf_g = " << deposit_expr("t", lo) << ";\n";
        os << "const u32 pf_b = (u32)__cvta_generic_to_shared(ptile), pf_w = qm_swz(t);\n";
    }
    auto prefetch = [&](const char* item_expr) {
        if (!piped) return;
        os << "{ const long long it = " << item_expr << ";\nif (it < total) {\n"
           << "const V* src = s0 + (u64)(int)(it >> P.cta_shift) * P.state_stride + (qm_deposit((u32)it & cta_mask, P.outer_mask) | pf_g);\n";
        for (int r = 0; r < NR; ++r) {
            uint32_t hi = 0;
            for (int m = 0; m < R; ++m)
                if ((r >> m) & 1) hi |= 1u << p.q[p.k - R + m];
            // slot of local index t + nt*r: the swizzle is linear, so qm_swz(t) ^ qm_swz(nt*r)
            os << (fp64 ? "qm_cp16(" : "qm_cp8(") << "pf_b + ((pf_w ^ " << hexu(swz_host((uint32_t)(nt * r), fp64))
               << ") << " << (fp64 ? 4 : 3) << "), src + " << hexu(hi) << ");\n";
        }
        os << "}\nqm_cp_commit(); }\n";
    };
    // a team's work items: every other one of the block's (team 0 the even, team 1 the odd)
    const char* next_item = teams ? "item + 2 * (long long)gridDim.x" : "item + gridDim.x";
    prefetch(teams ? "(long long)blockIdx.x + (long long)team * gridDim.x" : "(long long)blockIdx.x");
    os << "int current = -1;\n";
    if (hist) {
        os << "for (long long u = blockIdx.x; u < total / " << chunk << "; u += gridDim.x) {\n";
        os << "for (int i = t; i < " << warps * hist_bins << "; i += " << nt << ") hacc[i] = 0.0;\n";
        os << "for (int cc = 0; cc < " << chunk << "; ++cc) {\nconst long long item = u * " << chunk << " + cc;\n";
    } else if (teams) {
        os << "const u32 tok_in = team ? 4u : 3u, tok_out = team ? 3u : 4u;\n";
        os << "if (team == 1u) qm_arrive(3u, " << 2 * nt << "u);\n";
        os << "for (long long k2 = 0; (long long)blockIdx.x + k2 * gridDim.x < total; k2 += 2) {\n";
        os << "const long long item = (long long)blockIdx.x + (k2 + (long long)team) * gridDim.x;\n";
        os << "if (item >= total) { for (int j = 0; j < " << segs << "; ++j) { " << acquire << release << "} continue; }\n";
    } else {
        os << "for (long long item = blockIdx.x; item < total; item += gridDim.x) {\n";
    }
    os << "const int b = (int)(item >> P.cta_shift);\nconst u32 cta = (u32)item & cta_mask;\n";
    if (piped) os << "qm_cp_wait();\n";
    os << g.bar;
    if (tabled)
        os << "if (P.table_slots > 0 && b != current) { const double* row = P.table + (u64)b * P.table_stride;\n"
           << "  for (int i = t; i < 8 * P.table_slots; i += " << nt << ") table[i] = __ldg(row + i); __syncthreads(); }\n";
    os << "current = b;\n";
    os << "V* __restrict__ s = s0 + (u64)b * P.state_stride;\n";
    os << "const u32 outer = qm_deposit(cta, P.outer_mask);\n";
    os << g.T << " x0";
    for (int i = 1; i < NR; ++i) os << ", x" << i;
    for (int i = 0; i < NR; ++i) os << ", y" << i;
    os << ";\n";
    if (piped) {
        os << "u32 base = " << g.base_expr() << ";\n";
        os << "{ const u32 sn = qm_swz(base);\n";
        for (int i = 0; i < NR; ++i)
            os << "{ const V v = ptile[sn ^ " << hexu(g.const_slot(i)) << "]; x" << i << " = v.x; y" << i << " = v.y; }\n";
        os << "}\n";
        if (second || last_stage < 0) {
            os << g.bar;
            prefetch(next_item);
        }
        os << acquire;
    } else {
        os << "{ const u32 g0 = outer | " << deposit_expr("t", thread_in) << ";\n";
        for (int i = 0; i < NR; ++i) {
            uint32_t gi = 0;
            for (int m = 0; m < R; ++m)
                if ((i >> m) & 1) gi |= reg_in_g[m];
            if (zero_start)  // |0...0>: amplitude 1 at index 0 of every state, nothing read
                os << "x" << i << " = (g0 | " << hexu(gi) << ") == 0u ? (" << g.T << ")1 : (" << g.T << ")0; y" << i
                   << " = (" << g.T << ")0;\n";
            else
                os << "{ const V v = s[g0 | " << hexu(gi) << "]; x" << i << " = v.x; y" << i << " = v.y; }\n";
        }
        os << "}\n";
        os << "u32 base = " << g.base_expr() << ";\n";
    }
    g.defer_ok = sign_deferrals(p, fold.ops, tabled);
    for (int o = 0; o < p.op_count; ++o) {
        const size_t gi = (size_t)(p.op_begin + o);
        const FusedOp& op = fold.ops[gi];
        if (fold.cz[gi]) {
            g.cz(op);
            continue;
        }
        if (fold.forced[gi]) {
            g.rotation(op, split_unitary(op.coef));
            continue;
        }
        if (op.code == OP_STAGE) {
            os << release;
            g.stage(op.reg_pos, op.reserved);
            if (late && o == last_stage) {
                os << g.bar;  // every thread has read the exchange tile
                prefetch(next_item);
            }
            os << acquire;
            continue;
        }
        if (op.code == OP_DIAG_GROUP) {
            const int count = (int)op.reserved;
            g.group(o, plan_ops, p.op_begin + o + 1, count);
            o += count;
            continue;
        }
        g.op(o, op);
    }
    if (carry && !last) {
        // |g m| <= 1 per rotation, so the stored amplitudes grow by 1 / |G| until a rescale;
        // rescaling once |G| falls below 1e-60 (complex128) or 1e-9 (complex64) keeps them far
        // from overflow and saves a multiply per amplitude in most passes
        if (std::abs(g.G) < (fp64 ? 1e-60 : 1e-9)) g.rescale();
        g.normalize();
        carry->pend.clear();
        for (const Pend& e : g.pend) {
            uint32_t gm = e.omask;
            for (int b = 0; b < p.k; ++b)  // where the pass writes each local bit
                if (e.lmask & (1u << b)) gm |= 1u << p.q_out[b];
            carry->pend.push_back({gm, e.v});
        }
        carry->g = g.G;
    } else {
        g.flush_all();
        if (carry) {
            carry->pend.clear();
            carry->g = cplx(1.0, 0.0);
        }
    }
    if (hist) {
        // bin bit j is the j-th group qubit; in the store layout each is a register bit, a
        // thread bit (a lane bit when below 5) or a qubit outside the block
        uint32_t reg_gm = 0, lane_gm = 0;
        int reg_bin[R] = {};
        std::string rt = "0u";
        int tb = 0;
        std::vector<int> thread_rank((size_t)p.k, -1);
        for (int b = 0; b < p.k; ++b)
            if (!(g.regmask() & (1u << b))) thread_rank[(size_t)b] = tb++;
        int j = 0;
        for (int q = 0; q < qubits; ++q) {
            if (!(hist_mask & (1u << q))) continue;
            int lb = -1;
            for (int b = 0; b < p.k; ++b)
                if (p.q[b] == q) lb = b;
            if (lb < 0) {
                rt += " | (((outer >> " + std::to_string(q) + ") & 1u) << " + std::to_string(j) + ")";
            } else if (g.reg_of_local(lb) >= 0) {
                const int m = g.reg_of_local(lb);
                reg_gm |= 1u << m;
                reg_bin[m] = j;
            } else {
                const int r = thread_rank[(size_t)lb];
                rt += " | (((t >> " + std::to_string(r) + ") & 1u) << " + std::to_string(j) + ")";
                if (r < 5) lane_gm |= 1u << r;
            }
            ++j;
        }
        os << "{ const u32 hb = " << rt << ";\n";
        os << "const bool hw = (t & " << hexu(~lane_gm & 31u) << ") == 0u;\nconst int hwarp = (int)(t >> 5);\n";
        for (uint32_t pat = 0; pat < (uint32_t)NR; ++pat) {
            if ((pat & ~reg_gm) != 0) continue;
            uint32_t bin = 0;
            for (int m = 0; m < R; ++m)
                if ((pat >> m) & 1u) bin |= 1u << reg_bin[m];
            os << "{ double v = 0.0;\n";
            for (int i = 0; i < NR; ++i)
                if (((uint32_t)i & reg_gm) == pat)
                    os << "v += (double)" << g.X(i) << " * " << g.X(i) << " + (double)" << g.Y(i) << " * " << g.Y(i)
                       << ";\n";
            for (int l = 0; l < 5; ++l)
                if (!((lane_gm >> l) & 1u)) os << "v += __shfl_xor_sync(0xffffffffu, v, " << (1 << l) << ");\n";
            os << "if (hw) hacc[hwarp * " << hist_bins << " + (hb | " << hexu(bin) << ")] += v; }\n";
        }
        os << "}\n";
    }
    os << release;
    os << "{ const u32 g1 = outer | " << permute_expr("t", p.out_bit, p.k - R) << ";\n";
    for (int i = 0; i < NR; ++i) {
        uint32_t gi = 0;
        for (int m = 0; m < R; ++m)
            if ((i >> m) & 1) gi |= reg_out_g[m];
        os << "{ V v; v.x = " << g.X(i) << "; v.y = " << g.Y(i) << "; s[g1 | " << hexu(gi) << "] = v; }\n";
    }
    os << "}\n(void)base;\n}\n";
    if (teams) os << "if (team == 0u) qm_bar(3u, " << 2 * nt << "u);\n";  // team 1's last hand-over
    if (hist) {
        os << "__syncthreads();\n";
        os << "for (int k = t; k < " << hist_bins << "; k += " << nt << ") { double sum = 0.0;\n"
           << "  for (int w = 0; w < " << warps << "; ++w) sum += hacc[w * " << hist_bins << " + k];\n"
           << "  hist[u * " << hist_bins << " + k] = sum; }\n";
        os << "__syncthreads();\n}\n";
    }
    os << "}\n";

    std::ostringstream hd;
    hd << kPrelude;
    hd << "typedef " << (fp64 ? "double2" : "float2") << " V;\n";
    if (fp64)
        hd << "__device__ __forceinline__ u32 qm_swz(u32 j) { const u32 h = j >> 3; return j ^ ((h ^ (h >> 3) ^ (h >> 6) "
              "^ (h >> 9)) & 7u); }\n";
    else
        hd << "__device__ __forceinline__ u32 qm_swz(u32 j) { const u32 h = j >> 4; return j ^ ((h ^ (h >> 4) ^ (h >> 8)) "
              "& 15u); }\n";
    const size_t na = std::max<size_t>(1, g.aux.size());
    hd << "struct Aux { " << g.T << " v[" << na << "]; };\n";
    hd << "extern \"C\" __global__ void __launch_bounds__(" << nt * (teams ? 2 : 1) << ", " << minb
       << ") qm_pass(V* __restrict__ s0, const __grid_constant__ FusedLaunch P, const __grid_constant__ Aux A"
       << (hist ? ", double* __restrict__ hist" : "") << ") {\n";
    Generated out;
    // the constants travel as a kernel parameter (at most 32764 bytes with the launch record)
    if (g.aux.size() > kMaxAuxValues + 1000) return out;
    out.src = hd.str() + os.str();
    out.tiles = tiles;
    out.teams = teams ? 2 : 1;
    out.hist_bins = hist_bins;
    out.zero_start = zero_start;
    if (fp64) {
        std::vector<double> v(na, 0.0);
        std::copy(g.aux.begin(), g.aux.end(), v.begin());
        out.aux.resize(na * sizeof(double));
        std::memcpy(out.aux.data(), v.data(), out.aux.size());
    } else {
        std::vector<float> v(na, 0.0f);
        for (size_t i = 0; i < g.aux.size(); ++i) v[i] = (float)g.aux[i];
        out.aux.resize(na * sizeof(float));
        std::memcpy(out.aux.data(), v.data(), out.aux.size());
    }
    return out;
}

// Every pass of a plan: chained (phases carried from pass to pass, flushed by the last) or
// self-contained.
std::vector<Generated> generate_plan(const Plan& plan, bool chained) {
    const bool fp64 = plan.precision != QM_FP32;
    std::vector<Generated> out;
    out.reserve(plan.passes.size());
    Carry carry;
    const Fold fold = fold_plan(plan, chained);
    for (size_t i = 0; i < plan.passes.size(); ++i)
        out.push_back(generate(plan.passes[i], plan.ops, fold, plan.qubits, fp64, chained ? &carry : nullptr,
                               i + 1 == plan.passes.size(), i + 1 == plan.passes.size() ? plan.hist_mask : 0u,
                               i == 0 && plan.start_zero));
    return out;
}

// ---------------------------------------------------------------- compiled-kernel cache
struct Entry {
    cudaKernel_t kernel = nullptr;
    bool failed = false;
};

std::mutex g_cache_mu;
std::atomic<bool> g_self_contained{false};  // some plan compiled self-contained passes
std::unordered_map<std::string, Entry> g_cache;
std::atomic<int64_t> g_compiled{0}, g_failed{0}, g_launches{0};

// Compiles one source (without the cache lock held); returns null on failure.
cudaKernel_t compile_source(const std::string& src) {
    const Nvrtc& n = nvrtc();
    if (!n.ok) return nullptr;
    nvrtcProgram prog;
    if (n.create(&prog, src.c_str(), "qm_pass.cu", 0, nullptr, nullptr) != NVRTC_SUCCESS) return nullptr;
    const char* opts[] = {"--gpu-architecture=sm_100a", "--std=c++17", "--fmad=true", "-lineinfo"};
    const nvrtcResult rc = n.compile(prog, 4, opts);
    cudaKernel_t kernel = nullptr;
    if (rc == NVRTC_SUCCESS) {
        size_t size = 0;
        if (n.cubin_size(prog, &size) == NVRTC_SUCCESS && size > 0) {
            std::vector<char> cubin(size);
            if (n.cubin(prog, cubin.data()) == NVRTC_SUCCESS) {
                cudaLibrary_t lib = nullptr;
                if (cudaLibraryLoadData(&lib, cubin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0) == cudaSuccess &&
                    cudaLibraryGetKernel(&kernel, lib, src.find("qm_expect(") != std::string::npos ? "qm_expect" : "qm_pass") ==
                        cudaSuccess) {
                    int dev = 0, optin = 0;
                    if (cudaGetDevice(&dev) != cudaSuccess ||
                        cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess ||
                        cudaFuncSetAttribute(reinterpret_cast<const void*>(kernel),
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, optin) != cudaSuccess)
                        kernel = nullptr;
                } else {
                    kernel = nullptr;
                }
                cudaGetLastError();  // a failed load must not linger as the sticky last error
            }
        }
    }
    n.destroy(&prog);
    return kernel;
}

cudaKernel_t kernel_for(const std::string& src) {
    if (src.empty()) return nullptr;  // a pass whose constants do not fit a kernel parameter
    {
        std::lock_guard<std::mutex> lock(g_cache_mu);
        auto it = g_cache.find(src);
        if (it != g_cache.end()) return it->second.failed ? nullptr : it->second.kernel;
    }
    cudaKernel_t k = compile_source(src);
    std::lock_guard<std::mutex> lock(g_cache_mu);
    Entry& e = g_cache[src];
    if (!e.kernel && !e.failed) {
        e.kernel = k;
        e.failed = k == nullptr;
        (k ? g_compiled : g_failed)++;
    }
    return e.failed ? nullptr : e.kernel;
}

bool jit_enabled() { return kRegBits == 4 && nvrtc().ok; }

}  // namespace

namespace {

// Compiles the distinct sources in parallel; returns whether every one compiled.
bool compile_all(const std::vector<Generated>& gen) {
    std::vector<size_t> todo;
    {
        std::unordered_map<std::string, size_t> first;
        for (size_t i = 0; i < gen.size(); ++i)
            if (first.emplace(gen[i].src, i).second) todo.push_back(i);
    }
    int device = 0;
    cudaGetDevice(&device);
    std::atomic<size_t> next{0};
    const size_t workers = std::max<size_t>(1, std::min<size_t>(todo.size(), std::thread::hardware_concurrency()));
    std::vector<std::thread> pool;
    for (size_t w = 0; w < workers; ++w)
        pool.emplace_back([&]() {
            cudaSetDevice(device);
            for (size_t j; (j = next.fetch_add(1)) < todo.size();) kernel_for(gen[todo[j]].src);
        });
    for (auto& th : pool) th.join();
    bool all = true;
    for (const Generated& g : gen)
        if (!kernel_for(g.src)) all = false;
    return all;
}

void install(Plan& plan, std::vector<Generated>& gen, bool cached_only) {
    for (size_t i = 0; i < gen.size(); ++i) {
        const void* k = nullptr;
        if (cached_only) {
            std::lock_guard<std::mutex> lock(g_cache_mu);
            auto it = g_cache.find(gen[i].src);
            if (it != g_cache.end() && !it->second.failed) k = reinterpret_cast<const void*>(it->second.kernel);
        } else {
            k = reinterpret_cast<const void*>(kernel_for(gen[i].src));
        }
        plan.jit[i] = k;
        if (k) {
            plan.jit_aux[i] = std::move(gen[i].aux);
            plan.jit_tiles[i] = gen[i].tiles;
            plan.jit_teams[i] = gen[i].teams;
            plan.jit_hist_bins[i] = gen[i].hist_bins;
        }
    }
    plan.hist_fused = !gen.empty() && plan.jit.back() && gen.back().hist_bins > 0;
    plan.zero_fused = !gen.empty() && plan.jit.front() && gen.front().zero_start;
}

bool all_cached(const std::vector<Generated>& gen) {
    std::lock_guard<std::mutex> lock(g_cache_mu);
    for (const Generated& g : gen) {
        if (g.src.empty()) return false;
        auto it = g_cache.find(g.src);
        if (it == g_cache.end() || it->second.failed) return false;
    }
    return true;
}

}  // namespace

// Chained passes need every pass compiled; otherwise each pass is made self-contained and those
// that compile run compiled, the others on the interpreter.
void jit_prepare(Plan& plan) {
    plan.jit.assign(plan.passes.size(), nullptr);
    plan.jit_aux.assign(plan.passes.size(), {});
    plan.jit_tiles.assign(plan.passes.size(), 1);
    plan.jit_teams.assign(plan.passes.size(), 1);
    plan.jit_hist_bins.assign(plan.passes.size(), 0);
    plan.hist_fused = false;
    plan.zero_fused = false;
    if (!jit_enabled() || plan.passes.empty()) return;
    std::vector<Generated> gen = generate_plan(plan, true);
    if (compile_all(gen)) {
        install(plan, gen, false);
        return;
    }
    gen = generate_plan(plan, false);
    compile_all(gen);
    g_self_contained.store(true);
    install(plan, gen, false);
}

void jit_lookup(Plan& plan) {
    plan.jit.assign(plan.passes.size(), nullptr);
    plan.jit_aux.assign(plan.passes.size(), {});
    plan.jit_tiles.assign(plan.passes.size(), 1);
    plan.jit_teams.assign(plan.passes.size(), 1);
    plan.jit_hist_bins.assign(plan.passes.size(), 0);
    plan.hist_fused = false;
    plan.zero_fused = false;
    if (!jit_enabled() || plan.passes.empty()) return;
    {
        std::lock_guard<std::mutex> lock(g_cache_mu);
        if (g_cache.empty()) return;
    }
    std::vector<Generated> gen = generate_plan(plan, true);
    if (all_cached(gen)) {
        install(plan, gen, true);
        return;
    }
    // self-contained passes are only compiled when a chained plan failed to; until then there
    // is nothing to find and the generation (about a millisecond per plan) is skipped
    if (!g_self_contained.load()) return;
    gen = generate_plan(plan, false);
    install(plan, gen, true);
}

cudaError_t launch_plan_pass(const Plan& plan, size_t pass, void* amps, const FusedBatch* batch, cudaStream_t st) {
    const FusedPass& p = plan.passes[pass];
    const void* kernel = pass < plan.jit.size() && pass < plan.jit_aux.size() && pass < plan.jit_tiles.size() &&
                                 !plan.jit_aux[pass].empty()
                             ? plan.jit[pass]
                             : nullptr;
    if (!kernel) return launch_fused(amps, plan.qubits, plan.precision, p, plan.d_ops, batch, st);
    if (batch && (batch->states < 1 || batch->states > 65535)) return cudaErrorInvalidValue;
    FusedLaunch L = fused_launch_params(plan.qubits, p, plan.d_ops, batch);
    const bool fp64 = plan.precision != QM_FP32;
    const int hist_bins = pass < plan.jit_hist_bins.size() ? plan.jit_hist_bins[pass] : 0;
    if (hist_bins > 0 && (!batch || !batch->hist)) return cudaErrorInvalidValue;
    const size_t smem = ((size_t)(fp64 ? 16 : 8) * (size_t)plan.jit_tiles[pass] << p.k) +
                        sizeof(double) * (size_t)((1 << (p.k - R)) / 32) * (size_t)hist_bins +
                        (((size_t)p.op_count * sizeof(FusedOp) + 15) & ~size_t(15)) +
                        sizeof(double) * 8 * (size_t)L.table_slots;
    static const int sms = [] {
        int dev = 0, v = 0;
        if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
            return 0;
        return v;
    }();
    if (sms <= 0) return cudaErrorInvalidDevice;
    const int teams = pass < plan.jit_teams.size() ? plan.jit_teams[pass] : 1;
    const int threads = teams << (p.k - R);
    int per_sm = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    int64_t items = (int64_t)L.states << L.cta_shift;
    if (hist_bins > 0)  // work units are chunks of tiles (the joint-mass partial rows)
        items = (int64_t)L.states * (plan.qubits > 16 ? (int64_t)1 << (plan.qubits - 16) : 1);
    const int64_t grid = std::min<int64_t>(items, (int64_t)sms * per_sm);
    void* arg0 = amps;
    double* hist = batch ? batch->hist : nullptr;
    void* args[] = {&arg0, &L, const_cast<unsigned char*>(plan.jit_aux[pass].data()), &hist};
    e = cudaLaunchKernel(kernel, dim3((unsigned)grid), dim3((unsigned)threads), args, smem, st);
    if (e == cudaSuccess) ++g_launches;
    return e;
}

// ---------------------------------------------------------------- tiled expectation, compiled
// The tiled expectation kernel (qm_expect.cu) generated for one tile pass's term list: flip
// masks, pivots, phases and the tile-local Z-sign bits are constants, so a flip group's loop is
// two shared loads, the FP64 overlap and one add or subtract per term.  The reduction order and
// the partial-table layout are those of the generic kernel.
namespace {

uint32_t insert_zero(uint32_t v, int bit) {
    const uint32_t below = (1u << bit) - 1u;
    return (v & below) | ((v & ~below) << 1);
}

std::string generate_expect(int qubits, bool fp64, const TilePass& tp, const TileTerm* all_terms) {
    const int K = tp.k, NT = 1 << (K - R), WARPS = NT / 32;
    const int T = tp.term_count;
    const TileTerm* terms = all_terms + tp.term_begin;
    const int NCOL = T + 1;
    uint32_t thread_mask = 0, reg_g[R];
    for (int b = 0; b < K - R; ++b) thread_mask |= 1u << tp.q[b];
    for (int m = 0; m < R; ++m) reg_g[m] = 1u << tp.q[K - R + m];
    const uint32_t all = qubits >= 32 ? 0xffffffffu : ((1u << qubits) - 1u);
    const uint32_t outer_all = all & ~tp.block_mask;
    auto local_of = [&](uint32_t global) {
        uint32_t l = 0;
        for (int b = 0; b < K; ++b)
            if (global & (1u << tp.q[b])) l |= 1u << b;
        return l;
    };
    const uint32_t lo_mask = (1u << (K - R)) - 1u;
    int ndiag = 0;
    while (ndiag < T && terms[ndiag].flip_local == 0) ++ndiag;
    const bool wht = ndiag >= 3;

    std::ostringstream os;
    os << "typedef unsigned int u32;\ntypedef unsigned long long u64;\n";
    os << "typedef " << (fp64 ? "double2" : "float2") << " V;\n";
    os << "struct ExpLaunch { u32 outer_mask; int row_offset; int rows_per_state; int columns; int mass_column; int pad;\n"
          "  u64 state_stride; double* partials; };\n";
    os << "__device__ __forceinline__ u32 qm_deposit(u32 value, u32 mask) {\n"
          "  u32 out = 0;\n"
          "  while (mask) { const u32 low = mask & (0u - mask); if (value & 1u) out |= low; value >>= 1; mask ^= low; }\n"
          "  return out;\n}\n";
    os << "__device__ __forceinline__ double warp_sum(double v) {\n"
          "  for (int d = 16; d > 0; d >>= 1) v += __shfl_down_sync(0xffffffffu, v, d);\n  return v;\n}\n";
    // per-term constants of the final write
    os << "__constant__ int c_col[" << std::max(1, T) << "] = {";
    for (int k = 0; k < T; ++k) os << (k ? ", " : "") << terms[k].column;
    os << "};\n__constant__ u32 c_loc[" << std::max(1, T) << "] = {";
    for (int k = 0; k < T; ++k) os << (k ? ", " : "") << hexu(local_of(terms[k].sign & tp.block_mask));
    os << "};\n__constant__ u32 c_sout[" << std::max(1, T) << "] = {";
    for (int k = 0; k < T; ++k) os << (k ? ", " : "") << hexu(terms[k].sign & outer_all);
    os << "};\n";
    os << "extern \"C\" __global__ void __launch_bounds__(" << NT << ", " << std::max(1, 512 / NT)
       << ") qm_expect(const V* __restrict__ s, const __grid_constant__ ExpLaunch P) {\n";
    os << "extern __shared__ __align__(16) unsigned char smem_raw[];\n";
    os << "V* tile = reinterpret_cast<V*>(smem_raw);\n";
    os << "double* red = reinterpret_cast<double*>(smem_raw + " << ((fp64 ? 16 : 8) << K) << ");\n";
    os << "const u32 t = threadIdx.x;\nconst int warp = t >> 5, lane = t & 31;\n(void)warp; (void)lane;\n";
    os << "s += (u64)blockIdx.y * P.state_stride;\n";
    os << "const u32 outer = qm_deposit(blockIdx.x, P.outer_mask);\n";
    os << "{ const u32 g0 = outer | " << deposit_expr("t", thread_mask) << ";\n";
    for (int i = 0; i < NR; ++i) {
        uint32_t off = 0;
        for (int m = 0; m < R; ++m)
            if ((i >> m) & 1) off |= reg_g[m];
        os << "tile[t | " << hexu((uint32_t)i << (K - R)) << "] = s[g0 | " << hexu(off) << "];\n";
    }
    os << "}\n__syncthreads();\n";

    // flip groups (and diagonal terms when fewer than three), at most 8 terms per loop
    for (int k = wht ? ndiag : 0; k < T;) {
        const uint32_t F = terms[k].flip_local;
        int cnt = 1;
        while (cnt < 8 && k + cnt < T && terms[k + cnt].flip_local == F) ++cnt;
        bool paired = F != 0;
        for (int u = 0; u < cnt; ++u) {
            const uint32_t sl = local_of(terms[k + u].sign & tp.block_mask);
            if (((__builtin_popcount(F & sl) ^ terms[k + u].phase) & 1) != 0) paired = false;
        }
        os << "{\n";
        for (int u = 0; u < cnt; ++u) os << "double a" << u << " = 0.0;\n";
        auto term_add = [&](int u, uint32_t j_const, const char* ore, const char* oim) {
            const TileTerm& tt = terms[k + u];
            const uint32_t sl = local_of(tt.sign & tp.block_mask);
            const bool neg = (tt.phase == 1 || tt.phase == 2) ^ (__builtin_popcount(j_const & sl) & 1);
            os << "a" << u << (neg ? " -= " : " += ") << ((tt.phase & 1) ? oim : ore) << ";\n";
        };
        std::string jt;
        uint32_t jt_bits = lo_mask;  // local bits the run-time index part can hold
        if (paired) {
            const int pivot = 31 - __builtin_clz(F);
            if (pivot >= K - R) {
                jt = "t";
            } else {
                jt_bits = (lo_mask << 1) | 1u;  // the thread index with a zero inserted at the pivot
                const uint32_t below = (1u << pivot) - 1u;
                os << "const u32 jt = (t & " << hexu(below) << ") | ((t & " << hexu(~below & lo_mask) << ") << 1);\n";
                jt = "jt";
            }
            for (int r = 0; r < NR / 2; ++r) {
                const uint32_t c = insert_zero((uint32_t)(NT * r), pivot);
                os << "{ const V a = tile[" << jt << " | " << hexu(c) << "], b = tile[(" << jt << " | " << hexu(c) << ") ^ "
                   << hexu(F) << "];\n";
                os << "const double ar = a.x, ai = a.y, br = b.x, bi = b.y;\n";
                os << "const double ore = br * ar + bi * ai, oim = br * ai - bi * ar;\n";
                for (int u = 0; u < cnt; ++u) term_add(u, c, "ore", "oim");
                os << "}\n";
            }
        } else {
            jt = "t";
            for (int i = 0; i < NR; ++i) {
                const uint32_t c = (uint32_t)i << (K - R);
                os << "{ const V a = tile[t | " << hexu(c) << "];\nconst double ar = a.x, ai = a.y;\n";
                if (F == 0) {
                    os << "const double ore = ar * ar + ai * ai, oim = 0.0;\n";
                } else {
                    os << "const V b = tile[(t | " << hexu(c) << ") ^ " << hexu(F) << "];\nconst double br = b.x, bi = b.y;\n";
                    os << "const double ore = br * ar + bi * ai, oim = br * ai - bi * ar;\n";
                }
                for (int u = 0; u < cnt; ++u) term_add(u, c, "ore", "oim");
                os << "}\n";
            }
        }
        for (int u = 0; u < cnt; ++u) {
            const TileTerm& tt = terms[k + u];
            const uint32_t sl = local_of(tt.sign & tp.block_mask) & jt_bits;  // run-time part of the local sign
            const uint32_t so = tt.sign & outer_all;
            std::string par;
            if (sl) par = "__popc(" + jt + " & " + hexu(sl) + ")";
            if (so) par += std::string(par.empty() ? "" : " + ") + "__popc(outer & " + hexu(so) + ")";
            const char* scale = paired ? "2.0" : "1.0";
            if (par.empty())
                os << "{ const double v = warp_sum(" << scale << " * a" << u << ");\n";
            else
                os << "{ const double v = warp_sum(((" << par << ") & 1) ? -" << scale << " * a" << u << " : " << scale
                   << " * a" << u << ");\n";
            os << "if (lane == 0) red[warp * " << NCOL << " + " << (k + u) << "] = v; }\n";
        }
        os << "}\n";
        k += cnt;
    }
    if (tp.with_mass) {
        os << "{ double m = 0.0;\n";
        for (int i = 0; i < NR; ++i)
            os << "{ const V a = tile[t | " << hexu((uint32_t)i << (K - R)) << "]; m += (double)a.x * a.x + (double)a.y * a.y; }\n";
        os << "m = warp_sum(m);\nif (lane == 0) red[warp * " << NCOL << " + " << T << "] = m; }\n";
    }
    if (wht) {
        // Walsh-Hadamard transform of the tile's Born probabilities (as the generic kernel)
        os << "double* wbuf = reinterpret_cast<double*>(smem_raw);\n{\ndouble w[" << NR << "];\n";
        for (int i = 0; i < NR; ++i)
            os << "{ const V a = tile[t | " << hexu((uint32_t)i << (K - R)) << "]; w[" << i
               << "] = (double)a.x * a.x + (double)a.y * a.y; }\n";
        for (int m = 0; m < R; ++m)
            for (int i = 0; i < NR; ++i)
                if (!((i >> m) & 1))
                    os << "{ const double x = w[" << i << "], y = w[" << (i | (1 << m)) << "]; w[" << i << "] = x + y; w["
                       << (i | (1 << m)) << "] = x - y; }\n";
        for (int m = 0; m < 5; ++m) {
            os << "#pragma unroll\nfor (int i = 0; i < " << NR << "; ++i) { const double y = __shfl_xor_sync(0xffffffffu, w[i], "
               << (1 << m) << "); w[i] = ((lane >> " << m << ") & 1) ? y - w[i] : w[i] + y; }\n";
        }
        os << "__syncthreads();\n";
        os << "#pragma unroll\nfor (int i = 0; i < " << NR << "; ++i) wbuf[t | ((u32)i << " << (K - R) << ")] = w[i];\n";
        for (int m = 5; m < K - R; ++m) {
            os << "__syncthreads();\n#pragma unroll\nfor (int i = 0; i < " << NR << "; ++i) { const u32 j = t | ((u32)i << "
               << (K - R) << "); const double x = wbuf[j], y = wbuf[j ^ " << (1u << m) << "u]; w[i] = ((j >> " << m
               << ") & 1u) ? y - x : x + y; }\n";
            os << "__syncthreads();\n#pragma unroll\nfor (int i = 0; i < " << NR << "; ++i) wbuf[t | ((u32)i << " << (K - R)
               << ")] = w[i];\n";
        }
        os << "}\n";
    }
    os << "__syncthreads();\n";
    os << "const u64 row = (u64)blockIdx.y * P.rows_per_state + P.row_offset + blockIdx.x;\n";
    os << "for (int k = t; k < " << (T + (tp.with_mass ? 1 : 0)) << "; k += " << NT << ") {\n";
    os << "double sum = 0.0;\n";
    if (wht) {
        os << "if (k < " << ndiag << ") { sum = reinterpret_cast<const double*>(smem_raw)[c_loc[k]];\n"
              "  if (__popc(outer & c_sout[k]) & 1) sum = -sum;\n"
              "  P.partials[row * P.columns + c_col[k]] = sum; continue; }\n";
    }
    os << "for (int w = 0; w < " << WARPS << "; ++w) sum += red[w * " << NCOL << " + k];\n";
    os << "const int col = k < " << T << " ? c_col[k < " << T << " ? k : 0] : P.mass_column;\n";
    os << "P.partials[row * P.columns + col] = sum;\n}\n}\n";
    return os.str();
}

struct ExpLaunchHost {
    uint32_t outer_mask;
    int32_t row_offset, rows_per_state, columns, mass_column, pad;
    uint64_t state_stride;
    double* partials;
};
static_assert(sizeof(ExpLaunchHost) == 40, "ExpLaunch layout is mirrored in the generated source");

}  // namespace

void jit_prepare_tiles(TilePlan& tp, int qubits, int precision) {
    tp.jit.assign(tp.passes.size(), nullptr);
    if (!jit_enabled() || tp.passes.empty()) return;
    std::vector<Generated> gen(tp.passes.size());
    for (size_t i = 0; i < tp.passes.size(); ++i)
        gen[i].src = generate_expect(qubits, precision != QM_FP32, tp.passes[i], tp.terms.data());
    compile_all(gen);
    for (size_t i = 0; i < gen.size(); ++i) tp.jit[i] = reinterpret_cast<const void*>(kernel_for(gen[i].src));
}

cudaError_t launch_expect_tile_jit(const void* kernel, const void* amps, int qubits, int precision, const TilePass& tp,
                                   int states, uint64_t state_stride, double* partials, int columns, int rows_per_state,
                                   int mass_column, cudaStream_t st) {
    if (states < 1 || states > 65535) return cudaErrorInvalidValue;
    ExpLaunchHost L{};
    const uint32_t all = qubits >= 32 ? 0xffffffffu : ((1u << qubits) - 1u);
    L.outer_mask = all & ~tp.block_mask;
    L.row_offset = tp.row_offset;
    L.rows_per_state = rows_per_state;
    L.columns = columns;
    L.mass_column = mass_column;
    L.state_stride = state_stride;
    L.partials = partials;
    const int K = tp.k;
    const size_t smem = ((size_t)(precision == QM_FP32 ? 8 : 16) << K) +
                        sizeof(double) * (size_t)((1 << (K - R)) / 32) * (size_t)(tp.term_count + 1);
    const void* arg0 = amps;
    void* args[] = {&arg0, &L};
    dim3 grid(1u << (qubits - K), (unsigned)states);
    const cudaError_t e = cudaLaunchKernel(kernel, grid, dim3(1u << (K - R)), args, smem, st);
    if (e == cudaSuccess) ++g_launches;
    return e;
}

}  // namespace qm

extern "C" int32_t qm_jit_expect_source(int32_t qubits, int32_t precision, const qm_pauli_term* terms, int32_t count,
                                        int32_t pass, char* buffer, size_t size, size_t* length) {
    using namespace qm;
    if (qubits < 9 || qubits > 30) return fail(QM_E_RANGE, "tiled expectations need 9 to 30 qubits");
    if (precision != QM_FP64 && precision != QM_FP32) return fail(QM_E_RANGE, "unknown precision");
    if (count < 0 || (count > 0 && !terms)) return fail(QM_E_ARG, "bad term list");
    TilePlan tp;
    std::string err;
    if (!plan_tiles(qubits, precision, terms, count, tp, err)) return fail(QM_E_ARG, err);
    if (pass < 0 || (size_t)pass >= tp.passes.size()) return fail(QM_E_RANGE, "pass index out of range");
    const std::string src = generate_expect(qubits, precision != QM_FP32, tp.passes[(size_t)pass], tp.terms.data());
    if (length) *length = src.size();
    if (buffer && size) {
        const size_t n = std::min(size - 1, src.size());
        std::memcpy(buffer, src.data(), n);
        buffer[n] = '\0';
    }
    return QM_OK;
}

extern "C" int32_t qm_jit_info(int32_t* available, int64_t* kernels, int64_t* failed, int64_t* launches) {
    if (available) *available = qm::jit_enabled() ? 1 : 0;
    if (kernels) *kernels = qm::g_compiled.load();
    if (failed) *failed = qm::g_failed.load();
    if (launches) *launches = qm::g_launches.load();
    return QM_OK;
}

// Source of the compiled kernel of one pass of a plan made for these gates (inspection and tests).
// The constant parameter block (kernel parameter A) of the same pass, as bytes.
extern "C" int32_t qm_jit_constants(int32_t qubits, int32_t precision, const qm_gate* gates, int32_t count,
                                    int32_t fusion_width, int32_t pass, void* buffer, size_t size, size_t* length) {
    using namespace qm;
    int32_t rc = validate_prepared_gates(gates, count, qubits);
    if (rc) return rc;
    Plan plan;
    std::string err;
    std::vector<qm_gate> list(gates, gates + count);
    if (!plan_fused(list, qubits, precision, fusion_width, plan, err)) return fail(QM_E_ARG, "planner: " + err);
    if (pass < 0 || (size_t)pass >= plan.passes.size()) return fail(QM_E_RANGE, "pass index out of range");
    const std::vector<unsigned char> aux = generate_plan(plan, true)[(size_t)pass].aux;
    if (length) *length = aux.size();
    if (buffer && size) std::memcpy(buffer, aux.data(), std::min(size, aux.size()));
    return QM_OK;
}

extern "C" int32_t qm_jit_source(int32_t qubits, int32_t precision, const qm_gate* gates, int32_t count,
                                 int32_t fusion_width, int32_t pass, char* buffer, size_t size, size_t* length) {
    using namespace qm;
    int32_t rc = validate_prepared_gates(gates, count, qubits);
    if (rc) return rc;
    Plan plan;
    std::string err;
    std::vector<qm_gate> list(gates, gates + count);
    if (!plan_fused(list, qubits, precision, fusion_width, plan, err)) return fail(QM_E_ARG, "planner: " + err);
    if (pass < 0 || (size_t)pass >= plan.passes.size()) return fail(QM_E_RANGE, "pass index out of range");
    const std::string src = generate_plan(plan, true)[(size_t)pass].src;
    if (length) *length = src.size();
    if (buffer && size) {
        const size_t n = std::min(size - 1, src.size());
        std::memcpy(buffer, src.data(), n);
        buffer[n] = '\0';
    }
    return QM_OK;
}
