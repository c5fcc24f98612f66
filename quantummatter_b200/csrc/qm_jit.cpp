// qm_jit.cpp -- fused passes compiled for their own op sequence (NVRTC, sm_100a).
//
// k_fused interprets a pass program: for every op it decodes the record, selects the register
// bit through a switch and, for an X or SWAP on register bits, moves the amplitudes between
// registers.  Here a pass's op sequence is turned into straight-line CUDA C++ and compiled once
// with NVRTC for sm_100a.  The generated kernel takes the same parameters and shared-memory
// layout as k_fused (the program is still staged, and every coefficient is still read from it
// or from the batch table), so one compiled kernel serves every pass with the same structure
// whatever its angles.  What the generation fixes at compile time:
//   - the register of every op, and the register pairs it touches;
//   - the control predicates: register bits select pairs at compile time, thread bits become
//     one uniform test per op, bits outside the block one test per work item;
//   - an X, CNOT or SWAP acting on register bits only renames registers: no instruction;
//   - the load, store and shared-memory exchange addresses as constants and bit deposits.
// NVRTC is loaded at run time; without it every pass runs on k_fused, the GPU interpreter.
#include <cuda_runtime.h>
#include <dlfcn.h>
#include <nvrtc.h>

#include <algorithm>
#include <atomic>
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
static_assert(sizeof(FusedLaunch) == 112, "FusedLaunch layout is mirrored in the generated source");
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
)SRC";

struct Gen {
    std::ostringstream os;
    bool fp64;
    int K;
    int phys[NR];
    uint32_t pm[R];  // local masks of the register bits in the current layout
    const char* T;

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
    std::string base_expr() const { return deposit_expr("t", ((1u << K) - 1u) & ~regmask()); }

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

    void stage(const int8_t* pos) {
        os << "{ const u32 sb = qm_swz(base);\n__syncthreads();\n";
        for (int i = 0; i < NR; ++i) {
            os << "{ V v; v.x = " << X(i) << "; v.y = " << Y(i) << "; tile[sb ^ " << hexu(const_slot(i)) << "] = v; }\n";
        }
        set_layout(pos);
        for (int i = 0; i < NR; ++i) phys[i] = i;
        os << "base = " << base_expr() << ";\n";
        os << "const u32 sn = qm_swz(base);\n__syncthreads();\n";
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
                negate(m);
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

    void op(int o, const FusedOp& op) {
        uint32_t rm, tb;
        split(op.cmask_local, rm, tb);
        switch (op.code) {
        case OP_MATRIX:
        case OP_MATRIX_REAL: {
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
        case OP_NEGATE: negate(op); break;
        default: break;
        }
    }
};

// The whole source of one pass's kernel; structurally equal passes give the same text.
std::string generate(const FusedPass& p, const std::vector<FusedOp>& plan_ops, bool fp64) {
    Gen g;
    g.fp64 = fp64;
    g.K = p.k;
    g.T = fp64 ? "double" : "float";
    for (int i = 0; i < NR; ++i) g.phys[i] = i;
    g.set_layout(p.reg_in);
    uint32_t thread_in = 0, thread_out = 0, reg_in_local = 0, reg_out_local = 0;
    uint32_t reg_in_g[R], reg_out_g[R];
    for (int m = 0; m < R; ++m) {
        reg_in_local |= 1u << p.reg_in[m];
        reg_out_local |= 1u << p.reg_out[m];
        reg_in_g[m] = 1u << p.q[p.reg_in[m]];
        reg_out_g[m] = 1u << p.q[p.reg_out[m]];
    }
    for (int b = 0; b < p.k; ++b) {
        if (!(reg_in_local & (1u << b))) thread_in |= 1u << p.q[b];
        if (!(reg_out_local & (1u << b))) thread_out |= 1u << p.q[b];
    }
    const int nt = 1 << (p.k - R);
    // 128 registers per thread: two 256-thread blocks per SM (complex128, 12 qubits), one
    // 512-thread block (complex64, 13 qubits); fewer would spill the 16 amplitudes
    const int minb = (fp64 && p.k == 12) ? 2 : 1;
    const size_t tile_bytes = (size_t)(fp64 ? 16 : 8) << p.k;
    const size_t prog_bytes = ((size_t)p.op_count * sizeof(FusedOp) + 15) & ~size_t(15);
    bool tabled = false;
    for (int o = 0; o < p.op_count; ++o)
        if (plan_ops[(size_t)(p.op_begin + o)].flags & kOpTable) tabled = true;
    std::ostringstream& os = g.os;
    os << kPrelude;
    os << "typedef " << (fp64 ? "double2" : "float2") << " V;\n";
    if (fp64)
        os << "__device__ __forceinline__ u32 qm_swz(u32 j) { const u32 h = j >> 3; return j ^ ((h ^ (h >> 3) ^ (h >> 6) "
              "^ (h >> 9)) & 7u); }\n";
    else
        os << "__device__ __forceinline__ u32 qm_swz(u32 j) { const u32 h = j >> 4; return j ^ ((h ^ (h >> 4) ^ (h >> 8)) "
              "& 15u); }\n";
    os << "extern \"C\" __global__ void __launch_bounds__(" << nt << ", " << minb
       << ") qm_pass(V* __restrict__ s0, const __grid_constant__ FusedLaunch P) {\n";
    os << "extern __shared__ __align__(16) unsigned char smem_raw[];\n";
    os << "V* tile = reinterpret_cast<V*>(smem_raw);\n";
    os << "FusedOp* prog = reinterpret_cast<FusedOp*>(smem_raw + " << tile_bytes << ");\n";
    os << "double* table = reinterpret_cast<double*>(smem_raw + " << (tile_bytes + prog_bytes) << ");\n";
    os << "const u32 t = threadIdx.x;\n";
    os << "{ const uint2* src = reinterpret_cast<const uint2*>(P.ops); uint2* dst = reinterpret_cast<uint2*>(prog);\n"
       << "  for (int i = t; i < " << p.op_count * (int)(sizeof(FusedOp) / 8) << "; i += " << nt
       << ") dst[i] = __ldg(src + i); }\n";
    os << "const long long total = (long long)P.states << P.cta_shift;\n";
    os << "const u32 cta_mask = (1u << P.cta_shift) - 1u;\n";
    os << "int current = -1;\n";
    os << "for (long long item = blockIdx.x; item < total; item += gridDim.x) {\n";
    os << "const int b = (int)(item >> P.cta_shift);\nconst u32 cta = (u32)item & cta_mask;\n__syncthreads();\n";
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
    os << "{ const u32 g0 = outer | " << deposit_expr("t", thread_in) << ";\n";
    for (int i = 0; i < NR; ++i) {
        uint32_t gi = 0;
        for (int m = 0; m < R; ++m)
            if ((i >> m) & 1) gi |= reg_in_g[m];
        os << "{ const V v = s[g0 | " << hexu(gi) << "]; x" << i << " = v.x; y" << i << " = v.y; }\n";
    }
    os << "}\n";
    os << "u32 base = " << g.base_expr() << ";\n";
    for (int o = 0; o < p.op_count; ++o) {
        const FusedOp& op = plan_ops[(size_t)(p.op_begin + o)];
        if (op.code == OP_STAGE) {
            g.stage(op.reg_pos);
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
    os << "{ const u32 g1 = outer | " << deposit_expr("t", thread_out) << ";\n";
    for (int i = 0; i < NR; ++i) {
        uint32_t gi = 0;
        for (int m = 0; m < R; ++m)
            if ((i >> m) & 1) gi |= reg_out_g[m];
        os << "{ V v; v.x = " << g.X(i) << "; v.y = " << g.Y(i) << "; s[g1 | " << hexu(gi) << "] = v; }\n";
    }
    os << "}\n(void)base;\n}\n}\n";
    return os.str();
}

// ---------------------------------------------------------------- compiled-kernel cache
struct Entry {
    cudaKernel_t kernel = nullptr;
    bool failed = false;
};

std::mutex g_cache_mu;
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
                    cudaLibraryGetKernel(&kernel, lib, "qm_pass") == cudaSuccess) {
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

void jit_prepare(Plan& plan) {
    plan.jit.assign(plan.passes.size(), nullptr);
    if (!jit_enabled() || plan.passes.empty()) return;
    const bool fp64 = plan.precision != QM_FP32;
    std::vector<std::string> src(plan.passes.size());
    for (size_t i = 0; i < plan.passes.size(); ++i) src[i] = generate(plan.passes[i], plan.ops, fp64);
    // compile the distinct sources in parallel
    std::vector<size_t> todo;
    {
        std::unordered_map<std::string, size_t> first;
        for (size_t i = 0; i < src.size(); ++i)
            if (first.emplace(src[i], i).second) todo.push_back(i);
    }
    int device = 0;
    cudaGetDevice(&device);
    std::atomic<size_t> next{0};
    const size_t workers = std::max<size_t>(1, std::min<size_t>(todo.size(), std::thread::hardware_concurrency()));
    std::vector<std::thread> pool;
    for (size_t w = 0; w < workers; ++w)
        pool.emplace_back([&]() {
            cudaSetDevice(device);
            for (size_t j; (j = next.fetch_add(1)) < todo.size();) kernel_for(src[todo[j]]);
        });
    for (auto& th : pool) th.join();
    for (size_t i = 0; i < src.size(); ++i) plan.jit[i] = reinterpret_cast<const void*>(kernel_for(src[i]));
}

void jit_lookup(Plan& plan) {
    plan.jit.assign(plan.passes.size(), nullptr);
    if (!jit_enabled() || plan.passes.empty()) return;
    {
        std::lock_guard<std::mutex> lock(g_cache_mu);
        if (g_cache.empty()) return;
    }
    const bool fp64 = plan.precision != QM_FP32;
    std::lock_guard<std::mutex> lock(g_cache_mu);
    for (size_t i = 0; i < plan.passes.size(); ++i) {
        auto it = g_cache.find(generate(plan.passes[i], plan.ops, fp64));
        if (it != g_cache.end() && !it->second.failed) plan.jit[i] = reinterpret_cast<const void*>(it->second.kernel);
    }
}

cudaError_t launch_plan_pass(const Plan& plan, size_t pass, void* amps, const FusedBatch* batch, cudaStream_t st) {
    const FusedPass& p = plan.passes[pass];
    const void* kernel = pass < plan.jit.size() ? plan.jit[pass] : nullptr;
    if (!kernel) return launch_fused(amps, plan.qubits, plan.precision, p, plan.d_ops, batch, st);
    if (batch && (batch->states < 1 || batch->states > 65535)) return cudaErrorInvalidValue;
    FusedLaunch L = fused_launch_params(plan.qubits, p, plan.d_ops, batch);
    const bool fp64 = plan.precision != QM_FP32;
    const size_t smem = ((size_t)(fp64 ? 16 : 8) << p.k) + (((size_t)p.op_count * sizeof(FusedOp) + 15) & ~size_t(15)) +
                        sizeof(double) * 8 * (size_t)L.table_slots;
    static const int sms = [] {
        int dev = 0, v = 0;
        if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
            return 0;
        return v;
    }();
    if (sms <= 0) return cudaErrorInvalidDevice;
    const int threads = 1 << (p.k - R);
    int per_sm = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    const int64_t items = (int64_t)L.states << L.cta_shift;
    const int64_t grid = std::min<int64_t>(items, (int64_t)sms * per_sm);
    void* arg0 = amps;
    void* args[] = {&arg0, &L};
    e = cudaLaunchKernel(kernel, dim3((unsigned)grid), dim3((unsigned)threads), args, smem, st);
    if (e == cudaSuccess) ++g_launches;
    return e;
}

}  // namespace qm

extern "C" int32_t qm_jit_info(int32_t* available, int64_t* kernels, int64_t* failed, int64_t* launches) {
    if (available) *available = qm::jit_enabled() ? 1 : 0;
    if (kernels) *kernels = qm::g_compiled.load();
    if (failed) *failed = qm::g_failed.load();
    if (launches) *launches = qm::g_launches.load();
    return QM_OK;
}

// Source of the compiled kernel of one pass of a plan made for these gates (inspection and tests).
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
    const std::string src = generate(plan.passes[(size_t)pass], plan.ops, precision != QM_FP32);
    if (length) *length = src.size();
    if (buffer && size) {
        const size_t n = std::min(size - 1, src.size());
        std::memcpy(buffer, src.data(), n);
        buffer[n] = '\0';
    }
    return QM_OK;
}
