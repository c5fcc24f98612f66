// qm_planner.cpp -- gate-fusion planner of libqmb200.so.
//
// Turns an ordered list of prepared gates into fused passes for qm_fused.cu.  The
// reference executes one launch per non-identity gate (CudaStateVectorBackend.cs:145-160)
// and, on the CPU, reuses tiles only across adjacent same-target uncontrolled gates
// (ParallelCpuStateVectorBackend.cs:109-181).  Here a pass may hold any gates whose
// non-diagonal targets fit in the pass's block of k qubits, in any order the gates'
// commutation allows:
//   * a gate acts non-diagonally ("x role") on its target (and both SWAP operands) and
//     diagonally ("z role") on its controls; a diagonal gate is z role on every qubit;
//   * two gates commute when every qubit they share is z role in both (both are then
//     block-diagonal in the shared qubits' computational basis);
//   * a gate may move ahead of a skipped gate only if they commute.
// Diagonal gates never need block or register space: their phase is a function of the
// global index, which every amplitude knows.
// Plans without per-state coefficients also relabel qubits: a pass may write its block back
// with the qubits permuted among the block's index bits, so that the lowest bits (the run every
// pass reads whole) hold the qubits the next pass can use best; the last passes restore the order.
// Such a plan is kept only when it needs fewer passes than the plain one.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "qm_internal.h"

namespace qm {

namespace {

struct GInfo {
    qm_gate g;
    int32_t slot;    // batch-table coefficient slot, -1 for constant coefficients
    bool diag;
    uint32_t touch;  // every qubit the gate reads
    uint32_t xmask;  // qubits acted on non-diagonally
    uint32_t zmask;  // qubits acted on diagonally
    uint32_t need;   // qubits that must be register bits
};

inline int popc(uint32_t x) { return __builtin_popcount(x); }

GInfo classify(const qm_gate& g) {
    GInfo gi{};
    gi.g = g;
    gi.slot = -1;
    uint32_t tb = 1u << g.target;
    uint32_t sb = g.kernel == QM_KERNEL_SWAP ? (1u << g.swap_control) : 0u;
    gi.touch = tb | sb | g.control_mask;
    if (g.kernel == QM_KERNEL_DIAGONAL) {
        gi.diag = true;
        gi.xmask = 0;
        gi.zmask = gi.touch;
        gi.need = 0;
    } else {
        gi.diag = false;
        gi.xmask = tb | sb;
        gi.zmask = g.control_mask;
        gi.need = tb | sb;
    }
    return gi;
}

inline bool blocked(const GInfo& g, uint32_t bx, uint32_t bz) { return (g.touch & bx) || (g.xmask & bz); }

// a gate's qubits renamed by a permutation of the index bits
void remap_gate(GInfo& gi, const int* perm) {
    qm_gate g = gi.g;
    g.target = perm[g.target];
    uint32_t cm = 0;
    for (int q = 0; q < 32; ++q)
        if (g.control_mask & (1u << q)) cm |= 1u << perm[q];
    g.control_mask = cm;
    if (g.kernel == QM_KERNEL_SWAP) g.swap_control = perm[g.swap_control];
    const int32_t slot = gi.slot;
    gi = classify(g);
    gi.slot = slot;
}

inline bool is_exact(const double* v, double re, double im) { return v[0] == re && v[1] == im; }

}  // namespace

DevGate to_dev_gate(const qm_gate& g) {
    DevGate d{};
    d.kernel = g.kernel;
    d.target = g.target;
    d.target_bit = 1u << g.target;
    d.control_mask = g.control_mask;
    d.swap_control = g.swap_control;
    d.swap_bit = g.kernel == QM_KERNEL_SWAP ? (1u << g.swap_control) : 0u;
    d.a_is_one = is_exact(g.a, 1.0, 0.0);
    d.d_is_one = is_exact(g.d, 1.0, 0.0);
    std::memcpy(d.a, g.a, sizeof d.a);
    std::memcpy(d.b, g.b, sizeof d.b);
    std::memcpy(d.c, g.c, sizeof d.c);
    std::memcpy(d.d, g.d, sizeof d.d);
    return d;
}

// 12 qubits for both precisions: two 256-thread blocks per SM overlap better than one block of
// 13 (complex64), which saves few passes
int default_block_qubits(int qubits, int precision) {
    (void)precision;
    return std::min(12, qubits);
}

namespace {

bool relabel_enabled() {
    static const bool on = [] {
        const char* e = std::getenv("QM_RELABEL");
        return !(e && e[0] == '0');
    }();
    return on;
}

bool plan_fused_with(const std::vector<qm_gate>& gates, int qubits, int precision, int width, Plan& plan,
                     std::string& error, const std::vector<int32_t>* slots, bool allow_relabel) {
    plan.qubits = qubits;
    plan.precision = precision;
    plan.passes.clear();
    plan.ops.clear();
    plan.gates.clear();
    plan.planned_bytes = 0;
    plan.launches = 0;
    const int64_t elem = precision == QM_FP32 ? 8 : 16;
    const int64_t n = int64_t(1) << qubits;

    if (width >= 2 && width <= 8) {
        if (slots) {
            error = "batched plans need a fused block of at least 9 qubits";
            return false;
        }
        if (width > kDenseMaxQubits) {
            error = "fusion width must be 0, 1, 2..6 (dense fused gates) or 9..14 (fused blocks)";
            return false;
        }
        return plan_dense(gates, qubits, precision, width, plan, error);
    }
    const int kmax = precision == QM_FP32 ? 13 : 12;
    int k = width <= 0 ? default_block_qubits(qubits, precision) : std::min(width, kmax);
    k = std::min(k, qubits);
    // Per-gate path: requested explicitly (width 1) or the state is too small for a block
    // of at least 9 qubits (32 threads of 16 registers).
    if (width == 1 || k < 9) {
        if (slots) {
            error = "batched plans need a fused block of at least 9 qubits";
            return false;
        }
        plan.width = 1;
        for (const qm_gate& g : gates) {
            if (g.kernel == QM_KERNEL_IDENTITY) continue;
            DevGate d = to_dev_gate(g);
            if (d.kernel == QM_KERNEL_DIAGONAL && d.a_is_one && d.d_is_one) continue;
            plan.gates.push_back(d);
            int active = popc(d.target_bit | d.control_mask | d.swap_bit);
            int64_t pairs = n >> active;
            int64_t touched = 2 * pairs;
            if (d.kernel == QM_KERNEL_DIAGONAL && (d.a_is_one || d.d_is_one)) touched = pairs;
            plan.planned_bytes += 2 * touched * elem;
        }
        plan.launches = (int32_t)plan.gates.size();
        return true;
    }
    plan.width = k;

    std::vector<GInfo> remaining;
    remaining.reserve(gates.size());
    for (size_t gi = 0; gi < gates.size(); ++gi) {
        const qm_gate& g = gates[gi];
        const int32_t slot = slots ? (*slots)[gi] : -1;
        if (g.kernel == QM_KERNEL_IDENTITY) continue;
        if (slot < 0 && g.kernel == QM_KERNEL_DIAGONAL && is_exact(g.a, 1.0, 0.0) && is_exact(g.d, 1.0, 0.0)) continue;
        if (g.kernel == QM_KERNEL_SWAP && (g.swap_control < 0 || g.swap_control == g.target)) {
            error = "swap operands must be distinct";
            return false;
        }
        if (slot >= 0 && g.kernel != QM_KERNEL_MATRIX && g.kernel != QM_KERNEL_HADAMARD &&
            g.kernel != QM_KERNEL_DIAGONAL) {
            error = "only matrix and diagonal gates can take per-state coefficients";
            return false;
        }
        if (slot >= 0 && (slot & kSlotBranch) && (g.kernel != QM_KERNEL_MATRIX || g.control_mask != 0)) {
            error = "a noise branch is an uncontrolled matrix placeholder";
            return false;
        }
        GInfo info = classify(g);
        info.slot = slot;
        remaining.push_back(info);
    }

    // Low qubits always in the block: 8 complex128 or 16 complex64 = one 128-byte run.
    const int low_bits = precision == QM_FP32 ? 4 : 3;
    const uint32_t low_mask = (1u << low_bits) - 1u;

    // Relabeling (plans without per-state coefficients): a pass may write its tile back with the
    // block's qubits permuted among the block's index bits.  Index bits 0..low_bits-1 (the run
    // every pass reads whole) then hold the qubits the next pass can use best, found by trying
    // every choice against the next pass's greedy absorption, and the remaining gates are
    // renamed to match.  Blocks then follow the circuit's light cone instead of carrying qubits
    // 0..low_bits-1 through every pass.  `at[b]` is the qubit held at index bit b; the last
    // passes put every qubit back at its own bit.
    const bool relabel = allow_relabel && !slots && qubits > k;
    const uint32_t all_qubits = qubits >= 32 ? 0xffffffffu : (1u << qubits) - 1u;
    int at[32];
    for (int q = 0; q < 32; ++q) at[q] = q;
    int perm[32];
    int lane_pos[8];

    auto build_pass = [&](uint32_t Q, const std::vector<GInfo>& absorbed) -> bool {
            FusedPass pass{};
            pass.k = k;
            pass.block_mask = Q;
            int local_of[32];
            for (int i = 0; i < 32; ++i) local_of[i] = -1;
            int nb = 0;
            for (int q = 0; q < qubits; ++q)
                if (Q & (1u << q)) {
                    local_of[q] = nb;
                    pass.q[nb++] = q;
                }
            for (int b = 0; b < 16; ++b) pass.q_out[b] = pass.out_bit[b] = -1;
            for (int b = 0; b < k; ++b) pass.q_out[b] = (int8_t)perm[pass.q[b]];
            // lanes: the local bits whose qubits go to index bits 0..low_bits-1, in that order; they
            // must be the lowest thread ranks of the store layout (the coalesced run)
            uint32_t lane_mask = 0, lane_code = 0;
            bool lanes_needed = false;
            for (int r = 0; r < low_bits; ++r) {
                const int lb = local_of[lane_pos[r]];
                lane_mask |= 1u << lb;
                lane_code |= (uint32_t)lb << (4 + 4 * r);
                if (lb != r) lanes_needed = true;
            }
            lane_code |= (uint32_t)low_bits;
            pass.op_begin = (int32_t)plan.ops.size();
            auto to_local = [&](uint32_t global) {
                uint32_t l = 0;
                for (int q = 0; q < qubits; ++q)
                    if (global & (1u << q)) l |= 1u << local_of[q];
                return l;
            };

            // 1) split the pass into stages: each stage holds gates whose register needs fit in
            //    kRegBits qubits, in commutation-respecting order
            std::vector<std::vector<GInfo>> stage_gates;
            std::vector<uint32_t> stage_need;  // local bits
            std::vector<uint32_t> stage_soft;  // local bits worth holding (controls of X gates)
            {
                std::vector<GInfo> pending = absorbed;
                while (!pending.empty()) {
                    uint32_t P = 0, sbx = 0, sbz = 0;
                    std::vector<GInfo> mine, later;
                    for (const GInfo& g : pending) {
                        if (!blocked(g, sbx, sbz)) {
                            if (g.diag) {
                                mine.push_back(g);
                                continue;
                            }
                            uint32_t np = P | g.need;
                            if (popc(np) <= kRegBits) {
                                P = np;
                                mine.push_back(g);
                                continue;
                            }
                        }
                        later.push_back(g);
                        sbx |= g.xmask;
                        sbz |= g.zmask;
                    }
                    // controls of X gates are worth holding in registers too: the X then becomes
                    // a fixed register permutation
                    uint32_t soft = 0;
                    for (const GInfo& g : mine)
                        if (g.g.kernel == QM_KERNEL_EXCHANGE) soft |= g.g.control_mask & Q;
                    stage_gates.push_back(mine);
                    stage_need.push_back(to_local(P));
                    stage_soft.push_back(to_local(soft) & ~((1u << low_bits) - 1u));
                    pending.swap(later);
                }
            }
            // 2) register layouts: keep the current layout when it already covers a stage's
            //    needs; otherwise take the needs, then the next stages' needs (so the following
            //    stage may not need a change), then the current layout, then the highest bits.
            //    Low local bits (the coalescing run) are never used as filler.
            const uint32_t low_local = (1u << low_bits) - 1u;
            const uint32_t canonical = ((1u << kRegBits) - 1u) << (k - kRegBits);
            auto fill = [&](uint32_t need, size_t from, uint32_t current) {
                uint32_t l = need;
                if (from >= 1 && from - 1 < stage_soft.size()) {
                    uint32_t soft = stage_soft[from - 1] & ~l;
                    for (int b = 0; b < k && popc(l) < kRegBits; ++b)
                        if (soft & (1u << b)) l |= 1u << b;
                }
                for (size_t s = from; s < stage_need.size() && popc(l) < kRegBits; ++s) {
                    uint32_t extra = stage_need[s] & ~l & ~low_local;
                    for (int b = 0; b < k && popc(l) < kRegBits; ++b)
                        if (extra & (1u << b)) l |= 1u << b;
                }
                // relabeling passes keep their lanes off the filler, so that the last layout can
                // take the lane order without one more exchange
                const uint32_t avoid = low_local | (lanes_needed ? lane_mask : 0u);
                for (int b = k - 1; b >= 0 && popc(l) < kRegBits; --b)
                    if ((current & (1u << b)) && !(avoid & (1u << b))) l |= 1u << b;
                for (int b = k - 1; b >= 0 && popc(l) < kRegBits; --b)
                    if (!(avoid & (1u << b))) l |= 1u << b;
                for (int b = k - 1; b >= 0 && popc(l) < kRegBits; --b)
                    if (!(low_local & (1u << b))) l |= 1u << b;
                return l;
            };
            auto emit_stage = [&](uint32_t layout) {
                FusedOp st{};
                st.code = OP_STAGE;
                st.reg = st.reg2 = st.local = -1;
                int m = 0;
                for (int b = 0; b < k; ++b)
                    if (layout & (1u << b)) st.reg_pos[m++] = (int8_t)b;
                plan.ops.push_back(st);
            };
            auto set_regs = [&](int8_t* dst, uint32_t layout) {
                int m = 0;
                for (int b = 0; b < k; ++b)
                    if (layout & (1u << b)) dst[m++] = (int8_t)b;
            };
            uint32_t layout = fill(stage_need.empty() ? 0 : stage_need[0], 1, canonical);
            int stages = 1;
            if (layout & low_local) {
                set_regs(pass.reg_in, canonical);
                emit_stage(layout);
                ++stages;
            } else {
                set_regs(pass.reg_in, layout);
            }
            for (size_t si = 0; si < stage_gates.size(); ++si) {
                if ((stage_need[si] & ~layout) != 0) {
                    layout = fill(stage_need[si], si + 1, layout);
                    emit_stage(layout);
                    ++stages;
                }
                int reg_of_local[32];
                for (int i = 0; i < 32; ++i) reg_of_local[i] = -1;
                {
                    int m = 0;
                    for (int b = 0; b < k; ++b)
                        if (layout & (1u << b)) reg_of_local[b] = m++;
                }
                // Commuting diagonals (uncontrolled phases, CZ/Z negates) collect in a group that is
                // emitted as one OP_DIAG_GROUP; a non-diagonal gate may run ahead of the group when
                // its target is none of the group's qubits (they commute), otherwise the group is
                // emitted first.
                std::vector<FusedOp> group;
                uint32_t group_qubits = 0;
                auto flush = [&]() {
                    if (group.size() > 1) {
                        FusedOp hdr{};
                        hdr.code = OP_DIAG_GROUP;
                        hdr.reg = hdr.reg2 = hdr.local = -1;
                        hdr.reserved = (uint32_t)group.size();
                        plan.ops.push_back(hdr);
                    }
                    for (const FusedOp& m : group) plan.ops.push_back(m);
                    group.clear();
                    group_qubits = 0;
                };
                for (const GInfo& gi : stage_gates[si]) {
                    const qm_gate& g = gi.g;
                    FusedOp op{};
                    op.reg = op.reg2 = -1;
                    op.local = -1;
                    for (int q = 0; q < qubits; ++q) {
                        if (!(g.control_mask & (1u << q))) continue;
                        if (local_of[q] >= 0) op.cmask_local |= (uint16_t)(1u << local_of[q]);
                        else op.cmask_outer |= 1u << q;
                    }
                    std::memcpy(&op.coef[0], g.a, 16);
                    std::memcpy(&op.coef[2], g.b, 16);
                    std::memcpy(&op.coef[4], g.c, 16);
                    std::memcpy(&op.coef[6], g.d, 16);
                    if (gi.slot >= 0 && (gi.slot & kSlotBranch)) {
                        // noise branch: per-state coefficients, tested at run time
                        op.flags = kOpTable | kOpBranch;
                        op.reserved = (uint32_t)(gi.slot & (kSlotBranch - 1));
                        op.code = OP_MATRIX;
                        op.reg = (int8_t)reg_of_local[local_of[g.target]];
                    } else if (gi.slot >= 0) {
                        // per-state coefficients: generic op reading the batch table
                        op.flags = kOpTable;
                        op.reserved = (uint32_t)gi.slot;
                        if (gi.diag) {
                            int lt = local_of[g.target];
                            op.code = OP_DIAG;
                            op.local = (int8_t)lt;
                            op.target_outer = lt >= 0 ? 0u : (1u << g.target);
                        } else {
                            bool real = g.a[1] == 0 && g.b[1] == 0 && g.c[1] == 0 && g.d[1] == 0;
                            op.code = real ? OP_MATRIX_REAL : OP_MATRIX;
                            op.reg = (int8_t)reg_of_local[local_of[g.target]];
                        }
                    } else if (gi.diag) {
                        bool a1 = is_exact(g.a, 1.0, 0.0), d1 = is_exact(g.d, 1.0, 0.0);
                        int lt = local_of[g.target];
                        if (a1 && is_exact(g.d, -1.0, 0.0)) {
                            op.code = OP_NEGATE;
                            if (lt >= 0) op.cmask_local |= (uint16_t)(1u << lt);
                            else op.cmask_outer |= 1u << g.target;
                        } else {
                            op.code = OP_DIAG;
                            op.local = (int8_t)lt;
                            op.target_outer = lt >= 0 ? 0u : (1u << g.target);
                            op.flags = (uint16_t)((a1 ? 1 : 0) | (d1 ? 2 : 0));
                        }
                    } else if (g.kernel == QM_KERNEL_EXCHANGE) {
                        op.code = OP_EXCHANGE;
                        op.reg = (int8_t)reg_of_local[local_of[g.target]];
                        for (int q = 0; q < qubits && op.reg2 < 0; ++q)
                            if ((g.control_mask & (1u << q)) && local_of[q] >= 0 && reg_of_local[local_of[q]] >= 0)
                                op.reg2 = (int8_t)reg_of_local[local_of[q]];
                    } else if (g.kernel == QM_KERNEL_SWAP) {
                        op.code = OP_SWAP;
                        op.reg = (int8_t)reg_of_local[local_of[g.target]];
                        op.reg2 = (int8_t)reg_of_local[local_of[g.swap_control]];
                    } else {
                        bool real = g.a[1] == 0 && g.b[1] == 0 && g.c[1] == 0 && g.d[1] == 0;
                        op.code = real ? OP_MATRIX_REAL : OP_MATRIX;
                        op.reg = (int8_t)reg_of_local[local_of[g.target]];
                    }
                    if ((op.code == OP_MATRIX || op.code == OP_MATRIX_REAL || op.code == OP_EXCHANGE) && op.reg < 0) {
                        error = "planner placed a gate outside the register layout";
                        return false;
                    }
                    if (op.code == OP_SWAP && (op.reg < 0 || op.reg2 < 0)) {
                        error = "planner placed a swap outside the register layout";
                        return false;
                    }
                    const bool groupable =
                        (op.code == OP_DIAG && op.cmask_local == 0 && op.cmask_outer == 0) ||
                        (op.code == OP_NEGATE && popc(op.cmask_local) + popc(op.cmask_outer) <= 2);
                    if (groupable) {
                        group.push_back(op);
                        group_qubits |= gi.touch;
                        continue;
                    }
                    if (!gi.diag && (gi.xmask & group_qubits)) flush();
                    plan.ops.push_back(op);
                }
                flush();
            }
            if (lanes_needed) {
                // the store layout keeps the lanes on thread bits, as the lowest thread ranks: the
                // pass's last stage takes the lane order when its registers leave the lanes free,
                // otherwise one more stage does
                int last_stage = -1;
                for (size_t o = (size_t)pass.op_begin; o < plan.ops.size(); ++o)
                    if (plan.ops[o].code == OP_STAGE) last_stage = (int)o;
                if (last_stage < 0 || (layout & lane_mask)) {
                    uint32_t l = layout & ~lane_mask;
                    for (int b = k - 1; b >= 0 && popc(l) < kRegBits; --b)
                        if (!(lane_mask & (1u << b))) l |= 1u << b;
                    layout = l;
                    emit_stage(layout);
                    ++stages;
                    last_stage = (int)plan.ops.size() - 1;
                }
                plan.ops[(size_t)last_stage].reserved = lane_code;
                set_regs(pass.reg_out, layout);
            } else if (layout & low_local) {
                emit_stage(canonical);
                ++stages;
                set_regs(pass.reg_out, canonical);
                layout = canonical;
            } else {
                set_regs(pass.reg_out, layout);
            }
            {
                // Without a stage nothing orders one thread's stores after another's loads: a
                // relabeling pass stores through another mapping than it loads, so a thread could
                // overwrite an amplitude of its tile before the thread that loads it has.  Such a
                // pass (a restoring pass without gates) takes one exchange in its store layout,
                // whose barriers order them.
                bool moves = false, staged = false;
                for (int b = 0; b < k; ++b) moves |= pass.q_out[b] != pass.q[b];
                for (size_t o = (size_t)pass.op_begin; o < plan.ops.size(); ++o) staged |= plan.ops[o].code == OP_STAGE;
                if (moves && !staged) {
                    emit_stage(layout);
                    ++stages;
                }
            }
            {
                // Exchanges go through shared memory in phases of 2^low_bits threads (thread ranks
                // 0..low_bits-1 vary), and the swizzle sends local bit p to bank-group bit
                // p mod low_bits: an exchange side is free of bank conflicts when those ranks
                // hold bits of distinct classes.  The load layout holds bits 0..low_bits-1 there
                // and the last stage's ranks are fixed by the store, so every other stage whose
                // ascending ranks collide takes lanes of distinct classes when its free bits have
                // them.
                int last_stage = -1;
                for (size_t o = (size_t)pass.op_begin; o < plan.ops.size(); ++o)
                    if (plan.ops[o].code == OP_STAGE) last_stage = (int)o;
                for (size_t o = (size_t)pass.op_begin; (int)o < last_stage; ++o) {
                    FusedOp& st = plan.ops[o];
                    if (st.code != OP_STAGE || st.reserved != 0) continue;
                    uint32_t regs = 0;
                    for (int m = 0; m < kRegBits; ++m) regs |= 1u << st.reg_pos[m];
                    uint32_t seen = 0;
                    int n = 0;
                    for (int b = 0; b < k && n < low_bits; ++b)
                        if (!(regs & (1u << b))) {
                            seen |= 1u << (b % low_bits);
                            ++n;
                        }
                    if (seen == (1u << low_bits) - 1u) continue;  // ascending ranks are conflict-free
                    uint32_t code = (uint32_t)low_bits;
                    bool found = true;
                    for (int c = 0; c < low_bits && found; ++c) {
                        int pick = -1;
                        for (int b = c; b < k && pick < 0; b += low_bits)
                            if (!(regs & (1u << b))) pick = b;
                        if (pick < 0) found = false;
                        else code |= (uint32_t)pick << (4 + 4 * c);
                    }
                    if (found) st.reserved = code;
                }
            }
            {
                // store order: the lanes (when given), then the other thread bits ascending
                int rank = 0;
                if (lanes_needed)
                    for (int r = 0; r < low_bits; ++r) pass.out_bit[rank++] = pass.q_out[stage_lane(lane_code, r)];
                for (int b = 0; b < k; ++b)
                    if (!(layout & (1u << b)) && !(lanes_needed && (lane_mask & (1u << b))))
                        pass.out_bit[rank++] = pass.q_out[b];
                for (int r = 0; r < low_bits; ++r)
                    if (pass.out_bit[r] != r) {
                        error = "planner lost the coalesced run of a store layout";
                        return false;
                    }
            }
            pass.op_count = (int32_t)plan.ops.size() - pass.op_begin;
            if (pass.op_count > kMaxPassOps) {
                error = "pass program exceeds the kernel-parameter capacity";
                return false;
            }
            pass.stages = stages;
            plan.passes.push_back(pass);
            plan.planned_bytes += 2 * n * elem;
            return true;
    };

    // where each qubit of block Q goes: the qubits at lane_pos[r] to index bit r, every other
    // qubit to its own bit when that bit is a free one of the block, else where it is when that is
    // free, else to the lowest free bit
    auto place = [&](uint32_t Q) {
        for (int q = 0; q < 32; ++q) perm[q] = q;
        uint32_t lanes = 0;
        for (int r = 0; r < low_bits; ++r) {
            perm[lane_pos[r]] = r;
            lanes |= 1u << lane_pos[r];
        }
        uint32_t open = Q & ~low_mask, todo = Q & ~lanes;
        for (int b = 0; b < 32; ++b)
            if ((todo >> b) & 1u) {
                const int home = at[b];
                if (home >= low_bits && ((open >> home) & 1u)) {
                    perm[b] = home;
                    open &= ~(1u << home);
                    todo &= ~(1u << b);
                }
            }
        for (int b = 0; b < 32; ++b)
            if (((todo >> b) & 1u) && ((open >> b) & 1u)) {
                open &= ~(1u << b);
                todo &= ~(1u << b);
            }
        for (int b = 0; b < 32; ++b)
            if ((todo >> b) & 1u) {
                const int to = __builtin_ctz(open);
                perm[b] = to;
                open &= ~(1u << to);
            }
    };
    // lanes from a set of low_bits index bits: a qubit 0..low_bits-1 to its own lane, the others
    // in ascending order
    auto set_lanes = [&](uint32_t F) {
        bool used[8] = {};
        for (int r = 0; r < low_bits; ++r) lane_pos[r] = -1;
        for (int b = 0; b < 32; ++b)
            if (((F >> b) & 1u) && at[b] < low_bits && !used[at[b]]) {
                lane_pos[at[b]] = b;
                used[at[b]] = true;
                F &= ~(1u << b);
            }
        for (int r = 0; r < low_bits; ++r)
            if (lane_pos[r] < 0) {
                lane_pos[r] = __builtin_ctz(F);
                F &= ~(1u << lane_pos[r]);
            }
    };
    auto apply = [&](std::vector<GInfo>& gates) {
        int moved[32];
        for (int q = 0; q < 32; ++q) moved[perm[q]] = at[q];
        for (int q = 0; q < 32; ++q) at[q] = moved[q];
        for (GInfo& g : gates) remap_gate(g, perm);
    };
    auto in_order = [&]() {
        for (int q = 0; q < qubits; ++q)
            if (at[q] != q) return false;
        return true;
    };
    // index bits of qubits 0..low_bits-1, then of displaced qubits along their cycles, up to k
    auto restoring_block = [&](uint32_t Q) {
        for (int b = 0; b < qubits && popc(Q) < k; ++b)
            if (at[b] < low_bits) Q |= 1u << b;
        for (int b = 0; b < qubits && popc(Q) < k; ++b) {
            if (at[b] == b || ((Q >> b) & 1u)) continue;
            for (int c = b; popc(Q) < k && !((Q >> c) & 1u); c = at[c]) Q |= 1u << c;
        }
        return Q;
    };

    while (!remaining.empty()) {
        uint32_t Q = low_mask;
        uint32_t bx = 0, bz = 0;
        std::vector<GInfo> absorbed, rest;
        for (const GInfo& g : remaining) {
            if ((int)absorbed.size() < kMaxPassGates && !blocked(g, bx, bz)) {
                uint32_t nq = Q | g.need;
                if (popc(nq) <= k) {
                    Q = nq;
                    absorbed.push_back(g);
                    continue;
                }
            }
            rest.push_back(g);
            bx |= g.xmask;
            bz |= g.zmask;
        }
        if (absorbed.empty()) {
            error = "planner made no progress";
            return false;
        }
        // fill the block to k qubits: qubits the remaining gates need first, then the lowest
        for (const GInfo& g : rest) {
            if (popc(Q) >= k) break;
            uint32_t extra = g.need & ~Q;
            if (extra && popc(Q | extra) <= k) Q |= extra;
        }
        // the last pass of the circuit takes the bits that put qubits back before the lowest ones
        if (relabel && rest.empty()) Q = restoring_block(Q);
        for (int q = 0; q < qubits && popc(Q) < k; ++q) Q |= 1u << q;

        for (int q = 0; q < 32; ++q) perm[q] = q;
        for (int r = 0; r < low_bits; ++r) lane_pos[r] = r;
        if (relabel && rest.empty()) {
            // the last pass of the circuit starts putting the qubits back
            uint32_t F = 0;
            for (int b = 0; b < qubits; ++b)
                if (at[b] < low_bits) F |= 1u << b;
            if ((F & ~Q) == 0) set_lanes(F);
            place(Q);
        } else if (relabel) {
            // the low_bits bits of Q whose qubits let the next pass absorb the most gates
            auto absorbable = [&](uint32_t start) {
                uint32_t QQ = start, cx = 0, cz = 0;
                int c = 0;
                for (const GInfo& g : rest) {
                    if (c >= kMaxPassGates || cx == all_qubits) break;
                    if (!blocked(g, cx, cz)) {
                        const uint32_t nq = QQ | g.need;
                        if (popc(nq) <= k) {
                            QQ = nq;
                            ++c;
                            continue;
                        }
                    }
                    cx |= g.xmask;
                    cz |= g.zmask;
                }
                return c;
            };
            int bits[32], nb = 0;
            for (int b = 0; b < qubits; ++b)
                if ((Q >> b) & 1u) bits[nb++] = b;
            int best = -1;
            uint32_t bestF = low_mask;
            int idx[8];
            for (int i = 0; i < low_bits; ++i) idx[i] = i;
            while (true) {
                uint32_t F = 0, classes = 0;
                for (int i = 0; i < low_bits; ++i) {
                    F |= 1u << bits[idx[i]];
                    classes |= 1u << (idx[i] % low_bits);  // idx[i] is the local bit
                }
                // ties go to lanes of distinct bank-group classes (a conflict-free last exchange),
                // then to keeping the layout
                const int score = 4 * absorbable(F) + (classes == (1u << low_bits) - 1u ? 2 : 0) + (F == low_mask ? 1 : 0);
                if (score > best) {
                    best = score;
                    bestF = F;
                }
                int i = low_bits - 1;
                while (i >= 0 && idx[i] == nb - low_bits + i) --i;
                if (i < 0) break;
                ++idx[i];
                for (int j = i + 1; j < low_bits; ++j) idx[j] = idx[j - 1] + 1;
            }
            set_lanes(bestF);
            place(Q);
        }
        if (!build_pass(Q, absorbed)) return false;
        if (relabel) apply(rest);
        remaining.swap(rest);
    }
    if (relabel) {
        std::vector<GInfo> none;
        for (int round = 0; !in_order(); ++round) {
            if (round >= 2 * qubits) {
                error = "planner could not put the qubits back in order";
                return false;
            }
            uint32_t Q = restoring_block(low_mask);
            for (int q = 0; q < qubits && popc(Q) < k; ++q) Q |= 1u << q;
            uint32_t F = 0;
            for (int b = 0; b < qubits; ++b)
                if (at[b] < low_bits) F |= 1u << b;
            set_lanes(F);
            place(Q);
            if (!build_pass(Q, none)) return false;
            apply(none);
        }
    }
    plan.launches = (int32_t)plan.passes.size();
    return true;
}

}  // namespace

// Plans without relabeling and, where relabeling applies, with it: the relabeling plan is kept
// only when it needs fewer passes, since its lane stages and restoring pass cost more than they
// save otherwise.
// CNOTs rewritten as CZs for fused blocks (QM_CZ_REWRITE=0 turns it off).  CNOT(c, t) =
// H_t CZ(c, t) H_t; where the gates before and after it on t are uncontrolled single-qubit
// matrices U_p and U_n, they become H U_p and U_n H and the CNOT a CZ.  A CZ is diagonal, so a
// stage need not hold t in a register for it and gates commute past it on c and t alike: the
// 30-qubit brick plans in 25 passes of 142 stages instead of 29 of 185 (complex64: 23 of 130
// instead of 34 of 191).  Exact up to the rounding of the two matrix products.
bool cz_rewrite_enabled() {
    const char* e = std::getenv("QM_CZ_REWRITE");
    return !(e && e[0] == '0');
}

std::vector<qm_gate> cnots_as_cz(const std::vector<qm_gate>& gates) {
    std::vector<qm_gate> out(gates);
    const size_t n = out.size();
    auto touches = [](const qm_gate& g, int q) {
        return g.target == q || ((g.control_mask >> q) & 1u) || g.swap_control == q;
    };
    auto plain = [](const qm_gate& g) {
        return (g.kernel == QM_KERNEL_MATRIX || g.kernel == QM_KERNEL_HADAMARD) && g.control_mask == 0 &&
               g.swap_control < 0;
    };
    // the previous and next gate on each CNOT's target (the rewrite keeps every gate's qubits)
    std::vector<long> before(n, -1), after(n, -1);
    {
        long last[32];
        std::fill(last, last + 32, -1L);
        for (size_t i = 0; i < n; ++i) {
            if (out[i].target >= 0 && out[i].target < 32) before[i] = last[out[i].target];
            for (int q = 0; q < 32; ++q)
                if (touches(out[i], q)) last[q] = (long)i;
        }
        std::fill(last, last + 32, -1L);
        for (size_t i = n; i-- > 0;) {
            if (out[i].target >= 0 && out[i].target < 32) after[i] = last[out[i].target];
            for (int q = 0; q < 32; ++q)
                if (touches(out[i], q)) last[q] = (long)i;
        }
    }
    const double h = std::sqrt(0.5);
    for (size_t i = 0; i < n; ++i) {
        const qm_gate& x = out[i];
        if (x.kernel != QM_KERNEL_EXCHANGE || __builtin_popcount(x.control_mask) != 1 || x.swap_control >= 0) continue;
        if (before[i] < 0 || after[i] < 0 || !plain(out[(size_t)before[i]]) || !plain(out[(size_t)after[i]])) continue;
        qm_gate& u = out[(size_t)before[i]];
        qm_gate& v = out[(size_t)after[i]];
        // H U: rows (a, b) and (c, d) mixed; U H: columns (a, c) and (b, d) mixed
        for (int k = 0; k < 2; ++k) {
            const double a = u.a[k], b = u.b[k], c = u.c[k], d = u.d[k];
            u.a[k] = h * (a + c);
            u.b[k] = h * (b + d);
            u.c[k] = h * (a - c);
            u.d[k] = h * (b - d);
            const double va = v.a[k], vb = v.b[k], vc = v.c[k], vd = v.d[k];
            v.a[k] = h * (va + vb);
            v.b[k] = h * (va - vb);
            v.c[k] = h * (vc + vd);
            v.d[k] = h * (vc - vd);
        }
        u.kernel = QM_KERNEL_MATRIX;
        v.kernel = QM_KERNEL_MATRIX;
        qm_gate& z = out[i];
        z.kernel = QM_KERNEL_DIAGONAL;
        z.a[0] = 1.0;
        z.a[1] = 0.0;
        z.b[0] = z.b[1] = z.c[0] = z.c[1] = 0.0;
        z.d[0] = -1.0;
        z.d[1] = 0.0;
    }
    return out;
}

bool plan_fused(const std::vector<qm_gate>& in, int qubits, int precision, int width, Plan& plan,
                std::string& error, const std::vector<int32_t>* slots) {
    std::vector<qm_gate> rewritten;
    const bool rewrite = !slots && cz_rewrite_enabled() && (width == 0 || width >= 9);
    if (rewrite) rewritten = cnots_as_cz(in);
    const std::vector<qm_gate>& gates = rewrite ? rewritten : in;
    if (!plan_fused_with(gates, qubits, precision, width, plan, error, slots, false)) return false;
    if (slots || !relabel_enabled() || plan.width == 1 || plan.passes.size() < 2) return true;
    Plan alt;
    std::string alt_error;
    if (plan_fused_with(gates, qubits, precision, width, alt, alt_error, slots, true) &&
        alt.passes.size() < plan.passes.size())
        plan = std::move(alt);
    return true;
}

}  // namespace qm
