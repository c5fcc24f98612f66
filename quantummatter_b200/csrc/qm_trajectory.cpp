// qm_trajectory.cpp -- batched noise trajectories (qm_trajectories_run) of libqmb200.so.
//
// NoisyStateVectorSimulator (src/QuantumMatter.Application/Noise/NoisyStateVectorSimulator.cs:
// 36-106) runs trajectories one after another, each through NoisyCircuit.Execute
// (src/QuantumMatter.Core/Noise/NoisyCircuit.cs:48-65): unitary segments through the backend
// port and every channel placement through CpuNoiseChannelBackend, one full pass (two for a
// damping) per placement.  Here a wave of trajectories lives in HBM as the states of one batch
// and the noisy circuit is compiled once into segments:
//   - a segment's gates, its Pauli placements and the damping Kraus ops decided just before it
//     share one fused schedule; every placement is a table op whose 2x2 coefficients differ per
//     trajectory (identity for "no error", which the fused kernel skips);
//   - a run of consecutive damping placements over at most 8 qubits ends a segment: one read
//     pass writes the joint Born masses over those qubits, and the decision kernel takes the
//     dampings one after another on those masses (each damping rescales or moves them exactly
//     as it rescales or moves the amplitudes) before the next segment applies the Kraus ops.
// Decisions are taken per trajectory, in program order, on the device from the trajectory's
// own draws, so the host never waits inside a wave.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "qm_internal.h"

using namespace qm;

namespace {

struct Segment {
    std::vector<qm_gate> gates;
    std::vector<int32_t> slots;
    std::vector<Decision> decisions;  // taken just before the segment runs
    int32_t local_slots = 0;
    int32_t group = -1;               // joint-mass group measured after the segment
    Plan plan;
    std::vector<int32_t> pass_first, pass_count;  // packed slot range of each pass
    int32_t packed = 0;
    int32_t decision_offset = 0;
};

struct Program {
    std::vector<Segment> segments;
    std::vector<uint32_t> groups;  // qubit masks of the joint-mass groups
    std::vector<int8_t> fixed;     // per channel: -2 decided on the device, else its branch
    int32_t max_draws = 0;         // draws of the decisions, an upper bound per trajectory
    int32_t max_packed = 0;
    int32_t max_bins = 1;
    int32_t passes = 0;
    std::vector<Decision> all_decisions;
    ~Program() {
        for (Segment& s : segments) plan_release(s.plan);
    }
};

enum GateClass { GC_SKIP, GC_X, GC_Y, GC_Z, GC_H, GC_S, GC_CNOT, GC_CZ, GC_SWAP, GC_OTHER };

// Pauli and Clifford gates recognised from their prepared records (exact coefficients only).
GateClass classify_gate(const qm_gate& g) {
    auto is = [](const double* v, double re, double im) { return v[0] == re && v[1] == im; };
    const int controls = __builtin_popcount(g.control_mask);
    switch (g.kernel) {
    case QM_KERNEL_IDENTITY: return GC_SKIP;
    case QM_KERNEL_EXCHANGE: return controls == 0 ? GC_X : controls == 1 ? GC_CNOT : GC_OTHER;
    case QM_KERNEL_SWAP: return controls == 0 ? GC_SWAP : GC_OTHER;
    case QM_KERNEL_HADAMARD: return controls == 0 ? GC_H : GC_OTHER;
    case QM_KERNEL_DIAGONAL:
        if (is(g.a, 1, 0) && is(g.d, 1, 0)) return GC_SKIP;
        if (is(g.a, 1, 0) && is(g.d, -1, 0)) return controls == 0 ? GC_Z : controls == 1 ? GC_CZ : GC_OTHER;
        if (controls == 0 && is(g.a, 1, 0) && (is(g.d, 0, 1) || is(g.d, 0, -1))) return GC_S;
        return GC_OTHER;
    case QM_KERNEL_MATRIX:
        if (controls == 0 && is(g.a, 0, 0) && is(g.b, 0, -1) && is(g.c, 0, 1) && is(g.d, 0, 0)) return GC_Y;
        return GC_OTHER;
    default: return GC_OTHER;
    }
}

Decision step(int32_t kind, int32_t a, int32_t b = -1) {
    Decision d{};
    d.kind = kind;
    d.channel = -1;
    d.slot = -1;
    d.bit = 0;
    d.a = a;
    d.b = b;
    return d;
}

// The fused schedule's placeholder for a noise branch; its coefficients come from the table.
qm_gate branch_placeholder(int target) {
    qm_gate g{};
    g.kernel = QM_KERNEL_MATRIX;
    g.target = target;
    g.control_mask = 0;
    g.swap_control = -1;
    g.a[0] = 1.0;
    g.d[0] = 1.0;
    return g;
}

int32_t compile(const qm_gate* gates, int32_t gate_count, const qm_channel* ch, int32_t nch, int32_t qubits,
                int32_t exec_qubits, int32_t precision, Program& P) {
    P.fixed.assign((size_t)nch, -1);
    Segment cur;
    bool open = false;  // a run of dampings is open: its steps wait for the joint masses
    uint32_t mask = 0;
    std::vector<Decision> pending;  // steps of the open run, in program order
    auto add_step = [&](const Decision& d) { (open ? pending : cur.decisions).push_back(d); };
    auto close_group = [&]() {
        P.groups.push_back(mask);
        cur.group = (int32_t)P.groups.size() - 1;
        P.segments.push_back(std::move(cur));
        cur = Segment();
        for (Decision d : pending) {
            if (d.kind == STEP_DAMPING) {
                d.bit = __builtin_popcount(mask & ((1u << d.a) - 1u));
                d.slot = cur.local_slots++;
                cur.gates.push_back(branch_placeholder(d.a));
                cur.slots.push_back(d.slot | kSlotBranch);
            }
            cur.decisions.push_back(d);
        }
        P.max_bins = std::max(P.max_bins, 1 << __builtin_popcount(mask));
        pending.clear();
        open = false;
        mask = 0;
    };
    auto add_gate = [&](const qm_gate& g) -> int32_t {
        const GateClass gc = classify_gate(g);
        switch (gc) {
        case GC_SKIP: return QM_OK;
        case GC_X: add_step(step(STEP_FRAME_X, g.target)); return QM_OK;
        case GC_Y: add_step(step(STEP_FRAME_Y, g.target)); return QM_OK;
        case GC_Z: add_step(step(STEP_FRAME_Z, g.target)); return QM_OK;
        default: break;
        }
        if (open) close_group();
        const int ctrl = g.control_mask ? __builtin_ctz(g.control_mask) : -1;
        if (gc != GC_OTHER) {  // a Clifford gate: runs unchanged, conjugates the frame
            cur.gates.push_back(g);
            cur.slots.push_back(-1);
            const int32_t kind = gc == GC_H ? STEP_FRAME_H : gc == GC_S ? STEP_FRAME_S : gc == GC_CNOT ? STEP_FRAME_CNOT
                                 : gc == GC_CZ ? STEP_FRAME_CZ : STEP_FRAME_SWAP;
            cur.decisions.push_back(step(kind, g.target, gc == GC_SWAP ? g.swap_control : ctrl));
            return QM_OK;
        }
        if (g.kernel == QM_KERNEL_SWAP) return fail(QM_E_UNSUPPORTED, "controlled swap is not a reference gate");
        // the frame's X on a control would turn "control on one" into "control on zero": apply it first
        for (int q = 0; q < 32; ++q)
            if (g.control_mask & (1u << q)) {
                Decision f = step(STEP_FLUSH_X, q);
                f.slot = cur.local_slots++;
                cur.gates.push_back(branch_placeholder(q));
                cur.slots.push_back(f.slot | kSlotBranch);
                cur.decisions.push_back(f);
            }
        qm_gate ph = g;
        if (g.kernel == QM_KERNEL_EXCHANGE) {  // Toffoli: X on the target as a matrix
            ph.kernel = QM_KERNEL_MATRIX;
            ph.a[0] = ph.a[1] = ph.b[1] = ph.c[1] = ph.d[0] = ph.d[1] = 0.0;
            ph.b[0] = ph.c[0] = 1.0;
        } else if (g.kernel == QM_KERNEL_HADAMARD) {
            ph.kernel = QM_KERNEL_MATRIX;
        }
        Decision c = step(STEP_CONJ, g.target);
        c.slot = cur.local_slots++;
        std::memcpy(&c.coef[0], ph.a, 16);
        std::memcpy(&c.coef[2], ph.b, 16);
        std::memcpy(&c.coef[4], ph.c, 16);
        std::memcpy(&c.coef[6], ph.d, 16);
        cur.gates.push_back(ph);
        cur.slots.push_back(c.slot);
        cur.decisions.push_back(c);
        return QM_OK;
    };
    int32_t done = 0;
    int32_t rc = QM_OK;
    auto gates_until = [&](int32_t pos) -> int32_t {
        for (; done < pos; ++done) {
            int32_t r = add_gate(gates[done]);
            if (r) return r;
        }
        return QM_OK;
    };
    int32_t last = 0;
    for (int32_t j = 0; j < nch; ++j) {
        const qm_channel& c = ch[j];
        if (c.kind < 0 || c.kind > 3) return fail(QM_E_UNSUPPORTED, "unknown noise kind");
        if ((uint32_t)c.target >= (uint32_t)qubits) return fail(QM_E_RANGE, "channel target out of range");
        if (!std::isfinite(c.probability) || c.probability < 0 || c.probability > 1)
            return fail(QM_E_RANGE, "Channel probability must be finite and in [0,1].");
        if (c.position < last || c.position > gate_count)
            return fail(QM_E_ARG, "channel positions must be nondecreasing and within the gate list");
        last = c.position;
        if ((rc = gates_until(c.position))) return rc;
        if (c.probability == 0) continue;  // NoisyCircuit.Execute skips it without a draw
        if (c.kind == 3) {
            const uint32_t bit = 1u << c.target;
            if (open && !(mask & bit) && __builtin_popcount(mask) == kGroupMaxBits) close_group();
            open = true;
            mask |= bit;
            Decision d = step(STEP_DAMPING, c.target);
            d.channel = j;
            d.p = c.probability;
            pending.push_back(d);
            P.fixed[(size_t)j] = -2;
            ++P.max_draws;
            continue;
        }
        if (c.kind != 2 && c.probability == 1) {  // a certain flip takes no draw
            P.fixed[(size_t)j] = (int8_t)(c.kind == 0 ? 1 : 3);
            add_step(step(c.kind == 0 ? STEP_FRAME_X : STEP_FRAME_Z, c.target));
            continue;
        }
        P.fixed[(size_t)j] = -2;
        ++P.max_draws;
        Decision d = step(c.kind, c.target);
        d.channel = j;
        d.p = c.probability;
        add_step(d);
    }
    if ((rc = gates_until(gate_count))) return rc;
    if (open) close_group();
    P.segments.push_back(std::move(cur));

    // fused schedules; table slots renumbered so that each pass stages one contiguous range
    for (Segment& s : P.segments) {
        std::string err;
        if (!plan_fused(s.gates, exec_qubits, precision, 0, s.plan, err, &s.slots))
            return fail(QM_E_ARG, "planner: " + err);
        std::vector<int32_t> packed_of((size_t)s.local_slots, -1);
        int32_t next = 0;
        for (const FusedPass& p : s.plan.passes) {
            const int32_t first = next;
            for (int32_t o = p.op_begin; o < p.op_begin + p.op_count; ++o) {
                FusedOp& op = s.plan.ops[(size_t)o];
                if (!(op.flags & kOpTable)) continue;
                if (op.reserved >= (uint32_t)s.local_slots) return fail(QM_E_DEVICE, "noise branch slot out of range");
                packed_of[op.reserved] = next;
                op.reserved = (uint32_t)(next - first);
                ++next;
            }
            s.pass_first.push_back(first);
            s.pass_count.push_back(next - first);
        }
        s.packed = next;
        P.max_packed = std::max(P.max_packed, next);
        P.passes += (int32_t)s.plan.passes.size();
        for (Decision& d : s.decisions) {
            if (d.slot < 0) continue;
            if (packed_of[(size_t)d.slot] < 0) return fail(QM_E_DEVICE, "a per-trajectory op was not scheduled");
            d.slot = packed_of[(size_t)d.slot];
        }
        s.decision_offset = (int32_t)P.all_decisions.size();
        P.all_decisions.insert(P.all_decisions.end(), s.decisions.begin(), s.decisions.end());
    }
    return QM_OK;
}

// Device buffers of one run: freed after the context stream has drained.
struct Buffers {
    cudaStream_t stream;
    qm_context* ctx;
    int64_t accounted = 0;
    std::vector<void*> ptrs;
    Buffers(qm_context* c) : stream(c->stream), ctx(c) {}
    ~Buffers() {
        cudaStreamSynchronize(stream);
        for (void* p : ptrs) cudaFree(p);
        ctx->device_in_use -= accounted;
    }
    template <typename T>
    int32_t get(T*& out, size_t bytes) {
        void* p = nullptr;
        QM_CUDA(cudaMalloc(&p, std::max<size_t>(bytes, 16)));
        ptrs.push_back(p);
        out = static_cast<T*>(p);
        return QM_OK;
    }
};

}  // namespace

extern "C" int32_t qm_trajectories_run(qm_context* ctx, int32_t qubits, int32_t precision, const qm_gate* gates,
                                       int32_t gate_count, const qm_channel* channels, int32_t channel_count,
                                       int32_t trajectories, const double* draws, int32_t draw_stride,
                                       const qm_pauli_term* terms, int32_t term_count,
                                       const qm_trajectory_outputs* outputs, qm_trajectory_stats* stats) {
    const auto wall0 = std::chrono::steady_clock::now();
    if (!ctx) return fail(QM_E_ARG, "context is null");
    if (ctx->disposed) return fail(QM_E_DISPOSED, "context disposed");
    if (qubits < 1 || qubits > 30) return fail(QM_E_RANGE, "qubits must be between 1 and 30");
    if (precision != QM_FP64 && precision != QM_FP32) return fail(QM_E_RANGE, "unknown precision");
    if (trajectories < 1) return fail(QM_E_RANGE, "trajectories must be positive");
    if (channel_count < 0 || (channel_count > 0 && !channels)) return fail(QM_E_ARG, "channels is null");
    if (term_count < 0 || (term_count > 0 && !terms)) return fail(QM_E_ARG, "terms is null");
    if (draw_stride < 0 || (draw_stride > 0 && !draws)) return fail(QM_E_ARG, "draws is null");
    int32_t rc = validate_prepared_gates(gates, gate_count, qubits);
    if (rc) return rc;
    const uint32_t all = (uint32_t)((1ull << qubits) - 1);
    for (int32_t i = 0; i < term_count; ++i)
        if ((terms[i].flip_mask | terms[i].sign_mask) & ~all) return fail(QM_E_ARG, "Observable and state sizes must match.");
    qm_trajectory_outputs out{};
    if (outputs) out = *outputs;
    const bool welford = out.probability_means || out.probability_stderr;
    if (out.probability_stderr && trajectories < 2)
        return fail(QM_E_RANGE, "estimating probabilities needs at least two trajectories");
    for (int64_t i = 0; i < (int64_t)trajectories * draw_stride; ++i)
        if (!(draws[i] >= 0.0 && draws[i] < 1.0)) return fail(QM_E_RANGE, "draws must lie in [0,1)");

    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    QM_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    const int32_t n = std::max(qubits, 9);  // batched states hold at least 9 qubits; the extra ones stay |0>
    Program P;
    rc = compile(gates, gate_count, channels, channel_count, qubits, n, precision, P);
    if (rc) return rc;

    const bool tiles = out.values || out.masses || welford;
    TilePlan tp;
    if (tiles) {
        std::string err;
        if (!plan_tiles(n, precision, terms, term_count, tp, err)) return fail(QM_E_ARG, err);
    }
    const int64_t state_bytes = (precision == QM_FP32 ? 8ll : 16ll) << n;
    const int64_t len = int64_t(1) << qubits;
    auto per_state = [&](int states) {
        int64_t b = state_bytes + 64ll * std::max(1, P.max_packed) + 8ll * draw_stride + 24 + channel_count;
        b += 8ll * histogram_ctas(n) * P.max_bins;
        if (tiles) b += 8ll * (tp.rows_per_state + 1) * tp.columns;
        return b;
    };
    const int64_t fixed = (welford ? 16 * len : 0) + (int64_t)P.all_decisions.size() * (int64_t)sizeof(Decision);
    const int64_t room = ctx->device_budget - ctx->device_in_use - fixed;
    int64_t B = std::min<int64_t>(trajectories, 65535);
    if (room <= 0) B = 0;
    while (B > 0 && B * per_state((int)B) > room) B = std::min<int64_t>(B - 1, room / per_state((int)B));
    if (B < 1) return fail(QM_E_BUDGET, "one trajectory exceeds the context's device memory budget");
    const int ctas = histogram_ctas(n);

    Buffers buf(ctx);
    buf.accounted = B * per_state((int)B) + fixed;
    ctx->device_in_use += buf.accounted;
    void* amps = nullptr;
    double *table = nullptr, *partials = nullptr, *d_draws = nullptr, *tpart = nullptr, *tout = nullptr;
    double *d_masses = nullptr, *mean = nullptr, *m2 = nullptr;
    int32_t *counters = nullptr, *status = nullptr, *ambiguous = nullptr;
    uint32_t *frame_x = nullptr, *frame_z = nullptr;
    int8_t* d_branches = nullptr;
    Decision* d_decisions = nullptr;
    const uint64_t table_stride = 8ull * (uint64_t)std::max(1, P.max_packed);
    if ((rc = buf.get(amps, (size_t)(B * state_bytes))) ||
        (rc = buf.get(table, sizeof(double) * table_stride * (size_t)B)) ||
        (rc = buf.get(partials, sizeof(double) * (size_t)B * ctas * P.max_bins)) ||
        (rc = buf.get(d_draws, sizeof(double) * (size_t)B * draw_stride)) ||
        (rc = buf.get(counters, sizeof(int32_t) * (size_t)B)) || (rc = buf.get(status, sizeof(int32_t) * (size_t)B)) ||
        (rc = buf.get(ambiguous, sizeof(int32_t) * (size_t)B)) ||
        (rc = buf.get(frame_x, sizeof(uint32_t) * (size_t)B)) || (rc = buf.get(frame_z, sizeof(uint32_t) * (size_t)B)) ||
        (rc = buf.get(d_decisions, sizeof(Decision) * P.all_decisions.size())))
        return rc;
    if (out.branches && channel_count > 0 && (rc = buf.get(d_branches, (size_t)B * channel_count))) return rc;
    if (tiles && ((rc = buf.get(tpart, sizeof(double) * (size_t)B * tp.rows_per_state * tp.columns)) ||
                  (rc = buf.get(tout, sizeof(double) * (size_t)B * tp.columns))))
        return rc;
    if (welford && ((rc = buf.get(d_masses, sizeof(double) * (size_t)B)) || (rc = buf.get(mean, sizeof(double) * len)) ||
                    (rc = buf.get(m2, sizeof(double) * len))))
        return rc;
    if (welford) {
        QM_CUDA(cudaMemsetAsync(mean, 0, sizeof(double) * len, st));
        QM_CUDA(cudaMemsetAsync(m2, 0, sizeof(double) * len, st));
    }
    if (!P.all_decisions.empty())
        QM_CUDA(cudaMemcpyAsync(d_decisions, P.all_decisions.data(), sizeof(Decision) * P.all_decisions.size(),
                                cudaMemcpyHostToDevice, st));
    for (Segment& s : P.segments) {
        // a segment followed by a damping group computes the group's joint masses in the
        // epilogue of its last pass when that pass compiles
        if (s.group >= 0 && !s.plan.passes.empty()) s.plan.hist_mask = P.groups[(size_t)s.group];
        jit_prepare(s.plan);  // layers repeat: most segments share compiled passes
        rc = plan_upload(s.plan, st);
        if (rc) return rc;
    }

    const double margin = precision == QM_FP32 ? 1e-5 : 1e-12;
    std::vector<double> h_out;
    std::vector<int32_t> h_counters((size_t)B), h_status((size_t)B), h_amb((size_t)B);
    std::vector<uint32_t> h_fx((size_t)B), h_fz((size_t)B);
    std::vector<int8_t> h_branches;
    float device_ms = 0;
    int32_t waves = 0;
    for (int64_t t0 = 0; t0 < trajectories; t0 += B) {
        const int Bw = (int)std::min<int64_t>(B, trajectories - t0);
        ++waves;
        QM_CUDA(cudaEventRecord(ctx->ev_start, st));
        QM_CUDA(launch_reset_batched(amps, n, precision, Bw, st));
        QM_CUDA(cudaMemsetAsync(counters, 0, sizeof(int32_t) * Bw, st));
        QM_CUDA(cudaMemsetAsync(status, 0, sizeof(int32_t) * Bw, st));
        QM_CUDA(cudaMemsetAsync(ambiguous, 0, sizeof(int32_t) * Bw, st));
        QM_CUDA(cudaMemsetAsync(frame_x, 0, sizeof(uint32_t) * Bw, st));
        QM_CUDA(cudaMemsetAsync(frame_z, 0, sizeof(uint32_t) * Bw, st));
        if (d_branches) QM_CUDA(cudaMemsetAsync(d_branches, 0xff, (size_t)Bw * channel_count, st));
        if (draw_stride > 0)
            QM_CUDA(cudaMemcpyAsync(d_draws, draws + t0 * draw_stride, sizeof(double) * (size_t)Bw * draw_stride,
                                    cudaMemcpyHostToDevice, st));
        int32_t prev_group = -1;
        for (const Segment& s : P.segments) {
            DecideArgs da{};
            da.decisions = d_decisions + s.decision_offset;
            da.count = (int32_t)s.decisions.size();
            da.partials = prev_group >= 0 ? partials : nullptr;
            da.ctas = ctas;
            da.bins = prev_group >= 0 ? 1 << __builtin_popcount(P.groups[(size_t)prev_group]) : 0;
            da.draws = d_draws;
            da.draw_stride = draw_stride;
            da.counters = counters;
            da.status = status;
            da.ambiguous = ambiguous;
            da.table = table;
            da.table_stride = table_stride;
            da.branches = d_branches;
            da.channels = channel_count;
            da.margin = margin;
            da.frame_x = frame_x;
            da.frame_z = frame_z;
            QM_CUDA(launch_decide(da, Bw, st));
            for (size_t p = 0; p < s.plan.passes.size(); ++p) {
                FusedBatch fb{Bw, 1ull << n, table, table_stride, s.pass_first[p], s.pass_count[p]};
                fb.hist = partials;
                QM_CUDA(launch_plan_pass(s.plan, p, amps, &fb, st));
            }
            if (s.group >= 0 && !s.plan.hist_fused)
                QM_CUDA(launch_group_histogram(amps, n, precision, Bw, P.groups[(size_t)s.group], partials, st));
            prev_group = s.group;
        }
        if (tiles) QM_CUDA(enqueue_tile_expectation(amps, n, precision, tp, Bw, tpart, tout, st));
        QM_CUDA(cudaEventRecord(ctx->ev_stop, st));
        if (tiles) {
            h_out.resize((size_t)Bw * tp.columns);
            QM_CUDA(cudaMemcpyAsync(h_out.data(), tout, sizeof(double) * h_out.size(), cudaMemcpyDeviceToHost, st));
        }
        QM_CUDA(cudaMemcpyAsync(h_counters.data(), counters, sizeof(int32_t) * Bw, cudaMemcpyDeviceToHost, st));
        QM_CUDA(cudaMemcpyAsync(h_status.data(), status, sizeof(int32_t) * Bw, cudaMemcpyDeviceToHost, st));
        QM_CUDA(cudaMemcpyAsync(h_amb.data(), ambiguous, sizeof(int32_t) * Bw, cudaMemcpyDeviceToHost, st));
        QM_CUDA(cudaMemcpyAsync(h_fx.data(), frame_x, sizeof(uint32_t) * Bw, cudaMemcpyDeviceToHost, st));
        QM_CUDA(cudaMemcpyAsync(h_fz.data(), frame_z, sizeof(uint32_t) * Bw, cudaMemcpyDeviceToHost, st));
        if (d_branches) {
            h_branches.resize((size_t)Bw * channel_count);
            QM_CUDA(cudaMemcpyAsync(h_branches.data(), d_branches, h_branches.size(), cudaMemcpyDeviceToHost, st));
        }
        QM_CUDA(cudaStreamSynchronize(st));
        float ms = 0;
        QM_CUDA(cudaEventElapsedTime(&ms, ctx->ev_start, ctx->ev_stop));
        device_ms += ms;
        for (int b = 0; b < Bw; ++b) {
            if (h_status[(size_t)b] == QM_E_RANGE)
                return fail(QM_E_RANGE, "trajectory " + std::to_string(t0 + b) + " needs more than draw_stride draws");
            if (h_status[(size_t)b] != QM_OK)
                return fail(QM_E_MASS, "trajectory " + std::to_string(t0 + b) +
                                           ": The state has no finite positive probability mass.");
        }
        if (out.outcomes) {  // the true state: the frame's X applied to the stored one
            QM_CUDA(launch_frame_flip(amps, n, precision, Bw, frame_x, st));
            QM_CUDA(cudaStreamSynchronize(st));
        }
        for (int b = 0; b < Bw; ++b) {
            const int64_t t = t0 + b;
            int32_t consumed = h_counters[(size_t)b];
            if (tiles) {
                const double mass = h_out[(size_t)b * tp.columns + tp.mass_column];
                if (!std::isfinite(mass) || mass <= 0)
                    return fail(QM_E_MASS, "trajectory " + std::to_string(t) + ": The state has no finite positive probability mass.");
                if (out.masses) out.masses[t] = mass;
                for (int32_t k = 0; k < term_count && out.values; ++k) {
                    const double raw = h_out[(size_t)b * tp.columns + k];
                    if (!std::isfinite(raw)) return fail(QM_E_MASS, "The observable accumulation is nonfinite.");
                    // <F psi|P|F psi> = -<psi|P|psi> when the frame anticommutes with P
                    const int odd = (__builtin_popcount(h_fx[(size_t)b] & terms[k].sign_mask) +
                                     __builtin_popcount(h_fz[(size_t)b] & terms[k].flip_mask)) & 1;
                    out.values[t * term_count + k] = odd ? -(raw / mass) : raw / mass;
                }
            }
            if (out.ambiguous) out.ambiguous[t] = h_amb[(size_t)b];
            if (out.branches) {
                for (int32_t j = 0; j < channel_count; ++j) {
                    const int8_t f = P.fixed[(size_t)j];
                    out.branches[t * channel_count + j] = f == -2 ? h_branches[(size_t)b * channel_count + j] : f;
                }
            }
            if (out.outcomes) {
                if (consumed >= draw_stride)
                    return fail(QM_E_RANGE, "trajectory " + std::to_string(t) + " needs more than draw_stride draws");
                const double u = draws[t * draw_stride + consumed];
                int64_t outcome = -1;
                int32_t amb = 0;
                char* base = static_cast<char*>(amps) + (size_t)b * state_bytes;
                rc = qm_sample_amplitudes(ctx, base, n, precision, &u, 1, &outcome, &amb);
                if (rc) return rc;
                out.outcomes[t] = outcome;
                if (out.ambiguous) out.ambiguous[t] += amb;
                ++consumed;
            }
            if (out.consumed) out.consumed[t] = consumed;
        }
        if (welford) {
            std::vector<double> hm((size_t)Bw);
            for (int b = 0; b < Bw; ++b) hm[(size_t)b] = h_out[(size_t)b * tp.columns + tp.mass_column];
            QM_CUDA(cudaMemcpyAsync(d_masses, hm.data(), sizeof(double) * Bw, cudaMemcpyHostToDevice, st));
            // after a frame flip (outcomes) the stored states are the true ones
            if (out.outcomes) QM_CUDA(cudaMemsetAsync(frame_x, 0, sizeof(uint32_t) * Bw, st));
            QM_CUDA(launch_welford(amps, precision, Bw, 1ull << n, len, d_masses, frame_x, t0, mean, m2, st));
            QM_CUDA(cudaStreamSynchronize(st));
        }
    }
    if (welford) {
        if (out.probability_means)
            QM_CUDA(cudaMemcpyAsync(out.probability_means, mean, sizeof(double) * len, cudaMemcpyDeviceToHost, st));
        if (out.probability_stderr) {
            QM_CUDA(launch_welford_finish(m2, len, trajectories, st));
            QM_CUDA(cudaMemcpyAsync(out.probability_stderr, m2, sizeof(double) * len, cudaMemcpyDeviceToHost, st));
        }
        QM_CUDA(cudaStreamSynchronize(st));
    }
    if (stats) {
        stats->segments = (int32_t)P.segments.size();
        stats->passes = P.passes;
        stats->mass_passes = (int32_t)P.groups.size();
        stats->waves = waves;
        stats->batch_states = (int32_t)B;
        stats->reserved = 0;
        stats->device_seconds = device_ms * 1e-3;
        stats->wall_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - wall0).count();
    }
    return QM_OK;
}
