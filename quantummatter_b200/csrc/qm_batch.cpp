// qm_batch.cpp -- batches of states with one shared schedule, tiled Pauli-sum evaluation
// and the batched variational energy/gradient evaluator of libqmb200.so.
//
// VariationalEnergyEvaluator.EvaluateWithGradient (src/QuantumMatter.Application/Variational/
// VariationalEnergyEvaluator.cs:34-86) runs 1 + 2R circuits one after another, each a full
// upload/evolve/download through the backend port followed by one host pass per term.  Here
// every circuit of many parameter vectors is a state of a device batch: the circuits share
// one fused schedule (the template's structure) and differ only in the rotation coefficients,
// which each state reads from a coefficient table.  A parameter-shift circuit appends a
// same-axis rotation after one occurrence (ParameterizedCircuit.cs:87-88); the two rotations
// are combined on the host as the product of their host-prepared matrices, so the shift is
// never added to a possibly huge angle.  Per-term expectations come from the tiled kernel;
// energies and gradients are assembled on the host in the reference's order with its
// Neumaier compensation.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <memory>
#include <numeric>
#include <string>
#include <vector>

#include "qm_internal.h"

using namespace qm;

struct qm_batch {
    qm_context* ctx = nullptr;
    int32_t qubits = 0;
    int32_t precision = QM_FP64;
    int32_t capacity = 0;
    int64_t state_bytes = 0;
    void* amps = nullptr;
    double* table = nullptr;
    size_t table_bytes = 0;
    double* partials = nullptr;
    size_t partial_bytes = 0;
    double* out = nullptr;
    size_t out_bytes = 0;
};

namespace qm {

bool plan_tiles(int qubits, int precision, const qm_pauli_term* terms, int count, TilePlan& plan, std::string& error) {
    plan = TilePlan();
    const int k = tile_block_qubits(qubits, precision);
    if (k < 9) {
        error = "tiled expectation needs at least 9 qubits";
        return false;
    }
    const int low = precision == QM_FP32 ? 4 : 3;
    const int rows = 1 << (qubits - k);
    plan.columns = count + 1;
    plan.mass_column = count;
    std::vector<int> pending(count);
    std::iota(pending.begin(), pending.end(), 0);
    bool first = true;
    int row_offset = 0;
    while (first || !pending.empty()) {
        uint32_t Q;
        std::vector<int> mine, rest;
        if (first) {
            Q = (1u << k) - 1u;
            for (int t : pending) ((terms[t].flip_mask & ~Q) == 0 ? mine : rest).push_back(t);
        } else {
            Q = (1u << low) - 1u;
            for (int t : pending) {
                uint32_t nq = Q | terms[t].flip_mask;
                if (__builtin_popcount(nq) <= k) {
                    Q = nq;
                    mine.push_back(t);
                } else {
                    rest.push_back(t);
                }
            }
            for (int q = 0; q < qubits && __builtin_popcount(Q) < k; ++q) Q |= 1u << q;
            if (mine.empty()) {
                error = "a Pauli flip mask spans more qubits than a tile";
                return false;
            }
        }
        int local_of[32];
        int q_list[kMaxBlockQubits];
        int nb = 0;
        for (int q = 0; q < qubits; ++q) {
            local_of[q] = -1;
            if (Q & (1u << q)) {
                local_of[q] = nb;
                q_list[nb++] = q;
            }
        }
        size_t at = 0;
        do {
            TilePass p{};
            p.k = k;
            for (int i = 0; i < k; ++i) p.q[i] = q_list[i];
            p.block_mask = Q;
            p.term_begin = (int32_t)plan.terms.size();
            p.with_mass = (first && at == 0) ? 1 : 0;
            p.row_offset = row_offset;
            size_t end = std::min(mine.size(), at + (size_t)kTileMaxTerms);
            for (; at < end; ++at) {
                const qm_pauli_term& term = terms[mine[at]];
                uint32_t fl = 0;
                for (int q = 0; q < qubits; ++q)
                    if (term.flip_mask & (1u << q)) fl |= 1u << local_of[q];
                plan.terms.push_back(TileTerm{fl, term.sign_mask, term.y_count & 3, mine[at]});
            }
            p.term_count = (int32_t)plan.terms.size() - p.term_begin;
            // terms sharing a flip mask sit together: the kernel evaluates them as a group
            std::stable_sort(plan.terms.begin() + p.term_begin, plan.terms.end(),
                             [](const TileTerm& x, const TileTerm& y) { return x.flip_local < y.flip_local; });
            plan.passes.push_back(p);
            row_offset += rows;
        } while (at < mine.size());
        first = false;
        pending.swap(rest);
    }
    plan.rows_per_state = row_offset;
    return true;
}

cudaError_t enqueue_tile_expectation(const void* amps, int qubits, int precision, const TilePlan& tp, int states,
                                     double* partials, double* out, cudaStream_t st) {
    const size_t partial = sizeof(double) * (size_t)states * tp.rows_per_state * tp.columns;
    cudaError_t e = cudaMemsetAsync(partials, 0, partial, st);
    for (size_t i = 0; e == cudaSuccess && i < tp.passes.size(); ++i) {
        const void* k = i < tp.jit.size() ? tp.jit[i] : nullptr;
        e = k ? launch_expect_tile_jit(k, amps, qubits, precision, tp.passes[i], states, (uint64_t)1 << qubits, partials,
                                       tp.columns, tp.rows_per_state, tp.mass_column, st)
              : launch_expect_tile(amps, qubits, precision, tp.passes[i], tp.terms.data(), states, (uint64_t)1 << qubits,
                                   partials, tp.columns, tp.rows_per_state, tp.mass_column, st);
    }
    if (e == cudaSuccess) e = launch_finish_batched(partials, states, tp.rows_per_state, tp.columns, out, st);
    return e;
}

}  // namespace qm

namespace {

int32_t check_batch(qm_batch* b) {
    if (!b || !b->ctx) return fail(QM_E_ARG, "batch is null");
    if (b->ctx->disposed) return fail(QM_E_DISPOSED, "context disposed");
    return QM_OK;
}

template <typename T>
int32_t grow(T*& ptr, size_t& have, size_t need) {
    if (have >= need) return QM_OK;
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    have = 0;
    QM_CUDA(cudaMalloc(reinterpret_cast<void**>(&ptr), need));
    have = need;
    return QM_OK;
}

// Enqueues the schedule on `states` states of the batch (no synchronisation).
int32_t enqueue_plan(qm_batch* b, const Plan& plan, int states, const double* d_table, size_t table_stride,
                     cudaStream_t st) {
    FusedBatch fb{states, (uint64_t)1 << b->qubits, d_table, table_stride};
    for (size_t i = 0; i < plan.passes.size(); ++i) QM_CUDA(launch_plan_pass(plan, i, b->amps, &fb, st));
    return QM_OK;
}

// Enqueues the tiled expectation of `states` states into b->out ([states][columns], raw sums
// and the mass in the last column).
int32_t enqueue_tiles(qm_batch* b, const TilePlan& tp, int states, cudaStream_t st) {
    const size_t partial = sizeof(double) * (size_t)states * tp.rows_per_state * tp.columns;
    int32_t rc = grow(b->partials, b->partial_bytes, partial);
    if (rc) return rc;
    rc = grow(b->out, b->out_bytes, sizeof(double) * (size_t)states * tp.columns);
    if (rc) return rc;
    QM_CUDA(enqueue_tile_expectation(b->amps, b->qubits, b->precision, tp, states, b->partials, b->out, st));
    return QM_OK;
}

void cmat(const double* a1, const double* b1, const double* c1, const double* d1, const double* a2, const double* b2,
          const double* c2, const double* d2, double* out) {
    auto mul = [](const double* x, const double* y, double* o) {
        o[0] = x[0] * y[0] - x[1] * y[1];
        o[1] = x[0] * y[1] + x[1] * y[0];
    };
    double t1[2], t2[2];
    mul(a1, a2, t1); mul(b1, c2, t2); out[0] = t1[0] + t2[0]; out[1] = t1[1] + t2[1];
    mul(a1, b2, t1); mul(b1, d2, t2); out[2] = t1[0] + t2[0]; out[3] = t1[1] + t2[1];
    mul(c1, a2, t1); mul(d1, c2, t2); out[4] = t1[0] + t2[0]; out[5] = t1[1] + t2[1];
    mul(c1, b2, t1); mul(d1, d2, t2); out[6] = t1[0] + t2[0]; out[7] = t1[1] + t2[1];
}

}  // namespace

// ====================================================================== batch API

extern "C" int32_t qm_batch_create(qm_context* ctx, int32_t qubits, int32_t precision, int32_t capacity, qm_batch** out) {
    if (!ctx || !out) return fail(QM_E_ARG, "null argument");
    *out = nullptr;
    if (qubits < 9 || qubits > 30) return fail(QM_E_RANGE, "batched states need 9 to 30 qubits");
    if (precision != QM_FP64 && precision != QM_FP32) return fail(QM_E_RANGE, "unknown precision");
    if (capacity < 1 || capacity > 65535) return fail(QM_E_RANGE, "batch capacity must be in [1, 65535]");
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    if (ctx->disposed) return fail(QM_E_DISPOSED, "context disposed");
    const int64_t state_bytes = (precision == QM_FP32 ? 8ll : 16ll) << qubits;
    const int64_t bytes = state_bytes * capacity;
    if (ctx->device_in_use + bytes > ctx->device_budget)
        return fail(QM_E_BUDGET, "batch exceeds the context's device memory budget");
    QM_CUDA(cudaSetDevice(ctx->device));
    std::unique_ptr<qm_batch> b(new qm_batch());
    b->ctx = ctx;
    b->qubits = qubits;
    b->precision = precision;
    b->capacity = capacity;
    b->state_bytes = state_bytes;
    QM_CUDA(cudaMalloc(&b->amps, (size_t)bytes));
    cudaError_t e = launch_reset_batched(b->amps, qubits, precision, capacity, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
        cudaFree(b->amps);
        return cuda_fail(e, "qm_batch_create");
    }
    ctx->device_in_use += bytes;
    *out = b.release();
    return QM_OK;
}

extern "C" int32_t qm_batch_destroy(qm_batch* b) {
    if (!b) return QM_OK;
    if (b->ctx) {
        std::lock_guard<std::recursive_mutex> lock(b->ctx->mu);
        cudaSetDevice(b->ctx->device);
        cudaStreamSynchronize(b->ctx->stream);
        cudaFree(b->amps);
        if (b->table) cudaFree(b->table);
        if (b->partials) cudaFree(b->partials);
        if (b->out) cudaFree(b->out);
        b->ctx->device_in_use -= b->state_bytes * b->capacity;
    }
    delete b;
    return QM_OK;
}

extern "C" int32_t qm_batch_reset(qm_batch* b, int32_t states) {
    int32_t rc = check_batch(b);
    if (rc) return rc;
    if (states < 1 || states > b->capacity) return fail(QM_E_RANGE, "states out of range");
    std::lock_guard<std::recursive_mutex> lock(b->ctx->mu);
    QM_CUDA(cudaSetDevice(b->ctx->device));
    QM_CUDA(launch_reset_batched(b->amps, b->qubits, b->precision, states, b->ctx->stream));
    QM_CUDA(cudaStreamSynchronize(b->ctx->stream));
    return QM_OK;
}

extern "C" int32_t qm_batch_state(qm_batch* b, int32_t index, double* amplitudes, int64_t length, int32_t upload) {
    int32_t rc = check_batch(b);
    if (rc) return rc;
    if (index < 0 || index >= b->capacity) return fail(QM_E_RANGE, "state index out of range");
    if (!amplitudes || length != (int64_t(1) << b->qubits)) return fail(QM_E_ARG, "Buffer length must equal 2^qubitCount.");
    std::lock_guard<std::recursive_mutex> lock(b->ctx->mu);
    qm_context* ctx = b->ctx;
    QM_CUDA(cudaSetDevice(ctx->device));
    char* base = static_cast<char*>(b->amps) + (size_t)index * b->state_bytes;
    if (b->precision == QM_FP64) {
        if (upload) QM_CUDA(cudaMemcpyAsync(base, amplitudes, (size_t)b->state_bytes, cudaMemcpyHostToDevice, ctx->stream));
        else QM_CUDA(cudaMemcpyAsync(amplitudes, base, (size_t)b->state_bytes, cudaMemcpyDeviceToHost, ctx->stream));
    } else {
        double* tmp = nullptr;
        QM_CUDA(cudaMalloc(&tmp, (size_t)(16 * length)));
        cudaError_t e;
        if (upload) {
            e = cudaMemcpyAsync(tmp, amplitudes, (size_t)(16 * length), cudaMemcpyHostToDevice, ctx->stream);
            if (e == cudaSuccess) e = launch_convert_from_f64(base, tmp, length, ctx->stream);
        } else {
            e = launch_convert_to_f64(tmp, base, length, ctx->stream);
            if (e == cudaSuccess) e = cudaMemcpyAsync(amplitudes, tmp, (size_t)(16 * length), cudaMemcpyDeviceToHost, ctx->stream);
        }
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        cudaFree(tmp);
        if (e != cudaSuccess) return cuda_fail(e, "qm_batch_state");
    }
    QM_CUDA(cudaStreamSynchronize(ctx->stream));
    return QM_OK;
}

extern "C" int32_t qm_batch_execute(qm_batch* b, int32_t states, const qm_gate* gates, const int32_t* slots,
                                    int32_t count, const double* table, int32_t slot_count, int32_t width) {
    int32_t rc = check_batch(b);
    if (rc) return rc;
    if (states < 1 || states > b->capacity) return fail(QM_E_RANGE, "states out of range");
    if (count < 0 || (count > 0 && !gates)) return fail(QM_E_ARG, "gates is null");
    if (slot_count < 0 || (slot_count > 0 && !table)) return fail(QM_E_ARG, "coefficient table is null");
    std::vector<qm_gate> list(gates, gates + count);
    std::vector<int32_t> sl((size_t)count, -1);
    for (int32_t i = 0; i < count; ++i) {
        if (slots) sl[(size_t)i] = slots[i];
        if (sl[(size_t)i] >= slot_count) return fail(QM_E_RANGE, "coefficient slot out of range");
    }
    if (slot_count > 0)
        for (int64_t i = 0; i < (int64_t)states * slot_count * 8; ++i)
            if (!std::isfinite(table[i])) return fail(QM_E_RANGE, "coefficients must be finite");
    std::lock_guard<std::recursive_mutex> lock(b->ctx->mu);
    qm_context* ctx = b->ctx;
    QM_CUDA(cudaSetDevice(ctx->device));
    Plan plan;
    std::string err;
    if (width == 0) width = ctx->fusion_width;
    if (!plan_fused(list, b->qubits, b->precision, width, plan, err, &sl)) return fail(QM_E_ARG, "planner: " + err);
    struct Release {
        Plan& p;
        ~Release() { plan_release(p); }
    } release{plan};
    rc = plan_upload(plan, ctx->stream);
    if (rc) return rc;
    const size_t tbytes = sizeof(double) * (size_t)states * slot_count * 8;
    if (tbytes) {
        rc = grow(b->table, b->table_bytes, tbytes);
        if (rc) return rc;
        QM_CUDA(cudaMemcpyAsync(b->table, table, tbytes, cudaMemcpyHostToDevice, ctx->stream));
    }
    rc = enqueue_plan(b, plan, states, tbytes ? b->table : nullptr, (size_t)slot_count * 8, ctx->stream);
    if (rc) {
        cudaStreamSynchronize(ctx->stream);
        return rc;
    }
    QM_CUDA(cudaStreamSynchronize(ctx->stream));
    return QM_OK;
}

extern "C" int32_t qm_batch_expectation(qm_batch* b, int32_t states, const qm_pauli_term* terms, int32_t count,
                                        double* values, double* masses) {
    int32_t rc = check_batch(b);
    if (rc) return rc;
    if (states < 1 || states > b->capacity) return fail(QM_E_RANGE, "states out of range");
    if (count < 0 || (count > 0 && (!terms || !values))) return fail(QM_E_ARG, "null argument");
    const uint32_t all = (uint32_t)((1ull << b->qubits) - 1);
    for (int32_t i = 0; i < count; ++i)
        if ((terms[i].flip_mask | terms[i].sign_mask) & ~all) return fail(QM_E_ARG, "Observable and state sizes must match.");
    std::lock_guard<std::recursive_mutex> lock(b->ctx->mu);
    qm_context* ctx = b->ctx;
    QM_CUDA(cudaSetDevice(ctx->device));
    TilePlan tp;
    std::string err;
    if (!plan_tiles(b->qubits, b->precision, terms, count, tp, err)) return fail(QM_E_ARG, err);
    rc = enqueue_tiles(b, tp, states, ctx->stream);
    if (rc) {
        cudaStreamSynchronize(ctx->stream);
        return rc;
    }
    std::vector<double> host((size_t)states * tp.columns);
    QM_CUDA(cudaMemcpyAsync(host.data(), b->out, sizeof(double) * host.size(), cudaMemcpyDeviceToHost, ctx->stream));
    QM_CUDA(cudaStreamSynchronize(ctx->stream));
    int32_t status = QM_OK;
    for (int32_t s = 0; s < states; ++s) {
        const double mass = host[(size_t)s * tp.columns + tp.mass_column];
        if (masses) masses[s] = mass;
        const bool ok = std::isfinite(mass) && mass > 0;
        if (!ok) status = QM_E_MASS;
        for (int32_t t = 0; t < count; ++t) {
            const double raw = host[(size_t)s * tp.columns + t];
            if (!std::isfinite(raw)) status = QM_E_MASS;
            values[(size_t)s * count + t] = ok ? raw / mass : 0.0;
        }
    }
    if (status) return fail(status, "The state has no finite positive probability mass or a nonfinite observable sum.");
    return QM_OK;
}

// ====================================================================== variational evaluator

namespace {

struct Rotation {
    int op;         // template op index
    int parameter;
    int kind;       // QM_GATE_RX / RY / RZ
};

// Prepared coefficients of a rotation (PreparedStateVectorGate.cs:231-241).
void rotation_coefficients(int kind, double angle, double* c8) {
    qm_operation o{};
    o.kind = kind;
    o.target = 0;
    o.control = -1;
    o.second_control = -1;
    o.angle = angle;
    qm_gate g;
    qm_prepare_gates(&o, 1, 1, &g);
    std::memcpy(c8, g.a, 16);
    std::memcpy(c8 + 2, g.b, 16);
    std::memcpy(c8 + 4, g.c, 16);
    std::memcpy(c8 + 6, g.d, 16);
}

void neumaier_add(double& sum, double& correction, double value) {
    double next = sum + value;
    correction += std::fabs(sum) >= std::fabs(value) ? (sum - next) + value : (value - next) + sum;
    sum = next;
}

}  // namespace

namespace {

// One parameter-shift evaluation problem: a template, a Hamiltonian and `vectors` parameter
// vectors; every base and shifted circuit is a state of this problem's device batch.
// coefficients: [vectors][term_count] per-vector term coefficients, or null for the terms' own.
struct VqeProblem {
    // inputs
    int32_t qubits = 0, precision = QM_FP64;
    const qm_template_op* ops = nullptr;
    int32_t op_count = 0, parameter_count = 0;
    const qm_pauli_term* terms = nullptr;
    int32_t term_count = 0;
    const double* coefficients = nullptr;
    const double* parameters = nullptr;
    int32_t vectors = 0, with_gradient = 0;
    double* energies = nullptr;
    double* gradients = nullptr;
    // derived
    std::vector<qm_gate> gates;
    std::vector<int32_t> slots;
    std::vector<Rotation> rot;
    int R = 0, per_vector = 1, slot_count = 1;
    int64_t circuits = 0;
    int32_t exec_qubits = 0;
    Plan plan;
    TilePlan tp;
    qm_batch* batch = nullptr;
    int B = 0;
    double* h_table[2] = {nullptr, nullptr};
    double* h_out[2] = {nullptr, nullptr};
    std::vector<double> base;
    std::vector<double> results;
    double shift_plus[3][8], shift_minus[3][8];
    int64_t pending_first[2] = {-1, -1};
    int pending_count[2] = {0, 0};
    cudaStream_t stream = nullptr;
    bool own_stream = false;

    VqeProblem() = default;
    VqeProblem(const VqeProblem&) = delete;
    VqeProblem& operator=(const VqeProblem&) = delete;
    ~VqeProblem() {
        plan_release(plan);
        for (int i = 0; i < 2; ++i) {
            if (h_table[i]) cudaFreeHost(h_table[i]);
            if (h_out[i]) cudaFreeHost(h_out[i]);
        }
        if (batch) qm_batch_destroy(batch);
        if (own_stream && stream) cudaStreamDestroy(stream);
    }

    double coef(int v, int t) const {
        return coefficients ? coefficients[(size_t)v * term_count + t] : terms[t].coefficient;
    }
    int64_t state_bytes() const { return (precision == QM_FP32 ? 8ll : 16ll) << exec_qubits; }
    int64_t waves() const { return B ? (circuits + B - 1) / B : 0; }

    // Arguments, template and coefficients (host only).
    int32_t validate() {
        if (qubits < 1 || qubits > 30) return fail(QM_E_RANGE, "qubits must be between 1 and 30");
        if (precision != QM_FP64 && precision != QM_FP32) return fail(QM_E_RANGE, "unknown precision");
        if (op_count < 0 || (op_count > 0 && !ops)) return fail(QM_E_ARG, "template is null");
        if (parameter_count < 0) return fail(QM_E_RANGE, "parameter count must be nonnegative");
        if (vectors < 1) return fail(QM_E_RANGE, "vectors must be positive");
        if (!parameters && parameter_count > 0) return fail(QM_E_ARG, "parameters is null");
        if (!energies) return fail(QM_E_ARG, "energies is null");
        if (with_gradient && parameter_count > 0 && !gradients) return fail(QM_E_ARG, "gradients is null");
        if (term_count < 0 || (term_count > 0 && !terms)) return fail(QM_E_ARG, "terms is null");
        const uint32_t all = (uint32_t)((1ull << qubits) - 1);
        for (int32_t t = 0; t < term_count; ++t) {
            if ((terms[t].flip_mask | terms[t].sign_mask) & ~all)
                return fail(QM_E_ARG, "Circuit and Hamiltonian sizes must match.");
            if (!coefficients && !std::isfinite(terms[t].coefficient)) return fail(QM_E_RANGE, "coefficient must be finite");
        }
        if (coefficients)
            for (int64_t i = 0; i < (int64_t)vectors * term_count; ++i)
                if (!std::isfinite(coefficients[i])) return fail(QM_E_RANGE, "coefficient must be finite");
        for (int64_t i = 0; i < (int64_t)vectors * parameter_count; ++i)
            if (!std::isfinite(parameters[i])) return fail(QM_E_RANGE, "Parameters must be finite.");
        // template: constant gates prepared once; rotations get one coefficient slot each
        gates.assign((size_t)op_count, qm_gate{});
        slots.assign((size_t)op_count, -1);
        rot.clear();
        for (int32_t i = 0; i < op_count; ++i) {
            const qm_template_op& t = ops[i];
            if (t.parameter >= 0) {
                if (t.parameter >= parameter_count) return fail(QM_E_RANGE, "parameter index out of range");
                const int k = t.operation.kind;
                if ((k != QM_GATE_RX && k != QM_GATE_RY && k != QM_GATE_RZ) || t.operation.control != -1 ||
                    t.operation.second_control != -1)
                    return fail(QM_E_ARG, "parameterized operations are uncontrolled Rx, Ry or Rz");
                qm_operation rep = t.operation;
                rep.angle = 1.0;  // fixes the kernel kind (real matrix, complex matrix or diagonal)
                int32_t rc = qm_prepare_gates(&rep, 1, qubits, &gates[(size_t)i]);
                if (rc) return rc;
                slots[(size_t)i] = (int32_t)rot.size();
                rot.push_back(Rotation{i, t.parameter, k});
            } else {
                int32_t rc = qm_prepare_gates(&t.operation, 1, qubits, &gates[(size_t)i]);
                if (rc) return rc;
            }
        }
        R = (int)rot.size();
        per_vector = with_gradient ? 1 + 2 * R : 1;
        circuits = (int64_t)vectors * per_vector;
        slot_count = std::max(R, 1);
        // Registers below the 9-qubit minimum block run embedded in 9 qubits: the extra qubits stay
        // |0> and no term touches them, so energies and gradients are those of the small register.
        exec_qubits = std::max(qubits, 9);
        return QM_OK;
    }

    // Schedule, compiled passes and tile plan (context locked).
    int32_t prepare(qm_context* ctx) {
        std::string err;
        if (!plan_fused(gates, exec_qubits, precision, ctx->fusion_width, plan, err, &slots))
            return fail(QM_E_ARG, "planner: " + err);
        plan.start_zero = true;  // every circuit starts from |0...0>
        jit_prepare(plan);       // one structure for every circuit of every wave
        int32_t rc = plan_upload(plan, ctx->stream);
        if (rc) return rc;
        if (!plan_tiles(exec_qubits, precision, terms, term_count, tp, err)) return fail(QM_E_ARG, err);
        jit_prepare_tiles(tp, exec_qubits, precision);  // one term list for every circuit of every wave
        const double half_pi = M_PI / 2;
        for (int k = 0; k < 3; ++k) {
            rotation_coefficients(QM_GATE_RX + k, half_pi, shift_plus[k]);
            rotation_coefficients(QM_GATE_RX + k, -half_pi, shift_minus[k]);
        }
        base.assign((size_t)vectors * slot_count * 8, 0.0);
        for (int v = 0; v < vectors; ++v)
            for (int r = 0; r < R; ++r)
                rotation_coefficients(rot[(size_t)r].kind,
                                      parameters[(size_t)v * parameter_count + rot[(size_t)r].parameter],
                                      &base[((size_t)v * slot_count + r) * 8]);
        results.assign((size_t)circuits * tp.columns, 0.0);
        return QM_OK;
    }

    // The device batch: as many states as `bytes` allow (at least one), its table, tile partials
    // and pinned host buffers, all at full size before any capture.
    int32_t allocate(qm_context* ctx, int64_t bytes) {
        const int64_t cap = std::min<int64_t>({circuits, 65535, bytes / std::max<int64_t>(state_bytes(), 1), 8192});
        if (cap < 1) return fail(QM_E_BUDGET, "a single state exceeds the context's device memory budget");
        int32_t rc = qm_batch_create(ctx, exec_qubits, precision, (int32_t)cap, &batch);
        if (rc) return rc;
        B = (int)cap;
        const size_t table_doubles = (size_t)B * slot_count * 8;
        rc = grow(batch->table, batch->table_bytes, sizeof(double) * table_doubles);
        if (rc) return rc;
        rc = grow(batch->partials, batch->partial_bytes, sizeof(double) * (size_t)B * tp.rows_per_state * tp.columns);
        if (rc) return rc;
        rc = grow(batch->out, batch->out_bytes, sizeof(double) * (size_t)B * tp.columns);
        if (rc) return rc;
        for (int i = 0; i < 2; ++i) {
            QM_CUDA(cudaMallocHost(reinterpret_cast<void**>(&h_table[i]), sizeof(double) * table_doubles));
            QM_CUDA(cudaMallocHost(reinterpret_cast<void**>(&h_out[i]), sizeof(double) * (size_t)B * tp.columns));
        }
        return QM_OK;
    }

    void fill_table(int buf, int64_t first, int count) {
        double* dst = h_table[buf];
        for (int i = 0; i < count; ++i) {
            const int64_t c = first + i;
            const int v = (int)(c / per_vector), which = (int)(c % per_vector);
            double* row = dst + (size_t)i * slot_count * 8;
            std::memcpy(row, &base[(size_t)v * slot_count * 8], sizeof(double) * slot_count * 8);
            if (which > 0) {
                const int r = (which - 1) / 2;
                const double* shift = ((which - 1) % 2 == 0) ? shift_plus[rot[(size_t)r].kind - QM_GATE_RX]
                                                             : shift_minus[rot[(size_t)r].kind - QM_GATE_RX];
                const double* m = &base[((size_t)v * slot_count + r) * 8];
                // the shift gate is applied after the rotation: combined matrix = shift * rotation
                cmat(shift, shift + 2, shift + 4, shift + 6, m, m + 2, m + 4, m + 6, row + (size_t)r * 8);
            }
        }
    }

    // Coefficient upload, evolution from |0...0>, tiled expectation and the download of the raw
    // sums of `count` circuits, on stream st (capturable: no allocation, no synchronisation).
    int32_t enqueue_wave(int buf, int count, cudaStream_t st) {
        QM_CUDA(cudaMemcpyAsync(batch->table, h_table[buf], sizeof(double) * (size_t)count * slot_count * 8,
                                cudaMemcpyHostToDevice, st));
        if (!plan.zero_fused) QM_CUDA(launch_reset_batched(batch->amps, exec_qubits, precision, count, st));
        int32_t rc = enqueue_plan(batch, plan, count, batch->table, (size_t)slot_count * 8, st);
        if (rc) return rc;
        rc = enqueue_tiles(batch, tp, count, st);
        if (rc) return rc;
        QM_CUDA(cudaMemcpyAsync(h_out[buf], batch->out, sizeof(double) * (size_t)count * tp.columns,
                                cudaMemcpyDeviceToHost, st));
        return QM_OK;
    }

    // after the wave's completion event: its sums into the results
    void collect(int buf) {
        if (pending_first[buf] < 0) return;
        std::memcpy(&results[(size_t)pending_first[buf] * tp.columns], h_out[buf],
                    sizeof(double) * (size_t)pending_count[buf] * tp.columns);
        pending_first[buf] = -1;
    }

    // energies and gradients in the reference's order (StateVector.Energy.cs:22-45,
    // VariationalEnergyEvaluator.cs:45-85)
    int32_t assemble() {
        auto value = [&](int64_t c, int t, double& out) -> bool {
            const double mass = results[(size_t)c * tp.columns + tp.mass_column];
            const double raw = results[(size_t)c * tp.columns + t];
            if (!std::isfinite(mass) || mass <= 0 || !std::isfinite(raw)) return false;
            out = raw / mass;
            return true;
        };
        for (int v = 0; v < vectors; ++v) {
            const int64_t c0 = (int64_t)v * per_vector;
            {
                const double mass = results[(size_t)c0 * tp.columns + tp.mass_column];
                if (!std::isfinite(mass) || mass <= 0)
                    return fail(QM_E_MASS, "The state has no finite positive probability mass.");
            }
            double sum = 0, corr = 0;
            for (int t = 0; t < term_count; ++t) {
                const double ct = coef(v, t);
                if (ct == 0) continue;
                double e;
                if (!value(c0, t, e)) return fail(QM_E_MASS, "The observable accumulation is nonfinite.");
                neumaier_add(sum, corr, ct * e);
                if (!std::isfinite(sum) || !std::isfinite(corr))
                    return fail(QM_E_MASS, "The energy accumulation is nonfinite.");
            }
            const double energy = sum + corr;
            if (!std::isfinite(energy)) return fail(QM_E_MASS, "The energy is nonfinite.");
            energies[v] = energy;
            if (!with_gradient) continue;
            double* grad = gradients + (size_t)v * parameter_count;
            std::vector<double> correction((size_t)parameter_count, 0.0);
            for (int p = 0; p < parameter_count; ++p) grad[p] = 0.0;
            for (int r = 0; r < R; ++r) {
                const int64_t cp = c0 + 1 + 2 * r, cm = cp + 1;
                for (int64_t c : {cp, cm}) {
                    const double mass = results[(size_t)c * tp.columns + tp.mass_column];
                    if (!std::isfinite(mass) || mass <= 0)
                        return fail(QM_E_MASS, "The state has no finite positive probability mass.");
                }
                const int p = rot[(size_t)r].parameter;
                for (int t = 0; t < term_count; ++t) {
                    double plus, minus;
                    if (!value(cp, t, plus) || !value(cm, t, minus))
                        return fail(QM_E_MASS, "The observable accumulation is nonfinite.");
                    const double contribution = coef(v, t) * (0.5 * plus - 0.5 * minus);
                    neumaier_add(grad[p], correction[(size_t)p], contribution);
                    if (!std::isfinite(grad[p]) || !std::isfinite(correction[(size_t)p]))
                        return fail(QM_E_MASS, "The gradient accumulation is nonfinite.");
                }
            }
            for (int p = 0; p < parameter_count; ++p) {
                grad[p] += correction[(size_t)p];
                if (!std::isfinite(grad[p])) return fail(QM_E_MASS, "The gradient is nonfinite.");
            }
        }
        return QM_OK;
    }
};

// Runs problems of any sizes together.  The device budget is shared in proportion to each
// problem's state bytes; in every round each problem runs its next wave, on its own stream when
// there are several (forked from and joined to the context's stream), so the sizes overlap on
// the device.  Rounds in which every problem runs a full wave replay a captured CUDA graph (one
// per host buffer): a single launch covers all sizes of the round.
int32_t run_problems(qm_context* ctx, std::vector<std::unique_ptr<VqeProblem>>& problems, qm_vqe_stats* stats) {
    auto wall0 = std::chrono::steady_clock::now();
    if (!ctx) return fail(QM_E_ARG, "context is null");
    for (auto& p : problems) {
        int32_t rc = p->validate();
        if (rc) return rc;
    }
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    if (ctx->disposed) return fail(QM_E_DISPOSED, "context disposed");
    QM_CUDA(cudaSetDevice(ctx->device));
    for (auto& p : problems) {
        int32_t rc = p->prepare(ctx);
        if (rc) return rc;
    }
    const int64_t free_budget = ctx->device_budget - ctx->device_in_use;
    double total_work = 0;
    for (auto& p : problems) total_work += (double)p->circuits * (double)p->state_bytes();
    for (auto& p : problems) {
        const int64_t share = problems.size() == 1
                                  ? free_budget
                                  : (int64_t)((double)free_budget * ((double)p->circuits * p->state_bytes() / total_work));
        int32_t rc = p->allocate(ctx, share);
        if (rc) return rc;
    }
    const bool multi = problems.size() > 1;
    cudaStream_t main = ctx->stream;
    for (auto& p : problems) {
        if (multi) {
            QM_CUDA(cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking));
            p->own_stream = true;
        } else {
            p->stream = main;
        }
    }
    std::vector<cudaEvent_t> events;
    struct EventGuard {
        std::vector<cudaEvent_t>& e;
        ~EventGuard() {
            for (cudaEvent_t x : e) cudaEventDestroy(x);
        }
    } eg{events};
    auto make_event = [&](unsigned flags, cudaEvent_t* out) -> int32_t {
        QM_CUDA(cudaEventCreateWithFlags(out, flags));
        events.push_back(*out);
        return QM_OK;
    };
    cudaEvent_t done[2], e0, e1, fork;
    std::vector<cudaEvent_t> join(problems.size());
    int32_t rc = make_event(cudaEventDisableTiming, &done[0]);
    if (!rc) rc = make_event(cudaEventDisableTiming, &done[1]);
    if (!rc) rc = make_event(cudaEventDefault, &e0);
    if (!rc) rc = make_event(cudaEventDefault, &e1);
    if (!rc) rc = make_event(cudaEventDisableTiming, &fork);
    for (size_t i = 0; !rc && i < problems.size(); ++i) rc = make_event(cudaEventDisableTiming, &join[i]);
    if (rc) return rc;

    int64_t rounds = 0;
    for (auto& p : problems) rounds = std::max(rounds, p->waves());
    // one round: every active problem's wave, forked from and joined to the context's stream
    auto enqueue_round = [&](int buf, int64_t r) -> int32_t {
        if (multi) QM_CUDA(cudaEventRecord(fork, main));
        for (size_t i = 0; i < problems.size(); ++i) {
            VqeProblem& p = *problems[i];
            if (r >= p.waves()) continue;
            const int count = (int)std::min<int64_t>(p.B, p.circuits - r * p.B);
            if (multi) QM_CUDA(cudaStreamWaitEvent(p.stream, fork, 0));
            int32_t r2 = p.enqueue_wave(buf, count, p.stream);
            if (r2) return r2;
            if (multi) {
                QM_CUDA(cudaEventRecord(join[i], p.stream));
                QM_CUDA(cudaStreamWaitEvent(main, join[i], 0));
            }
        }
        return QM_OK;
    };
    auto full_round = [&](int64_t r) {
        for (auto& p : problems)
            if (r >= p->waves() || (r + 1) * p->B > p->circuits) return false;
        return true;
    };
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    struct GraphGuard {
        cudaGraphExec_t* g;
        ~GraphGuard() {
            for (int i = 0; i < 2; ++i)
                if (g[i]) cudaGraphExecDestroy(g[i]);
        }
    } gg{graph};
    const bool use_graphs = rounds >= 3;
    QM_CUDA(cudaEventRecord(e0, main));
    bool pending[2] = {false, false};
    auto collect = [&](int buf) -> int32_t {
        if (!pending[buf]) return QM_OK;
        QM_CUDA(cudaEventSynchronize(done[buf]));
        for (auto& p : problems) p->collect(buf);
        pending[buf] = false;
        return QM_OK;
    };
    for (int64_t r = 0; r < rounds; ++r) {
        const int buf = (int)(r & 1);
        rc = collect(buf);  // the host buffers of this parity are free again
        if (rc) return rc;
        for (auto& p : problems) {
            if (r >= p->waves()) continue;
            const int64_t first = r * p->B;
            const int count = (int)std::min<int64_t>(p->B, p->circuits - first);
            p->fill_table(buf, first, count);
            p->pending_first[buf] = first;
            p->pending_count[buf] = count;
        }
        if (use_graphs && full_round(r)) {
            if (!graph[buf] && r < 2) {
                // first use of this buffer runs eagerly (configures kernel attributes), then captures
                rc = enqueue_round(buf, r);
                if (rc) {
                    cudaStreamSynchronize(main);
                    return rc;
                }
                QM_CUDA(cudaEventRecord(done[buf], main));
                pending[buf] = true;
                cudaGraph_t g;
                QM_CUDA(cudaStreamSynchronize(main));
                QM_CUDA(cudaStreamBeginCapture(main, cudaStreamCaptureModeThreadLocal));
                int32_t r3 = enqueue_round(buf, r);
                cudaError_t ce = cudaStreamEndCapture(main, &g);
                if (r3) return r3;
                if (ce != cudaSuccess) return cuda_fail(ce, "cudaStreamEndCapture");
                ce = cudaGraphInstantiate(&graph[buf], g, 0);
                cudaGraphDestroy(g);
                if (ce != cudaSuccess) return cuda_fail(ce, "cudaGraphInstantiate");
                continue;
            }
            if (graph[buf]) {
                QM_CUDA(cudaGraphLaunch(graph[buf], main));
            } else {
                rc = enqueue_round(buf, r);
                if (rc) {
                    cudaStreamSynchronize(main);
                    return rc;
                }
            }
        } else {
            rc = enqueue_round(buf, r);
            if (rc) {
                cudaStreamSynchronize(main);
                return rc;
            }
        }
        QM_CUDA(cudaEventRecord(done[buf], main));
        pending[buf] = true;
    }
    rc = collect(0);
    if (rc) return rc;
    rc = collect(1);
    if (rc) return rc;
    QM_CUDA(cudaEventRecord(e1, main));
    QM_CUDA(cudaStreamSynchronize(main));
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    for (auto& p : problems) {
        rc = p->assemble();
        if (rc) return rc;
    }
    if (stats) {
        std::memset(stats, 0, sizeof *stats);
        for (auto& p : problems) {
            stats->circuits += p->circuits;
            stats->batch_states += p->B;
            stats->passes_per_circuit = std::max(stats->passes_per_circuit, (int32_t)p->plan.passes.size());
            stats->tile_passes = std::max(stats->tile_passes, (int32_t)p->tp.passes.size());
        }
        stats->waves = (int32_t)rounds;
        stats->device_seconds = ms * 1e-3;
        stats->wall_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - wall0).count();
    }
    return QM_OK;
}

int32_t vqe_evaluate(qm_context* ctx, int32_t qubits, int32_t precision, const qm_template_op* ops, int32_t op_count,
                     int32_t parameter_count, const qm_pauli_term* terms, int32_t term_count, const double* coefficients,
                     const double* parameters, int32_t vectors, int32_t with_gradient, double* energies,
                     double* gradients, qm_vqe_stats* stats) {
    std::vector<std::unique_ptr<VqeProblem>> problems;
    problems.emplace_back(new VqeProblem());
    VqeProblem& p = *problems[0];
    p.qubits = qubits;
    p.precision = precision;
    p.ops = ops;
    p.op_count = op_count;
    p.parameter_count = parameter_count;
    p.terms = terms;
    p.term_count = term_count;
    p.coefficients = coefficients;
    p.parameters = parameters;
    p.vectors = vectors;
    p.with_gradient = with_gradient;
    p.energies = energies;
    p.gradients = gradients;
    return run_problems(ctx, problems, stats);
}

}  // namespace

extern "C" int32_t qm_vqe_evaluate(qm_context* ctx, int32_t qubits, int32_t precision, const qm_template_op* ops,
                                   int32_t op_count, int32_t parameter_count, const qm_pauli_term* terms,
                                   int32_t term_count, const double* parameters, int32_t vectors, int32_t with_gradient,
                                   double* energies, double* gradients, qm_vqe_stats* stats) {
    return vqe_evaluate(ctx, qubits, precision, ops, op_count, parameter_count, terms, term_count, nullptr, parameters,
                        vectors, with_gradient, energies, gradients, stats);
}

extern "C" int32_t qm_vqe_evaluate_coefficients(qm_context* ctx, int32_t qubits, int32_t precision,
                                                const qm_template_op* ops, int32_t op_count, int32_t parameter_count,
                                                const qm_pauli_term* terms, int32_t term_count,
                                                const double* coefficients, const double* parameters, int32_t vectors,
                                                int32_t with_gradient, double* energies, double* gradients,
                                                qm_vqe_stats* stats) {
    if (term_count > 0 && !coefficients) return fail(QM_E_ARG, "coefficients is null");
    return vqe_evaluate(ctx, qubits, precision, ops, op_count, parameter_count, terms, term_count, coefficients,
                        parameters, vectors, with_gradient, energies, gradients, stats);
}

static_assert(sizeof(qm_vqe_problem) == 80, "qm_vqe_problem layout");

extern "C" int32_t qm_vqe_evaluate_mixed(qm_context* ctx, const qm_vqe_problem* list, int32_t count,
                                         qm_vqe_stats* stats) {
    if (count < 1 || !list) return fail(QM_E_ARG, "problems");
    std::vector<std::unique_ptr<VqeProblem>> problems;
    for (int32_t i = 0; i < count; ++i) {
        const qm_vqe_problem& q = list[i];
        problems.emplace_back(new VqeProblem());
        VqeProblem& p = *problems.back();
        p.qubits = q.qubits;
        p.precision = q.precision;
        p.ops = q.operations;
        p.op_count = q.operation_count;
        p.parameter_count = q.parameter_count;
        p.terms = q.terms;
        p.term_count = q.term_count;
        p.coefficients = q.coefficients;
        p.parameters = q.parameters;
        p.vectors = q.vectors;
        p.with_gradient = q.with_gradient;
        p.energies = q.energies;
        p.gradients = q.gradients;
    }
    return run_problems(ctx, problems, stats);
}
