// qm_serve.cpp -- the request server of libqmb200.so (qm_serve_* in include/qm_b200.h).
//
// The reference serves one request at a time: an application calls StateVector.Evolve and
// ExpectationValue (StateVector.Observations.cs:107-141), StateVectorSimulator.Run
// (StateVectorSimulator.cs:37-101) or VariationalEnergyEvaluator.EvaluateWithGradient
// (VariationalEnergyEvaluator.cs:34-86) in sequence.  This server takes a stream of such requests
// from any host thread and runs them concurrently on one GPU:
//   - admission by HBM footprint and VQE batching follow qm_serve_policy.h;
//   - each worker thread owns a context (its own CUDA stream), so jobs of different workers overlap
//     on the device, and keeps device states of recent sizes for reuse;
//   - a VQE session's parameters stay in the server between steps; the waiting steps of sessions
//     that share an ansatz structure and Pauli strings run as one device batch
//     (qm_vqe_evaluate_coefficients), each with its own coefficients and parameters, followed by
//     the steepest-descent update p - step * g with one rounding (VqeSolver.cs:76).
// Every result is the one the request gets alone: requests never share a state, the batched
// evaluator's results do not depend on batch position, and sampling takes the caller's draws.
#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <list>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "qm_internal.h"
#include "qm_serve_policy.h"

static_assert(sizeof(qm_serve_options) == 56 && sizeof(qm_serve_result) == 72 && sizeof(qm_serve_stats) == 80,
              "serving ABI sizes");

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
    int64_t id = 0;
    int32_t kind = 0;
    int32_t qubits = 0, precision = QM_FP64;
    std::vector<qm_gate> gates;
    std::vector<qm_pauli_term> terms;
    std::vector<double> draws;
    int64_t session = -1;
    int64_t bytes = 0;
    // progress and results
    bool done = false;
    int32_t status = QM_OK;
    std::string error;
    int32_t batch = 1, ambiguous = 0;
    double mass = 0.0, energy = 0.0;
    double submitted = 0.0, started = 0.0, finished = 0.0;
    std::vector<double> values;      // expectations, or the VQE gradient
    std::vector<int64_t> outcomes;   // shots
    std::vector<double> parameters;  // the session's parameters after the step
};

struct Session {
    int64_t id = 0;
    int32_t qubits = 0, precision = QM_FP64;
    std::vector<qm_template_op> ops;
    int32_t parameter_count = 0;
    std::vector<qm_pauli_term> terms;
    std::vector<double> coefficients;
    std::vector<double> parameters;
    double step = 0.0;
    std::string key;
    int64_t steps = 0;
    int32_t in_flight = 0;  // steps submitted and not finished
};

// a * b + c with one rounding (Math.FusedMultiplyAdd); plain arithmetic for non-finite inputs
double fused(double a, double b, double c) {
    if (!std::isfinite(a) || !std::isfinite(b) || !std::isfinite(c)) return a * b + c;
    return std::fma(a, b, c);
}

std::string last_error_text() {
    char buf[512];
    qm_last_error(buf, sizeof buf);
    return buf;
}

class Worker {
public:
    Worker(qm_context* ctx, int64_t cache_bytes) : ctx_(ctx), cache_bytes_(cache_bytes) {}

    ~Worker() {
        for (auto& e : states_) qm_state_destroy(e.second);
        if (ctx_) qm_context_destroy(ctx_);
    }

    qm_context* context() const { return ctx_; }

    // a device state of this size at |0...0>, reused when one is cached
    int32_t state(int32_t qubits, int32_t precision, qm_state** out) {
        const std::pair<int32_t, int32_t> key(qubits, precision);
        for (auto it = states_.begin(); it != states_.end(); ++it)
            if (it->first == key) {
                qm_state* st = it->second;
                states_.erase(it);
                states_.emplace_back(key, st);
                *out = st;
                return qm_state_reset(st);
            }
        const int64_t need = (int64_t)(precision == QM_FP32 ? 8 : 16) << qubits;
        while (!states_.empty() && cached_bytes() + need > cache_bytes_) evict();
        qm_state* st = nullptr;
        int32_t rc = qm_state_create(ctx_, qubits, precision, &st);
        while (rc == QM_E_BUDGET && !states_.empty()) {
            evict();
            rc = qm_state_create(ctx_, qubits, precision, &st);
        }
        if (rc) return rc;
        states_.emplace_back(key, st);
        *out = st;
        return QM_OK;
    }

private:
    int64_t cached_bytes() const {
        int64_t b = 0;
        for (const auto& e : states_) b += (int64_t)(e.first.second == QM_FP32 ? 8 : 16) << e.first.first;
        return b;
    }
    void evict() {
        qm_state_destroy(states_.front().second);
        states_.pop_front();
    }

    qm_context* ctx_;
    int64_t cache_bytes_;
    std::list<std::pair<std::pair<int32_t, int32_t>, qm_state*>> states_;  // least recently used first
};

}  // namespace

struct qm_server {
    std::mutex mu;
    std::condition_variable cv;
    qm::serve::Policy policy;
    std::unordered_map<int64_t, std::shared_ptr<Request>> requests;
    std::unordered_map<int64_t, std::shared_ptr<Session>> sessions;
    std::vector<std::unique_ptr<Worker>> workers;
    std::vector<std::thread> threads;
    bool closed = false;
    int64_t next_id = 1;
    Clock::time_point start = Clock::now();
    qm_serve_stats stats{};

    qm_server(int64_t budget, int max_batch) : policy(budget, max_batch) {}

    double now() const { return std::chrono::duration<double>(Clock::now() - start).count(); }

    void run_job(Worker& w, const qm::serve::Job& job);
    void loop(Worker* w);
};

namespace {

int32_t execute_circuit(Worker& w, const Request& r, qm_state** st) {
    int32_t rc = w.state(r.qubits, r.precision, st);
    if (rc) return rc;
    return qm_execute(*st, r.gates.data(), (int32_t)r.gates.size(), 0, nullptr);
}

}  // namespace

void qm_server::run_job(Worker& w, const qm::serve::Job& job) {
    std::vector<std::shared_ptr<Request>> reqs;
    {
        std::lock_guard<std::mutex> lock(mu);
        for (const auto& p : job.items) reqs.push_back(requests.at(p.id));
    }
    const double t_start = now();
    for (auto& r : reqs) r->started = t_start;
    if (!job.vqe) {
        Request& r = *reqs[0];
        qm_state* st = nullptr;
        int32_t rc = execute_circuit(w, r, &st);
        if (rc == QM_OK && r.kind == QM_SERVE_EXPECTATION) {
            r.values.assign(r.terms.size(), 0.0);
            rc = qm_expectation_pauli(st, r.terms.data(), (int32_t)r.terms.size(),
                                      r.values.empty() ? nullptr : r.values.data(), &r.mass);
        } else if (rc == QM_OK) {
            r.outcomes.assign(r.draws.size(), 0);
            rc = qm_sample(st, r.draws.data(), (int32_t)r.draws.size(), r.outcomes.data(), &r.ambiguous);
        }
        r.status = rc;
        if (rc) r.error = last_error_text();
        return;
    }
    // VQE steps of one batch key: one batched evaluation, then each session's update
    std::vector<std::shared_ptr<Session>> ss;
    {
        std::lock_guard<std::mutex> lock(mu);
        for (const auto& p : job.items) ss.push_back(sessions.at(p.session));
    }
    const Session& s0 = *ss[0];
    const int32_t V = (int32_t)ss.size(), P = s0.parameter_count, T = (int32_t)s0.terms.size();
    std::vector<double> params((size_t)V * P), coef((size_t)V * T), energies(V), grads((size_t)V * P);
    for (int32_t v = 0; v < V; ++v) {
        std::copy(ss[v]->parameters.begin(), ss[v]->parameters.end(), params.begin() + (size_t)v * P);
        std::copy(ss[v]->coefficients.begin(), ss[v]->coefficients.end(), coef.begin() + (size_t)v * T);
    }
    const int32_t rc = qm_vqe_evaluate_coefficients(w.context(), s0.qubits, s0.precision, s0.ops.data(),
                                                    (int32_t)s0.ops.size(), P, s0.terms.data(), T, coef.data(),
                                                    params.data(), V, 1, energies.data(), grads.data(), nullptr);
    const std::string err = rc ? last_error_text() : std::string();
    std::lock_guard<std::mutex> lock(mu);
    for (int32_t v = 0; v < V; ++v) {
        Request& r = *reqs[v];
        Session& s = *ss[v];
        r.batch = V;
        r.status = rc;
        if (rc) {
            r.error = err;
            continue;
        }
        r.energy = energies[v];
        r.values.assign(grads.begin() + (size_t)v * P, grads.begin() + (size_t)(v + 1) * P);
        for (int32_t p = 0; p < P; ++p) s.parameters[p] = fused(-s.step, r.values[p], s.parameters[p]);
        s.steps += 1;
        r.parameters = s.parameters;
    }
}

void qm_server::loop(Worker* w) {
    for (;;) {
        qm::serve::Job job;
        {
            std::unique_lock<std::mutex> lock(mu);
            while (!closed && !policy.take(job)) cv.wait(lock);
            if (closed) return;
            stats.running += (int32_t)job.items.size();
            stats.jobs += 1;
            if (job.vqe) {
                stats.vqe_jobs += 1;
                stats.vqe_steps += (int64_t)job.items.size();
                if ((int32_t)job.items.size() > stats.max_batch) stats.max_batch = (int32_t)job.items.size();
            }
        }
        run_job(*w, job);
        const double t_done = now();
        std::lock_guard<std::mutex> lock(mu);
        policy.release(job);
        stats.running -= (int32_t)job.items.size();
        stats.completed += (int64_t)job.items.size();
        for (const auto& p : job.items) {
            auto it = requests.find(p.id);
            if (it == requests.end()) continue;
            it->second->finished = t_done;
            it->second->done = true;
            if (p.session >= 0) {
                auto s = sessions.find(p.session);
                if (s != sessions.end()) s->second->in_flight -= 1;
            }
        }
        cv.notify_all();
    }
}

namespace {

int32_t submit(qm_server* sv, std::shared_ptr<Request> r, const std::string& key, int64_t* out) {
    std::lock_guard<std::mutex> lock(sv->mu);
    if (sv->closed) return qm::fail(QM_E_DISPOSED, "the server is closed");
    r->id = sv->next_id++;
    r->submitted = sv->now();
    qm::serve::Pending p;
    p.id = r->id;
    p.bytes = r->bytes;
    p.session = r->session;
    p.key = key;
    if (!sv->policy.push(p))
        return qm::fail(QM_E_BUDGET, "the request's state exceeds the server's admission budget");
    sv->requests[r->id] = r;
    sv->stats.submitted += 1;
    *out = r->id;
    sv->cv.notify_all();
    return QM_OK;
}

int32_t check_circuit(int32_t qubits, int32_t precision, const qm_operation* ops, int32_t count,
                      std::vector<qm_gate>& gates) {
    if (qubits < 1 || qubits > 30) return qm::fail(QM_E_RANGE, "qubits must be between 1 and 30");
    if (precision != QM_FP64 && precision != QM_FP32) return qm::fail(QM_E_RANGE, "unknown precision");
    if (count < 0 || (count > 0 && !ops)) return qm::fail(QM_E_ARG, "operations");
    gates.resize((size_t)count);
    return count ? qm_prepare_gates(ops, count, qubits, gates.data()) : QM_OK;
}

}  // namespace

extern "C" int32_t qm_serve_create(const qm_serve_options* options, qm_server** out) {
    if (!options || !out) return qm::fail(QM_E_ARG, "null argument");
    *out = nullptr;
    const qm_serve_options& o = *options;
    if (o.workers < 1 || o.workers > 64) return qm::fail(QM_E_RANGE, "workers must be between 1 and 64");
    if (o.budget_bytes <= 0 || o.context_budget_bytes <= 0 || o.cache_bytes < 0)
        return qm::fail(QM_E_RANGE, "budgets must be positive");
    std::unique_ptr<qm_server> sv(new qm_server(o.budget_bytes, o.max_batch > 0 ? o.max_batch : 64));
    for (int32_t i = 0; i < o.workers; ++i) {
        qm_options co;
        qm_options_default(&co);
        co.device_index = o.device_index;
        co.device_budget_bytes = o.context_budget_bytes;
        co.staging_budget_bytes = 1 << 30;
        qm_context* ctx = nullptr;
        const int32_t rc = qm_context_create(&co, &ctx);
        if (rc) return rc;
        sv->workers.emplace_back(new Worker(ctx, o.cache_bytes));
    }
    for (auto& w : sv->workers) sv->threads.emplace_back(&qm_server::loop, sv.get(), w.get());
    *out = sv.release();
    return QM_OK;
}

extern "C" int32_t qm_serve_destroy(qm_server* sv) {
    if (!sv) return QM_OK;
    {
        std::lock_guard<std::mutex> lock(sv->mu);
        sv->closed = true;
        for (int64_t id : sv->policy.drain()) {
            auto it = sv->requests.find(id);
            if (it == sv->requests.end()) continue;
            it->second->status = QM_E_CANCELLED;
            it->second->error = "the server closed before the request ran";
            it->second->done = true;
        }
        sv->cv.notify_all();
    }
    for (auto& t : sv->threads) t.join();
    sv->workers.clear();
    delete sv;
    return QM_OK;
}

extern "C" int32_t qm_serve_submit_expectation(qm_server* sv, int32_t qubits, int32_t precision,
                                               const qm_operation* ops, int32_t count, const qm_pauli_term* terms,
                                               int32_t term_count, int64_t* request) {
    if (!sv || !request) return qm::fail(QM_E_ARG, "null argument");
    if (term_count < 0 || (term_count > 0 && !terms)) return qm::fail(QM_E_ARG, "terms");
    auto r = std::make_shared<Request>();
    int32_t rc = check_circuit(qubits, precision, ops, count, r->gates);
    if (rc) return rc;
    const uint32_t all = (uint32_t)((1ull << qubits) - 1);
    for (int32_t t = 0; t < term_count; ++t)
        if ((terms[t].flip_mask | terms[t].sign_mask) & ~all)
            return qm::fail(QM_E_ARG, "Observable and state sizes must match.");
    r->kind = QM_SERVE_EXPECTATION;
    r->qubits = qubits;
    r->precision = precision;
    r->terms.assign(terms, terms + term_count);
    r->bytes = (int64_t)(precision == QM_FP32 ? 8 : 16) << qubits;
    return submit(sv, r, std::string(), request);
}

extern "C" int32_t qm_serve_submit_shots(qm_server* sv, int32_t qubits, int32_t precision, const qm_operation* ops,
                                         int32_t count, const double* draws, int32_t shots, int64_t* request) {
    if (!sv || !request) return qm::fail(QM_E_ARG, "null argument");
    if (shots < 0 || (shots > 0 && !draws)) return qm::fail(QM_E_ARG, "draws");
    auto r = std::make_shared<Request>();
    int32_t rc = check_circuit(qubits, precision, ops, count, r->gates);
    if (rc) return rc;
    for (int32_t i = 0; i < shots; ++i)
        if (!(draws[i] >= 0.0 && draws[i] < 1.0)) return qm::fail(QM_E_RANGE, "draws must lie in [0, 1)");
    r->kind = QM_SERVE_SHOTS;
    r->qubits = qubits;
    r->precision = precision;
    r->draws.assign(draws, draws + shots);
    r->bytes = (int64_t)(precision == QM_FP32 ? 8 : 16) << qubits;
    return submit(sv, r, std::string(), request);
}

extern "C" int32_t qm_serve_session_create(qm_server* sv, int32_t qubits, int32_t precision,
                                           const qm_template_op* ops, int32_t op_count, int32_t parameter_count,
                                           const qm_pauli_term* terms, int32_t term_count, const double* parameters,
                                           double step_size, int64_t* session) {
    if (!sv || !session || (op_count > 0 && !ops) || (term_count > 0 && !terms) ||
        (parameter_count > 0 && !parameters))
        return qm::fail(QM_E_ARG, "null argument");
    if (qubits < 1 || qubits > 30) return qm::fail(QM_E_RANGE, "qubits must be between 1 and 30");
    if (precision != QM_FP64 && precision != QM_FP32) return qm::fail(QM_E_RANGE, "unknown precision");
    if (op_count < 0 || parameter_count < 0 || term_count < 0) return qm::fail(QM_E_RANGE, "counts");
    if (!(step_size > 0.0) || !std::isfinite(step_size)) return qm::fail(QM_E_RANGE, "step_size must be positive");
    for (int32_t i = 0; i < op_count; ++i)
        if (ops[i].parameter >= parameter_count) return qm::fail(QM_E_RANGE, "parameter index out of range");
    auto s = std::make_shared<Session>();
    s->qubits = qubits;
    s->precision = precision;
    s->ops.assign(ops, ops + op_count);
    s->parameter_count = parameter_count;
    s->terms.assign(terms, terms + term_count);
    for (const auto& t : s->terms) s->coefficients.push_back(t.coefficient);
    s->parameters.assign(parameters, parameters + parameter_count);
    s->step = step_size;
    s->key = qm::serve::batch_key(qubits, precision, parameter_count, s->ops, s->terms);
    std::lock_guard<std::mutex> lock(sv->mu);
    if (sv->closed) return qm::fail(QM_E_DISPOSED, "the server is closed");
    s->id = sv->next_id++;
    sv->sessions[s->id] = s;
    *session = s->id;
    return QM_OK;
}

extern "C" int32_t qm_serve_session_parameters(qm_server* sv, int64_t session, double* parameters, int32_t count,
                                               int64_t* steps) {
    if (!sv) return qm::fail(QM_E_ARG, "null argument");
    std::lock_guard<std::mutex> lock(sv->mu);
    auto it = sv->sessions.find(session);
    if (it == sv->sessions.end()) return qm::fail(QM_E_ARG, "unknown session");
    const Session& s = *it->second;
    if (parameters) {
        if (count < s.parameter_count) return qm::fail(QM_E_RANGE, "parameters buffer too small");
        std::copy(s.parameters.begin(), s.parameters.end(), parameters);
    }
    if (steps) *steps = s.steps;
    return QM_OK;
}

extern "C" int32_t qm_serve_session_destroy(qm_server* sv, int64_t session) {
    if (!sv) return qm::fail(QM_E_ARG, "null argument");
    std::lock_guard<std::mutex> lock(sv->mu);
    auto it = sv->sessions.find(session);
    if (it == sv->sessions.end()) return qm::fail(QM_E_ARG, "unknown session");
    if (it->second->in_flight) return qm::fail(QM_E_ARG, "the session has steps in flight");
    sv->sessions.erase(it);
    return QM_OK;
}

extern "C" int32_t qm_serve_submit_vqe_step(qm_server* sv, int64_t session, int64_t* request) {
    if (!sv || !request) return qm::fail(QM_E_ARG, "null argument");
    std::shared_ptr<Session> s;
    {
        std::lock_guard<std::mutex> lock(sv->mu);
        auto it = sv->sessions.find(session);
        if (it == sv->sessions.end()) return qm::fail(QM_E_ARG, "unknown session");
        s = it->second;
        s->in_flight += 1;
    }
    auto r = std::make_shared<Request>();
    r->kind = QM_SERVE_VQE_STEP;
    r->qubits = s->qubits;
    r->precision = s->precision;
    r->session = session;
    r->bytes = (int64_t)(s->precision == QM_FP32 ? 8 : 16) << s->qubits;
    const int32_t rc = submit(sv, r, s->key, request);
    if (rc) {
        std::lock_guard<std::mutex> lock(sv->mu);
        s->in_flight -= 1;
    }
    return rc;
}

extern "C" int32_t qm_serve_wait(qm_server* sv, int64_t request, double timeout_seconds, int32_t* done) {
    if (!sv) return qm::fail(QM_E_ARG, "null argument");
    std::unique_lock<std::mutex> lock(sv->mu);
    auto it = sv->requests.find(request);
    if (it == sv->requests.end()) return qm::fail(QM_E_ARG, "unknown request");
    std::shared_ptr<Request> r = it->second;
    if (timeout_seconds > 0)
        sv->cv.wait_for(lock, std::chrono::duration<double>(timeout_seconds), [&] { return r->done; });
    if (done) *done = r->done ? 1 : 0;
    return QM_OK;
}

extern "C" int32_t qm_serve_take_result(qm_server* sv, int64_t request, qm_serve_result* result, double* values,
                                        int32_t max_values, int64_t* outcomes, int32_t max_outcomes,
                                        double* parameters, int32_t max_parameters) {
    if (!sv || !result) return qm::fail(QM_E_ARG, "null argument");
    std::shared_ptr<Request> r;
    {
        std::lock_guard<std::mutex> lock(sv->mu);
        auto it = sv->requests.find(request);
        if (it == sv->requests.end()) return qm::fail(QM_E_ARG, "unknown request");
        if (!it->second->done) return qm::fail(QM_E_ARG, "the request has not finished");
        r = it->second;
        const int32_t need_v = (int32_t)r->values.size(), need_o = (int32_t)r->outcomes.size(),
                      need_p = (int32_t)r->parameters.size();
        if ((need_v && (!values || max_values < need_v)) || (need_o && (!outcomes || max_outcomes < need_o)) ||
            (need_p && (!parameters || max_parameters < need_p)))
            return qm::fail(QM_E_RANGE, "output buffers too small for the request's results");
        sv->requests.erase(it);
    }
    std::memset(result, 0, sizeof *result);
    result->kind = r->kind;
    result->status = r->status;
    result->batch = r->batch;
    result->ambiguous = r->ambiguous;
    result->mass = r->mass;
    result->energy = r->energy;
    result->submitted = r->submitted;
    result->started = r->started;
    result->finished = r->finished;
    result->values = (int32_t)r->values.size();
    result->outcomes = (int32_t)r->outcomes.size();
    result->parameters = (int32_t)r->parameters.size();
    if (!r->values.empty()) std::copy(r->values.begin(), r->values.end(), values);
    if (!r->outcomes.empty()) std::copy(r->outcomes.begin(), r->outcomes.end(), outcomes);
    if (!r->parameters.empty()) std::copy(r->parameters.begin(), r->parameters.end(), parameters);
    if (r->status) qm::set_error(r->error);
    return QM_OK;
}

extern "C" int32_t qm_serve_get_stats(qm_server* sv, qm_serve_stats* stats) {
    if (!sv || !stats) return qm::fail(QM_E_ARG, "null argument");
    std::lock_guard<std::mutex> lock(sv->mu);
    *stats = sv->stats;
    stats->queued = (int32_t)sv->policy.queued();
    stats->reserved_bytes = sv->policy.reserved();
    stats->peak_reserved_bytes = sv->policy.peak_reserved();
    stats->budget_bytes = sv->policy.budget();
    return QM_OK;
}
