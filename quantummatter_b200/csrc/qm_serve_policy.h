// qm_serve_policy.h -- admission and batching policy of the request server (qm_serve.cpp).
//
// No device work and no locking: the server holds its mutex around every call.  Header-only so
// that the host tests compile it alone (tests/serve_policy_test.cpp).
//
// Admission: a request reserves the bytes of its state (16 * 2^n for complex128, 8 * 2^n for
// complex64) against the budget; the oldest waiting request that is ready and fits goes first, and
// a younger one passes it only while it does not fit.  A VQE step is ready when its session has no
// step in flight.  Batching: the waiting steps whose sessions share the first step's batch key
// (ansatz structure, Pauli strings, qubits, precision) join its job, up to max_batch, while the
// reservation fits.
#pragma once

#include <cstdint>
#include <deque>
#include <set>
#include <sstream>
#include <string>
#include <vector>

#include "qm_b200.h"

namespace qm {
namespace serve {

// VQE steps batch together when their sessions agree on everything but coefficients and
// parameters: qubits, precision, the ansatz template (gates, constant angles, parameter slots) and
// the Pauli strings of the Hamiltonian in order.
inline std::string batch_key(int32_t qubits, int32_t precision, int32_t parameter_count,
                             const std::vector<qm_template_op>& ops, const std::vector<qm_pauli_term>& terms) {
    std::ostringstream k;
    k.precision(17);
    k << qubits << '/' << precision << '/' << parameter_count << '/';
    for (const qm_template_op& t : ops) {
        const qm_operation& o = t.operation;
        k << o.kind << ',' << o.target << ',' << o.control << ',' << o.second_control << ',' << t.parameter << ',';
        if (t.parameter < 0) k << o.angle << ',';
        if (o.kind == QM_GATE_UNITARY)
            for (double u : o.unitary) k << u << ',';
        k << ';';
    }
    k << '/';
    for (const qm_pauli_term& t : terms) k << t.flip_mask << ',' << t.sign_mask << ',' << t.y_count << ';';
    return k.str();
}

struct Pending {
    int64_t id = 0;
    int64_t bytes = 0;
    int64_t session = -1;  // VQE steps: the session; -1 otherwise
    std::string key;       // VQE steps: the session's batch key
};

struct Job {
    std::vector<Pending> items;
    int64_t bytes = 0;
    bool vqe = false;
};

class Policy {
public:
    Policy(int64_t budget, int max_batch, int lookahead = 64)
        : budget_(budget), max_batch_(max_batch < 1 ? 1 : max_batch), lookahead_(lookahead) {}

    // false when the request can never fit the budget
    bool push(const Pending& p) {
        if (p.bytes > budget_) return false;
        queue_.push_back(p);
        return true;
    }

    bool take(Job& job) {
        job = Job();
        size_t pick = queue_.size();
        for (size_t i = 0; i < queue_.size() && (int)i < lookahead_; ++i)
            if (ready(queue_[i]) && reserved_ + queue_[i].bytes <= budget_) {
                pick = i;
                break;
            }
        if (pick == queue_.size()) return false;
        const Pending head = queue_[pick];
        queue_.erase(queue_.begin() + (std::ptrdiff_t)pick);
        job.items.push_back(head);
        job.bytes = head.bytes;
        job.vqe = head.session >= 0;
        if (job.vqe) {
            busy_.insert(head.session);
            std::deque<Pending> rest;
            while (!queue_.empty()) {
                Pending p = queue_.front();
                queue_.pop_front();
                if ((int)job.items.size() < max_batch_ && p.session >= 0 && p.key == head.key && ready(p) &&
                    reserved_ + job.bytes + p.bytes <= budget_) {
                    busy_.insert(p.session);
                    job.bytes += p.bytes;
                    job.items.push_back(p);
                } else {
                    rest.push_back(p);
                }
            }
            queue_.swap(rest);
        }
        reserved_ += job.bytes;
        if (reserved_ > peak_reserved_) peak_reserved_ = reserved_;
        return true;
    }

    void release(const Job& job) {
        reserved_ -= job.bytes;
        for (const Pending& p : job.items)
            if (p.session >= 0) busy_.erase(p.session);
    }

    // drops every waiting request, returning their ids
    std::vector<int64_t> drain() {
        std::vector<int64_t> ids;
        for (const Pending& p : queue_) ids.push_back(p.id);
        queue_.clear();
        return ids;
    }

    int64_t budget() const { return budget_; }
    int64_t reserved() const { return reserved_; }
    int64_t peak_reserved() const { return peak_reserved_; }
    size_t queued() const { return queue_.size(); }

private:
    bool ready(const Pending& p) const { return p.session < 0 || busy_.count(p.session) == 0; }

    int64_t budget_;
    int max_batch_;
    int lookahead_;
    int64_t reserved_ = 0;
    int64_t peak_reserved_ = 0;
    std::deque<Pending> queue_;
    std::set<int64_t> busy_;
};

}  // namespace serve
}  // namespace qm
