// TEST INFRASTRUCTURE: the request server's admission and batching policy
// (quantummatter_b200/csrc/qm_serve_policy.h) on the host, scenario by scenario.  Prints one line
// per passed scenario; exits non-zero at the first failure.
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "qm_serve_policy.h"

using qm::serve::Job;
using qm::serve::Pending;
using qm::serve::Policy;

#define CHECK(cond)                                                        \
    do {                                                                   \
        if (!(cond)) {                                                     \
            std::printf("FAIL %s:%d: %s\n", __FILE__, __LINE__, #cond);    \
            std::exit(1);                                                  \
        }                                                                  \
    } while (0)

static int64_t bytes(int qubits, bool fp32 = false) { return (int64_t)(fp32 ? 8 : 16) << qubits; }

static Pending req(int64_t id, int qubits, bool fp32 = false) {
    Pending p;
    p.id = id;
    p.bytes = bytes(qubits, fp32);
    return p;
}

static Pending step(int64_t id, int64_t session, const std::string& key, int qubits, bool fp32 = false) {
    Pending p = req(id, qubits, fp32);
    p.session = session;
    p.key = key;
    return p;
}

static std::vector<int64_t> ids(const Job& j) {
    std::vector<int64_t> out;
    for (const auto& p : j.items) out.push_back(p.id);
    return out;
}

static void reservations_never_exceed_the_budget() {
    Policy s(bytes(12) * 3, 64);
    const int sizes[] = {12, 12, 11, 12, 10};
    for (int i = 0; i < 5; ++i) CHECK(s.push(req(i, sizes[i])));
    std::vector<Job> jobs;
    Job j;
    while (s.take(j)) {
        jobs.push_back(j);
        CHECK(s.reserved() <= s.budget());
    }
    // 12 + 12 + 11 fit; the fourth (12) waits and the 10-qubit one passes it
    CHECK(jobs.size() == 4);
    CHECK(ids(jobs[0]) == std::vector<int64_t>{0} && ids(jobs[1]) == std::vector<int64_t>{1});
    CHECK(ids(jobs[2]) == std::vector<int64_t>{2} && ids(jobs[3]) == std::vector<int64_t>{4});
    CHECK(s.peak_reserved() <= s.budget());
    s.release(jobs[0]);
    CHECK(s.take(j) && ids(j) == std::vector<int64_t>{3} && s.reserved() <= s.budget());
    CHECK(!s.take(j));
    std::puts("ok reservations_never_exceed_the_budget");
}

static void oversized_requests_are_rejected() {
    Policy s(bytes(10), 64);
    CHECK(!s.push(req(0, 11)));
    CHECK(s.push(req(1, 11, true)));  // 8 * 2^11 fits 16 * 2^10
    std::puts("ok oversized_requests_are_rejected");
}

static void vqe_steps_batch_by_key_and_sessions_serialise() {
    Policy s(int64_t(1) << 40, 3);
    // sessions 1, 2, 3: one key; 4: other size; 5: other precision
    const std::string k6 = "6/fp64", k7 = "7/fp64", k6f = "6/fp32";
    std::vector<Pending> order = {step(10, 1, k6, 6), req(11, 6), step(12, 2, k6, 6), step(13, 4, k7, 7),
                                  step(14, 1, k6, 6), step(15, 3, k6, 6), step(16, 5, k6f, 6, true),
                                  step(17, 2, k6, 6)};
    for (const auto& p : order) CHECK(s.push(p));
    Job j1, j2, j3, j4, j5, none;
    CHECK(s.take(j1) && j1.vqe);
    // sessions 1, 2 and 3 share the key; session 1's second step waits for its first
    CHECK(ids(j1) == (std::vector<int64_t>{10, 12, 15}));
    CHECK(s.take(j2) && !j2.vqe && ids(j2) == std::vector<int64_t>{11});
    CHECK(s.take(j3) && ids(j3) == std::vector<int64_t>{13});
    CHECK(s.take(j4) && ids(j4) == std::vector<int64_t>{16});  // the complex64 session: its own batch
    CHECK(!s.take(none));                                      // sessions 1 and 2 are busy
    s.release(j1);
    CHECK(s.take(j5) && ids(j5) == (std::vector<int64_t>{14, 17}));
    CHECK(!s.take(none));
    std::puts("ok vqe_steps_batch_by_key_and_sessions_serialise");
}

static void keys_ignore_coefficients_and_parameters() {
    std::vector<qm_template_op> ops(2);
    ops[0].operation.kind = QM_GATE_RY;
    ops[0].operation.target = 0;
    ops[0].operation.control = ops[0].operation.second_control = -1;
    ops[0].parameter = 0;
    ops[1] = ops[0];
    ops[1].operation.kind = QM_GATE_CNOT;
    ops[1].operation.target = 1;
    ops[1].operation.control = 0;
    ops[1].parameter = -1;
    std::vector<qm_pauli_term> a(2), b;
    a[0].flip_mask = 1;
    a[0].coefficient = 0.5;
    a[1].sign_mask = 3;
    a[1].coefficient = -1.0;
    b = a;
    b[0].coefficient = 2.0;
    CHECK(qm::serve::batch_key(2, QM_FP64, 1, ops, a) == qm::serve::batch_key(2, QM_FP64, 1, ops, b));
    CHECK(qm::serve::batch_key(2, QM_FP64, 1, ops, a) != qm::serve::batch_key(2, QM_FP32, 1, ops, a));
    b[1].sign_mask = 2;
    CHECK(qm::serve::batch_key(2, QM_FP64, 1, ops, a) != qm::serve::batch_key(2, QM_FP64, 1, ops, b));
    auto ops2 = ops;
    ops2[1].operation.angle = 0.25;  // constant angle of a fixed gate: part of the structure
    ops2[1].parameter = -1;
    ops2[1].operation.kind = QM_GATE_RZ;
    ops2[1].operation.control = -1;
    auto ops3 = ops2;
    ops3[1].operation.angle = 0.5;
    CHECK(qm::serve::batch_key(2, QM_FP64, 1, ops2, a) != qm::serve::batch_key(2, QM_FP64, 1, ops3, a));
    std::puts("ok keys_ignore_coefficients_and_parameters");
}

static void drain_returns_waiting_requests() {
    Policy s(bytes(10), 64);
    CHECK(s.push(req(1, 10)) && s.push(req(2, 10)));
    Job j;
    CHECK(s.take(j));
    auto left = s.drain();
    CHECK(left == std::vector<int64_t>{2} && s.queued() == 0);
    std::puts("ok drain_returns_waiting_requests");
}

int main() {
    reservations_never_exceed_the_budget();
    oversized_requests_are_rejected();
    vqe_steps_batch_by_key_and_sessions_serialise();
    keys_ignore_coefficients_and_parameters();
    drain_returns_waiting_requests();
    return 0;
}
