// qm_dense.cpp -- dense fused gates of at most k qubits (fusion widths 2..6).
//
// The conventional gate-fusion scheme: consecutive gates are merged into fused gates acting on at
// most k qubits, each fused gate is a dense 2^m x 2^m unitary (m <= k) built on the host, and each
// runs as one sweep of the state (qm_dense.cu).  The reference applies one launch per non-identity
// gate (CudaStateVectorBackend.cs:145-160) with the per-gate semantics of
// CpuStateVectorBackend.cs:93-177; the fused unitary is the ordered product of those gates, built
// column by column by applying them to the basis vectors of the m-qubit space.  Gates wider than k
// (a CNOT at k = 1, a Toffoli at k = 2) run alone on the per-gate kernel.
//
// Grouping: a gate may join any group at or after the last group touching one of its qubits (the
// groups after that one share no qubit with it, so it commutes past them), provided the union
// stays within k qubits; the group growing least is chosen, the earliest on ties.  Otherwise it
// opens a new group at the end.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstring>
#include <string>
#include <vector>

#include "qm_internal.h"

namespace qm {

namespace {

using cd = std::complex<double>;

inline int popc(uint32_t x) { return __builtin_popcount(x); }

uint32_t gate_qubits(const qm_gate& g) {
    uint32_t m = (1u << g.target) | g.control_mask;
    if (g.kernel == QM_KERNEL_SWAP) m |= 1u << g.swap_control;
    return m;
}

// local bit of global qubit q in the ascending qubit list of `mask`
int local_bit(uint32_t mask, int q) { return popc(mask & ((1u << q) - 1u)); }

uint32_t local_mask(uint32_t mask, uint32_t global) {
    uint32_t out = 0;
    for (int q = 0; q < 32; ++q)
        if (global & (1u << q)) out |= 1u << local_bit(mask, q);
    return out;
}

// Applies one prepared gate to a vector over the local qubits of `mask` in place, with the
// per-gate semantics of the reference's scalar backend.
void apply_local(const qm_gate& g, uint32_t mask, std::vector<cd>& v) {
    const int m = popc(mask);
    const uint32_t dim = 1u << m;
    const uint32_t t = 1u << local_bit(mask, g.target);
    const uint32_t ctl = local_mask(mask, g.control_mask);
    const cd a(g.a[0], g.a[1]), b(g.b[0], g.b[1]), c(g.c[0], g.c[1]), d(g.d[0], g.d[1]);
    if (g.kernel == QM_KERNEL_SWAP) {
        const uint32_t s = 1u << local_bit(mask, g.swap_control);
        for (uint32_t i = 0; i < dim; ++i)
            if (!(i & t) && (i & s) && (i & ctl) == ctl) std::swap(v[i], v[(i ^ s) | t]);
        return;
    }
    for (uint32_t i = 0; i < dim; ++i) {
        if ((i & t) || (i & ctl) != ctl) continue;
        cd& x = v[i];
        cd& y = v[i | t];
        switch (g.kernel) {
        case QM_KERNEL_MATRIX: {
            const cd x0 = x, y0 = y;
            x = a * x0 + b * y0;
            y = c * x0 + d * y0;
            break;
        }
        case QM_KERNEL_HADAMARD: {
            const double h = g.a[0];
            const cd x0 = x, y0 = y;
            x = cd(h * x0.real() + h * y0.real(), h * x0.imag() + h * y0.imag());
            y = cd(h * x0.real() - h * y0.real(), h * x0.imag() - h * y0.imag());
            break;
        }
        case QM_KERNEL_EXCHANGE: std::swap(x, y); break;
        case QM_KERNEL_DIAGONAL:
            x = a * x;
            y = d * y;
            break;
        default: break;
        }
    }
}

struct Group {
    bool dense;
    uint32_t mask;
    std::vector<qm_gate> gates;
};

bool trivial(const qm_gate& g) {
    if (g.kernel == QM_KERNEL_IDENTITY) return true;
    return g.kernel == QM_KERNEL_DIAGONAL && g.a[0] == 1.0 && g.a[1] == 0.0 && g.d[0] == 1.0 && g.d[1] == 0.0;
}

}  // namespace

bool plan_dense(const std::vector<qm_gate>& gates, int qubits, int precision, int width, Plan& plan,
                std::string& error) {
    if (width < 1 || width > kDenseMaxQubits) {
        error = "dense fusion widths are 1 to 6 qubits";
        return false;
    }
    plan.qubits = qubits;
    plan.precision = precision;
    plan.width = width;
    plan.passes.clear();
    plan.ops.clear();
    plan.gates.clear();
    plan.dense.clear();
    plan.dense_matrices.clear();
    plan.dense_tc.clear();
    plan.planned_bytes = 0;
    plan.launches = 0;
    const int64_t elem = precision == QM_FP32 ? 8 : 16;
    const int64_t n = int64_t(1) << qubits;

    std::vector<Group> groups;
    std::vector<int> last(32, -1);
    for (const qm_gate& g : gates) {
        if (trivial(g)) continue;
        if (g.kernel == QM_KERNEL_SWAP && (g.swap_control < 0 || g.swap_control == g.target)) {
            error = "swap operands must be distinct";
            return false;
        }
        const uint32_t qs = gate_qubits(g);
        int cand = -1;
        for (int q = 0; q < 32; ++q)
            if (qs & (1u << q)) cand = std::max(cand, last[q]);
        int chosen = -1;
        if (popc(qs) <= width) {
            int best_growth = 1 << 30;
            for (int i = std::max(cand, 0); i < (int)groups.size(); ++i) {
                if (!groups[i].dense) continue;
                const uint32_t u = groups[i].mask | qs;
                if (popc(u) > width) continue;
                const int growth = popc(u) - popc(groups[i].mask);
                if (growth < best_growth) {
                    best_growth = growth;
                    chosen = i;
                }
            }
        }
        if (chosen < 0) {
            groups.push_back(Group{popc(qs) <= width, qs, {}});
            chosen = (int)groups.size() - 1;
        }
        groups[chosen].mask |= qs;
        groups[chosen].gates.push_back(g);
        for (int q = 0; q < 32; ++q)
            if (qs & (1u << q)) last[q] = chosen;
    }

    for (const Group& gr : groups) {
        DenseOp op{};
        op.gates = (int32_t)gr.gates.size();
        if (!gr.dense) {
            op.m = 0;
            op.gate = to_dev_gate(gr.gates[0]);
            const DevGate& d = op.gate;
            const int active = popc(d.target_bit | d.control_mask | d.swap_bit);
            int64_t touched = 2 * (n >> active);
            if (d.kernel == QM_KERNEL_DIAGONAL && (d.a_is_one || d.d_is_one)) touched /= 2;
            plan.planned_bytes += 2 * touched * elem;
        } else {
            uint32_t mask = gr.mask;
            // complex64 5-qubit gates join the tensor-core path as 6-qubit gates (U x I on one more
            // qubit): the extra multiply-adds are cheap there, the FP32 pipes are not.  The qubit next
            // to the group keeps its bits in one run (a scattered one would split the tile's copies).
            if (precision == QM_FP32 && popc(mask) == 5 && qubits >= 11 && dense_tc_enabled()) {
                const int top = 31 - __builtin_clz(mask), bottom = __builtin_ctz(mask);
                if (top + 1 < qubits)
                    mask |= 1u << (top + 1);
                else if (bottom > 0)
                    mask |= 1u << (bottom - 1);
                else
                    for (int q = 0; q < qubits; ++q)
                        if (!(mask & (1u << q))) {
                            mask |= 1u << q;
                            break;
                        }
            }
            const int m = popc(mask);
            op.m = m;
            op.tc_image = -1;
            int i = 0;
            for (int q = 0; q < 32; ++q)
                if (mask & (1u << q)) op.q[i++] = q;
            // Transposed unitary: row j is the image of basis vector j (column j of U), so the
            // kernel reads U(a, b) for consecutive a as one contiguous row.
            const uint32_t dim = 1u << m;
            op.matrix = (int64_t)plan.dense_matrices.size() / 2;
            std::vector<cd> v(dim);
            for (uint32_t j = 0; j < dim; ++j) {
                std::fill(v.begin(), v.end(), cd(0.0, 0.0));
                v[j] = cd(1.0, 0.0);
                for (const qm_gate& g : gr.gates) apply_local(g, mask, v);
                for (uint32_t a = 0; a < dim; ++a) {
                    if (!std::isfinite(v[a].real()) || !std::isfinite(v[a].imag())) {
                        error = "fused gate has non-finite coefficients";
                        return false;
                    }
                    plan.dense_matrices.push_back(v[a].real());
                    plan.dense_matrices.push_back(v[a].imag());
                }
            }
            if (dense_tc_supported(qubits, precision, op)) {
                std::vector<float> image;
                dense_tc_image(plan.dense_matrices.data() + 2 * op.matrix, image);
                op.tc_image = (int64_t)plan.dense_tc.size();
                plan.dense_tc.insert(plan.dense_tc.end(), image.begin(), image.end());
            }
            plan.planned_bytes += 2 * n * elem;
        }
        plan.dense.push_back(op);
    }
    plan.launches = (int32_t)plan.dense.size();
    return true;
}

}  // namespace qm
