/*
 * qm_oracle.c -- TEST INFRASTRUCTURE: CPU restatement of QuantumMatter's scalar path.
 *
 * This file is the oracle the CUDA library is checked against.  It is not shipped
 * and the product path never calls it.  Build: oracle/Makefile (gcc -O2
 * -ffp-contract=off, so that products are rounded separately, as .NET's
 * System.Numerics.Complex does).  Reference file paths are inside the
 * olgerd007/QuantumMatter project.
 */
#include "qm_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef struct { double re, im; } cpx;

/* System.Numerics.Complex multiplication: (ac - bd, bc + ad), rounded per product. */
static inline cpx cmul(cpx l, cpx r) {
    cpx o;
    o.re = l.re * r.re - l.im * r.im;
    o.im = l.im * r.re + l.re * r.im;
    return o;
}
static inline cpx cadd(cpx l, cpx r) { cpx o = { l.re + r.re, l.im + r.im }; return o; }
static inline cpx mk(double re, double im) { cpx o = { re, im }; return o; }
static inline cpx ld(const double* amps, int64_t i) { return mk(amps[2 * i], amps[2 * i + 1]); }
static inline void st(double* amps, int64_t i, cpx v) { amps[2 * i] = v.re; amps[2 * i + 1] = v.im; }
/* Complex.FromPolarCoordinates(1, phase) */
static inline cpx polar1(double phase) { return mk(cos(phase), sin(phase)); }

/* ---------------------------------------------------------------- validation */

/* Builder validation of src/QuantumMatter.Core/QuantumCircuit.cs:97-134: operands in
 * range and distinct, finite angle.  Returns 0, 1 (argument) or 10 (range). */
int qmo_validate(const qmo_operation* ops, int32_t count, int32_t qubits) {
    if (qubits < 1 || qubits > 30) return 10;
    for (int32_t g = 0; g < count; ++g) {
        const qmo_operation* o = &ops[g];
        if (o->kind < 0 || o->kind > QMO_TOFFOLI) return 9;
        if ((uint32_t)o->target >= (uint32_t)qubits) return 10;
        if (o->control >= 0) {
            if (o->control >= qubits) return 10;
            if (o->control == o->target) return 1;
        } else if (o->control != -1) return 10;
        if (o->second_control >= 0) {
            if (o->second_control >= qubits) return 10;
            if (o->second_control == o->target || o->second_control == o->control) return 1;
        } else if (o->second_control != -1) return 10;
        if (!isfinite(o->angle)) return 10;
        if ((o->kind == QMO_CNOT || o->kind == QMO_SWAP) && o->control < 0) return 1;
        if (o->kind == QMO_TOFFOLI && (o->control < 0 || o->second_control < 0)) return 1;
    }
    return 0;
}

/* ---------------------------------------------------------------- scalar backend */

/* CpuStateVectorBackend.ApplyMatrix (src/QuantumMatter.Infrastructure/CpuStateVectorBackend.cs:93-118) */
static void apply_matrix(double* s, int64_t len, int target, cpx a, cpx b, cpx c, cpx d, int64_t cmask) {
    int64_t bit = (int64_t)1 << target;
    for (int64_t pair = 0; pair < len / 2; ++pair) {
        int64_t low = pair & (bit - 1);
        int64_t first = ((pair - low) << 1) | low;
        if ((first & cmask) != cmask) continue;
        int64_t second = first | bit;
        cpx x = ld(s, first), y = ld(s, second);
        st(s, first, cadd(cmul(a, x), cmul(b, y)));
        st(s, second, cadd(cmul(c, x), cmul(d, y)));
    }
}

/* CpuStateVectorBackend.ApplyX (:120-140) -- X, CNOT and Toffoli */
static void apply_x(double* s, int64_t len, int target, int64_t cmask) {
    int64_t bit = (int64_t)1 << target;
    for (int64_t pair = 0; pair < len / 2; ++pair) {
        int64_t low = pair & (bit - 1);
        int64_t first = ((pair - low) << 1) | low;
        if ((first & cmask) != cmask) continue;
        int64_t second = first | bit;
        cpx x = ld(s, first), y = ld(s, second);
        st(s, first, y);
        st(s, second, x);
    }
}

/* CpuStateVectorBackend.ApplyDiagonal (:142-158) */
static void apply_diagonal(double* s, int64_t len, int target, cpx zero, cpx one, int64_t cmask) {
    int64_t bit = (int64_t)1 << target;
    for (int64_t i = 0; i < len; ++i) {
        if ((i & cmask) == cmask) st(s, i, cmul(ld(s, i), (i & bit) == 0 ? zero : one));
    }
}

/* CpuStateVectorBackend.ApplySwap (:160-177) */
static void apply_swap(double* s, int64_t len, int control, int target) {
    int64_t cb = (int64_t)1 << control, tb = (int64_t)1 << target;
    for (int64_t i = 0; i < len; ++i) {
        if ((i & cb) != 0 && (i & tb) == 0) {
            int64_t other = i ^ cb ^ tb;
            cpx x = ld(s, i), y = ld(s, other);
            st(s, i, y);
            st(s, other, x);
        }
    }
}

/* CpuStateVectorBackend.Execute (:10-91): coefficients built inline per gate. */
void qmo_execute(const qmo_operation* ops, int32_t count, int32_t qubits, double* amps) {
    int64_t len = (int64_t)1 << qubits;
    for (int32_t g = 0; g < count; ++g) {
        const qmo_operation* o = &ops[g];
        int64_t cmask = o->control >= 0 ? ((int64_t)1 << o->control) : 0;
        if (o->second_control >= 0) cmask |= (int64_t)1 << o->second_control;
        switch (o->kind) {
        case QMO_I: break;
        case QMO_CNOT: case QMO_TOFFOLI: case QMO_X:
            apply_x(amps, len, o->target, cmask); break;
        case QMO_SWAP:
            apply_swap(amps, len, o->control, o->target); break;
        case QMO_H: {
            double h = sqrt(0.5);
            apply_matrix(amps, len, o->target, mk(h, 0), mk(h, 0), mk(h, 0), mk(-h, 0), cmask);
            break;
        }
        case QMO_Y:
            apply_matrix(amps, len, o->target, mk(0, 0), mk(-0.0, -1), mk(0, 1), mk(0, 0), cmask); break;
        case QMO_Z:
            apply_diagonal(amps, len, o->target, mk(1, 0), mk(-1, 0), cmask); break;
        case QMO_S:
            apply_diagonal(amps, len, o->target, mk(1, 0), mk(0, 1), cmask); break;
        case QMO_SDG:
            apply_diagonal(amps, len, o->target, mk(1, 0), mk(-0.0, -1), cmask); break;
        case QMO_T: case QMO_TDG: case QMO_PHASE: {
            double phase = o->kind == QMO_T ? M_PI / 4 : o->kind == QMO_TDG ? -M_PI / 4 : o->angle;
            apply_diagonal(amps, len, o->target, mk(1, 0), polar1(phase), cmask);
            break;
        }
        case QMO_RX: case QMO_RY: {
            double cosine = cos(o->angle / 2), sine = sin(o->angle / 2);
            /* -i * sine for Rx (Complex product -ImaginaryOne * sine), -sine / sine for Ry */
            cpx upper = o->kind == QMO_RX ? mk(-0.0 * sine, -1.0 * sine) : mk(-sine, 0);
            cpx lower = o->kind == QMO_RX ? upper : mk(sine, 0);
            apply_matrix(amps, len, o->target, mk(cosine, 0), upper, lower, mk(cosine, 0), cmask);
            break;
        }
        case QMO_RZ:
            apply_diagonal(amps, len, o->target, polar1(-o->angle / 2), polar1(o->angle / 2), cmask); break;
        case QMO_UNITARY: {
            const double* u = o->unitary;
            apply_matrix(amps, len, o->target, mk(u[0], u[1]), mk(u[2], u[3]), mk(u[4], u[5]), mk(u[6], u[7]), cmask);
            break;
        }
        default: break;
        }
    }
}

/* ---------------------------------------------------------------- prepared gates */

/* PreparedStateVectorGate.Prepare (src/QuantumMatter.Infrastructure/PreparedStateVectorGate.cs:13-70) */
int qmo_prepare(const qmo_operation* ops, int32_t count, qmo_gate* out) {
    for (int32_t g = 0; g < count; ++g) {
        const qmo_operation* o = &ops[g];
        qmo_gate* p = &out[g];
        memset(p, 0, sizeof(*p));
        uint32_t mask = o->control >= 0 ? (1u << o->control) : 0u;
        if (o->second_control >= 0) mask |= 1u << o->second_control;
        p->target = o->target;
        p->control_mask = mask;
        p->swap_control = -1;
        cpx a = mk(0, 0), b = mk(0, 0), c = mk(0, 0), d = mk(0, 0);
        int kernel = QMO_K_MATRIX;
        switch (o->kind) {
        case QMO_I: kernel = QMO_K_IDENTITY; break;
        case QMO_X: case QMO_CNOT: case QMO_TOFFOLI: kernel = QMO_K_EXCHANGE; break;
        case QMO_SWAP: kernel = QMO_K_SWAP; p->control_mask = 0; p->swap_control = o->control; break;
        case QMO_H: { double h = sqrt(0.5); kernel = QMO_K_HADAMARD; a = b = c = mk(h, 0); d = mk(-h, 0); break; }
        case QMO_Y: b = mk(-0.0, -1); c = mk(0, 1); break;
        case QMO_Z: kernel = QMO_K_DIAGONAL; a = mk(1, 0); d = mk(-1, 0); break;
        case QMO_S: kernel = QMO_K_DIAGONAL; a = mk(1, 0); d = mk(0, 1); break;
        case QMO_SDG: kernel = QMO_K_DIAGONAL; a = mk(1, 0); d = mk(-0.0, -1); break;
        case QMO_T: kernel = QMO_K_DIAGONAL; a = mk(1, 0); d = polar1(M_PI / 4); break;
        case QMO_TDG: kernel = QMO_K_DIAGONAL; a = mk(1, 0); d = polar1(-M_PI / 4); break;
        case QMO_PHASE: kernel = QMO_K_DIAGONAL; a = mk(1, 0); d = polar1(o->angle); break;
        case QMO_RX: {
            double xc = cos(o->angle / 2);
            cpx xs = mk(-0.0 * sin(o->angle / 2), -1.0 * sin(o->angle / 2));
            a = mk(xc, 0); b = xs; c = xs; d = mk(xc, 0);
            break;
        }
        case QMO_RY: {
            double yc = cos(o->angle / 2), ys = sin(o->angle / 2);
            a = mk(yc, 0); b = mk(-ys, 0); c = mk(ys, 0); d = mk(yc, 0);
            break;
        }
        case QMO_RZ: kernel = QMO_K_DIAGONAL; a = polar1(-o->angle / 2); d = polar1(o->angle / 2); break;
        case QMO_UNITARY: {
            const double* u = o->unitary;
            a = mk(u[0], u[1]); b = mk(u[2], u[3]); c = mk(u[4], u[5]); d = mk(u[6], u[7]);
            break;
        }
        default: return 9;
        }
        p->kernel = kernel;
        p->a[0] = a.re; p->a[1] = a.im; p->b[0] = b.re; p->b[1] = b.im;
        p->c[0] = c.re; p->c[1] = c.im; p->d[0] = d.re; p->d[1] = d.im;
    }
    return 0;
}

/* Scalar branch of ParallelCpuStateVectorBackend.ApplyRange
 * (src/QuantumMatter.Infrastructure/ParallelCpuStateVectorBackend.cs:278-333), which is the
 * same per-pair arithmetic as the reference CUDA kernel (CudaStateVectorKernel.cs:38-77). */
void qmo_apply_prepared(const qmo_gate* gates, int32_t count, int32_t qubits, double* s) {
    int64_t len = (int64_t)1 << qubits;
    for (int32_t g = 0; g < count; ++g) {
        const qmo_gate* p = &gates[g];
        if (p->kernel == QMO_K_IDENTITY) continue;
        int64_t bit = (int64_t)1 << p->target;
        int64_t cmask = p->control_mask;
        cpx a = mk(p->a[0], p->a[1]), b = mk(p->b[0], p->b[1]);
        cpx c = mk(p->c[0], p->c[1]), d = mk(p->d[0], p->d[1]);
        if (p->kernel == QMO_K_DIAGONAL) {
            for (int64_t i = 0; i < len; ++i)
                if ((i & cmask) == cmask) st(s, i, cmul(ld(s, i), (i & bit) == 0 ? a : d));
            continue;
        }
        int64_t swap_bit = p->kernel == QMO_K_SWAP ? ((int64_t)1 << p->swap_control) : 0;
        for (int64_t pair = 0; pair < len / 2; ++pair) {
            int64_t low = pair & (bit - 1);
            int64_t first = ((pair - low) << 1) | low;
            if ((first & cmask) != cmask) continue;
            int64_t second = first | bit;
            if (p->kernel == QMO_K_SWAP) {
                if ((first & swap_bit) == 0) continue;
                second ^= swap_bit;
            }
            cpx x = ld(s, first), y = ld(s, second);
            if (p->kernel == QMO_K_SWAP || p->kernel == QMO_K_EXCHANGE) {
                st(s, first, y); st(s, second, x);
            } else {
                st(s, first, cadd(cmul(a, x), cmul(b, y)));
                st(s, second, cadd(cmul(c, x), cmul(d, y)));
            }
        }
    }
}

/* ---------------------------------------------------------------- observables */

/* StateVector.ExpectationValue (src/QuantumMatter.Core/StateVector.Observations.cs:107-141).
 * Returns the raw sequential sum; *mass_out receives the Born mass of the same pass.
 * The normalised value is raw / mass. */
double qmo_expectation(const double* s, int32_t qubits, uint32_t flip, uint32_t sign,
                       int32_t ycount, double* mass_out) {
    int64_t len = (int64_t)1 << qubits;
    double total = 0, expectation = 0;
    for (int64_t i = 0; i < len; ++i) {
        cpx v = ld(s, i);
        total += v.re * v.re + v.im * v.im;
        cpx partner = ld(s, i ^ (int64_t)flip);
        cpx conj = mk(partner.re, -partner.im);
        cpx overlap = cmul(conj, v);
        double contribution;
        switch (ycount & 3) {
        case 0: contribution = overlap.re; break;
        case 1: contribution = -overlap.im; break;
        case 2: contribution = -overlap.re; break;
        default: contribution = overlap.im; break;
        }
        expectation += (__builtin_popcountll((uint64_t)(i & (int64_t)sign)) & 1) == 0 ? contribution : -contribution;
    }
    if (mass_out) *mass_out = total;
    return expectation;
}

/* StateVector.ExpectationEnergy (src/QuantumMatter.Core/StateVector.Energy.cs:10-46):
 * mass validation pass, then per nonzero term c * <P>, Neumaier-summed in term order.
 * Returns 0 or 7 (no finite positive mass / nonfinite accumulation). */
int qmo_energy(const double* s, int32_t qubits, const uint32_t* flip, const uint32_t* sign,
               const int32_t* ycount, const double* coeff, int32_t terms, double* energy_out) {
    int64_t len = (int64_t)1 << qubits;
    double mass = 0;
    for (int64_t i = 0; i < len; ++i) { cpx v = ld(s, i); mass += v.re * v.re + v.im * v.im; }
    if (!isfinite(mass) || mass <= 0) return 7;
    double sum = 0, correction = 0;
    for (int32_t t = 0; t < terms; ++t) {
        if (coeff[t] == 0) continue;
        double total;
        double raw = qmo_expectation(s, qubits, flip[t], sign[t], ycount[t], &total);
        if (!isfinite(total) || total <= 0) return 7;
        if (!isfinite(raw)) return 7;
        double value = coeff[t] * (raw / total);
        double next = sum + value;
        correction += fabs(sum) >= fabs(value) ? (sum - next) + value : (value - next) + sum;
        sum = next;
        if (!isfinite(sum) || !isfinite(correction)) return 7;
    }
    double energy = sum + correction;
    if (!isfinite(energy)) return 7;
    *energy_out = energy;
    return 0;
}

/* ---------------------------------------------------------------- noise */

static void add_mass(double value, double* sum, double* compensation) {
    double corrected = value - *compensation;
    double next = *sum + corrected;
    *compensation = (next - *sum) - corrected;
    *sum = next;
}

/* Kahan masses of CpuNoiseChannelBackend.ApplyDamping (CpuNoiseChannelBackend.cs:88-106) */
void qmo_qubit_masses(const double* s, int32_t qubits, int32_t target, double* m0, double* m1) {
    int64_t len = (int64_t)1 << qubits, bit = (int64_t)1 << target;
    double zm = 0, om = 0, zc = 0, oc = 0;
    for (int64_t i = 0; i < len; ++i) {
        cpx v = ld(s, i);
        double mass = v.re * v.re + v.im * v.im;
        if ((i & bit) == 0) add_mass(mass, &zm, &zc); else add_mass(mass, &om, &oc);
    }
    *m0 = zm; *m1 = om;
}

/* CpuNoiseChannelBackend.Apply / ApplyDamping (src/QuantumMatter.Infrastructure/CpuNoiseChannelBackend.cs:10-145) */
/* *branch: -1 for p == 0 (nothing happens), Pauli 0..3 = I, X, Y, Z, damping 0 = stay, 1 = jump. */
static int noise_apply(int32_t kind, double p, int32_t target, double* s, int32_t qubits, const double* draws,
                       int32_t ndraws, int32_t* used, int32_t* branch) {
    int64_t len = (int64_t)1 << qubits, bit = (int64_t)1 << target;
    int32_t consumed = 0;
#define NEXT_DRAW() (consumed < ndraws ? draws[consumed++] : (consumed++, 0.0))
    if (used) *used = 0;
    *branch = -1;
    if (p == 0) return 0;
    if (kind == 3) {
        double zero_mass, one_mass;
        qmo_qubit_masses(s, qubits, target, &zero_mass, &one_mass);
        double jump_mass = p * one_mass;
        double stay_mass = zero_mass + (1 - p) * one_mass;
        double total = jump_mass + stay_mass;
        if (!isfinite(total) || total <= 0) return 7;
        int jump = jump_mass > 0 && (stay_mass == 0 || NEXT_DRAW() < jump_mass / total);
        *branch = jump;
        double branch_mass = jump ? jump_mass : stay_mass;
        double scale = 1 / sqrt(branch_mass);
        double jump_scale = sqrt(p) * scale;
        double stay_scale = sqrt(1 - p) * scale;
        for (int64_t pair = 0; pair < len / 2; ++pair) {
            int64_t low = pair & (bit - 1);
            int64_t first = ((pair - low) << 1) | low;
            int64_t second = first | bit;
            if (jump) {
                cpx y = ld(s, second);
                st(s, first, mk(jump_scale * y.re, jump_scale * y.im));
                st(s, second, mk(0, 0));
            } else {
                cpx x = ld(s, first), y = ld(s, second);
                st(s, first, mk(x.re * scale, x.im * scale));
                st(s, second, mk(y.re * stay_scale, y.im * stay_scale));
            }
        }
        if (used) *used = consumed;
        return 0;
    }
    int pauli;
    if (kind == 2) {
        double draw = NEXT_DRAW();
        double quarter = p / 4;
        pauli = draw < quarter ? 1 : draw < 2 * quarter ? 2 : draw < 3 * quarter ? 3 : 0;
    } else {
        int apply = p == 1 || NEXT_DRAW() < p;
        pauli = !apply ? 0 : kind == 0 ? 1 : 3;
    }
    if (used) *used = consumed;
    *branch = pauli;
    if (pauli == 0) return 0;
    for (int64_t pair = 0; pair < len / 2; ++pair) {
        int64_t low = pair & (bit - 1);
        int64_t first = ((pair - low) << 1) | low;
        int64_t second = first | bit;
        cpx zero = ld(s, first), one = ld(s, second);
        if (pauli == 3) {
            st(s, second, mk(-one.re, -one.im));
        } else {
            st(s, first, pauli == 1 ? one : mk(one.im, -one.re));
            st(s, second, pauli == 1 ? zero : mk(-zero.im, zero.re));
        }
    }
    return 0;
#undef NEXT_DRAW
}

int qmo_noise_apply(int32_t kind, double p, int32_t target, double* s, int32_t qubits,
                    const double* draws, int32_t ndraws, int32_t* used) {
    int32_t branch;
    return noise_apply(kind, p, target, s, qubits, draws, ndraws, used, &branch);
}

/* One trajectory of NoisyCircuit.Execute (src/QuantumMatter.Core/Noise/NoisyCircuit.cs:48-65)
 * through CpuStateVectorBackend and CpuNoiseChannelBackend: the operations run in order and
 * channel j is applied after the first channels[j].position operations; p == 0 placements
 * are skipped without a draw.  Draws are consumed from `draws` in order; *used receives the
 * count (it may exceed ndraws, in which case the missing draws read as 0).  branches (may be
 * NULL) receives one entry per channel (see noise_apply). */
int qmo_trajectory(const qmo_operation* ops, int32_t count, const qmo_channel* channels, int32_t nch,
                   int32_t qubits, double* amps, const double* draws, int32_t ndraws, int32_t* used,
                   int8_t* branches) {
    int32_t done = 0, consumed = 0;
    for (int32_t j = 0; j < nch; ++j) {
        int32_t pos = channels[j].position;
        if (pos < done || pos > count) return 1;
        qmo_execute(ops + done, pos - done, qubits, amps);
        done = pos;
        int32_t step = 0, branch = -1;
        const double* rest = consumed < ndraws ? draws + consumed : draws;
        int32_t left = consumed < ndraws ? ndraws - consumed : 0;
        int rc = noise_apply(channels[j].kind, channels[j].probability, channels[j].target, amps, qubits, rest,
                             left, &step, &branch);
        if (rc) {
            if (used) *used = consumed;
            return rc;
        }
        consumed += step;
        if (branches) branches[j] = (int8_t)branch;
    }
    qmo_execute(ops + done, count - done, qubits, amps);
    if (used) *used = consumed;
    return 0;
}

/* ---------------------------------------------------------------- sampling */

/* StateVectorSimulator.Run (src/QuantumMatter.Application/StateVectorSimulator.cs:44-90):
 * sequential FP64 CDF, then per shot draw*total and a strict upper-bound search. */
int qmo_sample(const double* s, int32_t qubits, const double* draws, int32_t shots, int64_t* out) {
    int64_t len = (int64_t)1 << qubits;
    double total = 0;
    int64_t last = -1;
    double* cdf = (double*)malloc((size_t)len * sizeof(double));
    if (!cdf) return 3;
    for (int64_t i = 0; i < len; ++i) {
        cpx v = ld(s, i);
        double prob = v.re * v.re + v.im * v.im;
        total += prob;
        cdf[i] = total;
        if (prob > 0) last = i;
    }
    if (!isfinite(total) || total <= 0) { free(cdf); return 7; }
    for (int32_t shot = 0; shot < shots; ++shot) {
        double draw = draws[shot] * total;
        int64_t low = 0, high = len;
        while (low < high) {
            int64_t middle = low + (high - low) / 2;
            if (cdf[middle] <= draw) low = middle + 1; else high = middle;
        }
        out[shot] = low < len ? low : last;
    }
    free(cdf);
    return 0;
}

/* StateVector.MeasureAll (src/QuantumMatter.Core/StateVector.cs:106-153) */
int qmo_measure_all(double* s, int32_t qubits, double u, int64_t* outcome) {
    int64_t len = (int64_t)1 << qubits;
    double total = 0;
    int64_t last = -1;
    for (int64_t i = 0; i < len; ++i) {
        cpx v = ld(s, i);
        double prob = v.re * v.re + v.im * v.im;
        total += prob;
        if (prob > 0) last = i;
    }
    if (!isfinite(total) || total <= 0) return 7;
    double draw = u * total, cumulative = 0;
    int64_t result = last;
    for (int64_t i = 0; i < len; ++i) {
        cpx v = ld(s, i);
        cumulative += v.re * v.re + v.im * v.im;
        if (draw < cumulative) { result = i; break; }
    }
    memset(s, 0, (size_t)len * 2 * sizeof(double));
    s[2 * result] = 1.0;
    *outcome = result;
    return 0;
}

/* StateVector.MarginalProbability (src/QuantumMatter.Core/StateVector.Observations.cs:10-36):
 * plain sequential sums of the total and the selected Born masses.  Bit k of outcome refers to
 * qubits[k].  Returns 0, 1 for a bad selection, 7 for no finite positive mass. */
int qmo_marginal_probability(const double* s, int32_t nq, const int32_t* qubits, int32_t count, int32_t outcome,
                             double* probability) {
    int64_t len = (int64_t)1 << nq, mask = 0, pattern = 0;
    if (count < 1 || count > nq) return 1;
    for (int32_t k = 0; k < count; ++k) {
        if (qubits[k] < 0 || qubits[k] >= nq || (mask >> qubits[k]) & 1) return 1;
        mask |= (int64_t)1 << qubits[k];
        pattern |= (int64_t)((outcome >> k) & 1) << qubits[k];
    }
    double total = 0, selected = 0;
    for (int64_t i = 0; i < len; ++i) {
        cpx v = ld(s, i);
        double prob = v.re * v.re + v.im * v.im;
        total += prob;
        if ((i & mask) == pattern) selected += prob;
    }
    if (!isfinite(total) || total <= 0) return 7;
    *probability = selected / total;
    return 0;
}

/* StateVector.Measure (StateVector.Observations.cs:38-97): one full-basis Born draw with the
 * strict upper-bound search, the matching branch's mass, then the projection (matching
 * amplitudes divided by the square root of that mass, the rest zero). */
int qmo_measure(double* s, int32_t nq, const int32_t* qubits, int32_t count, double u, int32_t* outcome) {
    int64_t len = (int64_t)1 << nq, mask = 0;
    if (count < 1 || count > nq) return 1;
    for (int32_t k = 0; k < count; ++k) {
        if (qubits[k] < 0 || qubits[k] >= nq || (mask >> qubits[k]) & 1) return 1;
        mask |= (int64_t)1 << qubits[k];
    }
    double total = 0;
    int64_t last = -1;
    for (int64_t i = 0; i < len; ++i) {
        cpx v = ld(s, i);
        double prob = v.re * v.re + v.im * v.im;
        total += prob;
        if (prob > 0) last = i;
    }
    if (!isfinite(total) || total <= 0) return 7;
    double draw = u * total, cumulative = 0;
    int64_t basis = last;
    for (int64_t i = 0; i < len; ++i) {
        cpx v = ld(s, i);
        cumulative += v.re * v.re + v.im * v.im;
        if (draw < cumulative) { basis = i; break; }
    }
    int64_t pattern = basis & mask;
    double branch = 0;
    for (int64_t i = 0; i < len; ++i) {
        if ((i & mask) != pattern) continue;
        cpx v = ld(s, i);
        branch += v.re * v.re + v.im * v.im;
    }
    if (!isfinite(branch) || branch <= 0) return 7;
    double norm = sqrt(branch);
    for (int64_t i = 0; i < len; ++i) {
        cpx v = ld(s, i);
        if ((i & mask) == pattern) st(s, i, mk(v.re / norm, v.im / norm));
        else st(s, i, mk(0, 0));
    }
    int32_t out = 0;
    for (int32_t k = 0; k < count; ++k) out |= (int32_t)((basis >> qubits[k]) & 1) << k;
    *outcome = out;
    return 0;
}

/* ---------------------------------------------------------------- System.Random */

/* Seeded System.Random: Knuth's subtractive generator (Numerical Recipes "ran3"),
 * which .NET keeps for seeded instances for compatibility.  Call sites in the
 * reference: StateVectorSimulator.cs:42,71; NoisyStateVectorSimulator.cs:42,72,111;
 * CpuNoiseChannelBackend.cs:43,49,117.  Restated from the published algorithm. */
void qmo_random_init(qmo_random* r, int32_t seed) {
    const int32_t MBIG = 2147483647, MSEED = 161803398;
    int32_t subtraction = seed == INT32_MIN ? MBIG : (seed < 0 ? -seed : seed);
    int32_t mj = MSEED - subtraction;
    int32_t mk = 1, ii = 0;
    memset(r, 0, sizeof(*r));
    r->seed_array[55] = mj;
    for (int i = 1; i < 55; ++i) {
        ii += 21;
        if (ii >= 55) ii -= 55;
        r->seed_array[ii] = mk;
        mk = mj - mk;
        if (mk < 0) mk += MBIG;
        mj = r->seed_array[ii];
    }
    for (int k = 1; k < 5; ++k) {
        for (int i = 1; i < 56; ++i) {
            int n = i + 30;
            if (n >= 55) n -= 55;
            r->seed_array[i] -= r->seed_array[1 + n];
            if (r->seed_array[i] < 0) r->seed_array[i] += MBIG;
        }
    }
    r->inext = 0;
    r->inextp = 21;
}

double qmo_random_next_double(qmo_random* r) {
    const int32_t MBIG = 2147483647;
    int32_t a = r->inext + 1, b = r->inextp + 1;
    if (a >= 56) a = 1;
    if (b >= 56) b = 1;
    int32_t v = r->seed_array[a] - r->seed_array[b];
    if (v == MBIG) v--;
    if (v < 0) v += MBIG;
    r->seed_array[a] = v;
    r->inext = a;
    r->inextp = b;
    return v * (1.0 / MBIG);
}
