/*
 * qm_oracle.h -- CPU restatement of QuantumMatter's scalar state-vector path.
 *
 * TEST INFRASTRUCTURE ONLY.  This oracle is the checker for the CUDA library in
 * quantummatter_b200/.  Only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline / --impl reference legs may load it.  The product path never
 * calls it and has no CPU fallback.
 *
 * It is plain C compiled with -ffp-contract=off so that every complex product is
 * rounded the way .NET's System.Numerics.Complex rounds it (no fused multiply-add).
 * Each function names the reference source it restates (paths inside the
 * olgerd007/QuantumMatter project).
 *
 * Parity pinning: the reference is C# and has no runtime in this environment, so
 * the oracle is pinned against the reference test suite's known answers
 * (gate matrix columns, CNOT/SWAP truth tables, GHZ amplitudes, Pauli eigenvalues,
 * Hamiltonian cancellation, Kraus branch thresholds) and against an independent
 * dense-matrix model, both in tests/test_oracle_pinning.py.  The seeded random
 * stream (System.Random) is restated from its published algorithm; no .NET-produced
 * draw values exist here, so RNG parity is unpinned.
 */
#ifndef QM_ORACLE_H
#define QM_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* GateKind numbering of src/QuantumMatter.Core/QuantumCircuit.cs:4-40. */
enum {
    QMO_H = 0, QMO_X = 1, QMO_Y = 2, QMO_Z = 3, QMO_S = 4, QMO_T = 5,
    QMO_RX = 6, QMO_RY = 7, QMO_RZ = 8, QMO_CNOT = 9, QMO_SWAP = 10, QMO_I = 11,
    QMO_SDG = 12, QMO_TDG = 13, QMO_PHASE = 14, QMO_UNITARY = 15, QMO_TOFFOLI = 16
};

/* GateOperation record (QuantumCircuit.cs:49-51).  unitary = row-major m00,m01,m10,m11
 * as (re,im) pairs; only read for QMO_UNITARY. */
typedef struct qmo_operation {
    int32_t kind;
    int32_t target;
    int32_t control;        /* -1 when absent; first SWAP operand for Swap */
    int32_t second_control; /* -1 when absent */
    double angle;
    double unitary[8];
} qmo_operation;

/* StateVectorKernelKind of src/QuantumMatter.Infrastructure/PreparedStateVectorGate.cs:6 */
enum { QMO_K_IDENTITY = 0, QMO_K_MATRIX = 1, QMO_K_HADAMARD = 2, QMO_K_EXCHANGE = 3,
       QMO_K_DIAGONAL = 4, QMO_K_SWAP = 5 };

/* PreparedStateVectorGate record (PreparedStateVectorGate.cs:9-11); same memory layout
 * as qm_gate in include/qm_b200.h. */
typedef struct qmo_gate {
    int32_t kernel;
    int32_t target;
    uint32_t control_mask;
    int32_t swap_control;
    double a[2], b[2], c[2], d[2];
} qmo_gate;

/* ---- gates ---- */
int  qmo_validate(const qmo_operation* ops, int32_t count, int32_t qubits);
void qmo_execute(const qmo_operation* ops, int32_t count, int32_t qubits, double* amps);
int  qmo_prepare(const qmo_operation* ops, int32_t count, qmo_gate* out);
void qmo_apply_prepared(const qmo_gate* gates, int32_t count, int32_t qubits, double* amps);

/* ---- observables ---- */
double qmo_expectation(const double* amps, int32_t qubits, uint32_t flip_mask,
                       uint32_t sign_mask, int32_t y_count, double* mass_out);
int    qmo_energy(const double* amps, int32_t qubits, const uint32_t* flip, const uint32_t* sign,
                  const int32_t* ycount, const double* coeff, int32_t terms, double* energy_out);

/* ---- noise (draws supplied by the caller, consumed in reference order) ---- */
/* kind: 0 bit flip, 1 phase flip, 2 depolarizing, 3 amplitude damping
 * (src/QuantumMatter.Core/Noise/NoiseChannel.cs:4-14).
 * draws/ndraws: available draws; *used receives the number consumed (0 or 1).
 * Returns 0, or 7 when the state has no finite positive mass. */
int qmo_noise_apply(int32_t kind, double p, int32_t target, double* amps, int32_t qubits,
                    const double* draws, int32_t ndraws, int32_t* used);
void qmo_qubit_masses(const double* amps, int32_t qubits, int32_t target, double* m0, double* m1);

/* One channel placement of a NoisyCircuit: NoiseKind, target, probability, and the number of
 * operations that precede it (Noise/NoisyCircuit.cs:38-48).  Same layout as qm_channel. */
typedef struct qmo_channel {
    int32_t kind;
    int32_t target;
    double probability;
    int32_t position;
    int32_t reserved;
} qmo_channel;
int qmo_trajectory(const qmo_operation* ops, int32_t count, const qmo_channel* channels, int32_t nch,
                   int32_t qubits, double* amps, const double* draws, int32_t ndraws, int32_t* used,
                   int8_t* branches);

/* ---- sampling ---- */
int qmo_sample(const double* amps, int32_t qubits, const double* draws, int32_t shots, int64_t* out);
int qmo_measure_all(double* amps, int32_t qubits, double draw, int64_t* outcome);
int qmo_marginal_probability(const double* amps, int32_t qubits, const int32_t* selection, int32_t count,
                             int32_t outcome, double* probability);
int qmo_measure(double* amps, int32_t qubits, const int32_t* selection, int32_t count, double draw, int32_t* outcome);

/* ---- System.Random (seeded) restatement ---- */
typedef struct qmo_random { int32_t seed_array[56]; int32_t inext, inextp; } qmo_random;
void   qmo_random_init(qmo_random* r, int32_t seed);
double qmo_random_next_double(qmo_random* r);

#ifdef __cplusplus
}
#endif
#endif
