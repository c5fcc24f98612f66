/*
 * qm_b200.h -- C ABI of libqmb200.so, the B200 (sm_100a) state-vector engine behind
 * QuantumMatter's execution-backend ports.
 *
 * Everything here is plain C: fixed-width integers, doubles, opaque handles and
 * caller-owned arrays.  Amplitude arrays on the host are interleaved complex128
 * (re, im), the layout of System.Numerics.Complex[].  Every call returns a qm_status;
 * qm_last_error() gives the message of the last failure on the calling thread.
 *
 * Reference interfaces replaced (paths inside the olgerd007/QuantumMatter project):
 *   IStateVectorBackend.Execute        src/QuantumMatter.Core/IStateVectorBackend.cs:13
 *   INoiseChannelBackend.Apply         src/QuantumMatter.Core/Noise/INoiseChannelBackend.cs:13-14
 *   CudaStateVectorBackend             src/QuantumMatter.Infrastructure/CudaStateVectorBackend.cs:21-216
 *   PreparedStateVectorGate.Prepare    src/QuantumMatter.Infrastructure/PreparedStateVectorGate.cs:13-70
 * and, as additive device-resident APIs, the host-side loops of
 *   StateVector.ExpectationValue/ExpectationEnergy  src/QuantumMatter.Core/StateVector.Observations.cs:107-141,
 *                                                   src/QuantumMatter.Core/StateVector.Energy.cs:10-46
 *   StateVector.MeasureAll                          src/QuantumMatter.Core/StateVector.cs:106-153
 *   StateVectorSimulator.Run sampling               src/QuantumMatter.Application/StateVectorSimulator.cs:44-90
 */
#ifndef QM_B200_H
#define QM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define QM_ABI_VERSION 2  /* 2: qm_fused_pass_info gained qubits_out and out_bit (relabeling passes) */

/* Status codes.  The right-hand comment is the exception the reference raises for
 * the same condition, which is what a .NET shim maps the code to. */
typedef enum qm_status {
    QM_OK = 0,
    QM_E_ARG = 1,          /* ArgumentException / ArgumentNullException */
    QM_E_BUDGET = 2,       /* InvalidOperationException: state exceeds a memory budget (CudaStateVectorBackend.cs:120-124) */
    QM_E_OOM = 3,          /* OutOfMemoryException: device or pinned allocation failed */
    QM_E_DEVICE = 4,       /* PlatformNotSupportedException / CUDA runtime error (CudaStateVectorBackend.cs:31-35) */
    QM_E_CANCELLED = 5,    /* OperationCanceledException */
    QM_E_TIMEOUT = 6,      /* a bounded device wait ran out */
    QM_E_MASS = 7,         /* InvalidOperationException: no finite positive probability mass */
    QM_E_DISPOSED = 8,     /* ObjectDisposedException */
    QM_E_UNSUPPORTED = 9,  /* NotSupportedException: unknown gate kind */
    QM_E_RANGE = 10        /* ArgumentOutOfRangeException */
} qm_status;

/* Element type of a device state. */
typedef enum qm_precision {
    QM_FP64 = 0,           /* complex128, the drop-in form */
    QM_FP32 = 1            /* complex64; reductions, masses and CDFs stay FP64 */
} qm_precision;

/* ---------------------------------------------------------------- gates */

/* GateKind numbering (src/QuantumMatter.Core/QuantumCircuit.cs:4-40). */
enum {
    QM_GATE_H = 0, QM_GATE_X = 1, QM_GATE_Y = 2, QM_GATE_Z = 3, QM_GATE_S = 4, QM_GATE_T = 5,
    QM_GATE_RX = 6, QM_GATE_RY = 7, QM_GATE_RZ = 8, QM_GATE_CNOT = 9, QM_GATE_SWAP = 10,
    QM_GATE_I = 11, QM_GATE_SDG = 12, QM_GATE_TDG = 13, QM_GATE_PHASE = 14,
    QM_GATE_UNITARY = 15, QM_GATE_TOFFOLI = 16
};

/* One GateOperation record (QuantumCircuit.cs:49-51).  unitary holds the row-major
 * m00, m01, m10, m11 entries as (re, im) pairs and is read only for QM_GATE_UNITARY. */
typedef struct qm_operation {
    int32_t kind;
    int32_t target;
    int32_t control;         /* -1 when absent; the first SWAP operand for QM_GATE_SWAP */
    int32_t second_control;  /* -1 when absent */
    double angle;
    double unitary[8];
} qm_operation;              /* 88 bytes */

/* StateVectorKernelKind (PreparedStateVectorGate.cs:6). */
enum {
    QM_KERNEL_IDENTITY = 0, QM_KERNEL_MATRIX = 1, QM_KERNEL_HADAMARD = 2,
    QM_KERNEL_EXCHANGE = 3, QM_KERNEL_DIAGONAL = 4, QM_KERNEL_SWAP = 5
};

/* One prepared gate, the record PreparedStateVectorGate holds (PreparedStateVectorGate.cs:9-11):
 * coefficients are evaluated once on the host.  Matrix/Hadamard: [a b; c d] on the
 * target pair.  Diagonal: a on target-zero, d on target-one.  Exchange: X.  Swap:
 * exchanges the target and swap_control qubits.  A gate acts only where every bit of
 * control_mask is set. */
typedef struct qm_gate {
    int32_t kernel;
    int32_t target;
    uint32_t control_mask;
    int32_t swap_control;    /* -1 unless kernel == QM_KERNEL_SWAP */
    double a[2], b[2], c[2], d[2];
} qm_gate;                   /* 80 bytes */

/* ---------------------------------------------------------------- options */

/* CudaBackendOptions (src/QuantumMatter.Infrastructure/CudaBackendOptions.cs:4-21) plus the
 * engine's own knobs.  Zero-initialise, then set fields; qm_options_default fills the
 * reference defaults (512 MiB budgets, device 0). */
typedef struct qm_options {
    int32_t device_index;
    int32_t enable_profiling;       /* fills qm_profile in the *_profiled calls */
    int64_t device_budget_bytes;    /* maximum bytes of device states held by the context */
    int64_t staging_budget_bytes;   /* maximum pinned host staging bytes */
    int32_t fusion_width;           /* 0 = planner default (fused blocks of 12 qubits); 1 = one launch
                                       per gate; 2..6 = dense fused gates of at most that many qubits,
                                       one sweep of the state each; 9..14 = fused blocks of that many
                                       qubits.  7 and 8 give QM_E_RANGE. */
    int32_t reserved[7];
} qm_options;

/* CudaExecutionProfile (CudaBackendOptions.cs:35): device time of the gate sequence
 * (CUDA events, launch gaps included, transfers excluded), state bytes, launches. */
typedef struct qm_profile {
    double device_seconds;
    double transfer_seconds;        /* host<->device copies of the host-buffer entry points */
    int64_t state_bytes;
    int32_t kernel_launches;
    int32_t passes;                 /* fused passes (0 on the per-gate path) */
    int64_t planned_bytes;          /* DRAM bytes the plan reads+writes */
} qm_profile;

typedef struct qm_device_info {
    int32_t index;
    int32_t sm_count;
    int32_t major, minor;
    int32_t driver_version;
    int32_t reserved;
    int64_t memory_bytes;
    char name[256];
} qm_device_info;

typedef struct qm_context qm_context;
typedef struct qm_state qm_state;
typedef struct qm_plan qm_plan;

/* ---------------------------------------------------------------- runtime */

int32_t qm_abi_version(void);
/* Copies the calling thread's last error message (NUL-terminated, truncated). */
int32_t qm_last_error(char* buffer, size_t size);
void qm_options_default(qm_options* options);
/* CudaStateVectorBackend.GetDevices (CudaStateVectorBackend.cs:70-85). */
int32_t qm_device_count(int32_t* count);
int32_t qm_device_info_get(int32_t index, qm_device_info* info);

/* CudaStateVectorBackend constructor / Dispose (CudaStateVectorBackend.cs:21-64,191-216).
 * QM_E_DEVICE when no device exists, QM_E_RANGE for a bad device index. */
int32_t qm_context_create(const qm_options* options, qm_context** context);
int32_t qm_context_destroy(qm_context* context);

/* Pinned host memory from the context's device, for callers that keep amplitude
 * arrays in page-locked memory (the copies then run at full PCIe/C2C rate). */
int32_t qm_host_alloc(qm_context* context, int64_t bytes, void** pointer);
int32_t qm_host_free(qm_context* context, void* pointer);

/* PreparedStateVectorGate.Prepare for `count` operations on a `qubits`-qubit register,
 * after the builder validation of QuantumCircuit.cs:97-134. */
int32_t qm_prepare_gates(const qm_operation* operations, int32_t count, int32_t qubits, qm_gate* gates);

/* ---------------------------------------------------------------- drop-in port */

/* IStateVectorBackend.Execute on a host buffer (CudaStateVectorBackend.ExecuteCore,
 * CudaStateVectorBackend.cs:103-188): validates length == 2^qubits (QM_E_ARG), checks
 * the budgets before touching the buffer (QM_E_BUDGET), uploads, runs every gate in
 * insertion order on the device, downloads and commits.  *cancel (may be NULL) is
 * polled before work, between launch chunks of at most 32 gates and before the
 * commit; QM_E_CANCELLED or any failure before the commit leaves the buffer unchanged.
 * profile may be NULL. */
int32_t qm_execute_host(qm_context* context, int32_t qubits, const qm_operation* operations,
                        int32_t count, double* amplitudes, int64_t length,
                        const volatile int32_t* cancel, qm_profile* profile);

/* INoiseChannelBackend.Apply on a host buffer (CpuNoiseChannelBackend.cs:10-145).
 * kind: 0 bit flip, 1 phase flip, 2 depolarizing, 3 amplitude damping
 * (src/QuantumMatter.Core/Noise/NoiseChannel.cs:4-14).  Random draws come from the
 * caller's generator through next_double (System.Random.NextDouble in the .NET shim),
 * consumed exactly where the reference consumes them: none when p == 0, none for a
 * flip with p == 1, none for damping when either branch has zero mass. */
typedef double (*qm_next_double_fn)(void* user);
int32_t qm_noise_apply_host(qm_context* context, int32_t kind, double probability, int32_t target,
                            double* amplitudes, int64_t length, qm_next_double_fn next_double,
                            void* user, const volatile int32_t* cancel);

/* ---------------------------------------------------------------- device states */

/* Allocates a device state of 2^qubits amplitudes (qubits in [1,30]) set to |0...0>.
 * QM_E_BUDGET when the context's device budget would be exceeded. */
int32_t qm_state_create(qm_context* context, int32_t qubits, int32_t precision, qm_state** state);
int32_t qm_state_destroy(qm_state* state);
int32_t qm_state_reset(qm_state* state);                       /* StateVector.Reset */
int32_t qm_state_upload(qm_state* state, const double* amplitudes, int64_t length);
int32_t qm_state_download(qm_state* state, double* amplitudes, int64_t length);
/* Device address of the amplitude array (complex128 or complex64, interleaved). */
int32_t qm_state_device_pointer(qm_state* state, void** pointer);

/* Runs prepared gates in order on a device state.  fusion_width as in qm_options
 * (0 = context default).  profile may be NULL. */
int32_t qm_execute(qm_state* state, const qm_gate* gates, int32_t count, int32_t fusion_width,
                   qm_profile* profile);

/* A reusable fused schedule for one gate list: planned once, executed many times. */
int32_t qm_plan_create(qm_context* context, int32_t qubits, int32_t precision, const qm_gate* gates,
                       int32_t count, int32_t fusion_width, qm_plan** plan);
int32_t qm_plan_execute(qm_plan* plan, qm_state* state, qm_profile* profile);
/* passes, kernel launches and planned DRAM bytes of one execution. */
int32_t qm_plan_stats(const qm_plan* plan, int32_t* passes, int32_t* launches, int64_t* planned_bytes);
int32_t qm_plan_destroy(qm_plan* plan);

/* The engine's autotuner: plans the gates at each candidate fusion width, times one execution of
 * each on a scratch state of that size (after an untimed one that compiles its kernels; the
 * scratch is freed before returning), and returns the plan of the fastest, as qm_plan_create does,
 * with its width in *chosen (may be NULL).  The choice is cached for the process per qubit count,
 * precision and gate structure (kernels, targets, controls; not coefficients), so circuits that
 * differ only in angles are timed once.  candidates NULL / candidate_count 0: fused blocks of 10,
 * 11 and 12 qubits, plus 13 and dense fused gates of 5 and 6 qubits for QM_FP32.  Additive. */
int32_t qm_plan_autotune(qm_context* context, int32_t qubits, int32_t precision, const qm_gate* gates,
                         int32_t count, const int32_t* candidates, int32_t candidate_count, qm_plan** plan,
                         int32_t* chosen);

/* One execution of a plan on a state captured as a CUDA graph: every pass (or fused gate) of the
 * plan becomes a node, and a launch replays them with one submission on the context's stream.
 * The plan and the state must outlive the graph; a launch evolves the state it was captured on,
 * in place, exactly as qm_plan_execute does (the capture itself runs nothing).  Execute the plan
 * once before capturing it, so that its kernels are loaded.  Additive (the reference launches one
 * kernel per gate and synchronises every 32, CudaStateVectorBackend.cs:155-159). */
typedef struct qm_graph qm_graph;
int32_t qm_graph_create(qm_plan* plan, qm_state* state, qm_graph** graph);
int32_t qm_graph_launch(qm_graph* graph, qm_profile* profile);
int32_t qm_graph_destroy(qm_graph* graph);

/* Host-only inspection of the fused schedule the planner builds for a gate list (no
 * device needed): pass headers and the op program each pass's kernel interprets.
 * Counts are always written; records are written when the arrays are large enough.
 * The records mirror the engine's internal layout (op codes: 0 stage change, 1 complex
 * matrix, 2 real matrix, 3 X, 4 diagonal, 5 negate, 6 swap). */
typedef struct qm_fused_pass_info {
    int32_t block_qubits;
    int32_t op_begin, op_count;
    int32_t qubits[14];      /* ascending; local bit i of a block index is qubits[i] */
    uint32_t block_mask;
    int32_t stages;          /* register layouts used by the pass */
    int8_t reg_in[4];        /* local register bits of the load layout */
    int8_t reg_out[4];       /* local register bits of the store layout */
    int8_t qubits_out[16];   /* index bit each local bit is written to (a permutation of qubits[]
                                when the pass relabels qubits, qubits[] otherwise) */
    int8_t out_bit[16];      /* index bit written by each thread rank of the store layout */
} qm_fused_pass_info;        /* 116 bytes */

typedef struct qm_fused_op_info {
    uint8_t code;
    int8_t reg, reg2;        /* register bits of the current stage layout */
    int8_t local;            /* local bit of a diagonal target, -1 outside the block */
    int8_t reg_pos[4];       /* stage change: local bit of each register bit */
    uint16_t cmask_local;    /* controls (and negate target) as local-index bits */
    uint16_t flags;          /* bit0: a == 1, bit1: d == 1 */
    uint32_t cmask_outer;    /* controls (and negate target) outside the block, global bits */
    uint32_t target_outer;   /* outside-the-block diagonal target, global bit */
    uint32_t reserved;
    double coef[8];          /* a, b, c, d as (re, im) */
} qm_fused_op_info;          /* 88 bytes */

int32_t qm_plan_program(int32_t qubits, int32_t precision, const qm_gate* gates, int32_t count,
                        int32_t fusion_width, int32_t* passes, qm_fused_pass_info* pass_records,
                        int32_t max_passes, int32_t* ops, qm_fused_op_info* op_records, int32_t max_ops,
                        int64_t* planned_bytes);

/* Passes compiled for their own op sequence.  Persistent plans (qm_plan_create), the batched
 * variational evaluator and the trajectory runner compile each distinct pass structure once
 * (NVRTC for sm_100a; angles and the constants derived from them travel as kernel parameters,
 * so a kernel serves every pass with its structure and rotation forms) and run the
 * compiled kernel; without NVRTC, or with QM_JIT=0 in the environment, they run the
 * interpreting pass kernel.  qm_jit_info reports whether compilation is available and the
 * process-wide counts; qm_jit_source returns the generated source of one pass of the plan the
 * planner makes for `gates` (length receives the full size). */
int32_t qm_jit_info(int32_t* available, int64_t* kernels, int64_t* failed, int64_t* launches);
/* Dense fused gates (fusion widths 2..6): how many kernel launches the process has made, and how
 * many of them ran on the tensor cores (complex64 gates of 5 and 6 qubits in states of 11 qubits or
 * more; QM_DENSE_TC=0 in the environment at planning keeps them on the FP32 pipes).  Additive. */
int32_t qm_dense_info(int64_t* launches, int64_t* tensor_core_launches);
int32_t qm_jit_source(int32_t qubits, int32_t precision, const qm_gate* gates, int32_t count,
                      int32_t fusion_width, int32_t pass, char* buffer, size_t size, size_t* length);
/* The constant parameter block that the same compiled pass is launched with (the rotation and
 * phase constants of its kernel parameter `A`), as bytes; for inspection and tests. */
int32_t qm_jit_constants(int32_t qubits, int32_t precision, const qm_gate* gates, int32_t count,
                         int32_t fusion_width, int32_t pass, void* buffer, size_t size, size_t* length);

/* ---------------------------------------------------------------- noise primitives */

/* FP64 compensated masses of target-zero and target-one amplitudes
 * (CpuNoiseChannelBackend.cs:88-106). */
int32_t qm_qubit_masses(qm_state* state, int32_t target, double* zero_mass, double* one_mass);
/* Pauli branch on the target: 1 = X, 2 = Y, 3 = Z (CpuNoiseChannelBackend.cs:59-80). */
int32_t qm_apply_pauli(qm_state* state, int32_t target, int32_t pauli);
/* Damping branch (CpuNoiseChannelBackend.cs:118-142): jump != 0 writes
 * psi0 = jump_scale * psi1, psi1 = 0; otherwise psi0 *= scale, psi1 *= stay_scale. */
int32_t qm_apply_damping(qm_state* state, int32_t target, int32_t jump, double scale,
                         double jump_scale, double stay_scale);
/* INoiseChannelBackend.Apply on a resident state: qm_noise_apply_host's branch choice and draw
 * consumption (none when p == 0, none for a flip with p == 1, none for damping when either
 * branch has zero mass), with no copy of the state.  The device-resident noisy dynamic circuit
 * uses it between segments. */
int32_t qm_state_noise_apply(qm_state* state, int32_t kind, double probability, int32_t target,
                             qm_next_double_fn next_double, void* user);

/* ---------------------------------------------------------------- observables */

/* One Pauli term: PauliString masks (src/QuantumMatter.Core/PauliString.cs:37-39) and the
 * real coefficient of a PauliTerm (src/QuantumMatter.Core/Observables/PauliTerm.cs:7-13). */
typedef struct qm_pauli_term {
    uint32_t flip_mask;      /* X or Y positions */
    uint32_t sign_mask;      /* Z or Y positions */
    int32_t y_count;
    int32_t reserved;
    double coefficient;
} qm_pauli_term;             /* 24 bytes */

/* One fused pass: per_term[t] = <psi|P_t|psi> / <psi|psi> for every term (coefficients
 * ignored), *mass = <psi|psi>, FP64 accumulation.  QM_E_MASS when the mass is not
 * finite and positive or a term sum is not finite. */
int32_t qm_expectation_pauli(qm_state* state, const qm_pauli_term* terms, int32_t count,
                             double* per_term, double* mass);
/* StateVector.ExpectationEnergy: sum of c_t <P_t> over nonzero coefficients in term order
 * with Neumaier compensation.  An empty term list still validates the mass. */
int32_t qm_expectation_energy(qm_state* state, const qm_pauli_term* terms, int32_t count,
                              double* energy);
/* The batched variational evaluator compiles the tiled expectation for its term list (one
 * kernel per tile pass: flip masks, phases and tile-local signs as constants).  Returns the
 * generated source of tile pass `pass` for these terms on a `qubits`-qubit state (inspection
 * and tests; length receives the full size).  No reference counterpart. */
int32_t qm_jit_expect_source(int32_t qubits, int32_t precision, const qm_pauli_term* terms, int32_t count,
                             int32_t pass, char* buffer, size_t size, size_t* length);

/* ---------------------------------------------------------------- sampling */

/* StateVector.MeasureAll: u is the caller's NextDouble draw; collapses the state to the
 * sampled basis state with amplitude +1.  *ambiguous is set when u*total lies within the
 * device/host rounding margin of a CDF boundary (the outcome is then still the device's). */
int32_t qm_measure_all(qm_state* state, double u, int64_t* outcome, int32_t* ambiguous);
/* StateVectorSimulator.Run terminal sampling: FP64 CDF, draw*total, strict upper-bound
 * search per shot, without collapse.  *ambiguous counts shots near a boundary. */
int32_t qm_sample(qm_state* state, const double* draws, int32_t shots, int64_t* outcomes,
                  int32_t* ambiguous);
/* StateVector.MarginalProbability (src/QuantumMatter.Core/StateVector.Observations.cs:10-36): the
 * normalised Born probability that qubits[k] reads bit k of `outcome`, for all k.  Selections
 * are 1..qubits distinct in-range qubits (QM_E_ARG / QM_E_RANGE otherwise). */
int32_t qm_marginal_probability(qm_state* state, const int32_t* qubits, int32_t count, int32_t outcome,
                                double* probability);
/* StateVector.Measure (StateVector.Observations.cs:38-97): one full-basis Born draw (u is the
 * caller's NextDouble), then the state is projected onto the drawn values of the selected qubits
 * and renormalised, keeping the surviving phases.  Bit k of *outcome is qubits[k]'s value;
 * *ambiguous is set when u * total lies within the rounding margin of a CDF boundary.  The state
 * stays on the device: dynamic circuits keep their classical control on the host. */
int32_t qm_measure(qm_state* state, const int32_t* qubits, int32_t count, double u, int32_t* outcome,
                   int32_t* ambiguous);

/* ---------------------------------------------------------------- batches */

/* A device batch of `capacity` equally sized states (qubits in [9,30]).  All states of one
 * execution share a gate structure; gates with a nonnegative slot read their coefficients
 * (a, b, c, d as 8 doubles) per state from `table` ([states][slot_count][8]).  This is the
 * engine behind batched trajectories, parameter-shift circuits and served requests. */
typedef struct qm_batch qm_batch;
int32_t qm_batch_create(qm_context* context, int32_t qubits, int32_t precision, int32_t capacity, qm_batch** batch);
int32_t qm_batch_destroy(qm_batch* batch);
int32_t qm_batch_reset(qm_batch* batch, int32_t states);          /* first `states` states to |0...0> */
/* Copies one state to (upload = 0) or from (upload != 0) a host complex128 array. */
int32_t qm_batch_state(qm_batch* batch, int32_t index, double* amplitudes, int64_t length, int32_t upload);
int32_t qm_batch_execute(qm_batch* batch, int32_t states, const qm_gate* gates, const int32_t* slots, int32_t count,
                         const double* table, int32_t slot_count, int32_t fusion_width);
/* values[state][term] = <P_t> / mass (coefficients ignored), masses[state] (may be NULL). */
int32_t qm_batch_expectation(qm_batch* batch, int32_t states, const qm_pauli_term* terms, int32_t count,
                             double* values, double* masses);

/* ---------------------------------------------------------------- variational */

/* One operation of a ParameterizedCircuit template (src/QuantumMatter.Core/Variational/
 * ParameterizedCircuit.cs:98): a constant gate (parameter = -1) or an uncontrolled Rx/Ry/Rz
 * whose angle is parameters[parameter]. */
typedef struct qm_template_op {
    qm_operation operation;
    int32_t parameter;
    int32_t reserved;
} qm_template_op;            /* 96 bytes */

typedef struct qm_vqe_stats {
    int64_t circuits;         /* circuits evaluated: vectors * (1 + 2 * rotations) with gradients */
    int32_t waves;            /* batch waves (CUDA-graph replays for full waves) */
    int32_t batch_states;
    int32_t passes_per_circuit;
    int32_t tile_passes;
    double device_seconds;
    double wall_seconds;
} qm_vqe_stats;

/* VariationalEnergyEvaluator.Evaluate / EvaluateWithGradient
 * (src/QuantumMatter.Application/Variational/VariationalEnergyEvaluator.cs:23-86) for `vectors`
 * parameter vectors at once: parameters[vector][parameter_count] -> energies[vector] and, when
 * with_gradient != 0, gradients[vector][parameter_count] by the occurrence-wise +-pi/2
 * parameter-shift rule with termwise differencing and Neumaier accumulation.  Every base and
 * shifted circuit runs as a state of device batches (waves sized by the device budget).
 * stats may be NULL. */
int32_t qm_vqe_evaluate(qm_context* context, int32_t qubits, int32_t precision, const qm_template_op* operations,
                        int32_t operation_count, int32_t parameter_count, const qm_pauli_term* terms,
                        int32_t term_count, const double* parameters, int32_t vectors, int32_t with_gradient,
                        double* energies, double* gradients, qm_vqe_stats* stats);
/* qm_vqe_evaluate with its own Hamiltonian coefficients per vector: coefficients[vector][term]
 * replaces terms[t].coefficient, so vectors whose Hamiltonians share Pauli strings but not
 * coefficients (served requests on different chains) share one batch. */
int32_t qm_vqe_evaluate_coefficients(qm_context* context, int32_t qubits, int32_t precision,
                                     const qm_template_op* operations, int32_t operation_count, int32_t parameter_count,
                                     const qm_pauli_term* terms, int32_t term_count, const double* coefficients,
                                     const double* parameters, int32_t vectors, int32_t with_gradient,
                                     double* energies, double* gradients, qm_vqe_stats* stats);

/* Several evaluations of different sizes at once (the batched form of VariationalEnergyEvaluator
 * for a mix of registers, e.g. 16-, 18-, 20- and 22-qubit ansatzes).  Each problem is what one
 * qm_vqe_evaluate / qm_vqe_evaluate_coefficients call takes (coefficients NULL: the terms' own).
 * The device budget is shared in proportion to each problem's state bytes; every round runs each
 * problem's next wave on its own stream, forked from and joined to the context's stream, so the
 * sizes overlap on the device, and rounds in which every problem runs a full wave replay one
 * captured CUDA graph (one launch for all sizes).  Results equal the separate calls'. */
typedef struct qm_vqe_problem {
    int32_t qubits, precision;
    const qm_template_op* operations;
    int32_t operation_count, parameter_count;
    const qm_pauli_term* terms;
    int32_t term_count, vectors;
    const double* coefficients;     /* [vectors][term_count] or NULL */
    const double* parameters;       /* [vectors][parameter_count] */
    int32_t with_gradient, reserved;
    double* energies;               /* [vectors] */
    double* gradients;              /* [vectors][parameter_count] when with_gradient */
} qm_vqe_problem;                   /* 80 bytes */
int32_t qm_vqe_evaluate_mixed(qm_context* context, const qm_vqe_problem* problems, int32_t count,
                              qm_vqe_stats* stats);

/* ---------------------------------------------------------------- serving */

/* A request server on one GPU; no reference counterpart (applications call the reference's port
 * one circuit at a time: StateVector.Evolve + ExpectationValue, StateVector.Observations.cs:107-141;
 * StateVectorSimulator.Run, StateVectorSimulator.cs:37-101; VariationalEnergyEvaluator.
 * EvaluateWithGradient, VariationalEnergyEvaluator.cs:34-86).  Requests from any host thread are
 * admitted by the bytes of their state (16 * 2^n complex128, 8 * 2^n complex64) against
 * budget_bytes, oldest first (a younger request passes only while an older one does not fit); each
 * of `workers` threads runs jobs on its own context and CUDA stream, so jobs overlap on the device.
 * A VQE session keeps its parameters in the server; waiting steps of sessions that share an ansatz
 * structure and Pauli strings run as one batch (qm_vqe_evaluate_coefficients), a session never has
 * two steps in flight, and each step ends with p - step_size * gradient rounded once (VqeSolver.cs:76).
 * Results equal those of the request run alone. */
typedef struct qm_server qm_server;
typedef struct qm_serve_options {
    int32_t device_index;
    int32_t workers;                /* worker threads, 1..64 */
    int64_t budget_bytes;           /* admission budget over the requests in flight */
    int64_t context_budget_bytes;   /* device budget of each worker's context */
    int64_t cache_bytes;            /* device states each worker keeps for reuse */
    int32_t max_batch;              /* VQE steps per device batch (0: 64) */
    int32_t reserved[5];
} qm_serve_options;

enum { QM_SERVE_EXPECTATION = 0, QM_SERVE_SHOTS = 1, QM_SERVE_VQE_STEP = 2 };

typedef struct qm_serve_result {
    int32_t kind;                   /* QM_SERVE_* */
    int32_t status;                 /* QM_OK or the error of the request's execution (qm_last_error) */
    int32_t batch;                  /* requests evaluated in the same device batch */
    int32_t ambiguous;              /* shots drawn within the rounding margin of a CDF boundary */
    int32_t values;                 /* doubles written to values: per-term <P_t> or the VQE gradient */
    int32_t outcomes;               /* int64s written to outcomes: one basis index per shot */
    int32_t parameters;             /* doubles written to parameters: the session's after the step */
    int32_t reserved;
    double mass;                    /* expectation: Born mass of the final state */
    double energy;                  /* VQE step: the energy before the update */
    double submitted, started, finished;  /* seconds since qm_serve_create */
} qm_serve_result;

typedef struct qm_serve_stats {
    int64_t submitted, completed, jobs, vqe_jobs, vqe_steps;
    int64_t budget_bytes, reserved_bytes, peak_reserved_bytes;
    int32_t queued, running, max_batch, reserved;
} qm_serve_stats;

int32_t qm_serve_create(const qm_serve_options* options, qm_server** server);
/* Waits for the jobs on the device, cancels waiting requests (QM_E_CANCELLED) and frees everything. */
int32_t qm_serve_destroy(qm_server* server);
/* <P_t> / <psi|psi> of every term on the circuit's final state from |0...0> (coefficients ignored). */
int32_t qm_serve_submit_expectation(qm_server* server, int32_t qubits, int32_t precision,
                                    const qm_operation* operations, int32_t count, const qm_pauli_term* terms,
                                    int32_t term_count, int64_t* request);
/* Terminal samples of the circuit's final state, one per draw in [0, 1) (qm_sample). */
int32_t qm_serve_submit_shots(qm_server* server, int32_t qubits, int32_t precision, const qm_operation* operations,
                              int32_t count, const double* draws, int32_t shots, int64_t* request);
/* A VQE session: the ansatz template (qm_vqe_evaluate), the Hamiltonian with its coefficients,
 * the initial parameters and the steepest-descent step size. */
int32_t qm_serve_session_create(qm_server* server, int32_t qubits, int32_t precision,
                                const qm_template_op* operations, int32_t operation_count, int32_t parameter_count,
                                const qm_pauli_term* terms, int32_t term_count, const double* parameters,
                                double step_size, int64_t* session);
int32_t qm_serve_session_parameters(qm_server* server, int64_t session, double* parameters, int32_t count,
                                    int64_t* steps);
int32_t qm_serve_session_destroy(qm_server* server, int64_t session);  /* QM_E_ARG while steps are in flight */
/* One energy + parameter-shift gradient at the session's parameters, then the update. */
int32_t qm_serve_submit_vqe_step(qm_server* server, int64_t session, int64_t* request);
/* Waits up to timeout_seconds (0: polls) for the request; *done = 1 once it finished. */
int32_t qm_serve_wait(qm_server* server, int64_t request, double timeout_seconds, int32_t* done);
/* Copies a finished request's result and outputs and forgets the request.  Buffers may be NULL when
 * the request has no such output; QM_E_RANGE when one is too small (the request is kept). */
int32_t qm_serve_take_result(qm_server* server, int64_t request, qm_serve_result* result, double* values,
                             int32_t max_values, int64_t* outcomes, int32_t max_outcomes, double* parameters,
                             int32_t max_parameters);
int32_t qm_serve_get_stats(qm_server* server, qm_serve_stats* stats);

/* ---------------------------------------------------------------- noise trajectories */

/* One channel placement of a NoisyCircuit (src/QuantumMatter.Core/Noise/NoisyCircuit.cs:38-48):
 * kind is NoiseKind (0 bit flip, 1 phase flip, 2 depolarizing, 3 amplitude damping,
 * Noise/NoiseChannel.cs:4-14), the channel acts after the first `position` gates. */
typedef struct qm_channel {
    int32_t kind;
    int32_t target;
    double probability;
    int32_t position;
    int32_t reserved;
} qm_channel;                /* 24 bytes */

/* Per-trajectory outputs of qm_trajectories_run; every pointer may be NULL. */
typedef struct qm_trajectory_outputs {
    double* values;              /* [trajectories][term_count]: <P_t> / mass at the end */
    double* masses;              /* [trajectories]: final Born mass */
    int32_t* consumed;           /* [trajectories]: draws consumed (the measurement's included) */
    int8_t* branches;            /* [trajectories][channel_count]: -1 skipped (p == 0), Pauli
                                    0..3 = I/X/Y/Z, damping 0 = stay, 1 = jump */
    int32_t* ambiguous;          /* [trajectories]: damping selections whose draw lay within the
                                    rounding margin of jumpMass / total */
    int64_t* outcomes;           /* [trajectories]: StateVector.MeasureAll of the final state with
                                    the trajectory's next draw (NoisyStateVectorSimulator.Run) */
    double* probability_means;   /* [2^qubits]: Welford mean of |psi_i|^2 / mass over trajectories */
    double* probability_stderr;  /* [2^qubits]: sqrt(M2 / (T (T - 1)))
                                    (NoisyStateVectorSimulator.EstimateProbabilities) */
} qm_trajectory_outputs;

typedef struct qm_trajectory_stats {
    int32_t segments;            /* fused schedules between damping decisions */
    int32_t passes;              /* fused passes per trajectory */
    int32_t mass_passes;         /* joint-mass (histogram) passes per trajectory */
    int32_t waves;
    int32_t batch_states;
    int32_t reserved;
    double device_seconds;
    double wall_seconds;
} qm_trajectory_stats;

/* NoisyCircuit.Execute for `trajectories` independent trajectories at once
 * (NoisyStateVectorSimulator.cs:36-106, CpuNoiseChannelBackend.cs:10-145).  Every trajectory
 * starts from |0...0>, runs the prepared gates with the channel placements between them and
 * consumes its own draws, draws[t * draw_stride + k], in the reference's order: one per
 * depolarizing placement, one per flip unless p == 1, one per damping unless the jump or the
 * stay branch has zero mass, none for p == 0, then one for the measurement when `outcomes` is
 * requested.  Branch selection follows the reference's thresholds on the given draws; damping
 * renormalisation uses FP64 masses.  QM_E_RANGE when a trajectory needs more than draw_stride
 * draws, QM_E_MASS when a damping meets no finite positive mass.  stats may be NULL. */
int32_t qm_trajectories_run(qm_context* context, int32_t qubits, int32_t precision, const qm_gate* gates,
                            int32_t gate_count, const qm_channel* channels, int32_t channel_count,
                            int32_t trajectories, const double* draws, int32_t draw_stride,
                            const qm_pauli_term* terms, int32_t term_count, const qm_trajectory_outputs* outputs,
                            qm_trajectory_stats* stats);

/* The NextDouble() stream of a seeded System.Random (the reference's draw source for
 * measurements and Kraus selectors, NoisyStateVectorSimulator.cs:111): values skip .. skip +
 * count - 1 of Random(seed). */
int32_t qm_random_doubles(int32_t seed, int64_t skip, int64_t count, double* out);

/* ---------------------------------------------------------------- allocation-free expectation */

/* No counterpart in the reference: an additive entry point for hosts that cannot allocate
 * device memory at the call (their pool allocator owns the device memory, or the device-wide
 * synchronisation of cudaMalloc/cudaFree is not acceptable in their loop).
 *
 * Same results as qm_expectation_pauli on a caller-owned device state: per_term[t] =
 * <psi|P_t|psi> / <psi|psi> (coefficients ignored), *mass = <psi|psi> (mass may be NULL),
 * FP64 accumulation, QM_E_MASS as there.  `amplitudes` is the device address of 2^qubits
 * interleaved (re, im) pairs, complex128 for QM_FP64 or complex64 for QM_FP32, on the current
 * device; the kernels run on `stream` (NULL: the legacy default stream) and the call returns
 * after that stream has finished them.
 *
 * It allocates nothing: its scratch (the reduction's per-block partial sums) is a fixed
 * file-scope device array of about 304 KB per device, zeroed by the call itself.  The first
 * call on each device looks that array's address up (cudaGetSymbolAddress).  CUDA loads a
 * library's device code lazily, so that first call also loads the modules holding the array
 * and the kernels, which reserves about 304 KB plus their code on the device: a host whose pool
 * takes the GPU's memory makes one warm-up call (count = 0 is enough) before the pool does, and
 * before any stream capture begins.  The address is cached for the life of the process, so the
 * entry point must not be used across a cudaDeviceReset.  count > QM_NOALLOC_MAX_TERMS gives
 * QM_E_RANGE.  Calls whose work can overlap on one GPU (from several host threads, or on
 * several streams) race on that device's scratch and give wrong sums: serialise them. */
#define QM_NOALLOC_MAX_TERMS 64
int32_t qm_expectation_pauli_noalloc(const void* amplitudes, int32_t qubits, int32_t precision,
                                     const qm_pauli_term* terms, int32_t count, double* per_term,
                                     double* mass, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* QM_B200_H */
