// qm_internal.h -- declarations shared by the host runtime and the CUDA kernels of
// libqmb200.so.  Not part of the public ABI (that is include/qm_b200.h).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <mutex>
#include <string>
#include <vector>

#include "qm_b200.h"

namespace qm {

// ---------------------------------------------------------------- errors
void set_error(const std::string& message);
int32_t fail(int32_t status, const std::string& message);
int32_t cuda_fail(cudaError_t err, const char* what);

#define QM_CUDA(call)                                         \
    do {                                                      \
        cudaError_t qm_err_ = (call);                         \
        if (qm_err_ != cudaSuccess) return ::qm::cuda_fail(qm_err_, #call); \
    } while (0)

// ---------------------------------------------------------------- device gate record
// Device form of a prepared gate: masks instead of qubit numbers (DeviceGate,
// CudaStateVectorKernel.cs:24-34), coefficients as doubles.
struct DevGate {
    int32_t kernel;
    uint32_t target_bit;
    uint32_t control_mask;
    uint32_t swap_bit;
    int32_t target;
    int32_t swap_control;
    int32_t a_is_one;   // diagonal zero-phase is exactly 1: the target-zero half is untouched
    int32_t d_is_one;
    double a[2], b[2], c[2], d[2];
};
DevGate to_dev_gate(const qm_gate& g);
// Kernel ids, qubit ranges, control/target overlap and finite coefficients of prepared gates.
int32_t validate_prepared_gates(const qm_gate* gates, int32_t count, int32_t qubits);

// ---------------------------------------------------------------- fused-pass program
// One fused pass touches a block of 2^k amplitudes per CTA: the local index bits are
// the pass's block qubits q[0..k) (ascending, always including the lowest qubits so
// that global reads come in contiguous runs), the other qubits are fixed per CTA.
// Each thread keeps 2^R amplitudes in registers; a stage selects which R local bits
// are register bits, and every gate of the stage either targets a register bit or is
// diagonal.  Stage changes go through shared memory.  The pass's op program travels as
// a kernel parameter (constant bank), so every op field is a uniform constant load.
#ifndef QM_REG_BITS
#define QM_REG_BITS 4
#endif
constexpr int kRegBits = QM_REG_BITS;
constexpr int kMaxBlockQubits = 14;
constexpr int kMaxPassOps = 256;    // ops per pass: the program (88 B per op) is staged in shared memory
constexpr int kMaxPassGates = 120;  // gates absorbed per pass (stage changes add at most gates + 2)

constexpr uint16_t kOpTable = 4;    // FusedOp::flags: coefficients come from the batch's table
constexpr uint16_t kOpBranch = 8;   // FusedOp::flags: a table op realising a noise branch; the kernel
                                    // skips identities and applies real diagonals as scalings
// A coefficient slot passed to plan_fused with this bit set marks a noise-branch op (kOpBranch).
constexpr int32_t kSlotBranch = 1 << 24;

enum OpCode : uint8_t {
    OP_STAGE = 0,       // new register layout: reg_pos[0..R) local bit positions; `reserved` may name
                        // the local bits of the lowest thread ranks (stage_lanes)
    OP_MATRIX = 1,      // complex 2x2 on register bit `reg`
    OP_MATRIX_REAL = 2, // real 2x2 (imaginary parts all zero)
    OP_EXCHANGE = 3,    // X on register bit `reg`
    OP_DIAG = 4,        // diagonal: a on bit-zero, d on bit-one of local bit `local` (or outer bit)
    OP_NEGATE = 5,      // amplitude *= -1 where all of (cmask_local, cmask_outer) bits are set: CZ, Z
    OP_SWAP = 6,        // exchange register bits `reg` and `reg2`
    OP_DIAG_GROUP = 7,  // the next `reserved` ops are commuting diagonals (uncontrolled OP_DIAG,
                        // OP_NEGATE on at most two bits) applied together as one phase per register
};

struct FusedOp {            // 88 bytes
    uint8_t code;
    int8_t reg;             // register bit (0..R) of the target, or -1
    int8_t reg2;            // second register bit for OP_SWAP; control register bit for OP_EXCHANGE (-1: none)
    int8_t local;           // local bit of a diagonal target, -1 when the target is outside the block
    int8_t reg_pos[4];      // OP_STAGE: local bit positions of the register bits (ascending; kRegBits used)
    uint16_t cmask_local;   // controls inside the block, as local-index bits
    uint16_t flags;         // bit0: a == 1, bit1: d == 1 (diagonal)
    uint32_t cmask_outer;   // controls outside the block, as global-index bits
    uint32_t target_outer;  // outer target bit of a diagonal (global), 0 when local
    uint32_t reserved;      // kOpTable: coefficient slot in the batch table
    double coef[8];         // a, b, c, d as (re, im)
};

struct FusedPass {                  // 116 bytes
    int32_t k;                      // block qubits
    int32_t op_begin, op_count;     // range in the plan's op array
    int32_t q[kMaxBlockQubits];     // block qubits, ascending
    uint32_t block_mask;            // OR of 1<<q[i]
    int32_t stages;                 // number of register layouts
    int8_t reg_in[4];               // local register bits of the load layout (ascending; kRegBits used)
    int8_t reg_out[4];              // local register bits of the store layout (ascending; kRegBits used)
    // Local bit b is read from index bit q[b] and written to index bit q_out[b]: a permutation of
    // the block's bits when the pass relabels qubits, q itself otherwise.  Thread rank r of the
    // store layout writes index bit out_bit[r].
    int8_t q_out[16];
    int8_t out_bit[16];
};

// OP_STAGE lane order: `reserved` = n | lane[0] << 4 | lane[1] << 8 | ...; thread ranks 0..n-1 take
// local bits lane[0..n-1], the other thread ranks the remaining non-register local bits in
// ascending order.  n = 0: all thread ranks in ascending order.
inline int stage_lane_count(uint32_t reserved) { return (int)(reserved & 15u); }
inline int stage_lane(uint32_t reserved, int i) { return (int)((reserved >> (4 + 4 * i)) & 15u); }

// ---------------------------------------------------------------- dense fused gates
// Fusion widths 2..6: the circuit becomes a sequence of fused gates, each a dense 2^m x 2^m
// unitary on m <= width qubits applied as one sweep of the state (qm_dense.cpp, qm_dense.cu);
// gates wider than the width run alone on the per-gate kernel.
constexpr int kDenseMaxQubits = 6;
struct DenseOp {
    int32_t m;                      // qubits of the fused gate; 0: `gate` runs on the per-gate kernel
    int32_t q[kDenseMaxQubits];     // its qubits, ascending (local bit i is qubit q[i])
    int32_t gates;                  // circuit gates fused into it
    int64_t matrix;                 // first complex element of its transposed unitary in dense_matrices
    int64_t tc_image;               // first float of its tensor-core operand image in dense_tc, or -1
    DevGate gate;
};
// Tile geometry of one dense fused gate (states of at least 9 qubits).
struct DenseGeometry {
    uint32_t qmask, lmask, copy_mask, outer_mask;
    int32_t l_bits[12];
    int32_t cols_bits, run_bits, copies, stride, buf_elems, nbuf, buf_offset;
    uint32_t xfer_mask;
    int32_t xfer_bits, xfers, xfer_stride;
    int32_t tma_rank;   // tensor-map dimensions of the tile's box, 0 when it needs more than five
    int32_t tma_lo[5], tma_len[5], tma_tile[5];
    size_t smem;
    uint64_t items;
};

struct Plan {
    int32_t qubits = 0;
    int32_t precision = QM_FP64;
    int32_t width = 0;              // 1: per-gate path; 2..6: dense fused gates
    std::vector<DevGate> gates;     // per-gate path
    std::vector<FusedPass> passes;  // fused path
    std::vector<FusedOp> ops;
    FusedOp* d_ops = nullptr;       // device copy of ops (each pass's program is staged from it)
    std::vector<const void*> jit;   // per pass: compiled kernel (cudaKernel_t) or null
    std::vector<std::vector<unsigned char>> jit_aux;  // per pass: the compiled kernel's constants
    std::vector<int> jit_tiles;     // per pass: shared-memory tiles of the compiled kernel (2: pipelined)
    std::vector<int> jit_teams;     // per pass: teams of threads per block of the compiled kernel
    std::vector<int> jit_hist_bins; // per pass: bins of the compiled kernel's joint-mass epilogue (0: none)
    // Joint masses over these qubits (at most 8) are wanted after the plan (a damping group of the
    // trajectory runner): the last pass computes them in its epilogue when it compiles
    // (hist_fused), in the layout of launch_group_histogram.
    uint32_t hist_mask = 0;
    bool hist_fused = false;
    // Every state starts the plan as |0...0> (the batched variational evaluator): the first pass
    // writes that state into its registers instead of loading it when it compiles (zero_fused),
    // so the caller's reset can be skipped.
    bool start_zero = false;
    bool zero_fused = false;
    bool borrowed = false;          // d_ops belongs to a context buffer
    std::vector<DenseOp> dense;         // dense fused gates (widths 2..6)
    std::vector<double> dense_matrices; // their transposed unitaries, (re, im) pairs
    double* d_dense = nullptr;          // device copy of dense_matrices
    std::vector<float> dense_tc;        // tensor-core operand images of 6-qubit complex64 fused gates
    float* d_dense_tc = nullptr;
    int32_t* d_status = nullptr;        // status word the dense kernels set when a wait runs out
    int64_t planned_bytes = 0;
    int32_t launches = 0;
};
// Copies the plan's program to the device (stream-ordered) / frees it.  With `buffer`, the
// program goes into that growable device buffer instead of a new allocation (transient plans
// of one-shot executions).
int32_t plan_upload(Plan& plan, cudaStream_t stream, void** buffer = nullptr, size_t* buffer_bytes = nullptr);
void plan_release(Plan& plan);

// Builds the fused schedule (qm_planner.cpp).  Returns false with a message on error.
// slots (optional, one per gate): batch-table coefficient slot of each gate, -1 for gates
// whose coefficients are the same for every state of a batch.
bool plan_fused(const std::vector<qm_gate>& gates, int qubits, int precision, int width, Plan& plan,
                std::string& error, const std::vector<int32_t>* slots = nullptr);
int default_block_qubits(int qubits, int precision);
// Dense fused gates of at most `width` (1..6) qubits (qm_dense.cpp).
bool plan_dense(const std::vector<qm_gate>& gates, int qubits, int precision, int width, Plan& plan,
                std::string& error);
bool dense_geometry(int qubits, int precision, const DenseOp& op, DenseGeometry& g);
// Tiles of dense fused gates move as tensor-map boxes (cp.async.bulk.tensor) where their bit runs
// form at most five dimensions; QM_DENSE_TMA=0 keeps them on plain bulk copies.
constexpr int kDenseTmaMaxRank = 5;
bool dense_tma_enabled();
// Tensor-map dimensions of a tile (the runs of tile and outer index bits from bit 0 up); false when
// they need more than five.  encode_tile_map builds the map over the state at `amps` (tile runs at
// full extent in the box, outer runs at extent 1); false without the driver's encoder.
bool tile_map_dims(uint32_t tile_mask, int qubits, int32_t* lo, int32_t* len, int32_t* tile, int32_t* rank);
bool encode_tile_map(CUtensorMap* map, void* amps, int precision, int rank, const int32_t* lo, const int32_t* len,
                     const int32_t* tile);
// One dense fused gate on a state (qm_dense.cu); `matrix` is its transposed unitary in device memory.
cudaError_t launch_dense(void* amps, int qubits, int precision, const DenseOp& op, const double2* matrix,
                         int32_t* status, int sm_count, cudaStream_t s);
// 6-qubit fused gates on complex64 states of at least 11 qubits run on the tensor cores
// (qm_dense_tc.cu, 3xTF32) when QM_DENSE_TC=1; otherwise they stay on the FP32 pipes.
bool dense_tc_enabled();
extern std::atomic<int64_t> g_dense_launches, g_dense_tc_launches;  // launch counts (qm_dense_info)
bool dense_tc_supported(int qubits, int precision, const DenseOp& op);
void dense_tc_image(const double* transposed_unitary, std::vector<float>& image);
cudaError_t launch_dense_tc(void* amps, int qubits, const DenseOp& op, const float* a_image, int32_t* status,
                            int sm_count, cudaStream_t s);

// ---------------------------------------------------------------- launchers (qm_kernels.cu)
cudaError_t launch_gate(void* amps, int qubits, int precision, const DevGate& g, cudaStream_t s);
// A batch of equally sized states with one shared plan: state b at amps + b * state_stride
// (elements); ops flagged kOpTable read 8 coefficients at table + b * table_stride + 8 * op.reserved.
// With slot_count >= 0 a pass stages only slots [slot_offset, slot_offset + slot_count) of each
// row and op.reserved counts from slot_offset.
struct FusedBatch {
    int32_t states;
    uint64_t state_stride;
    const double* table;
    uint64_t table_stride;
    int32_t slot_offset = 0;
    int32_t slot_count = -1;
    double* hist = nullptr;  // joint-mass partial rows written by a compiled pass with a histogram epilogue
};
cudaError_t launch_fused(void* amps, int qubits, int precision, const FusedPass& p, const FusedOp* ops,
                         const FusedBatch* batch, cudaStream_t s);

// Kernel parameters of a fused pass (the interpreter k_fused and the passes compiled for their
// own op sequence take the same struct; its layout is mirrored in the compiled source).
struct FusedLaunch {
    uint32_t outer_mask;        // qubits outside the block
    uint32_t thread_in;         // global mask of the block qubits that are thread bits at load
    uint32_t thread_out;        // ... at store
    int32_t op_count;
    uint32_t reg_in_g[kRegBits];  // global bit of each register bit at load
    uint32_t reg_out_g[kRegBits]; // ... at store
    int32_t reg_in_l[kRegBits];   // local positions of the load layout
    int32_t cta_shift;          // log2 of the CTAs (blocks) per state
    int32_t states;
    int32_t table_slots;        // coefficient slots per state (0 without a table)
    int32_t pad;
    const FusedOp* ops;         // the pass program in device memory
    // Batches: state b lives at s + b * state_stride; ops flagged kOpTable take their
    // coefficients from table + b * table_stride + 8 * op.reserved.
    const double* table;
    uint64_t state_stride;
    uint64_t table_stride;
    uint8_t out_bit[16];        // index bit written by each thread rank at store (FusedPass::out_bit)
};
FusedLaunch fused_launch_params(int qubits, const FusedPass& p, const FusedOp* d_ops, const FusedBatch* batch);

// Passes compiled for their own op sequence (qm_jit.cpp).  A plan's passes are compiled by
// jit_prepare (NVRTC, sm_100a; structurally equal passes share a kernel); launch_plan_pass runs
// a pass with its compiled kernel when there is one, else with k_fused.
void jit_prepare(Plan& plan);
void jit_lookup(Plan& plan);  // compiled kernels already in the cache only (no compilation)
cudaError_t launch_plan_pass(const Plan& plan, size_t pass, void* amps, const FusedBatch* batch, cudaStream_t s);
cudaError_t launch_reset(void* amps, int qubits, int precision, cudaStream_t s);
cudaError_t launch_convert_from_f64(void* dst_f32, const double* src_f64, int64_t n, cudaStream_t s);
cudaError_t launch_convert_to_f64(double* dst_f64, const void* src_f32, int64_t n, cudaStream_t s);
// FP64 partial sums: writes `blocks` partial (sum, compensation) pairs into scratch.
cudaError_t launch_masses(const void* amps, int qubits, int precision, int target, double* scratch,
                          int* blocks_out, cudaStream_t s);
cudaError_t launch_pauli(void* amps, int qubits, int precision, int target, int pauli, cudaStream_t s);
cudaError_t launch_damping(void* amps, int qubits, int precision, int target, int jump, double scale,
                           double jump_scale, double stay_scale, cudaStream_t s);
// Expectation: per-block partial sums [blocks][terms + 1] (last column = mass).
struct DevPauli { uint32_t flip, sign; int32_t phase; int32_t pad; };
cudaError_t launch_expectation(const void* amps, int qubits, int precision, const DevPauli* d_terms,
                               int terms, double* scratch, int* blocks_out, cudaStream_t s);
cudaError_t launch_finish_sums(const double* partials, int blocks, int columns, double* out,
                               cudaStream_t s);
// One group of at most 8 terms sharing a flip mask into the [blocks][columns] partial table,
// blocks = expectation_blocks(qubits), never more than kReduceBlocksMax.
constexpr int kPauliGroupMax = 8;
// Grid cap of the reduction kernels (partial rows of masses, expectations, pattern masses): four
// blocks per SM of a 148-SM B200.  Fixed-size scratch (qm_noalloc.cu) is sized from it.
constexpr int kReduceBlocksMax = 148 * 4;
int expectation_blocks(int qubits);
cudaError_t launch_pauli_group(const void* amps, int qubits, int precision, uint32_t flip, int terms,
                               const uint32_t* sign, const int32_t* phase, const int32_t* column, int with_mass,
                               int mass_column, int columns, double* partials, cudaStream_t s);
// Sampling: per-block probability sums, then searches.
cudaError_t launch_block_probs(const void* amps, int qubits, int precision, double* block_sums,
                               int64_t* block_last, int* blocks_out, int* chunk_out, cudaStream_t s);
cudaError_t launch_search(const void* amps, int qubits, int precision, const double* block_prefix,
                          int blocks, int chunk, const double* targets, int shots, double margin,
                          int64_t* out, cudaStream_t s);
cudaError_t launch_collapse(void* amps, int qubits, int precision, int64_t outcome, cudaStream_t s);
// (selected sum, compensation, total sum, compensation) per block for amplitudes with
// (index & mask) == pattern; blocks = expectation_blocks(qubits).
cudaError_t launch_pattern_masses(const void* amps, int qubits, int precision, uint64_t mask, uint64_t pattern,
                                  double* scratch, int* blocks_out, cudaStream_t s);
cudaError_t launch_project(void* amps, int qubits, int precision, uint64_t mask, uint64_t pattern, double norm,
                           cudaStream_t s);

// ---------------------------------------------------------------- tiled expectation (qm_expect.cu)
constexpr int kTileMaxTerms = 256;
struct TileTerm {
    uint32_t flip_local;   // flip mask in the tile's local bits
    uint32_t sign;         // Z-sign mask over global bits
    int32_t phase;         // y_count & 3
    int32_t column;        // output column (term index)
};
struct TilePass {
    int32_t k;
    int32_t q[kMaxBlockQubits];  // tile qubits, ascending (the lowest qubits first)
    uint32_t block_mask;
    int32_t term_begin, term_count;
    int32_t with_mass;
    int32_t row_offset;          // first partial row of the pass (rows = 2^(n-k))
};
struct TilePlan {
    std::vector<TilePass> passes;
    std::vector<TileTerm> terms;
    int32_t rows_per_state = 0;
    int32_t columns = 0;         // terms + 1 (the mass)
    int32_t mass_column = 0;
    std::vector<const void*> jit;  // per pass: the kernel compiled for its term list, or null
};
// Compiles each tile pass's term list (NVRTC; cached by source) / launches one compiled pass.
void jit_prepare_tiles(TilePlan& plan, int qubits, int precision);
cudaError_t launch_expect_tile_jit(const void* kernel, const void* amps, int qubits, int precision, const TilePass& pass,
                                   int states, uint64_t state_stride, double* partials, int columns, int rows_per_state,
                                   int mass_column, cudaStream_t s);
int tile_block_qubits(int qubits, int precision);
bool plan_tiles(int qubits, int precision, const qm_pauli_term* terms, int count, TilePlan& plan, std::string& error);
cudaError_t launch_expect_tile(const void* amps, int qubits, int precision, const TilePass& pass, const TileTerm* terms,
                               int states, uint64_t state_stride, double* partials, int columns, int rows_per_state,
                               int mass_column, cudaStream_t s);
cudaError_t launch_finish_batched(const double* partials, int states, int rows, int columns, double* out,
                                  cudaStream_t s);
cudaError_t launch_reset_batched(void* amps, int qubits, int precision, int states, cudaStream_t s);
// Tiled expectation of `states` states (stride 2^qubits) into out ([states][columns]: raw sums,
// the mass in tp.mass_column); partials holds states * rows_per_state * columns doubles.
cudaError_t enqueue_tile_expectation(const void* amps, int qubits, int precision, const TilePlan& tp, int states,
                                     double* partials, double* out, cudaStream_t s);

// ---------------------------------------------------------------- noise trajectories (qm_noise.cu)
// Consecutive damping placements share one joint-mass histogram over their qubits (at most
// kGroupMaxBits of them): bins[b] = sum of |psi_i|^2 over the i whose group bits spell b.
constexpr int kGroupMaxBits = 8;
constexpr int kGroupMaxBins = 1 << kGroupMaxBits;

// Every trajectory carries a Pauli frame F = X^fx Z^fz: its true state is F applied to the stored
// state (up to a global phase).  Pauli errors and Pauli gates only update the frame, Clifford
// gates run unchanged and conjugate the frame, and every other gate or Kraus operator U runs as
// F U F on the stored state (per-trajectory coefficients in the batch table).
enum StepKind : int32_t {
    STEP_PAULI_BIT_FLIP = 0,    // NoiseKind values: a channel decision from one draw
    STEP_PAULI_PHASE_FLIP = 1,
    STEP_PAULI_DEPOLARIZING = 2,
    STEP_DAMPING = 3,           // a Kraus selection on the group's joint masses
    STEP_FRAME_X = 10,          // Pauli gate or certain flip on qubit a
    STEP_FRAME_Y = 11,
    STEP_FRAME_Z = 12,
    STEP_FRAME_H = 13,          // Clifford gates (they also run on the stored state)
    STEP_FRAME_S = 14,
    STEP_FRAME_CNOT = 15,       // control b, target a
    STEP_FRAME_CZ = 16,
    STEP_FRAME_SWAP = 17,
    STEP_CONJ = 20,             // write F U F (U = coef) for the gate on qubit a into `slot`
    STEP_FLUSH_X = 21,          // apply the frame's X on qubit a to the stored state (X or I into `slot`)
};

// One step of a trajectory's program, taken per trajectory in program order on the device.
struct Decision {
    int32_t kind;     // StepKind
    int32_t channel;  // placement index (branch output column), -1 for gate steps
    int32_t slot;     // coefficient slot (packed, per segment) written by the step, -1 for none
    int32_t bit;      // damping: bit of the target in the group's histogram
    int32_t a, b;     // qubits: target (a) and control or second operand (b)
    double p;
    double coef[8];   // STEP_CONJ: the gate's a, b, c, d
};
int histogram_ctas(int qubits);
// partials[state][cta][bin] for the group mask (global qubit bits, popcount <= kGroupMaxBits).
cudaError_t launch_group_histogram(const void* amps, int qubits, int precision, int states, uint32_t group_mask,
                                   double* partials, cudaStream_t s);
struct DecideArgs {
    const Decision* decisions;
    int32_t count;
    const double* partials;   // histogram partials of the group, or null when no damping is decided
    int32_t ctas;             // partial rows per state
    int32_t bins;
    const double* draws;      // [states][draw_stride]
    int32_t draw_stride;
    int32_t* counters;        // draws consumed so far, per state
    int32_t* status;          // per state: QM_OK, QM_E_RANGE (draws exhausted), QM_E_MASS
    int32_t* ambiguous;       // per state
    double* table;            // [states][table_stride]
    uint64_t table_stride;    // doubles
    int8_t* branches;         // [states][channels] or null
    int32_t channels;
    double margin;            // relative ambiguity margin of damping selections
    uint32_t group_mask;      // qubits of the histogram group (damping steps)
    uint32_t* frame_x;        // per state Pauli frame
    uint32_t* frame_z;
};
cudaError_t launch_decide(const DecideArgs& a, int states, cudaStream_t s);
// Welford update of mean/m2 over indices [0, len) with states first .. first+states-1 of the run;
// state b's true probability at i is the stored one at i ^ frame_x[b].
cudaError_t launch_welford(const void* amps, int precision, int states, uint64_t state_stride, int64_t len,
                           const double* masses, const uint32_t* frame_x, int64_t first, double* mean, double* m2,
                           cudaStream_t s);
// Applies X^frame_x[b] to every state b in place (pair swaps).
cudaError_t launch_frame_flip(void* amps, int qubits, int precision, int states, const uint32_t* frame_x,
                              cudaStream_t s);
cudaError_t launch_welford_finish(double* m2, int64_t len, int64_t trajectories, cudaStream_t s);

}  // namespace qm

// Born-rule sampling of one state at a raw device address (qm_sample's engine).
int32_t qm_sample_amplitudes(struct qm_context* ctx, void* amps, int32_t qubits, int32_t precision, const double* draws,
                             int32_t shots, int64_t* outcomes, int32_t* ambiguous);

// ---------------------------------------------------------------- handles
struct qm_context {
    int32_t device = 0;
    int32_t sm_count = 0;
    int32_t profiling = 0;
    int32_t fusion_width = 0;
    int64_t device_budget = 0;
    int64_t staging_budget = 0;
    int64_t device_in_use = 0;
    bool disposed = false;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev_start = nullptr, ev_stop = nullptr;
    std::recursive_mutex mu;
    // growable scratch (reduction partials, small uploads)
    void* scratch = nullptr;
    size_t scratch_bytes = 0;
    double* host_scratch = nullptr;   // pinned, for small downloads
    size_t host_scratch_bytes = 0;
    // device buffer of the host-buffer entry points (qm_execute_host, qm_noise_apply_host)
    void* staging = nullptr;
    size_t staging_bytes = 0;
    // device copy of the op program of one-shot executions (reused, grows as needed)
    void* program = nullptr;
    size_t program_bytes = 0;
    // page-locked bounce buffers of whole-state copies from pageable host memory (qm_transfer.cpp)
    void* bounce[2] = {nullptr, nullptr};
    cudaEvent_t bounce_done[2] = {nullptr, nullptr};
};
// Whole-state copies with a caller's host buffer on the context's stream (qm_transfer.cpp):
// host_to_device returns once the host buffer has been read (the device copy may still be in
// flight on the stream); device_to_host returns once the host buffer holds the data.
cudaError_t host_to_device(qm_context* ctx, void* dev, const void* host, size_t bytes);
cudaError_t device_to_host(qm_context* ctx, void* host, const void* dev, size_t bytes);
void release_bounce(qm_context* ctx);

struct qm_state {
    qm_context* ctx = nullptr;
    int32_t qubits = 0;
    int32_t precision = QM_FP64;
    void* amps = nullptr;
    int64_t bytes = 0;
};

struct qm_plan {
    qm_context* ctx = nullptr;
    qm::Plan plan;
};
