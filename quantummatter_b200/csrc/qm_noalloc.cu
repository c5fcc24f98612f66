// qm_noalloc.cu -- the allocation-free Pauli-sum expectation of libqmb200.so.
//
// Some callers cannot allocate device memory at the moment they need an expectation value:
// a host whose device memory all belongs to its own pool allocator (a stray cudaMalloc would
// bypass the pool and may find no memory left when the pool holds nearly all of the GPU's
// memory), or a latency-bound loop where the device-wide synchronisation implied by cudaMalloc
// and cudaFree is not acceptable.  qm_expectation_pauli_noalloc serves them: the caller passes
// the device amplitudes, the terms and host output arrays; the only scratch memory, the
// per-block partial sums of the reduction, is the file-scope device array below.
//
// The kernels are the same flip-group expectation passes and fixed-order column sum that
// qm_expectation_pauli runs for small states, so results agree with it to rounding of the
// summation order (FP64 accumulation either way).
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>

#include "qm_internal.h"

using namespace qm;

namespace {

constexpr int kMaxTerms = QM_NOALLOC_MAX_TERMS;
constexpr int kColumns = kMaxTerms + 1;  // the Born mass rides in the last column
constexpr int kMaxBlocks = kReduceBlocksMax;  // expectation_blocks() never returns more
static_assert(kMaxBlocks >= 1 && kMaxBlocks <= 4096, "the fixed scratch is sized from the reduction grid cap");
constexpr size_t kScratchDoubles = (size_t)(kMaxBlocks + 1) * kColumns;
constexpr int kMaxDevices = 64;

// [kMaxBlocks][kColumns] partial sums followed by one row of finished column sums: about
// 304 KB that every GPU which loads the library holds until the process exits.  Every call
// shares it and it keeps the last call's contents.
static __device__ __align__(256) double g_scratch[kScratchDoubles];

std::mutex g_mutex;
double* g_address[kMaxDevices] = {};

// Device address of g_scratch on the current device, looked up once per device.  In host
// code `g_scratch` names a host-side stand-in, not device memory, so the kernels get this
// address instead.  The address is cached for the life of the process: a cudaDeviceReset by
// the host unloads the module that holds the array, so the entry point must not be used across
// one.  The first lookup also loads that module (CUDA loads modules lazily), which reserves the
// array's memory on the device.
int32_t scratch_address(double** out) {
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    if (device < 0 || device >= kMaxDevices) return fail(QM_E_DEVICE, "device ordinal beyond the supported range");
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!g_address[device]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress");
        g_address[device] = static_cast<double*>(p);
    }
    *out = g_address[device];
    return QM_OK;
}

}  // namespace

extern "C" int32_t qm_expectation_pauli_noalloc(const void* amplitudes, int32_t qubits, int32_t precision,
                                                const qm_pauli_term* terms, int32_t count, double* per_term,
                                                double* mass, void* stream) {
    if (!amplitudes) return fail(QM_E_ARG, "amplitudes is null");
    if (qubits < 1 || qubits > 30) return fail(QM_E_RANGE, "qubits must be between 1 and 30");
    if (precision != QM_FP64 && precision != QM_FP32) return fail(QM_E_RANGE, "unknown precision");
    if (count < 0 || count > kMaxTerms)
        return fail(QM_E_RANGE, "qm_expectation_pauli_noalloc takes at most QM_NOALLOC_MAX_TERMS (64) terms");
    if (count > 0 && (!terms || !per_term)) return fail(QM_E_ARG, "terms or per_term is null");
    const uint32_t all = (uint32_t)((1ull << qubits) - 1);
    for (int32_t t = 0; t < count; ++t)
        if ((terms[t].flip_mask | terms[t].sign_mask) & ~all) return fail(QM_E_ARG, "Observable and state sizes must match.");
    double* scratch = nullptr;
    int32_t rc = scratch_address(&scratch);
    if (rc) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int blocks = expectation_blocks(qubits);
    if (blocks < 1 || blocks > kMaxBlocks)
        return fail(QM_E_RANGE, "the reduction grid exceeds the fixed scratch of qm_expectation_pauli_noalloc");
    const int columns = count + 1;
    double* partials = scratch;                            // [blocks][columns]
    double* sums = scratch + (size_t)kMaxBlocks * kColumns; // [columns]
    QM_CUDA(cudaMemsetAsync(partials, 0, sizeof(double) * (size_t)blocks * columns, st));
    // one pass per group of terms with the same flip mask (at most kPauliGroupMax per pass)
    bool used[kMaxTerms] = {};
    bool mass_done = false;
    for (int32_t i = 0; i < count; ++i) {
        if (used[i]) continue;
        const uint32_t flip = terms[i].flip_mask;
        uint32_t sign[kPauliGroupMax];
        int32_t phase[kPauliGroupMax], column[kPauliGroupMax];
        int n = 0;
        for (int32_t j = i; j < count && n < kPauliGroupMax; ++j) {
            if (used[j] || terms[j].flip_mask != flip) continue;
            used[j] = true;
            sign[n] = terms[j].sign_mask;
            phase[n] = terms[j].y_count & 3;
            column[n] = j;
            ++n;
        }
        QM_CUDA(launch_pauli_group(amplitudes, qubits, precision, flip, n, sign, phase, column, mass_done ? 0 : 1,
                                   count, columns, partials, st));
        mass_done = true;
    }
    if (!mass_done)
        QM_CUDA(launch_pauli_group(amplitudes, qubits, precision, 0, 0, nullptr, nullptr, nullptr, 1, count, columns,
                                   partials, st));
    QM_CUDA(launch_finish_sums(partials, blocks, columns, sums, st));
    double host[kColumns];
    QM_CUDA(cudaMemcpyAsync(host, sums, sizeof(double) * columns, cudaMemcpyDeviceToHost, st));
    QM_CUDA(cudaStreamSynchronize(st));
    const double total = host[count];
    if (mass) *mass = total;
    if (!std::isfinite(total) || total <= 0) return fail(QM_E_MASS, "The state has no finite positive probability mass.");
    for (int32_t t = 0; t < count; ++t) {
        if (!std::isfinite(host[t])) return fail(QM_E_MASS, "The observable accumulation is nonfinite.");
        per_term[t] = host[t] / total;
    }
    return QM_OK;
}
