// qm_api.cpp -- C ABI of libqmb200.so (declared in include/qm_b200.h).
//
// Host runtime: contexts (one CUDA stream each, calls serialised like the reference's
// SemaphoreSlim, CudaStateVectorBackend.cs:16,115,186), device states, fused plans, the
// drop-in host-buffer entry points, noise primitives, observables and sampling.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "qm_internal.h"

namespace qm {

static thread_local std::string g_last_error;

void set_error(const std::string& message) { g_last_error = message; }

int32_t fail(int32_t status, const std::string& message) {
    g_last_error = message;
    return status;
}

int32_t cuda_fail(cudaError_t err, const char* what) {
    std::string m = std::string(what) + ": " + cudaGetErrorString(err);
    if (err == cudaErrorMemoryAllocation) return fail(QM_E_OOM, m);
    if (err == cudaErrorNoDevice || err == cudaErrorInsufficientDriver) return fail(QM_E_DEVICE, m);
    return fail(QM_E_DEVICE, m);
}

}  // namespace qm

using namespace qm;

namespace {

constexpr int64_t kDefaultBudget = 512ll * 1024 * 1024;

bool cancelled(const volatile int32_t* cancel) { return cancel != nullptr && *cancel != 0; }

int32_t ensure_scratch(qm_context* ctx, size_t bytes) {
    if (ctx->scratch_bytes >= bytes) return QM_OK;
    if (ctx->scratch) {
        cudaStreamSynchronize(ctx->stream);
        cudaFree(ctx->scratch);
        ctx->scratch = nullptr;
        ctx->scratch_bytes = 0;
    }
    size_t sz = std::max<size_t>(bytes, 1 << 20);
    QM_CUDA(cudaMalloc(&ctx->scratch, sz));
    ctx->scratch_bytes = sz;
    return QM_OK;
}

int32_t ensure_host_scratch(qm_context* ctx, size_t bytes) {
    if (ctx->host_scratch_bytes >= bytes) return QM_OK;
    if (ctx->host_scratch) {
        cudaStreamSynchronize(ctx->stream);
        cudaFreeHost(ctx->host_scratch);
        ctx->host_scratch = nullptr;
        ctx->host_scratch_bytes = 0;
    }
    size_t sz = std::max<size_t>(bytes, 1 << 16);
    void* p = nullptr;
    QM_CUDA(cudaMallocHost(&p, sz));
    ctx->host_scratch = static_cast<double*>(p);
    ctx->host_scratch_bytes = sz;
    return QM_OK;
}

// ---------------------------------------------------------------- gate preparation

// Builder validation (src/QuantumMatter.Core/QuantumCircuit.cs:97-134).
int32_t validate_operations(const qm_operation* ops, int32_t count, int32_t qubits) {
    if (qubits < 1 || qubits > 30) return fail(QM_E_RANGE, "qubits must be between 1 and 30");
    if (count < 0) return fail(QM_E_RANGE, "gate count must be nonnegative");
    if (count > 0 && !ops) return fail(QM_E_ARG, "operations is null");
    for (int32_t i = 0; i < count; ++i) {
        const qm_operation& o = ops[i];
        if (o.kind < 0 || o.kind > QM_GATE_TOFFOLI) return fail(QM_E_UNSUPPORTED, "unsupported gate kind");
        if ((uint32_t)o.target >= (uint32_t)qubits) return fail(QM_E_RANGE, "target out of range");
        if (o.control >= 0) {
            if (o.control >= qubits) return fail(QM_E_RANGE, "control out of range");
            if (o.control == o.target) return fail(QM_E_ARG, "the two qubits must differ");
        } else if (o.control != -1) {
            return fail(QM_E_RANGE, "control out of range");
        }
        if (o.second_control >= 0) {
            if (o.second_control >= qubits) return fail(QM_E_RANGE, "second control out of range");
            if (o.second_control == o.target || o.second_control == o.control)
                return fail(QM_E_ARG, "all three qubits must differ");
        } else if (o.second_control != -1) {
            return fail(QM_E_RANGE, "second control out of range");
        }
        if (!std::isfinite(o.angle)) return fail(QM_E_RANGE, "angle must be finite");
        if ((o.kind == QM_GATE_CNOT || o.kind == QM_GATE_SWAP) && o.control < 0)
            return fail(QM_E_ARG, "two-qubit gate needs a second operand");
        if (o.kind == QM_GATE_TOFFOLI && (o.control < 0 || o.second_control < 0))
            return fail(QM_E_ARG, "Toffoli needs two controls");
        if (o.kind == QM_GATE_UNITARY)
            for (double v : o.unitary)
                if (!std::isfinite(v)) return fail(QM_E_RANGE, "matrix entries must be finite");
    }
    return QM_OK;
}

void set_c(double* dst, double re, double im) {
    dst[0] = re;
    dst[1] = im;
}

// PreparedStateVectorGate.Prepare (src/QuantumMatter.Infrastructure/PreparedStateVectorGate.cs:13-70),
// coefficients from the host libm exactly as the reference evaluates them.
void prepare_one(const qm_operation& o, qm_gate& p) {
    std::memset(&p, 0, sizeof p);
    uint32_t mask = o.control >= 0 ? (1u << o.control) : 0u;
    if (o.second_control >= 0) mask |= 1u << o.second_control;
    p.target = o.target;
    p.control_mask = mask;
    p.swap_control = -1;
    p.kernel = QM_KERNEL_MATRIX;
    switch (o.kind) {
    case QM_GATE_I: p.kernel = QM_KERNEL_IDENTITY; break;
    case QM_GATE_X:
    case QM_GATE_CNOT:
    case QM_GATE_TOFFOLI: p.kernel = QM_KERNEL_EXCHANGE; break;
    case QM_GATE_SWAP:
        p.kernel = QM_KERNEL_SWAP;
        p.control_mask = 0;
        p.swap_control = o.control;
        break;
    case QM_GATE_H: {
        double h = std::sqrt(0.5);
        p.kernel = QM_KERNEL_HADAMARD;
        set_c(p.a, h, 0); set_c(p.b, h, 0); set_c(p.c, h, 0); set_c(p.d, -h, 0);
        break;
    }
    case QM_GATE_Y: set_c(p.b, -0.0, -1.0); set_c(p.c, 0.0, 1.0); break;
    case QM_GATE_Z: p.kernel = QM_KERNEL_DIAGONAL; set_c(p.a, 1, 0); set_c(p.d, -1, 0); break;
    case QM_GATE_S: p.kernel = QM_KERNEL_DIAGONAL; set_c(p.a, 1, 0); set_c(p.d, 0, 1); break;
    case QM_GATE_SDG: p.kernel = QM_KERNEL_DIAGONAL; set_c(p.a, 1, 0); set_c(p.d, -0.0, -1); break;
    case QM_GATE_T:
        p.kernel = QM_KERNEL_DIAGONAL;
        set_c(p.a, 1, 0);
        set_c(p.d, std::cos(M_PI / 4), std::sin(M_PI / 4));
        break;
    case QM_GATE_TDG:
        p.kernel = QM_KERNEL_DIAGONAL;
        set_c(p.a, 1, 0);
        set_c(p.d, std::cos(-M_PI / 4), std::sin(-M_PI / 4));
        break;
    case QM_GATE_PHASE:
        p.kernel = QM_KERNEL_DIAGONAL;
        set_c(p.a, 1, 0);
        set_c(p.d, std::cos(o.angle), std::sin(o.angle));
        break;
    case QM_GATE_RX: {
        double c = std::cos(o.angle / 2), s = std::sin(o.angle / 2);
        // -i * sin as the Complex product (-ImaginaryOne) * sin
        set_c(p.a, c, 0); set_c(p.b, -0.0 * s, -1.0 * s); set_c(p.c, -0.0 * s, -1.0 * s); set_c(p.d, c, 0);
        break;
    }
    case QM_GATE_RY: {
        double c = std::cos(o.angle / 2), s = std::sin(o.angle / 2);
        set_c(p.a, c, 0); set_c(p.b, -s, 0); set_c(p.c, s, 0); set_c(p.d, c, 0);
        break;
    }
    case QM_GATE_RZ:
        p.kernel = QM_KERNEL_DIAGONAL;
        set_c(p.a, std::cos(-o.angle / 2), std::sin(-o.angle / 2));
        set_c(p.d, std::cos(o.angle / 2), std::sin(o.angle / 2));
        break;
    case QM_GATE_UNITARY:
        std::memcpy(p.a, &o.unitary[0], 16);
        std::memcpy(p.b, &o.unitary[2], 16);
        std::memcpy(p.c, &o.unitary[4], 16);
        std::memcpy(p.d, &o.unitary[6], 16);
        break;
    default: break;
    }
}

int32_t validate_gates(const qm_gate* gates, int32_t count, int32_t qubits) {
    if (count < 0) return fail(QM_E_RANGE, "gate count must be nonnegative");
    if (count > 0 && !gates) return fail(QM_E_ARG, "gates is null");
    uint32_t all = (uint32_t)((1ull << qubits) - 1);
    for (int32_t i = 0; i < count; ++i) {
        const qm_gate& g = gates[i];
        if (g.kernel < QM_KERNEL_IDENTITY || g.kernel > QM_KERNEL_SWAP) return fail(QM_E_UNSUPPORTED, "unknown kernel");
        if ((uint32_t)g.target >= (uint32_t)qubits) return fail(QM_E_RANGE, "target out of range");
        if (g.control_mask & ~all) return fail(QM_E_RANGE, "control out of range");
        if (g.control_mask & (1u << g.target)) return fail(QM_E_ARG, "control equals target");
        if (g.kernel == QM_KERNEL_SWAP) {
            if ((uint32_t)g.swap_control >= (uint32_t)qubits) return fail(QM_E_RANGE, "swap operand out of range");
            if (g.swap_control == g.target) return fail(QM_E_ARG, "swap operands must differ");
            if (g.control_mask & (1u << g.swap_control)) return fail(QM_E_ARG, "control equals swap operand");
        }
        const double* v[4] = {g.a, g.b, g.c, g.d};
        for (auto* c : v)
            if (!std::isfinite(c[0]) || !std::isfinite(c[1])) return fail(QM_E_RANGE, "coefficients must be finite");
    }
    return QM_OK;
}

// ---------------------------------------------------------------- plan execution

}  // namespace

namespace qm {

int32_t validate_prepared_gates(const qm_gate* gates, int32_t count, int32_t qubits) {
    return validate_gates(gates, count, qubits);
}

int32_t plan_upload(Plan& plan, cudaStream_t stream, void** buffer, size_t* buffer_bytes) {
    if (!plan.dense.empty() && !plan.d_status) {
        QM_CUDA(cudaMalloc(&plan.d_status, sizeof(int32_t)));
        QM_CUDA(cudaMemsetAsync(plan.d_status, 0, sizeof(int32_t), stream));
        if (!plan.dense_matrices.empty()) {
            const size_t mbytes = plan.dense_matrices.size() * sizeof(double);
            QM_CUDA(cudaMalloc(&plan.d_dense, mbytes));
            QM_CUDA(cudaMemcpyAsync(plan.d_dense, plan.dense_matrices.data(), mbytes, cudaMemcpyHostToDevice, stream));
        }
        if (!plan.dense_tc.empty()) {
            const size_t ibytes = plan.dense_tc.size() * sizeof(float);
            QM_CUDA(cudaMalloc(&plan.d_dense_tc, ibytes));
            QM_CUDA(cudaMemcpyAsync(plan.d_dense_tc, plan.dense_tc.data(), ibytes, cudaMemcpyHostToDevice, stream));
        }
    }
    if (plan.ops.empty() || plan.d_ops) return QM_OK;
    const size_t bytes = plan.ops.size() * sizeof(FusedOp);
    if (buffer) {
        if (*buffer_bytes < bytes) {
            if (*buffer) {
                cudaStreamSynchronize(stream);
                cudaFree(*buffer);
            }
            *buffer = nullptr;
            *buffer_bytes = 0;
            QM_CUDA(cudaMalloc(buffer, bytes * 2));
            *buffer_bytes = bytes * 2;
        }
        plan.d_ops = static_cast<FusedOp*>(*buffer);
        plan.borrowed = true;
    } else {
        QM_CUDA(cudaMalloc(&plan.d_ops, bytes));
    }
    QM_CUDA(cudaMemcpyAsync(plan.d_ops, plan.ops.data(), bytes, cudaMemcpyHostToDevice, stream));
    return QM_OK;
}

void plan_release(Plan& plan) {
    if (plan.d_ops && !plan.borrowed) cudaFree(plan.d_ops);  // cudaFree waits for work using the buffer
    plan.d_ops = nullptr;
    plan.borrowed = false;
    if (plan.d_dense) cudaFree(plan.d_dense);
    if (plan.d_dense_tc) cudaFree(plan.d_dense_tc);
    if (plan.d_status) cudaFree(plan.d_status);
    plan.d_dense = nullptr;
    plan.d_dense_tc = nullptr;
    plan.d_status = nullptr;
}

// After the stream has finished a dense plan: QM_E_TIMEOUT if one of its kernels gave up a wait.
int32_t dense_status(const Plan& plan) {
    if (!plan.d_status) return QM_OK;
    int32_t status = 0;
    QM_CUDA(cudaMemcpy(&status, plan.d_status, sizeof status, cudaMemcpyDeviceToHost));
    if (status == 0) return QM_OK;
    cudaMemset(plan.d_status, 0, sizeof(int32_t));
    return fail(QM_E_TIMEOUT, "a dense fused-gate kernel gave up waiting for its tile copies");
}

}  // namespace qm

namespace {

// Fusion widths: 0 = planner default, 1 = one launch per gate, 2..6 = dense fused gates of at
// most that many qubits, 9..14 = fused blocks of that many qubits.  7 and 8 are neither.
constexpr const char* kWidthRule =
    "fusion width must be 0, 1, 2..6 (dense fused gates) or 9..14 (fused blocks)";
bool valid_width(int32_t w) { return (w >= 0 && w <= kDenseMaxQubits) || (w >= 9 && w <= 14); }

// transient plans (one-shot executions) borrow the context's program buffer
int32_t build_plan(qm_context* ctx, int32_t qubits, int32_t precision, const qm_gate* gates, int32_t count,
                   int32_t width, Plan& plan, bool transient = false) {
    std::vector<qm_gate> list(gates, gates + count);
    std::string err;
    if (width == 0) width = ctx->fusion_width;
    if (!plan_fused(list, qubits, precision, width, plan, err)) return fail(QM_E_ARG, "planner: " + err);
    // one-shot executions of large states run the compiled passes already built for the same
    // structures; they never wait for a compilation.  Below 26 qubits a pass takes well under a
    // millisecond, about what generating the plan's sources for the lookup costs on the host,
    // so those run the interpreter.
    if (transient && qubits >= 26) jit_lookup(plan);
    if (transient) return plan_upload(plan, ctx->stream, &ctx->program, &ctx->program_bytes);
    return plan_upload(plan, ctx->stream);
}

void free_plan(Plan& plan) { plan_release(plan); }

// Launches the plan on `amps`.  With a cancel flag the stream is synchronised every 32
// launches and the flag polled, as the reference bounds queued work
// (CudaStateVectorBackend.cs:155-159).
int32_t run_plan(qm_context* ctx, const Plan& plan, void* amps, const volatile int32_t* cancel) {
    int launched = 0;
    auto chunk_boundary = [&]() -> int32_t {
        if (cancel && (++launched & 31) == 0) {
            QM_CUDA(cudaStreamSynchronize(ctx->stream));
            if (cancelled(cancel)) return fail(QM_E_CANCELLED, "operation cancelled");
        }
        return QM_OK;
    };
    if (plan.width == 1) {
        for (const DevGate& g : plan.gates) {
            QM_CUDA(launch_gate(amps, plan.qubits, plan.precision, g, ctx->stream));
            int32_t rc = chunk_boundary();
            if (rc) return rc;
        }
    } else if (plan.width <= kDenseMaxQubits) {
        for (const DenseOp& op : plan.dense) {
            if (op.m == 0)
                QM_CUDA(launch_gate(amps, plan.qubits, plan.precision, op.gate, ctx->stream));
            else if (op.tc_image >= 0)
                QM_CUDA(launch_dense_tc(amps, plan.qubits, op, plan.d_dense_tc + op.tc_image, plan.d_status,
                                        ctx->sm_count, ctx->stream));
            else
                QM_CUDA(launch_dense(amps, plan.qubits, plan.precision, op,
                                     reinterpret_cast<const double2*>(plan.d_dense) + op.matrix, plan.d_status,
                                     ctx->sm_count, ctx->stream));
            int32_t rc = chunk_boundary();
            if (rc) return rc;
        }
    } else {
        for (size_t i = 0; i < plan.passes.size(); ++i) {
            QM_CUDA(launch_plan_pass(plan, i, amps, nullptr, ctx->stream));
            int32_t rc = chunk_boundary();
            if (rc) return rc;
        }
    }
    return QM_OK;
}

int32_t check_state(qm_state* st) {
    if (!st || !st->ctx) return fail(QM_E_ARG, "state is null");
    if (st->ctx->disposed) return fail(QM_E_DISPOSED, "context disposed");
    return QM_OK;
}

int32_t device_buffer(qm_context* ctx, size_t bytes, void** out);

}  // namespace

// ====================================================================== runtime

extern "C" int32_t qm_abi_version(void) { return QM_ABI_VERSION; }

extern "C" int32_t qm_last_error(char* buffer, size_t size) {
    if (!buffer || size == 0) return QM_E_ARG;
    size_t n = std::min(size - 1, g_last_error.size());
    std::memcpy(buffer, g_last_error.data(), n);
    buffer[n] = '\0';
    return QM_OK;
}

extern "C" void qm_options_default(qm_options* o) {
    if (!o) return;
    std::memset(o, 0, sizeof *o);
    o->device_budget_bytes = kDefaultBudget;
    o->staging_budget_bytes = kDefaultBudget;
}

extern "C" int32_t qm_device_count(int32_t* count) {
    if (!count) return fail(QM_E_ARG, "count is null");
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        n = 0;
    }
    *count = n;
    return QM_OK;
}

extern "C" int32_t qm_device_info_get(int32_t index, qm_device_info* info) {
    if (!info) return fail(QM_E_ARG, "info is null");
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return fail(QM_E_DEVICE, "no compatible NVIDIA CUDA device or driver");
    }
    if (index < 0 || index >= n) return fail(QM_E_RANGE, "device index is not available");
    cudaDeviceProp prop;
    QM_CUDA(cudaGetDeviceProperties(&prop, index));
    std::memset(info, 0, sizeof *info);
    info->index = index;
    info->sm_count = prop.multiProcessorCount;
    info->major = prop.major;
    info->minor = prop.minor;
    int drv = 0;
    cudaDriverGetVersion(&drv);
    info->driver_version = drv;
    info->memory_bytes = (int64_t)prop.totalGlobalMem;
    std::snprintf(info->name, sizeof info->name, "%s", prop.name);
    return QM_OK;
}

extern "C" int32_t qm_context_create(const qm_options* options, qm_context** out) {
    if (!out) return fail(QM_E_ARG, "context out-pointer is null");
    *out = nullptr;
    qm_options o;
    if (options) o = *options; else qm_options_default(&o);
    if (o.device_index < 0) return fail(QM_E_RANGE, "device index must be nonnegative");
    if (o.device_budget_bytes < 32 || o.staging_budget_bytes < 32) return fail(QM_E_RANGE, "budgets must be at least 32 bytes");
    if (!valid_width(o.fusion_width)) return fail(QM_E_RANGE, kWidthRule);
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return fail(QM_E_DEVICE,
                    "No compatible NVIDIA CUDA device/driver was found. Select a CPU backend explicitly or install a "
                    "compatible NVIDIA driver.");
    }
    if (o.device_index >= n) return fail(QM_E_RANGE, "CUDA device index is not available.");
    std::unique_ptr<qm_context> ctx(new qm_context());
    ctx->device = o.device_index;
    ctx->profiling = o.enable_profiling;
    ctx->fusion_width = o.fusion_width;
    ctx->device_budget = o.device_budget_bytes;
    ctx->staging_budget = o.staging_budget_bytes;
    QM_CUDA(cudaSetDevice(ctx->device));
    cudaDeviceProp prop;
    QM_CUDA(cudaGetDeviceProperties(&prop, ctx->device));
    ctx->sm_count = prop.multiProcessorCount;
    QM_CUDA(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
    QM_CUDA(cudaEventCreate(&ctx->ev_start));
    QM_CUDA(cudaEventCreate(&ctx->ev_stop));
    *out = ctx.release();
    return QM_OK;
}

extern "C" int32_t qm_context_destroy(qm_context* ctx) {
    if (!ctx) return QM_OK;
    {
        std::lock_guard<std::recursive_mutex> lock(ctx->mu);
        cudaSetDevice(ctx->device);
        if (ctx->stream) cudaStreamSynchronize(ctx->stream);
        if (ctx->scratch) cudaFree(ctx->scratch);
        if (ctx->host_scratch) cudaFreeHost(ctx->host_scratch);
        if (ctx->staging) cudaFree(ctx->staging);
        if (ctx->program) cudaFree(ctx->program);
        release_bounce(ctx);
        if (ctx->ev_start) cudaEventDestroy(ctx->ev_start);
        if (ctx->ev_stop) cudaEventDestroy(ctx->ev_stop);
        if (ctx->stream) cudaStreamDestroy(ctx->stream);
        ctx->disposed = true;
    }
    delete ctx;
    return QM_OK;
}

extern "C" int32_t qm_host_alloc(qm_context* ctx, int64_t bytes, void** ptr) {
    if (!ctx || !ptr) return fail(QM_E_ARG, "null argument");
    if (bytes <= 0) return fail(QM_E_RANGE, "bytes must be positive");
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    QM_CUDA(cudaSetDevice(ctx->device));
    QM_CUDA(cudaHostAlloc(ptr, (size_t)bytes, cudaHostAllocPortable));
    return QM_OK;
}

extern "C" int32_t qm_host_free(qm_context* ctx, void* ptr) {
    if (!ctx) return fail(QM_E_ARG, "context is null");
    if (!ptr) return QM_OK;
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    QM_CUDA(cudaFreeHost(ptr));
    return QM_OK;
}

extern "C" int32_t qm_prepare_gates(const qm_operation* ops, int32_t count, int32_t qubits, qm_gate* gates) {
    int32_t rc = validate_operations(ops, count, qubits);
    if (rc) return rc;
    if (count > 0 && !gates) return fail(QM_E_ARG, "gates is null");
    for (int32_t i = 0; i < count; ++i) prepare_one(ops[i], gates[i]);
    return QM_OK;
}

// ====================================================================== drop-in port

namespace {

// The context keeps one device buffer for the host-buffer entry points (reused across
// calls; counted against the device budget while it exists).
int32_t device_buffer(qm_context* ctx, size_t bytes, void** out) {
    if (ctx->staging_bytes < bytes) {
        if (ctx->staging) {
            cudaStreamSynchronize(ctx->stream);
            cudaFree(ctx->staging);
            ctx->staging = nullptr;
            ctx->staging_bytes = 0;
        }
        QM_CUDA(cudaMalloc(&ctx->staging, bytes));
        ctx->staging_bytes = bytes;
    }
    *out = ctx->staging;
    return QM_OK;
}

double seconds_between(cudaEvent_t a, cudaEvent_t b) {
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    return ms * 1e-3;
}

}  // namespace

extern "C" int32_t qm_execute_host(qm_context* ctx, int32_t qubits, const qm_operation* ops, int32_t count,
                                   double* amps, int64_t length, const volatile int32_t* cancel, qm_profile* profile) {
    if (!ctx) return fail(QM_E_ARG, "context is null");
    if (qubits < 1 || qubits > 30) return fail(QM_E_RANGE, "qubits must be between 1 and 30");
    if (!amps || length != (int64_t(1) << qubits)) return fail(QM_E_ARG, "Buffer length must equal 2^qubitCount.");
    if (cancelled(cancel)) return fail(QM_E_CANCELLED, "operation cancelled");
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    if (ctx->disposed) return fail(QM_E_DISPOSED, "context disposed");
    if (cancelled(cancel)) return fail(QM_E_CANCELLED, "operation cancelled");
    const int64_t bytes = 16 * length;
    size_t free_b = 0, total_b = 0;
    QM_CUDA(cudaSetDevice(ctx->device));
    QM_CUDA(cudaMemGetInfo(&free_b, &total_b));
    if (bytes > ctx->device_budget || bytes > (int64_t)total_b || bytes > ctx->staging_budget)
        return fail(QM_E_BUDGET, "CUDA state exceeds the device or host staging memory budget.");
    int32_t rc = validate_operations(ops, count, qubits);
    if (rc) return rc;
    std::vector<qm_gate> gates((size_t)count);
    for (int32_t i = 0; i < count; ++i) prepare_one(ops[i], gates[(size_t)i]);
    void* dev = nullptr;
    rc = device_buffer(ctx, (size_t)bytes, &dev);
    if (rc) return rc;

    cudaEvent_t t0 = nullptr, t1 = nullptr, t2 = nullptr, t3 = nullptr;
    if (profile) {
        cudaEventCreate(&t0); cudaEventCreate(&t1); cudaEventCreate(&t2); cudaEventCreate(&t3);
        cudaEventRecord(t0, ctx->stream);
    }
    // The upload is queued first: from a page-locked buffer it returns at once, and the plan is
    // built (and its compiled passes looked up) on the host while the copy engine moves the state.
    cudaError_t e = host_to_device(ctx, dev, amps, (size_t)bytes);
    if (e == cudaSuccess && profile) cudaEventRecord(t1, ctx->stream);
    Plan plan;
    if (e == cudaSuccess) rc = build_plan(ctx, qubits, QM_FP64, gates.data(), count, 0, plan, true);
    if (e == cudaSuccess && rc == QM_OK) rc = run_plan(ctx, plan, dev, cancel);
    if (e == cudaSuccess && rc == QM_OK) {
        if (profile) cudaEventRecord(t2, ctx->stream);
        e = cudaStreamSynchronize(ctx->stream);
    }
    if (e == cudaSuccess && rc == QM_OK) rc = dense_status(plan);
    if (e == cudaSuccess && rc == QM_OK && cancelled(cancel)) rc = fail(QM_E_CANCELLED, "operation cancelled");
    // commit: only after every launch completed and the last cancellation check passed
    if (e == cudaSuccess && rc == QM_OK) {
        e = device_to_host(ctx, amps, dev, (size_t)bytes);
        if (e == cudaSuccess && profile) cudaEventRecord(t3, ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    }
    cudaStreamSynchronize(ctx->stream);  // nothing queued may outlive this call
    if (e != cudaSuccess) rc = cuda_fail(e, "qm_execute_host");
    if (profile) {
        if (rc == QM_OK) {
            profile->transfer_seconds = seconds_between(t0, t1) + seconds_between(t2, t3);
            profile->device_seconds = seconds_between(t1, t2);
            profile->state_bytes = bytes;
            profile->kernel_launches = plan.launches;
            profile->passes = (int32_t)plan.passes.size();
            profile->planned_bytes = plan.planned_bytes;
        }
        cudaEventDestroy(t0); cudaEventDestroy(t1); cudaEventDestroy(t2); cudaEventDestroy(t3);
    }
    free_plan(plan);
    return rc;
}

namespace {

// Masses of target-zero and target-one amplitudes of a device array.
int32_t device_masses(qm_context* ctx, void* amps, int qubits, int precision, int target, double* m0, double* m1) {
    int32_t rc = ensure_scratch(ctx, sizeof(double) * (4 * 148 * 4 + 8));
    if (rc) return rc;
    rc = ensure_host_scratch(ctx, 4 * sizeof(double));
    if (rc) return rc;
    double* partial = static_cast<double*>(ctx->scratch);
    int blocks = 0;
    QM_CUDA(launch_masses(amps, qubits, precision, target, partial, &blocks, ctx->stream));
    double* out = partial + 4 * blocks;
    QM_CUDA(launch_finish_sums(partial, blocks, 4, out, ctx->stream));
    QM_CUDA(cudaMemcpyAsync(ctx->host_scratch, out, 4 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    QM_CUDA(cudaStreamSynchronize(ctx->stream));
    *m0 = ctx->host_scratch[0] + ctx->host_scratch[1];
    *m1 = ctx->host_scratch[2] + ctx->host_scratch[3];
    return QM_OK;
}

// The branch selection of CpuNoiseChannelBackend.Apply (CpuNoiseChannelBackend.cs:26-57,108-121)
// on masses computed on the device.  draw() is called exactly where the reference calls
// random.NextDouble().
struct Branch {
    int pauli = 0;     // 0 identity, 1 X, 2 Y, 3 Z
    bool damping = false;
    bool jump = false;
    double scale = 1, jump_scale = 0, stay_scale = 1;
};

template <typename Draw>
int32_t choose_branch(int32_t kind, double p, Draw draw, bool have_masses, double zero_mass, double one_mass,
                      Branch& b) {
    if (kind == 3) {
        b.damping = true;
        if (!have_masses) return QM_OK;
        double jump_mass = p * one_mass;
        double stay_mass = zero_mass + (1 - p) * one_mass;
        double total = jump_mass + stay_mass;
        if (!std::isfinite(total) || total <= 0)
            return fail(QM_E_MASS, "The state has no finite positive probability mass.");
        b.jump = jump_mass > 0 && (stay_mass == 0 || draw() < jump_mass / total);
        double branch = b.jump ? jump_mass : stay_mass;
        b.scale = 1 / std::sqrt(branch);
        b.jump_scale = std::sqrt(p) * b.scale;
        b.stay_scale = std::sqrt(1 - p) * b.scale;
        return QM_OK;
    }
    if (kind == 2) {
        double u = draw();
        double quarter = p / 4;
        b.pauli = u < quarter ? 1 : u < 2 * quarter ? 2 : u < 3 * quarter ? 3 : 0;
    } else {
        bool apply = p == 1 || draw() < p;
        b.pauli = !apply ? 0 : kind == 0 ? 1 : 3;
    }
    return QM_OK;
}

}  // namespace

extern "C" int32_t qm_noise_apply_host(qm_context* ctx, int32_t kind, double p, int32_t target, double* amps,
                                       int64_t length, qm_next_double_fn next_double, void* user,
                                       const volatile int32_t* cancel) {
    if (!ctx) return fail(QM_E_ARG, "context is null");
    if (!next_double) return fail(QM_E_ARG, "random source is null");
    if (kind < 0 || kind > 3) return fail(QM_E_RANGE, "unknown noise kind");
    if (!std::isfinite(p) || p < 0 || p > 1) return fail(QM_E_RANGE, "Channel probability must be finite and in [0,1].");
    if (!amps || length < 2 || (length & (length - 1)) != 0 || length > (int64_t(1) << 30))
        return fail(QM_E_ARG, "State length must be a power of two, at least two.");
    int qubits = 63 - __builtin_clzll((unsigned long long)length);
    if ((uint32_t)target >= (uint32_t)qubits) return fail(QM_E_RANGE, "target out of range");
    if (cancelled(cancel)) return fail(QM_E_CANCELLED, "operation cancelled");
    if (p == 0) return QM_OK;
    auto draw = [&]() { return next_double(user); };
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    if (ctx->disposed) return fail(QM_E_DISPOSED, "context disposed");
    QM_CUDA(cudaSetDevice(ctx->device));
    Branch b;
    if (kind != 3) {
        int32_t rc = choose_branch(kind, p, draw, false, 0, 0, b);
        if (rc) return rc;
        if (cancelled(cancel)) return fail(QM_E_CANCELLED, "operation cancelled");
        if (b.pauli == 0) return QM_OK;
    }
    const int64_t bytes = 16 * length;
    if (bytes > ctx->device_budget || bytes > ctx->staging_budget)
        return fail(QM_E_BUDGET, "CUDA state exceeds the device or host staging memory budget.");
    void* dev = nullptr;
    int32_t rc = device_buffer(ctx, (size_t)bytes, &dev);
    if (rc) return rc;
    QM_CUDA(host_to_device(ctx, dev, amps, (size_t)bytes));
    if (kind == 3) {
        double m0 = 0, m1 = 0;
        rc = device_masses(ctx, dev, qubits, QM_FP64, target, &m0, &m1);
        if (rc) return rc;
        rc = choose_branch(kind, p, draw, true, m0, m1, b);
        if (rc) return rc;
        if (cancelled(cancel)) return fail(QM_E_CANCELLED, "operation cancelled");
        QM_CUDA(launch_damping(dev, qubits, QM_FP64, target, b.jump ? 1 : 0, b.scale, b.jump_scale, b.stay_scale,
                               ctx->stream));
    } else {
        QM_CUDA(launch_pauli(dev, qubits, QM_FP64, target, b.pauli, ctx->stream));
    }
    QM_CUDA(cudaStreamSynchronize(ctx->stream));
    QM_CUDA(device_to_host(ctx, amps, dev, (size_t)bytes));
    QM_CUDA(cudaStreamSynchronize(ctx->stream));
    return QM_OK;
}

// ====================================================================== device states

extern "C" int32_t qm_state_create(qm_context* ctx, int32_t qubits, int32_t precision, qm_state** out) {
    if (!ctx || !out) return fail(QM_E_ARG, "null argument");
    *out = nullptr;
    if (qubits < 1 || qubits > 30) return fail(QM_E_RANGE, "qubits must be between 1 and 30");
    if (precision != QM_FP64 && precision != QM_FP32) return fail(QM_E_RANGE, "unknown precision");
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    if (ctx->disposed) return fail(QM_E_DISPOSED, "context disposed");
    int64_t bytes = (precision == QM_FP32 ? 8ll : 16ll) << qubits;
    if (ctx->device_in_use + bytes > ctx->device_budget)
        return fail(QM_E_BUDGET, "state exceeds the context's device memory budget");
    QM_CUDA(cudaSetDevice(ctx->device));
    std::unique_ptr<qm_state> st(new qm_state());
    st->ctx = ctx;
    st->qubits = qubits;
    st->precision = precision;
    st->bytes = bytes;
    QM_CUDA(cudaMalloc(&st->amps, (size_t)bytes));
    cudaError_t e = launch_reset(st->amps, qubits, precision, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
        cudaFree(st->amps);
        return cuda_fail(e, "qm_state_create");
    }
    ctx->device_in_use += bytes;
    *out = st.release();
    return QM_OK;
}

extern "C" int32_t qm_state_destroy(qm_state* st) {
    if (!st) return QM_OK;
    qm_context* ctx = st->ctx;
    if (ctx) {
        std::lock_guard<std::recursive_mutex> lock(ctx->mu);
        cudaSetDevice(ctx->device);
        cudaStreamSynchronize(ctx->stream);
        cudaFree(st->amps);
        ctx->device_in_use -= st->bytes;
    }
    delete st;
    return QM_OK;
}

extern "C" int32_t qm_state_reset(qm_state* st) {
    int32_t rc = check_state(st);
    if (rc) return rc;
    std::lock_guard<std::recursive_mutex> lock(st->ctx->mu);
    QM_CUDA(cudaSetDevice(st->ctx->device));
    QM_CUDA(launch_reset(st->amps, st->qubits, st->precision, st->ctx->stream));
    QM_CUDA(cudaStreamSynchronize(st->ctx->stream));
    return QM_OK;
}

extern "C" int32_t qm_state_device_pointer(qm_state* st, void** ptr) {
    int32_t rc = check_state(st);
    if (rc) return rc;
    if (!ptr) return fail(QM_E_ARG, "pointer is null");
    *ptr = st->amps;
    return QM_OK;
}

extern "C" int32_t qm_state_upload(qm_state* st, const double* amps, int64_t length) {
    int32_t rc = check_state(st);
    if (rc) return rc;
    if (!amps || length != (int64_t(1) << st->qubits)) return fail(QM_E_ARG, "Buffer length must equal 2^qubitCount.");
    qm_context* ctx = st->ctx;
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    QM_CUDA(cudaSetDevice(ctx->device));
    if (st->precision == QM_FP64) {
        QM_CUDA(host_to_device(ctx, st->amps, amps, (size_t)(16 * length)));
    } else {
        const int64_t chunk = int64_t(1) << 21;  // amplitudes per staging chunk (32 MiB FP64)
        rc = ensure_scratch(ctx, (size_t)(16 * std::min(chunk, length)));
        if (rc) return rc;
        for (int64_t off = 0; off < length; off += chunk) {
            int64_t cnt = std::min(chunk, length - off);
            QM_CUDA(cudaMemcpyAsync(ctx->scratch, amps + 2 * off, (size_t)(16 * cnt), cudaMemcpyHostToDevice, ctx->stream));
            QM_CUDA(launch_convert_from_f64(static_cast<float*>(st->amps) + 2 * off, static_cast<double*>(ctx->scratch),
                                            cnt, ctx->stream));
        }
    }
    QM_CUDA(cudaStreamSynchronize(ctx->stream));
    return QM_OK;
}

extern "C" int32_t qm_state_download(qm_state* st, double* amps, int64_t length) {
    int32_t rc = check_state(st);
    if (rc) return rc;
    if (!amps || length != (int64_t(1) << st->qubits)) return fail(QM_E_ARG, "Buffer length must equal 2^qubitCount.");
    qm_context* ctx = st->ctx;
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    QM_CUDA(cudaSetDevice(ctx->device));
    if (st->precision == QM_FP64) {
        QM_CUDA(device_to_host(ctx, amps, st->amps, (size_t)(16 * length)));
    } else {
        const int64_t chunk = int64_t(1) << 21;
        rc = ensure_scratch(ctx, (size_t)(16 * std::min(chunk, length)));
        if (rc) return rc;
        for (int64_t off = 0; off < length; off += chunk) {
            int64_t cnt = std::min(chunk, length - off);
            QM_CUDA(launch_convert_to_f64(static_cast<double*>(ctx->scratch), static_cast<float*>(st->amps) + 2 * off, cnt,
                                          ctx->stream));
            QM_CUDA(cudaMemcpyAsync(amps + 2 * off, ctx->scratch, (size_t)(16 * cnt), cudaMemcpyDeviceToHost, ctx->stream));
            QM_CUDA(cudaStreamSynchronize(ctx->stream));
        }
    }
    QM_CUDA(cudaStreamSynchronize(ctx->stream));
    return QM_OK;
}

// ====================================================================== execution

extern "C" int32_t qm_plan_create(qm_context* ctx, int32_t qubits, int32_t precision, const qm_gate* gates,
                                  int32_t count, int32_t width, qm_plan** out) {
    if (!ctx || !out) return fail(QM_E_ARG, "null argument");
    *out = nullptr;
    if (qubits < 1 || qubits > 30) return fail(QM_E_RANGE, "qubits must be between 1 and 30");
    if (precision != QM_FP64 && precision != QM_FP32) return fail(QM_E_RANGE, "unknown precision");
    if (!valid_width(width)) return fail(QM_E_RANGE, kWidthRule);
    int32_t rc = validate_gates(gates, count, qubits);
    if (rc) return rc;
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    if (ctx->disposed) return fail(QM_E_DISPOSED, "context disposed");
    QM_CUDA(cudaSetDevice(ctx->device));
    std::unique_ptr<qm_plan> p(new qm_plan());
    p->ctx = ctx;
    rc = build_plan(ctx, qubits, precision, gates, count, width, p->plan);
    if (rc) { free_plan(p->plan); return rc; }
    jit_prepare(p->plan);  // a plan is made to be run again: compile its passes once
    QM_CUDA(cudaStreamSynchronize(ctx->stream));
    *out = p.release();
    return QM_OK;
}

extern "C" int32_t qm_plan_destroy(qm_plan* p) {
    if (!p) return QM_OK;
    if (p->ctx) {
        std::lock_guard<std::recursive_mutex> lock(p->ctx->mu);
        cudaSetDevice(p->ctx->device);
        cudaStreamSynchronize(p->ctx->stream);
        free_plan(p->plan);
    }
    delete p;
    return QM_OK;
}

extern "C" int32_t qm_plan_stats(const qm_plan* p, int32_t* passes, int32_t* launches, int64_t* bytes) {
    if (!p) return fail(QM_E_ARG, "plan is null");
    if (passes) *passes = (int32_t)p->plan.passes.size();
    if (launches) *launches = p->plan.launches;
    if (bytes) *bytes = p->plan.planned_bytes;
    return QM_OK;
}

static_assert(sizeof(qm_fused_op_info) == sizeof(FusedOp), "qm_fused_op_info mirrors FusedOp");
static_assert(sizeof(qm_fused_pass_info) == sizeof(FusedPass), "qm_fused_pass_info mirrors FusedPass");
static_assert(sizeof(qm_gate) == 80 && sizeof(qm_operation) == 88 && sizeof(qm_pauli_term) == 24, "ABI sizes");

extern "C" int32_t qm_plan_program(int32_t qubits, int32_t precision, const qm_gate* gates, int32_t count,
                                   int32_t width, int32_t* passes, qm_fused_pass_info* pass_records,
                                   int32_t max_passes, int32_t* ops, qm_fused_op_info* op_records, int32_t max_ops,
                                   int64_t* planned_bytes) {
    if (qubits < 1 || qubits > 30) return fail(QM_E_RANGE, "qubits must be between 1 and 30");
    if (precision != QM_FP64 && precision != QM_FP32) return fail(QM_E_RANGE, "unknown precision");
    if (!valid_width(width)) return fail(QM_E_RANGE, kWidthRule);
    int32_t rc = validate_gates(gates, count, qubits);
    if (rc) return rc;
    Plan plan;
    std::string err;
    std::vector<qm_gate> list(gates, gates + count);
    if (!plan_fused(list, qubits, precision, width, plan, err)) return fail(QM_E_ARG, "planner: " + err);
    if (passes) *passes = (int32_t)plan.passes.size();
    if (ops) *ops = (int32_t)plan.ops.size();
    if (planned_bytes) *planned_bytes = plan.planned_bytes;
    if (pass_records && max_passes >= (int32_t)plan.passes.size())
        std::memcpy(pass_records, plan.passes.data(), plan.passes.size() * sizeof(FusedPass));
    if (op_records && max_ops >= (int32_t)plan.ops.size())
        std::memcpy(op_records, plan.ops.data(), plan.ops.size() * sizeof(FusedOp));
    return QM_OK;
}

namespace {

int32_t execute_plan(qm_state* st, const Plan& plan, qm_profile* profile) {
    qm_context* ctx = st->ctx;
    QM_CUDA(cudaSetDevice(ctx->device));
    if (profile) QM_CUDA(cudaEventRecord(ctx->ev_start, ctx->stream));
    int32_t rc = run_plan(ctx, plan, st->amps, nullptr);
    if (rc) {
        cudaStreamSynchronize(ctx->stream);
        return rc;
    }
    if (profile) QM_CUDA(cudaEventRecord(ctx->ev_stop, ctx->stream));
    QM_CUDA(cudaStreamSynchronize(ctx->stream));
    rc = dense_status(plan);
    if (rc) return rc;
    if (profile) {
        std::memset(profile, 0, sizeof *profile);
        profile->device_seconds = seconds_between(ctx->ev_start, ctx->ev_stop);
        profile->state_bytes = st->bytes;
        profile->kernel_launches = plan.launches;
        profile->passes = (int32_t)plan.passes.size();
        profile->planned_bytes = plan.planned_bytes;
    }
    return QM_OK;
}

}  // namespace

extern "C" int32_t qm_plan_execute(qm_plan* p, qm_state* st, qm_profile* profile) {
    if (!p) return fail(QM_E_ARG, "plan is null");
    int32_t rc = check_state(st);
    if (rc) return rc;
    if (p->ctx != st->ctx) return fail(QM_E_ARG, "plan and state belong to different contexts");
    if (p->plan.qubits != st->qubits || p->plan.precision != st->precision)
        return fail(QM_E_ARG, "plan and state sizes must match");
    std::lock_guard<std::recursive_mutex> lock(st->ctx->mu);
    return execute_plan(st, p->plan, profile);
}

// ====================================================================== autotuning

namespace {

// Fusion widths chosen by qm_plan_autotune, per (qubits, precision, gate structure): the
// structure is every gate's kernel, target, controls and swap operand, not its coefficients, so
// circuits that differ only in angles share a choice.
std::mutex g_tune_mutex;
std::map<std::vector<int64_t>, int32_t> g_tune_cache;

std::vector<int64_t> structure_key(int32_t qubits, int32_t precision, const qm_gate* gates, int32_t count) {
    std::vector<int64_t> key;
    key.reserve(2 + (size_t)count);
    key.push_back(qubits);
    key.push_back(precision);
    for (int32_t i = 0; i < count; ++i) {
        const qm_gate& g = gates[i];
        key.push_back(((int64_t)g.kernel << 56) | ((int64_t)(g.target & 0xff) << 48) |
                      ((int64_t)((g.swap_control + 1) & 0xff) << 40) | (int64_t)g.control_mask);
    }
    return key;
}

}  // namespace

extern "C" int32_t qm_plan_autotune(qm_context* ctx, int32_t qubits, int32_t precision, const qm_gate* gates,
                                    int32_t count, const int32_t* candidates, int32_t candidate_count, qm_plan** out,
                                    int32_t* chosen) {
    if (!ctx || !out) return fail(QM_E_ARG, "null argument");
    *out = nullptr;
    if (qubits < 1 || qubits > 30) return fail(QM_E_RANGE, "qubits must be between 1 and 30");
    if (precision != QM_FP64 && precision != QM_FP32) return fail(QM_E_RANGE, "unknown precision");
    if (candidate_count < 0 || (candidate_count > 0 && !candidates)) return fail(QM_E_ARG, "candidates");
    int32_t rc = validate_gates(gates, count, qubits);
    if (rc) return rc;
    std::vector<int32_t> widths(candidates, candidates + candidate_count);
    if (widths.empty()) {
        widths = {10, 11, 12};
        if (precision == QM_FP32) widths.insert(widths.end(), {13, 5, 6});
    }
    for (int32_t w : widths)
        if (w == 0 || !valid_width(w)) return fail(QM_E_RANGE, kWidthRule);
    const std::vector<int64_t> key = structure_key(qubits, precision, gates, count);
    int32_t best = 0;
    {
        std::lock_guard<std::mutex> lock(g_tune_mutex);
        auto it = g_tune_cache.find(key);
        if (it != g_tune_cache.end()) best = it->second;
    }
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    if (ctx->disposed) return fail(QM_E_DISPOSED, "context disposed");
    QM_CUDA(cudaSetDevice(ctx->device));
    if (best == 0 && widths.size() == 1) best = widths[0];
    if (best == 0) {
        // time one execution of each candidate (after one untimed, which compiles and loads its
        // kernels) on a scratch state; the scratch is freed before the chosen plan is built
        const size_t bytes = (size_t)(precision == QM_FP32 ? 8 : 16) << qubits;
        if ((int64_t)bytes + ctx->device_in_use > ctx->device_budget)
            return fail(QM_E_BUDGET, "autotuning needs a scratch state within the device budget");
        void* scratch = nullptr;
        QM_CUDA(cudaMalloc(&scratch, bytes));
        double best_s = 0;
        for (int32_t w : widths) {
            Plan plan;
            rc = build_plan(ctx, qubits, precision, gates, count, w, plan);
            if (rc == QM_OK) {
                jit_prepare(plan);
                launch_reset(scratch, qubits, precision, ctx->stream);
                rc = run_plan(ctx, plan, scratch, nullptr);
            }
            if (rc == QM_OK) {
                cudaEventRecord(ctx->ev_start, ctx->stream);
                rc = run_plan(ctx, plan, scratch, nullptr);
                cudaEventRecord(ctx->ev_stop, ctx->stream);
            }
            const cudaError_t e = cudaStreamSynchronize(ctx->stream);
            if (rc == QM_OK && e == cudaSuccess) rc = dense_status(plan);
            free_plan(plan);
            if (e != cudaSuccess) {
                cudaFree(scratch);
                return cuda_fail(e, "qm_plan_autotune");
            }
            if (rc) continue;  // a candidate this circuit cannot use (e.g. a batch-only width)
            const double sec = seconds_between(ctx->ev_start, ctx->ev_stop);
            if (best == 0 || sec < best_s) {
                best = w;
                best_s = sec;
            }
        }
        cudaFree(scratch);
        if (best == 0) return fail(QM_E_ARG, "no candidate fusion width plans this circuit");
        std::lock_guard<std::mutex> tl(g_tune_mutex);
        g_tune_cache[key] = best;
    }
    rc = qm_plan_create(ctx, qubits, precision, gates, count, best, out);
    if (rc == QM_OK && chosen) *chosen = best;
    return rc;
}

// ====================================================================== captured executions

struct qm_graph {
    qm_context* ctx = nullptr;
    qm_plan* plan = nullptr;
    qm_state* state = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

extern "C" int32_t qm_graph_create(qm_plan* p, qm_state* st, qm_graph** out) {
    if (!p || !st || !out) return fail(QM_E_ARG, "null argument");
    *out = nullptr;
    if (p->ctx != st->ctx) return fail(QM_E_ARG, "plan and state belong to different contexts");
    if (p->plan.qubits != st->qubits || p->plan.precision != st->precision)
        return fail(QM_E_ARG, "plan and state sizes must match");
    qm_context* ctx = st->ctx;
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    if (ctx->disposed) return fail(QM_E_DISPOSED, "context disposed");
    QM_CUDA(cudaSetDevice(ctx->device));
    // The capture records the plan's launches only (nothing runs); kernel attributes and compiled
    // passes are set up by the plan's first execution, which the caller makes before capturing.
    QM_CUDA(cudaStreamSynchronize(ctx->stream));
    std::unique_ptr<qm_graph> g(new qm_graph());
    g->ctx = ctx;
    g->plan = p;
    g->state = st;
    QM_CUDA(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    int32_t rc = run_plan(ctx, p->plan, st->amps, nullptr);
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(ctx->stream, &graph);
    if (rc) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
    }
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
    g->graph = graph;
    const cudaError_t ie = cudaGraphInstantiate(&g->exec, graph, 0);
    if (ie != cudaSuccess) {
        cudaGraphDestroy(graph);
        return cuda_fail(ie, "cudaGraphInstantiate");
    }
    *out = g.release();
    return QM_OK;
}

extern "C" int32_t qm_graph_launch(qm_graph* g, qm_profile* profile) {
    if (!g) return fail(QM_E_ARG, "graph is null");
    qm_context* ctx = g->ctx;
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    if (ctx->disposed) return fail(QM_E_DISPOSED, "context disposed");
    QM_CUDA(cudaSetDevice(ctx->device));
    if (profile) QM_CUDA(cudaEventRecord(ctx->ev_start, ctx->stream));
    QM_CUDA(cudaGraphLaunch(g->exec, ctx->stream));
    if (profile) QM_CUDA(cudaEventRecord(ctx->ev_stop, ctx->stream));
    QM_CUDA(cudaStreamSynchronize(ctx->stream));
    int32_t rc = dense_status(g->plan->plan);
    if (rc) return rc;
    if (profile) {
        std::memset(profile, 0, sizeof *profile);
        profile->device_seconds = seconds_between(ctx->ev_start, ctx->ev_stop);
        profile->state_bytes = g->state->bytes;
        profile->kernel_launches = g->plan->plan.launches;
        profile->passes = (int32_t)g->plan->plan.passes.size();
        profile->planned_bytes = g->plan->plan.planned_bytes;
    }
    return QM_OK;
}

extern "C" int32_t qm_graph_destroy(qm_graph* g) {
    if (!g) return QM_OK;
    if (g->ctx) {
        std::lock_guard<std::recursive_mutex> lock(g->ctx->mu);
        cudaSetDevice(g->ctx->device);
        cudaStreamSynchronize(g->ctx->stream);
    }
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->graph) cudaGraphDestroy(g->graph);
    delete g;
    return QM_OK;
}

extern "C" int32_t qm_execute(qm_state* st, const qm_gate* gates, int32_t count, int32_t width, qm_profile* profile) {
    int32_t rc = check_state(st);
    if (rc) return rc;
    if (!valid_width(width)) return fail(QM_E_RANGE, kWidthRule);
    rc = validate_gates(gates, count, st->qubits);
    if (rc) return rc;
    std::lock_guard<std::recursive_mutex> lock(st->ctx->mu);
    QM_CUDA(cudaSetDevice(st->ctx->device));
    Plan plan;
    rc = build_plan(st->ctx, st->qubits, st->precision, gates, count, width, plan, true);
    if (rc == QM_OK) rc = execute_plan(st, plan, profile);
    cudaStreamSynchronize(st->ctx->stream);
    free_plan(plan);
    return rc;
}

// ====================================================================== noise primitives

extern "C" int32_t qm_qubit_masses(qm_state* st, int32_t target, double* m0, double* m1) {
    int32_t rc = check_state(st);
    if (rc) return rc;
    if (!m0 || !m1) return fail(QM_E_ARG, "null output");
    if ((uint32_t)target >= (uint32_t)st->qubits) return fail(QM_E_RANGE, "target out of range");
    std::lock_guard<std::recursive_mutex> lock(st->ctx->mu);
    QM_CUDA(cudaSetDevice(st->ctx->device));
    return device_masses(st->ctx, st->amps, st->qubits, st->precision, target, m0, m1);
}

extern "C" int32_t qm_apply_pauli(qm_state* st, int32_t target, int32_t pauli) {
    int32_t rc = check_state(st);
    if (rc) return rc;
    if ((uint32_t)target >= (uint32_t)st->qubits) return fail(QM_E_RANGE, "target out of range");
    if (pauli < 0 || pauli > 3) return fail(QM_E_RANGE, "pauli must be 0..3");
    if (pauli == 0) return QM_OK;
    std::lock_guard<std::recursive_mutex> lock(st->ctx->mu);
    QM_CUDA(cudaSetDevice(st->ctx->device));
    QM_CUDA(launch_pauli(st->amps, st->qubits, st->precision, target, pauli, st->ctx->stream));
    QM_CUDA(cudaStreamSynchronize(st->ctx->stream));
    return QM_OK;
}

extern "C" int32_t qm_apply_damping(qm_state* st, int32_t target, int32_t jump, double scale, double jump_scale,
                                    double stay_scale) {
    int32_t rc = check_state(st);
    if (rc) return rc;
    if ((uint32_t)target >= (uint32_t)st->qubits) return fail(QM_E_RANGE, "target out of range");
    if (!std::isfinite(scale) || !std::isfinite(jump_scale) || !std::isfinite(stay_scale))
        return fail(QM_E_RANGE, "scales must be finite");
    std::lock_guard<std::recursive_mutex> lock(st->ctx->mu);
    QM_CUDA(cudaSetDevice(st->ctx->device));
    QM_CUDA(launch_damping(st->amps, st->qubits, st->precision, target, jump ? 1 : 0, scale, jump_scale, stay_scale,
                           st->ctx->stream));
    QM_CUDA(cudaStreamSynchronize(st->ctx->stream));
    return QM_OK;
}

extern "C" int32_t qm_state_noise_apply(qm_state* st, int32_t kind, double p, int32_t target,
                                        qm_next_double_fn next_double, void* user) {
    int32_t rc = check_state(st);
    if (rc) return rc;
    if (!next_double) return fail(QM_E_ARG, "random source is null");
    if (kind < 0 || kind > 3) return fail(QM_E_RANGE, "unknown noise kind");
    if (!std::isfinite(p) || p < 0 || p > 1) return fail(QM_E_RANGE, "Channel probability must be finite and in [0,1].");
    if ((uint32_t)target >= (uint32_t)st->qubits) return fail(QM_E_RANGE, "target out of range");
    if (p == 0) return QM_OK;
    auto draw = [&]() { return next_double(user); };
    std::lock_guard<std::recursive_mutex> lock(st->ctx->mu);
    QM_CUDA(cudaSetDevice(st->ctx->device));
    Branch b;
    if (kind != 3) {
        rc = choose_branch(kind, p, draw, false, 0, 0, b);
        if (rc) return rc;
        if (b.pauli == 0) return QM_OK;
        QM_CUDA(launch_pauli(st->amps, st->qubits, st->precision, target, b.pauli, st->ctx->stream));
    } else {
        double m0 = 0, m1 = 0;
        rc = device_masses(st->ctx, st->amps, st->qubits, st->precision, target, &m0, &m1);
        if (rc) return rc;
        rc = choose_branch(kind, p, draw, true, m0, m1, b);
        if (rc) return rc;
        QM_CUDA(launch_damping(st->amps, st->qubits, st->precision, target, b.jump ? 1 : 0, b.scale, b.jump_scale,
                               b.stay_scale, st->ctx->stream));
    }
    QM_CUDA(cudaStreamSynchronize(st->ctx->stream));
    return QM_OK;
}

// ====================================================================== observables

namespace {

int32_t validate_terms(const qm_pauli_term* terms, int32_t count, int qubits) {
    if (count < 0) return fail(QM_E_RANGE, "term count must be nonnegative");
    if (count > 0 && !terms) return fail(QM_E_ARG, "terms is null");
    uint32_t all = (uint32_t)((1ull << qubits) - 1);
    for (int32_t i = 0; i < count; ++i) {
        if ((terms[i].flip_mask | terms[i].sign_mask) & ~all)
            return fail(QM_E_ARG, "Observable and state sizes must match.");
        if (!std::isfinite(terms[i].coefficient)) return fail(QM_E_RANGE, "coefficient must be finite");
    }
    return QM_OK;
}

// Raw term sums and mass into host arrays (raw[count], *mass).  States of 9 or more qubits use
// the tiled kernel (a few reads of the state for the whole term list); smaller ones run one
// pass per distinct flip mask.
int32_t device_expectation(qm_state* st, const qm_pauli_term* terms, int32_t count, double* raw, double* mass) {
    qm_context* ctx = st->ctx;
    TilePlan tp;
    std::string err;
    if (st->qubits >= 9 && plan_tiles(st->qubits, st->precision, terms, count, tp, err)) {
        const size_t cells = (size_t)tp.rows_per_state * tp.columns;
        int32_t rc = ensure_scratch(ctx, sizeof(double) * (cells + tp.columns));
        if (rc) return rc;
        rc = ensure_host_scratch(ctx, sizeof(double) * tp.columns);
        if (rc) return rc;
        double* partial = static_cast<double*>(ctx->scratch);
        double* out = partial + cells;
        QM_CUDA(cudaMemsetAsync(partial, 0, sizeof(double) * cells, ctx->stream));
        for (const TilePass& p : tp.passes)
            QM_CUDA(launch_expect_tile(st->amps, st->qubits, st->precision, p, tp.terms.data(), 1, 0, partial,
                                       tp.columns, tp.rows_per_state, tp.mass_column, ctx->stream));
        QM_CUDA(launch_finish_batched(partial, 1, tp.rows_per_state, tp.columns, out, ctx->stream));
        QM_CUDA(cudaMemcpyAsync(ctx->host_scratch, out, sizeof(double) * tp.columns, cudaMemcpyDeviceToHost,
                                ctx->stream));
        QM_CUDA(cudaStreamSynchronize(ctx->stream));
        for (int32_t i = 0; i < count; ++i) raw[i] = ctx->host_scratch[i];
        *mass = ctx->host_scratch[tp.mass_column];
        return QM_OK;
    }
    std::vector<DevPauli> dev((size_t)count);
    for (int32_t i = 0; i < count; ++i)
        dev[(size_t)i] = DevPauli{terms[i].flip_mask, terms[i].sign_mask, terms[i].y_count & 3, 0};
    const int columns = count + 1;
    const int max_blocks = 148 * 4;
    int32_t rc = ensure_scratch(ctx, sizeof(double) * ((size_t)max_blocks * columns + columns));
    if (rc) return rc;
    rc = ensure_host_scratch(ctx, sizeof(double) * columns);
    if (rc) return rc;
    double* partial = static_cast<double*>(ctx->scratch);
    int blocks = 0;
    QM_CUDA(launch_expectation(st->amps, st->qubits, st->precision, dev.data(), count, partial, &blocks, ctx->stream));
    double* out = partial + (size_t)blocks * columns;
    QM_CUDA(launch_finish_sums(partial, blocks, columns, out, ctx->stream));
    QM_CUDA(cudaMemcpyAsync(ctx->host_scratch, out, sizeof(double) * columns, cudaMemcpyDeviceToHost, ctx->stream));
    QM_CUDA(cudaStreamSynchronize(ctx->stream));
    for (int32_t i = 0; i < count; ++i) raw[i] = ctx->host_scratch[i];
    *mass = ctx->host_scratch[count];
    return QM_OK;
}

}  // namespace

extern "C" int32_t qm_expectation_pauli(qm_state* st, const qm_pauli_term* terms, int32_t count, double* per_term,
                                        double* mass) {
    int32_t rc = check_state(st);
    if (rc) return rc;
    rc = validate_terms(terms, count, st->qubits);
    if (rc) return rc;
    if (count > 0 && !per_term) return fail(QM_E_ARG, "per_term is null");
    std::lock_guard<std::recursive_mutex> lock(st->ctx->mu);
    QM_CUDA(cudaSetDevice(st->ctx->device));
    std::vector<double> raw((size_t)count);
    double total = 0;
    rc = device_expectation(st, terms, count, raw.data(), &total);
    if (rc) return rc;
    if (mass) *mass = total;
    if (!std::isfinite(total) || total <= 0) return fail(QM_E_MASS, "The state has no finite positive probability mass.");
    for (int32_t i = 0; i < count; ++i) {
        if (!std::isfinite(raw[(size_t)i])) return fail(QM_E_MASS, "The observable accumulation is nonfinite.");
        per_term[i] = raw[(size_t)i] / total;
    }
    return QM_OK;
}

extern "C" int32_t qm_expectation_energy(qm_state* st, const qm_pauli_term* terms, int32_t count, double* energy) {
    int32_t rc = check_state(st);
    if (rc) return rc;
    if (!energy) return fail(QM_E_ARG, "energy is null");
    rc = validate_terms(terms, count, st->qubits);
    if (rc) return rc;
    // only nonzero coefficients contribute (StateVector.Energy.cs:27)
    std::vector<qm_pauli_term> used;
    for (int32_t i = 0; i < count; ++i)
        if (terms[i].coefficient != 0) used.push_back(terms[i]);
    std::lock_guard<std::recursive_mutex> lock(st->ctx->mu);
    QM_CUDA(cudaSetDevice(st->ctx->device));
    std::vector<double> raw(used.size());
    double total = 0;
    rc = device_expectation(st, used.data(), (int32_t)used.size(), raw.data(), &total);
    if (rc) return rc;
    if (!std::isfinite(total) || total <= 0) return fail(QM_E_MASS, "The state has no finite positive probability mass.");
    double sum = 0, correction = 0;
    for (size_t i = 0; i < used.size(); ++i) {
        if (!std::isfinite(raw[i])) return fail(QM_E_MASS, "The observable accumulation is nonfinite.");
        double value = used[i].coefficient * (raw[i] / total);
        double next = sum + value;
        correction += std::fabs(sum) >= std::fabs(value) ? (sum - next) + value : (value - next) + sum;
        sum = next;
        if (!std::isfinite(sum) || !std::isfinite(correction))
            return fail(QM_E_MASS, "The energy accumulation is nonfinite.");
    }
    double e = sum + correction;
    if (!std::isfinite(e)) return fail(QM_E_MASS, "The energy is nonfinite.");
    *energy = e;
    return QM_OK;
}

// ====================================================================== sampling

namespace {

// Targets draw*total on the FP64 chunk prefix, then device searches.  outcomes[i] = index;
// returns the number of draws near a boundary in *ambiguous.
int32_t device_sample(qm_state* st, const double* draws, int32_t shots, int64_t* outcomes, int32_t* ambiguous) {
    qm_context* ctx = st->ctx;
    const uint64_t n = 1ull << st->qubits;
    uint64_t chunk = std::max<uint64_t>(1024, n / (148 * 8));
    uint64_t c = 1;
    while (c < chunk) c <<= 1;
    if (c > n) c = n;
    const int blocks = (int)(n / c);
    size_t need = sizeof(double) * (size_t)blocks           // sums
                  + sizeof(int64_t) * (size_t)blocks        // last
                  + sizeof(double) * ((size_t)blocks + 1)   // prefix
                  + sizeof(double) * (size_t)shots          // targets
                  + sizeof(int64_t) * 2 * (size_t)shots;    // outcomes + flags
    int32_t rc = ensure_scratch(ctx, need);
    if (rc) return rc;
    rc = ensure_host_scratch(ctx, std::max(sizeof(double) * (size_t)blocks * 2, sizeof(int64_t) * 2 * (size_t)shots) + 64);
    if (rc) return rc;
    char* base = static_cast<char*>(ctx->scratch);
    double* sums = reinterpret_cast<double*>(base);
    int64_t* last = reinterpret_cast<int64_t*>(sums + blocks);
    double* prefix = reinterpret_cast<double*>(last + blocks);
    double* targets = prefix + blocks + 1;
    int64_t* out = reinterpret_cast<int64_t*>(targets + shots);
    int blocks_out = 0, chunk_out = 0;
    QM_CUDA(launch_block_probs(st->amps, st->qubits, st->precision, sums, last, &blocks_out, &chunk_out, ctx->stream));
    if (blocks_out != blocks || (uint64_t)chunk_out != c) return fail(QM_E_DEVICE, "sampling chunk mismatch");
    double* h = ctx->host_scratch;
    QM_CUDA(cudaMemcpyAsync(h, sums, sizeof(double) * blocks, cudaMemcpyDeviceToHost, ctx->stream));
    QM_CUDA(cudaMemcpyAsync(h + blocks, last, sizeof(int64_t) * blocks, cudaMemcpyDeviceToHost, ctx->stream));
    QM_CUDA(cudaStreamSynchronize(ctx->stream));
    std::vector<double> pre((size_t)blocks + 1);
    pre[0] = 0;
    int64_t last_supported = -1;
    const int64_t* hl = reinterpret_cast<const int64_t*>(h + blocks);
    for (int b = 0; b < blocks; ++b) {
        pre[(size_t)b + 1] = pre[(size_t)b] + h[b];
        last_supported = std::max(last_supported, hl[b]);
    }
    double total = pre[(size_t)blocks];
    if (!std::isfinite(total) || total <= 0) return fail(QM_E_MASS, "The state has no finite positive probability mass.");
    std::vector<double> tg((size_t)shots);
    for (int32_t s = 0; s < shots; ++s) tg[(size_t)s] = draws[s] * total;
    QM_CUDA(cudaMemcpyAsync(prefix, pre.data(), sizeof(double) * (blocks + 1), cudaMemcpyHostToDevice, ctx->stream));
    QM_CUDA(cudaMemcpyAsync(targets, tg.data(), sizeof(double) * shots, cudaMemcpyHostToDevice, ctx->stream));
    QM_CUDA(launch_search(st->amps, st->qubits, st->precision, prefix, blocks, (int)c, targets, shots, 1e-12 * total, out,
                          ctx->stream));
    int64_t* ho = reinterpret_cast<int64_t*>(h);
    QM_CUDA(cudaMemcpyAsync(ho, out, sizeof(int64_t) * 2 * shots, cudaMemcpyDeviceToHost, ctx->stream));
    QM_CUDA(cudaStreamSynchronize(ctx->stream));
    int32_t amb = 0;
    for (int32_t s = 0; s < shots; ++s) {
        outcomes[s] = ho[s] >= 0 ? ho[s] : last_supported;
        amb += ho[shots + s] ? 1 : 0;
    }
    if (ambiguous) *ambiguous = amb;
    return QM_OK;
}

}  // namespace

int32_t qm_sample_amplitudes(qm_context* ctx, void* amps, int32_t qubits, int32_t precision, const double* draws,
                             int32_t shots, int64_t* outcomes, int32_t* ambiguous) {
    qm_state view;
    view.ctx = ctx;
    view.qubits = qubits;
    view.precision = precision;
    view.amps = amps;
    view.bytes = (precision == QM_FP32 ? 8ll : 16ll) << qubits;
    return device_sample(&view, draws, shots, outcomes, ambiguous);
}

extern "C" int32_t qm_sample(qm_state* st, const double* draws, int32_t shots, int64_t* outcomes, int32_t* ambiguous) {
    int32_t rc = check_state(st);
    if (rc) return rc;
    if (shots < 1) return fail(QM_E_RANGE, "shots must be positive");
    if (!draws || !outcomes) return fail(QM_E_ARG, "null argument");
    for (int32_t s = 0; s < shots; ++s)
        if (!std::isfinite(draws[s]) || draws[s] < 0 || draws[s] >= 1) return fail(QM_E_RANGE, "draws must be in [0,1)");
    std::lock_guard<std::recursive_mutex> lock(st->ctx->mu);
    QM_CUDA(cudaSetDevice(st->ctx->device));
    return device_sample(st, draws, shots, outcomes, ambiguous);
}

namespace {

// StateVector.ValidateSelection (StateVector.Observations.cs:143-168): the mask of the selection.
int32_t selection_mask(const int32_t* qubits, int32_t count, int32_t register_qubits, uint64_t* mask) {
    if (!qubits || count < 1 || count > register_qubits)
        return fail(QM_E_ARG, "Select between one and QubitCount distinct qubits.");
    uint64_t m = 0;
    for (int32_t k = 0; k < count; ++k) {
        if ((uint32_t)qubits[k] >= (uint32_t)register_qubits) return fail(QM_E_RANGE, "Selected qubits must be in range.");
        const uint64_t bit = 1ull << qubits[k];
        if (m & bit) return fail(QM_E_ARG, "Selected qubits must be distinct.");
        m |= bit;
    }
    *mask = m;
    return QM_OK;
}

// (selected, total) Born masses on the device, FP64 compensated.
int32_t pattern_masses(qm_state* st, uint64_t mask, uint64_t pattern, double* selected, double* total) {
    qm_context* ctx = st->ctx;
    int32_t rc = ensure_scratch(ctx, sizeof(double) * (4 * 148 * 4 + 8));
    if (rc) return rc;
    rc = ensure_host_scratch(ctx, 4 * sizeof(double));
    if (rc) return rc;
    double* partial = static_cast<double*>(ctx->scratch);
    int blocks = 0;
    QM_CUDA(launch_pattern_masses(st->amps, st->qubits, st->precision, mask, pattern, partial, &blocks, ctx->stream));
    double* out = partial + 4 * blocks;
    QM_CUDA(launch_finish_sums(partial, blocks, 4, out, ctx->stream));
    QM_CUDA(cudaMemcpyAsync(ctx->host_scratch, out, 4 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    QM_CUDA(cudaStreamSynchronize(ctx->stream));
    *selected = ctx->host_scratch[0] + ctx->host_scratch[1];
    *total = ctx->host_scratch[2] + ctx->host_scratch[3];
    return QM_OK;
}

}  // namespace

extern "C" int32_t qm_marginal_probability(qm_state* st, const int32_t* qubits, int32_t count, int32_t outcome,
                                           double* probability) {
    int32_t rc = check_state(st);
    if (rc) return rc;
    if (!probability) return fail(QM_E_ARG, "probability is null");
    uint64_t mask = 0;
    if ((rc = selection_mask(qubits, count, st->qubits, &mask))) return rc;
    if (outcome < 0 || (count < 31 && outcome >= (1 << count))) return fail(QM_E_RANGE, "outcome out of range");
    uint64_t pattern = 0;
    for (int32_t k = 0; k < count; ++k) pattern |= (uint64_t)((outcome >> k) & 1) << qubits[k];
    std::lock_guard<std::recursive_mutex> lock(st->ctx->mu);
    QM_CUDA(cudaSetDevice(st->ctx->device));
    double selected = 0, total = 0;
    if ((rc = pattern_masses(st, mask, pattern, &selected, &total))) return rc;
    if (!std::isfinite(total) || total <= 0) return fail(QM_E_MASS, "The state has no finite positive probability mass.");
    *probability = selected / total;
    return QM_OK;
}

extern "C" int32_t qm_measure(qm_state* st, const int32_t* qubits, int32_t count, double u, int32_t* outcome,
                              int32_t* ambiguous) {
    int32_t rc = check_state(st);
    if (rc) return rc;
    if (!outcome) return fail(QM_E_ARG, "outcome is null");
    uint64_t mask = 0;
    if ((rc = selection_mask(qubits, count, st->qubits, &mask))) return rc;
    if (!std::isfinite(u) || u < 0 || u >= 1) return fail(QM_E_RANGE, "draw must be in [0,1)");
    std::lock_guard<std::recursive_mutex> lock(st->ctx->mu);
    QM_CUDA(cudaSetDevice(st->ctx->device));
    // one full-basis Born draw (the device CDF and search of qm_sample)
    int64_t basis = -1;
    int32_t amb = 0;
    if ((rc = device_sample(st, &u, 1, &basis, &amb))) return rc;
    const uint64_t pattern = (uint64_t)basis & mask;
    double branch = 0, total = 0;
    if ((rc = pattern_masses(st, mask, pattern, &branch, &total))) return rc;
    if (!std::isfinite(branch) || branch <= 0) return fail(QM_E_MASS, "The state has no finite positive probability mass.");
    QM_CUDA(launch_project(st->amps, st->qubits, st->precision, mask, pattern, std::sqrt(branch), st->ctx->stream));
    QM_CUDA(cudaStreamSynchronize(st->ctx->stream));
    int32_t out = 0;
    for (int32_t k = 0; k < count; ++k) out |= (int32_t)((basis >> qubits[k]) & 1) << k;
    *outcome = out;
    if (ambiguous) *ambiguous = amb;
    return QM_OK;
}

extern "C" int32_t qm_measure_all(qm_state* st, double u, int64_t* outcome, int32_t* ambiguous) {
    int32_t rc = check_state(st);
    if (rc) return rc;
    if (!outcome) return fail(QM_E_ARG, "outcome is null");
    if (!std::isfinite(u) || u < 0 || u >= 1) return fail(QM_E_RANGE, "draw must be in [0,1)");
    std::lock_guard<std::recursive_mutex> lock(st->ctx->mu);
    QM_CUDA(cudaSetDevice(st->ctx->device));
    int64_t out = -1;
    int32_t amb = 0;
    rc = device_sample(st, &u, 1, &out, &amb);
    if (rc) return rc;
    QM_CUDA(launch_collapse(st->amps, st->qubits, st->precision, out, st->ctx->stream));
    QM_CUDA(cudaStreamSynchronize(st->ctx->stream));
    *outcome = out;
    if (ambiguous) *ambiguous = amb;
    return QM_OK;
}
