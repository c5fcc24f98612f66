// qm_cpu_parallel.cpp -- TEST INFRASTRUCTURE: timed CPU baseline.
//
// C++ restatement of QuantumMatter's parallel/AVX-512 CPU backend, used only as the
// CPU baseline that bench.py times beside the CUDA library (and as a second CPU
// checker in tests).  It is not shipped and the product path never calls it.
//
// Restates (paths inside the olgerd007/QuantumMatter project):
//   src/QuantumMatter.Infrastructure/ParallelCpuStateVectorBackend.cs:31-334
//     bounded data parallelism with a join after every gate or gate block,
//     contiguous pair ranges per worker, optional gate blocking of up to 32
//     adjacent uncontrolled same-target gates over 512-pair tiles;
//   src/QuantumMatter.Infrastructure/Avx512StateVectorKernel.cs:15-107
//     four complex values per zmm, separate multiply and add (no FMA);
//   src/QuantumMatter.Infrastructure/AvxStateVectorKernel.cs:14-140
//     256-bit kernels, including the target-0 in-register form;
//   src/QuantumMatter.Infrastructure/SimdHadamardKernel.cs:14-65.
// The worker pool is a persistent std::thread pool: each gate is one fork/join, as
// Parallel.For is in the reference.
#include "qm_oracle.h"

#include <immintrin.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

extern "C" {
typedef struct qmp_options {
    int32_t workers;             // ParallelCpuOptions.MaxDegreeOfParallelism
    int32_t min_parallel_qubits; // ParallelCpuOptions.MinimumParallelQubits
    int32_t simd;                // EnableSimd
    int32_t avx512;              // EnableAvx512
    int32_t blocking;            // EnableGateBlocking
} qmp_options;
int qmp_execute(const qmp_options* opt, const qmo_operation* ops, int32_t count, int32_t qubits, double* amps);
int qmp_hardware_threads(void);
}

namespace {

// ------------------------------------------------------------------ pool
class Pool {
public:
    explicit Pool(int n) : n_(n) {
        for (int i = 1; i < n_; ++i) threads_.emplace_back([this, i] { loop(i); });
    }
    ~Pool() {
        {
            std::lock_guard<std::mutex> g(m_);
            stop_ = true;
            ++gen_;
        }
        cv_.notify_all();
        for (auto& t : threads_) t.join();
    }
    int size() const { return n_; }
    // Runs f(worker) for worker in [0, workers) and joins.
    void run(int workers, const std::function<void(int)>& f) {
        if (workers <= 1) { f(0); return; }
        {
            std::lock_guard<std::mutex> g(m_);
            job_ = &f;
            active_ = workers;
            pending_.store(workers - 1, std::memory_order_relaxed);
            ++gen_;
        }
        cv_.notify_all();
        f(0);
        while (pending_.load(std::memory_order_acquire) != 0) std::this_thread::yield();
    }

private:
    void loop(int id) {
        uint64_t seen = 0;
        for (;;) {
            const std::function<void(int)>* job;
            int active;
            {
                std::unique_lock<std::mutex> g(m_);
                cv_.wait(g, [&] { return gen_ != seen; });
                seen = gen_;
                if (stop_) return;
                job = job_;
                active = active_;
            }
            if (id < active) {
                (*job)(id);
                pending_.fetch_sub(1, std::memory_order_acq_rel);
            }
        }
    }
    int n_;
    std::vector<std::thread> threads_;
    std::mutex m_;
    std::condition_variable cv_;
    uint64_t gen_ = 0;
    bool stop_ = false;
    const std::function<void(int)>* job_ = nullptr;
    int active_ = 0;
    std::atomic<int> pending_{0};
};

Pool& pool_for(int workers) {
    static std::mutex m;
    static std::unique_ptr<Pool> p;
    std::lock_guard<std::mutex> g(m);
    if (!p || p->size() < workers) p.reset(new Pool(workers));
    return *p;
}

struct cpx { double re, im; };
inline cpx cmul(cpx l, cpx r) { return { l.re * r.re - l.im * r.im, l.im * r.re + l.re * r.im }; }
inline cpx cadd(cpx l, cpx r) { return { l.re + r.re, l.im + r.im }; }
inline bool is_one(const double* v) { return v[0] == 1.0 && v[1] == 0.0; }

// ------------------------------------------------------------------ AVX-512 (Avx512StateVectorKernel.cs)
struct Coef512 {
    __m512d re, im;
    bool real;
    explicit Coef512(const double* c) {
        re = _mm512_set1_pd(c[0]);
        // lanes alternate (-imag, +imag): permuted (im, re) * (-i, +i) gives the cross terms
        im = _mm512_setr_pd(-c[1], c[1], -c[1], c[1], -c[1], c[1], -c[1], c[1]);
        real = c[1] == 0;
    }
    inline __m512d mul(__m512d v) const {
        if (real) return _mm512_mul_pd(v, re);
        __m512d sw = _mm512_permute_pd(v, 0x55);
        return _mm512_add_pd(_mm512_mul_pd(v, re), _mm512_mul_pd(sw, im));
    }
};

void avx512_diag(double* s, const qmo_gate& g, int64_t start, int64_t end) {
    int64_t bit = int64_t(1) << g.target;
    for (int64_t index = start; index < end;) {
        int64_t run = std::min(std::min(bit - (index & (bit - 1)), end - index), int64_t(4096));
        const double* phase = (index & bit) == 0 ? g.a : g.d;
        if (!is_one(phase)) {
            Coef512 c(phase);
            double* comp = s + 2 * index;
            int64_t lane = 0, n = 2 * run;
            for (; lane + 8 <= n; lane += 8) _mm512_storeu_pd(comp + lane, c.mul(_mm512_loadu_pd(comp + lane)));
            for (int64_t off = lane / 2; off < run; ++off) {
                cpx v = cmul({ s[2 * (index + off)], s[2 * (index + off) + 1] }, { phase[0], phase[1] });
                s[2 * (index + off)] = v.re; s[2 * (index + off) + 1] = v.im;
            }
        }
        index += run;
    }
}

void avx512_apply(double* s, const qmo_gate& g, int64_t start, int64_t end) {
    if (g.kernel == QMO_K_DIAGONAL) { avx512_diag(s, g, start, end); return; }
    int64_t bit = int64_t(1) << g.target;
    Coef512 a(g.a), b(g.b), c(g.c), d(g.d);
    __m512d scale = _mm512_set1_pd(g.a[0]);
    for (int64_t pair = start; pair < end;) {
        int64_t low = pair & (bit - 1);
        int64_t first = ((pair - low) << 1) | low, second = first | bit;
        int64_t run = std::min(std::min(bit - low, end - pair), int64_t(4096));
        double* zero = s + 2 * first;
        double* one = s + 2 * second;
        int64_t lane = 0, n = 2 * run;
        for (; lane + 8 <= n; lane += 8) {
            __m512d x = _mm512_loadu_pd(zero + lane), y = _mm512_loadu_pd(one + lane);
            if (g.kernel == QMO_K_EXCHANGE) {
                _mm512_storeu_pd(zero + lane, y);
                _mm512_storeu_pd(one + lane, x);
            } else if (g.kernel == QMO_K_HADAMARD) {
                __m512d sx = _mm512_mul_pd(x, scale), sy = _mm512_mul_pd(y, scale);
                _mm512_storeu_pd(zero + lane, _mm512_add_pd(sx, sy));
                _mm512_storeu_pd(one + lane, _mm512_sub_pd(sx, sy));
            } else {
                _mm512_storeu_pd(zero + lane, _mm512_add_pd(a.mul(x), b.mul(y)));
                _mm512_storeu_pd(one + lane, _mm512_add_pd(c.mul(x), d.mul(y)));
            }
        }
        for (int64_t off = lane / 2; off < run; ++off) {
            cpx x = { zero[2 * off], zero[2 * off + 1] }, y = { one[2 * off], one[2 * off + 1] };
            if (g.kernel == QMO_K_EXCHANGE) {
                zero[2 * off] = y.re; zero[2 * off + 1] = y.im; one[2 * off] = x.re; one[2 * off + 1] = x.im;
            } else {
                cpx o0 = cadd(cmul({ g.a[0], g.a[1] }, x), cmul({ g.b[0], g.b[1] }, y));
                cpx o1 = cadd(cmul({ g.c[0], g.c[1] }, x), cmul({ g.d[0], g.d[1] }, y));
                zero[2 * off] = o0.re; zero[2 * off + 1] = o0.im; one[2 * off] = o1.re; one[2 * off + 1] = o1.im;
            }
        }
        pair += run;
    }
}

// ------------------------------------------------------------------ AVX2 (AvxStateVectorKernel.cs)
struct Coef256 {
    __m256d re, im;
    bool real;
    Coef256(const double* f, const double* s) {
        re = _mm256_setr_pd(f[0], f[0], s[0], s[0]);
        im = _mm256_setr_pd(-f[1], f[1], -s[1], s[1]);
        real = f[1] == 0 && s[1] == 0;
    }
    inline __m256d mul(__m256d v) const {
        if (real) return _mm256_mul_pd(v, re);
        return _mm256_add_pd(_mm256_mul_pd(v, re), _mm256_mul_pd(_mm256_permute_pd(v, 0x05), im));
    }
};

void scalar_pair(double* s, const qmo_gate& g, int64_t first, int64_t second) {
    cpx x = { s[2 * first], s[2 * first + 1] }, y = { s[2 * second], s[2 * second + 1] };
    if (g.kernel == QMO_K_EXCHANGE) {
        s[2 * first] = y.re; s[2 * first + 1] = y.im; s[2 * second] = x.re; s[2 * second + 1] = x.im;
        return;
    }
    cpx o0 = cadd(cmul({ g.a[0], g.a[1] }, x), cmul({ g.b[0], g.b[1] }, y));
    cpx o1 = cadd(cmul({ g.c[0], g.c[1] }, x), cmul({ g.d[0], g.d[1] }, y));
    s[2 * first] = o0.re; s[2 * first + 1] = o0.im; s[2 * second] = o1.re; s[2 * second + 1] = o1.im;
}

void avx_diag(double* s, const qmo_gate& g, int64_t start, int64_t end) {
    int64_t bit = int64_t(1) << g.target;
    int64_t index = start;
    while (index < end) {
        if ((index & 1) != 0 || index + 1 == end) {
            const double* ph = (index & bit) == 0 ? g.a : g.d;
            cpx v = cmul({ s[2 * index], s[2 * index + 1] }, { ph[0], ph[1] });
            s[2 * index] = v.re; s[2 * index + 1] = v.im;
            ++index;
            continue;
        }
        const double* phase = (index & bit) == 0 ? g.a : g.d;
        int64_t run = std::min(std::min(bit == 1 ? end - index : bit - (index & (bit - 1)), end - index), int64_t(4096));
        run &= ~int64_t(1);
        if (bit != 1 && is_one(phase)) { index += run; continue; }
        Coef256 c = bit == 1 ? Coef256(g.a, g.d) : Coef256(phase, phase);
        double* comp = s + 2 * index;
        for (int64_t lane = 0; lane < 2 * run; lane += 4) _mm256_storeu_pd(comp + lane, c.mul(_mm256_loadu_pd(comp + lane)));
        index += run;
    }
}

void avx_apply(double* s, const qmo_gate& g, int64_t start, int64_t end) {
    int64_t bit = int64_t(1) << g.target;
    if (g.kernel == QMO_K_DIAGONAL) { avx_diag(s, g, start, end); return; }
    Coef256 a(g.a, g.a), b(g.b, g.b), c(g.c, g.c), d(g.d, g.d);
    Coef256 ac(g.a, g.c), bd(g.b, g.d);
    int64_t pair = start;
    while (pair < end) {
        int64_t low = pair & (bit - 1);
        int64_t first = ((pair - low) << 1) | low, second = first | bit;
        if (bit == 1) {
            int64_t cnt = std::min(int64_t(4096), end - pair);
            double* comp = s + 2 * first;
            for (int64_t off = 0; off < 4 * cnt; off += 4) {
                __m256d in = _mm256_loadu_pd(comp + off), out;
                if (g.kernel == QMO_K_EXCHANGE) out = _mm256_permute2f128_pd(in, in, 0x01);
                else {
                    __m256d x = _mm256_permute2f128_pd(in, in, 0x00), y = _mm256_permute2f128_pd(in, in, 0x11);
                    out = _mm256_add_pd(ac.mul(x), bd.mul(y));
                }
                _mm256_storeu_pd(comp + off, out);
            }
            pair += cnt;
            continue;
        }
        int64_t run = std::min(std::min(bit - low, end - pair), int64_t(4096));
        double* zero = s + 2 * first;
        double* one = s + 2 * second;
        int64_t lane = 0;
        for (; lane + 4 <= 2 * run; lane += 4) {
            __m256d x = _mm256_loadu_pd(zero + lane), y = _mm256_loadu_pd(one + lane);
            if (g.kernel == QMO_K_EXCHANGE) { _mm256_storeu_pd(zero + lane, y); _mm256_storeu_pd(one + lane, x); }
            else {
                _mm256_storeu_pd(zero + lane, _mm256_add_pd(a.mul(x), b.mul(y)));
                _mm256_storeu_pd(one + lane, _mm256_add_pd(c.mul(x), d.mul(y)));
            }
        }
        if (lane < 2 * run) scalar_pair(s, g, first + lane / 2, second + lane / 2);
        pair += run;
    }
}

// SimdHadamardKernel.cs (Vector<double> of 4 lanes = two complex values)
void simd_hadamard(double* s, int target, int64_t start, int64_t end) {
    int64_t bit = int64_t(1) << target;
    double h = std::sqrt(0.5);
    __m256d scale = _mm256_set1_pd(h);
    int64_t pair = start;
    while (pair < end) {
        int64_t low = pair & (bit - 1);
        int64_t first = ((pair - low) << 1) | low, second = first | bit;
        int64_t run = std::min(bit - low, end - pair);
        double* zero = s + 2 * first;
        double* one = s + 2 * second;
        int64_t off = 0;
        for (; off + 2 <= run; off += 2) {
            __m256d x = _mm256_loadu_pd(zero + 2 * off), y = _mm256_loadu_pd(one + 2 * off);
            __m256d sx = _mm256_mul_pd(x, scale), sy = _mm256_mul_pd(y, scale);
            _mm256_storeu_pd(zero + 2 * off, _mm256_add_pd(sx, sy));
            _mm256_storeu_pd(one + 2 * off, _mm256_sub_pd(sx, sy));
        }
        for (; off < run; ++off) {
            double xr = zero[2 * off], xi = zero[2 * off + 1], yr = one[2 * off], yi = one[2 * off + 1];
            zero[2 * off] = h * xr + h * yr; zero[2 * off + 1] = h * xi + h * yi;
            one[2 * off] = h * xr - h * yr; one[2 * off + 1] = h * xi - h * yi;
        }
        pair += run;
    }
}

// ParallelCpuStateVectorBackend.ApplyRange (:246-334)
void apply_range(double* s, const qmo_gate& g, int64_t start, int64_t end, bool simd, bool avx512) {
    int64_t bit = int64_t(1) << g.target;
    bool vec_kind = g.kernel == QMO_K_MATRIX || g.kernel == QMO_K_HADAMARD || g.kernel == QMO_K_EXCHANGE ||
                    g.kernel == QMO_K_DIAGONAL;
    if (simd && avx512 && g.control_mask == 0 && bit >= 4 && vec_kind) { avx512_apply(s, g, start, end); return; }
    if (simd && g.control_mask == 0 && vec_kind) {
        if (g.kernel != QMO_K_HADAMARD || bit == 1) { avx_apply(s, g, start, end); return; }
    }
    if (g.kernel == QMO_K_HADAMARD && g.control_mask == 0 && simd && bit >= 2) {
        simd_hadamard(s, g.target, start, end);
        return;
    }
    int64_t cmask = g.control_mask;
    if (g.kernel == QMO_K_DIAGONAL) {
        for (int64_t i = start; i < end; ++i)
            if ((i & cmask) == cmask) {
                const double* ph = (i & bit) == 0 ? g.a : g.d;
                cpx v = cmul({ s[2 * i], s[2 * i + 1] }, { ph[0], ph[1] });
                s[2 * i] = v.re; s[2 * i + 1] = v.im;
            }
        return;
    }
    int64_t swap_bit = g.kernel == QMO_K_SWAP ? (int64_t(1) << g.swap_control) : 0;
    for (int64_t pair = start; pair < end; ++pair) {
        int64_t low = pair & (bit - 1);
        int64_t first = ((pair - low) << 1) | low;
        if ((first & cmask) != cmask) continue;
        int64_t second = first | bit;
        if (g.kernel == QMO_K_SWAP) {
            if ((first & swap_bit) == 0) continue;
            second ^= swap_bit;
            cpx x = { s[2 * first], s[2 * first + 1] }, y = { s[2 * second], s[2 * second + 1] };
            s[2 * first] = y.re; s[2 * first + 1] = y.im; s[2 * second] = x.re; s[2 * second + 1] = x.im;
        } else {
            scalar_pair(s, g, first, second);
        }
    }
}

bool can_block(const qmo_gate& g) {
    return g.control_mask == 0 && (g.kernel == QMO_K_MATRIX || g.kernel == QMO_K_HADAMARD ||
                                   g.kernel == QMO_K_EXCHANGE || g.kernel == QMO_K_DIAGONAL);
}

// ParallelCpuStateVectorBackend.ApplyBlockedRange (:113-181)
void apply_blocked_range(double* s, const qmo_gate* gates, int count, int64_t start, int64_t end, bool simd, bool avx512) {
    int64_t bit = int64_t(1) << gates[0].target;
    alignas(64) double scratch[2 * 1024];
    bool packed = bit > 512;
    for (int64_t pair = start; pair < end;) {
        int64_t low = pair & (bit - 1);
        int64_t first = ((pair - low) << 1) | low;
        int64_t run = std::min(int64_t(512), end - pair);
        bool contiguous = low == 0 && bit <= run;
        if (contiguous) run -= run % bit;
        else run = std::min(run, bit - low);
        if (packed) {
            int local_target = 63 - __builtin_clzll((unsigned long long)run);
            run = int64_t(1) << local_target;
            int64_t second = first | bit;
            std::memcpy(scratch, s + 2 * first, size_t(run) * 16);
            std::memcpy(scratch + 2 * run, s + 2 * second, size_t(run) * 16);
            for (int gi = 0; gi < count; ++gi) {
                qmo_gate local = gates[gi];
                local.target = local_target;
                int64_t work = local.kernel == QMO_K_DIAGONAL ? 2 * run : run;
                apply_range(scratch, local, 0, work, simd, avx512);
            }
            std::memcpy(s + 2 * first, scratch, size_t(run) * 16);
            std::memcpy(s + 2 * second, scratch + 2 * run, size_t(run) * 16);
            pair += run;
            continue;
        }
        for (int gi = 0; gi < count; ++gi) {
            const qmo_gate& g = gates[gi];
            if (g.kernel != QMO_K_DIAGONAL) apply_range(s, g, pair, pair + run, simd, avx512);
            else if (contiguous) apply_range(s, g, first, first + 2 * run, simd, avx512);
            else {
                apply_range(s, g, first, first + run, simd, avx512);
                int64_t second = first | bit;
                apply_range(s, g, second, second + run, simd, avx512);
            }
        }
        pair += run;
    }
}

}  // namespace

extern "C" int qmp_hardware_threads(void) {
    unsigned n = std::thread::hardware_concurrency();
    return n ? int(n) : 1;
}

// ParallelCpuStateVectorBackend.Execute (:31-107)
extern "C" int qmp_execute(const qmp_options* opt, const qmo_operation* ops, int32_t count, int32_t qubits, double* s) {
    if (!opt || opt->workers < 1 || opt->workers > 256) return 10;
    if (opt->min_parallel_qubits < 1 || opt->min_parallel_qubits > 30) return 10;
    int rc = qmo_validate(ops, count, qubits);
    if (rc) return rc;
    int64_t len = int64_t(1) << qubits;
    bool parallel = qubits >= opt->min_parallel_qubits && opt->workers > 1;
    bool simd = opt->simd != 0, avx512 = opt->avx512 != 0;
    if (!parallel && !simd && !opt->blocking) { qmo_execute(ops, count, qubits, s); return 0; }
    std::vector<qmo_gate> prepared(static_cast<size_t>(count));
    if (count > 0 && (rc = qmo_prepare(ops, count, prepared.data())) != 0) return rc;
    Pool* pool = parallel ? &pool_for(opt->workers) : nullptr;
    for (int32_t oi = 0; oi < count; ++oi) {
        const qmo_gate& g = prepared[size_t(oi)];
        if (g.kernel == QMO_K_IDENTITY) continue;
        if (opt->blocking && can_block(g)) {
            int n = 1;
            while (n < 32 && oi + n < count) {
                const qmo_gate& next = prepared[size_t(oi + n)];
                if (next.target != g.target || !can_block(next)) break;
                ++n;
            }
            if (n > 1) {
                int64_t pairs = len / 2;
                int workers = parallel ? int(std::min<int64_t>(pairs, opt->workers)) : 1;
                const qmo_gate* block = &prepared[size_t(oi)];
                pool_for(workers).run(workers, [&](int w) {
                    int64_t a = pairs * w / workers, b = pairs * (w + 1) / workers;
                    apply_blocked_range(s, block, n, a, b, simd, avx512);
                });
                oi += n - 1;
                continue;
            }
        }
        int64_t items = g.kernel == QMO_K_DIAGONAL ? len : len / 2;
        int workers = parallel ? int(std::min<int64_t>(items, opt->workers)) : 1;
        if (workers == 1) { apply_range(s, g, 0, items, simd, avx512); continue; }
        pool->run(workers, [&](int w) {
            int64_t a = items * w / workers, b = items * (w + 1) / workers;
            apply_range(s, g, a, b, simd, avx512);
        });
    }
    return 0;
}
