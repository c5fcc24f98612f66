// qm_random.cpp -- the host draw stream of seeded simulations in libqmb200.so.
//
// The reference draws every measurement and Kraus selector from a seeded System.Random
// (NoisyStateVectorSimulator.cs:42,111; StateVectorSimulator.cs:42).  For a seed, .NET keeps
// the published subtractive generator of Knuth (TAOCP vol. 2, 3.6) with its 55-entry table,
// lag 21 and modulus 2^31 - 1; NextDouble() is the next sample divided by 2^31 - 1.  This
// file restates that algorithm; the library's kernels never call it.
#include <stdint.h>

#include <cstdlib>

#include "qm_b200.h"
#include "qm_internal.h"

namespace {

constexpr int32_t kModulus = 2147483647;  // 2^31 - 1
constexpr int32_t kSeedOffset = 161803398;

struct Subtractive {
    int32_t table[56];
    int32_t next = 0, next_lag = 21;

    explicit Subtractive(int32_t seed) {
        const int32_t magnitude = seed == INT32_MIN ? kModulus : std::abs(seed);
        int32_t value = kSeedOffset - magnitude;
        table[55] = value;
        int32_t prior = 1;
        int32_t index = 0;
        for (int32_t i = 1; i < 55; ++i) {  // spread the seed over the table in steps of 21
            index += 21;
            if (index >= 55) index -= 55;
            table[index] = prior;
            prior = value - prior;
            if (prior < 0) prior += kModulus;
            value = table[index];
        }
        for (int round = 1; round < 5; ++round)  // four warm-up rounds
            for (int32_t i = 1; i < 56; ++i) {
                int32_t j = i + 30;
                if (j >= 55) j -= 55;
                table[i] -= table[1 + j];
                if (table[i] < 0) table[i] += kModulus;
            }
    }

    int32_t sample() {
        if (++next >= 56) next = 1;
        if (++next_lag >= 56) next_lag = 1;
        int32_t v = table[next] - table[next_lag];
        if (v == kModulus) --v;
        if (v < 0) v += kModulus;
        table[next] = v;
        return v;
    }

    double next_double() { return sample() * (1.0 / kModulus); }
};

}  // namespace

extern "C" int32_t qm_random_doubles(int32_t seed, int64_t skip, int64_t count, double* out) {
    if (skip < 0 || count < 0) return qm::fail(QM_E_RANGE, "skip and count must be nonnegative");
    if (count > 0 && !out) return qm::fail(QM_E_ARG, "out is null");
    Subtractive r(seed);
    for (int64_t i = 0; i < skip; ++i) r.sample();
    for (int64_t i = 0; i < count; ++i) out[i] = r.next_double();
    return QM_OK;
}
