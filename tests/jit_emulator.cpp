// jit_emulator.cpp -- TEST INFRASTRUCTURE: runs one generated pass kernel (qm_pass) on the CPU.
//
// The source that the library compiles with NVRTC for sm_100a is included here as C++ with the
// CUDA keywords defined away: every thread of the block is a std::thread, __syncthreads is a
// std::barrier, shared memory is one static array, and the blocks of the grid run one after
// another, each walking its work items in order.  Tests compare the result with the oracle, so
// the generated arithmetic (rotations between deferred phases, phases carried across passes,
// flushes) is checked without a GPU.  The tile copies of the pipelined forms (cp.async) are
// copies made at once, and the named barriers of two-team blocks are std::barriers of the
// counts the kernel names: a team's own barrier (ids 1, 2) and the token barriers (ids 3, 4),
// where bar.sync is arrive_and_wait and bar.arrive is arrive.  A hand-over protocol whose
// arrivals do not match hangs here instead of on the GPU.  Built per pass by
// tests/jit_emulator.py with -DGENERATED="<file>".
#include <barrier>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

struct double2 { double x, y; };
struct float2 { float x, y; };
struct uint2 { unsigned x, y; };
struct EmuDim { unsigned x, y, z; };
thread_local EmuDim threadIdx{0, 0, 0};
thread_local EmuDim blockIdx{0, 0, 0};
static EmuDim gridDim{1, 1, 1};
static std::barrier<>* g_bar = nullptr;
static std::vector<std::barrier<>*> g_warp_bar;
static std::barrier<>* g_named[5] = {};
static unsigned g_named_count[5] = {};
static double g_shfl[64][32];

inline void __syncthreads() { g_bar->arrive_and_wait(); }
inline int __popc(unsigned v) { return __builtin_popcount(v); }
template <class T>
inline T __ldg(const T* p) { return *p; }
inline double __shfl_xor_sync(unsigned, double v, int m) {
    const unsigned w = threadIdx.x >> 5, l = threadIdx.x & 31;
    g_shfl[w][l] = v;
    g_warp_bar[w]->arrive_and_wait();
    const double r = g_shfl[w][l ^ (unsigned)m];
    g_warp_bar[w]->arrive_and_wait();
    return r;
}

#define __global__
#define __device__
#define __forceinline__ inline
#define __launch_bounds__(a, b)
#define __grid_constant__
#define __shared__
#define __align__(n) __attribute__((aligned(n)))

alignas(16) unsigned char smem_raw[1 << 21];

typedef unsigned int u32;
inline size_t __cvta_generic_to_shared(const void* p) {
    return (size_t)(static_cast<const unsigned char*>(p) - smem_raw);
}
inline void qm_cp16(u32 dst, const void* src) { std::memcpy(smem_raw + dst, src, 16); }
inline void qm_cp8(u32 dst, const void* src) { std::memcpy(smem_raw + dst, src, 8); }
inline void qm_cp_commit() {}
inline void qm_cp_wait() {}
inline void named_check(u32 id, u32 n) {
    if (id < 1 || id > 4 || !g_named[id] || g_named_count[id] != n) std::abort();
}
inline void qm_bar(u32 id, u32 n) {
    named_check(id, n);
    g_named[id]->arrive_and_wait();
}
inline void qm_arrive(u32 id, u32 n) {
    named_check(id, n);
    (void)g_named[id]->arrive();
}

#define QM_EMULATED
#include GENERATED

extern "C" int emu_run(void* s0, const void* launch, size_t launch_size, const void* aux, size_t aux_size, void* hist,
                       int threads, int teams, int grid) {
    FusedLaunch P;
    if (launch_size != sizeof(P)) return -1;
    std::memcpy(&P, launch, sizeof(P));
    Aux A;
    if (aux_size != sizeof(A)) return -2;
    std::memcpy(&A, aux, sizeof(A));
    if (teams < 1 || teams > 2 || grid < 1 || threads % (32 * teams) != 0) return -3;
    std::barrier<> bar(threads);
    g_bar = &bar;
    g_warp_bar.clear();
    for (int w = 0; w < threads / 32; ++w) g_warp_bar.push_back(new std::barrier<>(32));
    for (int id = 1; id <= 4; ++id) {
        g_named_count[id] = (unsigned)(id <= 2 ? threads / teams : threads);
        g_named[id] = new std::barrier<>(g_named_count[id]);
    }
    (void)hist;
    gridDim.x = (unsigned)grid;
    for (int blk = 0; blk < grid; ++blk) {
        std::vector<std::thread> pool;
        for (int t = 0; t < threads; ++t)
            pool.emplace_back([&, t, blk] {
                threadIdx.x = (unsigned)t;
                blockIdx.x = (unsigned)blk;
                qm_pass(static_cast<V*>(s0), P, A EMU_HIST_ARG);
            });
        for (auto& th : pool) th.join();
    }
    gridDim.x = 1;
    for (auto* b : g_warp_bar) delete b;
    g_warp_bar.clear();
    for (int id = 1; id <= 4; ++id) {
        delete g_named[id];
        g_named[id] = nullptr;
    }
    return 0;
}
