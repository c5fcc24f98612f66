// jit_emulator.cpp -- TEST INFRASTRUCTURE: runs one generated pass kernel (qm_pass) on the CPU.
//
// The source that the library compiles with NVRTC for sm_100a is included here as C++ with the
// CUDA keywords defined away: every thread of the block is a std::thread, __syncthreads is a
// std::barrier, shared memory is one static array, and a single block (gridDim.x = 1) walks
// every work item in order.  Tests compare the result with the oracle, so the generated
// arithmetic (rotations between deferred phases, phases carried across passes, flushes) is
// checked without a GPU.  Built per pass by tests/jit_emulator.py with -DGENERATED="<file>".
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

#include GENERATED

extern "C" int emu_run(void* s0, const void* launch, size_t launch_size, const void* aux, size_t aux_size, void* hist,
                       int threads) {
    FusedLaunch P;
    if (launch_size != sizeof(P)) return -1;
    std::memcpy(&P, launch, sizeof(P));
    Aux A;
    if (aux_size != sizeof(A)) return -2;
    std::memcpy(&A, aux, sizeof(A));
    std::barrier<> bar(threads);
    g_bar = &bar;
    g_warp_bar.clear();
    for (int w = 0; w < threads / 32; ++w) g_warp_bar.push_back(new std::barrier<>(32));
    (void)hist;
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t)
        pool.emplace_back([&, t] {
            threadIdx.x = (unsigned)t;
            blockIdx.x = 0;
            qm_pass(static_cast<V*>(s0), P, A EMU_HIST_ARG);
        });
    for (auto& th : pool) th.join();
    for (auto* b : g_warp_bar) delete b;
    g_warp_bar.clear();
    return 0;
}
