// cuda_host_emu.h -- host stand-ins for the CUDA built-ins that the
// library's device code uses, so that g++ can compile that code and the CPU
// tests can run it (tests/kernels_host.cpp, tests/adjoint32_host.cpp).
//
// Launches are emulated block by block (emu::launch).  Kernels with warp
// shuffles or block barriers run one host thread per CUDA thread: a shuffle
// is an exchange through per-lane slots between two barriers of the warp's
// 32 threads (a butterfly shuffle and a vote likewise), __syncthreads a
// barrier of the block's threads, atomics take a lock, and __shared__ arrays
// are static (one block runs at a time).  Kernels with neither run their
// threads one after another.  1/sqrt(x) and the two-wide FP32 operations of
// sm_100 are computed as 1/sqrt(x) and two correctly rounded operations.
// Include before the library's device headers.
#pragma once

#include <atomic>
#include <cmath>
#include <cstring>
#include <mutex>
#include <thread>
#include <type_traits>
#include <vector>

#include <cuda_runtime.h>

#undef __shared__
#define __shared__ static

static thread_local uint3 threadIdx;
static uint3 blockIdx;
static dim3 blockDim, gridDim;

namespace emu {
constexpr int kLanes = 32, kMaxWarps = 32;

// Generation barrier of n threads; waiters yield rather than sleep (the
// emulated warps run far more threads than cores, and a barrier releases
// within microseconds).
struct Barrier {
    std::atomic<int> count{0}, gen{0};
    int n = kLanes;
    void wait()
    {
        const int g = gen.load(std::memory_order_acquire);
        if (count.fetch_add(1, std::memory_order_acq_rel) == n - 1) {
            count.store(0, std::memory_order_relaxed);
            gen.fetch_add(1, std::memory_order_release);
        } else {
            while (gen.load(std::memory_order_acquire) == g) std::this_thread::yield();
        }
    }
};
static Barrier warp_bar[kMaxWarps];
static Barrier block_bar;
static unsigned char slot[kMaxWarps][kLanes][16];

inline int flat_thread() { return int(threadIdx.x + threadIdx.y * blockDim.x); }

// value of lane (lane + delta) of the caller's warp, or the caller's own
// where that lane is outside the warp, as the hardware shuffles do
template <typename T>
T exchange(T v, int delta)
{
    static_assert(sizeof(T) <= sizeof(slot[0][0]), "shuffle operand too wide");
    const int f = flat_thread(), w = f / kLanes, lane = f % kLanes;
    std::memcpy(slot[w][lane], &v, sizeof(T));
    warp_bar[w].wait();
    T r = v;
    const int src = lane + delta;
    if (src >= 0 && src < kLanes) std::memcpy(&r, slot[w][src], sizeof(T));
    warp_bar[w].wait();
    return r;
}

// lane ^ mask's value (butterfly shuffle)
template <typename T>
T exchange_xor(T v, int mask)
{
    const int lane = flat_thread() % kLanes;
    return exchange(v, (lane ^ mask) - lane);
}

// warp vote: nonzero if any lane's predicate is
inline int vote_any(int pred)
{
    const int f = flat_thread(), w = f / kLanes, lane = f % kLanes;
    std::memcpy(slot[w][lane], &pred, sizeof pred);
    warp_bar[w].wait();
    int any = 0;
    for (int l = 0; l < kLanes; ++l) {
        int q;
        std::memcpy(&q, slot[w][l], sizeof q);
        any |= q != 0;
    }
    warp_bar[w].wait();
    return any;
}

static std::mutex atomic_mutex;  // the atomics of threaded launches

// Runs `body` as the kernel body of every thread of every block of the grid:
// `threaded` for kernels that shuffle or wait at block barriers (whole warps
// of threads), else thread after thread.
template <class F>
void launch(dim3 grid, dim3 block, bool threaded, F body)
{
    gridDim = grid;
    blockDim = block;
    const int nt = int(block.x * block.y);
    block_bar.n = nt;
    for (unsigned by = 0; by < grid.y; ++by)
        for (unsigned bx = 0; bx < grid.x; ++bx) {
            blockIdx = make_uint3(bx, by, 0);
            auto run = [&](int t) {
                threadIdx = make_uint3(unsigned(t) % block.x, unsigned(t) / block.x, 0);
                body();
            };
            if (threaded) {
                std::vector<std::thread> th;
                for (int t = 0; t < nt; ++t) th.emplace_back(run, t);
                for (auto &x : th) x.join();
            } else {
                for (int t = 0; t < nt; ++t) run(t);
            }
        }
}
} // namespace emu

static inline double rsqrt(double x) { return 1.0 / std::sqrt(x); }
static inline float rsqrtf(float x) { return 1.0f / std::sqrt(x); }
// correctly rounded products and sums that the compiler may not contract
static inline double __dmul_rn(double a, double b) { return a * b; }
static inline double __dadd_rn(double a, double b) { return a + b; }
// sm_100's two-wide FP32 instructions: two correctly rounded operations
static inline float2 __fadd2_rn(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
static inline float2 __fmul2_rn(float2 a, float2 b) { return make_float2(a.x * b.x, a.y * b.y); }
static inline float2 __ffma2_rn(float2 a, float2 b, float2 c)
{
    return make_float2(std::fma(a.x, b.x, c.x), std::fma(a.y, b.y, c.y));
}
template <typename T>
static inline T __shfl_xor_sync(unsigned, T v, int m) { return emu::exchange_xor(v, m); }
template <typename T>
static inline T __shfl_down_sync(unsigned, T v, int d) { return emu::exchange(v, d); }
template <typename T>
static inline T __shfl_up_sync(unsigned, T v, int d) { return emu::exchange(v, -d); }
template <typename T>
static inline T __shfl_sync(unsigned, T v, int src)
{
    return emu::exchange(v, (src & (emu::kLanes - 1)) - emu::flat_thread() % emu::kLanes);
}
static inline void __syncthreads() { emu::block_bar.wait(); }
static inline void __syncwarp(unsigned = 0xffffffffu) { emu::warp_bar[emu::flat_thread() / emu::kLanes].wait(); }
static inline void __threadfence() {}
static inline int __any_sync(unsigned, int p) { return emu::vote_any(p); }
static inline long long __double_as_longlong(double x)
{
    long long r;
    std::memcpy(&r, &x, 8);
    return r;
}
static inline double __longlong_as_double(long long x)
{
    double r;
    std::memcpy(&r, &x, 8);
    return r;
}
template <typename T>
static inline T atomicAdd(T *p, T v)
{
    std::lock_guard<std::mutex> g(emu::atomic_mutex);
    const T o = *p;
    *p = o + v;
    return o;
}
template <typename T>
static inline T atomicMax(T *p, T v)
{
    std::lock_guard<std::mutex> g(emu::atomic_mutex);
    const T o = *p;
    if (v > o) *p = v;
    return o;
}
template <typename T>
static inline T atomicCAS(T *p, T c, T v)
{
    std::lock_guard<std::mutex> g(emu::atomic_mutex);
    const T o = *p;
    if (o == c) *p = v;
    return o;
}
#pragma GCC diagnostic ignored "-Wunknown-pragmas"
static inline int min(int a, int b) { return a < b ? a : b; }
static inline int max(int a, int b) { return a > b ? a : b; }
#define __launch_bounds__(...)
