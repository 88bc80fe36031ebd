// cuda_runtime.h stand-in for the CTA emulator (test infrastructure only).
//
// Compiles a one-CTA device function for the CPU: every CUDA thread is a
// std::thread, __shared__ variables are function statics, and every
// __syncthreads / __syncthreads_or / warp intrinsic is a barrier that first
// checks that every live thread of the CTA (or warp) reached the SAME call
// site.  A barrier reached from different sites -- undefined behaviour on the
// GPU, where sm_100 reports it as an illegal instruction -- is printed as
// "[emu] ... divergent ..." instead of faulting.  Warp intrinsics also report
// partial masks and lanes that have exited.  Memory accesses are plain host
// accesses, so the build can run under AddressSanitizer.
#pragma once
#include <algorithm>
#include <atomic>
#include <barrier>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>
using std::max;
using std::min;
#define __device__
#define __host__
#define __global__
#define __forceinline__ inline
#define __launch_bounds__(...)
#define __restrict__
#define __shared__ static
#define __align__(x) alignas(x)
struct float4 { float x, y, z, w; };
struct int2 { int x, y; };
struct alignas(16) ulonglong2 { unsigned long long x, y; };
struct dim3 { unsigned x = 0, y = 0, z = 0; };
inline float4 make_float4(float a, float b, float c, float d) { return {a, b, c, d}; }
inline int2 make_int2(int a, int b) { return {a, b}; }
typedef int cudaStream_t;
extern thread_local dim3 threadIdx;
extern dim3 blockIdx, blockDim, gridDim;

namespace emu {
extern int NT;                          // threads of the emulated CTA
extern std::barrier<>* cta_bar;
extern std::barrier<>* warp_bar[64];
extern int site[1024];                  // call site of each thread's current barrier (-1: exited)
extern unsigned long long xch[1024];    // warp exchange slots
extern std::atomic<int> live[64];       // live lanes per warp
extern std::atomic<long long> clk;
void report(const char* what, int line);

inline void cta_sync(int line)
{
    const int t = threadIdx.x;
    site[t] = line;
    cta_bar->arrive_and_wait();
    if (t == 0)
        for (int i = 0; i < NT; i++)
            if (site[i] != line && site[i] != -1) { report("divergent __syncthreads", line); break; }
    cta_bar->arrive_and_wait();
}
inline int warp_enter(unsigned mask, unsigned long long v, int line)
{
    const int t = threadIdx.x, w = t >> 5;
    if (mask != 0xffffffffu) report("partial warp mask", line);
    if (live[w].load() != 32) report("warp intrinsic with exited lanes", line);
    site[t] = line;
    xch[t] = v;
    warp_bar[w]->arrive_and_wait();
    for (int i = 0; i < 32; i++)
        if (site[w * 32 + i] != line) { report("divergent warp intrinsic", line); break; }
    return t & 31;
}
inline void warp_leave() { warp_bar[threadIdx.x >> 5]->arrive_and_wait(); }
template <class T> unsigned long long bits(T v) { unsigned long long b = 0; std::memcpy(&b, &v, sizeof(T)); return b; }
template <class T> T unbits(unsigned long long b) { T v; std::memcpy(&v, &b, sizeof(T)); return v; }
}  // namespace emu

#define __syncthreads() emu::cta_sync(__LINE__)
inline int emu_sync_or(int x, int line)
{
    static std::atomic<int> acc{0};
    emu::cta_sync(line);
    if (x) acc.fetch_or(1);
    emu::cta_sync(line);
    const int r = acc.load();
    emu::cta_sync(line);
    if (threadIdx.x == 0) acc.store(0);
    emu::cta_sync(line);
    return r;
}
#define __syncthreads_or(x) emu_sync_or((x), __LINE__)

template <class T> T emu_shfl(unsigned m, T v, int src, int line)
{
    emu::warp_enter(m, emu::bits(v), line);
    T r = emu::unbits<T>(emu::xch[(threadIdx.x & ~31u) + (src & 31)]);
    emu::warp_leave();
    return r;
}
template <class T> T emu_shfl_up(unsigned m, T v, int d, int line)
{
    const int lane = emu::warp_enter(m, emu::bits(v), line);
    T r = lane >= d ? emu::unbits<T>(emu::xch[threadIdx.x - d]) : v;
    emu::warp_leave();
    return r;
}
template <class T> T emu_shfl_xor(unsigned m, T v, int x, int line)
{
    const int lane = emu::warp_enter(m, emu::bits(v), line);
    T r = emu::unbits<T>(emu::xch[(threadIdx.x & ~31u) + (lane ^ x)]);
    emu::warp_leave();
    return r;
}
inline unsigned emu_ballot(unsigned m, int p, int line)
{
    emu::warp_enter(m, p ? 1ull : 0ull, line);
    unsigned b = 0;
    for (int i = 0; i < 32; i++) if (emu::xch[(threadIdx.x & ~31u) + i]) b |= 1u << i;
    emu::warp_leave();
    return b;
}
template <class T> unsigned emu_match_any(unsigned m, T v, int line)
{
    emu::warp_enter(m, emu::bits(v), line);
    const unsigned long long me = emu::xch[threadIdx.x];
    unsigned b = 0;
    for (int i = 0; i < 32; i++) if (emu::xch[(threadIdx.x & ~31u) + i] == me) b |= 1u << i;
    emu::warp_leave();
    return b;
}
#define __shfl_sync(m, v, s) emu_shfl((m), (v), (s), __LINE__)
#define __shfl_up_sync(m, v, d) emu_shfl_up((m), (v), (d), __LINE__)
#define __shfl_xor_sync(m, v, x) emu_shfl_xor((m), (v), (x), __LINE__)
#define __ballot_sync(m, p) emu_ballot((m), (p), __LINE__)
#define __any_sync(m, p) (emu_ballot((m), (p), __LINE__) != 0)
#define __match_any_sync(m, v) emu_match_any((m), (v), __LINE__)
#define __syncwarp(...) do { emu::warp_enter(0xffffffffu, 0, __LINE__); emu::warp_leave(); } while (0)
inline int __popc(unsigned x) { return __builtin_popcount(x); }
inline int __ffs(unsigned x) { return __builtin_ffs(x); }
inline int __float_as_int(float f) { int i; std::memcpy(&i, &f, 4); return i; }
inline float __int_as_float(int i) { float f; std::memcpy(&f, &i, 4); return f; }
inline long long clock64() { return emu::clk.fetch_add(1); }
inline void __threadfence() { std::atomic_thread_fence(std::memory_order_seq_cst); }
template <class T> T atomicAdd(T* p, T v) { return std::atomic_ref<T>(*p).fetch_add(v); }
template <class T> T atomicOr(T* p, T v) { return std::atomic_ref<T>(*p).fetch_or(v); }
template <class T> T atomicMin(T* p, T v)
{
    std::atomic_ref<T> a(*p);
    T o = a.load();
    while (v < o && !a.compare_exchange_weak(o, v)) {}
    return o;
}
template <class T> T atomicMax(T* p, T v)
{
    std::atomic_ref<T> a(*p);
    T o = a.load();
    while (v > o && !a.compare_exchange_weak(o, v)) {}
    return o;
}
template <class T> T atomicCAS(T* p, T c, T v) { std::atomic_ref<T>(*p).compare_exchange_strong(c, v); return c; }
template <class T> T atomicExch(T* p, T v) { return std::atomic_ref<T>(*p).exchange(v); }

// IEEE round-to-nearest float intrinsics: the host's float operations round
// the same way when built with -ffp-contract=off.
inline float __fdiv_rn(float a, float b) { return a / b; }
inline float __fadd_rn(float a, float b) { return a + b; }
inline float __fsub_rn(float a, float b) { return a - b; }
inline float __fmul_rn(float a, float b) { return a * b; }
inline int __float2int_rz(float x) { return (int)x; }
template <class T> T __ldcg(const T* p) { return std::atomic_ref<T>(*const_cast<T*>(p)).load(); }
template <class T> T atomicSub(T* p, T v) { return std::atomic_ref<T>(*p).fetch_sub(v); }
