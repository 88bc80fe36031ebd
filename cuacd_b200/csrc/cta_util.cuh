// cta_util.cuh — CTA-wide building blocks: in-place array scans and a
// bitonic sort of 64-bit keys (shared or global memory).
#pragma once
#include "common.cuh"

// In-place exclusive scan of n ints (any n), whole CTA.  Returns the total.
// `sh` needs 34 ints of shared memory.  Each warp owns a contiguous segment:
// pass 1 sums it, one CTA scan of the warp sums gives the segment offsets,
// pass 2 scans the segment 32 values at a time with a running carry, so the
// CTA meets three barriers whatever n is.
// kRankFlags: the entries are flags (non-zero = set); a set entry becomes
// the number of set entries before it, a clear one -1.
template <bool kRankFlags>
static __device__ int cta_scan_impl(int* data, int n, int* sh)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    const int seg = ((n + nw - 1) / nw + 31) & ~31;
    const int b = min(n, w * seg), e = min(n, b + seg);
    int sum = 0;
    for (int i = b + lane; i < e; i += 32) sum += kRankFlags ? (data[i] != 0) : data[i];
    #pragma unroll
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(FULL_MASK, sum, o);
    __syncthreads();                                   // sh may still be in use by the caller
    if (lane == 0) sh[w] = sum;
    __syncthreads();
    if (w == 0) {
        int v = lane < nw ? sh[lane] : 0, x = v;
        #pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(FULL_MASK, x, o);
            if (lane >= o) x += y;
        }
        if (lane < nw) sh[lane] = x - v;               // exclusive segment offsets
        if (lane == 31) sh[32] = x;                    // total
    }
    __syncthreads();
    int carry = sh[w];
    const int total = sh[32];
    for (int base = b; base < e; base += 32) {         // warp-uniform trip count
        const int i = base + lane;
        const int v = i < e ? (kRankFlags ? (data[i] != 0) : data[i]) : 0;
        int x = v;
        #pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(FULL_MASK, x, o);
            if (lane >= o) x += y;
        }
        if (i < e) data[i] = (kRankFlags && !v) ? -1 : carry + x - v;
        carry += __shfl_sync(FULL_MASK, x, 31);
    }
    __syncthreads();
    return total;
}

static __device__ int cta_scan_inplace(int* data, int n, int* sh) { return cta_scan_impl<false>(data, n, sh); }

// In-place ranks of set flags: data[i] != 0 becomes the number of set
// entries before i, data[i] == 0 becomes -1.  Returns the number set.
static __device__ int cta_rank_flags_inplace(int* data, int n, int* sh) { return cta_scan_impl<true>(data, n, sh); }

// Bitonic sort of keys[0..n) ascending; the array must hold next_pow2(n)
// entries (the tail is filled with ~0).  Whole CTA.
static __device__ void cta_sort_u64(unsigned long long* keys, int n)
{
    int N = 1;
    while (N < n) N <<= 1;
    for (int i = n + threadIdx.x; i < N; i += blockDim.x) keys[i] = ~0ull;
    __syncthreads();
    for (int k = 2; k <= N; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = threadIdx.x; i < N; i += blockDim.x) {
                int l = i ^ j;
                if (l > i) {
                    unsigned long long a = keys[i], b = keys[l];
                    bool up = (i & k) == 0;
                    if ((a > b) == up) { keys[i] = b; keys[l] = a; }
                }
            }
            __syncthreads();
        }
    }
}

__host__ __device__ inline int next_pow2_i(int x) { int p = 1; while (p < x) p <<= 1; return p; }

// lower_bound over sorted u64 keys
static __device__ __forceinline__ int lower_bound_u64(const unsigned long long* a, int n, unsigned long long k)
{
    int lo = 0, hi = n;
    while (lo < hi) { int m = (lo + hi) >> 1; if (a[m] < k) lo = m + 1; else hi = m; }
    return lo;
}

// Stable LSD radix sort of n 64-bit keys by bits [lo_bit, lo_bit + nbits),
// 8 bits per pass (whole CTA of NT threads).  `tmp` holds n keys; the
// result is in `keys`.  `cnt` needs 256 * NT/32 ints of shared memory, `sh`
// 34 ints.  Per pass: per-warp digit counts over contiguous segments, one
// CTA scan (digit-major, warp-minor), then a stable scatter ranked with
// __match_any_sync inside each 32-key chunk.
template <int NT>
static __device__ void cta_radix_sort_u64(unsigned long long* keys, unsigned long long* tmp, int n, int lo_bit,
                                          int nbits, int* cnt, int* sh)
{
    constexpr int NW = NT / 32;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int seg = (n + NW - 1) / NW;
    const int b = min(n, w * seg), e = min(n, b + seg);
    unsigned long long* src = keys;
    unsigned long long* dst = tmp;
    int passes = 0;
    for (int s = lo_bit; s < lo_bit + nbits; s += 8) {
        for (int c = threadIdx.x; c < 256 * NW; c += NT) cnt[c] = 0;
        __syncthreads();
        for (int i = b + lane; i < e; i += 32) atomicAdd(&cnt[(int)((src[i] >> s) & 255ull) * NW + w], 1);
        __syncthreads();
        cta_scan_inplace(cnt, 256 * NW, sh);
        for (int base = b; base < e; base += 32) {          // warp-uniform trip count
            const int i = base + lane;
            unsigned long long k = 0;
            int d = -1;
            if (i < e) { k = src[i]; d = (int)((k >> s) & 255ull); }
            const unsigned m = __match_any_sync(FULL_MASK, d);
            const int rank = __popc(m & ((1u << lane) - 1u));
            int p = 0;
            if (d >= 0) p = cnt[d * NW + w] + rank;
            __syncwarp();
            if (d >= 0 && rank == 0) cnt[d * NW + w] += __popc(m);
            __syncwarp();
            if (d >= 0) dst[p] = k;
        }
        __syncthreads();
        unsigned long long* t = src; src = dst; dst = t;
        passes++;
    }
    if (passes & 1) {
        for (int i = threadIdx.x; i < n; i += NT) keys[i] = src[i];
        __syncthreads();
    }
}
