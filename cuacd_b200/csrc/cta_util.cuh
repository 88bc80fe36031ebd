// cta_util.cuh — CTA-wide building blocks: in-place array scans and a
// bitonic sort of 64-bit keys (shared or global memory).
#pragma once
#include "common.cuh"

// In-place exclusive scan of n ints (any n), whole CTA.  Returns the total.
// `sh` needs 34 ints of shared memory.
static __device__ int cta_scan_inplace(int* data, int n, int* sh)
{
    int carry = 0;
    for (int base = 0; base < n; base += blockDim.x) {
        int i = base + threadIdx.x;
        int v = (i < n) ? data[i] : 0;
        int tot;
        int ex = block_exclusive_scan(v, sh, &tot);
        if (i < n) data[i] = carry + ex;
        carry += tot;
    }
    __syncthreads();
    return carry;
}

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
