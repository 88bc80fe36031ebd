// common.cuh — shared device conventions for the candidate-evaluation path.
//
// Error word: single-bit flags OR-ed into a device int, the same bit layout as
// the reference's KERR_* codes (cuda/error_codes.cuh:14-53) so hosts that decode
// them keep working.  Bits this build never raises are kept for the layout.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#define KERR_BT_WARP_OOM       (1 <<  0)
#define KERR_BT_SORT_STACK     (1 <<  1)
#define KERR_BT_DC_STACK       (1 <<  2)
#define KERR_BT_POOL_EXHAUST   (1 <<  3)   // hull scratch capacity exceeded
#define KERR_BT_HEAP_TO_WARP   (1 <<  4)
#define KERR_BT_HEAP_OUTPUT    (1 <<  5)   // hull output capacity exceeded
#define KERR_BT_EXTRACT_FAIL   (1 <<  6)   // hull construction inconsistent
#define KERR_PC_SCRATCH_OOM    (1 <<  7)   // plane-cut scratch capacity exceeded
#define KERR_PC_POOL_OOM       (1 <<  8)   // plane-cut output capacity exceeded
#define KERR_PC_SORT_ERR       (1 <<  9)
#define KERR_HD_SCRATCH_OOM    (1 << 10)   // Hausdorff scratch capacity exceeded
#define KERR_HD_SORT_ERR       (1 << 11)
#define KERR_DC_OOM            (1 << 12)
#define KERR_KDOP_SCRATCH_OOM  (1 << 13)
#define KERR_LA_OVERFLOW       (1 << 14)
#define KERR_LA_SORT_OOM       (1 << 15)
#define KERR_LA_SORT_STACK     (1 << 16)
#define KERR_LA_EVAL_OOM       (1 << 17)
#define KERR_MESH_INVALID      (1 << 18)
#define KERR_HEAP_OOM          (1 << 19)   // arena exhausted
#define KERR_HEAP_CORRUPT      (1 << 20)
#define KERR_HEAP_CORRUPT_PREV (1 << 21)
#define KERR_TIMEOUT           (1 << 22)   // a bounded device wait gave up
#define KERR_COUNT     23

#define WARP 32
#define FULL_MASK 0xffffffffu

// ---------------------------------------------------------------------------
// Arena: one device buffer, bump-allocated by atomicAdd; reset by the host
// between launches that own it.  Never waits, so no lock can hang the GPU.
// ---------------------------------------------------------------------------
struct Arena {
    char*               base;
    unsigned long long  capacity;
    unsigned long long  offset;       // bump pointer (bytes)
    unsigned long long  high_water;   // max offset ever reached
    unsigned long long  n_allocs;     // allocations served since init
    unsigned long long  n_resets;     // host resets since init
};

// Allocate `bytes` (rounded to 256) from the arena; nullptr + KERR_HEAP_OOM when
// exhausted.  Call from one thread.
static __device__ __forceinline__ void* arena_alloc(Arena* a, unsigned long long bytes, int* err)
{
    bytes = (bytes + 255ull) & ~255ull;
    unsigned long long off = atomicAdd(&a->offset, bytes);
    if (off + bytes > a->capacity) {
        if (err) atomicOr(err, KERR_HEAP_OOM);
        return nullptr;
    }
    atomicMax(&a->high_water, off + bytes);
    atomicAdd(&a->n_allocs, 1ull);
    return a->base + off;
}

// ---------------------------------------------------------------------------
// warp / block helpers
// ---------------------------------------------------------------------------
static __device__ __forceinline__ float warp_min(float v) {
    #pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(FULL_MASK, v, o));
    return v;
}
static __device__ __forceinline__ float warp_max(float v) {
    #pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(FULL_MASK, v, o));
    return v;
}
static __device__ __forceinline__ float warp_sum(float v) {
    #pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL_MASK, v, o);
    return v;
}
static __device__ __forceinline__ double warp_sum_d(double v) {
    #pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL_MASK, v, o);
    return v;
}
static __device__ __forceinline__ int warp_sum_i(int v) {
    #pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL_MASK, v, o);
    return v;
}

// Block-wide exclusive scan of one int per thread; returns the exclusive
// prefix, writes the block total to *total.  `sh` needs blockDim/32 + 1 ints.
static __device__ __forceinline__ int block_exclusive_scan(int v, int* sh, int* total)
{
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    int x = v;
    #pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(FULL_MASK, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) sh[w] = x;
    __syncthreads();
    if (w == 0) {
        int s = lane < nw ? sh[lane] : 0;
        #pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(FULL_MASK, s, o);
            if (lane >= o) s += y;
        }
        if (lane < nw) sh[lane] = s;          // inclusive per-warp totals
        if (lane == nw - 1) sh[32] = s;
    }
    __syncthreads();
    int excl = x - v + (w > 0 ? sh[w - 1] : 0);
    if (total) *total = sh[32];
    __syncthreads();
    return excl;
}

static __device__ __forceinline__ double block_sum_d(double v, double* sh)
{
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    v = warp_sum_d(v);
    if (lane == 0) sh[w] = v;
    __syncthreads();
    double r = 0.0;
    if (w == 0) {
        r = lane < nw ? sh[lane] : 0.0;
        r = warp_sum_d(r);
        if (lane == 0) sh[32] = r;
    }
    __syncthreads();
    r = sh[32];
    __syncthreads();
    return r;
}

// float atomic max for non-negative values (bit patterns order like ints)
static __device__ __forceinline__ void atomic_max_nonneg(float* addr, float v) {
    atomicMax(reinterpret_cast<int*>(addr), __float_as_int(v));
}

// ---------------------------------------------------------------------------
// mesh volume (divergence theorem), FP64 accumulation
// cuda/mesh_volume.cuh:20-57: signed-tet sum anchored at vertex 0.
// ---------------------------------------------------------------------------
static __device__ __forceinline__ double tet6_d(const float* __restrict__ v, int a, int b, int c,
                                         double ox, double oy, double oz)
{
    double ax = (double)v[3*a] - ox, ay = (double)v[3*a+1] - oy, az = (double)v[3*a+2] - oz;
    double bx = (double)v[3*b] - ox, by = (double)v[3*b+1] - oy, bz = (double)v[3*b+2] - oz;
    double cx = (double)v[3*c] - ox, cy = (double)v[3*c+1] - oy, cz = (double)v[3*c+2] - oz;
    double nx = by*cz - bz*cy, ny = bz*cx - bx*cz, nz = bx*cy - by*cx;
    return ax*nx + ay*ny + az*nz;
}

// Block-cooperative signed volume of one mesh (all threads call).
static __device__ __forceinline__ double block_mesh_signed_volume(const float* __restrict__ v, int nv,
                                                           const int* __restrict__ t, int nt,
                                                           double* sh)
{
    if (nt <= 0 || nv <= 0) return 0.0;
    double ox = v[0], oy = v[1], oz = v[2];
    double acc = 0.0;
    for (int i = threadIdx.x; i < nt; i += blockDim.x)
        acc += tet6_d(v, t[3*i], t[3*i+1], t[3*i+2], ox, oy, oz);
    return block_sum_d(acc, sh) / 6.0;
}

// ---------------------------------------------------------------------------
// part costs: cuda/la_common.cuh:21-34
// ---------------------------------------------------------------------------
static __device__ __forceinline__ float part_cost_rv(double hull_vol, double mesh_vol) {
    const double pi = 3.14159265358979;
    double g = hull_vol - mesh_vol; if (g < 0.0) g = 0.0;
    return (float)(0.3 * cbrt((3.0 / (4.0 * pi)) * g));
}
