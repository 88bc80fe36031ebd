/*
 * cuacd_b200_diag.h -- diagnostic entry points of libcuacd_b200.so, kept out
 * of the drop-in ABI of cuacd_b200.h: kernel work counters and phase
 * timers, a benchmark of the device arena, the scorer's GEMM staging
 * counters and the remesh's marching-cubes case table.  None has a
 * counterpart in the reference's host layer except where stated; the
 * library's benchmarks and tests use them.
 */
#ifndef CUACD_B200_DIAG_H
#define CUACD_B200_DIAG_H

#include "cuacd_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Diagnostic: allocation throughput of the device arena that replaces the
 * reference's device heap (heap_alloc/heap_free, cuda/allocator.cuh:110-362),
 * on the workload of its heap benchmark (bench/malloc_test_bench.cu:76-125):
 * `grid` blocks, thread 0 of each makes `iters` allocations of log-uniform
 * sizes in [size_min, size_max] into `slots` per-block slots.  The arena
 * frees by whole-arena reset, once per run (arena_bytes of pool).  Reports
 * the mean and deviation of the kernel time over `measure` runs after
 * `warmup`, and the allocations of the last run that did not fit. */
int cuacd_arena_bench(gpu_ctx_t ctx, int grid, int iters, int slots, unsigned size_min, unsigned size_max,
                      unsigned long long arena_bytes, int warmup, int measure, float* out_mean_ms,
                      float* out_std_ms, int* out_fail);

/* Diagnostic: exact hulls of a batch of clouds (host pointers) with the
 * hull kernels' work counters, 8 per cloud: BVH leaves kept by the wraps,
 * wraps, faces, points tested by the wraps, SM cycles spent in set-up (sort,
 * BVH, first face), device clock (ns) when the wrapping took the cloud's
 * first edge and when it finished, large faces (+ 2^32 per wrap on the
 * cloud's own node lists, + 2^48 per face built in its own buffers).  For a
 * cloud whose construction failed, slots 4-7 instead hold the first failure
 * as pairs of 32-bit values (low, high): (site, u), (v, c), (coplanar count,
 * corner count), and for a failed wrap the input indices of u and v. */
int cuacd_hull_stats(gpu_ctx_t ctx, const float* pts, int total_pts,
                     const int* offsets, int n_hulls, int* out_nv, int* out_nt,
                     float* out_vol, unsigned long long* out_stats);

/* Diagnostic (no counterpart in the reference): cut one mesh by n_planes
 * planes and report 8 ints per plane: crossing edges, boundary edges, cap
 * loops, cap triangles, and the SM cycles / 64 spent in the crossing,
 * split, boundary and cap+output phases of the cut kernel. */
int cuacd_cut_stats(gpu_ctx_t ctx, const float* verts, int nv, const int* tris, int nt,
                    const float* planes, int n_planes, int* out_stats);

/* Diagnostic (no counterpart in the reference): scorer GEMM launches so far
 * in this process, by how their A operand reached shared memory -- by TMA
 * (a K-major contiguous A whose tensor map the CUDA driver accepted) or by the
 * CTA's own copies (strided or broadcast operands). */
void cuacd_scorer_gemm_counts(unsigned long long* tma, unsigned long long* staged);

/* The remesh's marching-cubes case table (no counterpart in the reference,
 * which contours with a dual method): per case, 17 ints -- the number of
 * loops, four loop lengths, twelve cube edges (loops one after another, -1
 * padded).  Host only; for checking the table. */
void cuacd_remesh_case_table(int* out);

#ifdef __cplusplus
}
#endif
#endif
