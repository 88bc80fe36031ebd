/* Test driver for the reference's own concave-edge plane kernel.
 *
 * TEST INFRASTRUCTURE ONLY: tests/golden/make_ref_gpu.py loads this library
 * (built by Makefile.ref into oracle/_ref/ref_concave.so together with the
 * reference's unmodified csrc/heap.c) on a B200 to record which planes the
 * reference's la_find_concave_edges (cuda/la_concave.cu:48-363) emits for a
 * mesh.  The context comes from the reference's gpu_init (csrc/heap.c:59-220:
 * fatbin module, device pool, heap_init_kernel); this file only sets up the
 * one-part decomposition state the kernel reads and launches it the way the
 * reference's search does (csrc/lookahead.c:520-531: one 32-thread block per
 * cutting part).
 */
#include <stdint.h>
#include <string.h>
#include <cuda.h>
#include "heap.h"
#include "structs.h"

/* The kernel reads only decomp->parts[cutting_indices[i]], and a
 * LaDecompState starts with its part table (cuda/structs.cuh:73-78), so a
 * one-part table stands in for the whole state. */
int ref_concave_planes(gpu_ctx_t ctx, const float* verts, int nv, const int* tris, int nt,
                       int n_concave_edges, float concave_eps, float concave_threshold,
                       float* out_planes, int* out_n, int* out_err)
{
    struct gpu_ctx* c = (struct gpu_ctx*)ctx;
    CUdeviceptr d_v = 0, d_t = 0, d_part = 0, d_idx = 0, d_planes = 0, d_n = 0, d_err = 0;
    const size_t plane_bytes = (size_t)4 * n_concave_edges * 4 * sizeof(float);
    CUresult r = CUDA_SUCCESS;
    struct Part_h part;
    int zero = 0, n = 0, err = 0;
    *out_n = 0;
    *out_err = 0;
    if (nv <= 0 || nt <= 0 || n_concave_edges <= 0) return 0;
    if ((r = cuMemAlloc(&d_v, 12 * (size_t)nv)) != CUDA_SUCCESS) goto done;
    if ((r = cuMemAlloc(&d_t, 12 * (size_t)nt)) != CUDA_SUCCESS) goto done;
    if ((r = cuMemAlloc(&d_part, sizeof(struct Part_h))) != CUDA_SUCCESS) goto done;
    if ((r = cuMemAlloc(&d_idx, sizeof(int))) != CUDA_SUCCESS) goto done;
    if ((r = cuMemAlloc(&d_planes, plane_bytes)) != CUDA_SUCCESS) goto done;
    if ((r = cuMemAlloc(&d_n, sizeof(int))) != CUDA_SUCCESS) goto done;
    if ((r = cuMemAlloc(&d_err, sizeof(int))) != CUDA_SUCCESS) goto done;
    if ((r = cuMemcpyHtoD(d_v, verts, 12 * (size_t)nv)) != CUDA_SUCCESS) goto done;
    if ((r = cuMemcpyHtoD(d_t, tris, 12 * (size_t)nt)) != CUDA_SUCCESS) goto done;
    memset(&part, 0, sizeof(part));
    part.mesh.verts = d_v; part.mesh.tris = d_t; part.mesh.nv = nv; part.mesh.nt = nt;
    if ((r = cuMemcpyHtoD(d_part, &part, sizeof(part))) != CUDA_SUCCESS) goto done;
    if ((r = cuMemcpyHtoD(d_idx, &zero, sizeof(int))) != CUDA_SUCCESS) goto done;
    if ((r = cuMemsetD8(d_planes, 0, plane_bytes)) != CUDA_SUCCESS) goto done;
    if ((r = cuMemcpyHtoD(d_n, &zero, sizeof(int))) != CUDA_SUCCESS) goto done;
    if ((r = cuMemcpyHtoD(d_err, &zero, sizeof(int))) != CUDA_SUCCESS) goto done;
    {
        int n_cutting = 1;
        CUdeviceptr d_pool = c->d_pool_struct;
        void* args[] = { &d_part, &d_idx, &n_cutting, &n_concave_edges, &concave_eps, &concave_threshold,
                         &d_planes, &d_n, &d_pool, &d_err };
        if ((r = cuLaunchKernel(c->fn_la_find_concave_edges, 1, 1, 1, 32, 1, 1, 0, NULL, args, NULL)) != CUDA_SUCCESS)
            goto done;
    }
    if ((r = cuCtxSynchronize()) != CUDA_SUCCESS) goto done;
    if ((r = cuMemcpyDtoH(&n, d_n, sizeof(int))) != CUDA_SUCCESS) goto done;
    if ((r = cuMemcpyDtoH(&err, d_err, sizeof(int))) != CUDA_SUCCESS) goto done;
    if (n < 0) n = 0;
    if (n > 4 * n_concave_edges) n = 4 * n_concave_edges;
    if (n > 0 && (r = cuMemcpyDtoH(out_planes, d_planes, (size_t)n * 4 * sizeof(float))) != CUDA_SUCCESS) goto done;
    *out_n = n;
    *out_err = err;
done:
    if (d_v) cuMemFree(d_v);
    if (d_t) cuMemFree(d_t);
    if (d_part) cuMemFree(d_part);
    if (d_idx) cuMemFree(d_idx);
    if (d_planes) cuMemFree(d_planes);
    if (d_n) cuMemFree(d_n);
    if (d_err) cuMemFree(d_err);
    return (int)r;
}
