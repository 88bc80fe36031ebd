// components.cu — connected-components kernel, its launcher for the
// lookahead, and the gpu_test_postprocess_dc entry point (csrc/postprocess.h:20-27).
#include <vector>
#include <cstring>
#include "context.cuh"
#include "components.cuh"
#include "hausdorff.cuh"
#include "launch.h"

// Connected components of meshes 0..n, one CTA each.
__global__ void __launch_bounds__(CC_BLOCK)
k_components(const HDSurf* __restrict__ meshes, int n, Arena* scratch, Arena* out, CompResult* res)
{
    const int i = blockIdx.x;
    if (i >= n) return;
    const HDSurf m = meshes[i];
    components_cta(m.v, m.nv, m.t, m.nt, scratch, out, &res[i]);
}

void launch_components(const HDSurf* d_meshes, int n, Arena* scratch, Arena* out, CompResult* res, cudaStream_t s)
{
    if (n > 0) k_components<<<n, CC_BLOCK, 0, s>>>(d_meshes, n, scratch, out, res);
}

// Output layout of the reference's test entry: component c's vertices at
// out_verts[c*max_verts_per*3 ...], triangles at out_tris[c*max_tris_per*3 ...].
// A mesh that is one component comes back unchanged as component 0.
extern "C" int gpu_test_postprocess_dc(gpu_ctx_t ctx, const float* verts, int n_verts, const int* tris, int n_tris,
                                       int max_components, int max_verts_per, int max_tris_per,
                                       float* out_verts, int* out_tris, int* out_nv, int* out_nt,
                                       int* out_n_components)
{
    if (!ctx || !out_n_components) return -1;
    *out_n_components = 0;
    if (n_verts < 0 || n_tris < 0 || max_components < 0 || max_verts_per < 0 || max_tris_per < 0)
        return ctx_fail(ctx, KERR_MESH_INVALID, "negative size");
    for (int i = 0; i < 3 * n_tris; i++)
        if (tris[i] < 0 || tris[i] >= n_verts) return ctx_fail(ctx, KERR_MESH_INVALID, "triangle index out of range");
    if (n_verts == 0 || n_tris == 0) return 0;
    CK(cudaSetDevice(ctx->device));
    const size_t scr_bytes = cc_scratch_bytes(n_verts), out_bytes = cc_output_bytes(n_verts, n_tris);
    const size_t need = al256(12 * (size_t)n_verts) + al256(12 * (size_t)n_tris) + al256(sizeof(HDSurf))
                      + al256(sizeof(CompResult)) + al256(2 * sizeof(Arena)) + al256(scr_bytes) + al256(out_bytes);
    int rc = pool_begin(ctx, need);
    if (rc) return rc;
    float* d_v = pool_take<float>(ctx, 3 * (size_t)n_verts);
    int* d_t = pool_take<int>(ctx, 3 * (size_t)n_tris);
    HDSurf* d_m = pool_take<HDSurf>(ctx, 1);
    CompResult* d_res = pool_take<CompResult>(ctx, 1);
    Arena* d_ar = pool_take<Arena>(ctx, 2);
    char* scr = pool_take<char>(ctx, scr_bytes);
    char* outb = pool_take<char>(ctx, out_bytes);
    if (!outb) return ctx_fail(ctx, KERR_HEAP_OOM, "pool carve failed");
    cudaStream_t s = ctx->stream;
    HDSurf m = {d_v, d_t, n_verts, n_tris};
    CK(cudaMemcpyAsync(d_v, verts, 12 * (size_t)n_verts, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(d_t, tris, 12 * (size_t)n_tris, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(d_m, &m, sizeof(m), cudaMemcpyHostToDevice, s));
    launch_arena_reset(d_ar, scr, scr_bytes, s);
    launch_arena_reset(d_ar + 1, outb, out_bytes, s);
    launch_components(d_m, 1, d_ar, d_ar + 1, d_res, s);
    ctx->launches += 3;
    CK(cudaGetLastError());
    CompResult r;
    CK(cudaMemcpyAsync(&r, d_res, sizeof(r), cudaMemcpyDeviceToHost, s));
    rc = sync_and_check(ctx, "postprocess_dc");
    if (rc) return rc;
    if (r.err) return ctx_fail(ctx, r.err, "postprocess_dc failed (error word 0x%x)", r.err);
    if (r.n <= 0) {                                   // one component: the input itself
        if (max_components < 1 || n_verts > max_verts_per || n_tris > max_tris_per)
            return ctx_fail(ctx, KERR_DC_OOM, "output buffers too small for 1 component of %d/%d", n_verts, n_tris);
        memcpy(out_verts, verts, 12 * (size_t)n_verts);
        memcpy(out_tris, tris, 12 * (size_t)n_tris);
        out_nv[0] = n_verts; out_nt[0] = n_tris;
        *out_n_components = 1;
        return 0;
    }
    if (r.n > max_components) return ctx_fail(ctx, KERR_DC_OOM, "%d components, room for %d", r.n, max_components);
    std::vector<CompMesh> cm(r.n);
    CK(cudaMemcpy(cm.data(), r.comps, sizeof(CompMesh) * r.n, cudaMemcpyDeviceToHost));
    for (int c = 0; c < r.n; c++) {
        if (cm[c].nv > max_verts_per || cm[c].nt > max_tris_per)
            return ctx_fail(ctx, KERR_DC_OOM, "component %d has %d/%d vertices/triangles, room for %d/%d",
                            c, cm[c].nv, cm[c].nt, max_verts_per, max_tris_per);
    }
    for (int c = 0; c < r.n; c++) {
        CK(cudaMemcpyAsync(out_verts + 3 * (size_t)c * max_verts_per, cm[c].v, 12 * (size_t)cm[c].nv,
                           cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(out_tris + 3 * (size_t)c * max_tris_per, cm[c].t, 12 * (size_t)cm[c].nt,
                           cudaMemcpyDeviceToHost, s));
        out_nv[c] = cm[c].nv; out_nt[c] = cm[c].nt;
    }
    CK(cudaStreamSynchronize(s));
    *out_n_components = r.n;
    return 0;
}
