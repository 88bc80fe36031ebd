// cut.cu — plane-cut kernels (built with -fmad=false, see cut.cuh) and the
// gpu_test_plane_cut entry point.
#include <vector>
#include "context.cuh"
#include "cut.cuh"
#include "launch.h"

// One cut of one mesh into caller-sized buffers.
__global__ void __launch_bounds__(CUT_NT)
k_cut_one(const float* __restrict__ v, int nv, const int* __restrict__ t, int nt, float4 plane,
          Arena* arena, CutFixedOut fixed, CutResult* res)
{
    __shared__ CutShared sh;
    cut_cta(v, nv, t, nt, plane.x, plane.y, plane.z, plane.w, arena, fixed, res, sh);
}

// Many planes on one mesh; fragments go to the arena.  Degenerate planes
// (all-zero normal) produce an empty result.
__global__ void __launch_bounds__(CUT_NT, 1)
k_cut_planes(const float* __restrict__ v, int nv, const int* __restrict__ t, int nt,
             const float4* __restrict__ planes, int n_planes, Arena* arena, CutResult* res)
{
    __shared__ CutShared sh;
    int i = blockIdx.x;
    if (i >= n_planes) return;
    float4 p = planes[i];
    if (p.x == 0.f && p.y == 0.f && p.z == 0.f) {
        if (threadIdx.x == 0) memset(&res[i], 0, sizeof(CutResult));
        return;
    }
    CutFixedOut none;
    memset(&none, 0, sizeof(none));
    cut_cta(v, nv, t, nt, p.x, p.y, p.z, p.w, arena, none, &res[i], sh);
}

size_t cut_scratch_bytes(int nv, int nt)
{
    size_t occ = 1; while (occ < (size_t)2 * nt + 1) occ <<= 1;
    size_t b = 0;
    b += al256(nv) + al256(8 * occ) + 2 * al256(4 * occ) + al256(8 * occ) + 2 * al256(4 * occ);
    b += al256(12 * ((size_t)nv + occ)) + 2 * al256(4 * (size_t)nt);
    b += 2 * al256(12 * ((size_t)2 * nt + 8));                        // side triangles
    b += 2 * al256(8 * (occ * 4));                                    // boundary keys (bounded by 6*n_pos edges)
    b += al256(4 * (4 * occ + 6 * (occ * 4 + 64)));                   // loops / polygons / caps
    b += 2 * al256(4 * ((size_t)nv + occ));                           // remap + used
    b += 2 * (al256(12 * ((size_t)nv + occ)) + al256(12 * ((size_t)2 * nt + 8 + 4 * occ)));  // outputs
    return b + 64 * 256;
}

void launch_cut_planes(const float* v, int nv, const int* t, int nt, const float4* planes, int n_planes,
                       Arena* arena, CutResult* res, cudaStream_t s)
{
    if (n_planes > 0) k_cut_planes<<<n_planes, CUT_NT, 0, s>>>(v, nv, t, nt, planes, n_planes, arena, res);
}

extern "C" int gpu_test_plane_cut(gpu_ctx_t ctx, const float* vertices, int n_verts, const int* triangles, int n_tris,
                                  float pa, float pb, float pc_n, float pd,
                                  float* out_pos_verts, int out_pos_verts_cap, int* out_pos_tris, int out_pos_tris_cap,
                                  float* out_neg_verts, int out_neg_verts_cap, int* out_neg_tris, int out_neg_tris_cap,
                                  int* out_n_pv, int* out_n_pt, int* out_n_nv, int* out_n_nt)
{
    if (!ctx) return -1;
    if (n_verts < 0 || n_tris < 0) return ctx_fail(ctx, KERR_MESH_INVALID, "negative mesh size");
    for (int i = 0; i < 3 * n_tris; i++)
        if (triangles[i] < 0 || triangles[i] >= n_verts)
            return ctx_fail(ctx, KERR_MESH_INVALID, "triangle index out of range");
    CK(cudaSetDevice(ctx->device));
    size_t need = al256(12 * (size_t)n_verts) + al256(12 * (size_t)n_tris)
                + al256(12 * (size_t)out_pos_verts_cap) + al256(12 * (size_t)out_pos_tris_cap)
                + al256(12 * (size_t)out_neg_verts_cap) + al256(12 * (size_t)out_neg_tris_cap)
                + al256(sizeof(CutResult)) + cut_scratch_bytes(n_verts, n_tris);
    int rc = pool_begin(ctx, need);
    if (rc) return rc;
    float* d_v = pool_take<float>(ctx, 3 * (size_t)n_verts);
    int* d_t = pool_take<int>(ctx, 3 * (size_t)n_tris);
    CutFixedOut f;
    f.pv = pool_take<float>(ctx, 3 * (size_t)out_pos_verts_cap); f.pv_cap = out_pos_verts_cap;
    f.pt = pool_take<int>(ctx, 3 * (size_t)out_pos_tris_cap);   f.pt_cap = out_pos_tris_cap;
    f.nv = pool_take<float>(ctx, 3 * (size_t)out_neg_verts_cap); f.nv_cap = out_neg_verts_cap;
    f.nt = pool_take<int>(ctx, 3 * (size_t)out_neg_tris_cap);   f.nt_cap = out_neg_tris_cap;
    CutResult* d_res = pool_take<CutResult>(ctx, 1);
    cudaStream_t s = ctx->stream;
    if (n_verts) CK(cudaMemcpyAsync(d_v, vertices, 12 * (size_t)n_verts, cudaMemcpyHostToDevice, s));
    if (n_tris) CK(cudaMemcpyAsync(d_t, triangles, 12 * (size_t)n_tris, cudaMemcpyHostToDevice, s));
    launch_arena_reset(ctx->d_arena, ctx->pool + ctx->carve, ctx->cap - ctx->carve, s);
    k_cut_one<<<1, CUT_NT, 0, s>>>(d_v, n_verts, d_t, n_tris, make_float4(pa, pb, pc_n, pd), ctx->d_arena, f, d_res);
    ctx->launches += 2;
    CK(cudaGetLastError());
    CutResult r;
    CK(cudaMemcpyAsync(&r, d_res, sizeof(CutResult), cudaMemcpyDeviceToHost, s));
    rc = sync_and_check(ctx, "plane_cut");
    if (rc) return rc;
    if (r.err) return ctx_fail(ctx, r.err, "plane cut failed (error word 0x%x)", r.err);
    if (r.npv) CK(cudaMemcpy(out_pos_verts, r.pv, 12 * (size_t)r.npv, cudaMemcpyDeviceToHost));
    if (r.npt) CK(cudaMemcpy(out_pos_tris, r.pt, 12 * (size_t)r.npt, cudaMemcpyDeviceToHost));
    if (r.nnv) CK(cudaMemcpy(out_neg_verts, r.nv, 12 * (size_t)r.nnv, cudaMemcpyDeviceToHost));
    if (r.nnt) CK(cudaMemcpy(out_neg_tris, r.nt, 12 * (size_t)r.nnt, cudaMemcpyDeviceToHost));
    *out_n_pv = r.npv; *out_n_pt = r.npt; *out_n_nv = r.nnv; *out_n_nt = r.nnt;
    return 0;
}

// Diagnostic: cut one mesh by n planes (k_cut_planes, fragments into the
// arena) and report per plane 8 ints: crossing edges, boundary edges, loops,
// cap triangles, then SM cycles / 64 of the crossing, split, boundary and
// cap+output phases.
extern "C" int cuacd_cut_stats(gpu_ctx_t ctx, const float* verts, int nv, const int* tris, int nt,
                               const float* planes, int n_planes, int* out_stats)
{
    if (!ctx) return -1;
    if (n_planes <= 0) return 0;
    if (nv <= 0 || nt <= 0) return ctx_fail(ctx, KERR_MESH_INVALID, "empty mesh");
    for (int i = 0; i < 3 * nt; i++)
        if (tris[i] < 0 || tris[i] >= nv) return ctx_fail(ctx, KERR_MESH_INVALID, "triangle index out of range");
    CK(cudaSetDevice(ctx->device));
    size_t need = al256(12 * (size_t)nv) + al256(12 * (size_t)nt) + al256(16 * (size_t)n_planes)
                + al256(sizeof(CutResult) * (size_t)n_planes) + cut_scratch_bytes(nv, nt) * (size_t)n_planes;
    int rc = pool_begin(ctx, need);
    if (rc) return rc;
    float* d_v = pool_take<float>(ctx, 3 * (size_t)nv);
    int* d_t = pool_take<int>(ctx, 3 * (size_t)nt);
    float4* d_p = pool_take<float4>(ctx, n_planes);
    CutResult* d_res = pool_take<CutResult>(ctx, n_planes);
    if (!d_res) return ctx_fail(ctx, KERR_HEAP_OOM, "pool carve failed");
    cudaStream_t s = ctx->stream;
    CK(cudaMemcpyAsync(d_v, verts, 12 * (size_t)nv, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(d_t, tris, 12 * (size_t)nt, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(d_p, planes, 16 * (size_t)n_planes, cudaMemcpyHostToDevice, s));
    launch_arena_reset(ctx->d_arena, ctx->pool + ctx->carve, ctx->cap - ctx->carve, s);
    launch_cut_planes(d_v, nv, d_t, nt, d_p, n_planes, ctx->d_arena, d_res, s);
    ctx->launches += 2;
    CK(cudaGetLastError());
    std::vector<CutResult> r(n_planes);
    CK(cudaMemcpyAsync(r.data(), d_res, sizeof(CutResult) * n_planes, cudaMemcpyDeviceToHost, s));
    rc = sync_and_check(ctx, "cut_stats");
    if (rc) return rc;
    for (int i = 0; i < n_planes; i++) {
        int* o = out_stats + 8 * i;
        o[0] = r[i].n_cross; o[1] = r[i].n_boundary; o[2] = r[i].n_loops; o[3] = r[i].n_cap;
        for (int k = 0; k < 4; k++) o[4 + k] = (int)r[i].cyc[k];
    }
    return 0;
}
