// eval.cu — candidate evaluator: for each plane, cut the mesh with caps,
// compute both fragments' volumes and exact hulls, optionally the sampled
// Hausdorff distance fragment<->hull, and the part costs of
// cuda/la_common.cuh:21-34.  This is the per-candidate scorer of the
// reference's la_expand (cuda/la_expand.cu:65-340) + la_hull
// (:357-424) + la_hausdorff_parts (cuda/la_refine.cu:19-45), as one
// device-resident pipeline with no host round trip:
//   k_cut_planes  (cut.cu)   one CTA per plane, fragments into the arena
//   hull pipeline (hull.cu)  volume + exact hull of every fragment
//   Hausdorff prep/plan/query (hausdorff.cu), pairs (hull, fragment)
//   k_eval_finish            costs and the per-candidate record
#include <algorithm>
#include <cstdlib>
#include "context.cuh"
#include "hull.cuh"
#include "cut.cuh"
#include "hausdorff.cuh"
#include "launch.h"

typedef HullRes FragInfo;     // per fragment: hull, mesh and hull volume, error

// Hull jobs for both fragments of every candidate (empty when the cut failed
// or left one side empty).  The fragment's triangles give its mesh volume.
__global__ void k_frag_jobs(const CutResult* __restrict__ cuts, int n_cand, HullJob* jobs)
{
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= 2 * n_cand) return;
    const CutResult& C = cuts[f >> 1];
    const int side = f & 1;
    const bool empty = C.err != 0 || C.npv <= 0 || C.nnv <= 0;
    HullJob J;
    memset(&J, 0, sizeof(J));
    if (!empty) {
        J.pts = side ? C.nv : C.pv; J.n = side ? C.nnv : C.npv;
        J.tris = side ? C.nt : C.pt; J.nt = side ? C.nnt : C.npt;
    }
    jobs[f] = J;
}

// surfaces for the Hausdorff pairs: pair f = (hull of fragment f, fragment f)
__global__ void k_make_surfs(const CutResult* __restrict__ cuts, const FragInfo* __restrict__ frags, int n_frag,
                             HDSurf* surfs)
{
    int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= n_frag) return;
    const CutResult& C = cuts[f >> 1];
    const FragInfo& F = frags[f];
    bool ok = F.err == 0 && F.hnt > 0 && C.npv > 0 && C.nnv > 0;
    HDSurf A = {F.hv, F.ht, ok ? F.hnv : 0, ok ? F.hnt : 0};
    HDSurf B;
    if (f & 1) { B.v = C.nv; B.t = C.nt; B.nv = ok ? C.nnv : 0; B.nt = ok ? C.nnt : 0; }
    else       { B.v = C.pv; B.t = C.pt; B.nv = ok ? C.npv : 0; B.nt = ok ? C.npt : 0; }
    surfs[2 * f] = A;
    surfs[2 * f + 1] = B;
}

// The same pairs built in two steps, so that the fragments' Hausdorff prep
// can start before their hulls exist: the fragment surfaces (2f+1) from the
// cut alone, then the hull surfaces (2f) -- empty when the hull failed, which
// leaves the pair without queries, as k_make_surfs does.
__global__ void k_make_frag_surfs(const CutResult* __restrict__ cuts, int n_frag, HDSurf* surfs)
{
    int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= n_frag) return;
    const CutResult& C = cuts[f >> 1];
    const bool ok = C.err == 0 && C.npv > 0 && C.nnv > 0;
    HDSurf B;
    if (f & 1) { B.v = C.nv; B.t = C.nt; B.nv = ok ? C.nnv : 0; B.nt = ok ? C.nnt : 0; }
    else       { B.v = C.pv; B.t = C.pt; B.nv = ok ? C.npv : 0; B.nt = ok ? C.npt : 0; }
    surfs[2 * f + 1] = B;
}

__global__ void k_make_hull_surfs(const CutResult* __restrict__ cuts, const FragInfo* __restrict__ frags, int n_frag,
                                  HDSurf* surfs)
{
    int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= n_frag) return;
    const CutResult& C = cuts[f >> 1];
    const FragInfo& F = frags[f];
    const bool ok = F.err == 0 && F.hnt > 0 && C.npv > 0 && C.nnv > 0;
    HDSurf A = {F.hv, F.ht, ok ? F.hnv : 0, ok ? F.hnt : 0};
    surfs[2 * f] = A;
}

__global__ void k_eval_finish(const CutResult* __restrict__ cuts, const FragInfo* __restrict__ frags,
                              const float* __restrict__ hd, int n_cand, int with_hd, const int* arena_err,
                              cuacd_cand_result* out)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_cand) return;
    const CutResult& C = cuts[i];
    cuacd_cand_result r;
    memset(&r, 0, sizeof(r));
    r.err = C.err | frags[2 * i].err | frags[2 * i + 1].err | (arena_err ? *arena_err : 0);
    r.ok = (r.err == 0 && C.npv > 0 && C.nnv > 0) ? 1 : 0;
    r.nv[0] = C.npv; r.nv[1] = C.nnv; r.nt[0] = C.npt; r.nt[1] = C.nnt;
    r.n_cap = C.n_cap;
    if (r.ok) {
        float worst_rv = 0.f, worst_full = 0.f;
        for (int s = 0; s < 2; s++) {
            const FragInfo& F = frags[2 * i + s];
            r.hull_nv[s] = F.hnv; r.hull_nt[s] = F.hnt;
            r.mesh_vol[s] = (float)F.mesh_vol; r.hull_vol[s] = F.hull_vol;
            float h = with_hd ? hd[2 * i + s] : 0.f;
            r.hausdorff[s] = h;
            r.cost_rv[s] = part_cost_rv((double)F.hull_vol, F.mesh_vol);
            r.cost_full[s] = fmaxf(r.cost_rv[s], h);
            worst_rv = fmaxf(worst_rv, r.cost_rv[s]);
            worst_full = fmaxf(worst_full, r.cost_full[s]);
        }
        r.score_rv = worst_rv; r.score_full = worst_full;
    }
    out[i] = r;
}

// cuts[pos[i]] = all[i] for every plane i a selection kept (pos[i] >= 0).
__global__ void k_gather_cuts(const CutResult* __restrict__ all, const int* __restrict__ pos, int n,
                              CutResult* __restrict__ cuts)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int j = pos[i];
    if (j >= 0) cuts[j] = all[i];
}

// ---------------------------------------------------------------------------
// workspace and launch sequence (shared by the host and device entry points)
// ---------------------------------------------------------------------------
struct EvalWork {
    float4* planes; CutResult* cuts; FragInfo* frags; HDSurf* surfs; HDPrep* preps;
    char* dirs; int* i4; float* pmax; float* hd;
    HullJob* jobs; HullState* states; int* hctl; int* wbuf; int nwc;
    int max_pts;                       // largest fragment possible: the parent's vertex count
};

static size_t eval_fixed_bytes(int n, int nwc)
{
    return al256(sizeof(float4) * n) + al256(sizeof(CutResult) * n) + al256(sizeof(FragInfo) * 2 * n)
         + al256(sizeof(HDSurf) * 4 * n) + al256(sizeof(HDPrep) * 4 * n) + al256(hd_dir_bytes() * 4 * n)
         + al256(sizeof(int) * 4) + 2 * al256(sizeof(float) * 2 * n)
         + al256(sizeof(HullJob) * 2 * n) + al256(sizeof(HullState) * 2 * n) + al256(64)
         + al256(hull_wrap_buf_bytes(nwc));
}

static int eval_wrap_ctas(gpu_ctx* ctx, int nv, int n)
{
    return hull_wrap_ctas(2LL * n * nv, ctx->n_sm, nv);
}

static size_t eval_arena_bytes(int nv, int nt, int n)
{
    // per candidate: cut scratch + fragments; per fragment: hull scratch and
    // output, two Hausdorff preps (hull and fragment)
    int fv = nv + nv / 2 + 64, ft = nt + nt / 2 + 64;
    size_t per = cut_scratch_bytes(nv, nt)
               + 2 * (al256(hull_scratch_bytes(fv)) + al256(12 * (size_t)fv) + al256(12 * (size_t)(2 * fv + 4)))
               + 2 * (al256(hd_prep_bytes(2 * fv)) + al256(hd_prep_bytes(ft)))
               + 64 * 1024;
    return per * (size_t)n;
}

static int eval_take(gpu_ctx* ctx, int n, int nwc, EvalWork& W, int max_pts)
{
    W.max_pts = max_pts;
    W.nwc = nwc;
    W.jobs = pool_take<HullJob>(ctx, 2 * n);
    W.states = pool_take<HullState>(ctx, 2 * n);
    W.hctl = pool_take<int>(ctx, 16);
    W.wbuf = (int*)pool_take<char>(ctx, hull_wrap_buf_bytes(nwc));
    W.planes = pool_take<float4>(ctx, n);
    W.cuts = pool_take<CutResult>(ctx, n);
    W.frags = pool_take<FragInfo>(ctx, 2 * n);
    W.surfs = pool_take<HDSurf>(ctx, 4 * n);
    W.preps = pool_take<HDPrep>(ctx, 4 * n);
    W.dirs = pool_take<char>(ctx, hd_dir_bytes() * 4 * n);
    W.i4 = pool_take<int>(ctx, 4);
    W.pmax = pool_take<float>(ctx, 2 * n);
    W.hd = pool_take<float>(ctx, 2 * n);
    return W.hd ? 0 : -1;
}

static int sm_count_dev(int dev)
{
    int n = 148;
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    return n > 0 ? n : 148;
}

static int eval_aux_ready(gpu_ctx* ctx, int G);

// The stages after the cut (hulls, Hausdorff, part costs) of n planes whose
// cut results are in W.cuts, on stream s.
static void eval_launch_after_cut(gpu_ctx* ctx, int n, int flags, float res, int mins, int total, EvalWork& W,
                                  cuacd_cand_result* d_out, cudaStream_t s, bool may_overlap)
{
    auto mark = [&](int i) { if (ctx->profile) { cudaEventRecord(ctx->ev[i], s); ctx->n_ev = i + 1; } };
    const bool hd = flags & CUACD_EVAL_HAUSDORFF;
    // Outside stage profiling (whose events describe one serial pipeline),
    // the fragments' Hausdorff prep runs on a second stream beside the hull
    // pipeline: it needs only the cut.
    const bool overlap = hd && may_overlap && !ctx->profile && eval_aux_ready(ctx, 3) == 0;
    k_frag_jobs<<<(2 * n + 127) / 128, 128, 0, s>>>(W.cuts, n, W.jobs);
    if (overlap) {
        cudaStream_t a = ctx->aux[1];
        k_make_frag_surfs<<<(2 * n + 127) / 128, 128, 0, s>>>(W.cuts, 2 * n, W.surfs);
        cudaEventRecord(ctx->fork_ev, s);
        cudaStreamWaitEvent(a, ctx->fork_ev, 0);
        launch_hd_prep_subset(W.surfs, 2 * n, 1, 2, ctx->d_arena, res, mins, total, W.preps, W.i4 + 2, a);
        cudaEventRecord(ctx->join_ev[1], a);
        ctx->launches += 2;
    }
    launch_hull_jobs(W.jobs, 2 * n, W.states, W.frags, ctx->d_arena, ctx->d_arena, W.hctl, W.wbuf, W.nwc,
                     nullptr, s, W.max_pts);
    mark(2);
    ctx->launches += 6;
    if (hd && overlap) {
        k_make_hull_surfs<<<(2 * n + 127) / 128, 128, 0, s>>>(W.cuts, W.frags, 2 * n, W.surfs);
        launch_hd_prep_subset(W.surfs, 2 * n, 0, 2, ctx->d_arena, res, mins, total, W.preps, W.i4 + 2, s);
        cudaStreamWaitEvent(s, ctx->join_ev[1], 0);
        launch_hd_plan_query(W.surfs, 2 * n, W.preps, W.dirs, W.i4, W.pmax, sm_count_dev(ctx->device), s,
                             [](int) {});
        launch_hd_sqrt(W.pmax, 2 * n, W.hd, 1, s);
        ctx->launches += 5;
    } else if (hd) {
        k_make_surfs<<<(2 * n + 127) / 128, 128, 0, s>>>(W.cuts, W.frags, 2 * n, W.surfs);
        launch_hausdorff_stages(W.surfs, 2 * n, ctx->d_arena, res, mins, total, W.preps, W.dirs, W.i4, W.pmax,
                                W.i4 + 2, sm_count_dev(ctx->device), s, [&](int k) { mark(3 + k); });
        launch_hd_sqrt(W.pmax, 2 * n, W.hd, 1, s);
        ctx->launches += 5;
    } else { mark(3); mark(4); mark(5); }
    k_eval_finish<<<(n + 127) / 128, 128, 0, s>>>(W.cuts, W.frags, W.hd, n, hd ? 1 : 0, W.i4 + 2, d_out);
    mark(6);
    ctx->launches += 1;
}

// All launches of one evaluation of n planes (already in W.planes) on
// stream s.  The caller resets the arena first.
static void eval_launch(gpu_ctx* ctx, const float* d_v, int nv, const int* d_t, int nt, int n, int flags,
                        float res, int mins, int total, EvalWork& W, cuacd_cand_result* d_out, cudaStream_t s,
                        bool may_overlap)
{
    auto mark = [&](int i) { if (ctx->profile) { cudaEventRecord(ctx->ev[i], s); ctx->n_ev = i + 1; } };
    cudaMemsetAsync(W.i4, 0, 4 * sizeof(int), s);
    mark(0);
    launch_cut_planes(d_v, nv, d_t, nt, W.planes, n, ctx->d_arena, W.cuts, s);
    mark(1);
    eval_launch_after_cut(ctx, n, flags, res, mins, total, W, d_out, s, may_overlap);
}

// ---------------------------------------------------------------------------
// plane groups on concurrent streams (CUACD_EVAL_GROUPS, default 1).  Each
// group's stages run on their own stream with their own work buffers; all
// share the arena, reset once before.  Measured on the 30-plane,
// 40,960-triangle step: 1 group 2,348 candidates/s, 2 groups 1,976, 3 groups
// 1,486, 4 groups 2,028 -- the groups' persistent hull grids and Hausdorff
// queries contend for the SMs, so one group is the default.
// ---------------------------------------------------------------------------
#define EVAL_MAX_GROUPS 4

static int eval_groups(gpu_ctx* ctx, int n)
{
    if (ctx->profile) return 1;                       // stage events describe one serial pipeline
    if (ctx->eval_groups == 0) {                      // CUACD_EVAL_GROUPS overrides the default (1)
        const char* e = getenv("CUACD_EVAL_GROUPS");
        ctx->eval_groups = (e && atoi(e) > 0) ? atoi(e) : 1;
    }
    int g = ctx->eval_groups;
    g = std::min(g, std::min(EVAL_MAX_GROUPS, n / 4));
    return std::max(g, 1);
}

static void group_range(int n, int G, int g, int* o, int* m) { *o = (int)((long long)n * g / G); *m = (int)((long long)n * (g + 1) / G) - *o; }

static size_t eval_groups_fixed_bytes(gpu_ctx* ctx, int nv, int n, int G)
{
    size_t b = 0;
    for (int g = 0; g < G; g++) {
        int o, m; group_range(n, G, g, &o, &m);
        b += eval_fixed_bytes(m, eval_wrap_ctas(ctx, nv, m));
    }
    return b;
}

static int eval_groups_take(gpu_ctx* ctx, int nv, int n, int G, EvalWork* W)
{
    for (int g = 0; g < G; g++) {
        int o, m; group_range(n, G, g, &o, &m);
        if (eval_take(ctx, m, eval_wrap_ctas(ctx, nv, m), W[g], nv)) return -1;
    }
    return 0;
}

static int eval_aux_ready(gpu_ctx* ctx, int G)
{
    if (G > 1 && !ctx->fork_ev) CK(cudaEventCreateWithFlags(&ctx->fork_ev, cudaEventDisableTiming));
    for (int g = 1; g < G; g++) {
        if (!ctx->aux[g - 1]) CK(cudaStreamCreateWithFlags(&ctx->aux[g - 1], cudaStreamNonBlocking));
        if (!ctx->join_ev[g - 1]) CK(cudaEventCreateWithFlags(&ctx->join_ev[g - 1], cudaEventDisableTiming));
    }
    return 0;
}

// Evaluate n planes (device, d_planes) in G groups; results to d_out[0, n).
static int eval_run(gpu_ctx* ctx, const float* d_v, int nv, const int* d_t, int nt, const float4* d_planes, int n,
                    int flags, float res, int mins, int total, EvalWork* W, int G, cuacd_cand_result* d_out,
                    cudaStream_t s)
{
    if (eval_aux_ready(ctx, G)) return -1;
    launch_arena_reset(ctx->d_arena, ctx->pool + ctx->carve, ctx->cap - ctx->carve, s);
    ctx->launches += 1;
    if (G > 1) CK(cudaEventRecord(ctx->fork_ev, s));
    for (int g = 0; g < G; g++) {
        int o, m; group_range(n, G, g, &o, &m);
        cudaStream_t sg = g == 0 ? s : ctx->aux[g - 1];
        if (g > 0) CK(cudaStreamWaitEvent(sg, ctx->fork_ev, 0));
        CK(cudaMemcpyAsync(W[g].planes, d_planes + o, sizeof(float4) * m, cudaMemcpyDeviceToDevice, sg));
        eval_launch(ctx, d_v, nv, d_t, nt, m, flags, res, mins, total, W[g], d_out + o, sg, G == 1);
    }
    for (int g = 1; g < G; g++) {
        CK(cudaEventRecord(ctx->join_ev[g - 1], ctx->aux[g - 1]));
        CK(cudaStreamWaitEvent(s, ctx->join_ev[g - 1], 0));
    }
    CK(cudaGetLastError());
    return 0;
}

// ---------------------------------------------------------------------------
// Evaluation of the planes a selection keeps, with the cut of every plane
// overlapping the selection itself (the surrogate-pruned evaluator): the
// cuts of all n planes run on the context's auxiliary stream while the
// caller ranks the planes on s; then s waits for them, gathers the kept
// planes' cut results and runs the remaining stages on those alone.  The
// cut of a plane does not depend on which others are cut, so every kept
// plane's result equals the one the exact evaluator gives it.
// ---------------------------------------------------------------------------
int eval_precut_begin(gpu_ctx* ctx, const float* d_v, int nv, const int* d_t, int nt, const float4* d_planes, int n,
                      EvalPrecut& P, cudaStream_t s)
{
    P.n = n;
    P.nwc = eval_wrap_ctas(ctx, nv, n);
    if (eval_aux_ready(ctx, 2)) return -1;
    int rc = pool_begin(ctx, eval_fixed_bytes(n, P.nwc) + al256(sizeof(CutResult) * (size_t)n)
                             + eval_arena_bytes(nv, nt, n));
    if (rc) return rc;
    P.W = new EvalWork;
    if (eval_take(ctx, n, P.nwc, *P.W, nv)) return ctx_fail(ctx, KERR_HEAP_OOM, "pool too small");
    P.all_cuts = pool_take<CutResult>(ctx, n);
    if (!P.all_cuts) return ctx_fail(ctx, KERR_HEAP_OOM, "pool too small");
    cudaStream_t a = ctx->aux[0];
    launch_arena_reset(ctx->d_arena, ctx->pool + ctx->carve, ctx->cap - ctx->carve, s);
    CK(cudaMemsetAsync(P.W->i4, 0, 4 * sizeof(int), s));
    CK(cudaEventRecord(ctx->fork_ev, s));
    CK(cudaStreamWaitEvent(a, ctx->fork_ev, 0));
    CK(cudaMemcpyAsync(P.W->planes, d_planes, sizeof(float4) * (size_t)n, cudaMemcpyDeviceToDevice, a));
    launch_cut_planes(d_v, nv, d_t, nt, P.W->planes, n, ctx->d_arena, P.all_cuts, a);
    CK(cudaEventRecord(ctx->join_ev[0], a));
    ctx->launches += 2;
    CK(cudaGetLastError());
    return 0;
}

void eval_precut_release(EvalPrecut& P)
{
    delete P.W;
    P.W = nullptr;
}

int eval_precut_finish(gpu_ctx* ctx, EvalPrecut& P, const int* d_pos, int n_sel, int flags, float res, int mins,
                       int total, cuacd_cand_result* d_out, cudaStream_t s)
{
    CK(cudaStreamWaitEvent(s, ctx->join_ev[0], 0));
    int rc = 0;
    if (n_sel > 0) {
        if (res <= 0.f) res = 2000.f;
        if (mins < 0) mins = 1000;
        k_gather_cuts<<<(P.n + 127) / 128, 128, 0, s>>>(P.all_cuts, d_pos, P.n, P.W->cuts);
        ctx->launches += 1;
        eval_launch_after_cut(ctx, n_sel, flags, res, mins, total, *P.W, d_out, s, true);
        if (cudaGetLastError() != cudaSuccess) rc = ctx_fail(ctx, -1, "pruned evaluation launch failed");
    }
    eval_precut_release(P);
    return rc;
}

extern "C" int cuacd_profile_stages(gpu_ctx_t ctx, int enable)
{
    if (!ctx) return -1;
    CK(cudaSetDevice(ctx->device));
    if (enable && !ctx->ev[0])
        for (int i = 0; i < 8; i++) CK(cudaEventCreate(&ctx->ev[i]));
    ctx->profile = enable ? 1 : 0;
    ctx->n_ev = 0;
    return 0;
}

extern "C" int cuacd_stage_times(gpu_ctx_t ctx, float* ms_out)
{
    if (!ctx || !ms_out) return -1;
    if (ctx->n_ev < CUACD_N_STAGES + 1) return ctx_fail(ctx, -1, "no profiled evaluation recorded");
    CK(cudaEventSynchronize(ctx->ev[CUACD_N_STAGES]));
    for (int i = 0; i < CUACD_N_STAGES; i++) CK(cudaEventElapsedTime(&ms_out[i], ctx->ev[i], ctx->ev[i + 1]));
    return 0;
}

extern "C" int cuacd_eval_candidates_device(gpu_ctx_t ctx, const float* d_verts, int nv, const int* d_tris, int nt,
                                            const float* d_planes, int n_planes, int flags, float hd_resolution,
                                            int hd_min_samples, int hd_total, cuacd_cand_result* d_out, void* stream)
{
    if (!ctx) return -1;
    if (n_planes <= 0) return 0;
    if (nv <= 0 || nt <= 0) return ctx_fail(ctx, KERR_MESH_INVALID, "empty mesh");
    if (hd_resolution <= 0.f) { hd_resolution = 2000.f; }
    if (hd_min_samples < 0) hd_min_samples = 1000;
    CK(cudaSetDevice(ctx->device));
    cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
    const int G = eval_groups(ctx, n_planes);
    int rc = pool_begin(ctx, eval_groups_fixed_bytes(ctx, nv, n_planes, G) + eval_arena_bytes(nv, nt, n_planes));
    if (rc) return rc;
    EvalWork W[EVAL_MAX_GROUPS];
    if (eval_groups_take(ctx, nv, n_planes, G, W)) return ctx_fail(ctx, KERR_HEAP_OOM, "pool too small");
    return eval_run(ctx, d_verts, nv, d_tris, nt, (const float4*)d_planes, n_planes, flags, hd_resolution,
                    hd_min_samples, hd_total, W, G, d_out, s);
}

extern "C" int cuacd_eval_candidates(gpu_ctx_t ctx, const float* verts, int nv, const int* tris, int nt,
                                     const float* planes, int n_planes, int flags, float hd_resolution,
                                     int hd_min_samples, int hd_total, cuacd_cand_result* out)
{
    if (!ctx) return -1;
    if (n_planes <= 0) return 0;
    if (nv <= 0 || nt <= 0) return ctx_fail(ctx, KERR_MESH_INVALID, "empty mesh");
    for (int i = 0; i < 3 * nt; i++)
        if (tris[i] < 0 || tris[i] >= nv) return ctx_fail(ctx, KERR_MESH_INVALID, "triangle index out of range");
    if (hd_resolution <= 0.f) hd_resolution = 2000.f;
    if (hd_min_samples < 0) hd_min_samples = 1000;
    CK(cudaSetDevice(ctx->device));
    size_t extra = 0;
    const int G = eval_groups(ctx, n_planes);
    for (int attempt = 0; attempt < 4; attempt++) {
        size_t need = al256(12 * (size_t)nv) + al256(12 * (size_t)nt) + al256(sizeof(cuacd_cand_result) * n_planes)
                    + al256(sizeof(float4) * n_planes) + eval_groups_fixed_bytes(ctx, nv, n_planes, G)
                    + eval_arena_bytes(nv, nt, n_planes) + extra;
        int rc = pool_begin(ctx, need);
        if (rc) return rc;
        float* dv = pool_take<float>(ctx, 3 * (size_t)nv);
        int* dt = pool_take<int>(ctx, 3 * (size_t)nt);
        cuacd_cand_result* dout = pool_take<cuacd_cand_result>(ctx, n_planes);
        float4* dp = pool_take<float4>(ctx, n_planes);
        EvalWork W[EVAL_MAX_GROUPS];
        if (eval_groups_take(ctx, nv, n_planes, G, W)) return ctx_fail(ctx, KERR_HEAP_OOM, "pool too small");
        cudaStream_t s = ctx->stream;
        CK(cudaMemcpyAsync(dv, verts, 12 * (size_t)nv, cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(dt, tris, 12 * (size_t)nt, cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(dp, planes, sizeof(float4) * n_planes, cudaMemcpyHostToDevice, s));
        rc = eval_run(ctx, dv, nv, dt, nt, dp, n_planes, flags, hd_resolution, hd_min_samples, hd_total, W, G, dout, s);
        if (rc) return rc;
        CK(cudaMemcpyAsync(out, dout, sizeof(cuacd_cand_result) * n_planes, cudaMemcpyDeviceToHost, s));
        rc = sync_and_check(ctx, "eval_candidates");
        if (rc) return rc;
        bool oom = false;
        for (int i = 0; i < n_planes; i++)
            if (out[i].err & (KERR_HEAP_OOM | KERR_PC_SCRATCH_OOM | KERR_HD_SCRATCH_OOM)) oom = true;
        if (!oom) return 0;
        if (ctx->fixed) return ctx_fail(ctx, KERR_HEAP_OOM, "device pool too small for this evaluation");
        extra = (ctx->cap) * 2;       // grow and retry
    }
    return ctx_fail(ctx, KERR_HEAP_OOM, "device pool exhausted");
}
