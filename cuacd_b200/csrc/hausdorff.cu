// hausdorff.cu — Hausdorff kernels and the gpu_test_hausdorff /
// cuacd_hausdorff entry points.
#include <algorithm>
#include <mutex>
#include <vector>
#include "context.cuh"
#include "hausdorff.cuh"
#include "launch.h"

// One CTA per surface: budget, offsets, BVH.  Scratch from the arena.
// Surface i = first + blockIdx.x * step (a subset of the surfaces can be
// prepared while the rest are still being built).
__global__ void __launch_bounds__(HD_PREP_NT)
k_hd_prep(const HDSurf* __restrict__ surfs, int n_surf, Arena* arena, float resolution, int min_samples,
          int total_override, HDPrep* preps, int* err, int first = 0, int step = 1)
{
    __shared__ HDShared sh;
    __shared__ char* s_scr;
    int i = first + (int)blockIdx.x * step;
    if (i >= n_surf) return;
    HDSurf S = surfs[i];
    if (threadIdx.x == 0) {
        s_scr = nullptr;
        if (S.nt > 0 && S.nv > 0) {
            s_scr = (char*)arena_alloc(arena, hd_prep_bytes(S.nt), err);
            if (!s_scr) atomicOr(err, KERR_HD_SCRATCH_OOM);
        }
    }
    __syncthreads();
    if (!s_scr) {
        if (threadIdx.x == 0) { HDPrep P; memset(&P, 0, sizeof(P)); preps[i] = P; }
        return;
    }
    hd_prep_cta(S, s_scr, resolution, min_samples, total_override, &preps[i], sh);
}

// Plan the query directions: pair p has surfaces 2p (A) and 2p+1 (B);
// direction 2p samples A against B, 2p+1 samples B against A.
__global__ void k_hd_plan(const HDSurf* surfs, const HDPrep* preps, int n_pairs, HDDir* dirs, int* total_chunks,
                          int* counter, float* pair_max)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    int c = 0;
    for (int p = 0; p < n_pairs; p++) {
        bool valid = surfs[2 * p].nt > 0 && surfs[2 * p].nv > 0 && surfs[2 * p + 1].nt > 0 && surfs[2 * p + 1].nv > 0;
        bool has = valid && preps[2 * p].n_samples > 0 && preps[2 * p + 1].n_samples > 0;
        for (int d = 0; d < 2; d++) {
            HDDir D;
            D.src = 2 * p + d; D.dst = 2 * p + 1 - d; D.pair = p;
            D.n_samples = has ? preps[D.src].n_samples : 0;
            D.chunk0 = c;
            c += (D.n_samples + HD_CHUNK - 1) / HD_CHUNK;
            dirs[2 * p + d] = D;
        }
        pair_max[p] = 0.f;
    }
    *total_chunks = c;
    *counter = 0;
}

__global__ void __launch_bounds__(HD_NT)
k_hd_query(const HDSurf* __restrict__ surfs, const HDPrep* __restrict__ preps, const HDDir* __restrict__ dirs,
           int n_dirs, const int* total_chunks, int* counter, float* pair_max)
{
    hd_query_body(surfs, preps, dirs, n_dirs, total_chunks, counter, pair_max);
}

__global__ void k_hd_sqrt(const float* pair_max, int n, float* out, int stride_floats)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[(size_t)i * stride_floats] = sqrtf(pair_max[i]);
}

size_t hd_pairs_scratch_bytes(int n_pairs, int max_nt_a, int max_nt_b)
{
    return (size_t)n_pairs * (al256(hd_prep_bytes(max_nt_a)) + al256(hd_prep_bytes(max_nt_b)) + 2048)
         + al256(sizeof(HDDir) * 2 * (size_t)n_pairs) + al256(sizeof(HDPrep) * 2 * (size_t)n_pairs) + 4096;
}

// Launch the three Hausdorff stages for n_pairs pairs whose surfaces are in
// d_surfs[2p] (A) / d_surfs[2p+1] (B).  Work buffers: d_preps[2n], d_dirs[2n],
// d_i2[2] (total chunks, counter), d_pmax[n].
void launch_hausdorff_stages(const HDSurf* d_surfs, int n_pairs, Arena* arena, float resolution, int min_samples,
                             int total, HDPrep* d_preps, void* d_dirs, int* d_i2, float* d_pmax, int* d_err,
                             int n_sm, cudaStream_t s, const std::function<void(int)>& after)
{
    if (n_pairs > 0) k_hd_prep<<<2 * n_pairs, HD_PREP_NT, 0, s>>>(d_surfs, 2 * n_pairs, arena, resolution, min_samples, total, d_preps, d_err);
    after(0);
    if (n_pairs > 0) k_hd_plan<<<1, 32, 0, s>>>(d_surfs, d_preps, n_pairs, (HDDir*)d_dirs, d_i2, d_i2 + 1, d_pmax);
    after(1);
    if (n_pairs > 0) k_hd_query<<<n_sm * 8, HD_NT, 0, s>>>(d_surfs, d_preps, (const HDDir*)d_dirs, 2 * n_pairs, d_i2, d_i2 + 1, d_pmax);
    after(2);
}

// The stages split for overlap: prep of surfaces first, first + step, ...
// (below 2 * n_pairs), and plan + queries once every surface is prepared.
void launch_hd_prep_subset(const HDSurf* d_surfs, int n_pairs, int first, int step, Arena* arena, float resolution,
                           int min_samples, int total, HDPrep* d_preps, int* d_err, cudaStream_t s)
{
    const int n = (2 * n_pairs - first + step - 1) / step;
    if (n > 0) k_hd_prep<<<n, HD_PREP_NT, 0, s>>>(d_surfs, 2 * n_pairs, arena, resolution, min_samples, total, d_preps,
                                                 d_err, first, step);
}

void launch_hd_plan_query(const HDSurf* d_surfs, int n_pairs, HDPrep* d_preps, void* d_dirs, int* d_i2,
                          float* d_pmax, int n_sm, cudaStream_t s, const std::function<void(int)>& after)
{
    if (n_pairs > 0) k_hd_plan<<<1, 32, 0, s>>>(d_surfs, d_preps, n_pairs, (HDDir*)d_dirs, d_i2, d_i2 + 1, d_pmax);
    after(1);
    if (n_pairs > 0) k_hd_query<<<n_sm * 8, HD_NT, 0, s>>>(d_surfs, d_preps, (const HDDir*)d_dirs, 2 * n_pairs, d_i2, d_i2 + 1, d_pmax);
    after(2);
}

void launch_hausdorff_pairs(const HDSurf* d_surfs, int n_pairs, Arena* arena, float resolution, int min_samples,
                            int total, HDPrep* d_preps, void* d_dirs, int* d_i2, float* d_pmax, int* d_err,
                            int n_sm, cudaStream_t s)
{
    launch_hausdorff_stages(d_surfs, n_pairs, arena, resolution, min_samples, total, d_preps, d_dirs, d_i2, d_pmax,
                            d_err, n_sm, s, [](int) {});
}

size_t hd_dir_bytes() { return sizeof(HDDir); }

void launch_hd_sqrt(const float* pmax, int n, float* out, int stride_floats, cudaStream_t s)
{
    if (n > 0) k_hd_sqrt<<<(n + 127) / 128, 128, 0, s>>>(pmax, n, out, stride_floats);
}

static int sm_count(gpu_ctx* ctx)
{
    int n = 148;
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, ctx->device);
    return n > 0 ? n : 148;
}

extern "C" int cuacd_hausdorff(gpu_ctx_t ctx, const float* a_verts, int a_nv, const int* a_tris, int a_nt,
                               const float* b_verts, int b_nv, const int* b_tris, int b_nt,
                               float resolution, int min_samples, int total, float* out_hausdorff)
{
    if (!ctx) return -1;
    if (a_nv < 0 || a_nt < 0 || b_nv < 0 || b_nt < 0) return ctx_fail(ctx, KERR_MESH_INVALID, "negative size");
    for (int i = 0; i < 3 * a_nt; i++) if (a_tris[i] < 0 || a_tris[i] >= a_nv) return ctx_fail(ctx, KERR_MESH_INVALID, "mesh a: index out of range");
    for (int i = 0; i < 3 * b_nt; i++) if (b_tris[i] < 0 || b_tris[i] >= b_nv) return ctx_fail(ctx, KERR_MESH_INVALID, "mesh b: index out of range");
    if (resolution <= 0.f) resolution = 2000.f;
    if (min_samples < 0) min_samples = 1000;
    CK(cudaSetDevice(ctx->device));
    size_t need = al256(12 * (size_t)a_nv) + al256(12 * (size_t)a_nt) + al256(12 * (size_t)b_nv) + al256(12 * (size_t)b_nt)
                + al256(sizeof(HDSurf) * 2) + al256(sizeof(int) * 4) + al256(sizeof(float) * 2)
                + hd_pairs_scratch_bytes(1, a_nt, b_nt) + (1 << 20);
    int rc = pool_begin(ctx, need);
    if (rc) return rc;
    float* dav = pool_take<float>(ctx, 3 * (size_t)a_nv); int* dat = pool_take<int>(ctx, 3 * (size_t)a_nt);
    float* dbv = pool_take<float>(ctx, 3 * (size_t)b_nv); int* dbt = pool_take<int>(ctx, 3 * (size_t)b_nt);
    HDSurf* dsurf = pool_take<HDSurf>(ctx, 2);
    HDPrep* dprep = pool_take<HDPrep>(ctx, 2);
    char* ddirs = pool_take<char>(ctx, 2 * sizeof(HDDir));
    int* di = pool_take<int>(ctx, 4);
    float* dmax = pool_take<float>(ctx, 2);
    cudaStream_t s = ctx->stream;
    if (a_nv) CK(cudaMemcpyAsync(dav, a_verts, 12 * (size_t)a_nv, cudaMemcpyHostToDevice, s));
    if (a_nt) CK(cudaMemcpyAsync(dat, a_tris, 12 * (size_t)a_nt, cudaMemcpyHostToDevice, s));
    if (b_nv) CK(cudaMemcpyAsync(dbv, b_verts, 12 * (size_t)b_nv, cudaMemcpyHostToDevice, s));
    if (b_nt) CK(cudaMemcpyAsync(dbt, b_tris, 12 * (size_t)b_nt, cudaMemcpyHostToDevice, s));
    HDSurf hs[2] = {{dav, dat, a_nv, a_nt}, {dbv, dbt, b_nv, b_nt}};
    CK(cudaMemcpyAsync(dsurf, hs, sizeof(hs), cudaMemcpyHostToDevice, s));
    CK(cudaMemsetAsync(di, 0, 4 * sizeof(int), s));
    launch_arena_reset(ctx->d_arena, ctx->pool + ctx->carve, ctx->cap - ctx->carve, s);
    launch_hausdorff_pairs(dsurf, 1, ctx->d_arena, resolution, min_samples, total, dprep, ddirs, di, dmax, di + 2,
                           sm_count(ctx), s);
    launch_hd_sqrt(dmax, 1, dmax + 1, 1, s);
    ctx->launches += 5;
    CK(cudaGetLastError());
    int herr = 0;
    float h = 0.f;
    CK(cudaMemcpyAsync(&herr, di + 2, sizeof(int), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(&h, dmax + 1, sizeof(float), cudaMemcpyDeviceToHost, s));
    rc = sync_and_check(ctx, "hausdorff");
    if (rc) return rc;
    if (herr) return ctx_fail(ctx, herr, "hausdorff failed (error word 0x%x)", herr);
    *out_hausdorff = h;
    return 0;
}

extern "C" int gpu_test_hausdorff(gpu_ctx_t ctx, const float* hull_verts, int hull_nv, const int* hull_tris,
                                  int hull_nt, const float* mesh_verts, int mesh_nv, const int* mesh_tris,
                                  int mesh_nt, float* out_hausdorff)
{
    return cuacd_hausdorff(ctx, hull_verts, hull_nv, hull_tris, hull_nt, mesh_verts, mesh_nv, mesh_tris, mesh_nt,
                           2000.f, 1000, 0, out_hausdorff);
}

// ---------------------------------------------------------------------------
// Batched Hausdorff distance: n_pairs (A_i, B_i) pairs in one launch of each
// stage (the reference runs such a batch as one block per pair in
// bench/hausdorff_bench.cu:253-345 and, inside the search, in
// la_hausdorff_parts).  Meshes are packed back to back: vertex offsets
// voff[n+1], triangle offsets toff[n+1], triangle indices local to their mesh.
// ---------------------------------------------------------------------------
static int hd_batch_check(gpu_ctx* ctx, int n_pairs, const int* voff, const int* toff, const char* which,
                          int* max_nt)
{
    *max_nt = 0;
    if (voff[0] != 0 || toff[0] != 0) return ctx_fail(ctx, KERR_MESH_INVALID, "mesh %s: offsets must start at 0", which);
    for (int i = 0; i < n_pairs; i++) {
        if (voff[i + 1] < voff[i] || toff[i + 1] < toff[i])
            return ctx_fail(ctx, KERR_MESH_INVALID, "mesh %s %d: decreasing offsets", which, i);
        *max_nt = std::max(*max_nt, toff[i + 1] - toff[i]);
    }
    return 0;
}

static int hd_batch_run(gpu_ctx* ctx, int n_pairs, const float* dav, const int* a_voff, const int* dat,
                        const int* a_toff, const float* dbv, const int* b_voff, const int* dbt, const int* b_toff,
                        int max_a, int max_b, float resolution, int min_samples, int total, float* d_out,
                        cudaStream_t s)
{
    HDSurf* dsurf = pool_take<HDSurf>(ctx, 2 * (size_t)n_pairs);
    HDPrep* dprep = pool_take<HDPrep>(ctx, 2 * (size_t)n_pairs);
    char* ddirs = pool_take<char>(ctx, 2 * (size_t)n_pairs * sizeof(HDDir));
    int* di = pool_take<int>(ctx, 4);
    float* dmax = pool_take<float>(ctx, (size_t)n_pairs);
    if (!dsurf || !dprep || !ddirs || !di || !dmax) return ctx_fail(ctx, KERR_HEAP_OOM, "hausdorff batch: pool too small");
    std::vector<HDSurf> hs(2 * (size_t)n_pairs);
    for (int i = 0; i < n_pairs; i++) {
        hs[2 * i] = {dav + 3 * (size_t)a_voff[i], dat + 3 * (size_t)a_toff[i], a_voff[i + 1] - a_voff[i],
                     a_toff[i + 1] - a_toff[i]};
        hs[2 * i + 1] = {dbv + 3 * (size_t)b_voff[i], dbt + 3 * (size_t)b_toff[i], b_voff[i + 1] - b_voff[i],
                         b_toff[i + 1] - b_toff[i]};
    }
    CK(cudaMemcpyAsync(dsurf, hs.data(), sizeof(HDSurf) * hs.size(), cudaMemcpyHostToDevice, s));
    CK(cudaMemsetAsync(di, 0, 4 * sizeof(int), s));
    launch_arena_reset(ctx->d_arena, ctx->pool + ctx->carve, ctx->cap - ctx->carve, s);
    launch_hausdorff_pairs(dsurf, n_pairs, ctx->d_arena, resolution, min_samples, total, dprep, ddirs, di, dmax,
                           di + 2, sm_count(ctx), s);
    launch_hd_sqrt(dmax, n_pairs, d_out, 1, s);
    ctx->launches += 5;
    CK(cudaGetLastError());
    int herr = 0;
    CK(cudaMemcpyAsync(&herr, di + 2, sizeof(int), cudaMemcpyDeviceToHost, s));
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return ctx_fail(ctx, (int)e, "hausdorff batch: %s", cudaGetErrorString(e));
    if (herr) return ctx_fail(ctx, herr, "hausdorff batch failed (error word 0x%x)", herr);
    (void)max_a; (void)max_b;
    return 0;
}

static size_t hd_batch_pool_bytes(int n_pairs, int max_a, int max_b)
{
    return al256(sizeof(HDSurf) * 2 * (size_t)n_pairs) + al256(sizeof(HDPrep) * 2 * (size_t)n_pairs)
         + al256(sizeof(HDDir) * 2 * (size_t)n_pairs) + al256(sizeof(int) * 4) + al256(sizeof(float) * (size_t)n_pairs)
         + hd_pairs_scratch_bytes(n_pairs, max_a, max_b) + (1 << 20);
}

extern "C" int cuacd_hausdorff_batch(gpu_ctx_t ctx, int n_pairs,
                                     const float* a_verts, const int* a_voff, const int* a_tris, const int* a_toff,
                                     const float* b_verts, const int* b_voff, const int* b_tris, const int* b_toff,
                                     float resolution, int min_samples, int total, float* out_hausdorff)
{
    if (!ctx) return -1;
    if (n_pairs <= 0) return 0;
    int max_a = 0, max_b = 0;
    int rc = hd_batch_check(ctx, n_pairs, a_voff, a_toff, "a", &max_a);
    if (!rc) rc = hd_batch_check(ctx, n_pairs, b_voff, b_toff, "b", &max_b);
    if (rc) return rc;
    for (int i = 0; i < n_pairs; i++) {
        for (int k = 3 * a_toff[i]; k < 3 * a_toff[i + 1]; k++)
            if (a_tris[k] < 0 || a_tris[k] >= a_voff[i + 1] - a_voff[i])
                return ctx_fail(ctx, KERR_MESH_INVALID, "mesh a %d: index out of range", i);
        for (int k = 3 * b_toff[i]; k < 3 * b_toff[i + 1]; k++)
            if (b_tris[k] < 0 || b_tris[k] >= b_voff[i + 1] - b_voff[i])
                return ctx_fail(ctx, KERR_MESH_INVALID, "mesh b %d: index out of range", i);
    }
    if (resolution <= 0.f) resolution = 2000.f;
    if (min_samples < 0) min_samples = 1000;
    CK(cudaSetDevice(ctx->device));
    const size_t anv = a_voff[n_pairs], ant = a_toff[n_pairs], bnv = b_voff[n_pairs], bnt = b_toff[n_pairs];
    size_t need = al256(12 * anv) + al256(12 * ant) + al256(12 * bnv) + al256(12 * bnt)
                + al256(sizeof(float) * (size_t)n_pairs) + hd_batch_pool_bytes(n_pairs, max_a, max_b);
    rc = pool_begin(ctx, need);
    if (rc) return rc;
    float* dav = pool_take<float>(ctx, 3 * anv); int* dat = pool_take<int>(ctx, 3 * ant);
    float* dbv = pool_take<float>(ctx, 3 * bnv); int* dbt = pool_take<int>(ctx, 3 * bnt);
    float* dout = pool_take<float>(ctx, (size_t)n_pairs);
    cudaStream_t s = ctx->stream;
    if (anv) CK(cudaMemcpyAsync(dav, a_verts, 12 * anv, cudaMemcpyHostToDevice, s));
    if (ant) CK(cudaMemcpyAsync(dat, a_tris, 12 * ant, cudaMemcpyHostToDevice, s));
    if (bnv) CK(cudaMemcpyAsync(dbv, b_verts, 12 * bnv, cudaMemcpyHostToDevice, s));
    if (bnt) CK(cudaMemcpyAsync(dbt, b_tris, 12 * bnt, cudaMemcpyHostToDevice, s));
    rc = hd_batch_run(ctx, n_pairs, dav, a_voff, dat, a_toff, dbv, b_voff, dbt, b_toff, max_a, max_b, resolution,
                      min_samples, total, dout, s);
    if (rc) return rc;
    CK(cudaMemcpy(out_hausdorff, dout, sizeof(float) * (size_t)n_pairs, cudaMemcpyDeviceToHost));
    return 0;
}

extern "C" int cuacd_hausdorff_batch_device(gpu_ctx_t ctx, int n_pairs,
                                            const float* d_a_verts, const int* a_voff, const int* d_a_tris,
                                            const int* a_toff, const float* d_b_verts, const int* b_voff,
                                            const int* d_b_tris, const int* b_toff, float resolution,
                                            int min_samples, int total, float* d_out, void* stream)
{
    if (!ctx) return -1;
    if (n_pairs <= 0) return 0;
    int max_a = 0, max_b = 0;
    int rc = hd_batch_check(ctx, n_pairs, a_voff, a_toff, "a", &max_a);
    if (!rc) rc = hd_batch_check(ctx, n_pairs, b_voff, b_toff, "b", &max_b);
    if (rc) return rc;
    if (resolution <= 0.f) resolution = 2000.f;
    if (min_samples < 0) min_samples = 1000;
    CK(cudaSetDevice(ctx->device));
    rc = pool_begin(ctx, hd_batch_pool_bytes(n_pairs, max_a, max_b));
    if (rc) return rc;
    return hd_batch_run(ctx, n_pairs, d_a_verts, a_voff, d_a_tris, a_toff, d_b_verts, b_voff, d_b_tris, b_toff,
                        max_a, max_b, resolution, min_samples, total, d_out,
                        stream ? (cudaStream_t)stream : ctx->stream);
}

// ---------------------------------------------------------------------------
// Allocation-free Hausdorff distance.
//
// For callers that cannot allocate device memory themselves — code that runs
// inside a host framework which owns every device allocation, or a plugin
// loaded where cudaMalloc is forbidden or may block — this entry point uses a
// fixed block of static device memory instead of the context pool.  The block
// is a file-scope __device__ array, so every GPU that loads the library holds
// CUACD_HD_NOALLOC_BYTES of it until the process exits.  All calls share it:
// its contents persist between calls, the per-call state that must start at
// zero is cleared by the first kernel of each call, and two calls whose work
// overlaps on the GPU (different streams, no ordering between them) race on
// it.  The first call on a device resolves the array's device address; make
// that first call before any stream capture.
// ---------------------------------------------------------------------------
#define CUACD_HD_NOALLOC_BYTES (32ull << 20)
#define CUACD_HD_NOALLOC_MAX_TRIS (1 << 20)
static __device__ __align__(256) char g_hd_noalloc_scratch[CUACD_HD_NOALLOC_BYTES];

// Layout of the static block: [Arena | 2 HDSurf | 2 HDPrep | 2 HDDir |
// 4 ints | 2 floats | arena space for the two surfaces' preps].
static const size_t NOALLOC_HDR = 4096;

__global__ void k_hd_noalloc_setup(char* base, const float* av, int anv, const int* at, int ant,
                                   const float* bv, int bnv, const int* bt, int bnt)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    Arena* A = (Arena*)base;
    A->base = base + NOALLOC_HDR;
    A->capacity = CUACD_HD_NOALLOC_BYTES - NOALLOC_HDR;
    A->offset = 0;
    HDSurf* S = (HDSurf*)(base + 256);
    S[0].v = av; S[0].t = at; S[0].nv = anv; S[0].nt = ant;
    S[1].v = bv; S[1].t = bt; S[1].nv = bnv; S[1].nt = bnt;
    int* I = (int*)(base + 1024);
    I[0] = 0; I[1] = 0; I[2] = 0; I[3] = 0;            // chunks, counter, error word
    float* M = (float*)(base + 1088);
    M[0] = 0.f; M[1] = 0.f;
}

// Every triangle index must lie in [0, nv).  The allocating entry points
// check this on the host; here the indices are device memory, so a grid scan
// does it: a surface with a bad index gets the error word set and its
// triangle count zeroed before any kernel reads through its indices.
__global__ void k_hd_noalloc_check(char* base, const int* at, int ant, int anv, const int* bt, int bnt, int bnv)
{
    HDSurf* S = (HDSurf*)(base + 256);
    int* I = (int*)(base + 1024);
    const long long na = 3ll * ant, n = na + 3ll * bnt;
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        const bool in_a = k < na;
        const int x = in_a ? at[k] : bt[k - na];
        if (x < 0 || x >= (in_a ? anv : bnv)) {
            atomicOr(&I[2], KERR_MESH_INVALID);
            S[in_a ? 0 : 1].nt = 0;
        }
    }
}

// sqrt of the pair's squared maximum, or NaN when any kernel of the call set
// the error word (bad index, scratch overflow): never a silent 0.
__global__ void k_hd_noalloc_finish(const char* base, float* out)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const int err = ((const int*)(base + 1024))[2];
    const float m = ((const float*)(base + 1088))[0];
    *out = err ? __int_as_float(0x7fc00000) : sqrtf(m);
}

static char* g_noalloc_base[64];
static std::mutex g_noalloc_mu;

extern "C" int cuacd_hausdorff_noalloc(const float* d_av, int anv, const int* d_at, int ant,
                                       const float* d_bv, int bnv, const int* d_bt, int bnt,
                                       float resolution, int min_samples, int total,
                                       float* d_out, void* stream)
{
    if (anv < 0 || ant < 0 || bnv < 0 || bnt < 0 || !d_out) return CUACD_NOALLOC_BAD_ARGS;
    // No surface above this many triangles can fit the block; rejecting them
    // first keeps the sizing arithmetic below far from int overflow.
    if (ant > CUACD_HD_NOALLOC_MAX_TRIS || bnt > CUACD_HD_NOALLOC_MAX_TRIS) return CUACD_NOALLOC_TOO_LARGE;
    size_t need = NOALLOC_HDR + hd_prep_bytes(ant) + hd_prep_bytes(bnt) + 8 * 256;
    if (need > CUACD_HD_NOALLOC_BYTES) return CUACD_NOALLOC_TOO_LARGE;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return (int)e;
    if (dev < 0 || dev >= 64) return CUACD_NOALLOC_BAD_ARGS;
    char* base;
    {
        std::lock_guard<std::mutex> lock(g_noalloc_mu);
        if (!g_noalloc_base[dev]) {
            void* p = nullptr;
            e = cudaGetSymbolAddress(&p, g_hd_noalloc_scratch);
            if (e != cudaSuccess) return (int)e;
            g_noalloc_base[dev] = (char*)p;
        }
        base = g_noalloc_base[dev];
    }
    if (resolution <= 0.f) resolution = 2000.f;
    if (min_samples < 0) min_samples = 1000;
    int n_sm = 148;
    cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
    cudaStream_t s = (cudaStream_t)stream;
    k_hd_noalloc_setup<<<1, 32, 0, s>>>(base, d_av, anv, d_at, ant, d_bv, bnv, d_bt, bnt);
    if (ant + bnt > 0) {
        const long long n = 3ll * ((long long)ant + bnt);
        const int blocks = (int)std::min<long long>((n + 255) / 256, 4ll * (n_sm > 0 ? n_sm : 148));
        k_hd_noalloc_check<<<blocks, 256, 0, s>>>(base, d_at, ant, anv, d_bt, bnt, bnv);
    }
    HDSurf* surfs = (HDSurf*)(base + 256);
    HDPrep* preps = (HDPrep*)(base + 384);
    void* dirs = (void*)(base + 768);
    int* i4 = (int*)(base + 1024);
    float* pmax = (float*)(base + 1088);
    launch_hausdorff_pairs(surfs, 1, (Arena*)base, resolution, min_samples, total, preps, dirs, i4, pmax, i4 + 2,
                           n_sm > 0 ? n_sm : 148, s);
    k_hd_noalloc_finish<<<1, 32, 0, s>>>(base, d_out);
    e = cudaGetLastError();
    return e == cudaSuccess ? 0 : (int)e;
}
