// capi.cu — extern "C" entry points of libcuacd_b200.so (see
// include/cuacd_b200.h for the contract of each function).
#include <cstdlib>
#include <vector>
#include <algorithm>
#include "context.cuh"
#include "volume.cuh"
#include "hull.cuh"
#include "launch.h"

// ---------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------
__global__ void k_arena_reset(Arena* a, char* base, unsigned long long cap)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        a->base = base; a->capacity = cap; a->offset = 0;
        a->n_resets += 1;
    }
}

void launch_arena_reset(Arena* a, char* base, unsigned long long cap, cudaStream_t s)
{
    k_arena_reset<<<1, 32, 0, s>>>(a, base, cap);
}

// ---------------------------------------------------------------------------
// context
// ---------------------------------------------------------------------------
extern "C" void gpu_set_fatbin(const void* data, size_t len) { (void)data; (void)len; }

extern "C" int gpu_init(gpu_ctx_t* out, int device_ordinal, size_t pool_bytes)
{
    if (!out) return -1;
    *out = nullptr;
    gpu_ctx* ctx = (gpu_ctx*)calloc(1, sizeof(gpu_ctx));
    if (!ctx) return -1;
    int dev = device_ordinal;
    cudaError_t e;
    if (dev < 0) {
        e = cudaGetDevice(&dev);
        if (e != cudaSuccess) { free(ctx); return (int)e; }
    } else {
        e = cudaSetDevice(dev);
        if (e != cudaSuccess) { free(ctx); return (int)e; }
    }
    ctx->device = dev;
    ctx->n_sm = 0;
    cudaDeviceGetAttribute(&ctx->n_sm, cudaDevAttrMultiProcessorCount, dev);
    if (ctx->n_sm <= 0) ctx->n_sm = 148;
    e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) { free(ctx); return (int)e; }
    e = cudaMalloc(&ctx->d_arena, sizeof(Arena));
    if (e != cudaSuccess) { cudaStreamDestroy(ctx->stream); free(ctx); return (int)e; }
    cudaMemset(ctx->d_arena, 0, sizeof(Arena));
    ctx->fixed = pool_bytes > 0;
    size_t want = pool_bytes > 0 ? pool_bytes : ((size_t)256 << 20);
    e = cudaMalloc(&ctx->pool, want);
    if (e != cudaSuccess) {
        cudaFree(ctx->d_arena); cudaStreamDestroy(ctx->stream); free(ctx); return (int)e;
    }
    ctx->cap = want;
    cudaMemPoolProps props;
    memset(&props, 0, sizeof(props));
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    e = cudaMemPoolCreate(&ctx->parts_pool, &props);
    if (e != cudaSuccess) {
        cudaFree(ctx->pool); cudaFree(ctx->d_arena); cudaStreamDestroy(ctx->stream); free(ctx); return (int)e;
    }
    unsigned long long keep = ~0ull;
    cudaMemPoolSetAttribute(ctx->parts_pool, cudaMemPoolAttrReleaseThreshold, &keep);
    *out = ctx;
    return 0;
}

extern "C" void gpu_destroy(gpu_ctx_t ctx)
{
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    if (ctx->pool) cudaFree(ctx->pool);
    if (ctx->d_arena) cudaFree(ctx->d_arena);
    for (int i = 0; i < 3; i++) {
        if (ctx->aux[i]) cudaStreamDestroy(ctx->aux[i]);
        if (ctx->join_ev[i]) cudaEventDestroy(ctx->join_ev[i]);
    }
    if (ctx->fork_ev) cudaEventDestroy(ctx->fork_ev);
    cudaStreamDestroy(ctx->stream);
    if (ctx->parts_pool) cudaMemPoolDestroy(ctx->parts_pool);
    free(ctx);
}

extern "C" const char* gpu_last_error(gpu_ctx_t ctx) { return ctx ? ctx->last_error : "no context"; }

extern "C" int cuacd_device_info(gpu_ctx_t ctx, char* name, int cap, int* n_sm)
{
    if (!ctx) return -1;
    cudaDeviceProp prop;
    CK(cudaGetDeviceProperties(&prop, ctx->device));
    if (name && cap > 0) { strncpy(name, prop.name, (size_t)cap - 1); name[cap - 1] = 0; }
    if (n_sm) *n_sm = ctx->n_sm;
    return 0;
}
extern "C" int gpu_heap_compact(gpu_ctx_t ctx) { (void)ctx; return 0; }
extern "C" size_t gpu_pool_usage(gpu_ctx_t ctx)
{
    if (!ctx) return 0;
    Arena a;
    if (cudaMemcpy(&a, ctx->d_arena, sizeof(Arena), cudaMemcpyDeviceToHost) != cudaSuccess) return ctx->high_water;
    size_t dev_hw = (size_t)a.high_water;
    return ctx->high_water + dev_hw;
}
extern "C" int gpu_heap_stats(gpu_ctx_t ctx, unsigned long long out[6])
{
    if (!ctx || !out) return -1;
    Arena a;
    CK(cudaMemcpy(&a, ctx->d_arena, sizeof(Arena), cudaMemcpyDeviceToHost));
    out[0] = a.offset;            // output bytes live in the device arena
    out[1] = a.n_allocs;          // device allocations served
    out[2] = a.n_resets;          // arena releases (resets)
    out[3] = ctx->stats[3];       // scratch bytes carved by the last call
    out[4] = ctx->stats[4];       // scratch carves
    out[5] = ctx->stats[5];       // scratch releases
    return 0;
}
extern "C" unsigned long long cuacd_launch_count(gpu_ctx_t ctx) { return ctx ? ctx->launches : 0; }

// ---------------------------------------------------------------------------
// hulls
// ---------------------------------------------------------------------------
// Device bytes of one hull batch: jobs, states, results, control words,
// per-warp wrap lists and per-cloud scratch.  The public batch calls build
// every cloud with full-size tables in one round: callers' clouds are often
// near-convex (an input mesh's vertices), whose hulls outgrow reduced first
// tables, and the rebuild costs more than the clearing it saves (a lone
// 10,242-point sphere: 11.3 -> 8.0 ms).
static size_t hull_batch_need(int n_hulls, int max_pts, int nwc)
{
    return al256(sizeof(HullJob) * (size_t)n_hulls) + al256(sizeof(HullState) * (size_t)n_hulls)
         + al256(sizeof(HullRes) * (size_t)n_hulls) + al256(64) + al256(hull_wrap_buf_bytes(nwc))
         + al256(hull_scratch_bytes(max_pts, HULL_FIRST_CAP)) * (size_t)n_hulls + 4096;
}

static int launch_hull_batch(gpu_ctx* ctx, const float* d_pts, const int* d_off, int n_hulls,
                             int max_pts, int max_hv, int max_ht, float* d_v, int* d_t,
                             int* d_nv, int* d_nt, float* d_vol, int* d_err, cudaStream_t s,
                             unsigned long long* d_stats = nullptr)
{
    const int nwc = hull_wrap_ctas(hull_wrap_points(n_hulls, max_pts), ctx->n_sm, max_pts);
    HullJob* jobs = pool_take<HullJob>(ctx, n_hulls);
    HullState* states = pool_take<HullState>(ctx, n_hulls);
    HullRes* res = pool_take<HullRes>(ctx, n_hulls);
    int* ctl = pool_take<int>(ctx, 16);
    int* wbuf = (int*)pool_take<char>(ctx, hull_wrap_buf_bytes(nwc));
    const size_t scr_bytes = al256(hull_scratch_bytes(max_pts, HULL_FIRST_CAP)) * (size_t)n_hulls;
    char* scratch = pool_take<char>(ctx, scr_bytes);
    if (!scratch) return ctx_fail(ctx, KERR_HEAP_OOM, "hull scratch does not fit the pool");
    launch_arena_reset(ctx->d_arena, scratch, scr_bytes, s);
    launch_jobs_from_offsets(d_pts, d_off, n_hulls, d_v, d_t, max_hv, max_ht, jobs, s);
    launch_hull_jobs(jobs, n_hulls, states, res, ctx->d_arena, ctx->d_arena, ctl, wbuf, nwc, d_stats, s, max_pts,
                     false);
    launch_unpack_results(res, n_hulls, d_nv, d_nt, d_vol, d_err, s);
    ctx->launches += 6;
    CK(cudaGetLastError());
    return 0;
}

static int hull_common(gpu_ctx_t ctx, const float* pts, int total_pts, const int* offsets, int n_hulls,
                       int max_pts, int max_hv, int max_ht, float* out_verts, int* out_tris,
                       int* out_nv, int* out_nt, float* out_vol, int* out_err,
                       unsigned long long* out_stats = nullptr)
{
    if (!ctx) return -1;
    if (n_hulls <= 0) return 0;
    if (total_pts < 0 || max_pts < 0 || max_hv < 0 || max_ht < 0)
        return ctx_fail(ctx, KERR_MESH_INVALID, "negative size");
    for (int i = 0; i < n_hulls; i++) {
        int n = offsets[i + 1] - offsets[i];
        if (n < 0 || n > max_pts || offsets[i + 1] > total_pts)
            return ctx_fail(ctx, KERR_MESH_INVALID, "hull %d: bad offsets", i);
    }
    if (max_pts >= (1 << 22)) return ctx_fail(ctx, KERR_MESH_INVALID, "more than 2^22 points in one cloud");
    CK(cudaSetDevice(ctx->device));
    size_t need = al256(sizeof(float) * 3 * (size_t)total_pts) + al256(sizeof(int) * (size_t)(n_hulls + 1))
                + al256(sizeof(float) * 3 * (size_t)n_hulls * max_hv) + al256(sizeof(int) * 3 * (size_t)n_hulls * max_ht)
                + 4 * al256(sizeof(int) * (size_t)n_hulls)
                + hull_batch_need(n_hulls, max_pts, hull_wrap_ctas(hull_wrap_points(n_hulls, max_pts), ctx->n_sm, max_pts))
                + al256(64 * (size_t)n_hulls);
    int rc = pool_begin(ctx, need);
    if (rc) return rc;
    unsigned long long* d_stats = out_stats ? pool_take<unsigned long long>(ctx, 8 * (size_t)n_hulls) : nullptr;
    float* d_pts = pool_take<float>(ctx, 3 * (size_t)total_pts);
    int* d_off = pool_take<int>(ctx, n_hulls + 1);
    float* d_v = pool_take<float>(ctx, 3 * (size_t)n_hulls * max_hv);
    int* d_t = pool_take<int>(ctx, 3 * (size_t)n_hulls * max_ht);
    int* d_nv = pool_take<int>(ctx, n_hulls);
    int* d_nt = pool_take<int>(ctx, n_hulls);
    float* d_vol = pool_take<float>(ctx, n_hulls);
    int* d_err = pool_take<int>(ctx, n_hulls);
    cudaStream_t s = ctx->stream;
    if (total_pts > 0) CK(cudaMemcpyAsync(d_pts, pts, sizeof(float) * 3 * (size_t)total_pts, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(d_off, offsets, sizeof(int) * (size_t)(n_hulls + 1), cudaMemcpyHostToDevice, s));
    rc = launch_hull_batch(ctx, d_pts, d_off, n_hulls, max_pts, max_hv, max_ht, d_v, d_t, d_nv, d_nt, d_vol, d_err, s,
                           d_stats);
    if (rc) return rc;
    if (out_stats) CK(cudaMemcpyAsync(out_stats, d_stats, 64 * (size_t)n_hulls, cudaMemcpyDeviceToHost, s));
    if (out_verts) CK(cudaMemcpyAsync(out_verts, d_v, sizeof(float) * 3 * (size_t)n_hulls * max_hv, cudaMemcpyDeviceToHost, s));
    if (out_tris) CK(cudaMemcpyAsync(out_tris, d_t, sizeof(int) * 3 * (size_t)n_hulls * max_ht, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(out_nv, d_nv, sizeof(int) * n_hulls, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(out_nt, d_nt, sizeof(int) * n_hulls, cudaMemcpyDeviceToHost, s));
    if (out_vol) CK(cudaMemcpyAsync(out_vol, d_vol, sizeof(float) * n_hulls, cudaMemcpyDeviceToHost, s));
    if (out_err) CK(cudaMemcpyAsync(out_err, d_err, sizeof(int) * n_hulls, cudaMemcpyDeviceToHost, s));
    return sync_and_check(ctx, "hull");
}

extern "C" int gpu_hull_dandc(gpu_ctx_t ctx, const float* pts, int total_pts, const int* offsets, int n_hulls,
                              int max_pts_per_hull, int max_hull_verts, int max_hull_tris,
                              float* out_verts, int* out_tris, int* out_nv, int* out_nt, int* out_errors)
{
    return hull_common(ctx, pts, total_pts, offsets, n_hulls, max_pts_per_hull, max_hull_verts, max_hull_tris,
                       out_verts, out_tris, out_nv, out_nt, nullptr, out_errors);
}

extern "C" int gpu_kdop_hull(gpu_ctx_t ctx, const float* pts, int total_pts, const int* offsets, int n_hulls,
                             int max_hull_verts, int max_hull_tris, float* out_verts, int* out_tris,
                             int* out_nv, int* out_nt, float* out_volumes, int* out_errors)
{
    if (!ctx) return -1;
    int max_pts = 0;
    for (int i = 0; i < n_hulls; i++) max_pts = std::max(max_pts, offsets[i + 1] - offsets[i]);
    return hull_common(ctx, pts, total_pts, offsets, n_hulls, max_pts, max_hull_verts, max_hull_tris,
                       out_verts, out_tris, out_nv, out_nt, out_volumes, out_errors);
}

extern "C" int cuacd_hull_batch_device(gpu_ctx_t ctx, const float* d_pts, const int* d_offsets, int n_hulls,
                                       int max_pts, int max_hv, int max_ht, float* d_v, int* d_t,
                                       int* d_nv, int* d_nt, float* d_vol, int* d_err, void* stream)
{
    if (!ctx) return -1;
    if (n_hulls <= 0) return 0;
    if (max_pts >= (1 << 22)) return ctx_fail(ctx, KERR_MESH_INVALID, "more than 2^22 points in one cloud");
    CK(cudaSetDevice(ctx->device));
    int rc = pool_begin(ctx, hull_batch_need(n_hulls, max_pts, hull_wrap_ctas(hull_wrap_points(n_hulls, max_pts), ctx->n_sm, max_pts)));
    if (rc) return rc;
    return launch_hull_batch(ctx, d_pts, d_offsets, n_hulls, max_pts, max_hv, max_ht, d_v, d_t, d_nv, d_nt,
                             d_vol, d_err, stream ? (cudaStream_t)stream : ctx->stream);
}

// ---------------------------------------------------------------------------
// volumes
// ---------------------------------------------------------------------------
extern "C" int gpu_batch_mesh_volume(gpu_ctx_t ctx, const float* verts, int total_verts, const int* tris,
                                     int total_tris, const int* tri_offsets, const int* vert_offsets,
                                     int n_meshes, float* out_volumes)
{
    if (!ctx) return -1;
    if (n_meshes <= 0) return 0;
    for (int m = 0; m < n_meshes; m++) {
        if (tri_offsets[m + 1] < tri_offsets[m] || tri_offsets[m + 1] > total_tris)
            return ctx_fail(ctx, KERR_MESH_INVALID, "mesh %d: bad tri offsets", m);
        if (vert_offsets && (vert_offsets[m + 1] < vert_offsets[m] || vert_offsets[m + 1] > total_verts))
            return ctx_fail(ctx, KERR_MESH_INVALID, "mesh %d: bad vert offsets", m);
    }
    // tiles never straddle meshes; empty meshes get no tile (volume 0)
    std::vector<int> tile_mesh, tile_first, mesh_tile0(n_meshes + 1);
    for (int m = 0; m < n_meshes; m++) {
        mesh_tile0[m] = (int)tile_mesh.size();
        bool has_verts = vert_offsets ? vert_offsets[m + 1] > vert_offsets[m] : total_verts > 0;
        if (!has_verts) continue;
        for (int t = tri_offsets[m]; t < tri_offsets[m + 1]; t += VOL_TILE) {
            tile_mesh.push_back(m); tile_first.push_back(t);
        }
    }
    mesh_tile0[n_meshes] = (int)tile_mesh.size();
    int n_tiles = (int)tile_mesh.size();
    CK(cudaSetDevice(ctx->device));
    size_t need = al256(sizeof(float) * 3 * (size_t)total_verts) + al256(sizeof(int) * 3 * (size_t)total_tris)
                + 2 * al256(sizeof(int) * (size_t)(n_meshes + 1)) + 2 * al256(sizeof(int) * (size_t)n_tiles)
                + al256(sizeof(int) * (size_t)(n_meshes + 1)) + al256(sizeof(double) * (size_t)n_tiles)
                + al256(sizeof(float) * (size_t)n_meshes) + 4096;
    int rc = pool_begin(ctx, need);
    if (rc) return rc;
    float* d_v = pool_take<float>(ctx, 3 * (size_t)total_verts);
    int* d_t = pool_take<int>(ctx, 3 * (size_t)total_tris);
    int* d_to = pool_take<int>(ctx, n_meshes + 1);
    int* d_vo = vert_offsets ? pool_take<int>(ctx, n_meshes + 1) : nullptr;
    int* d_tm = pool_take<int>(ctx, n_tiles);
    int* d_tf = pool_take<int>(ctx, n_tiles);
    int* d_mt0 = pool_take<int>(ctx, n_meshes + 1);
    double* d_part = pool_take<double>(ctx, n_tiles);
    float* d_out = pool_take<float>(ctx, n_meshes);
    cudaStream_t s = ctx->stream;
    if (total_verts > 0) CK(cudaMemcpyAsync(d_v, verts, sizeof(float) * 3 * (size_t)total_verts, cudaMemcpyHostToDevice, s));
    if (total_tris > 0) CK(cudaMemcpyAsync(d_t, tris, sizeof(int) * 3 * (size_t)total_tris, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(d_to, tri_offsets, sizeof(int) * (size_t)(n_meshes + 1), cudaMemcpyHostToDevice, s));
    if (d_vo) CK(cudaMemcpyAsync(d_vo, vert_offsets, sizeof(int) * (size_t)(n_meshes + 1), cudaMemcpyHostToDevice, s));
    if (n_tiles) {
        CK(cudaMemcpyAsync(d_tm, tile_mesh.data(), sizeof(int) * n_tiles, cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(d_tf, tile_first.data(), sizeof(int) * n_tiles, cudaMemcpyHostToDevice, s));
    }
    CK(cudaMemcpyAsync(d_mt0, mesh_tile0.data(), sizeof(int) * (n_meshes + 1), cudaMemcpyHostToDevice, s));
    if (n_tiles) {
        k_volume_tiles<<<n_tiles, VOL_NT, 0, s>>>(d_v, d_t, d_to, d_vo, d_tm, d_tf, n_tiles, d_part);
        ctx->launches++;
    }
    k_volume_reduce<<<(n_meshes + 127) / 128, 128, 0, s>>>(d_mt0, d_part, n_meshes, d_out);
    ctx->launches++;
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(out_volumes, d_out, sizeof(float) * n_meshes, cudaMemcpyDeviceToHost, s));
    return sync_and_check(ctx, "batch_mesh_volume");
}

extern "C" int gpu_test_mesh_volume(gpu_ctx_t ctx, const float* verts, int n_verts, const int* tris,
                                    int n_tris, float* out_volume)
{
    int to[2] = {0, n_tris};
    int vo[2] = {0, n_verts};
    return gpu_batch_mesh_volume(ctx, verts, n_verts, tris, n_tris, to, vo, 1, out_volume);
}

// ---------------------------------------------------------------------------
// Allocation throughput of the device arena on the workload of the
// reference's heap benchmark (bench/malloc_test_bench.cu:76-125, an
// mstress-style loop): `grid` blocks of 32 threads; thread 0 of each makes
// `iters` allocations of log-uniform sizes in [size_min, size_max]
// (xorshift32 draws, seeded per block) and keeps each in one of `slots`
// per-block slots.  The arena has no single free: the memory of a whole run
// is released by resetting the arena before the next one, as every
// evaluation and every lookahead wave does.  Allocations that do not fit are
// counted in fail.
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned bench_xorshift32(unsigned& r)
{
    r ^= r << 13; r ^= r >> 17; r ^= r << 5;
    return r;
}

__global__ void k_arena_mstress(Arena* a, void** slots, int n_slots, int iters, unsigned size_min, unsigned size_max,
                                float ln_min, float ln_delta, int* fail)
{
    if (threadIdx.x != 0) return;
    unsigned r = (unsigned)(blockIdx.x + 1) * 2654435761u;
    void** mine = slots + (size_t)blockIdx.x * n_slots;
    int nf = 0;
    for (int i = 0; i < iters; i++) {
        const int slot = (int)(bench_xorshift32(r) % (unsigned)n_slots);
        const float u = (float)(bench_xorshift32(r) >> 8) * (1.0f / 16777216.0f);
        unsigned sz = (unsigned)expf(ln_min + u * ln_delta);
        sz = min(max(sz, size_min), size_max);
        void* p = arena_alloc(a, sz, nullptr);
        if (!p) nf++;
        mine[slot] = p;
    }
    if (nf) atomicAdd(fail, nf);
}

extern "C" int cuacd_arena_bench(gpu_ctx_t ctx, int grid, int iters, int slots, unsigned size_min, unsigned size_max,
                                 unsigned long long arena_bytes, int warmup, int measure, float* out_mean_ms,
                                 float* out_std_ms, int* out_fail)
{
    if (!ctx || grid <= 0 || iters <= 0 || slots <= 0 || size_min == 0 || size_max < size_min || measure <= 0)
        return -1;
    CK(cudaSetDevice(ctx->device));
    const size_t slot_bytes = sizeof(void*) * (size_t)grid * slots;
    int rc = pool_begin(ctx, al256(slot_bytes) + al256(sizeof(int)) + arena_bytes + 4096);
    if (rc) return rc;
    void** d_slots = pool_take<void*>(ctx, (size_t)grid * slots);
    int* d_fail = pool_take<int>(ctx, 1);
    cudaStream_t s = ctx->stream;
    const float ln_min = logf((float)size_min), ln_delta = logf((float)size_max) - ln_min;
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    std::vector<float> ms;
    int fail = 0;
    for (int run = 0; run < warmup + measure; run++) {
        launch_arena_reset(ctx->d_arena, ctx->pool + ctx->carve, ctx->cap - ctx->carve, s);
        CK(cudaMemsetAsync(d_slots, 0, slot_bytes, s));
        CK(cudaMemsetAsync(d_fail, 0, sizeof(int), s));
        CK(cudaEventRecord(e0, s));
        k_arena_mstress<<<grid, 32, 0, s>>>(ctx->d_arena, d_slots, slots, iters, size_min, size_max, ln_min,
                                            ln_delta, d_fail);
        CK(cudaEventRecord(e1, s));
        CK(cudaEventSynchronize(e1));
        CK(cudaGetLastError());
        float t = 0.f;
        CK(cudaEventElapsedTime(&t, e0, e1));
        if (run >= warmup) ms.push_back(t);
        CK(cudaMemcpy(&fail, d_fail, sizeof(int), cudaMemcpyDeviceToHost));
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    double m = 0.0, v = 0.0;
    for (float t : ms) m += t;
    m /= ms.size();
    for (float t : ms) v += (t - m) * (t - m);
    v /= ms.size();
    if (out_mean_ms) *out_mean_ms = (float)m;
    if (out_std_ms) *out_std_ms = (float)sqrt(v);
    if (out_fail) *out_fail = fail;
    ctx->launches += (unsigned long long)(warmup + measure) * 2;
    return 0;
}

// ---------------------------------------------------------------------------
// entry points implemented in the remaining translation units
// ---------------------------------------------------------------------------

extern "C" int cuacd_hull_stats(gpu_ctx_t ctx, const float* pts, int total_pts, const int* offsets, int n_hulls,
                                int* out_nv, int* out_nt, float* out_vol, unsigned long long* out_stats)
{
    if (!ctx) return -1;
    int max_pts = 0;
    for (int i = 0; i < n_hulls; i++) max_pts = std::max(max_pts, offsets[i + 1] - offsets[i]);
    return hull_common(ctx, pts, total_pts, offsets, n_hulls, max_pts, max_pts, 2 * max_pts + 4,
                       nullptr, nullptr, out_nv, out_nt, out_vol, nullptr, out_stats);
}
