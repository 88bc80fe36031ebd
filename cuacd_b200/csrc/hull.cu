// hull.cu — kernels and launcher of the batched hull pipeline (hull.cuh):
// set-up (one CTA per cloud), shares of the wrap grid, persistent wrapping
// (up to one CTA per SM; each CTA wraps its home cloud, then helps others),
// output (one CTA per cloud).
#include <mutex>
#include "context.cuh"
#include "hull.cuh"
#include "hull_kernels.cuh"
#include "launch.h"

__global__ void __launch_bounds__(HULL_NT)
k_hull_setup(const HullJob* __restrict__ jobs, int n_jobs, Arena* scratch, HullState* states, int* ctl,
             int seed_min_n, int retry_round, int reduce_max_n)
{
    hull_setup_body(jobs, n_jobs, scratch, states, ctl, seed_min_n, retry_round, reduce_max_n);
}

// Wrap-grid shares (one CTA): prefix of the active hulls' weights, a hull's
// point count plus a floor.  With H active hulls and G > H wrap CTAs the
// floor ceil(sum n / (G - H)) makes every share at least one CTA spacing
// wide, so every hull has a home CTA from the start.
__global__ void __launch_bounds__(1024)
k_hull_assign(HullState* states, int n_jobs, int n_ctas, long long* total)
{
    hull_assign_body(states, n_jobs, n_ctas, total);
}

__global__ void __launch_bounds__(HULL_NT, 1)
k_hull_wrap(HullState* states, int n_jobs, int* ctl, const long long* total, int* wbuf)
{
    extern __shared__ int wsm_dyn[];                      // HULL_WRAP_DSMEM bytes
    hull_wrap_body(states, n_jobs, ctl, total, wbuf, wsm_dyn);
}

__global__ void __launch_bounds__(HULL_NT)
k_hull_output(const HullJob* __restrict__ jobs, HullState* states, int n_jobs, Arena* out, const int* ctl,
              HullRes* res, unsigned long long* stats, int retry_round)
{
    hull_output_body(jobs, states, n_jobs, out, ctl, res, stats, retry_round);
}

size_t hull_wrap_buf_bytes(int n_wrap_ctas)
{
    return (size_t)n_wrap_ctas * (HULL_NT / 32) * 2 * HULL_SGCAP * sizeof(int);
}

// Opt in to the wrap kernel's dynamic shared memory (once per process and
// device) and return its resident CTAs per SM.
static int hull_wrap_per_sm()
{
    static int cached[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) dev = 0;
    if (cached[dev] <= 0) {
        cudaFuncSetAttribute(k_hull_wrap, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)HULL_WRAP_DSMEM);
        int b = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_hull_wrap, HULL_NT, HULL_WRAP_DSMEM) != cudaSuccess || b < 1)
            b = 1;
        cached[dev] = b;
    }
    return cached[dev];
}

// Tuned launch shape per size class of a batch's largest cloud (< 4,096
// points, < 65,536, larger): points of the batch per wrap CTA (so warps per
// cloud) and the cloud size from which wrapping starts at HULL_SEEDS seed
// faces.  Per device; the defaults hold until cuacd_hull_set_tuning (the
// autotuner, cuacd_b200/autotune.py) replaces them.
struct HullTune { int pts_per_cta, seed_min_n, reduce_max_n; };
static HullTune g_hull_tune[64][HULL_TUNE_CLASSES] = {};
static std::mutex g_hull_tune_mu;

static int cur_device()
{
    int dev = 0;
    cudaGetDevice(&dev);
    return dev >= 0 && dev < 64 ? dev : 0;
}

int hull_size_class(int max_pts) { return max_pts < 4096 ? 0 : (max_pts < 65536 ? 1 : 2); }

static HullTune hull_tune(int cls)
{
    std::lock_guard<std::mutex> lock(g_hull_tune_mu);
    HullTune t = g_hull_tune[cur_device()][cls];
    if (t.pts_per_cta <= 0) t.pts_per_cta = 4096;
    if (t.seed_min_n <= 0) t.seed_min_n = 1 << 30;
    if (t.reduce_max_n <= 0) t.reduce_max_n = HULL_REDUCE_MAX_N;
    return t;
}

extern "C" int cuacd_hull_set_tuning(gpu_ctx_t ctx, int size_class, int pts_per_cta, int seed_min_n)
{
    if (!ctx || size_class < 0 || size_class >= HULL_TUNE_CLASSES || pts_per_cta < 0 || seed_min_n < 0) return -1;
    cudaSetDevice(ctx->device);
    std::lock_guard<std::mutex> lock(g_hull_tune_mu);
    HullTune& t = g_hull_tune[ctx->device >= 0 && ctx->device < 64 ? ctx->device : 0][size_class];
    t.pts_per_cta = pts_per_cta; t.seed_min_n = seed_min_n;
    return 0;
}

extern "C" int cuacd_hull_get_tuning(gpu_ctx_t ctx, int size_class, int* pts_per_cta, int* seed_min_n)
{
    if (!ctx || size_class < 0 || size_class >= HULL_TUNE_CLASSES || !pts_per_cta || !seed_min_n) return -1;
    cudaSetDevice(ctx->device);
    const HullTune t = hull_tune(size_class);
    *pts_per_cta = t.pts_per_cta; *seed_min_n = t.seed_min_n;
    return 0;
}

extern "C" int cuacd_hull_set_table_limit(gpu_ctx_t ctx, int size_class, int reduce_max_n)
{
    if (!ctx || size_class < 0 || size_class >= HULL_TUNE_CLASSES || reduce_max_n < 0) return -1;
    cudaSetDevice(ctx->device);
    std::lock_guard<std::mutex> lock(g_hull_tune_mu);
    g_hull_tune[ctx->device >= 0 && ctx->device < 64 ? ctx->device : 0][size_class].reduce_max_n = reduce_max_n;
    return 0;
}

extern "C" int cuacd_hull_get_table_limit(gpu_ctx_t ctx, int size_class, int* reduce_max_n)
{
    if (!ctx || size_class < 0 || size_class >= HULL_TUNE_CLASSES || !reduce_max_n) return -1;
    cudaSetDevice(ctx->device);
    *reduce_max_n = hull_tune(size_class).reduce_max_n;
    return 0;
}

// Wrap grid size: total_points / the tuned points per CTA of the class of
// max_pts (default 4,096: about one warp per 256 points), at most the
// resident CTAs of the whole device.
int hull_wrap_ctas(long long total_points, int n_sm, int max_pts)
{
    const int ppc = hull_tune(hull_size_class(max_pts)).pts_per_cta;
    long long c = (total_points + ppc - 1) / ppc;
    const long long cap = (long long)n_sm * hull_wrap_per_sm();
    if (c < 1) c = 1;
    if (c > cap) c = cap;
    return (int)c;
}

void launch_hull_jobs(const HullJob* d_jobs, int n_jobs, HullState* d_states, HullRes* d_res, Arena* scratch,
                      Arena* out, int* d_ctl, int* d_wbuf, int n_wrap_ctas, unsigned long long* d_stats,
                      cudaStream_t s, int max_pts, bool reduce)
{
    if (n_jobs <= 0) return;
    HullTune tune = hull_tune(hull_size_class(max_pts));
    if (!reduce) tune.reduce_max_n = HULL_FIRST_CAP;
    const int seed_min_n = tune.seed_min_n;
    hull_wrap_per_sm();                                   // dynamic shared memory opt-in
    // round 0 builds every cloud with first-attempt tables; round 1 (only
    // launched when a cloud of the batch can outgrow them) rebuilds the
    // clouds whose tables overflowed at full capacity -- its kernels return
    // at once when there are none
    const int rounds = max_pts > HULL_FIRST_CAP && tune.reduce_max_n > HULL_FIRST_CAP ? 2 : 1;
    for (int r = 0; r < rounds; r++) {
        cudaMemsetAsync(d_ctl, 0, 4 * sizeof(int), s);
        k_hull_setup<<<n_jobs, HULL_NT, 0, s>>>(d_jobs, n_jobs, scratch, d_states, d_ctl, seed_min_n, r,
                                                tune.reduce_max_n);
        k_hull_assign<<<1, 1024, 0, s>>>(d_states, n_jobs, n_wrap_ctas, (long long*)(d_ctl + 2));
        k_hull_wrap<<<n_wrap_ctas, HULL_NT, HULL_WRAP_DSMEM, s>>>(d_states, n_jobs, d_ctl,
                                                                 (const long long*)(d_ctl + 2), d_wbuf);
        k_hull_output<<<n_jobs, HULL_NT, 0, s>>>(d_jobs, d_states, n_jobs, out, d_ctl, d_res, d_stats, r);
    }
}

// Jobs for clouds packed back to back (offsets), outputs in fixed slots.
__global__ void k_jobs_from_offsets(const float* pts, const int* offsets, int n, float* out_v, int* out_t,
                                    int max_hv, int max_ht, HullJob* jobs)
{
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    HullJob J;
    J.pts = pts + 3 * (size_t)offsets[j]; J.n = offsets[j + 1] - offsets[j];
    J.tris = nullptr; J.nt = 0;
    J.out_v = out_v + 3 * (size_t)j * max_hv; J.out_t = out_t + 3 * (size_t)j * max_ht;
    J.max_hv = max_hv; J.max_ht = max_ht;
    jobs[j] = J;
}

__global__ void k_unpack_results(const HullRes* res, int n, int* out_nv, int* out_nt, float* out_vol, int* out_err)
{
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    HullRes r = res[j];
    out_nv[j] = r.hnv; out_nt[j] = r.hnt;
    if (out_vol) out_vol[j] = r.hull_vol;
    if (out_err) out_err[j] = r.err;
}

void launch_jobs_from_offsets(const float* d_pts, const int* d_off, int n, float* d_v, int* d_t, int max_hv,
                              int max_ht, HullJob* d_jobs, cudaStream_t s)
{
    if (n > 0) k_jobs_from_offsets<<<(n + 127) / 128, 128, 0, s>>>(d_pts, d_off, n, d_v, d_t, max_hv, max_ht, d_jobs);
}

void launch_unpack_results(const HullRes* d_res, int n, int* d_nv, int* d_nt, float* d_vol, int* d_err, cudaStream_t s)
{
    if (n > 0) k_unpack_results<<<(n + 127) / 128, 128, 0, s>>>(d_res, n, d_nv, d_nt, d_vol, d_err);
}
