// launch.h — host-side launch wrappers shared between translation units.
#pragma once
#include <cuda_runtime.h>
#include <functional>
#include <vector>
#include "common.cuh"

struct CutResult;

// capi.cu
void launch_arena_reset(Arena* a, char* base, unsigned long long cap, cudaStream_t s);

// cut.cu
size_t cut_scratch_bytes(int nv, int nt);
void launch_cut_planes(const float* v, int nv, const int* t, int nt, const float4* planes, int n_planes,
                       Arena* arena, CutResult* res, cudaStream_t s);

// hausdorff.cu
struct HDSurf;
struct HDPrep;
size_t hd_pairs_scratch_bytes(int n_pairs, int max_nt_a, int max_nt_b);
size_t hd_dir_bytes();
void launch_hausdorff_pairs(const HDSurf* d_surfs, int n_pairs, Arena* arena, float resolution, int min_samples,
                            int total, HDPrep* d_preps, void* d_dirs, int* d_i2, float* d_pmax, int* d_err,
                            int n_sm, cudaStream_t s);
void launch_hausdorff_stages(const HDSurf* d_surfs, int n_pairs, Arena* arena, float resolution, int min_samples,
                             int total, HDPrep* d_preps, void* d_dirs, int* d_i2, float* d_pmax, int* d_err,
                             int n_sm, cudaStream_t s, const std::function<void(int)>& after);
void launch_hd_sqrt(const float* pmax, int n, float* out, int stride_floats, cudaStream_t s);
void launch_hd_prep_subset(const HDSurf* d_surfs, int n_pairs, int first, int step, Arena* arena, float resolution,
                           int min_samples, int total, HDPrep* d_preps, int* d_err, cudaStream_t s);
void launch_hd_plan_query(const HDSurf* d_surfs, int n_pairs, HDPrep* d_preps, void* d_dirs, int* d_i2,
                          float* d_pmax, int n_sm, cudaStream_t s, const std::function<void(int)>& after);

// components.cu
struct CompResult;
void launch_components(const HDSurf* d_meshes, int n, Arena* scratch, Arena* out, CompResult* res, cudaStream_t s);

// concave.cu
struct gpu_ctx;
int concave_planes_device_batch(gpu_ctx* ctx, int n, const float* const* d_v, const int* nv, const int* const* d_t,
                                const int* nt, int K, float eps, float thr, char* scr, size_t cap,
                                std::vector<std::vector<float4>>& out);

// hull.cu
struct HullJob;
struct HullRes;
struct HullState;
size_t hull_wrap_buf_bytes(int n_wrap_ctas);
#define HULL_TUNE_CLASSES 3
#define HULL_REDUCE_MAX_N 32768     // default: clouds of 4,097-32,768 points start with quarter-size tables
int hull_size_class(int max_pts);
// Wrap CTAs for a batch of total_points points whose largest cloud has
// max_pts (its size class picks the tuned points per CTA).
int hull_wrap_ctas(long long total_points, int n_sm, int max_pts = 1 << 30);
// Points that size the wrap grid of a batch of n_hulls clouds of at most
// max_pts points: small clouds count as 256 points each, so a batch of many
// tiny clouds still gets about one warp per cloud.
inline long long hull_wrap_points(int n_hulls, int max_pts)
{
    return (long long)n_hulls * (max_pts > 256 ? max_pts : 256);
}
// reduce = false: every cloud starts with full-size tables (one round).
void launch_hull_jobs(const HullJob* d_jobs, int n_jobs, HullState* d_states, HullRes* d_res, Arena* scratch,
                      Arena* out, int* d_ctl, int* d_wbuf, int n_wrap_ctas, unsigned long long* d_stats,
                      cudaStream_t s, int max_pts, bool reduce = true);
void launch_jobs_from_offsets(const float* d_pts, const int* d_off, int n, float* d_v, int* d_t, int max_hv,
                              int max_ht, HullJob* d_jobs, cudaStream_t s);
void launch_unpack_results(const HullRes* d_res, int n, int* d_nv, int* d_nt, float* d_vol, int* d_err, cudaStream_t s);

// scorer.cu
struct cuacd_scorer;
struct ScorerPart { const float* v; const int* t; int nv, nt; float hull_vol; int off, n; };
// Predicted scores (score units) of planes d_planes[p.off, p.off + p.n) of
// each part p into pred[0, n_rows) (host); synchronises `s`.
int scorer_predict_parts(gpu_ctx* ctx, cuacd_scorer* sc, const ScorerPart* parts, int n_parts,
                         const float4* d_planes, int n_rows, float* pred, cudaStream_t s);
// Feature rows of the last scorer_predict_parts call (n_rows x n_features floats) to the host.
int scorer_copy_features(gpu_ctx* ctx, cuacd_scorer* sc, int n_rows, float* out, cudaStream_t s);
int scorer_n_features();

// eval.cu: exact evaluation of the planes a selection keeps, the cut of all
// planes overlapping the selection (eval_precut_begin / eval_precut_finish,
// declared in context.cuh)
struct EvalWork;
struct EvalPrecut { EvalWork* W = nullptr; CutResult* all_cuts = nullptr; int n = 0, nwc = 0; };
