/*
 * cuacd_b200.h — C ABI of libcuacd_b200.so, the B200 (sm_100a) engine for
 * cuacd's lookahead candidate-evaluation path.
 *
 * The gpu_* / lookahead_decompose entry points keep the names, argument order,
 * meaning and return conventions of the reference's host layer, so the
 * reference's CPython module (csrc/module.c) can link against this library in
 * place of csrc/heap.c, csrc/test.c and csrc/lookahead.c:
 *   - every pointer is a HOST pointer; the call copies in, computes, copies
 *     out and synchronises before returning;
 *   - return 0 on success, otherwise a CUDA error code or a device error word
 *     (KERR_* bit flags, layout of the reference's cuda/error_codes.cuh:14-53);
 *     the message is available from gpu_last_error();
 *   - per-item error words go to out_errors.
 * The cuacd_* entry points are additions for callers that keep data on the
 * device (device pointers + a CUDA stream) and for the candidate evaluator.
 */
#ifndef CUACD_B200_H
#define CUACD_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct gpu_ctx* gpu_ctx_t;

/* ---- context and pool (reference csrc/heap.h:19-50) ---------------------- */

/* Replaces gpu_set_fatbin (csrc/heap.h:19).  The kernels are linked into this
 * library, so the blob is ignored; kept so existing callers still link. */
void gpu_set_fatbin(const void* data, size_t len);

/* Replaces gpu_init (csrc/heap.h:26).  device_ordinal < 0 keeps the calling
 * thread's current device.  pool_bytes = 0 lets the device pool grow on
 * demand; > 0 fixes its capacity. */
int  gpu_init(gpu_ctx_t* ctx, int device_ordinal, size_t pool_bytes);
/* Replaces gpu_destroy (csrc/heap.h:27). */
void gpu_destroy(gpu_ctx_t ctx);
/* Replaces gpu_last_error (csrc/heap.h:29). */
const char* gpu_last_error(gpu_ctx_t ctx);
/* Replaces gpu_heap_compact (csrc/heap.h:34); a no-op, as in the reference
 * (csrc/heap.c:274-277): the pool is an arena reset between calls. */
int  gpu_heap_compact(gpu_ctx_t ctx);
/* Replaces gpu_pool_usage (csrc/heap.h:40): high-water mark of pool bytes. */
size_t gpu_pool_usage(gpu_ctx_t ctx);
/* Replaces gpu_heap_stats (csrc/heap.h:45).  out = {output bytes live,
 * output allocations, output releases, scratch bytes live, scratch
 * allocations, scratch releases}. */
int gpu_heap_stats(gpu_ctx_t ctx, unsigned long long out[6]);

/* ---- batch kernels (reference csrc/test.h) ------------------------------- */

/* Replaces gpu_hull_dandc (csrc/test.h:30-43): exact convex hull of each
 * cloud.  Corners are the input floats in ascending input order; triangles
 * index into them (per-hull relative), canonical order. */
int gpu_hull_dandc(gpu_ctx_t ctx, const float* pts, int total_pts,
                   const int* offsets, int n_hulls, int max_pts_per_hull,
                   int max_hull_verts, int max_hull_tris,
                   float* out_verts, int* out_tris, int* out_nv, int* out_nt,
                   int* out_errors);

/* Replaces gpu_test_mesh_volume (csrc/test.h:48-54). */
int gpu_test_mesh_volume(gpu_ctx_t ctx, const float* verts, int n_verts,
                         const int* tris, int n_tris, float* out_volume);

/* Replaces gpu_batch_mesh_volume (csrc/test.h:64-73). vert_offsets may be
 * NULL (all meshes index one shared vertex array). */
int gpu_batch_mesh_volume(gpu_ctx_t ctx, const float* verts, int total_verts,
                          const int* tris, int total_tris,
                          const int* tri_offsets, const int* vert_offsets,
                          int n_meshes, float* out_volumes);

/* Replaces gpu_kdop_hull (csrc/test.h:78-91): the same exact hull (the
 * reference's extreme-point prefilter is subsumed by the BVH search) plus
 * its volume. */
int gpu_kdop_hull(gpu_ctx_t ctx, const float* pts, int total_pts,
                  const int* offsets, int n_hulls,
                  int max_hull_verts, int max_hull_tris,
                  float* out_verts, int* out_tris, int* out_nv, int* out_nt,
                  float* out_volumes, int* out_errors);

/* Replaces gpu_test_hausdorff (csrc/test.h:96-102): bidirectional sampled
 * Hausdorff distance (2000 samples per unit area, at least 1000). */
int gpu_test_hausdorff(gpu_ctx_t ctx,
                       const float* hull_verts, int hull_nv,
                       const int* hull_tris, int hull_nt,
                       const float* mesh_verts, int mesh_nv,
                       const int* mesh_tris, int mesh_nt,
                       float* out_hausdorff);

/* Replaces gpu_test_plane_cut (csrc/test.h:112-122): cut a closed mesh by
 * pa*x+pb*y+pc_n*z+pd = 0 and cap both halves. */
int gpu_test_plane_cut(gpu_ctx_t ctx,
                       const float* vertices, int n_verts,
                       const int* triangles, int n_tris,
                       float pa, float pb, float pc_n, float pd,
                       float* out_pos_verts, int out_pos_verts_cap,
                       int* out_pos_tris, int out_pos_tris_cap,
                       float* out_neg_verts, int out_neg_verts_cap,
                       int* out_neg_tris, int out_neg_tris_cap,
                       int* out_n_pv, int* out_n_pt,
                       int* out_n_nv, int* out_n_nt);

/* Replaces gpu_mesh_audit (csrc/test.h:124-132): topology audit of a
 * triangle mesh, *out_flags = a bitmask of the reference's verdict bits
 * (cuda/mesh_audit.cuh:21-26): a zero-area or repeated-index triangle, an
 * index outside [0, n_verts) (that triangle is skipped), an edge used by one
 * triangle, by more than two, or by two in the same direction. */
#define CUACD_MAV_OK          0u
#define CUACD_MAV_DEGEN_TRI   (1u << 0)
#define CUACD_MAV_BAD_INDEX   (1u << 1)
#define CUACD_MAV_OPEN_EDGE   (1u << 2)
#define CUACD_MAV_NONMANIFOLD (1u << 3)
#define CUACD_MAV_FLIPPED     (1u << 4)
int gpu_mesh_audit(gpu_ctx_t ctx, const float* verts, int n_verts, const int* tris, int n_tris,
                   unsigned int* out_flags);

/* Replaces gpu_preprocess (csrc/preprocess.h:17-24): remesh a triangle
 * soup into a watertight, manifold, consistently oriented surface on a
 * resolution^3 grid (a power of two in [8, 1024]) -- distance field within
 * 3 cells of the triangles, signed by a flood fill from the grid boundary,
 * moved out by 0.9 cells, contoured by marching cubes.  *out_verts /
 * *out_tris are malloc'd (the caller frees them with free()); returns 0, 1
 * for bad arguments (a null pointer, an empty mesh, an index outside
 * [0, nv), a non-finite coordinate, a bad resolution, no extent), or a
 * KERR_* / CUDA error. */
int gpu_preprocess(gpu_ctx_t ctx, const float* verts, int nv, const int* tris, int nt,
                   int resolution, float** out_verts, int* out_nv, int** out_tris, int* out_nt);


/* Replaces gpu_test_postprocess_dc (csrc/postprocess.h:20-27): split a mesh
 * into its vertex-connected components.  Component c's vertices go to
 * out_verts[c*max_verts_per*3 ...] and its triangles (component-local
 * indices) to out_tris[c*max_tris_per*3 ...]; components are numbered by
 * their smallest input vertex, vertices and triangles keep input order.
 * Components with negative signed volume (inner shells) are dropped when
 * outer shells exist.  A mesh that is one component comes back unchanged
 * as component 0; an empty mesh gives 0 components.  Buffers too small for
 * the result: non-zero return, message from gpu_last_error. */
int gpu_test_postprocess_dc(gpu_ctx_t ctx,
                            const float* verts, int n_verts,
                            const int* tris, int n_tris,
                            int max_components, int max_verts_per, int max_tris_per,
                            float* out_verts, int* out_tris,
                            int* out_nv, int* out_nt,
                            int* out_n_components);

/* Replaces gpu_test_warp_sort (csrc/test.h:19-20): sort each sub-array of
 * (x,y,z,index) int records by (y,x,z,index) in place. */
int gpu_test_warp_sort(gpu_ctx_t ctx, int* points, int total_pts,
                       const int* offsets, int n_arrays);

/* ---- candidate evaluator (additions) ------------------------------------- */

/* Per-candidate result of cut + volumes + hulls (+ Hausdorff). */
typedef struct {
    int   ok;              /* both halves non-empty */
    int   nv[2], nt[2];    /* fragment sizes (pos, neg), caps included */
    int   n_cap;           /* cap triangles */
    int   hull_nv[2], hull_nt[2];
    float mesh_vol[2], hull_vol[2], hausdorff[2];
    float cost_rv[2], cost_full[2];
    float score_rv, score_full;   /* worst part cost of the candidate */
    int   err;             /* KERR_* bits raised for this candidate */
} cuacd_cand_result;

#define CUACD_EVAL_HAUSDORFF 1

/* Evaluate n_planes candidate planes (4 floats each) on one closed mesh:
 * cut with caps, volume of both halves, exact hull of both halves,
 * optionally the sampled Hausdorff distance fragment<->hull, and the part
 * costs of cuda/la_common.cuh:21-34.  Host pointers.  hd_resolution <= 0
 * selects the reference defaults (2000 per unit area, min 1000 samples);
 * hd_total > 0 fixes the per-surface sample budget instead. */
int cuacd_eval_candidates(gpu_ctx_t ctx, const float* verts, int nv,
                          const int* tris, int nt, const float* planes,
                          int n_planes, int flags, float hd_resolution,
                          int hd_min_samples, int hd_total,
                          cuacd_cand_result* out);

/* Same with device pointers on `stream` (cudaStream_t as void*); results
 * stay on the device in d_out.  Does not synchronise. */
int cuacd_eval_candidates_device(gpu_ctx_t ctx, const float* d_verts, int nv,
                                 const int* d_tris, int nt,
                                 const float* d_planes, int n_planes, int flags,
                                 float hd_resolution, int hd_min_samples,
                                 int hd_total, cuacd_cand_result* d_out,
                                 void* stream);

/* Candidate planes of one mesh (host pointers): the concave-edge planes of
 * la_find_concave_edges (cuda/la_concave.cu:48-363; up to 4 per sampled
 * edge, written first, count in *out_n_concave) followed by the `width`
 * axis-aligned cuts of la_axis_cut_candidate/la_expand
 * (cuda/la_axis_cut.cuh:10-19, cuda/la_expand.cu:182-199), 4 floats each.
 * out_planes holds 4*n_concave_edges + width planes; out_axis_valid[i] = 0
 * marks an axis too narrow to cut (its plane is all zeros). */
int cuacd_candidate_planes(gpu_ctx_t ctx, const float* verts, int nv,
                           const int* tris, int nt, int n_concave_edges,
                           float concave_eps, float concave_threshold,
                           int width, float min_edge_dist, float* out_planes,
                           int* out_n_concave, int* out_axis_valid);

/* Hausdorff with an explicit sample budget (config of a fixed total), host
 * pointers. */
int cuacd_hausdorff(gpu_ctx_t ctx,
                    const float* a_verts, int a_nv, const int* a_tris, int a_nt,
                    const float* b_verts, int b_nv, const int* b_tris, int b_nt,
                    float resolution, int min_samples, int total,
                    float* out_hausdorff);


/* Batched Hausdorff distance of n_pairs mesh pairs (A_i, B_i), each stage
 * launched once for the whole batch.  Replaces the reference's batch of
 * hausdorff_block calls, one block per pair (bench/hausdorff_bench.cu:253-345;
 * la_hausdorff_parts in cuda/la_lifecycle.cu), with the sampling rule of
 * gpu_test_hausdorff (csrc/test.h:96-102).  Meshes are packed back to back:
 * vertex offsets voff[n_pairs+1] and triangle offsets toff[n_pairs+1] (host
 * arrays, starting at 0), triangle indices local to their mesh.  Host
 * variant: host arrays in, out_hausdorff[n_pairs] on the host.  Device
 * variant: vertex/triangle arrays and d_out on the device, offsets on the
 * host, work on `stream` (NULL: the context's), synchronised before return;
 * the caller guarantees the indices are in range. */
int cuacd_hausdorff_batch(gpu_ctx_t ctx, int n_pairs,
                          const float* a_verts, const int* a_voff, const int* a_tris, const int* a_toff,
                          const float* b_verts, const int* b_voff, const int* b_tris, const int* b_toff,
                          float resolution, int min_samples, int total, float* out_hausdorff);
int cuacd_hausdorff_batch_device(gpu_ctx_t ctx, int n_pairs,
                                 const float* d_a_verts, const int* a_voff, const int* d_a_tris,
                                 const int* a_toff, const float* d_b_verts, const int* b_voff,
                                 const int* d_b_tris, const int* b_toff, float resolution,
                                 int min_samples, int total, float* d_out, void* stream);

/* Allocation-free Hausdorff distance (no counterpart in the reference).
 * For callers that cannot allocate device memory — plugins inside a host
 * framework that owns all device allocations, or code where cudaMalloc is
 * not allowed — and so cannot create a gpu_ctx_t either: no context, no
 * cudaMalloc/cudaFree, no allocating library call.  Inputs and the output
 * (one float) are device pointers the caller owns; work is enqueued on
 * `stream` (cudaStream_t as void*, NULL = legacy default stream) and the call
 * does not synchronise.  Scratch is a static 32 MiB device array held by
 * every GPU that loads this library until exit; all calls share it, so calls
 * whose work overlaps on the GPU race.  The first call on a device looks up
 * the array's device address and keeps it for the life of the process;
 * make that first call before any stream capture, and do not use the entry
 * point on a device after cudaDeviceReset (the kept address is stale).
 * Every triangle index must lie in [0, nv) of its surface; a device-side scan
 * checks this before any kernel reads through the indices.  Returns 0,
 * CUACD_NOALLOC_TOO_LARGE when the two surfaces' prep data would not fit
 * (two surfaces of up to 161,000 triangles each fit; the exact test is the
 * sum of both surfaces' per-triangle prep sizes; more than 2^20 triangles on
 * a surface is refused before any sizing), CUACD_NOALLOC_BAD_ARGS, or a CUDA
 * error code.  A failure found on the device (an index out of range, scratch
 * overflow) cannot be returned by a call that does not synchronise: *d_out
 * is then NaN, never a distance. */
#define CUACD_NOALLOC_TOO_LARGE (-2)
#define CUACD_NOALLOC_BAD_ARGS  (-3)
int cuacd_hausdorff_noalloc(const float* d_a_verts, int a_nv,
                            const int* d_a_tris, int a_nt,
                            const float* d_b_verts, int b_nv,
                            const int* d_b_tris, int b_nt,
                            float resolution, int min_samples, int total,
                            float* d_out, void* stream);

/* Device-pointer batch hull for callers with resident data (used by the
 * benchmark's device-resident leg).  Does not synchronise. */
int cuacd_hull_batch_device(gpu_ctx_t ctx, const float* d_pts,
                            const int* d_offsets, int n_hulls, int max_pts,
                            int max_hull_verts, int max_hull_tris,
                            float* d_out_verts, int* d_out_tris,
                            int* d_out_nv, int* d_out_nt, float* d_out_vol,
                            int* d_out_errors, void* stream);


/* Launch-shape tuning of the batched hull pipeline (no counterpart in the
 * reference, whose launch shapes are fixed: csrc/lookahead.c:572-573,
 * 606-607).  Per device and per size class of a batch's largest cloud
 * (0: < 4,096 points, 1: < 65,536, 2: larger): pts_per_cta = points of the
 * batch per wrap CTA, i.e. how many warps share a cloud (0: the default
 * 4,096); seed_min_n = clouds of at least this many points start wrapping
 * from six seed faces instead of one (0: never).  cuacd_b200/autotune.py
 * sweeps both with CUDA-event timing and stores the best per device. */
int cuacd_hull_set_tuning(gpu_ctx_t ctx, int size_class, int pts_per_cta, int seed_min_n);
int cuacd_hull_get_tuning(gpu_ctx_t ctx, int size_class, int* pts_per_cta, int* seed_min_n);

/* Table sizing of the candidate evaluator's fragment hulls, per size class
 * (no counterpart in the reference): a fragment of 4,097 to reduce_max_n
 * points first builds in tables for a quarter of its points (at least
 * 4,096) and only one whose hull outgrows them is built again at full size;
 * larger fragments start at full size (0: the default 32,768).  The public
 * batch hull calls and the lookahead search always start at full size. */
int cuacd_hull_set_table_limit(gpu_ctx_t ctx, int size_class, int reduce_max_n);
int cuacd_hull_get_table_limit(gpu_ctx_t ctx, int size_class, int* reduce_max_n);

/* The context's device: its name (NUL-terminated, at most cap bytes) and
 * streaming multiprocessor count (no counterpart in the reference). */
int cuacd_device_info(gpu_ctx_t ctx, char* name, int cap, int* n_sm);


/* Number of kernel launches issued by this context so far (a counter the
 * benchmark reads around its timed region). */
unsigned long long cuacd_launch_count(gpu_ctx_t ctx);

/* Per-stage timing of the candidate evaluator: when enabled, CUDA events are
 * recorded on the evaluator's stream between its launches.  After a call,
 * cuacd_stage_times fills ms[i] (i < CUACD_N_STAGES, in launch order: cut,
 * fragment hull+volume, Hausdorff prep, Hausdorff plan, Hausdorff query,
 * finish) for the last evaluation; it synchronises on the last event. */
#define CUACD_N_STAGES 6
int cuacd_profile_stages(gpu_ctx_t ctx, int enable);
int cuacd_stage_times(gpu_ctx_t ctx, float* ms_out);

/* ---- learned candidate scorer (no counterpart in the reference) ---------- */

/* A 240-256-256-1 MLP (BF16 operands, FP32 accumulation, ReLU) that
 * predicts a candidate plane's score_full from cuacd_candidate_features.
 * Parameters are FP32 master copies, flattened as W1[240][256], b1[256],
 * W2[256][256], b2[256], W3[256], b3[1] (row k of W holds input k's
 * weights).  The loss is the mean squared error of (prediction - target)
 * scaled by 10. */
typedef struct cuacd_scorer* cuacd_scorer_t;
int  cuacd_scorer_n_params(void);
int  cuacd_scorer_n_features(void);
int  cuacd_scorer_create(gpu_ctx_t ctx, unsigned seed, cuacd_scorer_t* out);
void cuacd_scorer_free(cuacd_scorer_t s);
/* set_params also resets the optimizer state. */
int  cuacd_scorer_set_params(cuacd_scorer_t s, const float* params);
int  cuacd_scorer_get_params(cuacd_scorer_t s, float* params);
/* Feature standardisation applied before the first layer, x' = (x - mean) *
 * inv_std (n_features floats each; identity after create). */
int  cuacd_scorer_set_normalizer(cuacd_scorer_t s, const float* mean, const float* inv_std);
int  cuacd_scorer_get_normalizer(cuacd_scorer_t s, float* mean, float* inv_std);

/* Feature rows (n_features floats each) of n planes on one part; hull_vol is
 * the part's convex-hull volume. */
int cuacd_candidate_features(gpu_ctx_t ctx, cuacd_scorer_t s, const float* verts, int nv,
                             const int* tris, int nt, float hull_vol,
                             const float* planes, int n, float* out);

/* Loss and parameter gradients (n_params floats) of one batch of n rows. */
int cuacd_scorer_grad(gpu_ctx_t ctx, cuacd_scorer_t s, const float* X, const float* T,
                      int n, float* loss, float* grads);

/* AdamW (beta 0.9/0.999, eps 1e-8, decoupled weight decay wd on weights)
 * over `epochs` shuffled passes of n rows in batches of `batch`; rows stay
 * on the device.  *final_loss: mean unscaled MSE over the last epoch. */
int cuacd_scorer_train(gpu_ctx_t ctx, cuacd_scorer_t s, const float* X, const float* T,
                       int n, int epochs, int batch, float lr, float wd,
                       unsigned seed, float* final_loss);

int cuacd_scorer_predict(gpu_ctx_t ctx, cuacd_scorer_t s, const float* X, int n, float* out);


/* Surrogate-pruned evaluation (at most 1024 planes): predicted scores for
 * all planes, the exact evaluator for the top_k best predictions plus every
 * plane predicted within `margin` of the k-th.  Unevaluated planes get
 * ok = 0 and scores FLT_MAX.  hull_vol < 0 computes the part's hull volume.
 * Runs the device-pointer form on staged copies of the inputs; kept planes
 * that meet a full arena are evaluated again through cuacd_eval_candidates,
 * which grows the pool. */
int cuacd_eval_candidates_pruned(gpu_ctx_t ctx, cuacd_scorer_t s, const float* verts, int nv,
                                 const int* tris, int nt, float hull_vol,
                                 const float* planes, int n_planes, int flags,
                                 float hd_resolution, int hd_min_samples, int hd_total,
                                 int top_k, float margin, cuacd_cand_result* out,
                                 float* out_pred, int* out_evaluated, int* out_n_evaluated);

/* Device-pointer form on `stream` (at most 1024 planes): features, network,
 * selection and the scatter of results run on the device, and the cuts of
 * all planes run on a second stream while the network ranks them; the call
 * waits once for the selected count, then launches the remaining exact
 * stages on the selected planes and returns without synchronising.  d_pred and
 * d_evaluated may be NULL; hull_vol must be the part's hull volume. */
int cuacd_eval_candidates_pruned_device(gpu_ctx_t ctx, cuacd_scorer_t s, const float* d_verts, int nv,
                                        const int* d_tris, int nt, float hull_vol,
                                        const float* d_planes, int n_planes, int flags,
                                        float hd_resolution, int hd_min_samples, int hd_total,
                                        int top_k, float margin, cuacd_cand_result* d_out,
                                        float* d_pred, int* d_evaluated, int* out_n_evaluated,
                                        void* stream);

/* ---- lookahead search (reference csrc/lookahead.h, csrc/heap.h) ---------- */

struct gpu_part_result {
    float* verts;       /* malloc'd, nv*3 floats */
    int*   tris;        /* malloc'd, nt*3 ints */
    int    nv;
    int    nt;
    float* hull_verts;  /* malloc'd, hull_nv*3 floats */
    int*   hull_tris;   /* malloc'd, hull_nt*3 ints */
    int    hull_nv;
    int    hull_nt;
    float  mesh_vol;
    float  hull_vol;
    float  hausdorff;
};

struct gpu_result {
    struct gpu_part_result* parts;
    int nparts;
};

/* Replaces gpu_result_free (csrc/heap.h:85). */
void gpu_result_free(struct gpu_result* result);

/* Replaces lookahead_decompose (csrc/lookahead.h:28-43).  quick_depth adds
 * the reference's quick levels after the `depth` full ones
 * (cuda/la_refine.cu:52-351); the last level runs the reference's branch and
 * bound (cuda/la_expand.cu:380-457), with the path bound taken per cutting
 * part; merge_hulls runs the merge-hulls post-pass
 * (cuda/postprocess_merge.cu:41-679). */
int lookahead_decompose(gpu_ctx_t ctx,
                        const float* verts, int nv, const int* tris, int nt,
                        const float* hull_verts, int hull_nv,
                        const int* hull_tris, int hull_nt,
                        int max_iters, int width, int width2, float threshold,
                        int depth, int quick_depth, int max_n_cutting,
                        int verbose, int debug, int decompose_components,
                        int decompose_components_per_iter,
                        int n_concave_edges, float concave_eps,
                        float concave_threshold, int concave_iters,
                        int merge_hulls, struct gpu_result* out);

/* lookahead_decompose with pruning (no counterpart in the reference).  With
 * a scorer, it ranks each cutting part's level-0 planes and only the top_k,
 * plus every plane predicted within `margin` of the k-th, are cut and scored
 * exactly (scorer NULL: all are).  With beam > 0, only the `beam` level-0
 * cuts of each part with the lowest exact level-0 cost are expanded to the
 * next level.  Deeper levels, the choice of the cut and every part cost stay
 * exact.  out_stats (optional, 3 values): level-0 planes ranked, planes cut,
 * level-0 cuts expanded.  Other arguments as lookahead_decompose. */
int cuacd_lookahead_decompose_pruned(gpu_ctx_t ctx, cuacd_scorer_t scorer, int top_k, float margin,
                                     int beam, unsigned long long* out_stats,
                                     const float* verts, int nv, const int* tris, int nt,
                                     const float* hull_verts, int hull_nv,
                                     const int* hull_tris, int hull_nt,
                                     int max_iters, int width, int width2, float threshold,
                                     int depth, int max_n_cutting, int verbose,
                                     int decompose_components, int decompose_components_per_iter,
                                     int n_concave_edges, float concave_eps,
                                     float concave_threshold, int concave_iters,
                                     struct gpu_result* out);

/* lookahead_decompose over a batch of meshes (no counterpart in the
 * reference, whose call takes one mesh).  Mesh m is vertices
 * [vert_off[m], vert_off[m+1]) and triangles [tri_off[m], tri_off[m+1]) of
 * the packed arrays, with indices relative to its own first vertex; its
 * convex hull likewise (hull_vert_off / hull_tri_off).  The meshes are
 * searched together -- every level's cuts and hulls of all meshes still
 * running go out as shared launches -- and every choice stays per part, so
 * out[m] holds exactly the parts a lookahead_decompose of mesh m alone
 * returns (with the same scorer, top_k, margin and beam as
 * cuacd_lookahead_decompose_pruned when scorer != NULL or beam > 0).
 * branch_and_bound = 0 turns the last level's bound off.  out_stats
 * (optional, 8 values): level-0 planes ranked, planes cut, level-0 cuts
 * expanded, fragment hulls built, items cut off by the bound, iterations
 * run, 0, 0.  out: n_meshes results, each freed with gpu_result_free. */
int cuacd_lookahead_decompose_batch(gpu_ctx_t ctx, int n_meshes,
                                    const float* verts, const int* vert_off,
                                    const int* tris, const int* tri_off,
                                    const float* hull_verts, const int* hull_vert_off,
                                    const int* hull_tris, const int* hull_tri_off,
                                    int max_iters, int width, int width2, float threshold,
                                    int depth, int quick_depth, int max_n_cutting, int verbose,
                                    int decompose_components, int decompose_components_per_iter,
                                    int n_concave_edges, float concave_eps, float concave_threshold,
                                    int concave_iters, int merge_hulls, int branch_and_bound,
                                    cuacd_scorer_t scorer, int top_k, float margin, int beam,
                                    unsigned long long* out_stats, struct gpu_result* out);

/* Exact lookahead_decompose that also records, for every level-0 candidate
 * that splits its part, the scorer's feature row followed by 4 floats: the
 * exact level-0 cost, the path cost the search ranks it by (mean level cost
 * of its best descendant leaf), a part key (iteration * 4096 + cutting-part
 * index) and 1 if the part's candidates had leaves (else the path cost is the
 * level-0 cost).  Up to max_rows rows of n_features + 4 floats go to
 * out_rows; *out_n_rows receives the count.  The training pairs of the
 * scorer's path-cost target (no counterpart in the reference). */
int cuacd_lookahead_trace(gpu_ctx_t ctx, cuacd_scorer_t scorer, float* out_rows, int max_rows,
                          int* out_n_rows, const float* verts, int nv, const int* tris, int nt,
                          const float* hull_verts, int hull_nv, const int* hull_tris, int hull_nt,
                          int max_iters, int width, int width2, float threshold, int depth,
                          int max_n_cutting, int n_concave_edges, float concave_eps,
                          float concave_threshold, int concave_iters, struct gpu_result* out);

/* Diagnostics (work counters, phase timers, an allocator benchmark, the
 * remesh's case table) are declared in cuacd_b200_diag.h. */

#ifdef __cplusplus
}
#endif
#endif
