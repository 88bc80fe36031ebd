/*
 * cuacd_oracle.h — CPU oracle for the lookahead candidate-evaluation path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product (the cuacd_b200 package,
 * libcuacd_b200.so) links, loads or calls this code; only tests/, the smoke
 * check and bench.py's CPU-baseline leg do, and only as the checker.
 *
 * It restates, in plain C (FP64 / exact int64), what the reference computes
 * for each candidate plane of cuacd's lookahead search:
 *   - mesh volume            cuda/mesh_volume.cuh:20-57, cuda/geometry.cuh:68-77
 *   - hull quantisation      cuda/hull_dandc.cuh:1351-1411
 *   - exact convex hull      cuda/hull_dandc.cuh:1678-1861 (vertex set of the
 *                            quantised points; computed here by gift wrapping)
 *   - plane cut with caps    cuda/plane_cut.cuh:167-1562
 *   - Hausdorff sampling     cuda/hausdorff.cuh:26-29,68-115,368-558,1453
 *   - concave-edge planes    cuda/la_concave.cu:48-363
 *   - axis candidates        cuda/la_axis_cut.cuh:10-19, cuda/la_expand.cu:182-199
 *   - part costs             cuda/la_common.cuh:21-34
 *   - connected components   cuda/postprocess.cuh:139-527
 *
 * Output orders are canonical (see each function) so the CUDA path can be
 * compared bit-for-bit on integer results.  Parity pins for this oracle live
 * in tests/golden/ (reference golden vectors and scipy/Qhull hull fixtures).
 */
#ifndef CUACD_ORACLE_H
#define CUACD_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------- volume ---------------- */
/* Signed volume (divergence theorem, anchored at vertex 0), FP64. */
double orc_mesh_signed_volume(const float* verts, int nv, const int* tris, int nt);

/* ---------------- hull ---------------- */
/* Quantise points onto the reference hull grid (hull_dandc.cuh:1351-1411),
 * with IEEE-rounded division.  out_q receives n*3 ints in the permuted axis
 * order (med, max, min).  Returns 0. */
int orc_quantize(const float* pts, int n, int* out_q);

/* Exact convex hull of the quantised points.
 * out_vidx: hull corner input indices, ascending (cap vcap)
 * out_tris: triangles as positions into out_vidx, canonical fan
 *           triangulation of each (coplanar-merged) face from its smallest
 *           corner, triangles sorted lexicographically (cap tcap)
 * out_vol : FP64 volume of the output mesh over the float input coords.
 * Returns 0 on success, 1 if degenerate (n<4 or collinear: empty output),
 * -1 on capacity overflow. */
int orc_hull(const float* pts, int n, int* out_vidx, int vcap, int* out_nv,
             int* out_tris, int tcap, int* out_nt, double* out_vol);

/* ---------------- plane cut ---------------- */
typedef struct {
    int n_pos_tris;     /* side triangles before caps */
    int n_neg_tris;
    int n_cap;          /* cap triangles (shared by both sides) */
    int n_loops;        /* boundary loops found */
    int n_boundary;     /* boundary edges */
    int cap_failed;     /* 1: returned the mesh unsplit */
    int n_cross;        /* unique crossing edges */
} orc_cut_info;

/* Cut a closed mesh by plane pa*x+pb*y+pc*z+pd = 0.
 * Outputs are caller-sized (caps below); counts written to out_n*.
 * Returns 0 on success, -1 on capacity overflow. */
int orc_plane_cut(const float* verts, int nv, const int* tris, int nt,
                  float pa, float pb, float pc, float pd,
                  float* pos_v, int pos_v_cap, int* pos_t, int pos_t_cap,
                  float* neg_v, int neg_v_cap, int* neg_t, int neg_t_cap,
                  int* n_pv, int* n_pt, int* n_nv, int* n_nt,
                  orc_cut_info* info);

/* ---------------- Hausdorff ---------------- */
/* Sample count for one surface (hausdorff.cuh:368-466 with a deterministic
 * fixed-point area total).  resolution = samples per unit area,
 * min_samples = floor, total_override > 0 replaces resolution*area. */
int orc_hd_sample_count(const float* v, int nv, const int* t, int nt,
                        float resolution, int min_samples, int total_override);
/* Write the samples of one surface (n*3 floats); returns the count. */
int orc_hd_samples(const float* v, int nv, const int* t, int nt,
                   float resolution, int min_samples, int total_override,
                   float* out, int cap);
/* Bidirectional sampled Hausdorff distance, FP64 nearest-triangle search.
 * Returns sqrt(max(d_ab^2, d_ba^2)) (hausdorff.cuh:1453). */
double orc_hausdorff(const float* av, int anv, const int* at, int ant,
                     const float* bv, int bnv, const int* bt, int bnt,
                     float resolution, int min_samples, int total_override,
                     int n_threads);

/* ---------------- candidate planes ---------------- */
/* Concave-edge planes (la_concave.cu:48-363), canonical order: reservoir
 * slot order, per slot [face-offset n1, face-offset n0, bisector +eps,
 * bisector -eps].  Returns the number of planes (<= 4*n_concave_edges). */
int orc_concave_planes(const float* verts, int nv, const int* tris, int nt,
                       int n_concave_edges, float concave_eps,
                       float concave_threshold, float* out_planes);
/* Axis-aligned candidate plane cut_idx of width (la_axis_cut.cuh:10-19,
 * la_expand.cu:182-199). Returns 0 if valid, 1 if the axis is too narrow. */
int orc_axis_plane(const float* verts, int nv, int width, int cut_idx,
                   float min_edge_dist, float* out_plane);

/* ---------------- candidate evaluator ---------------- */
typedef struct {
    int    ok;            /* both halves non-empty */
    int    nv[2], nt[2];  /* fragment sizes (pos, neg) incl. caps */
    int    n_cap;
    int    hull_nv[2], hull_nt[2];
    double mesh_vol[2], hull_vol[2], hausdorff[2];
    double cost_rv[2], cost_full[2];
    double score_rv, score_full;   /* worst part cost of the candidate */
} orc_cand_result;

#define ORC_EVAL_HAUSDORFF 1

int orc_eval_candidates(const float* verts, int nv, const int* tris, int nt,
                        const float* planes, int n_planes, int flags,
                        float hd_resolution, int hd_min_samples,
                        int hd_total_override, int n_threads,
                        orc_cand_result* out);

/* ---------------- connected components ---------------- */
/* Split into vertex-connected components (postprocess.cuh:139-527).
 * Components are written back to back: out_v (component vertices, input
 * order), out_t (component-local indices, input order), comp_nv/comp_nt/
 * comp_vol per component (|signed volume|, FP64).  Returns the number of
 * components written; 0 when the mesh is one component (or empty, or has
 * more than 4096 components); -1 when a capacity is exceeded. */
int orc_components(const float* v, int nv, const int* t, int nt, int max_comp, int max_out_v, int max_out_t,
                   float* out_v, int* out_t, int* comp_nv, int* comp_nt, double* comp_vol);

/* Part costs (la_common.cuh:21-34). */
double orc_cost_rv(double hull_vol, double mesh_vol);
double orc_cost_full(double hull_vol, double mesh_vol, double hausdorff);

#ifdef __cplusplus
}
#endif
#endif
