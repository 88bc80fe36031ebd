// lookahead.cu — lookahead_decompose: the tree search that calls the
// candidate evaluator (reference csrc/lookahead.c:144-1124 and the la_*
// kernels of cuda/la_expand.cu, la_refine.cu, la_lifecycle.cu, la_concave.cu).
//
// One iteration:
//   0. with decompose_components_per_iter, every part not yet known to be
//      connected is split into its connected components, each with a fresh
//      exact hull (la_decompose_components + la_hull_decomp,
//      csrc/lookahead.c:329-347 and :909-925; components.cuh);
//   1. Hausdorff of every part whose rv cost is below tau and not yet known
//      (la_hausdorff_parts, la_refine.cu:19-45);
//   2. parts sorted by full cost max(rv, H); the up-to-max_n_cutting
//      costliest parts with cost >= tau are cut this iteration
//      (la_sort_and_count_cutting, la_lifecycle.cu:90-144);
//   3. concave-edge planes of each cutting part (la_concave.cu);
//   4. `depth` expansion levels: level 0 cuts each cutting part with `width`
//      axis cuts + its edge planes, level d > 0 cuts the worst part of every
//      surviving item with `width2` axis cuts (la_expand.cu:65-340); every new
//      fragment gets its volume and exact hull (la_hull, :357-424; the
//      batched hull pipeline of hull.cu); the item
//      records its worst rv cost per level (la_sort_and_record,
//      la_refine.cu:359-409); a part too small on every axis ends its branch
//      as a leaf padded with zero costs (la_expand.cu:155-174);
//   5. per cutting part the initial cut with the lowest mean level cost over
//      its descendant leaves wins, with the greedy level-0 fallback
//      (la_evaluate, la_refine.cu:418-527);
//   6. the part is replaced by the two halves of its winning level-0 item
//      (la_apply_cuts, la_lifecycle.cu:151-261), whose hulls are already known.
// Cuts and hulls run as device jobs in waves: fragments and hulls go to an
// output arena kept for the iteration, scratch to a second arena reset
// between waves.
//   4b. `quick_depth` quick levels after the full ones (la_expand_quick,
//      la_refine.cu:52-351): each item's worst part is cut at its box midpoint
//      on the three axes and the most even volume split makes its one child;
//   4c. branch and bound on the last level (la_compute_best_ub + la_hull's
//      rough-hull bound, la_expand.cu:380-457): an item whose new fragment's
//      rough hull (exact hull of its extreme points along 40 directions)
//      already leaves a volume gap too large to beat the best path bound of
//      its cutting part gets no exact hulls and is not evaluated.
// merge_hulls runs the merge-hulls post-pass (merge_hulls_pass) after the
// last iteration.  A batch of meshes runs as one search whose levels share
// their launches (cuacd_lookahead_decompose_batch); every choice is per part,
// so each mesh's parts are those of a search of that mesh alone.
#include <vector>
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include "context.cuh"
#include "cut.cuh"
#include "hull.cuh"
#include "hausdorff.cuh"
#include "components.cuh"
#include "launch.h"

struct CutJob {
    const float* v; const int* t; int nv, nt;
    float4 plane;
    int axis, slice, cpa, _pad;     // axis >= 0: axis-aligned cut computed on the part's bbox
};

typedef HullRes FragRes;            // per fragment: hull + volumes

// The plane of cut job J, computed by the whole CTA into *s_plane / *s_flags
// (la_axis_cut_candidate + la_expand's bbox rules, cuda/la_axis_cut.cuh:10-19,
// cuda/la_expand.cu:155-199): an axis job cuts its part's bbox at slice /
// (cpa + 1) inside a min_edge_dist margin; a part too small on every axis is
// flagged SMALL, an axis too narrow NOPLANE; an explicit zero plane is NOPLANE.
static __device__ void cut_job_plane(const CutJob& J, float min_edge_dist, float (*red)[CUT_NT / 32], float* s_lo,
                                     float* s_hi, float4* s_plane, int* s_flags)
{
    if (threadIdx.x == 0) { *s_flags = 0; *s_plane = J.plane; }
    if (J.axis >= 0) {
        float l[3] = {1e30f, 1e30f, 1e30f}, h[3] = {-1e30f, -1e30f, -1e30f};
        for (int i = threadIdx.x; i < J.nv; i += CUT_NT)
            for (int k = 0; k < 3; k++) { float x = J.v[3 * i + k]; l[k] = fminf(l[k], x); h[k] = fmaxf(h[k], x); }
        for (int k = 0; k < 3; k++) { l[k] = warp_min(l[k]); h[k] = warp_max(h[k]); }
        if ((threadIdx.x & 31) == 0) for (int k = 0; k < 3; k++) { red[k][threadIdx.x >> 5] = l[k]; red[3 + k][threadIdx.x >> 5] = h[k]; }
        __syncthreads();
        if (threadIdx.x == 0) {
            for (int k = 0; k < 3; k++) {
                float a = 1e30f, b = -1e30f;
                for (int w = 0; w < CUT_NT / 32; w++) { a = fminf(a, red[k][w]); b = fmaxf(b, red[3 + k][w]); }
                s_lo[k] = a; s_hi[k] = b;
            }
            const float eps = 1e-6f;
            bool all_small = (s_hi[0] - s_lo[0] <= 2.f * min_edge_dist + eps) &&
                             (s_hi[1] - s_lo[1] <= 2.f * min_edge_dist + eps) &&
                             (s_hi[2] - s_lo[2] <= 2.f * min_edge_dist + eps);
            if (all_small) *s_flags = CUT_FLAG_SMALL | CUT_FLAG_NOPLANE;
            else if (J.cpa < 0) {       // quick level: the box midpoint (la_expand_quick, cuda/la_refine.cu:151-159)
                if (s_hi[J.axis] - s_lo[J.axis] <= 2.f * min_edge_dist + eps) *s_flags = CUT_FLAG_NOPLANE;
                else {
                    const float mid = (s_lo[J.axis] + s_hi[J.axis]) * 0.5f;
                    *s_plane = make_float4(J.axis == 0 ? 1.f : 0.f, J.axis == 1 ? 1.f : 0.f, J.axis == 2 ? 1.f : 0.f, -mid);
                }
            } else {
                float lv = s_lo[J.axis] + min_edge_dist, hv = s_hi[J.axis] - min_edge_dist;
                if (lv >= hv) *s_flags = CUT_FLAG_NOPLANE;
                else {
                    float frac = ((float)J.slice + 1.0f) / ((float)J.cpa + 1.0f);
                    float cut = fmaf(frac, hv - lv, lv);
                    *s_plane = make_float4(J.axis == 0 ? 1.f : 0.f, J.axis == 1 ? 1.f : 0.f, J.axis == 2 ? 1.f : 0.f, -cut);
                }
            }
        }
    } else if (threadIdx.x == 0 && J.plane.x == 0.f && J.plane.y == 0.f && J.plane.z == 0.f) {
        *s_flags = CUT_FLAG_NOPLANE;
    }
    __syncthreads();
}

__global__ void __launch_bounds__(CUT_NT)
k_cut_jobs(const CutJob* __restrict__ jobs, int j0, int j1, Arena* scratch, Arena* out, float min_edge_dist,
           CutResult* res, const int* __restrict__ order = nullptr)
{
    __shared__ CutShared sh;
    __shared__ float s_lo[3], s_hi[3];
    __shared__ float4 s_plane;
    __shared__ int s_flags;
    __shared__ float red[6][CUT_NT / 32];
    // order: the wave's jobs largest first, so the longest cuts start first
    const int j = order ? order[j0 + blockIdx.x] : j0 + blockIdx.x;
    if (j >= j1) return;
    const CutJob J = jobs[j];
    cut_job_plane(J, min_edge_dist, red, s_lo, s_hi, &s_plane, &s_flags);
    if (s_flags & CUT_FLAG_NOPLANE) {
        if (threadIdx.x == 0) { CutResult r; memset(&r, 0, sizeof(r)); r.flags = s_flags; res[j] = r; }
        return;
    }
    CutFixedOut none;
    memset(&none, 0, sizeof(none));
    float4 p = s_plane;
    cut_cta(J.v, J.nv, J.t, J.nt, p.x, p.y, p.z, p.w, scratch, none, &res[j], sh, out);
}

// The planes and flags of jobs [0, n) without cutting (what k_cut_jobs would
// cut with), for the learned scorer's ranking of level-0 candidates.
__global__ void __launch_bounds__(CUT_NT)
k_job_planes(const CutJob* __restrict__ jobs, int n, float min_edge_dist, float4* planes, int* flags)
{
    __shared__ float s_lo[3], s_hi[3];
    __shared__ float4 s_plane;
    __shared__ int s_flags;
    __shared__ float red[6][CUT_NT / 32];
    const int j = blockIdx.x;
    if (j >= n) return;
    const CutJob J = jobs[j];
    cut_job_plane(J, min_edge_dist, red, s_lo, s_hi, &s_plane, &s_flags);
    if (threadIdx.x == 0) { planes[j] = s_plane; flags[j] = s_flags; }
}

// Hull jobs for fragments f0..f1 (2 per cut, empty when the cut produced
// no split) into jobs[f - f0].
__global__ void k_cut_frag_jobs(const CutResult* __restrict__ cuts, int f0, int f1, HullJob* jobs,
                                const unsigned char* __restrict__ skip = nullptr)
{
    const int f = f0 + blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= f1) return;
    const CutResult& C = cuts[f >> 1];
    const int side = f & 1;
    const bool empty = C.err != 0 || C.npv <= 0 || C.nnv <= 0 || (skip && skip[f >> 1]);
    HullJob J;
    memset(&J, 0, sizeof(J));
    if (!empty) {
        J.pts = side ? C.nv : C.pv; J.n = side ? C.nnv : C.npv;
        J.tris = side ? C.nt : C.pt; J.nt = side ? C.nnt : C.npt;
    }
    jobs[f - f0] = J;
}

// Hull jobs for meshes f0..f1 (connected components of split parts).
__global__ void k_surf_jobs(const HDSurf* __restrict__ meshes, int f0, int f1, HullJob* jobs)
{
    const int f = f0 + blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= f1) return;
    const HDSurf m = meshes[f];
    HullJob J;
    memset(&J, 0, sizeof(J));
    if (m.nv > 0 && m.nt > 0) { J.pts = m.v; J.n = m.nv; J.tris = m.t; J.nt = m.nt; }
    jobs[f - f0] = J;
}

__global__ void k_mesh_volumes(const HDSurf* meshes, int n, double* out)
{
    __shared__ double sh[33];
    int i = blockIdx.x;
    if (i >= n) return;
    double v = block_mesh_signed_volume(meshes[i].v, meshes[i].nv, meshes[i].t, meshes[i].nt, sh);
    if (threadIdx.x == 0) out[i] = fabs(v);
}

// ---------------------------------------------------------------------------
// branch-and-bound rough hulls (la_hull's bound, cuda/la_expand.cu:380-401 with
// kdop_hull_block's step 3b, cuda/kdop_hull.cuh:184-213): the exact hull of a
// fragment's extreme points along LA_ROUGH_DIRS directions lies inside the
// fragment's hull, so its volume bounds the hull volume from below.
// ---------------------------------------------------------------------------
#define LA_ROUGH_DIRS 40
#define LA_ROUGH_PTS (2 * LA_ROUGH_DIRS)
#define LA_ROUGH_MIN_NV 1024       // smaller fragments get their exact hull directly (kdop_hull.cuh:95)

// Direction k of a Fibonacci lattice on the upper half sphere.
static __device__ __forceinline__ float3 rough_dir(int k)
{
    const float z = 1.0f - ((float)k + 0.5f) / (float)LA_ROUGH_DIRS;
    const float r = sqrtf(fmaxf(0.f, 1.0f - z * z));
    const float phi = 2.39996322972865332f * (float)k;          // golden angle
    return make_float3(r * cosf(phi), r * sinf(phi), z);
}

// Order-preserving map of a float to 32 unsigned bits.
static __device__ __forceinline__ unsigned long long ord32(float f)
{
    const unsigned u = __float_as_uint(f);
    return (u & 0x80000000u) ? (unsigned long long)(~u) : (unsigned long long)(u | 0x80000000u);
}

// One CTA (256 threads) per fragment: its extreme vertex along +-each
// direction (ties: the smallest index), written as LA_ROUGH_PTS points.
__global__ void __launch_bounds__(256) k_rough_points(const HDSurf* __restrict__ frags, int n, float* out)
{
    __shared__ unsigned long long best[LA_ROUGH_PTS];
    const int i = blockIdx.x;
    if (i >= n) return;
    const HDSurf F = frags[i];
    for (int k = threadIdx.x; k < LA_ROUGH_PTS; k += 256) best[k] = 0ull;
    __syncthreads();
    for (int g = 0; g < LA_ROUGH_DIRS; g += 8) {
        float3 d[8];
        for (int k = 0; k < 8; k++) d[k] = rough_dir(g + k);
        unsigned long long hi[8], lo[8];
        for (int k = 0; k < 8; k++) { hi[k] = 0ull; lo[k] = 0ull; }
        for (int v = threadIdx.x; v < F.nv; v += 256) {
            const float x = F.v[3 * v], y = F.v[3 * v + 1], z = F.v[3 * v + 2];
            const unsigned long long tag = 0xffffffffull - (unsigned)v;     // larger for smaller indices
            for (int k = 0; k < 8; k++) {
                const float t = fmaf(d[k].x, x, fmaf(d[k].y, y, d[k].z * z));
                const unsigned long long a = (ord32(t) << 32) | tag, b = (ord32(-t) << 32) | tag;
                hi[k] = a > hi[k] ? a : hi[k];
                lo[k] = b > lo[k] ? b : lo[k];
            }
        }
        for (int k = 0; k < 8; k++) {
            for (int o = 16; o > 0; o >>= 1) {
                const unsigned long long a = __shfl_xor_sync(FULL_MASK, hi[k], o);
                const unsigned long long b = __shfl_xor_sync(FULL_MASK, lo[k], o);
                hi[k] = a > hi[k] ? a : hi[k];
                lo[k] = b > lo[k] ? b : lo[k];
            }
            if ((threadIdx.x & 31) == 0) {
                atomicMax(&best[2 * (g + k)], hi[k]);
                atomicMax(&best[2 * (g + k) + 1], lo[k]);
            }
        }
    }
    __syncthreads();
    for (int k = threadIdx.x; k < LA_ROUGH_PTS; k += 256) {
        const int v = F.nv > 0 ? (int)(0xffffffffull - (best[k] & 0xffffffffull)) : 0;
        for (int c = 0; c < 3; c++) out[(size_t)i * 3 * LA_ROUGH_PTS + 3 * k + c] = F.nv > 0 ? F.v[3 * v + c] : 0.f;
    }
}

// Hull jobs over the rough point clouds.
__global__ void k_rough_jobs(const float* pts, int n, HullJob* jobs)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    HullJob J;
    memset(&J, 0, sizeof(J));
    J.pts = pts + (size_t)i * 3 * LA_ROUGH_PTS; J.n = LA_ROUGH_PTS;
    jobs[i] = J;
}

// ---------------------------------------------------------------------------
// merge-hulls post-pass kernels (cuda/postprocess_merge.cu:41-679)
// ---------------------------------------------------------------------------
// Axis-aligned box of every mesh: out[6i..6i+5] = min xyz, max xyz.
__global__ void __launch_bounds__(256) k_mesh_boxes(const HDSurf* __restrict__ meshes, int n, float* out)
{
    __shared__ float red[6][8];
    const int i = blockIdx.x;
    if (i >= n) return;
    const HDSurf M = meshes[i];
    float l[3] = {1e30f, 1e30f, 1e30f}, h[3] = {-1e30f, -1e30f, -1e30f};
    for (int v = threadIdx.x; v < M.nv; v += 256)
        for (int k = 0; k < 3; k++) { const float x = M.v[3 * v + k]; l[k] = fminf(l[k], x); h[k] = fmaxf(h[k], x); }
    for (int k = 0; k < 3; k++) { l[k] = warp_min(l[k]); h[k] = warp_max(h[k]); }
    if ((threadIdx.x & 31) == 0) for (int k = 0; k < 3; k++) { red[k][threadIdx.x >> 5] = l[k]; red[3 + k][threadIdx.x >> 5] = h[k]; }
    __syncthreads();
    if (threadIdx.x < 6) {
        const int k = threadIdx.x;
        float r = k < 3 ? 1e30f : -1e30f;
        for (int w = 0; w < 8; w++) r = k < 3 ? fminf(r, red[k][w]) : fmaxf(r, red[k][w]);
        out[6 * i + k] = r;
    }
}

// One merge candidate: parts a and b (meshes and hulls), where its buffers live.
struct MergeJob {
    const float* av; const int* at; int anv, ant;      // part a's mesh
    const float* bv; const int* bt; int bnv, bnt;      // part b's mesh
    const float* ahv; const int* aht; int ahnv, ahnt;  // hulls
    const float* bhv; int bhnv;
    float* cat_pts;                                    // ahnv + bhnv points (hull vertices of a, then b)
    float* mv; int* mt;                                // concatenated mesh (filtered triangles)
    int* mnt;                                          // filtered triangle count
};

// Hull vertices of a then b, one CTA per candidate.
__global__ void __launch_bounds__(256) k_merge_cat_points(const MergeJob* __restrict__ jobs, int n)
{
    const int j = blockIdx.x;
    if (j >= n) return;
    const MergeJob J = jobs[j];
    for (int i = threadIdx.x; i < 3 * J.ahnv; i += 256) J.cat_pts[i] = J.ahv[i];
    for (int i = threadIdx.x; i < 3 * J.bhnv; i += 256) J.cat_pts[3 * J.ahnv + i] = J.bhv[i];
}

// The concatenated mesh of a and b for the merged part's Hausdorff test:
// vertices of a then b; triangles of a then b (b's indices offset), minus
// those whose three vertices lie within 1e-3 of the shared plane -- a face
// plane of a's hull with every vertex of a's hull on or below it and every
// vertex of b's hull on it (la_merge_find_shared_plane_warp, cuda/merge.cuh;
// the lowest such face of a's hull, where the reference takes the first lane
// to find one).  Triangles keep their input order.  One CTA per candidate.
__global__ void __launch_bounds__(256) k_merge_cat_mesh(const MergeJob* __restrict__ jobs, int n)
{
    __shared__ int s_face;
    __shared__ float4 s_plane;
    __shared__ int scan[34];
    const int j = blockIdx.x;
    if (j >= n) return;
    const MergeJob J = jobs[j];
    const float tol = 1e-3f;
    if (threadIdx.x == 0) s_face = 0x7fffffff;
    __syncthreads();
    for (int f = threadIdx.x; f < J.ahnt; f += 256) {
        const int ia = J.aht[3 * f], ib = J.aht[3 * f + 1], ic = J.aht[3 * f + 2];
        const float ax = J.ahv[3 * ia], ay = J.ahv[3 * ia + 1], az = J.ahv[3 * ia + 2];
        const float e1x = J.ahv[3 * ib] - ax, e1y = J.ahv[3 * ib + 1] - ay, e1z = J.ahv[3 * ib + 2] - az;
        const float e2x = J.ahv[3 * ic] - ax, e2y = J.ahv[3 * ic + 1] - ay, e2z = J.ahv[3 * ic + 2] - az;
        float nx = e1y * e2z - e1z * e2y, ny = e1z * e2x - e1x * e2z, nz = e1x * e2y - e1y * e2x;
        const float len = sqrtf(nx * nx + ny * ny + nz * nz);
        if (len < 1e-20f) continue;
        const float inv = 1.0f / len;
        nx *= inv; ny *= inv; nz *= inv;
        const float d = nx * ax + ny * ay + nz * az;
        bool ok = true;
        for (int k = 0; k < J.ahnv && ok; k++) ok = nx * J.ahv[3 * k] + ny * J.ahv[3 * k + 1] + nz * J.ahv[3 * k + 2] - d <= tol;
        for (int k = 0; k < J.bhnv && ok; k++) ok = fabsf(nx * J.bhv[3 * k] + ny * J.bhv[3 * k + 1] + nz * J.bhv[3 * k + 2] - d) <= tol;
        if (ok) { atomicMin(&s_face, f); }
    }
    __syncthreads();
    if (threadIdx.x == 0 && s_face != 0x7fffffff) {
        const int f = s_face;
        const int ia = J.aht[3 * f], ib = J.aht[3 * f + 1], ic = J.aht[3 * f + 2];
        const float ax = J.ahv[3 * ia], ay = J.ahv[3 * ia + 1], az = J.ahv[3 * ia + 2];
        const float e1x = J.ahv[3 * ib] - ax, e1y = J.ahv[3 * ib + 1] - ay, e1z = J.ahv[3 * ib + 2] - az;
        const float e2x = J.ahv[3 * ic] - ax, e2y = J.ahv[3 * ic + 1] - ay, e2z = J.ahv[3 * ic + 2] - az;
        float nx = e1y * e2z - e1z * e2y, ny = e1z * e2x - e1x * e2z, nz = e1x * e2y - e1y * e2x;
        const float inv = 1.0f / sqrtf(nx * nx + ny * ny + nz * nz);
        nx *= inv; ny *= inv; nz *= inv;
        s_plane = make_float4(nx, ny, nz, nx * ax + ny * ay + nz * az);
    }
    __syncthreads();
    const bool has_plane = s_face != 0x7fffffff;
    const float4 P = s_plane;
    for (int i = threadIdx.x; i < 3 * J.anv; i += 256) J.mv[i] = J.av[i];
    for (int i = threadIdx.x; i < 3 * J.bnv; i += 256) J.mv[3 * J.anv + i] = J.bv[i];
    // keep flags in input order, then an exclusive scan gives each kept triangle its slot
    const int nt = J.ant + J.bnt;
    int written = 0;
    for (int base = 0; base < nt; base += 256) {
        const int t = base + threadIdx.x;
        int keep = 0, i0 = 0, i1 = 0, i2 = 0;
        if (t < nt) {
            const bool inb = t >= J.ant;
            const float* V = inb ? J.bv : J.av;
            const int* T = inb ? J.bt + 3 * (t - J.ant) : J.at + 3 * t;
            i0 = T[0]; i1 = T[1]; i2 = T[2];
            keep = 1;
            if (has_plane) {
                const float s0 = P.x * V[3 * i0] + P.y * V[3 * i0 + 1] + P.z * V[3 * i0 + 2] - P.w;
                const float s1 = P.x * V[3 * i1] + P.y * V[3 * i1 + 1] + P.z * V[3 * i1 + 2] - P.w;
                const float s2 = P.x * V[3 * i2] + P.y * V[3 * i2 + 1] + P.z * V[3 * i2 + 2] - P.w;
                if (fabsf(s0) <= tol && fabsf(s1) <= tol && fabsf(s2) <= tol) keep = 0;
            }
            if (inb) { i0 += J.anv; i1 += J.anv; i2 += J.anv; }
        }
        int tot;
        const int ex = block_exclusive_scan(keep, scan, &tot);
        if (keep) { J.mt[3 * (written + ex)] = i0; J.mt[3 * (written + ex) + 1] = i1; J.mt[3 * (written + ex) + 2] = i2; }
        written += tot;
        __syncthreads();
    }
    if (threadIdx.x == 0) *J.mnt = written;
}

// The merged part's mesh: vertices of a then b, triangles of a then b with
// b's indices offset (la_merge_apply, cuda/postprocess_merge.cu:520-620).
__global__ void __launch_bounds__(256) k_merge_concat(const float* av, const int* at, int anv, int ant, const float* bv,
                                                      const int* bt, int bnv, int bnt, float* ov, int* ot)
{
    const int i = blockIdx.x * 256 + threadIdx.x;
    if (i < 3 * anv) ov[i] = av[i];
    if (i < 3 * bnv) ov[3 * anv + i] = bv[i];
    if (i < 3 * ant) ot[i] = at[i];
    if (i < 3 * bnt) ot[3 * ant + i] = bt[i] + anv;
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
namespace {

struct HPart {                 // a part of the decomposition (persistent storage)
    float* v; int* t; int nv, nt;
    float* hv; int* ht; int hnv, hnt;
    double mesh_vol, hull_vol;
    double hd;                 // < 0: not computed
    char* block;               // owning allocation (nullptr: caller's input)
    int cc_id = 0;             // source connected component (0: not assigned)
    bool checked = false;      // already known to be one connected component
    int mesh = 0;              // input mesh of a batch the part belongs to
};

struct LPart {                 // a part inside a search item (arena or persistent)
    const float* v; const int* t; int nv, nt;
    double mesh_vol, hull_vol;
    const float* hv; const int* ht; int hnv, hnt;
};

struct Item {
    int src;                   // index into the cutting list
    int cut0;                  // initial cut index
    std::vector<LPart> parts;
    std::vector<float> costs;  // level costs
    bool leaf_small = false;
};

float cost_rv(double hull_vol, double mesh_vol)
{
    const double pi = 3.14159265358979;
    double g = hull_vol - mesh_vol; if (g < 0) g = 0;
    return (float)(0.3 * std::cbrt((3.0 / (4.0 * pi)) * g));
}
float cost_rv(const LPart& p) { return cost_rv(p.hull_vol, p.mesh_vol); }

struct Axis { int axis, slice, cpa; };
Axis axis_candidate(int width, int idx)
{
    int count = width / 3, rem = width % 3;
    int xc = count + (rem > 0), yc = count + (rem > 1);
    if (idx < xc) return {0, idx, xc};
    if (idx < xc + yc) return {1, idx - xc, yc};
    return {2, idx - xc - yc, count};
}

struct Lookahead {
    gpu_ctx* ctx;
    cudaStream_t s;
    char* out_base; size_t out_cap;       // output arena memory
    char* scr_base; size_t scr_cap;       // scratch arena memory
    Arena* d_out; Arena* d_scr;           // device arena structs
    char* tmp_base; size_t tmp_cap;       // arena for the last level's fragments (reset per wave)
    Arena* d_tmp;
    Arena* d_cur = nullptr;               // where run_level / run_hulls write: d_out or d_tmp
    float min_edge = 0.0125f;
    int debug = 0;                        // write the points of failed fragment hulls to files
    // buffers for the components pass
    HDSurf* d_surfs = nullptr; int surf_cap = 0;
    CompResult* d_cres = nullptr;
    FragRes* d_frags = nullptr; int frag_cap = 0;
    // hull pipeline: jobs/states (frag_cap each), control words, wrap lists
    HullJob* d_hjobs = nullptr; HullState* d_hstates = nullptr; int* d_hctl = nullptr; int* d_wbuf = nullptr;
    int nwc = 1; size_t wbuf_bytes = 0;

    // Hulls of jobs [0, n) already in d_hjobs, results into res[0, n); waves
    // keep the per-hull scratch within the scratch arena.  The search's
    // fragments start with full-size hull tables: many are near-convex
    // pieces of smooth meshes whose hulls outgrow quarter-size tables, and
    // rebuilding those cost more (config-4 sample: 1.03 s against 0.87 s)
    // than clearing full tables.
    int run_hulls(const std::vector<int>& sizes, FragRes* res)
    {
        const int n = (int)sizes.size();
        int f = 0;
        while (f < n) {
            size_t acc = 0; int f1 = f;
            while (f1 < n) {
                size_t e = al256(hull_scratch_bytes(sizes[f1] > 4 ? sizes[f1] : 4, HULL_FIRST_CAP)) + 256;
                if (f1 > f && acc + e > scr_cap) break;
                acc += e; f1++;
            }
            long long pts = 0; int mx = 0;
            for (int k = f; k < f1; k++) { pts += std::max(sizes[k], 256); mx = std::max(mx, sizes[k]); }
            reset_scr();
            launch_hull_jobs(d_hjobs + f, f1 - f, d_hstates + f, res + f, d_scr, d_cur, d_hctl, d_wbuf,
                             std::min(nwc, hull_wrap_ctas(pts, ctx->n_sm, mx)), nullptr, s, mx, false);
            ctx->launches += 5;
            f = f1;
        }
        CK(cudaGetLastError());
        return 0;
    }

    void reset_out() { launch_arena_reset(d_out, out_base, out_cap, s); }
    void reset_tmp() { launch_arena_reset(d_tmp, tmp_base, tmp_cap, s); }

    // Branch-and-bound buffers (2 per job): rough-hull sources, points, mesh
    // volumes, and the per-job skip mask of the fragment hulls.
    HDSurf* d_bnb_surf = nullptr; float* d_bnb_pts = nullptr; double* d_bnb_mvol = nullptr;
    unsigned char* d_skip = nullptr;
    int bnb_cap = 0;                                 // fragments the rough-hull buffers hold
    int* d_order = nullptr;                          // cut jobs, largest first per wave (max_jobs)
    unsigned long long n_hulls = 0, n_pruned = 0;    // fragment hulls built, items pruned

    // The last level's fragments are only needed for their costs: its jobs
    // run in waves whose output fits the temporary arena, reset per wave.
    // bound / pruned as in run_level.
    int run_last_level(const std::vector<CutJob>& jobs, std::vector<CutResult>& cuts, std::vector<FragRes>& frags,
                       CutJob* d_jobs, CutResult* d_cuts, FragRes* d_fr, const std::vector<float>* bound = nullptr,
                       std::vector<char>* pruned = nullptr)
    {
        cuts.clear(); frags.clear();
        if (pruned) pruned->clear();
        std::vector<CutResult> c1; std::vector<FragRes> f1;
        std::vector<float> b1; std::vector<char> p1;
        size_t j = 0;
        while (j < jobs.size()) {
            size_t acc = 0, j1 = j;
            while (j1 < jobs.size()) {
                size_t e = 64 * ((size_t)jobs[j1].nv + jobs[j1].nt) + (64 << 10);
                if (j1 > j && acc + e > tmp_cap) break;
                acc += e; j1++;
            }
            std::vector<CutJob> part(jobs.begin() + j, jobs.begin() + j1);
            if (bound) b1.assign(bound->begin() + j, bound->begin() + j1);
            reset_tmp();
            d_cur = d_tmp;
            int rc = run_level(part, c1, f1, d_jobs, d_cuts, d_fr, bound ? &b1 : nullptr, pruned ? &p1 : nullptr);
            d_cur = d_out;
            if (rc) return rc;
            cuts.insert(cuts.end(), c1.begin(), c1.end());
            frags.insert(frags.end(), f1.begin(), f1.end());
            if (pruned) pruned->insert(pruned->end(), p1.begin(), p1.end());
            j = j1;
        }
        return 0;
    }
    void reset_scr() { launch_arena_reset(d_scr, scr_base, scr_cap, s); }

    // Cut jobs [0, n) into waves of the scratch arena; results to the host.
    int run_cuts(const std::vector<CutJob>& jobs, std::vector<CutResult>& cuts, CutJob* d_jobs, CutResult* d_cuts)
    {
        const int n = (int)jobs.size();
        cuts.assign(n, CutResult());
        if (n == 0) return 0;
        CK(cudaMemcpyAsync(d_jobs, jobs.data(), sizeof(CutJob) * n, cudaMemcpyHostToDevice, s));
        // waves by the scratch estimate; inside a wave the CTAs take the jobs
        // largest first (longest-processing-time order: the block scheduler
        // hands out blocks in index order, so the tail is the short cuts)
        std::vector<int> order(n);
        std::vector<std::pair<int, int>> waves;
        int j = 0;
        while (j < n) {
            size_t acc = 0; int j1 = j;
            while (j1 < n) {
                size_t e = 48 * ((size_t)jobs[j1].nv + 2 * (size_t)jobs[j1].nt) + (256 << 10);
                if (j1 > j && acc + e > scr_cap) break;
                acc += e; j1++;
            }
            for (int k = j; k < j1; k++) order[k] = k;
            std::stable_sort(order.begin() + j, order.begin() + j1,
                             [&](int a, int b) { return jobs[a].nt > jobs[b].nt; });
            waves.push_back({j, j1});
            j = j1;
        }
        CK(cudaMemcpyAsync(d_order, order.data(), sizeof(int) * n, cudaMemcpyHostToDevice, s));
        for (const auto& w : waves) {
            reset_scr();
            k_cut_jobs<<<w.second - w.first, CUT_NT, 0, s>>>(d_jobs, w.first, w.second, d_scr, d_cur, min_edge, d_cuts,
                                                            d_order);
            ctx->launches += 2;
        }
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(cuts.data(), d_cuts, sizeof(CutResult) * n, cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        for (auto& c : cuts) if (c.err & (KERR_HEAP_OOM | KERR_PC_SCRATCH_OOM | KERR_PC_POOL_OOM)) return KERR_HEAP_OOM;
        return 0;
    }

    // Branch and bound over the cut results of one level: bound[j] is job j's
    // rv budget (the best bound on its source part's path sum less the job's
    // item's own partial sum; >= 1e29: none).  A job whose fragment (of more
    // than LA_ROUGH_MIN_NV vertices) already has a rough-hull volume gap above
    // the gap that budget allows -- any gap when the budget is <= 0 -- is
    // pruned: its item cannot beat the bound (la_hull, cuda/la_expand.cu:380-401).
    int bnb_prune(const std::vector<CutResult>& cuts, const std::vector<float>& bound, std::vector<char>& pruned,
                  FragRes* d_fr)
    {
        const int n = (int)cuts.size();
        pruned.assign(n, 0);
        std::vector<HDSurf> src;
        std::vector<int> src_job;
        for (int j = 0; j < n; j++) {
            const CutResult& c = cuts[j];
            if (bound[j] >= 1e29f || c.err || c.npv <= 0 || c.nnv <= 0) continue;
            if (c.npv > LA_ROUGH_MIN_NV) { src.push_back({c.pv, c.pt, c.npv, c.npt}); src_job.push_back(j); }
            if (c.nnv > LA_ROUGH_MIN_NV) { src.push_back({c.nv, c.nt, c.nnv, c.nnt}); src_job.push_back(j); }
        }
        const int m = (int)src.size();
        if (m == 0) return 0;
        std::vector<FragRes> fr(m);
        std::vector<double> mv(m);
        for (int b = 0; b < m; b += bnb_cap) {                  // chunks of the rough-hull buffers
            const int q = std::min(bnb_cap, m - b);
            CK(cudaMemcpyAsync(d_bnb_surf, src.data() + b, sizeof(HDSurf) * q, cudaMemcpyHostToDevice, s));
            k_rough_points<<<q, 256, 0, s>>>(d_bnb_surf, q, d_bnb_pts);
            k_mesh_volumes<<<q, 256, 0, s>>>(d_bnb_surf, q, d_bnb_mvol);
            k_rough_jobs<<<(q + 127) / 128, 128, 0, s>>>(d_bnb_pts, q, d_hjobs);
            ctx->launches += 3;
            CK(cudaGetLastError());
            std::vector<int> sizes(q, LA_ROUGH_PTS);
            int rh = run_hulls(sizes, d_fr);
            if (rh) return rh;
            CK(cudaMemcpyAsync(fr.data() + b, d_fr, sizeof(FragRes) * q, cudaMemcpyDeviceToHost, s));
            CK(cudaMemcpyAsync(mv.data() + b, d_bnb_mvol, sizeof(double) * q, cudaMemcpyDeviceToHost, s));
            CK(cudaStreamSynchronize(s));
        }
        const double pi = 3.14159265358979;
        for (int k = 0; k < m; k++) {
            if (fr[k].err || fr[k].hnt <= 0) continue;          // no rough hull (degenerate points): no bound
            const int j = src_job[k];
            const double thr = bound[j];
            bool cut_off;
            if (thr <= 0.0) cut_off = true;
            else {
                const double r = thr / 0.3;
                const double gap_thr = r * r * r * (4.0 * pi / 3.0);
                // a relative slack keeps the bound item's own children (whose gap
                // can equal the budget's) clear of rounding in the budget
                cut_off = std::max((double)fr[k].hull_vol - mv[k], 0.0) > gap_thr * (1.0 + 1e-4) + 1e-12;
            }
            if (cut_off) pruned[j] = 1;
        }
        for (int j = 0; j < n; j++) n_pruned += pruned[j] ? 1 : 0;
        return 0;
    }

    // Run cut jobs then hull jobs; returns 0 or an error (OOM -> KERR_HEAP_OOM).
    // With `bound`, jobs that branch and bound cuts off get no fragment hulls
    // and are flagged in *pruned.
    int run_level(const std::vector<CutJob>& jobs, std::vector<CutResult>& cuts, std::vector<FragRes>& frags,
                  CutJob* d_jobs, CutResult* d_cuts, FragRes* d_fr, const std::vector<float>* bound = nullptr,
                  std::vector<char>* pruned = nullptr)
    {
        const int n = (int)jobs.size();
        cuts.assign(n, CutResult());
        frags.assign(2 * n, FragRes());
        if (pruned) pruned->assign(n, 0);
        if (n == 0) return 0;
        int rc = run_cuts(jobs, cuts, d_jobs, d_cuts);
        if (rc) return rc;
        const bool use_bnb = bound && pruned;
        if (use_bnb) {
            rc = bnb_prune(cuts, *bound, *pruned, d_fr);
            if (rc) return rc;
            CK(cudaMemcpyAsync(d_skip, pruned->data(), (size_t)n, cudaMemcpyHostToDevice, s));
        }
        // hulls of all fragments (exact sizes known now)
        std::vector<int> sizes(2 * n);
        for (int f = 0; f < 2 * n; f++) {
            const CutResult& c = cuts[f >> 1];
            const bool empty = c.err != 0 || c.npv <= 0 || c.nnv <= 0 || (use_bnb && (*pruned)[f >> 1]);
            sizes[f] = empty ? 0 : ((f & 1) ? c.nnv : c.npv);
            n_hulls += empty ? 0 : 1;
        }
        k_cut_frag_jobs<<<(2 * n + 127) / 128, 128, 0, s>>>(d_cuts, 0, 2 * n, d_hjobs, use_bnb ? d_skip : nullptr);
        ctx->launches += 1;
        int rh = run_hulls(sizes, d_fr);
        if (rh) return rh;
        CK(cudaMemcpyAsync(frags.data(), d_fr, sizeof(FragRes) * 2 * n, cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        if (debug) {
            static int n_dump = 0;
            for (int f = 0; f < 2 * n && n_dump < 16; f++) {
                if (!frags[f].err) continue;
                const CutResult& c = cuts[f >> 1];
                const int nvf = (f & 1) ? c.nnv : c.npv;
                std::vector<float> pts(3 * (size_t)(nvf > 0 ? nvf : 1));
                CK(cudaMemcpy(pts.data(), (f & 1) ? c.nv : c.pv, 12 * (size_t)nvf, cudaMemcpyDeviceToHost));
                char name[64];
                snprintf(name, sizeof(name), "cuacd_failed_hull_%d.f32", n_dump++);
                FILE* fp = fopen(name, "wb");
                if (fp) { fwrite(pts.data(), 12, (size_t)nvf, fp); fclose(fp); }
                fprintf(stderr, "[la] fragment hull failed (0x%x), %d points written to %s\n", frags[f].err, nvf, name);
            }
        }
        for (auto& r : frags) if (r.err & (KERR_HEAP_OOM | KERR_BT_POOL_EXHAUST)) return KERR_HEAP_OOM;
        return 0;
    }

    // A persistent part holding copies of a mesh and its hull.
    int make_part(HPart& p, const float* v, const int* t, int nv, int nt,
                  const float* hv, const int* ht, int hnv, int hnt)
    {
        size_t b0 = al256(12 * (size_t)nv), b1 = al256(12 * (size_t)nt), b2 = al256(12 * (size_t)hnv);
        size_t b3 = al256(12 * (size_t)hnt);
        char* blk = nullptr;
        CK(cudaMallocFromPoolAsync((void**)&blk, b0 + b1 + b2 + b3 + 256, ctx->parts_pool, s));
        p.block = blk;
        p.v = (float*)blk; p.t = (int*)(blk + b0); p.hv = (float*)(blk + b0 + b1); p.ht = (int*)(blk + b0 + b1 + b2);
        p.nv = nv; p.nt = nt; p.hnv = hnv; p.hnt = hnt;
        CK(cudaMemcpyAsync(p.v, v, 12 * (size_t)nv, cudaMemcpyDeviceToDevice, s));
        CK(cudaMemcpyAsync(p.t, t, 12 * (size_t)nt, cudaMemcpyDeviceToDevice, s));
        if (hnv) CK(cudaMemcpyAsync(p.hv, hv, 12 * (size_t)hnv, cudaMemcpyDeviceToDevice, s));
        if (hnt) CK(cudaMemcpyAsync(p.ht, ht, 12 * (size_t)hnt, cudaMemcpyDeviceToDevice, s));
        return 0;
    }
    void free_part(HPart& p) { if (p.block) cudaFreeAsync(p.block, s); p.block = nullptr; }

    int split_components(std::vector<HPart>& parts, const std::vector<int>& idx, std::vector<int>& cc_counter);
};

// Replace every part of `idx` that has several connected components by its
// components, each with a fresh exact hull and volumes (la_decompose_components
// + la_hull_decomp, csrc/lookahead.c:329-347 and :909-925).  The first
// component takes the part's slot, the others are appended
// (la_lifecycle.cu:384-406); cc ids follow la_lifecycle.cu:363-378.
int Lookahead::split_components(std::vector<HPart>& parts, const std::vector<int>& idx, std::vector<int>& cc_counter)
{
    size_t gi = 0;
    while (gi < idx.size()) {
        size_t g1 = gi, oacc = 0, sacc = 0;
        while (g1 < idx.size() && g1 - gi < (size_t)surf_cap) {
            const HPart& p = parts[idx[g1]];
            const size_t nc = (size_t)std::min(p.nv, CC_MAX_COMP);
            size_t oe = cc_output_bytes(p.nv, p.nt) + 36 * (size_t)p.nv + 600 * nc + 4096;
            size_t se = cc_scratch_bytes(p.nv) + 4096;
            if (g1 > gi && (oacc + oe > out_cap || sacc + se > scr_cap)) break;
            oacc += oe; sacc += se; g1++;
        }
        const int m = (int)(g1 - gi);
        std::vector<HDSurf> sf(m);
        for (int k = 0; k < m; k++) { const HPart& p = parts[idx[gi + k]]; sf[k] = {p.v, p.t, p.nv, p.nt}; }
        CK(cudaMemcpyAsync(d_surfs, sf.data(), sizeof(HDSurf) * m, cudaMemcpyHostToDevice, s));
        reset_out();
        reset_scr();
        launch_components(d_surfs, m, d_scr, d_out, d_cres, s);
        ctx->launches += 3;
        CK(cudaGetLastError());
        std::vector<CompResult> cr(m);
        CK(cudaMemcpyAsync(cr.data(), d_cres, sizeof(CompResult) * m, cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        std::vector<CompMesh> comps;
        for (int k = 0; k < m; k++) {
            if (cr[k].err) return ctx_fail(ctx, cr[k].err, "connected components failed (0x%x)", cr[k].err);
            parts[idx[gi + k]].checked = true;
            if (cr[k].n <= 0) continue;
            size_t o = comps.size();
            comps.resize(o + cr[k].n);
            CK(cudaMemcpyAsync(comps.data() + o, cr[k].comps, sizeof(CompMesh) * cr[k].n, cudaMemcpyDeviceToHost, s));
        }
        CK(cudaStreamSynchronize(s));
        // exact hull of every component, in chunks and scratch waves
        std::vector<FragRes> fr(comps.size());
        const size_t chunk = (size_t)std::min(surf_cap, frag_cap);
        for (size_t c0 = 0; c0 < comps.size(); c0 += chunk) {
            const int cn = (int)std::min(chunk, comps.size() - c0);
            std::vector<HDSurf> hs(cn);
            for (int k = 0; k < cn; k++) hs[k] = {comps[c0 + k].v, comps[c0 + k].t, comps[c0 + k].nv, comps[c0 + k].nt};
            CK(cudaMemcpyAsync(d_surfs, hs.data(), sizeof(HDSurf) * cn, cudaMemcpyHostToDevice, s));
            k_surf_jobs<<<(cn + 127) / 128, 128, 0, s>>>(d_surfs, 0, cn, d_hjobs);
            ctx->launches += 1;
            std::vector<int> sizes(cn);
            for (int k = 0; k < cn; k++) sizes[k] = hs[k].nv;
            int rh = run_hulls(sizes, d_frags);
            if (rh) return rh;
            CK(cudaMemcpyAsync(fr.data() + c0, d_frags, sizeof(FragRes) * cn, cudaMemcpyDeviceToHost, s));
            CK(cudaStreamSynchronize(s));
        }
        for (auto& r : fr)
            if (r.err) return ctx_fail(ctx, r.err, "component hull failed (0x%x)", r.err);
        size_t c = 0;
        for (int k = 0; k < m; k++) {
            if (cr[k].n <= 0) continue;
            const int slot = idx[gi + k];
            const int parent_cc = parts[slot].cc_id;
            const int mesh = parts[slot].mesh;
            const int base_cc = cc_counter[mesh];
            if (parent_cc == 0) cc_counter[mesh] += cr[k].n;
            std::vector<HPart> made(cr[k].n);
            for (int j = 0; j < cr[k].n; j++, c++) {
                HPart& p = made[j];
                int rc = make_part(p, comps[c].v, comps[c].t, comps[c].nv, comps[c].nt,
                                   fr[c].hv, fr[c].ht, fr[c].hnv, fr[c].hnt);
                if (rc) return rc;
                p.hull_vol = fr[c].hull_vol;
                p.mesh_vol = std::min(comps[c].vol, (double)fr[c].hull_vol);   // la_hull_decomp clamp
                p.hd = -1;
                p.checked = true;
                p.cc_id = parent_cc ? parent_cc : base_cc + j + 1;
                p.mesh = mesh;
            }
            free_part(parts[slot]);
            parts[slot] = made[0];
            for (int j = 1; j < cr[k].n; j++) parts.push_back(made[j]);
        }
        CK(cudaStreamSynchronize(s));      // copies out of the output arena are done
        gi = g1;
    }
    return 0;
}

} // namespace

extern "C" void gpu_result_free(struct gpu_result* r)
{
    if (!r) return;
    for (int i = 0; i < r->nparts; i++) {
        free(r->parts[i].verts); free(r->parts[i].tris);
        free(r->parts[i].hull_verts); free(r->parts[i].hull_tris);
    }
    free(r->parts);
    r->parts = nullptr; r->nparts = 0;
}

// Merge-hulls post-pass (cuda/postprocess_merge.cu:41-679, driven as in
// csrc/lookahead.c:987-1063).  For every pair of parts (p1 > p2) of the same
// connected component: reject when the sum of their hull-minus-mesh gaps
// already costs tau or more, or when their boxes are tau/2 or more apart;
// else the exact hull of both hulls' vertices gives the merged rv cost, and
// below tau the sampled Hausdorff distance between that hull and both meshes
// (less the triangles lying in a shared face plane) raises it to
// max(rv, H).  Then one greedy round: the cheapest pair below tau merges, its
// two parts leave the pool, repeat; each merged part is both meshes
// concatenated with the merged hull.  Costs use the reference's FP32 forms.
static int merge_hulls_pass(gpu_ctx* ctx, Lookahead& L, std::vector<HPart>& parts, float tau, HDSurf* d_surfs,
                            HDPrep* d_preps, char* d_dirs, int* d_i4, float* d_pmax)
{
    cudaStream_t s = L.s;
    const int P = (int)parts.size();
    const float pi_f = 3.14159265358979f;
    auto rv_of = [&](float gap) { return 0.3f * cbrtf((3.0f / (4.0f * pi_f)) * gap); };
    // boxes of every part's mesh
    std::vector<float> box(6 * (size_t)P);
    for (int b = 0; b < P; b += 1024) {                // d_pmax holds 8192 floats: 6 per part
        const int m = std::min(1024, P - b);
        std::vector<HDSurf> sf(m);
        for (int k = 0; k < m; k++) sf[k] = {parts[b + k].v, parts[b + k].t, parts[b + k].nv, parts[b + k].nt};
        CK(cudaMemcpyAsync(d_surfs, sf.data(), sizeof(HDSurf) * m, cudaMemcpyHostToDevice, s));
        k_mesh_boxes<<<m, 256, 0, s>>>(d_surfs, m, d_pmax);
        ctx->launches++;
        CK(cudaMemcpyAsync(box.data() + 6 * (size_t)b, d_pmax, sizeof(float) * 6 * m, cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
    }
    // candidates surviving the quick rejects (reference order of pair indices)
    std::vector<std::pair<int, int>> cand;
    for (int p1 = 1; p1 < P; p1++)
        for (int p2 = 0; p2 < p1; p2++) {
            const HPart& A = parts[p1]; const HPart& B = parts[p2];
            if (A.cc_id != 0 && B.cc_id != 0 && A.cc_id != B.cc_id) continue;
            const float msum = (float)A.mesh_vol + (float)B.mesh_vol;
            if (rv_of(fmaxf((float)A.hull_vol + (float)B.hull_vol - msum, 0.0f)) >= tau) continue;
            const float* a = &box[6 * (size_t)p1]; const float* b = &box[6 * (size_t)p2];
            float g2 = 0.f;
            for (int k = 0; k < 3; k++) { const float g = fmaxf(0.0f, fmaxf(a[k] - b[3 + k], b[k] - a[3 + k])); g2 += g * g; }
            if (g2 >= (tau * 0.5f) * (tau * 0.5f)) continue;
            cand.push_back({p1, p2});
        }
    std::vector<float> cost(cand.size(), 1e30f);
    std::vector<FragRes> mres(cand.size());
    L.reset_out();                                   // the search's fragments are no longer needed
    const int CH = std::min(2048, L.frag_cap);
    for (size_t c0 = 0; c0 < cand.size(); c0 += CH) {
        const int m = (int)std::min<size_t>(CH, cand.size() - c0);
        // device buffers for this chunk
        size_t pts = 0, mv = 0, mt = 0;
        for (int k = 0; k < m; k++) {
            const HPart& A = parts[cand[c0 + k].first]; const HPart& B = parts[cand[c0 + k].second];
            pts += 3 * (size_t)(A.hnv + B.hnv); mv += 3 * (size_t)(A.nv + B.nv); mt += 3 * (size_t)(A.nt + B.nt);
        }
        char* blk = nullptr;
        const size_t bj = al256(sizeof(MergeJob) * m), bp = al256(4 * pts), bv = al256(4 * mv), bt = al256(4 * mt);
        const size_t bn = al256(4 * (size_t)m);
        CK(cudaMallocFromPoolAsync((void**)&blk, bj + bp + bv + bt + bn, ctx->parts_pool, s));
        MergeJob* d_jobs = (MergeJob*)blk;
        float* d_pts = (float*)(blk + bj); float* d_mv = (float*)(blk + bj + bp); int* d_mt = (int*)(blk + bj + bp + bv);
        int* d_mnt = (int*)(blk + bj + bp + bv + bt);
        std::vector<MergeJob> jobs(m);
        std::vector<HullJob> hj(m);
        std::vector<int> sizes(m);
        size_t op = 0, ov = 0, ot = 0;
        for (int k = 0; k < m; k++) {
            const HPart& A = parts[cand[c0 + k].first]; const HPart& B = parts[cand[c0 + k].second];
            MergeJob& J = jobs[k];
            J.av = A.v; J.at = A.t; J.anv = A.nv; J.ant = A.nt;
            J.bv = B.v; J.bt = B.t; J.bnv = B.nv; J.bnt = B.nt;
            J.ahv = A.hv; J.aht = A.ht; J.ahnv = A.hnv; J.ahnt = A.hnt;
            J.bhv = B.hv; J.bhnv = B.hnv;
            J.cat_pts = d_pts + op; J.mv = d_mv + ov; J.mt = d_mt + ot; J.mnt = d_mnt + k;
            HullJob& H = hj[k];
            memset(&H, 0, sizeof(H));
            H.pts = J.cat_pts; H.n = A.hnv + B.hnv;
            sizes[k] = H.n;
            op += 3 * (size_t)(A.hnv + B.hnv); ov += 3 * (size_t)(A.nv + B.nv); ot += 3 * (size_t)(A.nt + B.nt);
        }
        CK(cudaMemcpyAsync(d_jobs, jobs.data(), sizeof(MergeJob) * m, cudaMemcpyHostToDevice, s));
        k_merge_cat_points<<<m, 256, 0, s>>>(d_jobs, m);
        CK(cudaMemcpyAsync(L.d_hjobs, hj.data(), sizeof(HullJob) * m, cudaMemcpyHostToDevice, s));
        ctx->launches++;
        int rh = L.run_hulls(sizes, L.d_frags);
        if (rh) { cudaFreeAsync(blk, s); return rh; }
        std::vector<FragRes> fr(m);
        CK(cudaMemcpyAsync(fr.data(), L.d_frags, sizeof(FragRes) * m, cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        std::vector<int> hd_idx;                        // candidates that go on to the Hausdorff test
        for (int k = 0; k < m; k++) {
            const HPart& A = parts[cand[c0 + k].first]; const HPart& B = parts[cand[c0 + k].second];
            mres[c0 + k] = fr[k];
            if (fr[k].err || fr[k].hnt == 0) { if (fr[k].err & (KERR_HEAP_OOM | KERR_BT_POOL_EXHAUST)) { cudaFreeAsync(blk, s); return ctx_fail(ctx, KERR_HEAP_OOM, "merge hulls: pool exhausted"); } continue; }
            const float msum = (float)A.mesh_vol + (float)B.mesh_vol;
            const float rv = rv_of(fmaxf(fr[k].hull_vol - msum, 0.0f));
            cost[c0 + k] = rv;
            if (rv < tau) hd_idx.push_back(k);
        }
        if (!hd_idx.empty()) {
            k_merge_cat_mesh<<<m, 256, 0, s>>>(d_jobs, m);
            ctx->launches++;
            std::vector<int> mnt(m);
            CK(cudaMemcpyAsync(mnt.data(), d_mnt, sizeof(int) * m, cudaMemcpyDeviceToHost, s));
            CK(cudaStreamSynchronize(s));
            std::vector<int> keep;                      // no triangle left: Hausdorff 0 (reference)
            for (int k : hd_idx) if (mnt[k] > 0) keep.push_back(k);
            hd_idx.swap(keep);
            for (size_t b = 0; b < hd_idx.size(); b += 4096) {
                const int q = (int)std::min<size_t>(4096, hd_idx.size() - b);
                std::vector<HDSurf> sf(2 * q);
                std::vector<int> with(q, 1);
                for (int r = 0; r < q; r++) {
                    const int k = hd_idx[b + r];
                    const MergeJob& J = jobs[k];
                    sf[2 * r] = {fr[k].hv, fr[k].ht, fr[k].hnv, fr[k].hnt};
                    sf[2 * r + 1] = {J.mv, J.mt, J.anv + J.bnv, mnt[k]};
                }
                CK(cudaMemcpyAsync(d_surfs, sf.data(), sizeof(HDSurf) * 2 * q, cudaMemcpyHostToDevice, s));
                CK(cudaMemsetAsync(d_i4, 0, 16 * sizeof(int), s));
                L.reset_scr();
                launch_hausdorff_pairs(d_surfs, q, L.d_scr, 2000.f, 1000, 0, d_preps, d_dirs, d_i4, d_pmax, d_i4 + 2,
                                       ctx->n_sm, s);
                launch_hd_sqrt(d_pmax, q, d_pmax + 4096, 1, s);
                ctx->launches += 5;
                std::vector<float> h(q);
                int herr = 0;
                CK(cudaMemcpyAsync(h.data(), d_pmax + 4096, sizeof(float) * q, cudaMemcpyDeviceToHost, s));
                CK(cudaMemcpyAsync(&herr, d_i4 + 2, sizeof(int), cudaMemcpyDeviceToHost, s));
                CK(cudaStreamSynchronize(s));
                if (herr) { cudaFreeAsync(blk, s); return ctx_fail(ctx, herr, "merge hulls: Hausdorff failed (0x%x)", herr); }
                for (int r = 0; r < q; r++) {
                    const int k = hd_idx[b + r];
                    if (with[r]) cost[c0 + k] = fmaxf(cost[c0 + k], h[r]);
                }
            }
        }
        // merged hulls of pairs that may still merge stay in the output arena;
        // the chunk's own buffers go
        CK(cudaFreeAsync(blk, s));
    }
    // greedy matching: cheapest pair below tau first (ties: lower pair index)
    std::vector<int> order;
    for (size_t k = 0; k < cand.size(); k++) if (cost[k] < tau) order.push_back((int)k);
    auto pair_index = [&](int k) { const int p1 = cand[k].first, p2 = cand[k].second; return (long long)p1 * (p1 - 1) / 2 + p2; };
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
        return cost[a] < cost[b] || (cost[a] == cost[b] && pair_index(a) < pair_index(b));
    });
    std::vector<char> used(P, 0), dead(P, 0);
    for (int k : order) {
        const int p1 = cand[k].first, p2 = cand[k].second;
        if (used[p1] || used[p2]) continue;
        used[p1] = used[p2] = 1;
        const HPart A = parts[p1], B = parts[p2];
        const FragRes& H = mres[k];
        HPart M;
        const int nv = A.nv + B.nv, nt = A.nt + B.nt;
        const size_t b0 = al256(12 * (size_t)nv), b1 = al256(12 * (size_t)nt), b2 = al256(12 * (size_t)H.hnv);
        const size_t b3 = al256(12 * (size_t)H.hnt);
        char* blk = nullptr;
        CK(cudaMallocFromPoolAsync((void**)&blk, b0 + b1 + b2 + b3 + 256, ctx->parts_pool, s));
        M.block = blk;
        M.v = (float*)blk; M.t = (int*)(blk + b0); M.hv = (float*)(blk + b0 + b1); M.ht = (int*)(blk + b0 + b1 + b2);
        M.nv = nv; M.nt = nt; M.hnv = H.hnv; M.hnt = H.hnt;
        const int big = 3 * std::max(std::max(A.nv, B.nv), std::max(A.nt, B.nt));
        k_merge_concat<<<(big + 255) / 256, 256, 0, s>>>(A.v, A.t, A.nv, A.nt, B.v, B.t, B.nv, B.nt, M.v, M.t);
        ctx->launches++;
        CK(cudaMemcpyAsync(M.hv, H.hv, 12 * (size_t)H.hnv, cudaMemcpyDeviceToDevice, s));
        CK(cudaMemcpyAsync(M.ht, H.ht, 12 * (size_t)H.hnt, cudaMemcpyDeviceToDevice, s));
        M.mesh_vol = (double)((float)A.mesh_vol + (float)B.mesh_vol);
        M.hull_vol = H.hull_vol;
        M.hd = 0.0;                                    // la_merge_apply resets it
        M.cc_id = A.cc_id ? A.cc_id : B.cc_id;
        M.checked = true;
        M.mesh = A.mesh;
        L.free_part(parts[p1]);
        L.free_part(parts[p2]);
        parts[p1] = M;
        dead[p2] = 1;
    }
    std::vector<HPart> kept;
    for (int i = 0; i < P; i++) if (!dead[i]) kept.push_back(parts[i]);
    parts.swap(kept);
    CK(cudaStreamSynchronize(s));
    return 0;
}

struct Prune;
static int prune_level0(gpu_ctx* ctx, Lookahead& L, const Prune& P, const std::vector<Item>& cur,
                        std::vector<CutJob>& jobs, std::vector<std::pair<int, int>>& job_of, CutJob* d_jobs,
                        float4* d_planes, int* d_flags);

// Optional pruning.  With a scorer, it ranks each cutting part's level-0
// planes and only the top_k (plus those predicted within `margin` of the
// k-th) are cut; planes the cut would skip (no plane, part too small) are
// always kept.  With beam > 0, only the `beam` level-0 items of each part
// with the lowest exact level-0 cost are expanded further.  stats[0] +=
// level-0 candidates ranked, stats[1] += those cut, stats[2] += level-0
// items expanded.
struct Prune {
    cuacd_scorer* sc; int top_k; float margin; int beam; unsigned long long* stats;
    // trace mode (top_k <= 0 with a scorer): nothing is pruned; every level-0
    // candidate's feature row is kept with its exact level-0 cost and its
    // path cost (mean level cost of its best leaf), rows of n_features + 4
    // floats: features, level-0 cost, path cost, part key, 1 if it has leaves
    std::vector<float>* trace; size_t trace_cap; int iter;
    mutable std::vector<float> tfeat; mutable std::vector<std::pair<int, int>> tkey;
};

static int prune_level0(gpu_ctx* ctx, Lookahead& L, const Prune& P, const std::vector<Item>& cur,
                        std::vector<CutJob>& jobs, std::vector<std::pair<int, int>>& job_of, CutJob* d_jobs,
                        float4* d_planes, int* d_flags)
{
    const int n = (int)jobs.size();
    if (n == 0) return 0;
    cudaStream_t s = L.s;
    CK(cudaMemcpyAsync(d_jobs, jobs.data(), sizeof(CutJob) * n, cudaMemcpyHostToDevice, s));
    k_job_planes<<<n, CUT_NT, 0, s>>>(d_jobs, n, L.min_edge, d_planes, d_flags);
    ctx->launches++;
    CK(cudaGetLastError());
    std::vector<int> flags(n);
    CK(cudaMemcpyAsync(flags.data(), d_flags, sizeof(int) * n, cudaMemcpyDeviceToHost, s));
    // one scorer part per item: its jobs are consecutive
    std::vector<ScorerPart> sp;
    for (int j = 0; j < n;) {
        const int ii = job_of[j].first;
        int j1 = j;
        while (j1 < n && job_of[j1].first == ii) j1++;
        const LPart& w = cur[ii].parts.back();
        sp.push_back({w.v, w.t, w.nv, w.nt, (float)w.hull_vol, j, j1 - j});
        j = j1;
    }
    std::vector<float> pred(n);
    int rc = scorer_predict_parts(ctx, P.sc, sp.data(), (int)sp.size(), d_planes, n, pred.data(), s);
    if (rc) return rc;
    if (P.top_k <= 0) {                                // trace: keep every job, remember its row
        P.tfeat.resize((size_t)n * scorer_n_features());
        rc = scorer_copy_features(ctx, P.sc, n, P.tfeat.data(), s);
        if (rc) return rc;
        P.tkey.assign(job_of.begin(), job_of.end());
        return 0;
    }
    std::vector<char> keep(n, 0);
    for (const ScorerPart& p : sp) {
        std::vector<int> valid;
        for (int k = p.off; k < p.off + p.n; k++) {
            if (flags[k] & CUT_FLAG_NOPLANE) keep[k] = 1;     // skipped by the cut; keeps the small-part rule
            else valid.push_back(k);
        }
        P.stats[0] += valid.size();
        std::vector<float> key(valid.size());
        for (size_t r = 0; r < valid.size(); r++) {
            const float y = pred[valid[r]];
            key[r] = y == y ? y : 3.402823466e38f;             // NaN ranks last
        }
        std::vector<int> order(valid.size());
        for (size_t r = 0; r < valid.size(); r++) order[r] = (int)r;
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return key[a] < key[b]; });
        const int k = std::min<int>(P.top_k, (int)valid.size());
        const float kth = k > 0 ? key[order[k - 1]] : 0.f;
        for (int r = 0; r < (int)order.size(); r++)
            if (r < k || key[order[r]] <= kth + P.margin) { keep[valid[order[r]]] = 1; P.stats[1]++; }
    }
    std::vector<CutJob> kj;
    std::vector<std::pair<int, int>> ko;
    for (int j = 0; j < n; j++) if (keep[j]) { kj.push_back(jobs[j]); ko.push_back(job_of[j]); }
    jobs.swap(kj);
    job_of.swap(ko);
    return 0;
}

// One input mesh of a batch: the mesh and its convex hull (host pointers).
struct MeshIn { const float* v; int nv; const int* t; int nt; const float* hv; int hnv; const int* ht; int hnt; };

struct SearchParams {
    int max_iters, width, width2; float threshold; int depth, quick_depth, max_n_cutting, verbose, debug;
    int decompose_components, decompose_components_per_iter, n_concave_edges;
    float concave_eps, concave_threshold; int concave_iters, merge_hulls, bnb;
};

// Branch-and-bound budgets of the last level's jobs.  Per source part, the
// best bound on a path sum over the current items: partial sum plus the
// worst (latest) level cost for every level left, since a part's volume gap
// never grows when it is cut (la_compute_best_ub, cuda/la_expand.cu:434-457).
// The bound is taken per source part: the reference takes one minimum over
// the items of every cutting part, which lets one part's bound cut off all
// of another part's leaves and send that part to its greedy fallback.
// A job's budget is that bound less its item's partial sum (1e30: none).
static std::vector<float> bnb_budgets(const std::vector<Item>& cur, int n_src, int total_levels,
                                      const std::vector<std::pair<int, int>>& job_of)
{
    std::vector<double> ub(n_src, 1e30);
    for (const Item& it : cur) {
        const int nl = (int)it.costs.size();
        if (nl <= 0) continue;
        double ps = 0;
        for (float c : it.costs) ps += c;
        ub[it.src] = std::min(ub[it.src], ps + (double)it.costs.back() * (total_levels - nl));
    }
    std::vector<float> b(job_of.size(), 1e30f);
    for (size_t j = 0; j < job_of.size(); j++) {
        const Item& it = cur[job_of[j].first];
        const int nl = (int)it.costs.size();
        if (ub[it.src] >= 1e29 || nl <= 0 || nl >= total_levels) continue;
        double ps = 0;
        for (float c : it.costs) ps += c;
        b[j] = (float)(ub[it.src] - ps);
    }
    return b;
}

// Search statistics of a call (cuacd_lookahead_decompose_batch's out_stats).
enum { ST_RANKED = 0, ST_CUT = 1, ST_EXPANDED = 2, ST_HULLS = 3, ST_PRUNED = 4, ST_ITERS = 5, ST_N = 8 };

// The lookahead search over a group of meshes at once.  Every decision is
// per part, so each mesh gets exactly the parts a search of it alone gets;
// what the group shares are the launches: one cut wave and one hull wave
// per level serve the cutting parts of every mesh still running.
static int search_group(gpu_ctx_t ctx, int n_mesh, const MeshIn* M, const SearchParams& P, const Prune* prune,
                        unsigned long long* st, struct gpu_result* outs)
{
    if (!ctx || !outs) return -1;
    for (int m = 0; m < n_mesh; m++) { outs[m].parts = nullptr; outs[m].nparts = 0; }
    if (n_mesh <= 0) return 0;
    if (n_mesh > 2048) return ctx_fail(ctx, KERR_MESH_INVALID, "more than 2048 meshes in one search group");
    if (P.width < 1 || P.width2 < 1 || P.depth < 1 || P.depth > 4 || P.quick_depth < 0 || P.quick_depth > 4 ||
        P.max_n_cutting < 1 || P.n_concave_edges < 0 || P.n_concave_edges > 256)
        return ctx_fail(ctx, KERR_MESH_INVALID, "bad search parameters");
    size_t sum_v = 0, sum_t = 0, sum_hv = 0, sum_ht = 0;
    int max_nv = 0;
    for (int m = 0; m < n_mesh; m++) {
        const MeshIn& I = M[m];
        if (I.nv <= 0 || I.nt <= 0) return ctx_fail(ctx, KERR_MESH_INVALID, "mesh %d: empty mesh", m);
        if (I.hnv < 0 || I.hnt < 0) return ctx_fail(ctx, KERR_MESH_INVALID, "mesh %d: negative hull size", m);
        for (int i = 0; i < 3 * I.nt; i++)
            if (I.t[i] < 0 || I.t[i] >= I.nv) return ctx_fail(ctx, KERR_MESH_INVALID, "mesh %d: index out of range", m);
        for (int i = 0; i < 3 * I.hnt; i++)
            if (I.ht[i] < 0 || I.ht[i] >= I.hnv)
                return ctx_fail(ctx, KERR_MESH_INVALID, "mesh %d: hull index out of range", m);
        sum_v += I.nv; sum_t += I.nt; sum_hv += I.hnv; sum_ht += I.hnt;
        max_nv = std::max(max_nv, I.nv);
    }
    CK(cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->stream;
    const int K = P.n_concave_edges;
    const int tw_max = P.width + 4 * K;
    const int total_levels = P.depth + P.quick_depth;
    const size_t n_cut_cap = (size_t)P.max_n_cutting * n_mesh;
    // ---- pool: fixed buffers + output arena + scratch arena + temporary arena
    size_t items_last = n_cut_cap * tw_max;             // items after the full levels
    for (int d = 1; d < P.depth; d++) items_last *= P.width2;
    const size_t max_jobs = items_last * (P.quick_depth > 0 ? 3 : 1);
    const size_t hjob_cap = std::max<size_t>(2 * max_jobs, 2 * 4096);
    const size_t bnb_cap = std::min<size_t>(hjob_cap, 16384);
    size_t fixed = al256(sizeof(CutJob) * max_jobs) + al256(sizeof(CutResult) * max_jobs) + al256(sizeof(FragRes) * 2 * max_jobs)
                 + al256(sizeof(float4) * n_cut_cap * tw_max) + al256(sizeof(int) * n_cut_cap * tw_max)
                 + al256(3 * sizeof(Arena)) + al256(12 * (sum_v + sum_t)) + al256(12 * (sum_hv + sum_ht))
                 + al256(sizeof(HDSurf) * 2 * 4096) + al256(sizeof(HDPrep) * 2 * 4096) + al256(hd_dir_bytes() * 2 * 4096)
                 + al256(64) + al256(sizeof(float) * 2 * 4096) + al256(sizeof(double) * 4096)
                 + al256(sizeof(CompResult) * 2 * 4096)
                 + al256(sizeof(HullJob) * hjob_cap) + al256(sizeof(HullState) * hjob_cap) + al256(64)
                 + al256(hull_wrap_buf_bytes(hull_wrap_ctas(1LL << 40, ctx->n_sm)))
                 + al256(sizeof(HDSurf) * bnb_cap) + al256(sizeof(float) * 3 * LA_ROUGH_PTS * bnb_cap)
                 + al256(sizeof(double) * bnb_cap) + al256(max_jobs) + al256(sizeof(int) * max_jobs);
    // Output arena: the fragments and hulls of every level whose items outlive
    // it.  A level-0 candidate set outputs about 64 bytes per input vertex and
    // triangle per plane; a further level multiplies that by width2 at most.
    const size_t lvl0 = (size_t)tw_max * 64 * (sum_v + sum_t) * 5 / 4;
    size_t kept = 0, mult = 1;
    const int kept_full = P.quick_depth > 0 ? P.depth : P.depth - 1;
    for (int d = 0; d < kept_full; d++) { kept += mult; mult *= P.width2; }
    if (P.quick_depth > 1) kept += (size_t)(P.quick_depth - 1) * (mult / P.width2 > 0 ? mult / P.width2 : 1);
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    const size_t out_limit = std::max<size_t>((size_t)1 << 30, std::min<size_t>((size_t)96 << 30, free_b / 2));
    size_t out_cap = std::min<size_t>(std::max<size_t>((size_t)1 << 30, lvl0 * std::max<size_t>(kept, 1)), out_limit);
    size_t tmp_cap = std::min<size_t>(std::max<size_t>((size_t)1 << 30, (size_t)P.width2 * 64 * (sum_v + sum_t) * 2),
                                      (size_t)16 << 30);
    size_t scr_cap = std::max<size_t>((size_t)2 << 30, hull_scratch_bytes(max_nv) * 64);
    int rc = pool_begin(ctx, fixed + out_cap + tmp_cap + scr_cap + (1 << 20));
    if (rc) return rc;
    CutJob* d_jobs = pool_take<CutJob>(ctx, max_jobs);
    float4* d_jplanes = pool_take<float4>(ctx, n_cut_cap * tw_max);
    int* d_jflags = pool_take<int>(ctx, n_cut_cap * tw_max);
    CutResult* d_cuts = pool_take<CutResult>(ctx, max_jobs);
    FragRes* d_frags = pool_take<FragRes>(ctx, 2 * max_jobs);
    Arena* d_arenas = pool_take<Arena>(ctx, 3);
    float* d_v0 = pool_take<float>(ctx, 3 * sum_v);
    int* d_t0 = pool_take<int>(ctx, 3 * sum_t);
    float* d_hv0 = pool_take<float>(ctx, 3 * sum_hv);
    int* d_ht0 = pool_take<int>(ctx, 3 * sum_ht);
    HDSurf* d_surfs = pool_take<HDSurf>(ctx, 2 * 4096);
    HDPrep* d_preps = pool_take<HDPrep>(ctx, 2 * 4096);
    char* d_dirs = pool_take<char>(ctx, hd_dir_bytes() * 2 * 4096);
    int* d_i4 = pool_take<int>(ctx, 16);
    float* d_pmax = pool_take<float>(ctx, 2 * 4096);
    double* d_vols = pool_take<double>(ctx, 4096);
    CompResult* d_cres = pool_take<CompResult>(ctx, 2 * 4096);
    HullJob* d_hjobs = pool_take<HullJob>(ctx, hjob_cap);
    HullState* d_hstates = pool_take<HullState>(ctx, hjob_cap);
    int* d_hctl = pool_take<int>(ctx, 16);
    int* d_wbuf = (int*)pool_take<char>(ctx, hull_wrap_buf_bytes(hull_wrap_ctas(1LL << 40, ctx->n_sm)));
    HDSurf* d_bnb_surf = pool_take<HDSurf>(ctx, bnb_cap);
    float* d_bnb_pts = pool_take<float>(ctx, 3 * LA_ROUGH_PTS * bnb_cap);
    double* d_bnb_mvol = pool_take<double>(ctx, bnb_cap);
    unsigned char* d_skip = pool_take<unsigned char>(ctx, max_jobs);
    int* d_order = pool_take<int>(ctx, max_jobs);
    char* out_base = pool_take<char>(ctx, out_cap);
    char* scr_base = pool_take<char>(ctx, scr_cap);
    char* tmp_base = pool_take<char>(ctx, tmp_cap);
    if (!scr_base || !tmp_base) return ctx_fail(ctx, KERR_HEAP_OOM, "pool carve failed");
    Lookahead L;
    L.ctx = ctx; L.s = s; L.out_base = out_base; L.out_cap = out_cap; L.scr_base = scr_base; L.scr_cap = scr_cap;
    L.d_out = d_arenas; L.d_scr = d_arenas + 1; L.d_tmp = d_arenas + 2; L.d_cur = L.d_out;
    L.tmp_base = tmp_base; L.tmp_cap = tmp_cap;
    L.min_edge = std::min(P.threshold * 0.25f, 0.015f);
    L.debug = P.debug;
    L.d_surfs = d_surfs; L.surf_cap = 2 * 4096; L.d_cres = d_cres;
    L.d_frags = d_frags; L.frag_cap = (int)std::min<size_t>(2 * max_jobs, 1 << 30);
    L.d_hjobs = d_hjobs; L.d_hstates = d_hstates; L.d_hctl = d_hctl; L.d_wbuf = d_wbuf; L.nwc = hull_wrap_ctas(1LL << 40, ctx->n_sm);
    L.d_bnb_surf = d_bnb_surf; L.d_bnb_pts = d_bnb_pts; L.d_bnb_mvol = d_bnb_mvol; L.d_skip = d_skip;
    L.bnb_cap = (int)bnb_cap;
    L.d_order = d_order;
    // ---- initial parts: each mesh and the caller's hull (la_initialize, la_lifecycle.cu:18-81)
    std::vector<HPart> parts;
    {
        size_t ov = 0, ot = 0, ohv = 0, oht = 0;
        std::vector<HDSurf> sf(2 * (size_t)n_mesh);
        for (int m = 0; m < n_mesh; m++) {
            const MeshIn& I = M[m];
            CK(cudaMemcpyAsync(d_v0 + 3 * ov, I.v, 12 * (size_t)I.nv, cudaMemcpyHostToDevice, s));
            CK(cudaMemcpyAsync(d_t0 + 3 * ot, I.t, 12 * (size_t)I.nt, cudaMemcpyHostToDevice, s));
            if (I.hnv) CK(cudaMemcpyAsync(d_hv0 + 3 * ohv, I.hv, 12 * (size_t)I.hnv, cudaMemcpyHostToDevice, s));
            if (I.hnt) CK(cudaMemcpyAsync(d_ht0 + 3 * oht, I.ht, 12 * (size_t)I.hnt, cudaMemcpyHostToDevice, s));
            HPart p;
            p.v = d_v0 + 3 * ov; p.t = d_t0 + 3 * ot; p.nv = I.nv; p.nt = I.nt;
            p.hv = d_hv0 + 3 * ohv; p.ht = d_ht0 + 3 * oht; p.hnv = I.hnv; p.hnt = I.hnt;
            p.hd = -1; p.block = nullptr; p.mesh = m;
            parts.push_back(p);
            sf[2 * m] = {p.v, p.t, p.nv, p.nt};
            sf[2 * m + 1] = {p.hv, p.ht, p.hnv, p.hnt};
            ov += I.nv; ot += I.nt; ohv += I.hnv; oht += I.hnt;
        }
        for (int b = 0; b < 2 * n_mesh; b += 4096) {
            const int q = std::min(4096, 2 * n_mesh - b);
            std::vector<double> vols(q);
            CK(cudaMemcpyAsync(d_surfs, sf.data() + b, sizeof(HDSurf) * q, cudaMemcpyHostToDevice, s));
            k_mesh_volumes<<<q, 256, 0, s>>>(d_surfs, q, d_vols);
            ctx->launches++;
            CK(cudaMemcpyAsync(vols.data(), d_vols, sizeof(double) * q, cudaMemcpyDeviceToHost, s));
            CK(cudaStreamSynchronize(s));
            for (int k = 0; k < q; k++) {
                HPart& p = parts[(b + k) >> 1];
                if (((b + k) & 1) == 0) p.mesh_vol = vols[k]; else p.hull_vol = vols[k];
            }
        }
    }
    int result = 0;
    std::vector<int> cc_counter(n_mesh, 0);
    std::vector<char> done(n_mesh, 0);
    auto unchecked = [&]() {
        std::vector<int> u;
        for (int i = 0; i < (int)parts.size(); i++) if (!parts[i].checked && !done[parts[i].mesh]) u.push_back(i);
        return u;
    };
    std::vector<CutJob> jobs;
    std::vector<CutResult> cuts;
    std::vector<FragRes> frs;
    // verbose >= 2: wall time per phase (the stream is drained at each mark)
    double tph[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    auto tnow = [&]() { cudaStreamSynchronize(s); return std::chrono::steady_clock::now(); };
    std::chrono::steady_clock::time_point tmark = std::chrono::steady_clock::now();
    auto tacc = [&](int k) {
        if (P.verbose < 2) return;
        auto t = tnow();
        tph[k] += std::chrono::duration<double>(t - tmark).count();
        tmark = t;
    };
    int n_iters_run = 0;
    for (int iter = 0; iter < P.max_iters && result == 0; iter++) {
        bool any_active = false;
        for (int m = 0; m < n_mesh; m++) any_active |= !done[m];
        if (!any_active) break;
        n_iters_run++;
        tacc(7);
        // ---- 0. split parts made of several connected components
        //      (dc_pre_eval / dc_post_cuts, csrc/lookahead.c:329-347, :909-925)
        if (P.decompose_components_per_iter) {
            result = L.split_components(parts, unchecked(), cc_counter);
            if (result) break;
        }
        tacc(0);
        // ---- 1. Hausdorff of parts below tau
        {
            std::vector<int> need;
            for (int i = 0; i < (int)parts.size(); i++)
                if (!done[parts[i].mesh] && parts[i].hd < 0 && parts[i].hnt > 0 &&
                    cost_rv(parts[i].hull_vol, parts[i].mesh_vol) < P.threshold)
                    need.push_back(i);
            for (size_t b = 0; b < need.size(); b += 4096) {
                int m = (int)std::min<size_t>(4096, need.size() - b);
                std::vector<HDSurf> sf(2 * m);
                for (int k = 0; k < m; k++) {
                    const HPart& p = parts[need[b + k]];
                    sf[2 * k] = {p.hv, p.ht, p.hnv, p.hnt};
                    sf[2 * k + 1] = {p.v, p.t, p.nv, p.nt};
                }
                CK(cudaMemcpyAsync(d_surfs, sf.data(), sizeof(HDSurf) * 2 * m, cudaMemcpyHostToDevice, s));
                CK(cudaMemsetAsync(d_i4, 0, 16 * sizeof(int), s));
                L.reset_scr();
                launch_hausdorff_pairs(d_surfs, m, L.d_scr, 2000.f, 1000, 0, d_preps, d_dirs, d_i4, d_pmax, d_i4 + 2,
                                       ctx->n_sm, s);
                launch_hd_sqrt(d_pmax, m, d_pmax + 4096, 1, s);
                ctx->launches += 5;
                std::vector<float> h(m);
                int herr = 0;
                CK(cudaMemcpyAsync(h.data(), d_pmax + 4096, sizeof(float) * m, cudaMemcpyDeviceToHost, s));
                CK(cudaMemcpyAsync(&herr, d_i4 + 2, sizeof(int), cudaMemcpyDeviceToHost, s));
                CK(cudaStreamSynchronize(s));
                if (herr) { result = ctx_fail(ctx, herr, "hausdorff failed at iter %d (0x%x)", iter, herr); break; }
                for (int k = 0; k < m; k++) parts[need[b + k]].hd = h[k];
            }
            if (result) break;
        }
        // ---- 2. cutting parts of every running mesh (costliest first, la_sort_and_count_cutting)
        auto full = [&](int i) {
            const HPart& p = parts[i];
            float rv = cost_rv(p.hull_vol, p.mesh_vol);
            return std::max(rv, p.hd > 0 ? (float)p.hd : 0.f);
        };
        std::vector<std::vector<int>> of_mesh(n_mesh);
        for (int i = 0; i < (int)parts.size(); i++) if (!done[parts[i].mesh]) of_mesh[parts[i].mesh].push_back(i);
        std::vector<int> cutting;
        for (int m = 0; m < n_mesh; m++) {
            if (done[m]) continue;
            std::vector<int>& order = of_mesh[m];
            std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return full(a) < full(b); });
            int first_above = (int)order.size();
            for (int i = 0; i < (int)order.size(); i++) if (full(order[i]) >= P.threshold) { first_above = i; break; }
            const int start = std::max(first_above, (int)order.size() - P.max_n_cutting);
            size_t before = cutting.size();
            for (int i = start; i < (int)order.size(); i++) if (full(order[i]) >= P.threshold) cutting.push_back(order[i]);
            if (cutting.size() == before) done[m] = 1;           // nothing above tau: this mesh is finished
        }
        if (P.verbose == 1 || P.verbose >= 3)
            fprintf(stderr, "[la] iter %d: parts=%zu cutting=%zu\n", iter, parts.size(), cutting.size());
        if (cutting.empty()) break;
        const int nc = (int)cutting.size();
        tacc(1);
        // ---- 3. concave-edge planes per cutting part
        std::vector<std::vector<float4>> eplanes(nc);
        if (K > 0 && iter < P.concave_iters) {      // all cutting parts in one launch
            std::vector<const float*> pv(nc); std::vector<const int*> pt(nc);
            std::vector<int> pnv(nc), pnt(nc);
            for (int c = 0; c < nc; c++) {
                const HPart& p = parts[cutting[c]];
                pv[c] = p.v; pt[c] = p.t; pnv[c] = p.nv; pnt[c] = p.nt;
            }
            rc = concave_planes_device_batch(ctx, nc, pv.data(), pnv.data(), pt.data(), pnt.data(), K, P.concave_eps,
                                             P.concave_threshold, L.scr_base, L.scr_cap, eplanes);
            if (rc) { result = rc; break; }
        }
        int n_edge = 0;
        for (auto& e : eplanes) n_edge = std::max(n_edge, (int)e.size());
        const int tw0 = P.width + n_edge;
        tacc(2);
        // ---- 4. expansion levels: `depth` full levels, then `quick_depth` quick ones
        std::vector<Item> cur, leaves, extra;
        for (int c = 0; c < nc; c++) {
            Item it; it.src = c; it.cut0 = -1;
            const HPart& p = parts[cutting[c]];
            it.parts.push_back({p.v, p.t, p.nv, p.nt, p.mesh_vol, p.hull_vol, p.hv, p.ht, p.hnv, p.hnt});
            cur.push_back(it);
        }
        std::vector<int> cur_src_of_item0(cur.size());  // level-0 item -> cutting part
        for (size_t ii = 0; ii < cur.size(); ii++) cur_src_of_item0[ii] = cur[ii].src;
        std::vector<Item> level0;              // level-0 items by (src, cut) for apply
        std::vector<std::vector<int>> l0index(nc, std::vector<int>(tw0, -1));
        L.reset_out();
        // a part too small on every axis ends its branch as a leaf padded with
        // zero costs (la_expand.cu:155-174, la_refine.cu:103-118)
        auto small_leaf = [&](const Item& it, int d, int ci) {
            Item x = it;
            if (d == 0) x.cut0 = ci;
            while ((int)x.costs.size() < total_levels) x.costs.push_back(0.f);
            x.leaf_small = true;
            extra.push_back(x);
        };
        // the item that replaces its worst part by the two fragments of cut j
        auto child = [&](const Item& it, int d, int ci, const CutResult& c, const FragRes& a, const FragRes& b) {
            Item x;
            x.src = it.src; x.cut0 = d == 0 ? ci : it.cut0;
            x.parts.assign(it.parts.begin(), it.parts.end() - 1);
            x.parts.push_back({c.pv, c.pt, c.npv, c.npt, a.mesh_vol, (double)a.hull_vol, a.hv, a.ht, a.hnv, a.hnt});
            x.parts.push_back({c.nv, c.nt, c.nnv, c.nnt, b.mesh_vol, (double)b.hull_vol, b.hv, b.ht, b.hnv, b.hnt});
            std::stable_sort(x.parts.begin(), x.parts.end(), [](const LPart& p, const LPart& q) { return cost_rv(p) < cost_rv(q); });
            x.costs = it.costs;
            x.costs.push_back(cost_rv(x.parts.back()));
            return x;
        };
        for (int d = 0; d < P.depth && !cur.empty() && result == 0; d++) {
            const int wd = d == 0 ? P.width : P.width2;
            jobs.clear();
            std::vector<std::pair<int, int>> job_of;   // (item, cut idx)
            for (int ii = 0; ii < (int)cur.size(); ii++) {
                const Item& it = cur[ii];
                const LPart& w = it.parts.back();      // worst part (parts sorted by rv)
                int tw = d == 0 ? tw0 : wd;
                for (int ci = 0; ci < tw; ci++) {
                    CutJob J;
                    J.v = w.v; J.t = w.t; J.nv = w.nv; J.nt = w.nt; J._pad = 0;
                    if (ci < wd) {
                        Axis a = axis_candidate(wd, ci);
                        J.axis = a.axis; J.slice = a.slice; J.cpa = a.cpa; J.plane = make_float4(0, 0, 0, 0);
                    } else {
                        const auto& ep = eplanes[it.src];
                        int k = ci - wd;
                        J.axis = -1; J.slice = 0; J.cpa = 0;
                        J.plane = k < (int)ep.size() ? ep[k] : make_float4(0, 0, 0, 0);
                    }
                    jobs.push_back(J);
                    job_of.push_back({ii, ci});
                }
            }
            if (d == 0 && prune && prune->sc) {
                result = prune_level0(ctx, L, *prune, cur, jobs, job_of, d_jobs, d_jplanes, d_jflags);
                if (result) break;
                tacc(3);
            }
            const bool last = d == total_levels - 1 && d > 0;
            const bool bnb = last && P.bnb;
            std::vector<float> budget;
            std::vector<char> pruned;
            if (bnb) budget = bnb_budgets(cur, nc, total_levels, job_of);
            int lr = last ? L.run_last_level(jobs, cuts, frs, d_jobs, d_cuts, d_frags, bnb ? &budget : nullptr,
                                             bnb ? &pruned : nullptr)
                          : L.run_level(jobs, cuts, frs, d_jobs, d_cuts, d_frags);
            tacc(d == 0 ? 4 : 5);
            if (lr) { result = ctx_fail(ctx, lr, "lookahead level %d failed at iter %d (0x%x)", d, iter, lr); break; }
            std::vector<Item> next;
            std::vector<bool> small_done(cur.size(), false);
            for (size_t j = 0; j < jobs.size(); j++) {
                const int ii = job_of[j].first, ci = job_of[j].second;
                const Item& it = cur[ii];
                const CutResult& c = cuts[j];
                if (c.flags & CUT_FLAG_SMALL) {
                    if (!small_done[ii]) { small_done[ii] = true; small_leaf(it, d, ci); }
                    continue;
                }
                if (c.flags & CUT_FLAG_NOPLANE) continue;
                if (c.err || c.npv == 0 || c.nnv == 0) continue;
                if (bnb && pruned[j]) continue;            // cannot beat its source part's bound
                const FragRes& a = frs[2 * j];
                const FragRes& b = frs[2 * j + 1];
                if (a.err || b.err) { result = ctx_fail(ctx, a.err | b.err, "fragment hull failed (0x%x)", a.err | b.err); break; }
                Item x = child(it, d, ci, c, a, b);
                if (d == 0) { l0index[x.src][ci] = (int)level0.size(); level0.push_back(x); }
                next.push_back(std::move(x));
            }
            if (result) break;
            if (d == 0 && prune && prune->beam > 0 && total_levels > 1) {
                std::vector<std::vector<int>> by_src(nc);
                for (int k = 0; k < (int)next.size(); k++) by_src[next[k].src].push_back(k);
                std::vector<char> keep(next.size(), 0);
                for (auto& ks : by_src) {
                    std::stable_sort(ks.begin(), ks.end(), [&](int a, int b) { return next[a].costs[0] < next[b].costs[0]; });
                    for (int r = 0; r < (int)ks.size() && r < prune->beam; r++) keep[ks[r]] = 1;
                }
                std::vector<Item> kept_items;
                for (size_t k = 0; k < next.size(); k++) if (keep[k]) kept_items.push_back(std::move(next[k]));
                next.swap(kept_items);
            }
            if (d == 0 && prune) prune->stats[2] += next.size();
            cur.swap(next);
        }
        // quick levels (la_expand_quick, cuda/la_refine.cu:52-351): each item's
        // worst part is cut at its box midpoint on each axis; the cut with the
        // most even volume split (max / sum, first axis on ties) makes the
        // item's one child.  The three cuts are made in the temporary arena to
        // compare them, then the chosen one again where its level keeps it.
        for (int q = 0; q < P.quick_depth && !cur.empty() && result == 0; q++) {
            const int d = P.depth + q;
            const int ni = (int)cur.size();
            jobs.clear();
            for (int ii = 0; ii < ni; ii++) {
                const LPart& w = cur[ii].parts.back();
                for (int a = 0; a < 3; a++) {
                    CutJob J;
                    J.v = w.v; J.t = w.t; J.nv = w.nv; J.nt = w.nt; J._pad = 0;
                    J.axis = a; J.slice = 0; J.cpa = -1; J.plane = make_float4(0, 0, 0, 0);
                    jobs.push_back(J);
                }
            }
            std::vector<int> choice(ni, -1);
            std::vector<char> is_small(ni, 0);
            {
                std::vector<double> bal(jobs.size(), 1e30);
                size_t j = 0;
                while (j < jobs.size() && result == 0) {
                    size_t acc = 0, j1 = j;
                    while (j1 < jobs.size()) {
                        size_t e = 64 * ((size_t)jobs[j1].nv + jobs[j1].nt) + (64 << 10);
                        if (j1 > j && acc + e > L.tmp_cap) break;
                        acc += e; j1++;
                    }
                    std::vector<CutJob> part(jobs.begin() + j, jobs.begin() + j1);
                    std::vector<CutResult> c1;
                    L.reset_tmp();
                    L.d_cur = L.d_tmp;
                    int lr = L.run_cuts(part, c1, d_jobs, d_cuts);
                    if (lr) { L.d_cur = L.d_out; result = ctx_fail(ctx, lr, "quick level %d failed at iter %d (0x%x)", q, iter, lr); break; }
                    std::vector<HDSurf> src;
                    std::vector<size_t> src_job;
                    for (size_t k = 0; k < c1.size(); k++) {
                        const CutResult& c = c1[k];
                        if (c.flags & CUT_FLAG_SMALL) is_small[(j + k) / 3] = 1;
                        if ((c.flags & CUT_FLAG_NOPLANE) || c.err || c.npv <= 0 || c.nnv <= 0) continue;
                        src.push_back({c.pv, c.pt, c.npv, c.npt});
                        src.push_back({c.nv, c.nt, c.nnv, c.nnt});
                        src_job.push_back(j + k);
                    }
                    std::vector<double> vol(src.size());
                    for (size_t b = 0; b < src.size(); b += bnb_cap) {
                        const int m = (int)std::min<size_t>(bnb_cap, src.size() - b);
                        CK(cudaMemcpyAsync(d_bnb_surf, src.data() + b, sizeof(HDSurf) * m, cudaMemcpyHostToDevice, s));
                        k_mesh_volumes<<<m, 256, 0, s>>>(d_bnb_surf, m, d_bnb_mvol);
                        ctx->launches++;
                        CK(cudaMemcpyAsync(vol.data() + b, d_bnb_mvol, sizeof(double) * m, cudaMemcpyDeviceToHost, s));
                        CK(cudaStreamSynchronize(s));
                    }
                    for (size_t k = 0; k < src_job.size(); k++) {
                        const double vp = vol[2 * k], vn = vol[2 * k + 1];
                        bal[src_job[k]] = std::max(vp, vn) / (vp + vn + 1e-10);
                    }
                    L.d_cur = L.d_out;
                    j = j1;
                }
                if (result) break;
                for (int ii = 0; ii < ni; ii++) {
                    double best = 1e30;
                    for (int a = 0; a < 3; a++)
                        if (bal[3 * ii + a] < best) { best = bal[3 * ii + a]; choice[ii] = a; }
                }
            }
            // the chosen cuts, kept where their level's items live
            std::vector<CutJob> cj;
            std::vector<std::pair<int, int>> job_of;
            for (int ii = 0; ii < ni; ii++) {
                if (is_small[ii]) { small_leaf(cur[ii], d, 0); continue; }
                if (choice[ii] < 0) continue;                // no axis splits it: the item ends here
                cj.push_back(jobs[3 * ii + choice[ii]]);
                job_of.push_back({ii, 0});
            }
            const bool last = d == total_levels - 1;
            const bool bnb = last && P.bnb;
            std::vector<float> budget;
            std::vector<char> pruned;
            if (bnb) budget = bnb_budgets(cur, nc, total_levels, job_of);
            int lr = last ? L.run_last_level(cj, cuts, frs, d_jobs, d_cuts, d_frags, bnb ? &budget : nullptr,
                                             bnb ? &pruned : nullptr)
                          : L.run_level(cj, cuts, frs, d_jobs, d_cuts, d_frags);
            tacc(5);
            if (lr) { result = ctx_fail(ctx, lr, "quick level %d failed at iter %d (0x%x)", q, iter, lr); break; }
            std::vector<Item> next;
            for (size_t j = 0; j < cj.size(); j++) {
                const Item& it = cur[job_of[j].first];
                const CutResult& c = cuts[j];
                if ((c.flags & (CUT_FLAG_SMALL | CUT_FLAG_NOPLANE)) || c.err || c.npv == 0 || c.nnv == 0) continue;
                if (bnb && pruned[j]) continue;
                const FragRes& a = frs[2 * j];
                const FragRes& b = frs[2 * j + 1];
                if (a.err || b.err) { result = ctx_fail(ctx, a.err | b.err, "fragment hull failed (0x%x)", a.err | b.err); break; }
                next.push_back(child(it, d, 0, c, a, b));
            }
            if (result) break;
            cur.swap(next);
        }
        if (result) break;
        for (auto& it : cur) leaves.push_back(it);
        for (auto& it : extra) leaves.push_back(it);
        // ---- 5. evaluate (la_evaluate)
        std::vector<int> best_cut(nc, -1);
        for (int c = 0; c < nc; c++) {
            std::vector<float> cb(tw0, 1e30f);
            for (const Item& it : leaves) {
                if (it.src != c || it.costs.empty() || it.cut0 < 0 || it.cut0 >= tw0) continue;
                float pc = 0.f;
                for (float x : it.costs) pc += x;
                pc /= (float)it.costs.size();
                cb[it.cut0] = std::min(cb[it.cut0], pc);
            }
            bool any = false;
            for (float x : cb) if (x < 1e30f) any = true;
            if (!any)
                for (int ci = 0; ci < tw0; ci++) {
                    int li = l0index[c][ci];
                    if (li >= 0 && !level0[li].costs.empty()) cb[ci] = level0[li].costs[0];
                }
            float best = 1e30f; int bi = -1;
            for (int ci = 0; ci < tw0; ci++) if (cb[ci] < best) { best = cb[ci]; bi = ci; }
            best_cut[c] = bi;
            if (prune && prune->trace && !prune->tkey.empty()) {
                const int KF = scorer_n_features();
                for (size_t j = 0; j < prune->tkey.size(); j++) {
                    if (cur_src_of_item0[prune->tkey[j].first] != c) continue;
                    const int ci = prune->tkey[j].second;
                    const int li = l0index[c][ci];
                    if (li < 0 || level0[li].costs.empty()) continue;      // no split: not a candidate
                    if (prune->trace->size() + KF + 4 > prune->trace_cap) break;
                    const float* f = prune->tfeat.data() + j * KF;
                    prune->trace->insert(prune->trace->end(), f, f + KF);
                    prune->trace->push_back(level0[li].costs[0]);
                    prune->trace->push_back(cb[ci] < 1e30f ? cb[ci] : level0[li].costs[0]);
                    prune->trace->push_back((float)(iter * 4096 + c));
                    prune->trace->push_back(any ? 1.f : 0.f);
                }
            }
        }
        if (prune) { prune->tkey.clear(); prune->tfeat.clear(); }
        tacc(6);
        // ---- 6. apply: the part becomes the two halves of its best level-0 item
        std::vector<char> applied(n_mesh, 0), had(n_mesh, 0);
        std::vector<HPart> added;
        for (int c = 0; c < nc; c++) {
            const int mesh = parts[cutting[c]].mesh;
            had[mesh] = 1;
            int bi = best_cut[c];
            if (bi < 0) continue;
            int li = l0index[c][bi];
            if (li < 0) continue;                    // winner was a small-part leaf: nothing to cut
            const Item& x = level0[li];
            HPart nw[2];
            for (int k = 0; k < 2; k++) {
                const LPart& q = x.parts[k];
                HPart& p = nw[k];
                rc = L.make_part(p, q.v, q.t, q.nv, q.nt, q.hv, q.ht, q.hnv, q.hnt);
                if (rc) { result = rc; break; }
                p.hull_vol = q.hull_vol;
                p.mesh_vol = std::min(q.mesh_vol, q.hull_vol);   // la_hull_decomp clamp (la_lifecycle.cu:294-297)
                p.hd = -1;
                p.cc_id = parts[cutting[c]].cc_id;             // cut pieces inherit (la_expand.cu:253-258)
                p.mesh = mesh;
            }
            if (result) break;
            L.free_part(parts[cutting[c]]);
            parts[cutting[c]] = nw[0];
            added.push_back(nw[1]);
            applied[mesh] = 1;
        }
        for (auto& p : added) parts.push_back(p);
        if (result) break;
        CK(cudaStreamSynchronize(s));
        for (int m = 0; m < n_mesh; m++) if (had[m] && !applied[m]) done[m] = 1;   // no cut applied: finished
    }
    tacc(7);
    if (P.verbose >= 2)
        fprintf(stderr, "[la] %d iterations, seconds: components %.4f hausdorff %.4f concave %.4f prune %.4f "
                "level0 %.4f deeper %.4f bookkeeping %.4f apply %.4f\n", n_iters_run, tph[0], tph[1], tph[2],
                tph[3], tph[4], tph[5], tph[6], tph[7]);
    if (st) { st[ST_HULLS] += L.n_hulls; st[ST_PRUNED] += L.n_pruned; st[ST_ITERS] += n_iters_run; }
    // ---- post-pass components (csrc/lookahead.c:969-985); with the per-iteration
    //      pass on, only the pieces of the last iteration's cuts are left
    if (result == 0 && (P.decompose_components || P.decompose_components_per_iter)) {
        std::fill(done.begin(), done.end(), 0);
        result = L.split_components(parts, unchecked(), cc_counter);
    }
    // ---- merge-hulls post-pass (csrc/lookahead.c:987-1063, cuda/postprocess_merge.cu:41-679):
    //      one greedy round of pairwise merges whose merged cost stays below tau, per mesh
    if (result == 0 && P.merge_hulls) {
        std::vector<HPart> merged;
        for (int m = 0; m < n_mesh && result == 0; m++) {
            std::vector<HPart> mine;
            for (auto& p : parts) if (p.mesh == m) mine.push_back(p);
            if (mine.size() >= 2)
                result = merge_hulls_pass(ctx, L, mine, P.threshold, d_surfs, d_preps, d_dirs, d_i4, d_pmax);
            merged.insert(merged.end(), mine.begin(), mine.end());
        }
        if (result == 0) parts.swap(merged);
    }
    // ---- results (host copies), per mesh in part order
    if (result == 0) {
        std::vector<int> count(n_mesh, 0);
        for (auto& p : parts) count[p.mesh]++;
        for (int m = 0; m < n_mesh; m++) {
            outs[m].parts = (gpu_part_result*)calloc(count[m] > 0 ? count[m] : 1, sizeof(gpu_part_result));
            outs[m].nparts = 0;
        }
        for (size_t i = 0; i < parts.size() && result == 0; i++) {
            const HPart& p = parts[i];
            gpu_part_result& r = outs[p.mesh].parts[outs[p.mesh].nparts++];
            r.nv = p.nv; r.nt = p.nt; r.hull_nv = p.hnv; r.hull_nt = p.hnt;
            r.verts = (float*)malloc(12 * (size_t)(p.nv > 0 ? p.nv : 1));
            r.tris = (int*)malloc(12 * (size_t)(p.nt > 0 ? p.nt : 1));
            r.hull_verts = (float*)malloc(12 * (size_t)(p.hnv > 0 ? p.hnv : 1));
            r.hull_tris = (int*)malloc(12 * (size_t)(p.hnt > 0 ? p.hnt : 1));
            r.mesh_vol = (float)p.mesh_vol; r.hull_vol = (float)p.hull_vol; r.hausdorff = (float)std::max(p.hd, 0.0);
            cudaError_t e1 = cudaMemcpyAsync(r.verts, p.v, 12 * (size_t)p.nv, cudaMemcpyDeviceToHost, s);
            cudaError_t e2 = cudaMemcpyAsync(r.tris, p.t, 12 * (size_t)p.nt, cudaMemcpyDeviceToHost, s);
            cudaError_t e3 = p.hnv ? cudaMemcpyAsync(r.hull_verts, p.hv, 12 * (size_t)p.hnv, cudaMemcpyDeviceToHost, s) : cudaSuccess;
            cudaError_t e4 = p.hnt ? cudaMemcpyAsync(r.hull_tris, p.ht, 12 * (size_t)p.hnt, cudaMemcpyDeviceToHost, s) : cudaSuccess;
            if (e1 || e2 || e3 || e4) result = ctx_fail(ctx, -1, "result copy failed");
        }
        if (cudaStreamSynchronize(s) != cudaSuccess && result == 0) result = ctx_fail(ctx, -1, "result copy failed");
    }
    for (auto& p : parts) L.free_part(p);
    cudaStreamSynchronize(s);
    if (result) { for (int m = 0; m < n_mesh; m++) gpu_result_free(&outs[m]); return result; }
    return 0;
}

static SearchParams search_params(int max_iters, int width, int width2, float threshold, int depth, int quick_depth,
                                  int max_n_cutting, int verbose, int debug, int decompose_components,
                                  int decompose_components_per_iter, int n_concave_edges, float concave_eps,
                                  float concave_threshold, int concave_iters, int merge_hulls, int bnb)
{
    SearchParams P;
    P.max_iters = max_iters; P.width = width; P.width2 = width2; P.threshold = threshold; P.depth = depth;
    P.quick_depth = quick_depth; P.max_n_cutting = max_n_cutting; P.verbose = verbose; P.debug = debug;
    P.decompose_components = decompose_components; P.decompose_components_per_iter = decompose_components_per_iter;
    P.n_concave_edges = n_concave_edges; P.concave_eps = concave_eps; P.concave_threshold = concave_threshold;
    P.concave_iters = concave_iters; P.merge_hulls = merge_hulls; P.bnb = bnb;
    return P;
}

extern "C" int lookahead_decompose(gpu_ctx_t ctx, const float* verts, int nv, const int* tris, int nt,
                                   const float* hull_verts, int hull_nv, const int* hull_tris, int hull_nt,
                                   int max_iters, int width, int width2, float threshold,
                                   int depth, int quick_depth, int max_n_cutting,
                                   int verbose, int debug, int decompose_components,
                                   int decompose_components_per_iter,
                                   int n_concave_edges, float concave_eps, float concave_threshold,
                                   int concave_iters, int merge_hulls, struct gpu_result* out)
{
    if (!ctx || !out) return -1;
    MeshIn m{verts, nv, tris, nt, hull_verts, hull_nv, hull_tris, hull_nt};
    SearchParams P = search_params(max_iters, width, width2, threshold, depth, quick_depth, max_n_cutting, verbose,
                                   debug, decompose_components, decompose_components_per_iter, n_concave_edges,
                                   concave_eps, concave_threshold, concave_iters, merge_hulls, 1);
    return search_group(ctx, 1, &m, P, nullptr, nullptr, out);
}

extern "C" int cuacd_lookahead_decompose_pruned(gpu_ctx_t ctx, cuacd_scorer_t scorer, int top_k, float margin,
                                                int beam, unsigned long long* out_stats,
                                                const float* verts, int nv, const int* tris, int nt,
                                                const float* hull_verts, int hull_nv, const int* hull_tris,
                                                int hull_nt, int max_iters, int width, int width2, float threshold,
                                                int depth, int max_n_cutting, int verbose,
                                                int decompose_components, int decompose_components_per_iter,
                                                int n_concave_edges, float concave_eps, float concave_threshold,
                                                int concave_iters, struct gpu_result* out)
{
    if (!ctx || !out) return -1;
    unsigned long long st[3] = {0, 0, 0};
    Prune PR{scorer, top_k > 0 ? top_k : 1, margin, beam, st};
    MeshIn m{verts, nv, tris, nt, hull_verts, hull_nv, hull_tris, hull_nt};
    SearchParams P = search_params(max_iters, width, width2, threshold, depth, 0, max_n_cutting, verbose, 0,
                                   decompose_components, decompose_components_per_iter, n_concave_edges, concave_eps,
                                   concave_threshold, concave_iters, 0, 1);
    int rc = search_group(ctx, 1, &m, P, &PR, nullptr, out);
    if (out_stats) for (int k = 0; k < 3; k++) out_stats[k] = st[k];
    return rc;
}

extern "C" int cuacd_lookahead_decompose_batch(gpu_ctx_t ctx, int n_meshes,
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
                                               unsigned long long* out_stats, struct gpu_result* out)
{
    if (!ctx || !out || n_meshes < 0) return -1;
    if (n_meshes == 0) return 0;
    if (!verts || !vert_off || !tris || !tri_off || !hull_verts || !hull_vert_off || !hull_tris || !hull_tri_off)
        return ctx_fail(ctx, KERR_MESH_INVALID, "null mesh arrays");
    std::vector<MeshIn> M(n_meshes);
    for (int m = 0; m < n_meshes; m++) {
        if (vert_off[m + 1] < vert_off[m] || tri_off[m + 1] < tri_off[m] || hull_vert_off[m + 1] < hull_vert_off[m] ||
            hull_tri_off[m + 1] < hull_tri_off[m])
            return ctx_fail(ctx, KERR_MESH_INVALID, "mesh %d: decreasing offsets", m);
        M[m] = {verts + 3 * (size_t)vert_off[m], vert_off[m + 1] - vert_off[m], tris + 3 * (size_t)tri_off[m],
                tri_off[m + 1] - tri_off[m], hull_verts + 3 * (size_t)hull_vert_off[m],
                hull_vert_off[m + 1] - hull_vert_off[m], hull_tris + 3 * (size_t)hull_tri_off[m],
                hull_tri_off[m + 1] - hull_tri_off[m]};
    }
    for (int m = 0; m < n_meshes; m++) { out[m].parts = nullptr; out[m].nparts = 0; }
    unsigned long long pst[3] = {0, 0, 0};
    Prune PR{scorer, top_k > 0 ? top_k : 1, margin, beam, pst};
    const bool use_prune = scorer != nullptr || beam > 0;
    SearchParams P = search_params(max_iters, width, width2, threshold, depth, quick_depth, max_n_cutting, verbose,
                                   0, decompose_components, decompose_components_per_iter, n_concave_edges,
                                   concave_eps, concave_threshold, concave_iters, merge_hulls, branch_and_bound);
    unsigned long long st[ST_N] = {0, 0, 0, 0, 0, 0, 0, 0};
    // groups of consecutive meshes: the level output of a group's cutting parts
    // must fit one output arena
    const size_t group_elems = (size_t)3 << 20;
    const int group_meshes = 256;
    int g = 0, rc = 0;
    while (g < n_meshes && rc == 0) {
        size_t acc = 0;
        int g1 = g;
        while (g1 < n_meshes && g1 - g < group_meshes) {
            const size_t e = (size_t)M[g1].nv + M[g1].nt;
            if (g1 > g && acc + e > group_elems) break;
            acc += e; g1++;
        }
        rc = search_group(ctx, g1 - g, M.data() + g, P, use_prune ? &PR : nullptr, st, out + g);
        g = g1;
    }
    if (rc) { for (int m = 0; m < n_meshes; m++) gpu_result_free(&out[m]); }
    st[ST_RANKED] = pst[0]; st[ST_CUT] = pst[1]; st[ST_EXPANDED] = pst[2];
    if (out_stats) for (int k = 0; k < ST_N; k++) out_stats[k] = st[k];
    return rc;
}

extern "C" int cuacd_lookahead_trace(gpu_ctx_t ctx, cuacd_scorer_t scorer, float* out_rows, int max_rows,
                                     int* out_n_rows, const float* verts, int nv, const int* tris, int nt,
                                     const float* hull_verts, int hull_nv, const int* hull_tris, int hull_nt,
                                     int max_iters, int width, int width2, float threshold, int depth,
                                     int max_n_cutting, int n_concave_edges, float concave_eps,
                                     float concave_threshold, int concave_iters, struct gpu_result* out)
{
    if (!ctx) return -1;
    if (!scorer || !out_rows || !out_n_rows || max_rows < 0) return ctx_fail(ctx, -1, "bad trace arguments");
    *out_n_rows = 0;
    const int W = scorer_n_features() + 4;
    std::vector<float> rows;
    unsigned long long st[3] = {0, 0, 0};
    Prune PR{scorer, 0, 0.f, 0, st, &rows, (size_t)max_rows * W, 0, {}, {}};
    MeshIn m{verts, nv, tris, nt, hull_verts, hull_nv, hull_tris, hull_nt};
    // no branch and bound: every level-0 candidate's path cost is traced
    SearchParams P = search_params(max_iters, width, width2, threshold, depth, 0, max_n_cutting, 0, 0, 0, 1,
                                   n_concave_edges, concave_eps, concave_threshold, concave_iters, 0, 0);
    int rc = search_group(ctx, 1, &m, P, &PR, nullptr, out);
    if (rc) return rc;
    const int n = (int)(rows.size() / W);
    memcpy(out_rows, rows.data(), sizeof(float) * (size_t)n * W);
    *out_n_rows = n;
    return 0;
}
