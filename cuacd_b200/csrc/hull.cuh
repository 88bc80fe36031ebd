// hull.cuh — exact convex hulls of point clouds, batched (sm_100a).
//
// Replaces the reference's warp D&C hull (cuda/hull_dandc.cuh:1678-1861) and
// its k-DOP prefilter (cuda/kdop_hull.cuh:49-398) with one exact algorithm,
// run as three launches over a batch of clouds (kernels in hull.cu):
//
//   1. set-up, one CTA per cloud: quantise onto the reference grid
//      (hull_dandc.cuh:1351-1411: per-axis step span/10216, axes permuted to
//      (med,max,min), sign flip when (medAx+1)%3 != maxAx, truncation toward
//      zero, IEEE-rounded divisions; |q| <= 5109, stored as exact floats);
//      bucket by a 12-bit Morton code; implicit binary BVH over leaves of
//      HULL_LEAF points with per-leaf oriented boxes; the first face; the
//      frontier queue.
//   2. wrapping, a persistent grid: every warp takes frontier edges from any
//      cloud's queue.  The next face around edge (u,v) is found by a
//      depth-first branch-and-bound over the BVH that tightens the plane as
//      leaves are scanned.  Orientation tests run in FP32 with a static error
//      bound and fall back to exact FP64 near zero (grid predicates are
//      < 2^46, so FP64 is exact).  Coplanar points are merged into one polygon
//      face.  New faces go to a face hash set, their edges to an edge hash
//      set, unmatched edges to the queue.
//   3. output, one CTA per cloud: corners in ascending input index; each face
//      fanned from its smallest corner; triangles grouped by first vertex and
//      sorted; FP64 volume.
//
// Duplicate grid points resolve to the smallest input index, as the
// reference's (y,x,z,index) sort keeps the first (warp_sort.cuh:237-244).
#pragma once
#include "common.cuh"
#include "cta_util.cuh"

#ifndef HULL_NT
#define HULL_NT       512           // threads per hull CTA (set-up, wrap, output)
#endif
// Points per BVH leaf (8, 16 or 32).  32: a leaf is one point per lane of
// the scanning warp and the tree one level shallower; on the config-3 step
// the hull stage measured 5.06 ms (pruned) against 5.31 with 16 and 5.2
// with 8, the same hulls.
#ifndef HULL_LEAF
#define HULL_LEAF     32
#endif
#define HULL_SMALL_S  24
#define HULL_MORTON_BITS 4            // bits per axis for the bucket sort
#define HULL_CELLS    (1 << (3 * HULL_MORTON_BITS))
// Shared ints per warp while wrapping (dynamic) and, of which, the node
// stack; the rest is the kept-leaf list.  (The CPU emulation of the tests
// builds with much smaller lists to drive the overflow paths.)
#ifndef HULL_WSM
#define HULL_WSM      1024
#endif
#ifndef HULL_WQ
#define HULL_WQ       704
#endif
#define HULL_WL       (HULL_WSM - HULL_WQ)         //           kept-leaf list
#define HULL_WRAP_DSMEM ((size_t)(HULL_NT / 32) * HULL_WSM * sizeof(int))
#define HULL_SEEDS    6                            // seed faces that start the wrapping of a cloud of at
                                                   // least seed_min_n points (the tuned size class decides;
                                                   // smaller clouds start from one)

// Per-cloud scratch layout (bytes computed on the host by hull_scratch_bytes).
struct HullCaps {
    int n, m_leaves, P;      // points, leaves, leaf slots (pow2)
    int hcap, ccap, fcap, fr_cap, eh, fh;
};

__host__ __device__ inline int hull_pow2(int x) { int p = 1; while (p < x) p <<= 1; return p; }

// Hull vertex capacity of the first attempt at an n-point cloud: every
// point up to HULL_FIRST_CAP points, beyond that a quarter of them (at least
// HULL_FIRST_CAP).  Fragments of meshes have far fewer hull vertices than
// points (a 20,000-point sphere fragment about 2,800), so their edge set,
// face set and frontier queue -- cleared at set-up, probed while wrapping --
// start four times smaller; a cloud whose hull outgrows them (a convex
// cloud, such as the vertices of a fine sphere, has every point on its hull)
// is built again with h = n in the same launch sequence.
// Clouds above reduce_max_n points start at full size: large clouds are
// often convex-ish (a whole input mesh), and a second attempt at them would
// repeat most of the wrapping (the tuned size class sets the limit).
#define HULL_FIRST_CAP 4096
__host__ __device__ inline int hull_first_cap(int n, int reduce_max_n = 1 << 30)
{
    if (n <= HULL_FIRST_CAP || n > reduce_max_n) return n;
    return n / 4 > HULL_FIRST_CAP ? n / 4 : HULL_FIRST_CAP;
}

// Table capacities of an n-point cloud built with room for h hull vertices.
// Clouds are limited to 2^22 points, which keeps every table within int range.
__host__ __device__ inline HullCaps hull_caps(int n, int h)
{
    HullCaps c;
    c.n = n;
    c.m_leaves = (n + HULL_LEAF - 1) / HULL_LEAF;
    if (c.m_leaves < 1) c.m_leaves = 1;
    c.P = hull_pow2(c.m_leaves);
    if (h > n) h = n;
    if (h < 4) h = 4;
    if (h > (1 << 22)) h = 1 << 22;
    c.hcap = h;
    c.ccap = 6 * h + 64;
    c.fcap = 2 * h + 8;
    c.fr_cap = 6 * h + 64;
    c.eh = hull_pow2(2 * c.ccap);
    c.fh = hull_pow2(2 * c.fcap);
    return c;
}

__host__ __device__ inline size_t hull_align(size_t x) { return (x + 255) & ~(size_t)255; }


// ---------------------------------------------------------------------------
// exact grid geometry
// ---------------------------------------------------------------------------
struct HullCtx {
    const float4* __restrict__ pts;     // (qx,qy,qz, input index as int bits)
    const float4* __restrict__ nlo;     // node boxes, heap order [1, 2P)
    const float4* __restrict__ nhi;
    const float4* __restrict__ obb;     // per leaf: centre (w = 1 if valid), axes e1..e3 with half extents in w
    int m, P, nleaf;
};

// Bounds of N.(x - a) over a leaf's points from its oriented box:
// N.(c - a) -+ (sum_i h_i |N.e_i| + margin).  The margin covers the float
// rounding of the stored axes (|N|_1 * 1e-5 * (sum h + 1)).  c - a is formed
// in FP64, where it is exact: the centre is not on the grid, and a float
// difference would be off by up to half an ulp of |c - a| (5e-4 grid units),
// more than the margin of a flat leaf lying in the plane -- its points would
// then be cut from the face.
static __device__ __forceinline__ bool leaf_obb(const HullCtx& H, int leaf, double nx, double ny, double nz,
                                                float4 a, double* lo, double* hi)
{
    float4 c = H.obb[4 * leaf];
    if (c.w == 0.f) return false;
    float4 e1 = H.obb[4 * leaf + 1], e2 = H.obb[4 * leaf + 2], e3 = H.obb[4 * leaf + 3];
    double mid = nx * ((double)c.x - (double)a.x) + ny * ((double)c.y - (double)a.y) + nz * ((double)c.z - (double)a.z);
    double r = fabs(nx * e1.x + ny * e1.y + nz * e1.z) * e1.w + fabs(nx * e2.x + ny * e2.y + nz * e2.z) * e2.w
             + fabs(nx * e3.x + ny * e3.y + nz * e3.z) * e3.w;
    r += (fabs(nx) + fabs(ny) + fabs(nz)) * 1e-5 * ((double)e1.w + e2.w + e3.w + 1.0);
    *lo = mid - r; *hi = mid + r;
    return true;
}

static __device__ __forceinline__ int pidx(float4 p) { return __float_as_int(p.w); }

// Sign of N.(q - a) for integer-valued N (|N| < 2^30) and grid points,
// FP32 with error bound, exact FP64 fallback.
static __device__ __forceinline__ int plane_sign(double nx, double ny, double nz,
                                          float fx, float fy, float fz,
                                          float4 a, float4 q, unsigned& n64)
{
    float ex = q.x - a.x, ey = q.y - a.y, ez = q.z - a.z;     // exact
    float s = fmaf(fz, ez, fmaf(fy, ey, fx * ex));
    float bound = fmaf(fabsf(fz), fabsf(ez), fmaf(fabsf(fy), fabsf(ey), fabsf(fx) * fabsf(ex))) * 4.8e-7f;
    if (s > bound) return 1;
    if (s < -bound) return -1;
    n64++;
    double d = nx * (double)ex + ny * (double)ey + nz * (double)ez;   // exact
    return (d > 0.0) - (d < 0.0);
}

// Is q on the line through a with integer direction d?  (exact int32)
static __device__ __forceinline__ bool on_line(int dx, int dy, int dz, float4 a, float4 q)
{
    int ex = (int)(q.x - a.x), ey = (int)(q.y - a.y), ez = (int)(q.z - a.z);
    return (dy * ez - dz * ey) == 0 && (dz * ex - dx * ez) == 0 && (dx * ey - dy * ex) == 0;
}

// min over the box of N.(x - a)
static __device__ __forceinline__ double box_min(double nx, double ny, double nz, float4 lo, float4 hi, float4 a)
{
    double r = nx * (double)(nx >= 0 ? lo.x - a.x : hi.x - a.x)
             + ny * (double)(ny >= 0 ? lo.y - a.y : hi.y - a.y)
             + nz * (double)(nz >= 0 ? lo.z - a.z : hi.z - a.z);
    return r;
}
static __device__ __forceinline__ double box_max(double nx, double ny, double nz, float4 lo, float4 hi, float4 a)
{
    double r = nx * (double)(nx >= 0 ? hi.x - a.x : lo.x - a.x)
             + ny * (double)(ny >= 0 ? hi.y - a.y : lo.y - a.y)
             + nz * (double)(nz >= 0 ? hi.z - a.z : lo.z - a.z);
    return r;
}

// Wrap: rotate the supporting plane about the line (a, d) into the cloud and
// return the first point hit (sorted-point id), or -1 when every point lies
// on the line.  q replaces c when (d x (c - a)).(q - a) < 0.
static __device__ int hull_wrap(const HullCtx& H, int a_id, int dx, int dy, int dz, int start_leaf,
                                unsigned& n_pts, unsigned& n64)
{
    float4 a = H.pts[a_id];
    int c = -1;
    double mx = 0, my = 0, mz = 0;
    float fx = 0, fy = 0, fz = 0;
    auto consider = [&](int qi) {
        float4 q = H.pts[qi];
        n_pts++;
        if (on_line(dx, dy, dz, a, q)) return;
        bool take = (c < 0);
        if (!take) take = plane_sign(mx, my, mz, fx, fy, fz, a, q, n64) < 0;
        if (take) {
            c = qi;
            double ex = q.x - a.x, ey = q.y - a.y, ez = q.z - a.z;
            mx = dy * ez - dz * ey; my = dz * ex - dx * ez; mz = dx * ey - dy * ex;
            fx = (float)mx; fy = (float)my; fz = (float)mz;
        }
    };
    // seed from the leaf holding `a`
    {
        int lo = start_leaf * HULL_LEAF, hi = min(lo + HULL_LEAF, H.m);
        for (int i = lo; i < hi; i++) consider(i);
    }
    int stack[40];
    int sp = 0;
    stack[sp++] = 1;
    while (sp > 0) {
        int node = stack[--sp];
        float4 lo = H.nlo[node], hi = H.nhi[node];
        if (lo.x > hi.x) continue;                         // empty
        if (c >= 0 && box_min(mx, my, mz, lo, hi, a) >= 0.0) continue;
        if (node >= H.P) {
            int leaf = node - H.P;
            if (leaf == start_leaf) continue;
            int l0 = leaf * HULL_LEAF, l1 = min(l0 + HULL_LEAF, H.m);
            for (int i = l0; i < l1; i++) consider(i);
        } else {
            int l = 2 * node, r = 2 * node + 1;
            if (c >= 0) {
                double bl = box_min(mx, my, mz, H.nlo[l], H.nhi[l], a);
                double br = box_min(mx, my, mz, H.nlo[r], H.nhi[r], a);
                if (bl < br) { stack[sp++] = r; stack[sp++] = l; }
                else         { stack[sp++] = l; stack[sp++] = r; }
            } else { stack[sp++] = r; stack[sp++] = l; }
        }
    }
    return c;
}

// Collect up to `cap` points on the plane through a with outward normal N
// (all points satisfy N.(q-a) <= 0).  Returns the count (may exceed cap:
// the caller then treats the face as large).
static __device__ int hull_coplanar(const HullCtx& H, int a_id, double nx, double ny, double nz, int* out, int cap,
                                    unsigned& n_pts, unsigned& n64)
{
    float4 a = H.pts[a_id];
    float fx = (float)nx, fy = (float)ny, fz = (float)nz;
    int cnt = 0;
    int stack[40];
    int sp = 0;
    stack[sp++] = 1;
    while (sp > 0) {
        int node = stack[--sp];
        float4 lo = H.nlo[node], hi = H.nhi[node];
        if (lo.x > hi.x) continue;
        if (box_max(nx, ny, nz, lo, hi, a) < 0.0) continue;
        if (node >= H.P) {
            int leaf = node - H.P;
            int l0 = leaf * HULL_LEAF, l1 = min(l0 + HULL_LEAF, H.m);
            for (int i = l0; i < l1; i++) {
                n_pts++;
                if (plane_sign(nx, ny, nz, fx, fy, fz, a, H.pts[i], n64) == 0) {
                    if (cnt < cap) out[cnt] = i;
                    cnt++;
                }
            }
        } else {
            stack[sp++] = 2 * node + 1;
            stack[sp++] = 2 * node;
        }
    }
    return cnt;
}

// Per-warp scratch of the cooperative wrap.  The node queue and the leaf
// list live in global scratch sized to the whole tree, so they never overflow.
struct HullWarp {
    int S[HULL_SMALL_S + 8];   // coplanar points of the new face
};

// A warp's work lists (same value on every lane): the BVH node stack, reused
// as the coplanar leaf list, and the leaves reached by the sweep, with their
// capacities (shared memory first, the global 2P / P lists when too small).
struct WarpLists {
    int* q; int* leaf;
    int qcap, lcap;
};

// Is q strictly beyond the plane through a spanned by d and (c - a)?
static __device__ __forceinline__ bool wrap_better(float4 a, int dx, int dy, int dz, float4 c, float4 q, unsigned& n64)
{
    double ex = c.x - a.x, ey = c.y - a.y, ez = c.z - a.z;
    double mx = dy * ez - dz * ey, my = dz * ex - dx * ez, mz = dx * ey - dy * ex;
    return plane_sign(mx, my, mz, (float)mx, (float)my, (float)mz, a, q, n64) < 0;
}

// Warp-wide best candidate (comparator reduction), broadcast from lane 0.
static __device__ __forceinline__ void warp_best(int& ci, float4& cq, float4 a, int dx, int dy, int dz, unsigned& n64)
{
    #pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        int c2 = __shfl_xor_sync(FULL_MASK, ci, o);
        float4 q2;
        q2.x = __shfl_xor_sync(FULL_MASK, cq.x, o); q2.y = __shfl_xor_sync(FULL_MASK, cq.y, o);
        q2.z = __shfl_xor_sync(FULL_MASK, cq.z, o); q2.w = __shfl_xor_sync(FULL_MASK, cq.w, o);
        if (c2 >= 0 && (ci < 0 || wrap_better(a, dx, dy, dz, cq, q2, n64))) { ci = c2; cq = q2; }
    }
    ci = __shfl_sync(FULL_MASK, ci, 0);
    cq.x = __shfl_sync(FULL_MASK, cq.x, 0); cq.y = __shfl_sync(FULL_MASK, cq.y, 0);
    cq.z = __shfl_sync(FULL_MASK, cq.z, 0); cq.w = __shfl_sync(FULL_MASK, cq.w, 0);
}

// Warp-cooperative wrap about edge (u, v): seed the candidate from the
// leaves holding u and v, then sweep the BVH depth first keeping every box
// that reaches on or beyond the current plane (strict pruning, so the kept
// leaves also hold every point of the final face), scanning kept leaves'
// points on 32 lanes as they are reached and reducing with the exact
// comparator.
// Returns c (sorted id), -1 if all points are on the line, -2 if the warp
// queues overflowed (the caller then uses the serial search).
// ties_out (optional, edge mode): how many scanned points other than u, v
// and c lie on the final plane (every point of the line through u and v
// counts), same value on every lane; 0 means the face is the triangle
// (v, u, c).  Exact: every point on the final plane is scanned (its box is
// never strictly behind an earlier plane), and a point on it scanned under
// an earlier plane would have become the candidate, so each is either the
// candidate or counted against the plane it lies on -- a lane's count
// survives a reduction only when its own candidate lies on the winning
// plane (the two planes are then the same).
static __device__ int warp_wrap(const HullCtx& H, int u, int v, const WarpLists W, int lane, int* nleaf_out,
                                unsigned& n_pts, unsigned& n64, const int* dir = nullptr, int* ties_out = nullptr)
{
    // dir: wrap about the line through u with this direction (v unused)
    const unsigned lt = (1u << lane) - 1u;
    float4 a = H.pts[u], pv = dir ? a : H.pts[v];
    const int dx = dir ? dir[0] : (int)(pv.x - a.x), dy = dir ? dir[1] : (int)(pv.y - a.y);
    const int dz = dir ? dir[2] : (int)(pv.z - a.z);
    if (dir) v = u;
    int ci = -1; float4 cq = a;
    double mx = 0, my = 0, mz = 0; float fx = 0, fy = 0, fz = 0;
    auto setm = [&]() {
        double ex = cq.x - a.x, ey = cq.y - a.y, ez = cq.z - a.z;
        mx = dy * ez - dz * ey; my = dz * ex - dx * ez; mz = dx * ey - dy * ex;
        fx = (float)mx; fy = (float)my; fz = (float)mz;
    };
    int tie = 0, online = 0;         // points on this lane's plane / on the line (other than u, v)
    auto take = [&](int qi) {
        float4 q = H.pts[qi];
        n_pts++;
        if (on_line(dx, dy, dz, a, q)) { online += (qi != u && qi != v); return; }
        if (ci < 0) { ci = qi; cq = q; setm(); tie = 0; return; }
        const int sg = plane_sign(mx, my, mz, fx, fy, fz, a, q, n64);
        if (sg < 0) { ci = qi; cq = q; setm(); tie = 0; }
        else if (sg == 0 && qi != ci) tie++;
    };
    // warp reduction of the candidates; each lane's tie count follows it
    auto reduce = [&]() {
        const int c0 = ci; const float4 q0 = cq;
        warp_best(ci, cq, a, dx, dy, dz, n64);
        if (ci >= 0) setm();
        if (ci != c0) tie = (c0 >= 0 && plane_sign(mx, my, mz, fx, fy, fz, a, q0, n64) == 0) ? tie + 1 : 0;
    };
    {
        // the leaves of u and v (with leaves of 8 points, also their
        // siblings, the neighbouring stretch of the sorted points)
        const int lu = u / HULL_LEAF, lv = v / HULL_LEAF;
        constexpr int n_seed = HULL_LEAF >= 16 ? 2 : 4;
        for (int k = lane; k < n_seed * HULL_LEAF; k += 32) {
            const int sl = k / HULL_LEAF;
            if (sl == 1 && lv == lu) continue;
            const int lf = (sl & 1 ? lv : lu) ^ (sl >> 1);
            const int i = lf * HULL_LEAF + (k % HULL_LEAF);
            if (lf < H.nleaf && i < H.m) take(i);
        }
    }
    reduce();
    // Depth-first sweep, 32 nodes per step from the top of a warp stack.
    // Each step's newly kept leaves are scanned at once, so the plane
    // tightens while the sweep is still near the seed and later boxes are
    // pruned against it.  Every leaf not pruned when reached is recorded:
    // a point on the final plane is never strictly below an earlier (less
    // rotated) plane, so the list holds the final face's points.
    // The sweep starts from the tree level with min(32, P) nodes (fewer if
    // the stack is short) rather than the root: the levels above it hold fewer nodes than lanes, and walking
    // them costs dependent steps with idle lanes.  A box contains its
    // children's boxes, so a node the root walk would prune has every
    // descendant pruned here too; only the order of the visits changes.
    int d0 = 1;
    while (d0 < 32 && d0 < H.P && 4 * d0 <= W.qcap) d0 <<= 1;
    int sp = d0, nl = 0, scanned = 0;
    if (lane < d0) W.q[lane] = d0 + lane;
    __syncwarp();
    while (sp > 0) {
        // pop at most as many nodes as the stack has room for children of
        // (a step grows the stack by at most the nodes it pops)
        const int batch = min(min(32, sp), W.qcap - sp);
        if (batch <= 0) return -2;
        const int base = sp - batch;
        const int node = lane < batch ? W.q[base + lane] : 0;
        __syncwarp();                                   // all pops read before pushes overwrite
        bool kl = false, ki = false;
        if (lane < batch) {
            float4 lo = H.nlo[node], hi = H.nhi[node];
            bool pruned = lo.x > hi.x || (ci >= 0 && box_min(mx, my, mz, lo, hi, a) > 0.0);
            if (!pruned && ci >= 0 && node >= H.P) {
                double olo, ohi;
                if (leaf_obb(H, node - H.P, mx, my, mz, a, &olo, &ohi) && olo > 0.0) pruned = true;
            }
            if (!pruned) { if (node >= H.P) kl = true; else ki = true; }
        }
        const unsigned bl = __ballot_sync(FULL_MASK, kl), bi = __ballot_sync(FULL_MASK, ki);
        const int nbl = __popc(bl), nbi = __popc(bi);
        if (nl + nbl > W.lcap && ci >= 0) {
            // Leaf list full: drop the recorded leaves that the current
            // plane now prunes.  Their points were scanned already
            // (scanned == nl here), and a point of the final face is never
            // strictly beyond an earlier plane, so none of them can be on
            // it.  In place: an entry moves to a position <= its own, after
            // every lane has read its entry of the chunk.
            int nk = 0;
            for (int b0 = 0; b0 < nl; b0 += 32) {
                const int j = b0 + lane;
                int lf = 0;
                bool keep = false;
                if (j < nl) {
                    lf = W.leaf[j];
                    keep = !(box_min(mx, my, mz, H.nlo[lf + H.P], H.nhi[lf + H.P], a) > 0.0);
                    double olo, ohi;
                    if (keep && leaf_obb(H, lf, mx, my, mz, a, &olo, &ohi) && olo > 0.0) keep = false;
                }
                const unsigned bk = __ballot_sync(FULL_MASK, keep);
                if (keep) W.leaf[nk + __popc(bk & lt)] = lf;
                nk += __popc(bk);
                __syncwarp();
            }
            nl = nk; scanned = nk;
        }
        if (nl + nbl > W.lcap || base + 2 * nbi > W.qcap) return -2;
        if (kl) W.leaf[nl + __popc(bl & lt)] = node - H.P;
        if (ki) { int p = base + 2 * __popc(bi & lt); W.q[p] = 2 * node; W.q[p + 1] = 2 * node + 1; }
        __syncwarp();
        sp = base + 2 * nbi; nl += nbl;
        if (nl > scanned) {                             // scan the new leaves, tighten the plane
            const int total = (nl - scanned) * HULL_LEAF;
            const int ci0 = ci;
            for (int i = lane; i < total; i += 32) {
                int p = W.leaf[scanned + i / HULL_LEAF] * HULL_LEAF + (i % HULL_LEAF);
                if (p < H.m) take(p);
            }
            // reduce only when some lane found a better point
            if (__any_sync(FULL_MASK, ci != ci0)) reduce();
            scanned = nl;
        }
    }
    *nleaf_out = nl;
    if (ties_out) {
        int t = tie + online;
        #pragma unroll
        for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(FULL_MASK, t, o);
        *ties_out = t;
    }
    return ci;
}

// Points of the kept leaves lying on the plane through a with outward normal
// N (all points satisfy N.(q-a) <= 0).  Leaves whose box stays below the
// plane are skipped first.  Returns the count; the first `cap` ids go to W.S.
// Does any point of the kept leaves lie on the plane (a, N) but off the line
// through a with integer direction e?  (Whole warp; the answer is uniform.)
static __device__ bool warp_any_off_line(const HullCtx& H, const WarpLists L, int nl, float4 a, double nx, double ny,
                                         double nz, int ex, int ey, int ez, int lane, unsigned& n64)
{
    const float fx = (float)nx, fy = (float)ny, fz = (float)nz;
    const int total = nl * HULL_LEAF;
    bool any = false;
    for (int base = 0; base < total && !any; base += 32) {
        const int i = base + lane;
        bool off = false;
        if (i < total) {
            const int p = L.leaf[i / HULL_LEAF] * HULL_LEAF + (i % HULL_LEAF);
            if (p < H.m) {
                const float4 q = H.pts[p];
                off = plane_sign(nx, ny, nz, fx, fy, fz, a, q, n64) == 0 && !on_line(ex, ey, ez, a, q);
            }
        }
        any = __any_sync(FULL_MASK, off);
    }
    return any;
}

static __device__ int warp_coplanar(const HullCtx& H, float4 a, double nx, double ny, double nz, HullWarp& W,
                                    const WarpLists L, int nl, int lane, int cap, unsigned& n_pts, unsigned& n64)
{
    const unsigned lt = (1u << lane) - 1u;
    const float fx = (float)nx, fy = (float)ny, fz = (float)nz;
    int nk = 0;
    for (int base = 0; base < nl; base += 32) {
        int j = base + lane;
        bool keep = false;
        if (j < nl) {
            int node = L.leaf[j] + H.P;
            keep = box_max(nx, ny, nz, H.nlo[node], H.nhi[node], a) >= 0.0;
            double olo, ohi;
            if (keep && leaf_obb(H, L.leaf[j], nx, ny, nz, a, &olo, &ohi) && ohi < 0.0) keep = false;
        }
        unsigned b = __ballot_sync(FULL_MASK, keep);
        if (keep) L.q[nk + __popc(b & lt)] = L.leaf[j];
        nk += __popc(b);
    }
    __syncwarp();
    int cnt = 0;
    const int total = nk * HULL_LEAF;
    for (int base = 0; base < total; base += 32) {
        int i = base + lane, p = -1;
        bool on = false;
        if (i < total) {
            p = L.q[i / HULL_LEAF] * HULL_LEAF + (i % HULL_LEAF);
            if (p < H.m) { n_pts++; on = plane_sign(nx, ny, nz, fx, fy, fz, a, H.pts[p], n64) == 0; }
        }
        unsigned b = __ballot_sync(FULL_MASK, on);
        if (on) { int pos = cnt + __popc(b & lt); if (pos < cap) W.S[pos] = p; }
        cnt += __popc(b);
    }
    __syncwarp();
    return cnt;
}

// 2D projection dropping the dominant component of N; sign makes CCW
// (w.r.t. N) positive.
struct Proj { int ku, kv; int sgn; };
static __device__ __forceinline__ Proj make_proj(double nx, double ny, double nz)
{
    double ax = fabs(nx), ay = fabs(ny), az = fabs(nz);
    int k = (ax >= ay && ax >= az) ? 0 : (ay >= az ? 1 : 2);
    double nk = k == 0 ? nx : (k == 1 ? ny : nz);
    Proj p; p.ku = (k + 1) % 3; p.kv = (k + 2) % 3; p.sgn = nk > 0 ? 1 : -1;
    return p;
}
static __device__ __forceinline__ float comp(float4 p, int k) { return k == 0 ? p.x : (k == 1 ? p.y : p.z); }

// 2D orientation of (p, r, t) in projected grid units (exact in int64)
static __device__ __forceinline__ long long o2d(const Proj& P, float4 p, float4 r, float4 t)
{
    long long ux = (long long)(comp(r, P.ku) - comp(p, P.ku)), uy = (long long)(comp(r, P.kv) - comp(p, P.kv));
    long long wx = (long long)(comp(t, P.ku) - comp(p, P.ku)), wy = (long long)(comp(t, P.kv) - comp(p, P.kv));
    return (ux * wy - uy * wx) * P.sgn;
}
static __device__ __forceinline__ long long d2d(const Proj& P, float4 p, float4 r)
{
    long long ux = (long long)(comp(r, P.ku) - comp(p, P.ku)), uy = (long long)(comp(r, P.kv) - comp(p, P.kv));
    return ux * ux + uy * uy;
}
static __device__ __forceinline__ bool same_pos(float4 a, float4 b) { return a.x == b.x && a.y == b.y && a.z == b.z; }

// Is candidate t better than r as the next CCW corner after cur?
static __device__ __forceinline__ bool next_better(const Proj& P, float4 cur, float4 r, float4 t)
{
    long long o = o2d(P, cur, r, t);
    if (o < 0) return true;
    if (o > 0) return false;
    if (same_pos(t, r)) return pidx(t) < pidx(r);
    return d2d(P, cur, t) > d2d(P, cur, r);
}

// Serial polygon walk over a small coplanar set; writes corners (sorted-point
// ids) starting with prev, cur.  Returns the corner count or -1.
static __device__ int hull_small_polygon(const HullCtx& H, const int* S, int ns, double nx, double ny, double nz,
                                  int prev, int cur, int* out)
{
    Proj P = make_proj(nx, ny, nz);
    int k = 0;
    out[k++] = prev;
    for (int guard = 0; guard <= ns; guard++) {
        out[k++] = cur;
        float4 pc = H.pts[cur];
        int r = -1; float4 pr = pc;
        for (int i = 0; i < ns; i++) {
            float4 pt = H.pts[S[i]];
            if (same_pos(pt, pc)) continue;
            if (r < 0 || next_better(P, pc, pr, pt)) { r = S[i]; pr = pt; }
        }
        if (r < 0) return -1;
        if (same_pos(pr, H.pts[prev])) return k;
        cur = r;
        if (k >= ns + 1) return -1;
    }
    return -1;
}

// Large coplanar face (more than HULL_SMALL_S points) built by one warp:
// collect the face's points from the kept leaves into Sg, then walk the
// polygon CCW from (v, u) with a warp-wide comparator reduction per corner.
// Corners go to Pg; returns their count or -1.
static __device__ int warp_big_polygon(const HullCtx& H, int u, int v, double nx, double ny, double nz,
                                       const int* leaves, int nl, int* Sg, int* Pg, int lane,
                                       unsigned& n_pts, unsigned& n64)
{
    const unsigned lt = (1u << lane) - 1u;
    const float4 a = H.pts[u];
    const float fx = (float)nx, fy = (float)ny, fz = (float)nz;
    int ns = nl < 0 ? -nl : 0;     // nl < 0: Sg already holds -nl points
    for (int base = 0; nl > 0 && base < nl * HULL_LEAF; base += 32) {
        int i = base + lane, p = -1;
        bool on = false;
        if (i < nl * HULL_LEAF) {
            p = leaves[i / HULL_LEAF] * HULL_LEAF + (i % HULL_LEAF);
            if (p < H.m) { n_pts++; on = plane_sign(nx, ny, nz, fx, fy, fz, a, H.pts[p], n64) == 0; }
        }
        unsigned b = __ballot_sync(FULL_MASK, on);
        if (on) Sg[ns + __popc(b & lt)] = p;
        ns += __popc(b);
    }
    __syncwarp();
    const Proj PR = make_proj(nx, ny, nz);
    const float4 pv4 = H.pts[v];
    if (lane == 0) Pg[0] = v;
    int k = 1, cur = u;
    for (int guard = 0; guard <= ns; guard++) {
        if (lane == 0) Pg[k] = cur;
        k++;
        const float4 pc = H.pts[cur];
        int r = -1; float4 pr = pc;
        for (int i = lane; i < ns; i += 32) {
            float4 pt = H.pts[Sg[i]];
            if (same_pos(pt, pc)) continue;
            if (r < 0 || next_better(PR, pc, pr, pt)) { r = Sg[i]; pr = pt; }
        }
        #pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            int r2 = __shfl_xor_sync(FULL_MASK, r, o);
            float4 p2;
            p2.x = __shfl_xor_sync(FULL_MASK, pr.x, o); p2.y = __shfl_xor_sync(FULL_MASK, pr.y, o);
            p2.z = __shfl_xor_sync(FULL_MASK, pr.z, o); p2.w = __shfl_xor_sync(FULL_MASK, pr.w, o);
            if (r2 >= 0 && (r < 0 || next_better(PR, pc, pr, p2))) { r = r2; pr = p2; }
        }
        r = __shfl_sync(FULL_MASK, r, 0);
        pr.x = __shfl_sync(FULL_MASK, pr.x, 0); pr.y = __shfl_sync(FULL_MASK, pr.y, 0);
        pr.z = __shfl_sync(FULL_MASK, pr.z, 0); pr.w = __shfl_sync(FULL_MASK, pr.w, 0);
        if (r < 0) return -1;
        if (same_pos(pr, pv4)) { __syncwarp(); return k; }
        cur = r;
    }
    return -1;
}

// ---------------------------------------------------------------------------
// hash sets of 64-bit keys (open addressing, empty = ~0)
// ---------------------------------------------------------------------------
static __device__ __forceinline__ unsigned long long ekey(int u, int v) {
    return ((unsigned long long)(unsigned)u << 32) | (unsigned)v;
}
static __device__ __forceinline__ unsigned hslot(unsigned long long k, int cap) {
    return (unsigned)((k * 0x9E3779B97F4A7C15ull) >> 32) & (unsigned)(cap - 1);
}
// returns 1 inserted, 0 present, -1 full
static __device__ __forceinline__ int hset_insert(unsigned long long* tab, int cap, unsigned long long k) {
    unsigned s = hslot(k, cap);
    for (int i = 0; i < cap; i++) {
        unsigned long long prev = atomicCAS(&tab[s], ~0ull, k);
        if (prev == ~0ull) return 1;
        if (prev == k) return 0;
        s = (s + 1) & (unsigned)(cap - 1);
    }
    return -1;
}
static __device__ __forceinline__ bool hset_has(const unsigned long long* tab, int cap, unsigned long long k) {
    unsigned s = hslot(k, cap);
    for (int i = 0; i < cap; i++) {
        unsigned long long x = __ldcg(&tab[s]);
        if (x == k) return true;
        if (x == ~0ull) return false;
        s = (s + 1) & (unsigned)(cap - 1);
    }
    return false;
}

// ---------------------------------------------------------------------------
// batched hull pipeline: setup (one CTA per hull), wrapping (a persistent
// grid whose warps take frontier edges from any hull's queue), output (one
// CTA per hull).  Per-hull state lives in global memory (HullState).
// ---------------------------------------------------------------------------
struct HullJob {               // one hull to build (device pointers)
    const float* pts; int n;   // the cloud, AoS xyz
    const int* tris; int nt;   // optional: mesh triangles over pts (mesh volume)
    float* out_v; int* out_t;  // null: outputs are taken from the output arena
    int max_hv, max_ht;        //       (capacities n and 2n+4)
};

struct HullRes {               // per job
    float* hv; int* ht; int hnv, hnt;
    double mesh_vol;           // |signed volume| of (pts, tris), 0 without tris
    float hull_vol; int err;
};

struct HullState {             // per hull, global memory
    float4* P4; float4* nlo; float4* nhi; float4* obb;
    unsigned long long* eset; unsigned long long* fset; unsigned long long* Q;
    int2* faces; int* corners; int* Sbuf; int* posn; int* ocnt;
    int n, P, m_leaves, eh, fh, fcap, ccap, qcap;
    int hcap;                  // hull vertex capacity its tables were sized for
    int retry;                 // 1: its tables overflowed on the first attempt; build again at h = n
    int q_head, q_tail, q_pending, n_faces, n_corners, err;
    int active;                // 1 while its frontier queue has work
    int lock;                  // guards Sbuf/posn/ocnt while wrapping (large faces)
    long long wbase;           // wrap-grid share: prefix of the active hulls' point counts
    double mesh_vol;
    int fail[8];               // first construction failure: site, u, v, c, ns, k, input index of u, of v
    unsigned long long stats[8];   // leaves kept by wraps, wraps, faces, points
                                   // tested by wraps, set-up cycles, device
                                   // time (ns) of the first edge taken and of
                                   // completion, large faces (+ 2^32 per wrap
                                   // and 2^48 per face on the hull's own lists)
};

// Scratch of one attempt at an n-point cloud with room for h hull vertices.
__host__ __device__ inline size_t hull_attempt_bytes(int n, int h)
{
    HullCaps c = hull_caps(n, h);
    size_t nn = (size_t)(n > 0 ? n : 1);
    size_t b = 0;
    b += hull_align(sizeof(float4) * nn);                             // pts
    b += hull_align(sizeof(float4) * 2 * (size_t)(2 * c.P));          // node lo/hi
    b += hull_align(sizeof(unsigned long long) * (size_t)c.eh);       // edge set
    b += hull_align(sizeof(unsigned long long) * (size_t)c.fh);       // face keys
    b += hull_align(sizeof(int2) * (size_t)c.fcap);                   // faces
    b += hull_align(sizeof(int) * (size_t)c.ccap);                    // corners
    b += hull_align(sizeof(unsigned long long) * 2 * (size_t)c.fr_cap); // frontier queue
    b += hull_align(sizeof(int) * nn);                                // coplanar set (set-up)
    b += hull_align(sizeof(int) * nn);                                // output positions
    b += hull_align(sizeof(int) * nn * 2);                            // owner count / fill
    b += hull_align(sizeof(float4) * 4 * (size_t)c.P);                // leaf OBBs
    return b;
}

// Scratch a cloud may use over both attempts (the first one's stays
// allocated while the second runs): what callers reserve per cloud.
__host__ __device__ inline size_t hull_scratch_bytes(int n, int reduce_max_n = 1 << 30)
{
    const int h1 = hull_first_cap(n, reduce_max_n);
    return hull_align(hull_attempt_bytes(n, h1)) + (h1 < n ? hull_align(hull_attempt_bytes(n, n)) : 0);
}

// Per-warp global lists of the wrapping grid, sized for clouds of up to
// n_max points: coplanar set and polygon (n_max + 2 each), node stack (2P)
// and leaf list (P).
__host__ __device__ inline size_t hull_warp_bytes(int n_max)
{
    HullCaps c = hull_caps(n_max > 4 ? n_max : 4, n_max);
    return hull_align(sizeof(int) * (2 * (size_t)(n_max + 2) + 3 * (size_t)c.P));
}

struct HullSetupShared {
    HullWarp ws[8];                    // coplanar points of the seed planes (one per seed warp)
    float mn[3], mx[3];
    float cen[3], inv[3];
    int ax[3];
    unsigned long long lexmin;
    int n_faces, n_corners, err;
    int n_S;
    int red_id[HULL_NT / 32];
    int scan[33];
    double dsh[33];
    int cells[HULL_CELLS];
};

struct HullWrapShared {
    HullWarp ws[HULL_NT / 32];
};

struct HullOutShared {
    int scan[34];
    double dsh[33];
};

static __device__ __forceinline__ HullCtx hull_ctx(const HullState& S)
{
    HullCtx H;
    H.pts = S.P4; H.nlo = S.nlo; H.nhi = S.nhi; H.obb = S.obb; H.m = S.n; H.P = S.P; H.nleaf = S.m_leaves;
    return H;
}

// Set-up of one hull (all HULL_NT threads): quantise and bucket-sort the
// points, build the BVH and the leaf boxes, clear the tables, build the
// first face and seed the frontier queue.  Writes the hull's state to *S;
// S->active = 1 when the queue holds work.  `scratch` holds
// hull_scratch_bytes(n) bytes.
// Set every entry of a table of 64-bit words to ~0 (all HULL_NT threads);
// n even and the table 16-byte aligned, so two entries go per store.
static __device__ __forceinline__ void cta_fill_ones64(unsigned long long* tab, int n, int tid)
{
    ulonglong2* t2 = reinterpret_cast<ulonglong2*>(tab);
    ulonglong2 ones;
    ones.x = ~0ull; ones.y = ~0ull;
    for (int i = tid; i < (n >> 1); i += HULL_NT) t2[i] = ones;
}

static __device__ void hull_setup_cta(const float* __restrict__ pts, int n, char* scratch, HullState* S,
                                      HullSetupShared& sh, int seed_min_n = 1 << 30, int hcap = 1 << 30)
{
    const int tid = threadIdx.x;
    const long long t_begin = clock64();
    HullCaps C = hull_caps(n, hcap);
    char* p = scratch;
    float4* P4 = (float4*)p;            p += hull_align(sizeof(float4) * (size_t)n);
    float4* nlo = (float4*)p;           p += hull_align(sizeof(float4) * 2 * (size_t)(2 * C.P));
    float4* nhi = nlo + 2 * C.P;
    unsigned long long* eset = (unsigned long long*)p; p += hull_align(sizeof(unsigned long long) * (size_t)C.eh);
    unsigned long long* fset = (unsigned long long*)p; p += hull_align(sizeof(unsigned long long) * (size_t)C.fh);
    int2* faces = (int2*)p;             p += hull_align(sizeof(int2) * (size_t)C.fcap);
    int* corners = (int*)p;             p += hull_align(sizeof(int) * (size_t)C.ccap);
    unsigned long long* Q = (unsigned long long*)p; p += hull_align(sizeof(unsigned long long) * 2 * (size_t)C.fr_cap);
    int* Sbuf = (int*)p;                p += hull_align(sizeof(int) * (size_t)n);
    int* posn = (int*)p;                p += hull_align(sizeof(int) * (size_t)n);
    int* ocnt = (int*)p;                p += hull_align(sizeof(int) * (size_t)n * 2);
    float4* obb = (float4*)p;
    const int qcap = 2 * C.fr_cap;
    if (tid == 0) {
        S->P4 = P4; S->nlo = nlo; S->nhi = nhi; S->obb = obb; S->eset = eset; S->fset = fset; S->Q = Q;
        S->faces = faces; S->corners = corners; S->Sbuf = Sbuf; S->posn = posn; S->ocnt = ocnt;
        S->n = n; S->P = C.P; S->m_leaves = C.m_leaves; S->eh = C.eh; S->fh = C.fh; S->fcap = C.fcap;
        S->ccap = C.ccap; S->qcap = qcap; S->hcap = C.hcap;
        S->q_head = 0; S->q_tail = 0; S->q_pending = 0; S->n_faces = 0; S->n_corners = 0; S->err = 0;
        S->active = 0; S->lock = 0;
        for (int k = 0; k < 8; k++) S->stats[k] = 0;
        sh.err = 0;
    }

    // ---- 1. bounding box and quantisation parameters
    {
        float lo[3] = {1e30f, 1e30f, 1e30f}, hi[3] = {-1e30f, -1e30f, -1e30f};
        for (int i = tid; i < n; i += HULL_NT)
            for (int k = 0; k < 3; k++) {
                float x = pts[3 * i + k];
                lo[k] = fminf(lo[k], x); hi[k] = fmaxf(hi[k], x);
            }
        for (int k = 0; k < 3; k++) { lo[k] = warp_min(lo[k]); hi[k] = warp_max(hi[k]); }
        __shared__ float red[2][3][HULL_NT / 32];
        if ((tid & 31) == 0) for (int k = 0; k < 3; k++) { red[0][k][tid >> 5] = lo[k]; red[1][k][tid >> 5] = hi[k]; }
        __syncthreads();
        if (tid == 0) {
            for (int k = 0; k < 3; k++) {
                float a = 1e30f, b = -1e30f;
                for (int w = 0; w < HULL_NT / 32; w++) { a = fminf(a, red[0][k][w]); b = fmaxf(b, red[1][k][w]); }
                sh.mn[k] = a; sh.mx[k] = b;
            }
            float span[3] = {sh.mx[0] - sh.mn[0], sh.mx[1] - sh.mn[1], sh.mx[2] - sh.mn[2]};
            int maxAx = (span[0] >= span[1]) ? ((span[0] >= span[2]) ? 0 : 2) : ((span[1] >= span[2]) ? 1 : 2);
            int minAx = (span[0] <= span[1]) ? ((span[0] <= span[2]) ? 0 : 2) : ((span[1] <= span[2]) ? 1 : 2);
            if (minAx == maxAx) minAx = (maxAx + 1) % 3;
            int medAx = 3 - maxAx - minAx;
            float sc[3];
            for (int k = 0; k < 3; k++) sc[k] = __fdiv_rn(span[k], 10216.0f);
            if (((medAx + 1) % 3) != maxAx) for (int k = 0; k < 3; k++) sc[k] = -sc[k];
            sh.ax[0] = medAx; sh.ax[1] = maxAx; sh.ax[2] = minAx;
            for (int k = 0; k < 3; k++) {
                int a = sh.ax[k];
                sh.cen[k] = __fmul_rn(__fadd_rn(sh.mn[a], sh.mx[a]), 0.5f);
                float s = sc[a];
                sh.inv[k] = (s != 0.0f) ? __fdiv_rn(1.0f, s) : 0.0f;
            }
        }
        __syncthreads();
    }
    // ---- 2. quantise + bucket sort by a coarse Morton code
    for (int i = tid; i < HULL_CELLS; i += HULL_NT) sh.cells[i] = 0;
    __syncthreads();
    auto qpoint = [&](int i, int* q) {
        for (int k = 0; k < 3; k++) {
            float d = __fsub_rn(pts[3 * i + sh.ax[k]], sh.cen[k]);
            q[k] = __float2int_rz(__fmul_rn(d, sh.inv[k]));
        }
    };
    auto cell_of = [&](const int* q) {
        unsigned c = 0;
        for (int b = HULL_MORTON_BITS - 1; b >= 0; b--)
            for (int k = 0; k < 3; k++) {
                unsigned u = (unsigned)(q[k] + 5120) >> (14 - HULL_MORTON_BITS);   // 0..15
                c = (c << 1) | ((u >> b) & 1u);
            }
        return (int)c;
    };
    for (int i = tid; i < n; i += HULL_NT) {
        int q[3]; qpoint(i, q);
        atomicAdd(&sh.cells[cell_of(q)], 1);
    }
    __syncthreads();
    {
        // exclusive scan of HULL_CELLS counts (HULL_CELLS / HULL_NT per thread)
        const int per = HULL_CELLS / HULL_NT;
        int loc[per], s = 0;
        for (int j = 0; j < per; j++) { loc[j] = sh.cells[tid * per + j]; s += loc[j]; }
        int tot;
        int ex = block_exclusive_scan(s, sh.scan, &tot);
        for (int j = 0; j < per; j++) { sh.cells[tid * per + j] = ex; ex += loc[j]; }
        __syncthreads();
    }
    for (int i = tid; i < n; i += HULL_NT) {
        int q[3]; qpoint(i, q);
        int slot = atomicAdd(&sh.cells[cell_of(q)], 1);
        P4[slot] = make_float4((float)q[0], (float)q[1], (float)q[2], __int_as_float(i));
    }
    __syncthreads();
    // ---- 3. BVH boxes: leaves then levels bottom-up
    for (int l = tid; l < C.P; l += HULL_NT) {
        float4 lo = make_float4(1e30f, 1e30f, 1e30f, 0.f), hi = make_float4(-1e30f, -1e30f, -1e30f, 0.f);
        if (l < C.m_leaves) {
            int a = l * HULL_LEAF, b = min(a + HULL_LEAF, n);
            for (int i = a; i < b; i++) {
                float4 q = P4[i];
                lo.x = fminf(lo.x, q.x); lo.y = fminf(lo.y, q.y); lo.z = fminf(lo.z, q.z);
                hi.x = fmaxf(hi.x, q.x); hi.y = fmaxf(hi.y, q.y); hi.z = fmaxf(hi.z, q.z);
            }
        }
        nlo[C.P + l] = lo; nhi[C.P + l] = hi;
        // oriented box: e1 towards the farthest point from the first, e2 the
        // farthest direction off that line, e3 = e1 x e2
        float4 ob[4] = {make_float4(0.f, 0.f, 0.f, 0.f), make_float4(0.f, 0.f, 0.f, 0.f),
                        make_float4(0.f, 0.f, 0.f, 0.f), make_float4(0.f, 0.f, 0.f, 0.f)};
        if (l < C.m_leaves) {
            int a = l * HULL_LEAF, b = min(a + HULL_LEAF, n);
            float4 x0 = P4[a];
            double best = 0; double e1[3] = {0, 0, 0};
            for (int i = a + 1; i < b; i++) {
                float4 q = P4[i];
                double dx = q.x - x0.x, dy = q.y - x0.y, dz = q.z - x0.z, d2 = dx * dx + dy * dy + dz * dz;
                if (d2 > best) { best = d2; e1[0] = dx; e1[1] = dy; e1[2] = dz; }
            }
            if (best > 0) {
                double inv = 1.0 / sqrt(best);
                e1[0] *= inv; e1[1] *= inv; e1[2] *= inv;
                double best2 = 0; double e2[3] = {0, 0, 0};
                for (int i = a + 1; i < b; i++) {
                    float4 q = P4[i];
                    double dx = q.x - x0.x, dy = q.y - x0.y, dz = q.z - x0.z;
                    double t = dx * e1[0] + dy * e1[1] + dz * e1[2];
                    double ox = dx - t * e1[0], oy = dy - t * e1[1], oz = dz - t * e1[2], d2 = ox * ox + oy * oy + oz * oz;
                    if (d2 > best2) { best2 = d2; e2[0] = ox; e2[1] = oy; e2[2] = oz; }
                }
                if (best2 > 1e-12) {
                    double inv2 = 1.0 / sqrt(best2);
                    e2[0] *= inv2; e2[1] *= inv2; e2[2] *= inv2;
                    double e3[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
                    float fe[3][3];
                    for (int k = 0; k < 3; k++) { fe[0][k] = (float)e1[k]; fe[1][k] = (float)e2[k]; fe[2][k] = (float)e3[k]; }
                    double tmin[3] = {1e300, 1e300, 1e300}, tmax[3] = {-1e300, -1e300, -1e300};
                    for (int i = a; i < b; i++) {
                        float4 q = P4[i];
                        for (int k = 0; k < 3; k++) {
                            double t = (double)fe[k][0] * (q.x - x0.x) + (double)fe[k][1] * (q.y - x0.y) + (double)fe[k][2] * (q.z - x0.z);
                            tmin[k] = fmin(tmin[k], t); tmax[k] = fmax(tmax[k], t);
                        }
                    }
                    double cx = x0.x, cy = x0.y, cz = x0.z;
                    for (int k = 0; k < 3; k++) {
                        double mid = 0.5 * (tmin[k] + tmax[k]);
                        cx += mid * fe[k][0]; cy += mid * fe[k][1]; cz += mid * fe[k][2];
                    }
                    float4 cf = make_float4((float)cx, (float)cy, (float)cz, 1.f);
                    // half extents measured from the stored (rounded) centre and axes
                    double h[3] = {0, 0, 0};
                    for (int i = a; i < b; i++) {
                        float4 q = P4[i];
                        for (int k = 0; k < 3; k++) {
                            double t = (double)fe[k][0] * (q.x - cf.x) + (double)fe[k][1] * (q.y - cf.y) + (double)fe[k][2] * (q.z - cf.z);
                            h[k] = fmax(h[k], fabs(t));
                        }
                    }
                    ob[0] = cf;
                    for (int k = 0; k < 3; k++) ob[k + 1] = make_float4(fe[k][0], fe[k][1], fe[k][2], (float)(h[k] * (1.0 + 1e-6) + 1e-6));
                }
            }
        }
        for (int k = 0; k < 4; k++) obb[4 * l + k] = ob[k];
    }
    __syncthreads();
    for (int width = C.P >> 1; width >= 1; width >>= 1) {
        for (int j = tid; j < width; j += HULL_NT) {
            int node = width + j;
            float4 a = nlo[2 * node], b = nlo[2 * node + 1], c = nhi[2 * node], d = nhi[2 * node + 1];
            nlo[node] = make_float4(fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z), 0.f);
            nhi[node] = make_float4(fmaxf(c.x, d.x), fmaxf(c.y, d.y), fmaxf(c.z, d.z), 0.f);
        }
        __syncthreads();
    }
    // ---- 4. tables
    cta_fill_ones64(eset, C.eh, tid);                // sizes even (powers of two), 256-byte aligned
    cta_fill_ones64(fset, C.fh, tid);
    if (tid == 0) { sh.n_faces = 0; sh.n_corners = 0; sh.lexmin = ~0ull; }
    __syncthreads();
    HullCtx H; H.pts = P4; H.nlo = nlo; H.nhi = nhi; H.obb = obb; H.m = n; H.P = C.P; H.nleaf = C.m_leaves;

    // extreme point for seed sd: lexicographic minimum of (s0*q[ax0],
    // s1*q[ax1], s2*q[ax2], input index) -> sorted id
    __shared__ int s_p0;
    auto extreme = [&](int ax0, int s0, int ax1, int s1, int ax2, int s2) -> int {
        if (tid == 0) { sh.lexmin = ~0ull; s_p0 = -1; }
        __syncthreads();
        unsigned long long best = ~0ull;
        for (int i = tid; i < n; i += HULL_NT) {
            float4 q = P4[i];
            const int c0 = s0 * (int)comp(q, ax0), c1 = s1 * (int)comp(q, ax1), c2 = s2 * (int)comp(q, ax2);
            // duplicates resolve to the smaller input index
            unsigned long long k = ((unsigned long long)(c0 + 8192) << 50) | ((unsigned long long)(c1 + 8192) << 36) |
                                   ((unsigned long long)(c2 + 8192) << 22) | (unsigned long long)(unsigned)pidx(q);
            if (k < best) best = k;
        }
        atomicMin(&sh.lexmin, best);
        __syncthreads();
        const int want = (int)(sh.lexmin & ((1ull << 22) - 1));
        for (int i = tid; i < n; i += HULL_NT) if (pidx(P4[i]) == want) s_p0 = i;
        __syncthreads();
        return s_p0;
    };

    // ---- cooperative (large) face: collect S by scanning all points, walk
    // the polygon with CTA reductions, publish the face.  u<0: first face.
    __shared__ int s_face_ok;
    __shared__ int s_cur, s_first;
    auto coop_face = [&](int u, int v, double nx, double ny, double nz, int anchor) -> void {
        // anchor: a point on the plane
        if (tid == 0) { sh.n_S = 0; s_face_ok = 1; }
        __syncthreads();
        float4 a = P4[anchor];
        float fx = (float)nx, fy = (float)ny, fz = (float)nz;
        for (int base = 0; base < n; base += HULL_NT) {
            int i = base + tid;
            unsigned dummy = 0;
            bool on = i < n && plane_sign(nx, ny, nz, fx, fy, fz, a, P4[i], dummy) == 0;
            unsigned bal = __ballot_sync(FULL_MASK, on);
            int wbase = 0;
            if ((tid & 31) == 0 && bal) wbase = atomicAdd(&sh.n_S, __popc(bal));
            wbase = __shfl_sync(FULL_MASK, wbase, 0);
            if (on) Sbuf[wbase + __popc(bal & ((1u << (tid & 31)) - 1))] = i;
        }
        __syncthreads();
        const int ns = sh.n_S;
        Proj PR = make_proj(nx, ny, nz);
        // start corner
        if (u < 0) {
            // 2D lexmin (u, v, input index) among S
            __shared__ unsigned long long s_lm;
            if (tid == 0) s_lm = ~0ull;
            __syncthreads();
            unsigned long long best = ~0ull;
            for (int i = tid; i < ns; i += HULL_NT) {
                float4 q = P4[Sbuf[i]];
                unsigned long long k = ((unsigned long long)((int)comp(q, PR.ku) + 8192) << 44) |
                                       ((unsigned long long)((int)comp(q, PR.kv) + 8192) << 30) |
                                       (unsigned long long)(unsigned)i;
                // tie on position: smaller input index
                if (k < best) best = k;
            }
            atomicMin(&s_lm, best);
            __syncthreads();
            if (tid == 0) {
                int si = (int)(s_lm & ((1ull << 30) - 1));
                int f = Sbuf[si];
                // among duplicates at that position pick the smallest input index
                for (int i = 0; i < ns; i++) {
                    float4 q = P4[Sbuf[i]];
                    if (same_pos(q, P4[f]) && pidx(q) < pidx(P4[f])) f = Sbuf[i];
                }
                s_first = f; s_cur = f;
            }
        } else if (tid == 0) { s_first = v; s_cur = u; }
        __syncthreads();
        // corner list
        __shared__ int s_cstart, s_k;
        if (tid == 0) {
            s_cstart = atomicAdd(&sh.n_corners, 0);   // provisional: single writer below
            s_k = 0;
            if (u >= 0) { if (s_cstart < C.ccap) corners[s_cstart] = v; s_k = 1; }
        }
        __syncthreads();
        for (int guard = 0; guard <= ns + 1; guard++) {
            int cur = s_cur;
            if (tid == 0) {
                int slot = s_cstart + s_k;
                if (slot < C.ccap) corners[slot] = cur; else s_face_ok = 0;
                s_k++;
            }
            float4 pc = P4[cur];
            int r = -1; float4 pr = pc;
            for (int i = tid; i < ns; i += HULL_NT) {
                float4 pt = P4[Sbuf[i]];
                if (same_pos(pt, pc)) continue;
                if (r < 0 || next_better(PR, pc, pr, pt)) { r = Sbuf[i]; pr = pt; }
            }
            // warp reduce with the comparator
            for (int o = 16; o > 0; o >>= 1) {
                int r2 = __shfl_xor_sync(FULL_MASK, r, o);
                if (r2 >= 0) {
                    float4 p2 = P4[r2];
                    if (r < 0 || next_better(PR, pc, pr, p2)) { r = r2; pr = p2; }
                }
            }
            if ((tid & 31) == 0) sh.red_id[tid >> 5] = r;
            __syncthreads();
            if (tid == 0) {
                int rr = -1; float4 prr = pc;
                for (int w = 0; w < HULL_NT / 32; w++) {
                    int r2 = sh.red_id[w];
                    if (r2 < 0) continue;
                    float4 p2 = P4[r2];
                    if (rr < 0 || next_better(PR, pc, prr, p2)) { rr = r2; prr = p2; }
                }
                if (rr < 0) { s_face_ok = 0; s_cur = -1; }
                else if (same_pos(prr, P4[s_first])) s_cur = -1;
                else s_cur = rr;
            }
            __syncthreads();
            if (s_cur < 0) break;
        }
        if (tid == 0) {
            int k = s_k;
            if (s_face_ok && k >= 3 && s_cur < 0) {
                // canonical face key: (min input idx corner, successor)
                int mi = 0;
                for (int i = 1; i < k; i++)
                    if (pidx(P4[corners[s_cstart + i]]) < pidx(P4[corners[s_cstart + mi]])) mi = i;
                unsigned long long key = ekey(corners[s_cstart + mi], corners[s_cstart + (mi + 1) % k]);
                int ins = hset_insert(fset, C.fh, key);
                if (ins == 1) {
                    int f = sh.n_faces++;
                    if (f < C.fcap) { faces[f] = make_int2(s_cstart, k); sh.n_corners = s_cstart + k; }
                    else sh.err |= KERR_BT_POOL_EXHAUST;
                } else if (ins < 0) sh.err |= KERR_BT_POOL_EXHAUST;
            } else if (!s_face_ok || s_cur >= 0) {
                sh.err |= KERR_BT_EXTRACT_FAIL;
                if (S->fail[0] == 0) {
                    S->fail[0] = 2; S->fail[1] = u; S->fail[2] = v; S->fail[3] = s_cur; S->fail[4] = ns;
                    S->fail[5] = k; S->fail[6] = s_face_ok; S->fail[7] = anchor;
                }
            }
        }
        __syncthreads();
    };

    // ---- 5. seed faces.  Each seed is an extreme point p (a vertex of the
    // cloud's projection along d) and a direction d: wrapping a plane about
    // the line (p, d) gives a hull edge (p, c), whose outward face normal is
    // (c - p) x d; a collinear contact set is wrapped again about (p, c).
    // Seed 0 (lexicographic minimum, d = z) always runs; more seeds start the
    // wrapping from up to five more places, which shortens its longest
    // chain.  One warp finds each seed's plane (warp-cooperative wraps over
    // the output buffers, free until the output phase), then the CTA builds
    // the seed faces in order; a face already found is dropped by the face set.
    unsigned st_pts = 0, st_cop = 0, st_64 = 0;
    const int seeds[6][9] = {
        {0, 1, 1, 1, 2, 1, 0, 0, 1}, {0, -1, 1, -1, 2, 1, 0, 0, 1},
        {1, 1, 0, -1, 2, 1, 0, 0, 1}, {1, -1, 0, 1, 2, 1, 0, 0, 1},
        {2, 1, 1, 1, 0, 1, 1, 0, 0}, {2, -1, 1, -1, 0, 1, 1, 0, 0}};
    const int n_seeds = (n >= 64 && n >= seed_min_n) ? HULL_SEEDS : 1;
    __shared__ int s_sp[6], s_sok[6];
    __shared__ double s_sN[6][3];
    for (int sd = 0; sd < n_seeds; sd++) {
        const int* S6 = seeds[sd];
        const int pe = extreme(S6[0], S6[1], S6[2], S6[3], S6[4], S6[5]);
        if (tid == 0) s_sp[sd] = pe;
    }
    __syncthreads();
    {
        const int warp = tid >> 5, lane = tid & 31;
        if (warp < n_seeds) {
            const int sd = warp;
            const int p0 = s_sp[sd];
            const int dir[3] = {seeds[sd][6], seeds[sd][7], seeds[sd][8]};
            // lists: 3P ints per seed warp, seeds 0-3 in ocnt (2n), 4-5 in posn (n)
            int* base = sd < 4 ? ocnt + (size_t)sd * 3 * C.P : posn + (size_t)(sd - 4) * 3 * C.P;
            WarpLists L;
            L.q = base; L.leaf = base + 2 * C.P; L.qcap = 2 * C.P; L.lcap = C.P;
            int nl = 0;
            int ok = p0 >= 0;
            double nx = 0, ny = 0, nz = 0;
            int c = ok ? warp_wrap(H, p0, p0, L, lane, &nl, st_pts, st_64, dir) : -1;
            ok = c >= 0;
            if (ok) {
                const float4 a = P4[p0], q = P4[c];
                const double ex = q.x - a.x, ey = q.y - a.y, ez = q.z - a.z;
                nx = ey * dir[2] - ez * dir[1]; ny = ez * dir[0] - ex * dir[2]; nz = ex * dir[1] - ey * dir[0];
                // collinear contact set? then wrap again about (p0, c)
                const int ns = warp_coplanar(H, a, nx, ny, nz, sh.ws[sd], L, nl, lane, HULL_SMALL_S, st_cop, st_64);
                // (a large contact set may still be collinear: duplicates of
                // p0 or c, or points along the line)
                const int ix = (int)ex, iy = (int)ey, iz = (int)ez;
                int noncol = 0;
                if (ns > HULL_SMALL_S) noncol = warp_any_off_line(H, L, nl, a, nx, ny, nz, ix, iy, iz, lane, st_64);
                else {
                    if (lane == 0)
                        for (int i = 0; i < ns && !noncol; i++)
                            if (!on_line(ix, iy, iz, a, P4[sh.ws[sd].S[i]])) noncol = 1;
                    noncol = __shfl_sync(FULL_MASK, noncol, 0);
                }
                if (!noncol) {
                    const int c2 = warp_wrap(H, p0, c, L, lane, &nl, st_pts, st_64);
                    if (c2 < 0) ok = 0;
                    else {
                        const float4 q2 = P4[c2];
                        const double fx = q2.x - a.x, fy = q2.y - a.y, fz = q2.z - a.z;
                        nx = fy * ez - fz * ey; ny = fz * ex - fx * ez; nz = fx * ey - fy * ex;
                        if (nx == 0 && ny == 0 && nz == 0) ok = 0;
                    }
                }
            }
            if (lane == 0) { s_sok[sd] = ok; s_sN[sd][0] = nx; s_sN[sd][1] = ny; s_sN[sd][2] = nz; }
        }
    }
    __syncthreads();
    for (int sd = 0; sd < n_seeds; sd++) {
        if (!s_sok[sd]) {
            if (sd == 0) return;                     // degenerate: collinear input (no faces, no error)
            continue;
        }
        coop_face(-1, -1, s_sN[sd][0], s_sN[sd][1], s_sN[sd][2], s_sp[sd]);
        if (sh.err) break;
    }

    // ---- 6. frontier queue: every edge of the seed faces whose twin is unknown
    cta_fill_ones64(Q, qcap, tid);                   // qcap = 2 * fr_cap, even
    __syncthreads();
    if (tid == 0) {
        int qt = 0;
        const int nf0 = min(sh.n_faces, C.fcap);
        for (int f = 0; f < nf0; f++) {
            int2 F = faces[f];
            for (int i = 0; i < F.y; i++)
                if (hset_insert(eset, C.eh, ekey(corners[F.x + i], corners[F.x + (i + 1) % F.y])) < 0)
                    sh.err |= KERR_BT_POOL_EXHAUST;
        }
        for (int f = 0; f < nf0; f++) {
            int2 F = faces[f];
            for (int i = 0; i < F.y; i++) {
                int u = corners[F.x + i], v = corners[F.x + (i + 1) % F.y];
                if (!hset_has(eset, C.eh, ekey(v, u)) && qt < qcap) Q[qt++] = ekey(u, v);
            }
        }
        S->q_tail = qt; S->q_pending = qt;
        S->n_faces = sh.n_faces; S->n_corners = sh.n_corners; S->err = sh.err;
        S->active = (qt > 0 && sh.err == 0) ? 1 : 0;
        S->stats[4] = (unsigned long long)(clock64() - t_begin);
    }
    __syncthreads();
}

// Device-wide clock (ns) for the per-hull wrap timestamps.
static __device__ __forceinline__ unsigned long long hull_now()
{
    unsigned long long t;
#ifdef __CUDA_ARCH__
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
#else
    t = (unsigned long long)clock64();      // host builds of the device code (CPU emulation in the tests)
#endif
    return t;
}

#define HULL_SGCAP 4096   // per-warp coplanar set and polygon (ints each); larger faces use the hull's own buffers

// The hull's own buffers Sbuf/posn/ocnt are free while it is being wrapped;
// a warp that needs them for a large face or a long leaf list takes this
// lock (bounded wait; a timeout marks the hull failed).
static __device__ bool hull_lock(HullState* S, int lane)
{
    int ok = 0;
    if (lane == 0) {
        for (int spin = 0; spin < (1 << 22); spin++) {
            if (atomicCAS(&S->lock, 0, 1) == 0) { ok = 1; break; }
            __nanosleep(64);
        }
        if (!ok) atomicOr(&S->err, KERR_TIMEOUT);
        __threadfence();
    }
    return __shfl_sync(FULL_MASK, ok, 0) != 0;
}

static __device__ void hull_unlock(HullState* S, int lane)
{
    __syncwarp();
    if (lane == 0) { __threadfence(); atomicExch(&S->lock, 0); }
    __syncwarp();
}

// Wrap about frontier edge (u, v) of hull S and register the face found
// (whole warp): the first point hit, the face's coplanar points, its
// polygon; a new face is inserted in the face set, its edges in the edge
// set, and those whose twin is not known yet go to the frontier queue.
static __device__ void hull_wrap_edge(HullState* S, int u, int v, HullWarp& W, const WarpLists Ls,
                                      int* Sg, int* Pg, int lane, unsigned& st_pts, unsigned& st_cop,
                                      unsigned& st_64)
{
    const HullCtx H = hull_ctx(*S);
    const float4* P4 = H.pts;
    int nl = 0, ties = 1;
    WarpLists L = Ls;
    bool locked = false;
    int c = warp_wrap(H, u, v, L, lane, &nl, st_pts, st_64, nullptr, &ties);
    if (c == -2) {                                   // shared lists too small: the hull's own
        locked = hull_lock(S, lane);
        if (!locked) return;
        if (lane == 0) atomicAdd(&S->stats[7], 1ull << 32);
        L.q = S->ocnt; L.leaf = S->ocnt + 2 * S->P; L.qcap = 2 * S->P; L.lcap = S->P;
        c = warp_wrap(H, u, v, L, lane, &nl, st_pts, st_64, nullptr, &ties);
        if (c == -2) {                               // cannot happen: 2P + P hold the whole tree
            if (lane == 0) atomicOr(&S->err, KERR_BT_WARP_OOM);
            hull_unlock(S, lane);
            return;
        }
    }
    if (lane == 0) { atomicAdd(&S->stats[0], (unsigned long long)nl); atomicAdd(&S->stats[1], 1ull); }
    const float4 pu = P4[u], pv = P4[v];
    const int dx = (int)(pv.x - pu.x), dy = (int)(pv.y - pu.y), dz = (int)(pv.z - pu.z);
    int ns = 0;
    double nx = 0, ny = 0, nz = 0;
    if (c >= 0) {
        float4 pc = P4[c];
        double ex = pc.x - pu.x, ey = pc.y - pu.y, ez = pc.z - pu.z;
        nx = ey * dz - ez * dy; ny = ez * dx - ex * dz; nz = ex * dy - ey * dx;
        // no other point on the plane: the triangle (v, u, c) without a
        // coplanar pass
        ns = ties == 0 ? 3 : warp_coplanar(H, pu, nx, ny, nz, W, L, nl, lane, HULL_SMALL_S, st_cop, st_64);
    }
    int k = -1;
    const int* poly = Pg;
    if (c >= 0 && ns > HULL_SMALL_S) {
        int* bS = Sg; int* bP = Pg;
        if (ns + 2 > HULL_SGCAP) {                   // large face: the hull's own buffers
            if (!locked) { locked = hull_lock(S, lane); if (!locked) return; }
            if (lane == 0) atomicAdd(&S->stats[7], 1ull << 48);
            bS = S->Sbuf; bP = S->posn;
        }
        k = warp_big_polygon(H, u, v, nx, ny, nz, L.leaf, nl, bS, bP, lane, st_cop, st_64);
        poly = bP;
        if (lane == 0) atomicAdd(&S->stats[7], 1ull);
    } else if (c >= 0) {
        if (lane == 0) {
            if (ns == 3) { Pg[0] = v; Pg[1] = u; Pg[2] = c; k = 3; }
            else k = hull_small_polygon(H, W.S, ns, nx, ny, nz, v, u, Pg);
        }
        k = __shfl_sync(FULL_MASK, k, 0);
    }
    __syncwarp();
    // register the face: lane 0 claims it (face key = its smallest corner and
    // the next one), then the lanes insert its edges and queue the new ones
    int fs = -1;
    if (lane == 0) {
        if (c < 0 || k < 3) {
            atomicOr(&S->err, KERR_BT_EXTRACT_FAIL);
            if (atomicCAS(&S->fail[0], 0, 1) == 0) {
                S->fail[1] = u; S->fail[2] = v; S->fail[3] = c; S->fail[4] = ns; S->fail[5] = k;
                S->fail[6] = pidx(P4[u]); S->fail[7] = pidx(P4[v]);
            }
        } else {
            int mi = 0;
            for (int i = 1; i < k; i++) if (pidx(P4[poly[i]]) < pidx(P4[poly[mi]])) mi = i;
            int ins = hset_insert(S->fset, S->fh, ekey(poly[mi], poly[(mi + 1) % k]));
            if (ins == 1) {
                int cs = atomicAdd(&S->n_corners, k);
                int f = atomicAdd(&S->n_faces, 1);
                if (cs + k <= S->ccap && f < S->fcap) { S->faces[f] = make_int2(cs, k); fs = cs; }
                else atomicOr(&S->err, KERR_BT_POOL_EXHAUST);
            } else if (ins < 0) atomicOr(&S->err, KERR_BT_POOL_EXHAUST);
        }
    }
    fs = __shfl_sync(FULL_MASK, fs, 0);
    if (fs >= 0) {
        unsigned long long* eset = S->eset;
        const int eh = S->eh, qcap = S->qcap;
        for (int i = lane; i < k; i += 32) {
            S->corners[fs + i] = poly[i];
            if (hset_insert(eset, eh, ekey(poly[i], poly[(i + 1) % k])) < 0) atomicOr(&S->err, KERR_BT_POOL_EXHAUST);
        }
        for (int i = lane; i < k; i += 32) {
            int x = poly[i], y = poly[(i + 1) % k];
            if (!hset_has(eset, eh, ekey(y, x))) {
                atomicAdd(&S->q_pending, 1);
                int slot = atomicAdd(&S->q_tail, 1);
                if (slot < qcap) atomicExch(&S->Q[slot], ekey(x, y));
                else { atomicOr(&S->err, KERR_BT_POOL_EXHAUST); atomicSub(&S->q_pending, 1); }
            }
        }
    }
    if (locked) hull_unlock(S, lane);
}

// Persistent wrapping (all HULL_NT threads of every CTA of the grid).  Each
// CTA has a home hull (h0): the CTAs are shared out over the active hulls in
// proportion to their point counts, so a hull's BVH and points stay in the
// L1 of the few SMs that wrap it.  A warp takes frontier edges from its
// current hull, waits (backing off) while that hull still has edges in
// flight, and moves to another hull with queued edges once it is done.
// ctl[0] counts the hulls still wrapping; a hull is done when its last
// queued edge is done.  Every wait is bounded: ctl[1] collects KERR_TIMEOUT.
static __device__ void hull_wrap_grid(HullState* states, int n_jobs, int h0, int* ctl, int* wbuf,
                                      HullWrapShared& sh, int* wsm)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int gw = blockIdx.x * (HULL_NT / 32) + warp;
    HullWarp& W = sh.ws[warp];
    int* Sg = wbuf + (size_t)gw * 2 * HULL_SGCAP;
    int* Pg = Sg + HULL_SGCAP;
    WarpLists Ls;
    Ls.q = wsm + (size_t)warp * HULL_WSM; Ls.leaf = Ls.q + HULL_WQ; Ls.qcap = HULL_WQ; Ls.lcap = HULL_WL;
    unsigned st_pts = 0, st_cop = 0, st_64 = 0;
    int h = h0;
    int idle = 0;
    unsigned nap = 64;
    for (;;) {
        int idx = -1;
        if (lane == 0) {
            HullState* S = &states[h];
            if (*(volatile int*)&S->active) {
                int hd = *(volatile int*)&S->q_head;
                const int tl = *(volatile int*)&S->q_tail;
                while (hd < tl) {
                    int prev = atomicCAS(&S->q_head, hd, hd + 1);
                    if (prev == hd) { idx = hd; break; }
                    hd = prev;
                }
            }
        }
        // lane 0 reads the shared words and broadcasts: every lane takes the
        // same branch
        int done = 0, stay = 0;
        if (lane == 0 && idx < 0) {
            done = *(volatile int*)&ctl[0] <= 0;
            stay = *(volatile int*)&states[h].active;
        }
        idx = __shfl_sync(FULL_MASK, idx, 0);
        done = __shfl_sync(FULL_MASK, done, 0);
        stay = __shfl_sync(FULL_MASK, stay, 0);
        if (idx < 0) {
            if (done) break;                                         // every hull is done
            if (stay) {                                              // edges in flight: stay
                if (++idle > (1 << 20)) { if (lane == 0) atomicOr(&ctl[1], KERR_TIMEOUT); break; }
                __nanosleep(nap);
                nap = min(2 * nap, 2048u);
                continue;
            }
            int found = -1;
            for (int base = 1; base <= n_jobs && found < 0; base += 32) {   // warp-uniform trip count
                const int off = base + lane;
                const int cand = off <= n_jobs ? (h + off) % n_jobs : -1;
                bool av = false;
                if (cand >= 0) {
                    const HullState* C = &states[cand];
                    av = *(volatile const int*)&C->active &&
                         *(volatile const int*)&C->q_head < *(volatile const int*)&C->q_tail;
                }
                const unsigned b = __ballot_sync(FULL_MASK, av);
                if (b) found = __shfl_sync(FULL_MASK, cand, __ffs(b) - 1);      // same on every lane
            }
            if (found >= 0) { h = found; idle = 0; nap = 64; continue; }
            if (++idle > (1 << 20)) { if (lane == 0) atomicOr(&ctl[1], KERR_TIMEOUT); break; }
            __nanosleep(nap);                           // back off: idle warps must not flood L2
            nap = min(2 * nap, 8192u);
            continue;
        }
        idle = 0; nap = 64;
        HullState* S = &states[h];
        if (lane == 0 && idx == 0) S->stats[5] = hull_now();          // first edge taken
        unsigned long long key = ~0ull;
        int skip = 0;
        if (lane == 0) {
            for (int spin = 0; spin < (1 << 22); spin++) {
                key = atomicAdd(&S->Q[idx], 0ull);
                if (key != ~0ull) break;
                __nanosleep(32);
            }
            if (key == ~0ull) atomicOr(&S->err, KERR_TIMEOUT);
            else skip = (*(volatile int*)&S->err != 0) ||
                        hset_has(S->eset, S->eh, ekey((int)(key & 0xffffffffu), (int)(key >> 32)));
        }
        key = __shfl_sync(FULL_MASK, key, 0);
        skip = __shfl_sync(FULL_MASK, skip, 0);
        if (key != ~0ull && !skip) {
            const unsigned p0 = st_pts;
            hull_wrap_edge(S, (int)(key >> 32), (int)(key & 0xffffffffu), W, Ls, Sg, Pg, lane, st_pts, st_cop, st_64);
            unsigned d = st_pts - p0;
            #pragma unroll
            for (int o = 16; o > 0; o >>= 1) d += __shfl_xor_sync(FULL_MASK, d, o);
            if (lane == 0) atomicAdd(&S->stats[3], (unsigned long long)d);
        }
        __syncwarp();
        if (lane == 0) {
            if (atomicSub(&S->q_pending, 1) == 1) {                   // this hull is complete
                S->stats[6] = hull_now();
                atomicExch(&S->active, 0);
                __threadfence();
                atomicSub(&ctl[0], 1);
            }
        }
    }
}

// Output of one wrapped hull (all HULL_NT threads): corners in ascending
// input index, each face fanned from its smallest corner, triangles grouped
// by that corner and sorted; FP64 volume.  A hull without faces (fewer than
// 4 points, or collinear) gives empty output; a failed hull only its error.
static __device__ void hull_output_cta(const float* __restrict__ pts, const HullState* S, float* out_v, int* out_t,
                                       int max_hv, int max_ht, int* o_nv, int* o_nt, float* o_vol, int* o_err,
                                       HullOutShared& sh)
{
    const int tid = threadIdx.x;
    const int n = S->n;
    const int err0 = S->err;
    if (n < 4 || S->n_faces == 0 || err0) {          // nothing built, or failed: no buffers touched
        if (tid == 0) { *o_nv = 0; *o_nt = 0; *o_vol = 0.f; *o_err = err0; }
        return;
    }
    if (tid == 0) *o_err = 0;
    const float4* P4 = S->P4;
    const int2* faces = S->faces;
    const int* corners = S->corners;
    int* posn = S->posn;
    int* ocnt = S->ocnt;
    int* ofill = ocnt + n;
    // ---- 7. canonical output
    const int nfaces = min(S->n_faces, S->fcap);
    // mark corners by input index
    for (int i = tid; i < n; i += HULL_NT) { posn[i] = 0; ocnt[i] = 0; ofill[i] = 0; }
    __syncthreads();
    for (int f = tid; f < nfaces; f += HULL_NT) {
        int2 F = faces[f];
        for (int i = 0; i < F.y; i++) posn[pidx(P4[corners[F.x + i]])] = 1;
    }
    __syncthreads();
    // input index -> output position (rank among the corners), -1 if none
    const int nv_out = cta_rank_flags_inplace(posn, n, sh.scan);
    // triangles per owner (face's smallest corner)
    for (int f = tid; f < nfaces; f += HULL_NT) {
        int2 F = faces[f];
        int mi = 0;
        for (int i = 1; i < F.y; i++) if (pidx(P4[corners[F.x + i]]) < pidx(P4[corners[F.x + mi]])) mi = i;
        atomicAdd(&ocnt[posn[pidx(P4[corners[F.x + mi]])]], F.y - 2);
    }
    __syncthreads();
    const int nt_out = cta_scan_inplace(ocnt, nv_out, sh.scan);   // owner -> first triangle slot
    bool fits = nv_out <= max_hv && nt_out <= max_ht && !err0;
    if (fits) {
        for (int f = tid; f < nfaces; f += HULL_NT) {
            int2 F = faces[f];
            int k = F.y, mi = 0;
            for (int i = 1; i < k; i++) if (pidx(P4[corners[F.x + i]]) < pidx(P4[corners[F.x + mi]])) mi = i;
            int owner = posn[pidx(P4[corners[F.x + mi]])];
            int slot = ocnt[owner] + atomicAdd(&ofill[owner], k - 2);
            for (int i = 1; i + 1 < k; i++, slot++) {
                out_t[3 * slot]     = owner;
                out_t[3 * slot + 1] = posn[pidx(P4[corners[F.x + (mi + i) % k]])];
                out_t[3 * slot + 2] = posn[pidx(P4[corners[F.x + (mi + i + 1) % k]])];
            }
        }
        __syncthreads();
        // sort each owner's triangles by (t1, t2)
        for (int o = tid; o < nv_out; o += HULL_NT) {
            int a = ocnt[o], b = (o + 1 < nv_out) ? ocnt[o + 1] : nt_out;
            for (int i = a + 1; i < b; i++) {
                int k1 = out_t[3 * i + 1], k2 = out_t[3 * i + 2];
                int j = i - 1;
                while (j >= a && (out_t[3 * j + 1] > k1 || (out_t[3 * j + 1] == k1 && out_t[3 * j + 2] > k2))) {
                    out_t[3 * (j + 1) + 1] = out_t[3 * j + 1];
                    out_t[3 * (j + 1) + 2] = out_t[3 * j + 2];
                    j--;
                }
                out_t[3 * (j + 1) + 1] = k1; out_t[3 * (j + 1) + 2] = k2;
            }
        }
        for (int i = tid; i < n; i += HULL_NT) {
            int pos = posn[i];
            if (pos >= 0) {
                out_v[3 * pos] = pts[3 * i]; out_v[3 * pos + 1] = pts[3 * i + 1]; out_v[3 * pos + 2] = pts[3 * i + 2];
            }
        }
        __syncthreads();
        double vol = block_mesh_signed_volume(out_v, nv_out, out_t, nt_out, sh.dsh);
        if (tid == 0) { *o_nv = nv_out; *o_nt = nt_out; *o_vol = (float)fabs(vol); }
    } else {
        if (tid == 0) { *o_nv = 0; *o_nt = 0; *o_vol = 0.f; *o_err = err0 ? err0 : KERR_BT_HEAP_OUTPUT; }
    }
    __syncthreads();
}
