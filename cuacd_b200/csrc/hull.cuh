// hull.cuh — exact convex hull of a point cloud, one CTA per cloud (sm_100a).
//
// Replaces the reference's warp D&C hull (cuda/hull_dandc.cuh:1678-1861) and
// its k-DOP prefilter (cuda/kdop_hull.cuh:49-398) with one exact algorithm:
//
//   1. quantise onto the reference grid (hull_dandc.cuh:1351-1411): per-axis
//      step span/10216, axes permuted to (med,max,min), sign flip when
//      (medAx+1)%3 != maxAx, truncation toward zero; IEEE-rounded divisions.
//      Grid coordinates are |q| <= 5109, stored as exact floats.
//   2. bucket the points by a 12-bit Morton code and build an implicit binary
//      BVH over leaves of HULL_LEAF points (bounding boxes in grid units).
//   3. gift wrapping over polygon faces, one thread per frontier edge: the
//      next face around edge (u,v) is found by branch-and-bound over the BVH
//      (a box is skipped when no corner lies strictly beyond the current
//      plane).  Orientation tests run in FP32 with a static error bound and
//      fall back to exact FP64 (all grid predicates are < 2^46 in magnitude,
//      so FP64 is exact) near zero.  Coplanar points are merged into one
//      polygon face; faces with more than HULL_SMALL_S coplanar points are
//      finished cooperatively by the whole CTA.
//   4. canonical output: corners in ascending input index; each face fanned
//      from its smallest corner; triangles grouped by first vertex and sorted.
//
// Duplicate grid points resolve to the smallest input index, as the
// reference's (y,x,z,index) sort keeps the first (warp_sort.cuh:237-244).
#pragma once
#include "common.cuh"

#define HULL_NT       256
#define HULL_LEAF     16
#define HULL_SMALL_S  24
#define HULL_MORTON_BITS 4            // bits per axis for the bucket sort
#define HULL_CELLS    (1 << (3 * HULL_MORTON_BITS))

struct HullOut {
    float* verts;     // hull corner coordinates (input floats), cap max_hv
    int*   tris;      // triangles, cap max_ht
    int*   vidx;      // optional: input index of each corner (nullable)
    int    max_hv, max_ht;
};

// Per-cloud scratch layout (bytes computed on the host by hull_scratch_bytes).
struct HullCaps {
    int n, m_leaves, P;      // points, leaves, leaf slots (pow2)
    int hcap, ccap, fcap, fr_cap, eh, fh, bq_cap;
};

__host__ __device__ inline int hull_pow2(int x) { int p = 1; while (p < x) p <<= 1; return p; }

__host__ __device__ inline HullCaps hull_caps(int n)
{
    HullCaps c;
    c.n = n;
    c.m_leaves = (n + HULL_LEAF - 1) / HULL_LEAF;
    if (c.m_leaves < 1) c.m_leaves = 1;
    c.P = hull_pow2(c.m_leaves);
    int h = n < 4 ? 4 : n;
    if (h > 65536) h = 65536;
    c.hcap = h;
    c.ccap = 6 * h + 64;
    c.fcap = 2 * h + 8;
    c.fr_cap = 6 * h + 64;
    c.eh = hull_pow2(2 * c.ccap);
    c.fh = hull_pow2(2 * c.fcap);
    c.bq_cap = 1024;
    return c;
}

__host__ __device__ inline size_t hull_align(size_t x) { return (x + 255) & ~(size_t)255; }

__host__ __device__ inline size_t hull_scratch_bytes(int n)
{
    HullCaps c = hull_caps(n);
    size_t b = 0;
    b += hull_align(sizeof(float4) * (size_t)(n > 0 ? n : 1));        // pts
    b += hull_align(sizeof(float4) * 2 * (size_t)(2 * c.P));          // node lo/hi
    b += hull_align(sizeof(unsigned long long) * (size_t)c.eh);       // edge set
    b += hull_align(sizeof(unsigned long long) * (size_t)c.fh);       // face keys
    b += hull_align(sizeof(int2) * (size_t)c.fcap);                   // faces
    b += hull_align(sizeof(int) * (size_t)c.ccap);                    // corners
    b += hull_align(sizeof(int2) * 2 * (size_t)c.fr_cap);             // frontier x2
    b += hull_align(sizeof(int4) * (size_t)c.bq_cap);                 // big-face queue
    b += hull_align(sizeof(int) * (size_t)(n > 0 ? n : 1));           // S / per-point flags
    b += hull_align(sizeof(int) * (size_t)(n > 0 ? n : 1));           // positions
    b += hull_align(sizeof(int) * (size_t)(n > 0 ? n : 1) * 2);       // owner count/fill
    return b;
}

// ---------------------------------------------------------------------------
// exact grid geometry
// ---------------------------------------------------------------------------
struct HullCtx {
    const float4* __restrict__ pts;     // (qx,qy,qz, input index as int bits)
    const float4* __restrict__ nlo;     // node boxes, heap order [1, 2P)
    const float4* __restrict__ nhi;
    int m, P, nleaf;
};

static __device__ __forceinline__ int pidx(float4 p) { return __float_as_int(p.w); }

// Sign of N.(q - a) for integer-valued N (|N| < 2^30) and grid points,
// FP32 with error bound, exact FP64 fallback.
static __device__ __forceinline__ int plane_sign(double nx, double ny, double nz,
                                          float fx, float fy, float fz,
                                          float4 a, float4 q)
{
    float ex = q.x - a.x, ey = q.y - a.y, ez = q.z - a.z;     // exact
    float s = fmaf(fz, ez, fmaf(fy, ey, fx * ex));
    float bound = fmaf(fabsf(fz), fabsf(ez), fmaf(fabsf(fy), fabsf(ey), fabsf(fx) * fabsf(ex))) * 4.8e-7f;
    if (s > bound) return 1;
    if (s < -bound) return -1;
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
static __device__ int hull_wrap(const HullCtx& H, int a_id, int dx, int dy, int dz, int start_leaf)
{
    float4 a = H.pts[a_id];
    int c = -1;
    double mx = 0, my = 0, mz = 0;
    float fx = 0, fy = 0, fz = 0;
    auto consider = [&](int qi) {
        float4 q = H.pts[qi];
        if (on_line(dx, dy, dz, a, q)) return;
        bool take = (c < 0);
        if (!take) take = plane_sign(mx, my, mz, fx, fy, fz, a, q) < 0;
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
static __device__ int hull_coplanar(const HullCtx& H, int a_id, double nx, double ny, double nz, int* out, int cap)
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
                if (plane_sign(nx, ny, nz, fx, fy, fz, a, H.pts[i]) == 0) {
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
        unsigned long long x = tab[s];
        if (x == k) return true;
        if (x == ~0ull) return false;
        s = (s + 1) & (unsigned)(cap - 1);
    }
    return false;
}

// ---------------------------------------------------------------------------
// the CTA hull
// ---------------------------------------------------------------------------
struct HullShared {
    float mn[3], mx[3];
    float cen[3], inv[3];
    int ax[3];
    unsigned long long lexmin;
    int n_faces, n_corners, n_front, n_next, n_big, err;
    int n_S;
    int red_id[HULL_NT / 32];
    int scan[33];
    double dsh[33];
    int small_S[HULL_NT][HULL_SMALL_S];
    int cells[HULL_CELLS];
};

// Build one hull.  All HULL_NT threads call.  `pts` are the input floats
// (AoS xyz) of this cloud; `scratch` holds hull_scratch_bytes(n).
// Writes the hull into `out` and returns (via *o_nv, *o_nt, *o_vol from
// thread 0) the counts and FP64 volume; error bits go to *err_word.
static __device__ void hull_cta(const float* __restrict__ pts, int n, char* scratch,
                         HullOut out, int* o_nv, int* o_nt, float* o_vol, int* err_word,
                         HullShared& sh)
{
    const int tid = threadIdx.x;
    if (tid == 0) { sh.err = 0; }
    if (n < 4) {
        if (tid == 0) { *o_nv = 0; *o_nt = 0; if (o_vol) *o_vol = 0.f; }
        return;
    }
    HullCaps C = hull_caps(n);
    char* p = scratch;
    float4* P4 = (float4*)p;            p += hull_align(sizeof(float4) * (size_t)n);
    float4* nlo = (float4*)p;           p += hull_align(sizeof(float4) * 2 * (size_t)(2 * C.P));
    float4* nhi = nlo + 2 * C.P;
    unsigned long long* eset = (unsigned long long*)p; p += hull_align(sizeof(unsigned long long) * (size_t)C.eh);
    unsigned long long* fset = (unsigned long long*)p; p += hull_align(sizeof(unsigned long long) * (size_t)C.fh);
    int2* faces = (int2*)p;             p += hull_align(sizeof(int2) * (size_t)C.fcap);
    int* corners = (int*)p;             p += hull_align(sizeof(int) * (size_t)C.ccap);
    int2* front0 = (int2*)p;
    int2* front1 = front0 + C.fr_cap;   p += hull_align(sizeof(int2) * 2 * (size_t)C.fr_cap);
    int4* bigq = (int4*)p;              p += hull_align(sizeof(int4) * (size_t)C.bq_cap);
    int* Sbuf = (int*)p;                p += hull_align(sizeof(int) * (size_t)n);
    int* posn = (int*)p;                p += hull_align(sizeof(int) * (size_t)n);
    int* ocnt = (int*)p;                                 // [n] owner tri counts, [n] fill
    int* ofill = ocnt + n;

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
    for (int i = tid; i < C.eh; i += HULL_NT) eset[i] = ~0ull;
    for (int i = tid; i < C.fh; i += HULL_NT) fset[i] = ~0ull;
    if (tid == 0) { sh.n_faces = 0; sh.n_corners = 0; sh.n_front = 0; sh.n_next = 0; sh.n_big = 0; sh.lexmin = ~0ull; }
    __syncthreads();
    HullCtx H; H.pts = P4; H.nlo = nlo; H.nhi = nhi; H.m = n; H.P = C.P; H.nleaf = C.m_leaves;

    // lexmin (x,y,z,input index) -> first face seed
    {
        unsigned long long best = ~0ull;
        for (int i = tid; i < n; i += HULL_NT) {
            float4 q = P4[i];
            // key (x, y, z, input index): duplicates resolve to the smaller index
            unsigned long long k = ((unsigned long long)((int)q.x + 8192) << 50) |
                                   ((unsigned long long)((int)q.y + 8192) << 36) |
                                   ((unsigned long long)((int)q.z + 8192) << 22) |
                                   (unsigned long long)(unsigned)pidx(q);
            if (k < best) best = k;
        }
        atomicMin(&sh.lexmin, best);
        __syncthreads();
    }
    // convert lexmin key back to a sorted id (find the point with that input index)
    __shared__ int s_p0;
    if (tid == 0) s_p0 = -1;
    __syncthreads();
    {
        int want = (int)(sh.lexmin & ((1ull << 22) - 1));
        for (int i = tid; i < n; i += HULL_NT) if (pidx(P4[i]) == want) s_p0 = i;
        __syncthreads();
    }
    const int p0 = s_p0;

    // ---- cooperative (large) face: collect S by scanning all points, walk
    // the polygon with CTA reductions, publish the face.  u<0: first face.
    __shared__ int s_face_ok;
    __shared__ int s_cur, s_prev, s_first;
    __shared__ double s_N[3];
    auto coop_face = [&](int u, int v, double nx, double ny, double nz, int anchor) -> void {
        // anchor: a point on the plane
        if (tid == 0) { sh.n_S = 0; s_face_ok = 1; }
        __syncthreads();
        float4 a = P4[anchor];
        float fx = (float)nx, fy = (float)ny, fz = (float)nz;
        for (int base = 0; base < n; base += HULL_NT) {
            int i = base + tid;
            bool on = i < n && plane_sign(nx, ny, nz, fx, fy, fz, a, P4[i]) == 0;
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
                s_first = f; s_cur = f; s_prev = -1;
            }
        } else if (tid == 0) { s_first = v; s_prev = v; s_cur = u; }
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
            } else if (!s_face_ok || s_cur >= 0) sh.err |= KERR_BT_EXTRACT_FAIL;
        }
        __syncthreads();
    };

    // ---- 5. first face (cooperative, thread 0 finds the plane)
    if (tid == 0) {
        int c = hull_wrap(H, p0, 0, 0, 1, p0 / HULL_LEAF);
        double nx = 0, ny = 0, nz = 0;
        int ok = c >= 0;
        if (ok) {
            float4 a = P4[p0], q = P4[c];
            double ex = q.x - a.x, ey = q.y - a.y, ez = q.z - a.z;
            nx = ey; ny = -ex; nz = 0;                      // (c - p0) x (0,0,1)
            // collinear contact set? then wrap again about (p0, c)
            int tmp[HULL_SMALL_S];
            int cnt = hull_coplanar(H, p0, nx, ny, nz, tmp, HULL_SMALL_S);
            bool noncol = cnt > HULL_SMALL_S;
            int ix = (int)ex, iy = (int)ey, iz = (int)ez;
            for (int i = 0; i < cnt && i < HULL_SMALL_S && !noncol; i++)
                if (!on_line(ix, iy, iz, a, P4[tmp[i]])) noncol = true;
            if (!noncol) {
                int c2 = hull_wrap(H, p0, ix, iy, iz, p0 / HULL_LEAF);
                if (c2 < 0) ok = 0;
                else {
                    float4 q2 = P4[c2];
                    double fx = q2.x - a.x, fy = q2.y - a.y, fz = q2.z - a.z;
                    nx = fy * ez - fz * ey; ny = fz * ex - fx * ez; nz = fx * ey - fy * ex;
                    if (nx == 0 && ny == 0 && nz == 0) ok = 0;
                }
            }
        }
        s_N[0] = nx; s_N[1] = ny; s_N[2] = nz;
        s_face_ok = ok;
    }
    __syncthreads();
    if (!s_face_ok) {
        if (tid == 0) { *o_nv = 0; *o_nt = 0; if (o_vol) *o_vol = 0.f; }
        return;                                      // degenerate: collinear input
    }
    coop_face(-1, -1, s_N[0], s_N[1], s_N[2], p0);

    // ---- 6. rounds of parallel wrapping
    int2* cur_front = front0;
    int2* nxt_front = front1;
    __shared__ int s_round_f0;
    if (tid == 0) s_round_f0 = 0;
    __syncthreads();
    for (int round = 0; round < 4 * C.fcap + 8; round++) {
        // register edges of faces created since s_round_f0, build the frontier
        int f0 = s_round_f0, f1 = sh.n_faces;
        if (f1 > C.fcap) f1 = C.fcap;
        for (int f = f0 + tid; f < f1; f += HULL_NT) {
            int2 F = faces[f];
            for (int i = 0; i < F.y; i++) {
                int u = corners[F.x + i], v = corners[F.x + (i + 1) % F.y];
                if (hset_insert(eset, C.eh, ekey(u, v)) < 0) atomicOr(&sh.err, KERR_BT_POOL_EXHAUST);
            }
        }
        __syncthreads();
        if (tid == 0) sh.n_front = 0;
        __syncthreads();
        for (int f = f0 + tid; f < f1; f += HULL_NT) {
            int2 F = faces[f];
            for (int i = 0; i < F.y; i++) {
                int u = corners[F.x + i], v = corners[F.x + (i + 1) % F.y];
                if (!hset_has(eset, C.eh, ekey(v, u))) {
                    int s = atomicAdd(&sh.n_front, 1);
                    if (s < C.fr_cap) cur_front[s] = make_int2(u, v);
                    else atomicOr(&sh.err, KERR_BT_POOL_EXHAUST);
                }
            }
        }
        __syncthreads();
        if (tid == 0) { s_round_f0 = f1; sh.n_big = 0; }
        __syncthreads();
        int nf = min(sh.n_front, C.fr_cap);
        if (nf == 0 || sh.err) break;
        // wrap each frontier edge
        for (int e = tid; e < nf; e += HULL_NT) {
            int2 E = cur_front[e];
            int u = E.x, v = E.y;
            if (hset_has(eset, C.eh, ekey(v, u))) continue;
            float4 pu = P4[u], pv = P4[v];
            int dx = (int)(pv.x - pu.x), dy = (int)(pv.y - pu.y), dz = (int)(pv.z - pu.z);
            int c = hull_wrap(H, u, dx, dy, dz, u / HULL_LEAF);
            if (c < 0) { atomicOr(&sh.err, KERR_BT_EXTRACT_FAIL); continue; }
            float4 pc = P4[c];
            double ex = pc.x - pu.x, ey = pc.y - pu.y, ez = pc.z - pu.z;
            // outward normal (c - u) x d
            double nx = ey * dz - ez * dy, ny = ez * dx - ex * dz, nz = ex * dy - ey * dx;
            int* S = sh.small_S[tid];
            int ns = hull_coplanar(H, u, nx, ny, nz, S, HULL_SMALL_S);
            if (ns > HULL_SMALL_S) {
                int b = atomicAdd(&sh.n_big, 1);
                if (b < C.bq_cap) bigq[b] = make_int4(u, v, c, 0);
                else atomicOr(&sh.err, KERR_BT_POOL_EXHAUST);
                continue;
            }
            int poly[HULL_SMALL_S + 2];
            int k = (ns == 3) ? 3 : -1;
            if (ns == 3) { poly[0] = v; poly[1] = u; poly[2] = c; }
            else k = hull_small_polygon(H, S, ns, nx, ny, nz, v, u, poly);
            if (k < 3) { atomicOr(&sh.err, KERR_BT_EXTRACT_FAIL); continue; }
            int mi = 0;
            for (int i = 1; i < k; i++) if (pidx(P4[poly[i]]) < pidx(P4[poly[mi]])) mi = i;
            int ins = hset_insert(fset, C.fh, ekey(poly[mi], poly[(mi + 1) % k]));
            if (ins == 1) {
                int cs = atomicAdd(&sh.n_corners, k);
                int f = atomicAdd(&sh.n_faces, 1);
                if (cs + k <= C.ccap && f < C.fcap) {
                    for (int i = 0; i < k; i++) corners[cs + i] = poly[i];
                    faces[f] = make_int2(cs, k);
                } else atomicOr(&sh.err, KERR_BT_POOL_EXHAUST);
            } else if (ins < 0) atomicOr(&sh.err, KERR_BT_POOL_EXHAUST);
        }
        __syncthreads();
        // large faces, one at a time, whole CTA
        int nb = min(sh.n_big, C.bq_cap);
        for (int b = 0; b < nb; b++) {
            int4 B = bigq[b];
            int u = B.x, v = B.y, c = B.z;
            if (hset_has(eset, C.eh, ekey(v, u))) continue;
            float4 pu = P4[u], pv = P4[v], pc = P4[c];
            double dx = pv.x - pu.x, dy = pv.y - pu.y, dz = pv.z - pu.z;
            double ex = pc.x - pu.x, ey = pc.y - pu.y, ez = pc.z - pu.z;
            double nx = ey * dz - ez * dy, ny = ez * dx - ex * dz, nz = ex * dy - ey * dx;
            // skip if a face owning edge (v,u) was already added this round
            __shared__ int s_dup;
            if (tid == 0) s_dup = 0;
            __syncthreads();
            int fstart = s_round_f0, fend = min(sh.n_faces, C.fcap);
            for (int f = fstart + tid; f < fend; f += HULL_NT) {
                int2 F = faces[f];
                for (int i = 0; i < F.y; i++)
                    if (corners[F.x + i] == v && corners[F.x + (i + 1) % F.y] == u) s_dup = 1;
            }
            __syncthreads();
            if (s_dup) continue;
            coop_face(u, v, nx, ny, nz, u);
        }
        __syncthreads();
        int2* t = cur_front; cur_front = nxt_front; nxt_front = t;
    }
    __syncthreads();

    // ---- 7. canonical output
    const int nfaces = min(sh.n_faces, C.fcap);
    // mark corners by input index
    for (int i = tid; i < n; i += HULL_NT) { posn[i] = 0; ocnt[i] = 0; ofill[i] = 0; }
    __syncthreads();
    for (int f = tid; f < nfaces; f += HULL_NT) {
        int2 F = faces[f];
        for (int i = 0; i < F.y; i++) posn[pidx(P4[corners[F.x + i]])] = 1;
    }
    __syncthreads();
    // exclusive scan over input indices -> output position
    __shared__ int s_carry;
    if (tid == 0) s_carry = 0;
    __syncthreads();
    for (int base = 0; base < n; base += HULL_NT) {
        int i = base + tid;
        int v = (i < n) ? posn[i] : 0;
        int tot;
        int ex = block_exclusive_scan(v, sh.scan, &tot);
        if (i < n) posn[i] = v ? (s_carry + ex) : -1;
        __syncthreads();
        if (tid == 0) s_carry += tot;
        __syncthreads();
    }
    const int nv_out = s_carry;
    // triangles per owner (face's smallest corner)
    for (int f = tid; f < nfaces; f += HULL_NT) {
        int2 F = faces[f];
        int mi = 0;
        for (int i = 1; i < F.y; i++) if (pidx(P4[corners[F.x + i]]) < pidx(P4[corners[F.x + mi]])) mi = i;
        atomicAdd(&ocnt[posn[pidx(P4[corners[F.x + mi]])]], F.y - 2);
    }
    __syncthreads();
    if (tid == 0) s_carry = 0;
    __syncthreads();
    for (int base = 0; base < nv_out; base += HULL_NT) {
        int i = base + tid;
        int v = (i < nv_out) ? ocnt[i] : 0;
        int tot;
        int ex = block_exclusive_scan(v, sh.scan, &tot);
        if (i < nv_out) ocnt[i] = s_carry + ex;
        __syncthreads();
        if (tid == 0) s_carry += tot;
        __syncthreads();
    }
    const int nt_out = s_carry;
    bool fits = nv_out <= out.max_hv && nt_out <= out.max_ht && !sh.err;
    if (fits) {
        for (int f = tid; f < nfaces; f += HULL_NT) {
            int2 F = faces[f];
            int k = F.y, mi = 0;
            for (int i = 1; i < k; i++) if (pidx(P4[corners[F.x + i]]) < pidx(P4[corners[F.x + mi]])) mi = i;
            int owner = posn[pidx(P4[corners[F.x + mi]])];
            int slot = ocnt[owner] + atomicAdd(&ofill[owner], k - 2);
            for (int i = 1; i + 1 < k; i++, slot++) {
                out.tris[3 * slot]     = owner;
                out.tris[3 * slot + 1] = posn[pidx(P4[corners[F.x + (mi + i) % k]])];
                out.tris[3 * slot + 2] = posn[pidx(P4[corners[F.x + (mi + i + 1) % k]])];
            }
        }
        __syncthreads();
        // sort each owner's triangles by (t1, t2)
        for (int o = tid; o < nv_out; o += HULL_NT) {
            int a = ocnt[o], b = (o + 1 < nv_out) ? ocnt[o + 1] : nt_out;
            for (int i = a + 1; i < b; i++) {
                int k1 = out.tris[3 * i + 1], k2 = out.tris[3 * i + 2];
                int j = i - 1;
                while (j >= a && (out.tris[3 * j + 1] > k1 || (out.tris[3 * j + 1] == k1 && out.tris[3 * j + 2] > k2))) {
                    out.tris[3 * (j + 1) + 1] = out.tris[3 * j + 1];
                    out.tris[3 * (j + 1) + 2] = out.tris[3 * j + 2];
                    j--;
                }
                out.tris[3 * (j + 1) + 1] = k1; out.tris[3 * (j + 1) + 2] = k2;
            }
        }
        for (int i = tid; i < n; i += HULL_NT) {
            int pos = posn[i];
            if (pos >= 0) {
                out.verts[3 * pos] = pts[3 * i]; out.verts[3 * pos + 1] = pts[3 * i + 1]; out.verts[3 * pos + 2] = pts[3 * i + 2];
                if (out.vidx) out.vidx[pos] = i;
            }
        }
        __syncthreads();
        double vol = block_mesh_signed_volume(out.verts, nv_out, out.tris, nt_out, sh.dsh);
        if (tid == 0) { *o_nv = nv_out; *o_nt = nt_out; if (o_vol) *o_vol = (float)fabs(vol); }
    } else {
        if (tid == 0) {
            *o_nv = 0; *o_nt = 0; if (o_vol) *o_vol = 0.f;
            int e = sh.err ? sh.err : KERR_BT_HEAP_OUTPUT;
            atomicOr(err_word, e);
        }
    }
    __syncthreads();
}
