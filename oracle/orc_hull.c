/*
 * orc_hull.c — oracle: mesh volume, hull quantisation and exact hull.
 * TEST INFRASTRUCTURE ONLY (see cuacd_oracle.h).
 *
 * Hull semantics follow cuda/hull_dandc.cuh:
 *   - points are quantised onto an int grid whose per-axis step is
 *     span/10216, with axes permuted to (med, max, min) and a sign flip when
 *     (medAx+1)%3 != maxAx; coordinates are truncated toward zero
 *     (hull_dandc.cuh:1366-1408).  Divisions here are IEEE-rounded.
 *   - the hull is exact on that grid; identical grid points keep the first in
 *     (y,x,z,index) order, i.e. the smallest input index (warp_sort.cuh:237-244)
 *   - output vertices are the input floats of the hull corners
 *     (hull_dandc.cuh:1268-1274); coplanar faces are merged and fan
 *     triangulated (hull_dandc.cuh:1296-1320).
 * The reference builds the hull by divide & conquer (a Bullet port); this
 * oracle finds the same polytope by exact gift wrapping over polygon faces.
 */
#include "cuacd_oracle.h"
#include <stdlib.h>
#include <string.h>
#include <math.h>

/* ------------------------------------------------------------------ */
/* volume: cuda/mesh_volume.cuh:20-49 (anchor at vertex 0), in FP64     */
/* ------------------------------------------------------------------ */
double orc_mesh_signed_volume(const float* v, int nv, const int* t, int nt)
{
    if (nt <= 0 || nv <= 0) return 0.0;
    double ox = v[0], oy = v[1], oz = v[2];
    double acc = 0.0;
    for (int i = 0; i < nt; i++) {
        int a = t[3*i], b = t[3*i+1], c = t[3*i+2];
        double ax = v[3*a]-ox, ay = v[3*a+1]-oy, az = v[3*a+2]-oz;
        double bx = v[3*b]-ox, by = v[3*b+1]-oy, bz = v[3*b+2]-oz;
        double cx = v[3*c]-ox, cy = v[3*c+1]-oy, cz = v[3*c+2]-oz;
        double nx = by*cz - bz*cy, ny = bz*cx - bx*cz, nz = bx*cy - by*cx;
        acc += ax*nx + ay*ny + az*nz;
    }
    return acc / 6.0;
}

/* ------------------------------------------------------------------ */
/* quantisation: cuda/hull_dandc.cuh:1351-1411                          */
/* ------------------------------------------------------------------ */
int orc_quantize(const float* pts, int n, int* q)
{
    float mn[3] = {1e30f, 1e30f, 1e30f}, mx[3] = {-1e30f, -1e30f, -1e30f};
    for (int i = 0; i < n; i++)
        for (int k = 0; k < 3; k++) {
            float x = pts[3*i+k];
            if (x < mn[k]) mn[k] = x;
            if (x > mx[k]) mx[k] = x;
        }
    float span[3] = {mx[0]-mn[0], mx[1]-mn[1], mx[2]-mn[2]};
    int maxAx = (span[0] >= span[1]) ? ((span[0] >= span[2]) ? 0 : 2) : ((span[1] >= span[2]) ? 1 : 2);
    int minAx = (span[0] <= span[1]) ? ((span[0] <= span[2]) ? 0 : 2) : ((span[1] <= span[2]) ? 1 : 2);
    if (minAx == maxAx) minAx = (maxAx + 1) % 3;
    int medAx = 3 - maxAx - minAx;
    volatile float sc[3];
    for (int k = 0; k < 3; k++) sc[k] = span[k] / 10216.0f;
    if (((medAx + 1) % 3) != maxAx)
        for (int k = 0; k < 3; k++) sc[k] = -sc[k];
    float cen[3];
    for (int k = 0; k < 3; k++) cen[k] = (mn[k] + mx[k]) * 0.5f;
    int ax[3] = {medAx, maxAx, minAx};
    float inv[3];
    for (int k = 0; k < 3; k++) {
        float s = sc[ax[k]];
        inv[k] = (s != 0.0f) ? 1.0f / s : 0.0f;
    }
    for (int i = 0; i < n; i++)
        for (int k = 0; k < 3; k++) {
            volatile float d = pts[3*i+ax[k]] - cen[ax[k]];
            volatile float p = d * inv[k];
            q[3*i+k] = (int)p;
        }
    return 0;
}

/* ------------------------------------------------------------------ */
/* exact hull by gift wrapping over polygon faces                       */
/* ------------------------------------------------------------------ */
typedef struct { int64_t x, y, z; } v3;

static v3 pt(const int* q, int i) { v3 r = {q[3*i], q[3*i+1], q[3*i+2]}; return r; }
static v3 sub(v3 a, v3 b) { v3 r = {a.x-b.x, a.y-b.y, a.z-b.z}; return r; }
static v3 cross(v3 a, v3 b) {
    v3 r = {a.y*b.z - a.z*b.y, a.z*b.x - a.x*b.z, a.x*b.y - a.y*b.x}; return r;
}
static int64_t dot(v3 a, v3 b) { return a.x*b.x + a.y*b.y + a.z*b.z; }
static int is_zero(v3 a) { return a.x == 0 && a.y == 0 && a.z == 0; }
static int same(const int* q, int i, int j) {
    return q[3*i] == q[3*j] && q[3*i+1] == q[3*j+1] && q[3*i+2] == q[3*j+2];
}

typedef struct {
    const int* q; int n;
    int* canon;           /* canonical representative (smallest index) per point */
    /* faces */
    int* corner; int ncorner, ccap;
    int* fstart; int* fsize; int nface, fcap;
    /* directed edge hash: key -> face */
    uint64_t* hkey; int* hval; int hcap;
    /* frontier stack of directed edges */
    int* stk; int nstk, scap;
    int err;
} hstate;

static uint64_t ekey(int u, int v) { return ((uint64_t)(uint32_t)u << 32) | (uint32_t)v; }

static int h_find(hstate* s, uint64_t k) {
    uint64_t h = (k * 0x9E3779B97F4A7C15ull) >> 20;
    for (int i = 0; i < s->hcap; i++) {
        int slot = (int)((h + (uint64_t)i) & (uint64_t)(s->hcap - 1));
        if (s->hkey[slot] == ~0ull) return -1;
        if (s->hkey[slot] == k) return s->hval[slot];
    }
    return -1;
}
static int h_insert(hstate* s, uint64_t k, int val) {
    uint64_t h = (k * 0x9E3779B97F4A7C15ull) >> 20;
    for (int i = 0; i < s->hcap; i++) {
        int slot = (int)((h + (uint64_t)i) & (uint64_t)(s->hcap - 1));
        if (s->hkey[slot] == ~0ull) { s->hkey[slot] = k; s->hval[slot] = val; return 0; }
        if (s->hkey[slot] == k) return 1;   /* duplicate directed edge */
    }
    return -1;
}

/* Rotate the supporting plane about the line (a, dir) towards the points and
 * return the first point hit: q replaces c when (dir x (c-a)).(q-a) < 0.
 * Points on the line are skipped.  Returns -1 if every point is on the line. */
static int wrap(hstate* s, int a, v3 dir)
{
    v3 pa = pt(s->q, a);
    int c = -1; v3 m = {0, 0, 0};
    for (int i = 0; i < s->n; i++) {
        if (s->canon[i] != i) continue;
        v3 d = sub(pt(s->q, i), pa);
        if (is_zero(cross(dir, d))) continue;
        if (c < 0 || dot(m, d) < 0) { c = i; m = cross(dir, d); }
    }
    return c;
}

/* projected 2D orientation helpers for a face with normal N */
typedef struct { int ku, kv; int sgn; } proj;
static proj mkproj(v3 N) {
    int64_t ax = N.x < 0 ? -N.x : N.x, ay = N.y < 0 ? -N.y : N.y, az = N.z < 0 ? -N.z : N.z;
    int k = (ax >= ay && ax >= az) ? 0 : (ay >= az ? 1 : 2);
    int64_t nk = k == 0 ? N.x : (k == 1 ? N.y : N.z);
    proj p; p.ku = (k + 1) % 3; p.kv = (k + 2) % 3; p.sgn = nk > 0 ? 1 : -1;
    return p;
}
static int64_t o2(const int* q, proj P, int p, int r, int t) {
    int64_t ux = q[3*r+P.ku] - q[3*p+P.ku], uy = q[3*r+P.kv] - q[3*p+P.kv];
    int64_t wx = q[3*t+P.ku] - q[3*p+P.ku], wy = q[3*t+P.kv] - q[3*p+P.kv];
    return (ux*wy - uy*wx) * P.sgn;
}
static int64_t d2(const int* q, proj P, int p, int r) {
    int64_t ux = q[3*r+P.ku] - q[3*p+P.ku], uy = q[3*r+P.kv] - q[3*p+P.kv];
    return ux*ux + uy*uy;
}

/* Strict CCW polygon (w.r.t. N) of the coplanar set S.  If start>=0 the walk
 * starts at corner `start` whose predecessor is `prev`; else it starts at
 * the 2D-lexmin corner.  Corners are appended to s->corner.  Returns the
 * corner count (>=3) or -1. */
static int polygon(hstate* s, const int* S, int ns, v3 N, int start, int prev)
{
    proj P = mkproj(N);
    const int* q = s->q;
    int first;
    if (start < 0) {
        int b = S[0];
        for (int i = 1; i < ns; i++) {
            int t = S[i];
            int tu = q[3*t+P.ku], tv = q[3*t+P.kv], bu = q[3*b+P.ku], bv = q[3*b+P.kv];
            if (tu < bu || (tu == bu && (tv < bv || (tv == bv && t < b)))) b = t;
        }
        first = b;
    } else first = start;
    int base = s->ncorner;
    int cur = first, cnt = 0;
    int stop = (start < 0) ? first : prev;
    if (start >= 0) {
        if (s->ncorner + 1 > s->ccap) return -1;
        s->corner[s->ncorner++] = prev; cnt = 1;
    }
    for (int guard = 0; guard <= ns + 1; guard++) {
        if (s->ncorner + 1 > s->ccap) return -1;
        s->corner[s->ncorner++] = cur; cnt++;
        int r = -1;
        for (int i = 0; i < ns; i++) {
            int t = S[i];
            if (same(q, t, cur)) continue;
            if (r < 0) { r = t; continue; }
            int64_t o = o2(q, P, cur, r, t);
            if (o < 0) r = t;
            else if (o == 0) {
                if (same(q, t, r)) { if (t < r) r = t; }
                else if (d2(q, P, cur, t) > d2(q, P, cur, r)) r = t;
            }
        }
        if (r < 0) return -1;
        if (r == stop) {
            if (start < 0) return cnt;
            /* rotate so the list starts at prev: it already does */
            return cnt;
        }
        cur = r;
        if (cnt > ns + 1) break;
    }
    s->ncorner = base;
    return -1;
}

static int add_face(hstate* s, int cstart, int k)
{
    if (s->nface + 1 > s->fcap) return -1;
    int f = s->nface++;
    s->fstart[f] = cstart; s->fsize[f] = k;
    for (int i = 0; i < k; i++) {
        int u = s->corner[cstart + i], v = s->corner[cstart + (i + 1) % k];
        int r = h_insert(s, ekey(u, v), f);
        if (r != 0) return -1;
        if (h_find(s, ekey(v, u)) < 0) {
            if (s->nstk + 2 > s->scap) return -1;
            s->stk[s->nstk++] = u; s->stk[s->nstk++] = v;
        }
    }
    return f;
}

/* collect points on plane through a with normal N */
static int coplanar(hstate* s, int a, v3 N, int* S)
{
    v3 pa = pt(s->q, a);
    int ns = 0;
    for (int i = 0; i < s->n; i++) {
        if (s->canon[i] != i) continue;
        if (dot(N, sub(pt(s->q, i), pa)) == 0) S[ns++] = i;
    }
    return ns;
}

static const int* g_qsort_q;   /* qsort context (oracle is single-threaded per hull call) */
static int qcmp_ctx(const void* a, const void* b)
{
    int i = *(const int*)a, j = *(const int*)b;
    const int* q = g_qsort_q;
    for (int k = 0; k < 3; k++) if (q[3*i+k] != q[3*j+k]) return q[3*i+k] < q[3*j+k] ? -1 : 1;
    return (i > j) - (i < j);
}
static int cmp_int(const void* a, const void* b) {
    int x = *(const int*)a, y = *(const int*)b; return (x > y) - (x < y);
}
static int cmp_tri(const void* a, const void* b) {
    const int* x = (const int*)a; const int* y = (const int*)b;
    for (int k = 0; k < 3; k++) if (x[k] != y[k]) return x[k] < y[k] ? -1 : 1;
    return 0;
}

int orc_hull(const float* pts, int n, int* out_vidx, int vcap, int* out_nv,
             int* out_tris, int tcap, int* out_nt, double* out_vol)
{
    *out_nv = 0; *out_nt = 0; *out_vol = 0.0;
    if (n < 4) return 1;
    int* q = (int*)malloc(sizeof(int) * 3 * (size_t)n);
    orc_quantize(pts, n, q);
    hstate s; memset(&s, 0, sizeof(s));
    s.q = q; s.n = n;
    s.canon = (int*)malloc(sizeof(int) * (size_t)n);
    /* canonical representative: smallest index with identical grid coords */
    {
        int* order = (int*)malloc(sizeof(int) * (size_t)n);
        for (int i = 0; i < n; i++) order[i] = i;
        /* sort indices by (x,y,z,idx); runs of equal coords share the
         * first (smallest) index */
        for (int i = 0; i < n; i++) s.canon[i] = i;
        g_qsort_q = q;
        qsort(order, (size_t)n, sizeof(int), qcmp_ctx);
        for (int i = 1; i < n; i++)
            if (same(q, order[i], order[i-1])) s.canon[order[i]] = s.canon[order[i-1]];
        free(order);
    }
    s.ccap = 6 * n + 64; s.corner = (int*)malloc(sizeof(int) * (size_t)s.ccap);
    s.fcap = 2 * n + 8; s.fstart = (int*)malloc(sizeof(int) * (size_t)s.fcap);
    s.fsize = (int*)malloc(sizeof(int) * (size_t)s.fcap);
    s.hcap = 1; while (s.hcap < 4 * (6 * n + 64)) s.hcap <<= 1;
    s.hkey = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)s.hcap);
    memset(s.hkey, 0xff, sizeof(uint64_t) * (size_t)s.hcap);
    s.hval = (int*)malloc(sizeof(int) * (size_t)s.hcap);
    s.scap = 2 * (6 * n + 64); s.stk = (int*)malloc(sizeof(int) * (size_t)s.scap);
    int* S = (int*)malloc(sizeof(int) * (size_t)n);
    int rc = 0;

    /* initial face: p0 = lexmin (x,y,z,idx); wrap about the z-parallel line
     * through p0 starting from the supporting plane x = xmin. */
    int p0 = 0;
    for (int i = 1; i < n; i++) {
        if (s.canon[i] != i) continue;
        if (q[3*i] < q[3*p0] || (q[3*i] == q[3*p0] && (q[3*i+1] < q[3*p0+1] ||
            (q[3*i+1] == q[3*p0+1] && q[3*i+2] < q[3*p0+2])))) p0 = i;
    }
    v3 dz = {0, 0, 1};
    int c = wrap(&s, p0, dz);
    if (c < 0) { rc = 1; goto done; }
    v3 N = cross(sub(pt(q, c), pt(q, p0)), dz);
    int ns = coplanar(&s, p0, N, S);
    {
        /* is S collinear? */
        int noncol = 0;
        v3 e = sub(pt(q, c), pt(q, p0));
        for (int i = 0; i < ns; i++)
            if (!is_zero(cross(e, sub(pt(q, S[i]), pt(q, p0))))) { noncol = 1; break; }
        if (!noncol) {
            int c2 = wrap(&s, p0, e);
            if (c2 < 0) { rc = 1; goto done; }
            N = cross(sub(pt(q, c2), pt(q, p0)), e);
            if (is_zero(N)) { rc = 1; goto done; }
            ns = coplanar(&s, p0, N, S);
        }
    }
    {
        int cs = s.ncorner;
        int k = polygon(&s, S, ns, N, -1, -1);
        if (k < 3) { rc = 1; goto done; }
        if (add_face(&s, cs, k) < 0) { rc = -1; goto done; }
    }
    while (s.nstk > 0) {
        int v = s.stk[--s.nstk], u = s.stk[--s.nstk];
        if (h_find(&s, ekey(v, u)) >= 0) continue;
        v3 d = sub(pt(q, v), pt(q, u));
        int cc = wrap(&s, u, d);
        if (cc < 0) { rc = -1; goto done; }
        v3 NG = cross(sub(pt(q, cc), pt(q, u)), d);
        int m = coplanar(&s, u, NG, S);
        int cs = s.ncorner;
        int k = polygon(&s, S, m, NG, u, v);
        if (k < 3) { rc = -1; goto done; }
        if (add_face(&s, cs, k) < 0) { rc = -1; goto done; }
    }

    /* canonical output */
    {
        int nvtx = 0;
        int* mark = (int*)calloc((size_t)n, sizeof(int));
        for (int i = 0; i < s.ncorner; i++) mark[s.corner[i]] = 1;
        for (int i = 0; i < n; i++) if (mark[i]) nvtx++;
        int ntri = 0;
        for (int f = 0; f < s.nface; f++) ntri += s.fsize[f] - 2;
        if (nvtx > vcap || ntri > tcap) { free(mark); rc = -1; goto done; }
        int* pos = (int*)malloc(sizeof(int) * (size_t)n);
        int j = 0;
        for (int i = 0; i < n; i++) if (mark[i]) { pos[i] = j; out_vidx[j++] = i; }
        int t = 0;
        for (int f = 0; f < s.nface; f++) {
            int st = s.fstart[f], k = s.fsize[f];
            int mi = 0;
            for (int i = 1; i < k; i++) if (s.corner[st+i] < s.corner[st+mi]) mi = i;
            for (int i = 1; i + 1 < k; i++) {
                out_tris[3*t]   = pos[s.corner[st + mi]];
                out_tris[3*t+1] = pos[s.corner[st + (mi + i) % k]];
                out_tris[3*t+2] = pos[s.corner[st + (mi + i + 1) % k]];
                t++;
            }
        }
        qsort(out_tris, (size_t)ntri, 3 * sizeof(int), cmp_tri);
        *out_nv = nvtx; *out_nt = ntri;
        /* volume over float coords */
        float* hv = (float*)malloc(sizeof(float) * 3 * (size_t)(nvtx > 0 ? nvtx : 1));
        for (int i = 0; i < nvtx; i++)
            for (int kk = 0; kk < 3; kk++) hv[3*i+kk] = pts[3*out_vidx[i]+kk];
        double vol = orc_mesh_signed_volume(hv, nvtx, out_tris, ntri);
        *out_vol = vol < 0 ? -vol : vol;
        free(hv); free(pos); free(mark);
    }
done:
    free(S); free(s.stk); free(s.hval); free(s.hkey); free(s.fsize); free(s.fstart);
    free(s.corner); free(s.canon); free(q);
    (void)cmp_int;
    return rc;
}

