/*
 * orc_hausdorff.c — oracle: sampled bidirectional Hausdorff distance.
 * TEST INFRASTRUCTURE ONLY (see cuacd_oracle.h).
 *
 * Follows cuda/hausdorff.cuh:
 *   - per-surface sample budget res = max(HD_MIN_SAMPLES, (int)(HD_RESOLUTION*area))
 *     (:368-397); per-triangle count floor(res/area * a_t) with the parity rule
 *     for zero counts (:433-466).  The total area is accumulated here in
 *     64-bit fixed point (2^-36 units) so the total, and therefore every
 *     sample, is independent of summation order.
 *   - samples from the Wang hash of (t*65537 + k) with square-root
 *     barycentrics (:517-558), evaluated with an explicit FP32 operation order.
 *   - distance = exact nearest triangle (:68-115), here in FP64 by brute force
 *     over a uniform-grid candidate set; result sqrt(max(d_ab^2, d_ba^2)) (:1453).
 */
#include "cuacd_oracle.h"
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <pthread.h>

static unsigned int wang_hash(unsigned int seed)
{
    seed = (seed ^ 61u) ^ (seed >> 16);
    seed *= 9u;
    seed = seed ^ (seed >> 4);
    seed *= 0x27d4eb2du;
    seed = seed ^ (seed >> 15);
    return seed;
}

/* FP32 triangle area with a fixed operation order (fmaf where the product
 * pairs are summed) — the CUDA path evaluates the identical sequence. */
static float tri_area_f32(const float* v, int a, int b, int c)
{
    float abx = v[3*b] - v[3*a], aby = v[3*b+1] - v[3*a+1], abz = v[3*b+2] - v[3*a+2];
    float acx = v[3*c] - v[3*a], acy = v[3*c+1] - v[3*a+1], acz = v[3*c+2] - v[3*a+2];
    float nx = fmaf(aby, acz, -(abz * acy));
    float ny = fmaf(abz, acx, -(abx * acz));
    float nz = fmaf(abx, acy, -(aby * acx));
    float s = fmaf(nz, nz, fmaf(ny, ny, nx * nx));
    return 0.5f * sqrtf(s);
}

typedef struct { int res; float area; } hd_budget;

static hd_budget budget(const float* v, int nv, const int* t, int nt,
                        float resolution, int min_samples, int total_override)
{
    (void)nv;
    int64_t fx = 0;
    for (int i = 0; i < nt; i++) {
        float a = tri_area_f32(v, t[3*i], t[3*i+1], t[3*i+2]);
        fx += (int64_t)llrint(ldexp((double)a, 36));
    }
    double total = ldexp((double)fx, -36);
    hd_budget b;
    b.area = (float)total;
    int res;
    if (total_override > 0) res = total_override;
    else res = (int)((double)resolution * total);
    if (res < min_samples) res = min_samples;
    b.res = res;
    return b;
}

static int tri_count(float area_t, int t, int nt, hd_budget b)
{
    int area_count = (b.area > 1e-20f) ? (int)(((float)b.res / b.area) * area_t) : 0;
    if (nt > b.res) {
        int step = nt / b.res;
        return (area_count > 0) ? area_count : ((t % step == 0) ? 1 : 0);
    }
    return (area_count > 0) ? area_count : ((t % 2 == 0) ? 1 : 0);
}

int orc_hd_sample_count(const float* v, int nv, const int* t, int nt,
                        float resolution, int min_samples, int total_override)
{
    if (nt <= 0 || nv <= 0) return 0;
    hd_budget b = budget(v, nv, t, nt, resolution, min_samples, total_override);
    int total = 0;
    for (int i = 0; i < nt; i++)
        total += tri_count(tri_area_f32(v, t[3*i], t[3*i+1], t[3*i+2]), i, nt, b);
    return total;
}

int orc_hd_samples(const float* v, int nv, const int* t, int nt,
                   float resolution, int min_samples, int total_override,
                   float* out, int cap)
{
    if (nt <= 0 || nv <= 0) return 0;
    hd_budget b = budget(v, nv, t, nt, resolution, min_samples, total_override);
    int idx = 0;
    for (int i = 0; i < nt; i++) {
        int a = t[3*i], bb = t[3*i+1], c = t[3*i+2];
        int N = tri_count(tri_area_f32(v, a, bb, c), i, nt, b);
        for (int k = 0; k < N; k++) {
            unsigned int ha = wang_hash((unsigned int)i * 65537u + (unsigned int)k);
            unsigned int hb = wang_hash(ha + 0x9e3779b9u);
            float ra = (float)(ha & 0xFFFFFFu) / (float)0xFFFFFFu;
            float rb = (float)(hb & 0xFFFFFFu) / (float)0xFFFFFFu;
            float sqa = sqrtf(ra);
            float w0 = 1.0f - sqa;
            float w1 = sqa * (1.0f - rb);
            float w2 = sqa * rb;
            if (idx < cap) {
                for (int kk = 0; kk < 3; kk++)
                    out[3*idx+kk] = fmaf(w2, v[3*c+kk], fmaf(w1, v[3*bb+kk], w0 * v[3*a+kk]));
            }
            idx++;
        }
    }
    return idx;
}

/* FP64 point-triangle squared distance (hausdorff.cuh:68-115 structure). */
static double seg_d2(const double* p, const double* a, const double* b)
{
    double ab[3] = {b[0]-a[0], b[1]-a[1], b[2]-a[2]};
    double ap[3] = {p[0]-a[0], p[1]-a[1], p[2]-a[2]};
    double ab2 = ab[0]*ab[0] + ab[1]*ab[1] + ab[2]*ab[2];
    double t = ab2 > 1e-30 ? (ap[0]*ab[0] + ap[1]*ab[1] + ap[2]*ab[2]) / ab2 : 0.0;
    if (t < 0) t = 0; if (t > 1) t = 1;
    double d[3] = {ap[0]-t*ab[0], ap[1]-t*ab[1], ap[2]-t*ab[2]};
    return d[0]*d[0] + d[1]*d[1] + d[2]*d[2];
}

static double pt_tri_d2(const double* p, const double* a, const double* b, const double* c)
{
    double ab[3] = {b[0]-a[0], b[1]-a[1], b[2]-a[2]};
    double ac[3] = {c[0]-a[0], c[1]-a[1], c[2]-a[2]};
    double ap[3] = {p[0]-a[0], p[1]-a[1], p[2]-a[2]};
    double n[3] = {ab[1]*ac[2]-ab[2]*ac[1], ab[2]*ac[0]-ab[0]*ac[2], ab[0]*ac[1]-ab[1]*ac[0]};
    double n2 = n[0]*n[0] + n[1]*n[1] + n[2]*n[2];
    if (n2 < 1e-30) {
        double bp[3] = {p[0]-b[0], p[1]-b[1], p[2]-b[2]};
        double cp[3] = {p[0]-c[0], p[1]-c[1], p[2]-c[2]};
        double da = ap[0]*ap[0]+ap[1]*ap[1]+ap[2]*ap[2];
        double db = bp[0]*bp[0]+bp[1]*bp[1]+bp[2]*bp[2];
        double dc = cp[0]*cp[0]+cp[1]*cp[1]+cp[2]*cp[2];
        double m = da < db ? da : db; return m < dc ? m : dc;
    }
    double d00 = ab[0]*ab[0]+ab[1]*ab[1]+ab[2]*ab[2];
    double d01 = ab[0]*ac[0]+ab[1]*ac[1]+ab[2]*ac[2];
    double d02 = ab[0]*ap[0]+ab[1]*ap[1]+ab[2]*ap[2];
    double d11 = ac[0]*ac[0]+ac[1]*ac[1]+ac[2]*ac[2];
    double d12 = ac[0]*ap[0]+ac[1]*ap[1]+ac[2]*ap[2];
    double inv = 1.0 / (d00*d11 - d01*d01);
    double u = (d11*d02 - d01*d12) * inv;
    double w = (d00*d12 - d01*d02) * inv;
    if (u >= 0 && w >= 0 && u + w <= 1) {
        double dist = n[0]*ap[0] + n[1]*ap[1] + n[2]*ap[2];
        return dist * dist / n2;
    }
    double e0 = seg_d2(p, a, b), e1 = seg_d2(p, b, c), e2 = seg_d2(p, c, a);
    double m = e0 < e1 ? e0 : e1; return m < e2 ? m : e2;
}

/* ---- uniform grid over target triangles for exact nearest search ---- */
typedef struct {
    const float* v; const int* t; int nt;
    double lo[3], cell; int dim[3];
    int* cstart; int* items;     /* CSR: cell -> triangle list */
    double* tb;                  /* per-triangle bbox lo/hi (6) */
} grid;

static void grid_build(grid* g, const float* v, const int* t, int nt)
{
    g->v = v; g->t = t; g->nt = nt;
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    g->tb = (double*)malloc(sizeof(double) * 6 * (size_t)nt);
    for (int i = 0; i < nt; i++) {
        double* b = g->tb + 6*i;
        for (int k = 0; k < 3; k++) { b[k] = 1e300; b[3+k] = -1e300; }
        for (int j = 0; j < 3; j++) {
            int vi = t[3*i+j];
            for (int k = 0; k < 3; k++) {
                double x = v[3*vi+k];
                if (x < b[k]) b[k] = x; if (x > b[3+k]) b[3+k] = x;
            }
        }
        for (int k = 0; k < 3; k++) { if (b[k] < lo[k]) lo[k] = b[k]; if (b[3+k] > hi[k]) hi[k] = b[3+k]; }
    }
    double ext = 0; for (int k = 0; k < 3; k++) if (hi[k]-lo[k] > ext) ext = hi[k]-lo[k];
    if (ext <= 0) ext = 1;
    int r = (int)cbrt((double)nt) + 1; if (r > 128) r = 128;
    g->cell = ext / r * 1.000001;
    for (int k = 0; k < 3; k++) {
        g->lo[k] = lo[k];
        g->dim[k] = (int)((hi[k]-lo[k]) / g->cell) + 1;
    }
    int nc = g->dim[0]*g->dim[1]*g->dim[2];
    int* cnt = (int*)calloc((size_t)nc + 1, sizeof(int));
    for (int pass = 0; pass < 2; pass++) {
        for (int i = 0; i < nt; i++) {
            double* b = g->tb + 6*i;
            int c0[3], c1[3];
            for (int k = 0; k < 3; k++) {
                c0[k] = (int)((b[k]-g->lo[k]) / g->cell); c1[k] = (int)((b[3+k]-g->lo[k]) / g->cell);
                if (c0[k] < 0) c0[k] = 0; if (c1[k] >= g->dim[k]) c1[k] = g->dim[k]-1;
            }
            for (int x = c0[0]; x <= c1[0]; x++)
                for (int y = c0[1]; y <= c1[1]; y++)
                    for (int z = c0[2]; z <= c1[2]; z++) {
                        int c = (x*g->dim[1] + y)*g->dim[2] + z;
                        if (pass == 0) cnt[c+1]++;
                        else g->items[g->cstart[c] + (cnt[c]++)] = i;
                    }
        }
        if (pass == 0) {
            for (int c = 0; c < nc; c++) cnt[c+1] += cnt[c];
            g->cstart = (int*)malloc(sizeof(int) * ((size_t)nc + 1));
            memcpy(g->cstart, cnt, sizeof(int) * ((size_t)nc + 1));
            g->items = (int*)malloc(sizeof(int) * (size_t)(cnt[nc] > 0 ? cnt[nc] : 1));
            memset(cnt, 0, sizeof(int) * ((size_t)nc + 1));
        }
    }
    free(cnt);
}
static void grid_free(grid* g) { free(g->cstart); free(g->items); free(g->tb); }

/* exact nearest-triangle squared distance, visiting cells in growing shells */
static double grid_nearest(const grid* g, const double* p, int* stamp, int sid)
{
    double best = 1e300;
    int pc[3];
    for (int k = 0; k < 3; k++) {
        int c = (int)floor((p[k]-g->lo[k]) / g->cell);
        if (c < 0) c = 0; if (c >= g->dim[k]) c = g->dim[k]-1;
        pc[k] = c;
    }
    int maxr = g->dim[0]; if (g->dim[1] > maxr) maxr = g->dim[1]; if (g->dim[2] > maxr) maxr = g->dim[2];
    for (int r = 0; r <= maxr; r++) {
        /* cells at Chebyshev distance r; any point in them is >= (r-1)*cell away */
        double shell_lb = 0.0;
        if (r >= 1) {
            /* distance from p to the boundary of the (2r-1)^3 box of cells */
            double lbk = 1e300;
            for (int k = 0; k < 3; k++) {
                double lo = g->lo[k] + (pc[k] - (r - 1)) * g->cell;
                double hi = g->lo[k] + (pc[k] + r) * g->cell;
                double a = p[k] - lo, b = hi - p[k];
                if (a < lbk) lbk = a; if (b < lbk) lbk = b;
            }
            shell_lb = lbk > 0 ? lbk : 0;
        }
        if (shell_lb * shell_lb > best) break;
        for (int x = pc[0]-r; x <= pc[0]+r; x++) {
            if (x < 0 || x >= g->dim[0]) continue;
            for (int y = pc[1]-r; y <= pc[1]+r; y++) {
                if (y < 0 || y >= g->dim[1]) continue;
                for (int z = pc[2]-r; z <= pc[2]+r; z++) {
                    if (z < 0 || z >= g->dim[2]) continue;
                    int ax = abs(x-pc[0]), ay = abs(y-pc[1]), az = abs(z-pc[2]);
                    int cheb = ax > ay ? ax : ay; cheb = cheb > az ? cheb : az;
                    if (cheb != r) continue;
                    int c = (x*g->dim[1] + y)*g->dim[2] + z;
                    for (int it = g->cstart[c]; it < g->cstart[c+1]; it++) {
                        int ti = g->items[it];
                        if (stamp[ti] == sid) continue;
                        stamp[ti] = sid;
                        const double* b = g->tb + 6*ti;
                        double dd = 0;
                        for (int k = 0; k < 3; k++) {
                            double e = 0;
                            if (p[k] < b[k]) e = b[k]-p[k]; else if (p[k] > b[3+k]) e = p[k]-b[3+k];
                            dd += e*e;
                        }
                        if (dd >= best) continue;
                        double A[3], B[3], C[3];
                        int ia = g->t[3*ti], ib = g->t[3*ti+1], ic = g->t[3*ti+2];
                        for (int k = 0; k < 3; k++) { A[k] = g->v[3*ia+k]; B[k] = g->v[3*ib+k]; C[k] = g->v[3*ic+k]; }
                        double d = pt_tri_d2(p, A, B, C);
                        if (d < best) best = d;
                    }
                }
            }
        }
    }
    return best;
}

typedef struct {
    const grid* g; const float* s; int lo, hi; double out;
} hd_job;

static void* hd_worker(void* arg)
{
    hd_job* j = (hd_job*)arg;
    int* stamp = (int*)malloc(sizeof(int) * (size_t)(j->g->nt > 0 ? j->g->nt : 1));
    for (int i = 0; i < j->g->nt; i++) stamp[i] = -1;
    double m = 0;
    for (int i = j->lo; i < j->hi; i++) {
        double p[3] = {j->s[3*i], j->s[3*i+1], j->s[3*i+2]};
        double d = grid_nearest(j->g, p, stamp, i);
        if (d > m) m = d;
    }
    free(stamp);
    j->out = m;
    return NULL;
}

static double directed_max(const float* samples, int ns, const float* v, const int* t, int nt, int n_threads)
{
    if (ns <= 0 || nt <= 0) return 0.0;
    grid g; grid_build(&g, v, t, nt);
    if (n_threads < 1) n_threads = 1;
    if (n_threads > 256) n_threads = 256;
    hd_job jobs[256]; pthread_t th[256];
    int per = (ns + n_threads - 1) / n_threads;
    int nj = 0;
    for (int k = 0; k < n_threads; k++) {
        int lo = k * per, hi = lo + per; if (hi > ns) hi = ns;
        if (lo >= hi) break;
        jobs[nj].g = &g; jobs[nj].s = samples; jobs[nj].lo = lo; jobs[nj].hi = hi; jobs[nj].out = 0;
        nj++;
    }
    if (nj == 1) hd_worker(&jobs[0]);
    else {
        for (int k = 0; k < nj; k++) pthread_create(&th[k], NULL, hd_worker, &jobs[k]);
        for (int k = 0; k < nj; k++) pthread_join(th[k], NULL);
    }
    double m = 0; for (int k = 0; k < nj; k++) if (jobs[k].out > m) m = jobs[k].out;
    grid_free(&g);
    return m;
}

double orc_hausdorff(const float* av, int anv, const int* at, int ant,
                     const float* bv, int bnv, const int* bt, int bnt,
                     float resolution, int min_samples, int total_override,
                     int n_threads)
{
    if (ant <= 0 || anv <= 0 || bnt <= 0 || bnv <= 0) return 0.0;
    int na = orc_hd_sample_count(av, anv, at, ant, resolution, min_samples, total_override);
    int nb = orc_hd_sample_count(bv, bnv, bt, bnt, resolution, min_samples, total_override);
    if (na <= 0 || nb <= 0) return 0.0;
    float* sa = (float*)malloc(sizeof(float) * 3 * (size_t)na);
    float* sb = (float*)malloc(sizeof(float) * 3 * (size_t)nb);
    orc_hd_samples(av, anv, at, ant, resolution, min_samples, total_override, sa, na);
    orc_hd_samples(bv, bnv, bt, bnt, resolution, min_samples, total_override, sb, nb);
    double dab = directed_max(sa, na, bv, bt, bnt, n_threads);
    double dba = directed_max(sb, nb, av, at, ant, n_threads);
    free(sa); free(sb);
    return sqrt(dab > dba ? dab : dba);
}
