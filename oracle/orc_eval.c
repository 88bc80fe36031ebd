/*
 * orc_eval.c — oracle: candidate planes, part costs and the candidate
 * evaluator (cut -> volumes -> hulls -> Hausdorff -> costs).
 * TEST INFRASTRUCTURE ONLY (see cuacd_oracle.h).
 */
#include "cuacd_oracle.h"
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <pthread.h>

/* ------------------------------------------------------------------ */
/* part costs: cuda/la_common.cuh:21-34                                 */
/* ------------------------------------------------------------------ */
double orc_cost_rv(double hull_vol, double mesh_vol)
{
    const double pi = 3.14159265358979;
    double g = hull_vol - mesh_vol; if (g < 0) g = 0;
    return 0.3 * cbrt((3.0 / (4.0 * pi)) * g);
}
double orc_cost_full(double hull_vol, double mesh_vol, double hausdorff)
{
    double rv = orc_cost_rv(hull_vol, mesh_vol);
    return rv > hausdorff ? rv : hausdorff;
}

/* ------------------------------------------------------------------ */
/* axis candidates: cuda/la_axis_cut.cuh:10-19, la_expand.cu:129-199    */
/* ------------------------------------------------------------------ */
int orc_axis_plane(const float* v, int nv, int width, int cut_idx,
                   float min_edge_dist, float* out)
{
    float lo[3] = {1e30f, 1e30f, 1e30f}, hi[3] = {-1e30f, -1e30f, -1e30f};
    for (int i = 0; i < nv; i++)
        for (int k = 0; k < 3; k++) {
            float x = v[3*i+k];
            if (x < lo[k]) lo[k] = x;
            if (x > hi[k]) hi[k] = x;
        }
    int count = width / 3, rem = width % 3;
    int xc = count + (rem > 0), yc = count + (rem > 1);
    int axis, slice, cpa;
    if (cut_idx < xc) { axis = 0; slice = cut_idx; cpa = xc; }
    else if (cut_idx < xc + yc) { axis = 1; slice = cut_idx - xc; cpa = yc; }
    else { axis = 2; slice = cut_idx - xc - yc; cpa = count; }
    float lo_valid = lo[axis] + min_edge_dist;
    float hi_valid = hi[axis] - min_edge_dist;
    if (lo_valid >= hi_valid) return 1;
    float frac = ((float)slice + 1.0f) / ((float)cpa + 1.0f);
    float cut = fmaf(frac, hi_valid - lo_valid, lo_valid);
    out[0] = axis == 0 ? 1.0f : 0.0f;
    out[1] = axis == 1 ? 1.0f : 0.0f;
    out[2] = axis == 2 ? 1.0f : 0.0f;
    out[3] = -cut;
    return 0;
}

/* ------------------------------------------------------------------ */
/* concave-edge planes: cuda/la_concave.cu:48-363                       */
/* ------------------------------------------------------------------ */
typedef struct { int lo, hi, f; } ef;
static int cmp_ef(const void* a, const void* b) {
    const ef* x = (const ef*)a; const ef* y = (const ef*)b;
    if (x->lo != y->lo) return x->lo < y->lo ? -1 : 1;
    if (x->hi != y->hi) return x->hi < y->hi ? -1 : 1;
    if (x->f != y->f) return x->f < y->f ? -1 : 1;
    return 0;
}

/* unit face normal, fixed FP32 operation order; returns 0 if degenerate */
static int face_normal(const float* v, const int* t, int f, float* n)
{
    const float* a = v + 3*t[3*f]; const float* b = v + 3*t[3*f+1]; const float* c = v + 3*t[3*f+2];
    float e1x = b[0]-a[0], e1y = b[1]-a[1], e1z = b[2]-a[2];
    float e2x = c[0]-a[0], e2y = c[1]-a[1], e2z = c[2]-a[2];
    float nx = fmaf(e1y, e2z, -(e1z * e2y));
    float ny = fmaf(e1z, e2x, -(e1x * e2z));
    float nz = fmaf(e1x, e2y, -(e1y * e2x));
    float len = sqrtf(fmaf(nz, nz, fmaf(ny, ny, nx * nx)));
    if (len < 1e-12f) return 0;
    n[0] = nx / len; n[1] = ny / len; n[2] = nz / len;
    return 1;
}

static unsigned int lcg_next(unsigned int* s) { *s = *s * 1664525u + 1013904223u; return *s; }

/* The dihedral test `dihedral > threshold` with dihedral = pi +- acos(c)
 * (la_concave.cu:213-234) is evaluated without acos: it holds iff
 * d > 0 and c < cos(threshold - pi), or d <= 0 and c > cos(pi - threshold);
 * the two cosines are formed once in double. */
static void dihedral_cos(float thr, int* mode_pos, float* cpos, int* mode_neg, float* cneg)
{
    const double pi = 3.14159265358979;
    double xp = (double)thr - pi;          /* d > 0: need acos(c) > xp */
    if (xp < 0) *mode_pos = 1;             /* always */
    else if (xp >= pi) *mode_pos = 0;      /* never */
    else { *mode_pos = 2; *cpos = (float)cos(xp); }
    double xn = pi - (double)thr;          /* d <= 0: need acos(c) < xn */
    if (xn <= 0) *mode_neg = 0;
    else if (xn > pi) *mode_neg = 1;
    else { *mode_neg = 2; *cneg = (float)cos(xn); }
}

int orc_concave_planes(const float* v, int nv, const int* t, int nt,
                       int K, float eps, float thr, float* out)
{
    (void)nv;
    if (nt < 2 || K <= 0) return 0;
    int nd = 3 * nt;
    ef* e = (ef*)malloc(sizeof(ef) * (size_t)nd);
    for (int i = 0; i < nd; i++) {
        int f = i / 3, k = i % 3;
        int a = t[3*f+k], b = t[3*f+(k+1)%3];
        e[i].lo = a < b ? a : b; e[i].hi = a < b ? b : a; e[i].f = f;
    }
    qsort(e, (size_t)nd, sizeof(ef), cmp_ef);
    int mp, mn; float cp = 0, cn = 0;
    dihedral_cos(thr, &mp, &cp, &mn, &cn);
    int* res = (int*)malloc(sizeof(int) * 4 * (size_t)K);
    for (int i = 0; i < 4 * K; i++) res[i] = -1;
    int n_seen = 0, n_res = 0; unsigned int rng = 1u;
    for (int i = 0; i + 1 < nd; i++) {
        int first = (i == 0) || e[i-1].lo != e[i].lo || e[i-1].hi != e[i].hi;
        int shared = e[i].lo == e[i+1].lo && e[i].hi == e[i+1].hi && e[i].f != e[i+1].f;
        if (!(first && shared)) continue;
        int v0 = e[i].lo, v1 = e[i].hi, f0 = e[i].f, f1 = e[i+1].f;
        float n0[3], n1[3];
        if (!face_normal(v, t, f0, n0) || !face_normal(v, t, f1, n1)) continue;
        float c = fmaf(n0[2], n1[2], fmaf(n0[1], n1[1], n0[0] * n1[0]));
        c = fmaxf(-1.0f, fminf(1.0f, c));
        int other = -1;
        for (int k = 0; k < 3; k++) { int vv = t[3*f0+k]; if (vv != v0 && vv != v1) { other = vv; break; } }
        if (other < 0) continue;
        float dx = v[3*other] - v[3*v0], dy = v[3*other+1] - v[3*v0+1], dz = v[3*other+2] - v[3*v0+2];
        float d = fmaf(dz, n1[2], fmaf(dy, n1[1], dx * n1[0]));
        int valid;
        if (d > 0.0f) valid = (mp == 1) || (mp == 2 && c < cp);
        else          valid = (mn == 1) || (mn == 2 && c > cn);
        if (!valid) continue;
        n_seen++;
        if (n_res < K) {
            int s = n_res++;
            res[4*s] = v0; res[4*s+1] = v1; res[4*s+2] = f0; res[4*s+3] = f1;
        } else {
            unsigned int r = lcg_next(&rng);
            unsigned int th = (unsigned int)((float)K / (float)n_seen * 4294967295.0f);
            if (r < th) {
                unsigned int r2 = lcg_next(&rng);
                int s = (int)(r2 % (unsigned int)K);
                res[4*s] = v0; res[4*s+1] = v1; res[4*s+2] = f0; res[4*s+3] = f1;
            }
        }
    }
    int np = 0;
    for (int s = 0; s < n_res; s++) {
        int v0 = res[4*s], v1 = res[4*s+1], f0 = res[4*s+2], f1 = res[4*s+3];
        float n0[3], n1[3];
        if (!face_normal(v, t, f0, n0) || !face_normal(v, t, f1, n1)) continue;
        float mx = (v[3*v0] + v[3*v1]) * 0.5f, my = (v[3*v0+1] + v[3*v1+1]) * 0.5f, mz = (v[3*v0+2] + v[3*v1+2]) * 0.5f;
        float* o = out + 4 * np;
        o[0] = n1[0]; o[1] = n1[1]; o[2] = n1[2];
        o[3] = -(fmaf(n1[2], mz, fmaf(n1[1], my, n1[0] * mx)) + eps);
        o[4] = n0[0]; o[5] = n0[1]; o[6] = n0[2];
        o[7] = -(fmaf(n0[2], mz, fmaf(n0[1], my, n0[0] * mx)) + eps);
        np += 2;
        float bx = n0[0] + n1[0], by = n0[1] + n1[1], bz = n0[2] + n1[2];
        float bl = sqrtf(fmaf(bz, bz, fmaf(by, by, bx * bx)));
        if (bl >= 1e-4f) {
            bx = bx / bl; by = by / bl; bz = bz / bl;
            float bm = fmaf(bz, mz, fmaf(by, my, bx * mx));
            float* o2 = out + 4 * np;
            o2[0] = bx; o2[1] = by; o2[2] = bz; o2[3] = -(bm + eps);
            o2[4] = bx; o2[5] = by; o2[6] = bz; o2[7] = -(bm - eps);
            np += 2;
        }
    }
    free(res); free(e);
    return np;
}

/* ------------------------------------------------------------------ */
/* candidate evaluator                                                  */
/* ------------------------------------------------------------------ */
typedef struct {
    const float* v; int nv; const int* t; int nt;
    const float* planes; int n_planes; int flags;
    float res; int mins; int tot;
    orc_cand_result* out;
    int next; pthread_mutex_t mu;
} eval_ctx;

static void eval_one(eval_ctx* c, int i)
{
    orc_cand_result* r = &c->out[i];
    memset(r, 0, sizeof(*r));
    const float* P = c->planes + 4 * i;
    int cv = c->nv * 2 + 16, ct = c->nt * 3 + 16;
    float* sv[2]; int* st[2];
    for (int s = 0; s < 2; s++) {
        sv[s] = (float*)malloc(sizeof(float) * 3 * (size_t)cv);
        st[s] = (int*)malloc(sizeof(int) * 3 * (size_t)ct);
    }
    int nvs[2], nts[2];
    orc_cut_info info;
    int rc = orc_plane_cut(c->v, c->nv, c->t, c->nt, P[0], P[1], P[2], P[3],
                           sv[0], cv, st[0], ct, sv[1], cv, st[1], ct,
                           &nvs[0], &nts[0], &nvs[1], &nts[1], &info);
    r->n_cap = info.n_cap;
    r->ok = (rc == 0 && nvs[0] > 0 && nvs[1] > 0);
    if (r->ok) {
        for (int s = 0; s < 2; s++) {
            r->nv[s] = nvs[s]; r->nt[s] = nts[s];
            double mv = orc_mesh_signed_volume(sv[s], nvs[s], st[s], nts[s]);
            mv = mv < 0 ? -mv : mv;
            int* hidx = (int*)malloc(sizeof(int) * (size_t)nvs[s]);
            int htcap = 2 * nvs[s] + 8;
            int* htri = (int*)malloc(sizeof(int) * 3 * (size_t)htcap);
            int hnv = 0, hnt = 0; double hvol = 0;
            orc_hull(sv[s], nvs[s], hidx, nvs[s], &hnv, htri, htcap, &hnt, &hvol);
            r->hull_nv[s] = hnv; r->hull_nt[s] = hnt;
            r->mesh_vol[s] = mv; r->hull_vol[s] = hvol;
            double h = 0;
            if ((c->flags & ORC_EVAL_HAUSDORFF) && hnt > 0) {
                float* hv = (float*)malloc(sizeof(float) * 3 * (size_t)(hnv > 0 ? hnv : 1));
                for (int k = 0; k < hnv; k++) memcpy(hv + 3*k, sv[s] + 3*hidx[k], 12);
                h = orc_hausdorff(hv, hnv, htri, hnt, sv[s], nvs[s], st[s], nts[s],
                                  c->res, c->mins, c->tot, 1);
                free(hv);
            }
            r->hausdorff[s] = h;
            r->cost_rv[s] = orc_cost_rv(hvol, mv);
            r->cost_full[s] = orc_cost_full(hvol, mv, h);
            free(hidx); free(htri);
        }
        r->score_rv = r->cost_rv[0] > r->cost_rv[1] ? r->cost_rv[0] : r->cost_rv[1];
        r->score_full = r->cost_full[0] > r->cost_full[1] ? r->cost_full[0] : r->cost_full[1];
    }
    for (int s = 0; s < 2; s++) { free(sv[s]); free(st[s]); }
}

static void* eval_worker(void* arg)
{
    eval_ctx* c = (eval_ctx*)arg;
    for (;;) {
        pthread_mutex_lock(&c->mu);
        int i = c->next++;
        pthread_mutex_unlock(&c->mu);
        if (i >= c->n_planes) break;
        eval_one(c, i);
    }
    return NULL;
}

int orc_eval_candidates(const float* v, int nv, const int* t, int nt,
                        const float* planes, int n_planes, int flags,
                        float hd_resolution, int hd_min_samples,
                        int hd_total_override, int n_threads,
                        orc_cand_result* out)
{
    eval_ctx c;
    c.v = v; c.nv = nv; c.t = t; c.nt = nt; c.planes = planes; c.n_planes = n_planes;
    c.flags = flags; c.res = hd_resolution; c.mins = hd_min_samples; c.tot = hd_total_override;
    c.out = out; c.next = 0;
    pthread_mutex_init(&c.mu, NULL);
    if (n_threads < 1) n_threads = 1;
    if (n_threads > 512) n_threads = 512;
    if (n_threads == 1) eval_worker(&c);
    else {
        pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * (size_t)n_threads);
        for (int k = 0; k < n_threads; k++) pthread_create(&th[k], NULL, eval_worker, &c);
        for (int k = 0; k < n_threads; k++) pthread_join(th[k], NULL);
        free(th);
    }
    pthread_mutex_destroy(&c.mu);
    return 0;
}
