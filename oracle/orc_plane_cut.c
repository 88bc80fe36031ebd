/*
 * orc_plane_cut.c — oracle: mesh/plane cut with cap triangulation.
 * TEST INFRASTRUCTURE ONLY (see cuacd_oracle.h).
 *
 * Restates cuda/plane_cut.cuh:167-1562:
 *   - classify: d = plane(v), sign +1/-1 beyond +-1e-6, else 0 (:270-275);
 *     crossing edges are those whose effective signs differ with 0 counted
 *     as positive (:277-303)
 *   - unique crossing edges in (min,max) order; an edge with exactly one
 *     on-plane endpoint reuses it, otherwise a new vertex n_verts+k is
 *     created at t = d0/(d0-d1) (:536-569)
 *   - triangle split rules, incl. on-plane vertices and coplanar triangles
 *     (:582-652); side triangles are emitted in input-triangle order
 *   - boundary = unmatched edges of the positive side, loops, 2D projection
 *     dropping the largest normal component, CCW orientation, even/odd
 *     nesting, hole bridging and ear clipping (:661-1294), in FP64
 *   - cap failure returns the mesh unsplit on the positive side (:1341-1368)
 *   - per-side vertex compaction in index order and cap winding (:1394-1550)
 *   - n_cross == 0: whole mesh to one side, or per-triangle side split with
 *     first-use vertex order (:330-480)
 * Canonical choices (the reference's are order-nondeterministic): loops start
 * at the smallest unused directed boundary edge; a vertex with several
 * outgoing boundary edges continues along the smallest target.  Boundary
 * edges are sought only among edges whose endpoints both lie on the cut
 * (on-plane or new vertices); for closed input meshes this is the same set.
 */
#include "cuacd_oracle.h"
#include <stdlib.h>
#include <string.h>
#include <math.h>

#define PC_EPS 1e-6f

static float plane_eval(float pa, float pb, float pc, float pd, const float* v)
{
    return fmaf(pa, v[0], fmaf(pb, v[1], fmaf(pc, v[2], pd)));
}

typedef struct { int a, b; } e2;
static int cmp_e2(const void* x, const void* y) {
    const e2* p = (const e2*)x; const e2* q = (const e2*)y;
    if (p->a != q->a) return p->a < q->a ? -1 : 1;
    if (p->b != q->b) return p->b < q->b ? -1 : 1;
    return 0;
}

static int find_edge(const e2* arr, int n, int a, int b)
{
    int lo = 0, hi = n - 1;
    while (lo <= hi) {
        int mid = (lo + hi) >> 1;
        if (arr[mid].a < a || (arr[mid].a == a && arr[mid].b < b)) lo = mid + 1;
        else if (arr[mid].a == a && arr[mid].b == b) return mid;
        else hi = mid - 1;
    }
    return -1;
}

/* ---- FP64 2D helpers for caps ---- */
typedef struct { const float* V; int pu, pv; } cap2d;
static double U(const cap2d* c, int v) { return (double)c->V[3*v + c->pu]; }
static double W(const cap2d* c, int v) { return (double)c->V[3*v + c->pv]; }

static double signed_area(const cap2d* c, const int* poly, int n)
{
    double a = 0.0;
    for (int i = 0; i < n; i++) {
        int j = (i + 1) % n;
        a += U(c, poly[i]) * W(c, poly[j]) - U(c, poly[j]) * W(c, poly[i]);
    }
    return a * 0.5;
}
static void reverse_ints(int* a, int n) {
    for (int i = 0; i < n / 2; i++) { int t = a[i]; a[i] = a[n-1-i]; a[n-1-i] = t; }
}
static double cross2(double ax, double ay, double bx, double by, double cx, double cy) {
    return (bx - ax) * (cy - ay) - (by - ay) * (cx - ax);
}
static int pt_in_tri(double px, double py, double ax, double ay, double bx, double by, double cx, double cy)
{
    double d1 = cross2(ax, ay, bx, by, px, py);
    double d2 = cross2(bx, by, cx, cy, px, py);
    double d3 = cross2(cx, cy, ax, ay, px, py);
    int neg = (d1 < -1e-10) || (d2 < -1e-10) || (d3 < -1e-10);
    int pos = (d1 > 1e-10) || (d2 > 1e-10) || (d3 > 1e-10);
    return !(neg && pos);
}

/* Ear clipping (plane_cut.cuh:1166-1281 logic, FP64).  Returns triangles
 * written, appended to cap[] (3 ints each). */
static int ear_clip(const cap2d* c, const int* poly, int n, int* prv, int* nxt, int* cap)
{
    int nc = 0;
    for (int i = 0; i < n; i++) { prv[i] = (i + n - 1) % n; nxt[i] = (i + 1) % n; }
    int remaining = n, cur = 0, iter = 0;
    while (remaining > 3 && iter < remaining) {
        iter++;
        int p = prv[cur], q = nxt[cur];
        int vp = poly[p], vc = poly[cur], vn = poly[q];
        double up = U(c, vp), wp = W(c, vp), uc = U(c, vc), wc = W(c, vc), un = U(c, vn), wn = W(c, vn);
        double cr = (uc - up) * (wn - wp) - (wc - wp) * (un - up);
        if (cr < -1e-9) { cur = q; continue; }
        if (cr <= 1e-9) {
            cap[3*nc] = vp; cap[3*nc+1] = vc; cap[3*nc+2] = vn; nc++;
            nxt[p] = q; prv[q] = p; remaining--; cur = q; iter = 0;
            continue;
        }
        int ear = 1;
        for (int idx = 0; idx < n && ear; idx++) {
            if (idx == p || idx == cur || idx == q) continue;
            if (nxt[prv[idx]] != idx) continue;
            int vi = poly[idx];
            double cu = U(c, vi), cw = W(c, vi);
            if (fabs(cu - up) + fabs(cw - wp) > 1e-6 &&
                fabs(cu - uc) + fabs(cw - wc) > 1e-6 &&
                fabs(cu - un) + fabs(cw - wn) > 1e-6 &&
                pt_in_tri(cu, cw, up, wp, uc, wc, un, wn)) ear = 0;
        }
        if (ear) {
            cap[3*nc] = vp; cap[3*nc+1] = vc; cap[3*nc+2] = vn; nc++;
            nxt[p] = q; prv[q] = p; remaining--; cur = q; iter = 0;
        } else cur = q;
    }
    if (remaining == 3) {
        int p = prv[cur], q = nxt[cur];
        cap[3*nc] = poly[p]; cap[3*nc+1] = poly[cur]; cap[3*nc+2] = poly[q]; nc++;
    }
    return nc;
}

/* Build the caps from directed boundary edges (sorted by (a,b)).
 * Returns n_cap >= 0, or -1 on cap failure. */
static int build_caps(const float* V, int n_all, const e2* be, int nb,
                      float pa, float pb, float pc, int* cap_out, int* n_loops_out)
{
    *n_loops_out = 0;
    if (nb == 0) return 0;
    cap2d C; C.V = V;
    {
        float ax = fabsf(pa), ay = fabsf(pb), az = fabsf(pc);
        if (ax >= ay && ax >= az) { C.pu = 1; C.pv = 2; }
        else if (ay >= az)        { C.pu = 0; C.pv = 2; }
        else                      { C.pu = 0; C.pv = 1; }
    }
    /* outgoing edge lists: be is sorted by (a,b) so each vertex's edges are contiguous */
    int* used = (int*)calloc((size_t)nb, sizeof(int));
    int* lv = (int*)malloc(sizeof(int) * (size_t)nb);
    int* ls = (int*)malloc(sizeof(int) * (size_t)nb);
    int* lsz = (int*)malloc(sizeof(int) * (size_t)nb);
    int n_loops = 0, lvi = 0, fail = 0;
    for (int st = 0; st < nb && !fail; st++) {
        if (used[st]) continue;
        int first = be[st].a, cur = be[st].b;
        if (first < 0 || first >= n_all || cur < 0 || cur >= n_all) { fail = 1; break; }
        used[st] = 1;
        int start = lvi;
        lv[lvi++] = first;
        int guard = nb + 2;
        while (cur != first && guard-- > 0) {
            if (lvi >= nb) { fail = 1; break; }
            lv[lvi++] = cur;
            /* smallest unused edge leaving cur */
            int lo = 0, hi = nb;   /* lower_bound on a == cur */
            while (lo < hi) { int m = (lo + hi) >> 1; if (be[m].a < cur) lo = m + 1; else hi = m; }
            int found = -1;
            for (int k = lo; k < nb && be[k].a == cur; k++) if (!used[k]) { found = k; break; }
            if (found < 0) { fail = 1; break; }
            used[found] = 1;
            cur = be[found].b;
        }
        if (fail || cur != first) { fail = 1; break; }
        ls[n_loops] = start; lsz[n_loops] = lvi - start; n_loops++;
    }
    *n_loops_out = n_loops;
    if (n_loops > 128) fail = 1;
    int n_cap = 0;
    if (!fail) {
        for (int i = 0; i < n_loops; i++)
            if (signed_area(&C, lv + ls[i], lsz[i]) < 0) reverse_ints(lv + ls[i], lsz[i]);
        int parent[128], is_hole[128];
        for (int i = 0; i < n_loops; i++) { parent[i] = -1; is_hole[i] = 0; }
        for (int i = 0; i < n_loops; i++) {
            if (lsz[i] < 3) continue;
            int vi = lv[ls[i]];
            double pu_ = U(&C, vi), pv_ = W(&C, vi);
            double best_area = 1e300;
            for (int j = 0; j < n_loops; j++) {
                if (j == i || lsz[j] < 3) continue;
                const int* lp = lv + ls[j];
                int m = lsz[j], crossings = 0;
                for (int k = 0; k < m; k++) {
                    int kn = (k + 1) % m;
                    double ay = W(&C, lp[k]), by = W(&C, lp[kn]);
                    if ((ay <= pv_) == (by <= pv_)) continue;
                    double ax = U(&C, lp[k]), bx = U(&C, lp[kn]);
                    double t = (pv_ - ay) / (by - ay);
                    if (ax + t * (bx - ax) > pu_) crossings++;
                }
                if (crossings & 1) {
                    double a = fabs(signed_area(&C, lp, m));
                    if (a < best_area) { best_area = a; parent[i] = j; }
                }
            }
        }
        for (int i = 0; i < n_loops && !fail; i++) {
            int steps = 0;
            for (int p = parent[i]; p >= 0; p = parent[p]) if (++steps > n_loops) { fail = 1; break; }
        }
        if (!fail) {
            for (int i = 0; i < n_loops; i++) {
                int depth = 0;
                for (int p = parent[i]; p >= 0; p = parent[p]) depth++;
                is_hole[i] = depth & 1;
                if (!is_hole[i] && depth >= 2) parent[i] = -1;
            }
            for (int i = 0; i < n_loops; i++) if (is_hole[i]) reverse_ints(lv + ls[i], lsz[i]);
            int poly_cap = nb * 4 + 64;
            int* poly = (int*)malloc(sizeof(int) * (size_t)poly_cap);
            int* tmp = (int*)malloc(sizeof(int) * (size_t)poly_cap * 2);
            int expected = 0;
            for (int oi = 0; oi < n_loops && !fail; oi++) {
                if (is_hole[oi] || lsz[oi] < 3) continue;
                int pn = lsz[oi];
                for (int i = 0; i < pn; i++) poly[i] = lv[ls[oi] + i];
                int hidx[128]; double hmax[128]; int nin = 0;
                for (int i = 0; i < n_loops && nin < 128; i++) {
                    if (parent[i] != oi || lsz[i] < 3) continue;
                    double mu = -1e300;
                    for (int j = 0; j < lsz[i]; j++) { double u = U(&C, lv[ls[i] + j]); if (u > mu) mu = u; }
                    hidx[nin] = i; hmax[nin] = mu; nin++;
                }
                for (int i = 0; i < nin - 1; i++) {
                    int best = i;
                    for (int j = i + 1; j < nin; j++) if (hmax[j] > hmax[best]) best = j;
                    if (best != i) {
                        int ti = hidx[i]; hidx[i] = hidx[best]; hidx[best] = ti;
                        double tf = hmax[i]; hmax[i] = hmax[best]; hmax[best] = tf;
                    }
                }
                for (int ii = 0; ii < nin && !fail; ii++) {
                    int hi = hidx[ii], hs = lsz[hi];
                    const int* hole = lv + ls[hi];
                    int m_idx = 0; double max_u = -1e300;
                    for (int j = 0; j < hs; j++) { double u = U(&C, hole[j]); if (u > max_u) { max_u = u; m_idx = j; } }
                    double mu_ = U(&C, hole[m_idx]), mv_ = W(&C, hole[m_idx]);
                    double best_t = 1e300; int best_edge = -1;
                    for (int j = 0; j < pn; j++) {
                        int jn = (j + 1) % pn;
                        double au = U(&C, poly[j]), av = W(&C, poly[j]);
                        double bu = U(&C, poly[jn]), bv = W(&C, poly[jn]);
                        double dv = bv - av; if (fabs(dv) < 1e-12) continue;
                        double s_ = (mv_ - av) / dv;
                        if (s_ < -1e-12 || s_ > 1.0 + 1e-12) continue;
                        double tv = au + s_ * (bu - au) - mu_;
                        if (tv > 1e-12 && tv < best_t) { best_t = tv; best_edge = j; }
                    }
                    if (best_edge < 0) { fail = 1; break; }
                    int jn = (best_edge + 1) % pn;
                    int p_pos = (U(&C, poly[best_edge]) >= U(&C, poly[jn])) ? best_edge : jn;
                    if (pn + hs + 2 > poly_cap) { fail = 1; break; }
                    int k = 0;
                    for (int j = 0; j <= p_pos; j++) tmp[k++] = poly[j];
                    for (int j = 0; j < hs; j++) tmp[k++] = hole[(m_idx + j) % hs];
                    tmp[k++] = hole[m_idx]; tmp[k++] = poly[p_pos];
                    for (int j = p_pos + 1; j < pn; j++) tmp[k++] = poly[j];
                    for (int j = 0; j < k; j++) poly[j] = tmp[j];
                    pn = k;
                }
                if (fail) break;
                expected += pn - 2;
                if (pn >= 3) n_cap += ear_clip(&C, poly, pn, tmp, tmp + poly_cap, cap_out + 3 * n_cap);
            }
            if (!fail && n_cap < expected) fail = 1;
            free(poly); free(tmp);
        }
    }
    free(used); free(lv); free(ls); free(lsz);
    return fail ? -1 : n_cap;
}

static int copy_whole(const float* verts, int nv, const int* tris, int nt,
                      float* ov, int ovcap, int* ot, int otcap, int* onv, int* ont)
{
    if (nv > ovcap || nt > otcap) return -1;
    memcpy(ov, verts, sizeof(float) * 3 * (size_t)nv);
    memcpy(ot, tris, sizeof(int) * 3 * (size_t)nt);
    *onv = nv; *ont = nt;
    return 0;
}

int orc_plane_cut(const float* verts, int nv, const int* tris, int nt,
                  float pa, float pb, float pc, float pd,
                  float* pos_v, int pos_v_cap, int* pos_t, int pos_t_cap,
                  float* neg_v, int neg_v_cap, int* neg_t, int neg_t_cap,
                  int* n_pv, int* n_pt, int* n_nv, int* n_nt,
                  orc_cut_info* info)
{
    orc_cut_info dummy; if (!info) info = &dummy;
    memset(info, 0, sizeof(*info));
    *n_pv = *n_pt = *n_nv = *n_nt = 0;
    signed char* sg = (signed char*)malloc((size_t)(nv > 0 ? nv : 1));
    for (int v = 0; v < nv; v++) {
        float d = plane_eval(pa, pb, pc, pd, verts + 3*v);
        sg[v] = (d > PC_EPS) ? 1 : ((d < -PC_EPS) ? -1 : 0);
    }
    /* crossing edges */
    e2* ce = (e2*)malloc(sizeof(e2) * (size_t)(3 * nt > 0 ? 3 * nt : 1));
    int nce = 0;
    for (int t = 0; t < nt; t++) {
        for (int e = 0; e < 3; e++) {
            int va = tris[3*t+e], vb = tris[3*t+(e+1)%3];
            int ea = sg[va] >= 0 ? 1 : -1, eb = sg[vb] >= 0 ? 1 : -1;
            if (ea != eb) { ce[nce].a = va < vb ? va : vb; ce[nce].b = va < vb ? vb : va; nce++; }
        }
    }
    int rc = 0;
    if (nce == 0) {
        int any_pos = 0, any_neg = 0;
        for (int v = 0; v < nv; v++) { if (sg[v] > 0) any_pos = 1; if (sg[v] < 0) any_neg = 1; }
        if (!any_pos || !any_neg) {
            if (any_neg && !any_pos) rc = copy_whole(verts, nv, tris, nt, neg_v, neg_v_cap, neg_t, neg_t_cap, n_nv, n_nt);
            else rc = copy_whole(verts, nv, tris, nt, pos_v, pos_v_cap, pos_t, pos_t_cap, n_pv, n_pt);
            info->n_pos_tris = *n_pt; info->n_neg_tris = *n_nt;
        } else {
            int* vmap = (int*)malloc(sizeof(int) * (size_t)nv);
            for (int side = 0; side < 2 && rc == 0; side++) {
                float* ov = side == 0 ? pos_v : neg_v; int* ot = side == 0 ? pos_t : neg_t;
                int ovc = side == 0 ? pos_v_cap : neg_v_cap, otc = side == 0 ? pos_t_cap : neg_t_cap;
                for (int v = 0; v < nv; v++) vmap[v] = -1;
                int cnv = 0, cnt = 0;
                for (int t = 0; t < nt; t++) {
                    int i0 = tris[3*t], i1 = tris[3*t+1], i2 = tris[3*t+2];
                    int isneg = sg[i0] < 0 || sg[i1] < 0 || sg[i2] < 0;
                    if (isneg != side) continue;
                    int ii[3] = {i0, i1, i2};
                    for (int k = 0; k < 3; k++) if (vmap[ii[k]] < 0) vmap[ii[k]] = cnv++;
                    if (cnt >= otc) { rc = -1; break; }
                    for (int k = 0; k < 3; k++) ot[3*cnt+k] = vmap[ii[k]];
                    cnt++;
                }
                if (rc) break;
                if (cnv > ovc) { rc = -1; break; }
                for (int v = 0; v < nv; v++) if (vmap[v] >= 0) memcpy(ov + 3*vmap[v], verts + 3*v, 12);
                if (side == 0) { *n_pv = cnv; *n_pt = cnt; } else { *n_nv = cnv; *n_nt = cnt; }
            }
            free(vmap);
            info->n_pos_tris = *n_pt; info->n_neg_tris = *n_nt;
        }
        free(ce); free(sg);
        return rc;
    }
    qsort(ce, (size_t)nce, sizeof(e2), cmp_e2);
    int nu = 0;
    for (int i = 0; i < nce; i++) if (i == 0 || cmp_e2(&ce[i], &ce[i-1]) != 0) ce[nu++] = ce[i];
    info->n_cross = nu;
    int n_all = nv;
    int* isect = (int*)malloc(sizeof(int) * (size_t)nu);
    float* all = (float*)malloc(sizeof(float) * 3 * (size_t)(nv + nu));
    memcpy(all, verts, sizeof(float) * 3 * (size_t)nv);
    for (int i = 0; i < nu; i++) {
        int va = ce[i].a, vb = ce[i].b;
        float d0 = plane_eval(pa, pb, pc, pd, verts + 3*va);
        float d1 = plane_eval(pa, pb, pc, pd, verts + 3*vb);
        if (fabsf(d0) <= PC_EPS && fabsf(d1) > PC_EPS) isect[i] = va;
        else if (fabsf(d1) <= PC_EPS && fabsf(d0) > PC_EPS) isect[i] = vb;
        else {
            float t = d0 / (d0 - d1);
            for (int k = 0; k < 3; k++)
                all[3*n_all+k] = fmaf(t, verts[3*vb+k] - verts[3*va+k], verts[3*va+k]);
            isect[i] = n_all++;
        }
    }
    /* split triangles, input order */
    int cap_t = 2 * nt + 8;
    int* pt_ = (int*)malloc(sizeof(int) * 3 * (size_t)cap_t);
    int* nt_ = (int*)malloc(sizeof(int) * 3 * (size_t)cap_t);
    int np = 0, nn = 0;
#define EMIT(arr, cnt, x, y, z) do { arr[3*cnt] = (x); arr[3*cnt+1] = (y); arr[3*cnt+2] = (z); cnt++; } while (0)
#define ISECT(u, w) ({ int _m = (u) < (w) ? (u) : (w), _x = (u) < (w) ? (w) : (u); \
                      int _f = find_edge(ce, nu, _m, _x); _f >= 0 ? isect[_f] : -1; })
    for (int t = 0; t < nt; t++) {
        int i0 = tris[3*t], i1 = tris[3*t+1], i2 = tris[3*t+2];
        int s0 = sg[i0], s1 = sg[i1], s2 = sg[i2];
        int hp = s0 > 0 || s1 > 0 || s2 > 0, hn = s0 < 0 || s1 < 0 || s2 < 0;
        if (!hp || !hn) {
            if (hn) EMIT(nt_, nn, i0, i1, i2);
            else if (hp) EMIT(pt_, np, i0, i1, i2);
            else {
                float e1x = all[3*i1] - all[3*i0], e1y = all[3*i1+1] - all[3*i0+1], e1z = all[3*i1+2] - all[3*i0+2];
                float e2x = all[3*i2] - all[3*i0], e2y = all[3*i2+1] - all[3*i0+1], e2z = all[3*i2+2] - all[3*i0+2];
                double dot = (double)pa * ((double)e1y*e2z - (double)e1z*e2y)
                           + (double)pb * ((double)e1z*e2x - (double)e1x*e2z)
                           + (double)pc * ((double)e1x*e2y - (double)e1y*e2x);
                if (dot > 0) EMIT(pt_, np, i0, i1, i2); else EMIT(nt_, nn, i0, i1, i2);
            }
            continue;
        }
        int vi[3] = {i0, i1, i2}, si[3] = {s0, s1, s2};
        int on = -1;
        for (int k = 0; k < 3; k++) if (si[k] == 0) { on = k; break; }
        if (on >= 0) {
            int ov = vi[on], a_i = vi[(on+1)%3], b_i = vi[(on+2)%3], sa = si[(on+1)%3], sb = si[(on+2)%3];
            if (sa == sb) {
                if (sa > 0) EMIT(pt_, np, i0, i1, i2); else EMIT(nt_, nn, i0, i1, i2);
            } else {
                int nvi = ISECT(a_i, b_i);
                if (nvi < 0) continue;
                if (sa > 0) { EMIT(pt_, np, ov, a_i, nvi); EMIT(nt_, nn, ov, nvi, b_i); }
                else        { EMIT(nt_, nn, ov, a_i, nvi); EMIT(pt_, np, ov, nvi, b_i); }
            }
        } else {
            int lone = -1;
            for (int k = 0; k < 3; k++) if (si[k] != si[(k+1)%3] && si[k] != si[(k+2)%3]) { lone = k; break; }
            if (lone < 0) continue;
            int lv = vi[lone], ov1 = vi[(lone+1)%3], ov2 = vi[(lone+2)%3], ls = si[lone];
            int nv1 = ISECT(lv, ov1), nv2 = ISECT(lv, ov2);
            if (nv1 < 0 || nv2 < 0) continue;
            if (ls > 0) {
                EMIT(pt_, np, lv, nv1, nv2);
                EMIT(nt_, nn, ov1, nv2, nv1); EMIT(nt_, nn, ov1, ov2, nv2);
            } else {
                EMIT(nt_, nn, lv, nv1, nv2);
                EMIT(pt_, np, ov1, nv2, nv1); EMIT(pt_, np, ov1, ov2, nv2);
            }
        }
    }
#undef ISECT
    info->n_pos_tris = np; info->n_neg_tris = nn;
    /* boundary of the positive side among edges on the cut */
    signed char* oncut = (signed char*)calloc((size_t)n_all, 1);
    for (int v = 0; v < nv; v++) if (sg[v] == 0) oncut[v] = 1;
    for (int v = nv; v < n_all; v++) oncut[v] = 1;
    e2* de = (e2*)malloc(sizeof(e2) * (size_t)(3 * np + 1));
    int nde = 0;
    for (int t = 0; t < np; t++)
        for (int e = 0; e < 3; e++) {
            int a = pt_[3*t+e], b = pt_[3*t+(e+1)%3];
            if (oncut[a] && oncut[b]) { de[nde].a = a; de[nde].b = b; nde++; }
        }
    /* unordered-key grouping: a directed edge is boundary iff its key occurs once */
    e2* key = (e2*)malloc(sizeof(e2) * (size_t)(nde + 1));
    for (int i = 0; i < nde; i++) {
        key[i].a = de[i].a < de[i].b ? de[i].a : de[i].b;
        key[i].b = de[i].a < de[i].b ? de[i].b : de[i].a;
    }
    qsort(key, (size_t)nde, sizeof(e2), cmp_e2);
    e2* be = (e2*)malloc(sizeof(e2) * (size_t)(nde + 1));
    int nb = 0;
    for (int i = 0; i < nde; i++) {
        int lo = de[i].a < de[i].b ? de[i].a : de[i].b, hi = de[i].a < de[i].b ? de[i].b : de[i].a;
        int f = find_edge(key, nde, lo, hi);
        /* count occurrences around f */
        int c = 1;
        if (f > 0 && key[f-1].a == lo && key[f-1].b == hi) c++;
        if (f + 1 < nde && key[f+1].a == lo && key[f+1].b == hi) c++;
        if (c == 1) be[nb++] = de[i];
    }
    qsort(be, (size_t)nb, sizeof(e2), cmp_e2);
    info->n_boundary = nb;
    int* cap = (int*)malloc(sizeof(int) * 3 * (size_t)(nb * 4 + 64));
    int n_loops = 0;
    int n_cap = build_caps(all, n_all, be, nb, pa, pb, pc, cap, &n_loops);
    info->n_loops = n_loops;
    if (n_cap < 0) {
        info->cap_failed = 1;
        rc = copy_whole(verts, nv, tris, nt, pos_v, pos_v_cap, pos_t, pos_t_cap, n_pv, n_pt);
    } else {
        info->n_cap = n_cap;
        int flip;
        {
            float ax = fabsf(pa), ay = fabsf(pb), az = fabsf(pc);
            float n2d[3] = {0, 0, 0};
            if (ax >= ay && ax >= az) n2d[0] = 1.0f;          /* (pu,pv) = (1,2) */
            else if (ay >= az)        n2d[1] = -1.0f;         /* (0,2) */
            else                      n2d[2] = 1.0f;          /* (0,1) */
            flip = (n2d[0]*(-pa) + n2d[1]*(-pb) + n2d[2]*(-pc) < 0) ? 1 : 0;
        }
        int* remap = (int*)malloc(sizeof(int) * (size_t)n_all);
        for (int side = 0; side < 2 && rc == 0; side++) {
            const int* st = side == 0 ? pt_ : nt_; int ns = side == 0 ? np : nn;
            float* ov = side == 0 ? pos_v : neg_v; int* ot = side == 0 ? pos_t : neg_t;
            int ovc = side == 0 ? pos_v_cap : neg_v_cap, otc = side == 0 ? pos_t_cap : neg_t_cap;
            for (int v = 0; v < n_all; v++) remap[v] = -1;
            for (int i = 0; i < 3 * ns; i++) remap[st[i]] = 0;
            for (int i = 0; i < 3 * n_cap; i++) remap[cap[i]] = 0;
            int cnv = 0;
            for (int v = 0; v < n_all; v++) if (remap[v] == 0) remap[v] = cnv++;
            if (cnv > ovc || ns + n_cap > otc) { rc = -1; break; }
            for (int v = 0; v < n_all; v++) if (remap[v] >= 0) memcpy(ov + 3*remap[v], all + 3*v, 12);
            for (int i = 0; i < 3 * ns; i++) ot[i] = remap[st[i]];
            for (int t = 0; t < n_cap; t++) {
                int v0 = cap[3*t], v1 = cap[3*t+1], v2 = cap[3*t+2];
                int o = 3 * (ns + t);
                ot[o] = remap[v0];
                if (side == 0) { ot[o+1] = flip ? remap[v2] : remap[v1]; ot[o+2] = flip ? remap[v1] : remap[v2]; }
                else           { ot[o+1] = flip ? remap[v1] : remap[v2]; ot[o+2] = flip ? remap[v2] : remap[v1]; }
            }
            if (side == 0) { *n_pv = cnv; *n_pt = ns + n_cap; } else { *n_nv = cnv; *n_nt = ns + n_cap; }
        }
        free(remap);
    }
#undef EMIT
    free(cap); free(be); free(key); free(de); free(oncut);
    free(pt_); free(nt_); free(all); free(isect); free(ce); free(sg);
    return rc;
}
