/*
 * orc_components.c — connected components of a triangle mesh.
 * TEST INFRASTRUCTURE ONLY (see cuacd_oracle.h).
 *
 * Restates decompose_components_block (cuda/postprocess.cuh:139-527):
 * vertices joined by a triangle are in one component (union-find,
 * postprocess.cuh:215-238); components are numbered in order of their
 * smallest vertex (sequential numbering, postprocess.cuh:258-270); each
 * component's signed volume decides whether it is an unreachable inner shell
 * (negative), and inner shells are dropped when outer shells exist too
 * (postprocess.cuh:449-495).  Canonical order (the reference's is arbitrary
 * inside a component): vertices and triangles keep their input order.
 * Vertices used by no triangle belong to no component.
 */
#include <stdlib.h>
#include "cuacd_oracle.h"

static int uf_find(int* p, int x)
{
    while (p[x] != x) { p[x] = p[p[x]]; x = p[x]; }
    return x;
}

int orc_components(const float* v, int nv, const int* t, int nt, int max_comp, int max_out_v, int max_out_t,
                   float* out_v, int* out_t, int* comp_nv, int* comp_nt, double* comp_vol)
{
    if (nv <= 0 || nt <= 0) return 0;
    int* parent = (int*)malloc(sizeof(int) * nv);
    int* cid = (int*)malloc(sizeof(int) * nv);
    int* local = (int*)malloc(sizeof(int) * nv);
    int* used = (int*)calloc((size_t)nv, sizeof(int));
    int* root_id = (int*)malloc(sizeof(int) * nv);
    int* vstart = NULL;
    int* tstart = NULL;
    int rc = 0;
    for (int i = 0; i < nv; i++) { parent[i] = i; cid[i] = -1; root_id[i] = -1; }
    for (int i = 0; i < nt; i++) {
        for (int k = 1; k < 3; k++) {
            int a = uf_find(parent, t[3 * i]), b = uf_find(parent, t[3 * i + k]);
            if (a == b) continue;
            if (a < b) parent[b] = a; else parent[a] = b;
        }
    }
    /* component numbers in order of the smallest used vertex */
    for (int i = 0; i < 3 * nt; i++) used[t[i]] = 1;
    int C = 0;
    for (int i = 0; i < nv; i++) {
        if (!used[i]) continue;
        int r = uf_find(parent, i);
        if (root_id[r] < 0) root_id[r] = C++;
        cid[i] = root_id[r];
    }
    if (C <= 1 || C > 4096) { rc = 0; goto done; }
    if (C > max_comp) { rc = -1; goto done; }
    vstart = (int*)calloc((size_t)C + 1, sizeof(int));
    tstart = (int*)calloc((size_t)C + 1, sizeof(int));
    for (int i = 0; i < nv; i++) if (cid[i] >= 0) vstart[cid[i] + 1]++;
    for (int i = 0; i < nt; i++) tstart[cid[t[3 * i]] + 1]++;
    for (int c = 0; c < C; c++) { vstart[c + 1] += vstart[c]; tstart[c + 1] += tstart[c]; }
    if (vstart[C] > max_out_v || tstart[C] > max_out_t) { rc = -1; goto done; }
    {
        int* vf = (int*)calloc((size_t)C, sizeof(int));
        int* tf = (int*)calloc((size_t)C, sizeof(int));
        for (int i = 0; i < nv; i++) {
            int c = cid[i];
            if (c < 0) continue;
            int p = vstart[c] + vf[c]++;
            local[i] = p - vstart[c];
            out_v[3 * p] = v[3 * i]; out_v[3 * p + 1] = v[3 * i + 1]; out_v[3 * p + 2] = v[3 * i + 2];
        }
        for (int i = 0; i < nt; i++) {
            int c = cid[t[3 * i]];
            int p = tstart[c] + tf[c]++;
            for (int k = 0; k < 3; k++) out_t[3 * p + k] = local[t[3 * i + k]];
        }
        free(vf); free(tf);
    }
    {
        int n_inner = 0;
        double* vol = (double*)malloc(sizeof(double) * C);
        for (int c = 0; c < C; c++) {
            vol[c] = orc_mesh_signed_volume(out_v + 3 * (size_t)vstart[c], vstart[c + 1] - vstart[c],
                                            out_t + 3 * (size_t)tstart[c], tstart[c + 1] - tstart[c]);
            n_inner += vol[c] < 0.0;
        }
        int drop = n_inner > 0 && n_inner < C;
        /* compact in place (components only move towards the front) */
        int k = 0, vo = 0, to = 0;
        for (int c = 0; c < C; c++) {
            int cnv = vstart[c + 1] - vstart[c], cnt = tstart[c + 1] - tstart[c];
            if (drop && vol[c] < 0.0) continue;
            if (vo != vstart[c]) for (int i = 0; i < 3 * cnv; i++) out_v[3 * vo + i] = out_v[3 * vstart[c] + i];
            if (to != tstart[c]) for (int i = 0; i < 3 * cnt; i++) out_t[3 * to + i] = out_t[3 * tstart[c] + i];
            comp_nv[k] = cnv; comp_nt[k] = cnt; comp_vol[k] = vol[c] < 0 ? -vol[c] : vol[c];
            vo += cnv; to += cnt; k++;
        }
        free(vol);
        rc = k;
    }
done:
    free(parent); free(cid); free(local); free(used); free(root_id); free(vstart); free(tstart);
    return rc;
}
