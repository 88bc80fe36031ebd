// remesh.cuh — remesh front end (Context.preprocess / gpu_preprocess): the
// per-item work of every kernel in remesh.cu, as __host__ __device__
// functions so that a host build can run the same arithmetic (the CPU
// emulation test).  Replaces the reference's PaMO stage
// (csrc/preprocess.c:605-700, cuda/c2s_kernels.cu, cuda/pdmc_kernels.cu):
//   normalise   p_norm = ((p - vmin) / extent + band) / margin, band = 3/R,
//               margin = 1 + 2 band; grid units u = p_norm R - 0.5 (node g
//               samples p_norm = (g + 0.5) / R, csrc/preprocess.c:686-696)
//   distance    squared distance of every node within 3 cells of a
//               triangle (float32, least over triangles)
//   crossings   grid edges (node, node + e_k) that a triangle crosses
//   sign        nodes reachable from the grid's boundary through uncrossed
//               edges are outside (axis sweeps until nothing changes)
//   field       (outside ? d : -d) - 0.9 cells (csrc/preprocess.c:669-676)
//   contour     marching cubes with a generated case table: one vertex per
//               crossed grid edge, loops of three as triangles, longer
//               loops fanned around their mean
// All FP64 and in a fixed order; remesh.cu is built with -fmad=false.
#pragma once
#include <math.h>

#ifdef __CUDACC__
#define RM_HD __host__ __device__ __forceinline__
#else
#define RM_HD inline
#endif

#define RM_BAND   3.0          // cells of the distance band
#define RM_SHIFT  0.9          // cells the surface moves out
#define RM_TCLAMP 0.01         // edge parameter kept in [0.01, 0.99]
#define RM_FAR    0x7f7fffffu  // FLT_MAX bits: no triangle within the band
#define RM_MAXLOOP 4           // loops of one case (generated table: at most 4)
#define RM_MAXEDGE 12

struct RmParams {
    int R;
    float vmin[3];
    float extent;
    double band, margin;
};

// Marching-cubes loops per case (built on the host by rm_build_table).
struct RmTable {
    unsigned char nloop[256];
    unsigned char len[256][RM_MAXLOOP];
    signed char edge[256][RM_MAXEDGE];      // loops one after another
    unsigned char ntri[256], nctr[256];     // triangles, centre vertices
};

// cube corner c: (c & 1, c >> 1 & 1, c >> 2 & 1); edge e from corner
// RM_E0[e] along axis RM_EAX[e]
RM_HD int rm_e0(int e) { return e < 4 ? 2 * e : (e < 8 ? ((e - 4) & 1) | (((e - 4) >> 1) << 2) : e - 8); }
RM_HD int rm_eax(int e) { return e >> 2; }

RM_HD long long rm_lin(int x, int y, int z, int R) { return ((long long)z * R + y) * R + x; }

RM_HD double rm_dot(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
RM_HD void rm_cross(const double* a, const double* b, double* o)
{
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}
RM_HD void rm_sub(const double* a, const double* b, double* o) { o[0] = a[0] - b[0]; o[1] = a[1] - b[1]; o[2] = a[2] - b[2]; }

// grid units of one input coordinate
RM_HD double rm_norm(float p, int k, const RmParams& P)
{
    return (((double)p - (double)P.vmin[k]) / (double)P.extent + P.band) / P.margin * (double)P.R - 0.5;
}

// output coordinate of a grid-unit coordinate
RM_HD float rm_denorm(double g, int k, const RmParams& P)
{
    return (float)(((g + 0.5) / (double)P.R * P.margin - P.band) * (double)P.extent + (double)P.vmin[k]);
}

RM_HD double rm_seg_d2(const double* p, const double* a, const double* b)
{
    double ab[3], pa[3];
    rm_sub(b, a, ab);
    rm_sub(p, a, pa);
    const double ll = rm_dot(ab, ab);
    double t = ll > 0 ? rm_dot(pa, ab) / ll : 0.0;
    t = fmin(fmax(t, 0.0), 1.0);
    double d[3];
    for (int k = 0; k < 3; k++) d[k] = p[k] - (a[k] + t * ab[k]);
    return rm_dot(d, d);
}

// squared distance from node p to triangle abc
RM_HD double rm_point_tri_d2(const double* p, const double* a, const double* b, const double* c)
{
    double ab[3], bc[3], ca[3], ac[3], n[3];
    rm_sub(b, a, ab); rm_sub(c, b, bc); rm_sub(a, c, ca); rm_sub(c, a, ac);
    rm_cross(ab, ac, n);
    const double nn = rm_dot(n, n);
    double d2 = fmin(fmin(rm_seg_d2(p, a, b), rm_seg_d2(p, b, c)), rm_seg_d2(p, c, a));
    if (nn > 0) {
        double pa[3], pb[3], pc[3], x[3];
        rm_sub(p, a, pa); rm_sub(p, b, pb); rm_sub(p, c, pc);
        rm_cross(ab, pa, x); const double s0 = rm_dot(x, n);
        rm_cross(bc, pb, x); const double s1 = rm_dot(x, n);
        rm_cross(ca, pc, x); const double s2 = rm_dot(x, n);
        if (s0 >= 0 && s1 >= 0 && s2 >= 0) {
            const double dp = rm_dot(pa, n);
            d2 = fmin(d2, dp * dp / nn);
        }
    }
    return d2;
}

// node box of a triangle's distance band: lo[k] .. hi[k] (empty when any hi < lo)
RM_HD void rm_tri_box(const double* a, const double* b, const double* c, int R, int* lo, int* hi)
{
    for (int k = 0; k < 3; k++) {
        const double mn = fmin(fmin(a[k], b[k]), c[k]), mx = fmax(fmax(a[k], b[k]), c[k]);
        const double l = ceil(mn - RM_BAND), h = floor(mx + RM_BAND);
        lo[k] = l < 0 ? 0 : (l > R ? R : (int)l);
        hi[k] = h > R - 1 ? R - 1 : (h < -1 ? -1 : (int)h);
    }
}

RM_HD double rm_orient(const double* X, const double* Y, double pi, double pj, int i, int j)
{
    return (Y[i] - X[i]) * (pj - X[j]) - (Y[j] - X[j]) * (pi - X[i]);
}

// twice the signed area of the triangle's projection along axis k; lines
// along k do not cross a triangle whose projection is a segment
RM_HD double rm_tri_area2(const double* A, const double* B, const double* C, int k)
{
    const int i = (k + 1) % 3, j = (k + 2) % 3;
    return rm_orient(A, B, C[i], C[j], i, j);
}

// the line through integer (a, b) on axes (i, j) = ((k+1)%3, (k+2)%3):
// the node whose edge along k it crosses, or -1
RM_HD long long rm_line_cross(const double* A, const double* B, const double* C, int k, int a, int b, int R)
{
    const int i = (k + 1) % 3, j = (k + 2) % 3;
    const double pa = (double)a, pb = (double)b;
    const double w0 = rm_orient(B, C, pa, pb, i, j);
    const double w1 = rm_orient(C, A, pa, pb, i, j);
    const double w2 = rm_orient(A, B, pa, pb, i, j);
    const double ws = w0 + w1 + w2;
    const bool hit = ((w0 >= 0 && w1 >= 0 && w2 >= 0) || (w0 <= 0 && w1 <= 0 && w2 <= 0)) && ws != 0;
    if (!hit) return -1;
    const double z = floor((w0 * A[k] + w1 * B[k] + w2 * C[k]) / ws);
    if (!(z >= 0 && z <= (double)(R - 2))) return -1;
    int q[3];
    q[k] = (int)z; q[i] = a; q[j] = b;
    return rm_lin(q[0], q[1], q[2], R);
}

// line range of a triangle's projection on axes i, j (empty when hi < lo)
RM_HD void rm_tri_lines(const double* A, const double* B, const double* C, int k, int R, int* lo, int* hi)
{
    const int ax[2] = {(k + 1) % 3, (k + 2) % 3};
    for (int m = 0; m < 2; m++) {
        const int i = ax[m];
        const double l = ceil(fmin(fmin(A[i], B[i]), C[i])), h = floor(fmax(fmax(A[i], B[i]), C[i]));
        lo[m] = l < 0 ? 0 : (l > R ? R : (int)l);
        hi[m] = h > R - 1 ? R - 1 : (h < -1 ? -1 : (int)h);
    }
}

RM_HD float rm_field(unsigned d2bits, bool outside)
{
    float d2f;
#ifdef __CUDA_ARCH__
    d2f = __uint_as_float(d2bits);
#else
    __builtin_memcpy(&d2f, &d2bits, 4);
#endif
    const double u = d2bits == RM_FAR ? 1e9 : sqrt((double)d2f);
    return (float)((outside ? u : -u) - RM_SHIFT);
}

// grid-unit position of the vertex on edge (node n = (x, y, z), axis k)
RM_HD void rm_edge_pos(const float* sd, int x, int y, int z, int k, int R, double* g)
{
    int q[3] = {x, y, z};
    q[k] += 1;
    const double s0 = (double)sd[rm_lin(x, y, z, R)], s1 = (double)sd[rm_lin(q[0], q[1], q[2], R)];
    double t = s0 / (s0 - s1);
    t = fmin(fmax(t, RM_TCLAMP), 1.0 - RM_TCLAMP);
    g[0] = (double)x; g[1] = (double)y; g[2] = (double)z;
    g[k] = g[k] + t;
}

RM_HD int rm_case(const float* sd, int x, int y, int z, int R)
{
    int c = 0;
    for (int q = 0; q < 8; q++)
        if (sd[rm_lin(x + (q & 1), y + (q >> 1 & 1), z + (q >> 2 & 1), R)] < 0.0f) c |= 1 << q;
    return c;
}

// global edge id (3 * node + axis) of cube edge e of the cell at (x, y, z)
RM_HD long long rm_cell_edge(int e, int x, int y, int z, int R)
{
    const int c0 = rm_e0(e);
    return 3 * rm_lin(x + (c0 & 1), y + (c0 >> 1 & 1), z + (c0 >> 2 & 1), R) + rm_eax(e);
}

// Triangles and centre vertices of one cell: vid[] holds the scanned vertex
// id of every crossed grid edge; tri_base / ctr_base are the cell's first
// triangle and first centre (centres are numbered after the edge vertices).
RM_HD void rm_cell_emit(const RmTable& T, const float* sd, const int* vid, int x, int y, int z, int R,
                        const RmParams& P, int n_edge_verts, int tri_base, int ctr_base, float* out_v, int* out_t)
{
    const int cs = rm_case(sd, x, y, z, R);
    int off = 0, tri = tri_base, ctr = ctr_base;
    for (int l = 0; l < T.nloop[cs]; l++) {
        const int L = T.len[cs][l];
        int v[RM_MAXEDGE];
        for (int m = 0; m < L; m++) v[m] = vid[rm_cell_edge(T.edge[cs][off + m], x, y, z, R)];
        if (L == 3) {
            out_t[3 * tri] = v[0]; out_t[3 * tri + 1] = v[1]; out_t[3 * tri + 2] = v[2];
            tri++;
        } else {
            double s[3] = {0.0, 0.0, 0.0};
            for (int m = 0; m < L; m++) {
                const int e = T.edge[cs][off + m], c0 = rm_e0(e);
                double g[3];
                rm_edge_pos(sd, x + (c0 & 1), y + (c0 >> 1 & 1), z + (c0 >> 2 & 1), rm_eax(e), R, g);
                s[0] += g[0]; s[1] += g[1]; s[2] += g[2];
            }
            const int cv = n_edge_verts + ctr;
            for (int k = 0; k < 3; k++) out_v[3 * (long long)cv + k] = rm_denorm(s[k] / (double)L, k, P);
            for (int m = 0; m < L; m++) {
                out_t[3 * tri] = cv; out_t[3 * tri + 1] = v[m]; out_t[3 * tri + 2] = v[(m + 1) % L];
                tri++;
            }
            ctr++;
        }
        off += L;
    }
}

// The case table from its rule (host): on each face, a segment from every
// edge where the counter-clockwise cycle (seen from outside) passes from an
// inside corner to an outside one, back to the edge that opened that run of
// inside corners -- two diagonal inside corners on a face get one segment
// each, so the inside is 6-connected and neighbouring cells agree on every
// face.  The segments close into loops; each loop is reversed (normals then
// point from inside to outside) and starts at its first edge.
inline int rm_edge_of(int c0, int c1)
{
    const int lo = c0 < c1 ? c0 : c1, hi = c0 < c1 ? c1 : c0;
    for (int e = 0; e < 12; e++)
        if (rm_e0(e) == lo && (lo | (1 << rm_eax(e))) == hi) return e;
    return -1;
}

inline void rm_build_table(RmTable& T)
{
    int cyc[6][4];
    int f = 0;
    for (int a = 0; a < 3; a++) {
        const int b = (a + 1) % 3, c = (a + 2) % 3;
        for (int s = 0; s < 2; s++, f++) {
            const int pb[4] = {0, 1, 1, 0}, pc[4] = {0, 0, 1, 1};
            for (int i = 0; i < 4; i++) {
                const int q = (s << a) | (pb[i] << b) | (pc[i] << c);
                cyc[f][s ? i : 3 - i] = q;
            }
        }
    }
    for (int cs = 0; cs < 256; cs++) {
        int nxt[12];
        for (int e = 0; e < 12; e++) nxt[e] = -1;
        for (int fc = 0; fc < 6; fc++) {
            bool st[4];
            for (int i = 0; i < 4; i++) st[i] = cs >> cyc[fc][i] & 1;
            for (int i = 0; i < 4; i++) {
                if (!(st[i] && !st[(i + 1) % 4])) continue;
                int j = i;
                while (st[j]) j = (j + 3) % 4;
                nxt[rm_edge_of(cyc[fc][i], cyc[fc][(i + 1) % 4])] = rm_edge_of(cyc[fc][j], cyc[fc][(j + 1) % 4]);
            }
        }
        bool seen[12] = {false};
        int nl = 0, off = 0, ntri = 0, nctr = 0;
        for (int e = 0; e < 12; e++) {
            if (nxt[e] < 0 || seen[e]) continue;
            int loop[12], L = 0;
            loop[L++] = e; seen[e] = true;
            for (int g = nxt[e]; g != e; g = nxt[g]) { loop[L++] = g; seen[g] = true; }
            T.edge[cs][off] = (signed char)loop[0];
            for (int m = 1; m < L; m++) T.edge[cs][off + m] = (signed char)loop[L - m];
            T.len[cs][nl++] = (unsigned char)L;
            off += L;
            if (L == 3) ntri += 1; else { ntri += L; nctr += 1; }
        }
        for (int m = off; m < RM_MAXEDGE; m++) T.edge[cs][m] = -1;
        for (int l = nl; l < RM_MAXLOOP; l++) T.len[cs][l] = 0;
        T.nloop[cs] = (unsigned char)nl;
        T.ntri[cs] = (unsigned char)ntri;
        T.nctr[cs] = (unsigned char)nctr;
    }
}
