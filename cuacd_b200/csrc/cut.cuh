// cut.cuh — mesh/plane cut with cap triangulation, one CTA per cut (sm_100a).
//
// Replaces plane_cut_block (cuda/plane_cut.cuh:167-1562; 64 threads, ~15
// locked heap allocations, thread-0 serial phases).  Here:
//   classify (:270-275)         one pass over the vertices, all threads
//   crossing edges (:277-303)   per-triangle ballot compaction, CTA bitonic
//                               sort + dedup of 64-bit edge keys
//   new vertices (:536-569)     exclusive scan over the unique edges; an edge
//                               with one on-plane end reuses that vertex
//   split (:582-652)            per-triangle piece counts, exclusive scan,
//                               pieces written in input-triangle order
//   boundary (:661-811)         unmatched edges of the positive side among
//                               edges whose ends both lie on the cut, found
//                               by sorting (min,max,dir) keys
//   caps (:893-1294)            loops (smallest unused edge first), FP64
//                               orientation, even/odd nesting, hole bridging
//                               and ear clipping with a warp-parallel
//                               point-in-triangle scan
//   failure (:1341-1368)        the mesh is returned unsplit on the + side
//   output (:1394-1550)         per-side vertex compaction in index order,
//                               cap winding rule
// Every scratch buffer is bump-allocated from the arena once its size is
// known; nothing waits on a lock.  This translation unit is compiled with
// -fmad=false: the FP32 and FP64 expressions round exactly as written (the
// checker evaluates the same sequence), and every fused multiply-add that is
// wanted is spelled fmaf().
#pragma once
#include "common.cuh"
#include "cta_util.cuh"

#define CUT_NT  512
#define CUT_EPS 1e-6f

struct CutResult {
    float* pv; int* pt; int npv, npt;      // positive side (caps included)
    float* nv; int* nt; int nnv, nnt;      // negative side
    int n_pos_tris, n_neg_tris;            // before caps
    int n_cap, n_loops, n_boundary, cap_failed, n_cross;
    int err;
    int flags;                             // CUT_FLAG_* (set by callers that skip the cut)
    int _pad;
    unsigned cyc[4];                       // SM cycles / 64: crossings, split, boundary, caps + output
};

#define CUT_FLAG_SMALL   1    // the part is too small on every axis to be cut
#define CUT_FLAG_NOPLANE 2    // no valid plane: nothing was cut

struct CutFixedOut {          // caller-sized outputs; null -> allocate in the arena
    float* pv; int pv_cap; int* pt; int pt_cap;
    float* nv; int nv_cap; int* nt; int nt_cap;
};

static __device__ __forceinline__ float cut_plane_eval(float pa, float pb, float pc, float pd, const float* v)
{
    return fmaf(pa, v[0], fmaf(pb, v[1], fmaf(pc, v[2], pd)));
}

struct CutShared {
    int scan[34];
    int cnt[8];
    int ok;
    void* ptr[16];
    int ival[16];
};

// ---- FP64 cap helpers (same operation order as the checker) --------------
struct Cap2D { const float* V; int pu, pv; };
static __device__ __forceinline__ double cU(const Cap2D& c, int v) { return (double)c.V[3 * v + c.pu]; }
static __device__ __forceinline__ double cW(const Cap2D& c, int v) { return (double)c.V[3 * v + c.pv]; }

static __device__ double cut_signed_area(const Cap2D& c, const int* poly, int n)
{
    double a = 0.0;
    for (int i = 0; i < n; i++) {
        int j = (i + 1) % n;
        a += cU(c, poly[i]) * cW(c, poly[j]) - cU(c, poly[j]) * cW(c, poly[i]);
    }
    return a * 0.5;
}
static __device__ void cut_reverse(int* a, int n) {
    for (int i = 0; i < n / 2; i++) { int t = a[i]; a[i] = a[n - 1 - i]; a[n - 1 - i] = t; }
}
static __device__ __forceinline__ double cut_cross2(double ax, double ay, double bx, double by, double cx, double cy) {
    return (bx - ax) * (cy - ay) - (by - ay) * (cx - ax);
}
static __device__ __forceinline__ int cut_pt_in_tri(double px, double py, double ax, double ay, double bx, double by,
                                             double cx, double cy)
{
    double d1 = cut_cross2(ax, ay, bx, by, px, py);
    double d2 = cut_cross2(bx, by, cx, cy, px, py);
    double d3 = cut_cross2(cx, cy, ax, ay, px, py);
    int neg = (d1 < -1e-10) || (d2 < -1e-10) || (d3 < -1e-10);
    int pos = (d1 > 1e-10) || (d2 > 1e-10) || (d3 > 1e-10);
    return !(neg && pos);
}

// Ear clipping of one polygon by the whole CTA, with the decisions -- and
// so the triangles -- of the one-thread walk (cur, remaining, iter): at cur
// with prev p, clip (p, cur, next) when it is degenerate or convex with no
// remaining vertex inside, advancing to next either way.  Every thread
// follows the walk.  At a convex or degenerate cur the walk would, as long
// as it keeps clipping, clip the fan p, c0 = cur, c1, c2, ... (each clip
// makes p the prev of the next vertex), so the first K triangles of the fan
// are tested in one pass of the CTA, triangle k against the vertices that
// remain once c0 .. c(k-1) are clipped, and the walk clips up to the first
// triangle that fails (a reflex triangle ends the fan before it).  One
// barrier per pass instead of one per tested ear.  K adapts: it doubles
// (up to CUT_EAR_SPEC) after a fan clipped whole and restarts at 2 after a
// failed ear, so walks whose ears often fail test few triangles ahead.
// Every thread writes the same fan (s_chain) and links and reads its own
// writes; fan and inside masks are double-buffered by pass parity, and the
// links of pass r + 1 are only written after its barrier, which every thread
// reaches after its reads of pass r + 1.  U/W hold the polygon's 2D coordinates
// (FP64), prv/nxt its links.  Returns the triangle count.
#define CUT_EAR_SM 1024     // polygons up to this size keep U/W/prv/nxt in shared memory
#define CUT_EAR_SPEC 32     // most fan triangles tested per pass
static __device__ int cut_ear_clip_cta(const Cap2D& c, const int* poly, int n, double* U, double* W,
                                       int* prv, int* nxt, int* cap)
{
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    __shared__ int s_chain[2][CUT_EAR_SPEC + 1];
    __shared__ unsigned s_wm[2][CUT_NT / 32];
    for (int i = tid; i < n; i += CUT_NT) {
        prv[i] = (i + n - 1) % n; nxt[i] = (i + 1) % n;
        U[i] = cU(c, poly[i]); W[i] = cW(c, poly[i]);
    }
    __syncthreads();
    int nc = 0, remaining = n, cur = 0, iter = 0, kspec = 2;
    for (int pass = 0;; pass++) {
        const int b = pass & 1;
        bool done = false;
        for (;;) {                                   // reflex steps
            if (!(remaining > 3 && iter < remaining)) { done = true; break; }
            const int p = prv[cur], q = nxt[cur];
            const double up = U[p], wp = W[p], uc = U[cur], wc = W[cur], un = U[q], wn = W[q];
            const double cr = (uc - up) * (wn - wp) - (wc - wp) * (un - up);
            if (cr < -1e-9) { iter++; cur = q; continue; }
            break;
        }
        if (done) break;
        const int p = prv[cur];
        const double up = U[p], wp = W[p];
        const int kmax = min(kspec, remaining - 3);
        int K = 0, cv = cur;
        unsigned need = 0;                           // bit k: triangle k is convex (needs the inside test)
        s_chain[b][0] = cur;
        while (K < kmax) {
            const int q = nxt[cv];
            const double uc = U[cv], wc = W[cv], un = U[q], wn = W[q];
            const double cr = (uc - up) * (wn - wp) - (wc - wp) * (un - up);
            if (cr < -1e-9) break;                   // reflex: the fan ends before it
            if (cr > 1e-9) need |= 1u << K;
            s_chain[b][K + 1] = q;
            K++; cv = q;
        }
        unsigned bits = 0;                           // bit k: a remaining vertex lies in fan triangle k
        if (need) {
            for (int idx = tid; idx < n; idx += CUT_NT) {
                if (idx == p || nxt[prv[idx]] != idx) continue;
                int pos = -1;
                for (int j = 0; j <= K; j++) if (s_chain[b][j] == idx) { pos = j; break; }
                // triangle k skips its own corners and the clipped c0 .. c(k-1)
                const int kend = pos < 0 ? K : pos - 1;
                const double cu = U[idx], cw = W[idx];
                for (int k = 0; k < kend; k++) {
                    if (!((need >> k) & 1u) || ((bits >> k) & 1u)) continue;
                    const int ck = s_chain[b][k], cn = s_chain[b][k + 1];
                    const double uc = U[ck], wc = W[ck], un = U[cn], wn = W[cn];
                    if (fabs(cu - up) + fabs(cw - wp) > 1e-6 &&
                        fabs(cu - uc) + fabs(cw - wc) > 1e-6 &&
                        fabs(cu - un) + fabs(cw - wn) > 1e-6 &&
                        cut_pt_in_tri(cu, cw, up, wp, uc, wc, un, wn)) bits |= 1u << k;
                }
            }
        }
        #pragma unroll
        for (int o = 16; o > 0; o >>= 1) bits |= __shfl_xor_sync(FULL_MASK, bits, o);
        if (lane == 0) s_wm[b][warp] = bits;
        __syncthreads();
        unsigned inside = 0;
        for (int w = 0; w < CUT_NT / 32; w++) inside |= s_wm[b][w];
        const unsigned fail = need & inside;
        const int ks = fail ? __ffs(fail) - 1 : K;   // triangles clipped
        // the clips in the walk's order; each made p the prev of the next vertex
        if (tid == 0)
            for (int k = 0; k < ks; k++) {
                cap[3 * (nc + k)] = poly[p]; cap[3 * (nc + k) + 1] = poly[s_chain[b][k]];
                cap[3 * (nc + k) + 2] = poly[s_chain[b][k + 1]];
            }
        for (int j = 1; j <= ks; j++) prv[s_chain[b][j]] = p;
        if (ks > 0) nxt[p] = s_chain[b][ks];
        nc += ks; remaining -= ks;
        if (ks < K) { iter = (ks > 0 ? 0 : iter) + 1; cur = s_chain[b][ks + 1]; kspec = 2; }   // the failed ear
        else        { iter = 0; cur = s_chain[b][K]; kspec = min(2 * kspec, CUT_EAR_SPEC); }
    }
    if (remaining == 3) {
        const int p = prv[cur], q = nxt[cur];
        if (tid == 0) { cap[3 * nc] = poly[p]; cap[3 * nc + 1] = poly[cur]; cap[3 * nc + 2] = poly[q]; }
        nc++;
    }
    __syncthreads();
    return nc;
}

// i = tid, tid + CUT_NT, ... < n, each thread issuing the loads of
// CUT_ILP iterations before their stores, so that a thread keeps several
// independent global loads in flight.  For loops whose iterations are
// independent: load(i) reads nothing that store(j) writes.
#define CUT_ILP 4
template <class Load, class Store>
static __device__ __forceinline__ void cut_for_ilp(int n, Load load, Store store)
{
    for (int base = threadIdx.x; base < n; base += CUT_ILP * CUT_NT) {
        decltype(load(0)) v[CUT_ILP];
        #pragma unroll
        for (int u = 0; u < CUT_ILP; u++) { const int i = base + u * CUT_NT; if (i < n) v[u] = load(i); }
        #pragma unroll
        for (int u = 0; u < CUT_ILP; u++) { const int i = base + u * CUT_NT; if (i < n) store(i, v[u]); }
    }
}

// Corner indices and vertex signs of the triangles t = base + u * CUT_NT,
// u < CUT_ILP (those below nt): all index loads first, then all sign loads.
static __device__ __forceinline__ void cut_load_tris(const int* __restrict__ tris, const signed char* sg, int nt,
                                                     int base, int (&ix)[CUT_ILP][3], int (&sv)[CUT_ILP][3])
{
    #pragma unroll
    for (int u = 0; u < CUT_ILP; u++) {
        const int t = base + u * CUT_NT;
        #pragma unroll
        for (int k = 0; k < 3; k++) ix[u][k] = t < nt ? tris[3 * t + k] : 0;
    }
    #pragma unroll
    for (int u = 0; u < CUT_ILP; u++)
        #pragma unroll
        for (int k = 0; k < 3; k++) sv[u][k] = base + u * CUT_NT < nt ? sg[ix[u][k]] : 0;
}

// Corners of the split triangles t = base + u * CUT_NT below n and whether
// each lies on the cut (a new vertex, or an input vertex of sign 0).
static __device__ __forceinline__ void cut_load_on_cut(const int* tri, const signed char* sg, int nv, int n,
                                                       int base, int (&ix)[CUT_ILP][3], int (&on)[CUT_ILP][3])
{
    #pragma unroll
    for (int u = 0; u < CUT_ILP; u++) {
        const int t = base + u * CUT_NT;
        #pragma unroll
        for (int k = 0; k < 3; k++) ix[u][k] = t < n ? tri[3 * t + k] : 0;
    }
    #pragma unroll
    for (int u = 0; u < CUT_ILP; u++)
        #pragma unroll
        for (int k = 0; k < 3; k++)
            on[u][k] = base + u * CUT_NT < n && (ix[u][k] >= nv || sg[ix[u][k]] == 0);
}

// +1 / -1: every vertex on the positive / negative side or on the plane,
// and one off it -- the triangle is its own piece on that side; 0: the
// triangle crosses the plane or lies in it.
static __device__ __forceinline__ int cut_tri_side(const int (&s)[3])
{
    const int hp = s[0] > 0 || s[1] > 0 || s[2] > 0, hn = s[0] < 0 || s[1] < 0 || s[2] < 0;
    return hp && !hn ? 1 : (hn && !hp ? -1 : 0);
}

// CTA-wide minimum of (key, idx) pairs in lexicographic order, returned to
// every thread (all CUT_NT threads call).
static __device__ void cut_cta_lexmin(double& key, int& idx)
{
    __shared__ double s_k[CUT_NT / 32];
    __shared__ int s_i[CUT_NT / 32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    #pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double k2 = __shfl_xor_sync(FULL_MASK, key, o);
        const int i2 = __shfl_xor_sync(FULL_MASK, idx, o);
        if (k2 < key || (k2 == key && i2 < idx)) { key = k2; idx = i2; }
    }
    if (lane == 0) { s_k[w] = key; s_i[w] = idx; }
    __syncthreads();
    key = s_k[0]; idx = s_i[0];
    for (int q = 1; q < CUT_NT / 32; q++)
        if (s_k[q] < key || (s_k[q] == key && s_i[q] < idx)) { key = s_k[q]; idx = s_i[q]; }
    __syncthreads();                                   // s_k / s_i free for the next call
}

// Caps from the directed boundary edges be[] (sorted by (a,b), packed a<<32|b).
// Whole CTA: the loops are traced by pointer jumping when the boundary's
// successor map is a permutation (else by thread 0's walk), nesting counts
// ray crossings with the CTA, holes are bridged by CTA reductions and a
// parallel splice, and the ear clipping is CTA-wide; thread 0 keeps the
// short serial decisions (loop orientation, parent choice, hole order).
// gU/gW: 2*poly_cap doubles of global scratch for
// polygons longer than CUT_EAR_SM.  Returns n_cap >= 0 or -1 on failure.
static __device__ int cut_build_caps(const float* V, int n_all, const unsigned long long* be, int nb,
                              float pa, float pb, float pc, int* used, int* lv, int* ls, int* lsz,
                              int* poly, int* tmp, int poly_cap, int* cap_out, int* n_loops_out,
                              double* gU)
{
    const int tid = threadIdx.x;
    __shared__ int s_nl, s_fail, s_pn;
    __shared__ double s_U[CUT_EAR_SM], s_W[CUT_EAR_SM];
    __shared__ int s_prv[CUT_EAR_SM], s_nxt[CUT_EAR_SM];
    Cap2D C; C.V = V;
    {
        float ax = fabsf(pa), ay = fabsf(pb), az = fabsf(pc);
        if (ax >= ay && ax >= az) { C.pu = 1; C.pv = 2; }
        else if (ay >= az)        { C.pu = 0; C.pv = 2; }
        else                      { C.pu = 0; C.pv = 1; }
    }
    // Loops, orientation and nesting are serial decisions of thread 0.  When
    // the boundary fits the ear-clipping arrays (nb <= CUT_EAR_SM) they are
    // borrowed first: the CTA stages each edge's start-vertex coordinates
    // (s_U/s_W), the first edge leaving its end vertex (s_nxt) and a used
    // flag (s_prv), so thread 0 walks shared memory instead of binary
    // searches and scattered vertex loads; le[k] (in `used`) is the edge
    // whose start vertex is lv[k] (shared memory: thread 0 would otherwise
    // wait on L2 for every element it has just written).  Same values, same
    // order: same result.
    const bool fast = nb <= CUT_EAR_SM;
    __shared__ int s_le[CUT_EAR_SM];
    __shared__ int s_ea[CUT_EAR_SM], s_eb[CUT_EAR_SM];     // each edge's start and end vertex
    int* le = fast ? s_le : used;
    if (fast) {
        for (int i = tid; i < nb; i += CUT_NT) {
            const int a = (int)(be[i] >> 32), b = (int)(be[i] & 0xffffffffu);
            s_ea[i] = a; s_eb[i] = b;
            s_U[i] = (a >= 0 && a < n_all) ? cU(C, a) : 0.0;
            s_W[i] = (a >= 0 && a < n_all) ? cW(C, a) : 0.0;
            s_nxt[i] = lower_bound_u64(be, nb, (unsigned long long)(unsigned)b << 32);
            s_prv[i] = 0;
        }
        __syncthreads();
    }
    auto LU = [&](int k) -> double { return fast ? s_U[le[k]] : cU(C, lv[k]); };
    auto LW = [&](int k) -> double { return fast ? s_W[le[k]] : cW(C, lv[k]); };
    auto loop_area = [&](int start, int m) -> double {      // cut_signed_area of lv[start .. start+m)
        double a = 0.0;
        for (int i = 0; i < m; i++) {
            const int j = (i + 1) % m;
            a += LU(start + i) * LW(start + j) - LU(start + j) * LW(start + i);
        }
        return a * 0.5;
    };
    auto loop_reverse = [&](int start, int m) { cut_reverse(lv + start, m); if (fast) cut_reverse(le + start, m); };
    int n_loops = 0, fail = 0;
    // Parallel tracing.  When every boundary vertex starts exactly one edge
    // and ends exactly one, "the first unused edge leaving the walk's vertex"
    // is the successor permutation, and thread 0's walk (next loop at the
    // smallest unused edge) yields its cycles, each from its smallest edge,
    // in order of that edge.  The CTA finds each edge's cycle minimum and
    // its distance from it by pointer jumping (log2 nb rounds each) and
    // writes lv / le / ls / lsz as the walk would.  Any other boundary (a
    // vertex with two outgoing edges, an open chain) takes the walk.
    __shared__ int s_scanbuf[34];
    bool traced = false;
    if (fast && nb >= 64) {
        int* succ = tmp;                              // tmp: 2 * poly_cap >= 8 nb + 128 ints
        int* cnt = tmp + nb;
        int* mA = tmp + 2 * nb; int* mB = tmp + 3 * nb;
        int* jA = tmp + 4 * nb; int* jB = tmp + 5 * nb;
        int* dA = tmp + 6 * nb; int* dB = tmp + 7 * nb;
        for (int i = tid; i < nb; i += CUT_NT) cnt[i] = 0;
        __syncthreads();
        int bad = 0;
        for (int i = tid; i < nb; i += CUT_NT) {
            const int a = s_ea[i], b = s_eb[i];
            int sc = s_nxt[i];
            if (a < 0 || a >= n_all || b < 0 || b >= n_all) bad = 1;
            if (sc >= nb || s_ea[sc] != b || (sc + 1 < nb && s_ea[sc + 1] == b)) { bad = 1; sc = i; }
            succ[i] = sc;
            atomicAdd(&cnt[sc], 1);
        }
        __syncthreads();
        for (int i = tid; i < nb; i += CUT_NT) if (cnt[i] != 1) bad = 1;
        if (!__syncthreads_or(bad)) {
            int R = 0;
            while ((1 << R) < nb) R++;
            // cycle minimum: after R rounds each edge has seen 2^R >= nb edges of its cycle
            for (int i = tid; i < nb; i += CUT_NT) { mA[i] = i; jA[i] = succ[i]; }
            __syncthreads();
            int *mc = mA, *mn = mB, *jc = jA, *jn = jB;
            for (int r = 0; r < R; r++) {
                for (int i = tid; i < nb; i += CUT_NT) { const int j = jc[i]; mn[i] = min(mc[i], mc[j]); jn[i] = jc[j]; }
                __syncthreads();
                int* t = mc; mc = mn; mn = t; t = jc; jc = jn; jn = t;
            }
            // steps to the cycle's last edge (the one whose successor is the minimum)
            int *dc = dA, *dn = dB;
            jc = jA; jn = jB;
            for (int i = tid; i < nb; i += CUT_NT) {
                const int last = succ[i] == mc[i];
                jc[i] = last ? -1 : succ[i]; dc[i] = last ? 0 : 1;
            }
            __syncthreads();
            for (int r = 0; r < R; r++) {
                for (int i = tid; i < nb; i += CUT_NT) {
                    const int j = jc[i];
                    if (j >= 0) { dn[i] = dc[i] + dc[j]; jn[i] = jc[j]; } else { dn[i] = dc[i]; jn[i] = -1; }
                }
                __syncthreads();
                int* t = dc; dc = dn; dn = t; t = jc; jc = jn; jn = t;
            }
            // loops in order of their smallest edge: starts and indices by two scans
            int* start = jc;                          // free now
            int* lid = jn;
            for (int i = tid; i < nb; i += CUT_NT) {
                const int is_min = mc[i] == i;
                start[i] = is_min ? dc[i] + 1 : 0;
                lid[i] = is_min;
            }
            __syncthreads();
            cta_scan_inplace(start, nb, s_scanbuf);
            const int nloops = cta_scan_inplace(lid, nb, s_scanbuf);
            if (nloops <= 128) {
                for (int i = tid; i < nb; i += CUT_NT) {
                    const int m = mc[i];
                    const int off = start[m] + (dc[m] - dc[i]);
                    lv[off] = s_ea[i]; le[off] = i;
                    if (m == i) { ls[lid[i]] = start[i]; lsz[lid[i]] = dc[i] + 1; }
                }
            }
            if (tid == 0) { s_nl = nloops; s_fail = nloops > 128; }
            traced = true;
        }
    }
    if (tid == 0 && !traced) {
        int lvi = 0;
        if (!fast) for (int i = 0; i < nb; i++) used[i] = 0;
        for (int st = 0; st < nb && !fail; st++) {
            if (fast ? s_prv[st] : used[st]) continue;
            int first = fast ? s_ea[st] : (int)(be[st] >> 32), cur = fast ? s_eb[st] : (int)(be[st] & 0xffffffffu);
            if (first < 0 || first >= n_all || cur < 0 || cur >= n_all) { fail = 1; break; }
            int ce = st;
            if (fast) { s_prv[st] = 1; le[lvi] = st; } else used[st] = 1;
            int start = lvi;
            lv[lvi++] = first;
            int guard = nb + 2;
            while (cur != first && guard-- > 0) {
                if (lvi >= nb) { fail = 1; break; }
                lv[lvi] = cur;
                int found = -1;
                if (fast) {
                    for (int k = s_nxt[ce]; k < nb && s_ea[k] == cur; k++) if (!s_prv[k]) { found = k; break; }
                } else {
                    int lo = lower_bound_u64(be, nb, (unsigned long long)(unsigned)cur << 32);
                    for (int k = lo; k < nb && (int)(be[k] >> 32) == cur; k++) if (!used[k]) { found = k; break; }
                }
                if (found < 0) { fail = 1; break; }
                if (fast) { s_prv[found] = 1; le[lvi] = found; } else used[found] = 1;
                lvi++;
                ce = found;
                cur = fast ? s_eb[found] : (int)(be[found] & 0xffffffffu);
            }
            if (fail || cur != first) { fail = 1; break; }
            ls[n_loops] = start; lsz[n_loops] = lvi - start; n_loops++;
        }
        if (n_loops > 128) fail = 1;
        s_nl = n_loops; s_fail = fail;
    }
    __syncthreads();
    n_loops = s_nl;
    fail = s_fail;
    *n_loops_out = n_loops;
    if (fail) return -1;
    __shared__ int parent[128], is_hole[128], hidx[128];
    __shared__ double hmax[128];
    __shared__ double s_area[128];
    __shared__ int s_ls[128], s_lsz[128], s_cross[2][128];
    int n_cap = 0;
    // Nesting: a loop's parent is the smallest loop (by |area|) that a ray
    // from its first vertex crosses an odd number of times.  Orientation and
    // the areas (computed once per loop, after the orientation fix, in the
    // walk's order) are thread 0's; the crossings of each loop's ray are
    // counted by the CTA, edge by edge with the same test, so the parities
    // -- and the parents -- are those of the serial count.
    if (tid == 0) {
        for (int i = 0; i < n_loops; i++)
            if (loop_area(ls[i], lsz[i]) < 0) loop_reverse(ls[i], lsz[i]);
        for (int i = 0; i < n_loops; i++) {
            parent[i] = -1; is_hole[i] = 0; s_ls[i] = ls[i]; s_lsz[i] = lsz[i];
            s_area[i] = lsz[i] >= 3 ? fabs(loop_area(ls[i], lsz[i])) : 0.0;
        }
    }
    __syncthreads();
    if (n_loops > 1) {
        const int npos = s_ls[n_loops - 1] + s_lsz[n_loops - 1];
        int round = 0;                               // counts buffered by round parity
        for (int i = 0; i < n_loops; i++) {
            if (s_lsz[i] < 3) continue;
            int* cross = s_cross[round++ & 1];
            for (int j = tid; j < n_loops; j += CUT_NT) cross[j] = 0;
            __syncthreads();
            const double pu_ = LU(s_ls[i]), pv_ = LW(s_ls[i]);
            for (int pos = tid; pos < npos; pos += CUT_NT) {
                int lo = 0, hi = n_loops - 1;            // the loop holding pos
                while (lo < hi) { const int mid = (lo + hi + 1) >> 1; if (s_ls[mid] <= pos) lo = mid; else hi = mid - 1; }
                const int j = lo, m = s_lsz[j];
                if (j == i || m < 3) continue;
                const int k = pos - s_ls[j], kn = (k + 1) % m;
                const double ay = LW(s_ls[j] + k), by = LW(s_ls[j] + kn);
                if ((ay <= pv_) == (by <= pv_)) continue;
                const double ax = LU(s_ls[j] + k), bx = LU(s_ls[j] + kn);
                const double t = (pv_ - ay) / (by - ay);
                if (ax + t * (bx - ax) > pu_) atomicAdd(&cross[j], 1);
            }
            __syncthreads();
            if (tid == 0) {
                double best_area = 1e300;
                for (int j = 0; j < n_loops; j++) {
                    if (j == i || s_lsz[j] < 3) continue;
                    if ((cross[j] & 1) && s_area[j] < best_area) { best_area = s_area[j]; parent[i] = j; }
                }
            }
        }
    }
    if (tid == 0) {
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
            for (int i = 0; i < n_loops; i++) if (is_hole[i]) loop_reverse(ls[i], lsz[i]);
        }
        s_fail = fail;
    }
    __syncthreads();
    fail = s_fail;
    if (fail) return -1;
    int expected = 0;
    for (int oi = 0; oi < n_loops; oi++) {
        if (is_hole[oi] || lsz[oi] < 3) continue;
        int pn = 0;
        {                                                    // the outer loop, copied by the CTA
            const int o = ls[oi], m = lsz[oi];
            for (int i = tid; i < m; i += CUT_NT) poly[i] = lv[o + i];
            __syncthreads();
        }
        // holes of this loop, by decreasing largest u (thread 0: a short list)
        __shared__ int s_nin;
        if (tid == 0) {
            int nin = 0;
            for (int i = 0; i < n_loops && nin < 128; i++) {
                if (parent[i] != oi || lsz[i] < 3) continue;
                double mu = -1e300;
                for (int j = 0; j < lsz[i]; j++) { double u = cU(C, lv[ls[i] + j]); if (u > mu) mu = u; }
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
            s_nin = nin; s_pn = lsz[oi]; s_fail = 0;
        }
        __syncthreads();
        // Each hole is bridged to the loop by the CTA: its rightmost vertex
        // (the first of largest u) and the loop edge its rightward ray meets
        // first (the first of smallest t) are CTA reductions over the same
        // per-vertex and per-edge expressions as a serial scan, with the
        // serial scan's tie rule (smallest index); the spliced polygon is
        // written in parallel.
        const int nin = s_nin;
        for (int ii = 0; ii < nin; ii++) {
            const int pn0 = s_pn;
            const int hi = hidx[ii], hs = lsz[hi];
            const int* hole = lv + ls[hi];
            double key = 1e300; int idx = 0x7fffffff;
            for (int j = tid; j < hs; j += CUT_NT) {
                const double k = -cU(C, hole[j]);
                if (k < key || (k == key && j < idx)) { key = k; idx = j; }
            }
            cut_cta_lexmin(key, idx);
            const int m_idx = idx;
            const double mu_ = cU(C, hole[m_idx]), mv_ = cW(C, hole[m_idx]);
            key = 1e300; idx = 0x7fffffff;
            for (int j = tid; j < pn0; j += CUT_NT) {
                const int jn = (j + 1) % pn0;
                const double au = cU(C, poly[j]), av = cW(C, poly[j]);
                const double bu = cU(C, poly[jn]), bv = cW(C, poly[jn]);
                const double dv = bv - av;
                if (fabs(dv) < 1e-12) continue;
                const double s_ = (mv_ - av) / dv;
                if (s_ < -1e-12 || s_ > 1.0 + 1e-12) continue;
                const double tv = au + s_ * (bu - au) - mu_;
                if (tv > 1e-12 && (tv < key || (tv == key && j < idx))) { key = tv; idx = j; }
            }
            cut_cta_lexmin(key, idx);
            const int best_edge = idx;
            if (best_edge == 0x7fffffff || pn0 + hs + 2 > poly_cap) { fail = 1; break; }   // uniform
            const int jn = (best_edge + 1) % pn0;
            const int p_pos = (cU(C, poly[best_edge]) >= cU(C, poly[jn])) ? best_edge : jn;
            const int npn = pn0 + hs + 2;
            for (int k = tid; k < npn; k += CUT_NT) {
                int v;
                if (k <= p_pos) v = poly[k];
                else if (k <= p_pos + hs) v = hole[(m_idx + (k - p_pos - 1)) % hs];
                else if (k == p_pos + hs + 1) v = hole[m_idx];
                else if (k == p_pos + hs + 2) v = poly[p_pos];
                else v = poly[k - hs - 2];
                tmp[k] = v;
            }
            __syncthreads();
            for (int k = tid; k < npn; k += CUT_NT) poly[k] = tmp[k];
            if (tid == 0) s_pn = npn;
            __syncthreads();
        }
        if (tid == 0 && fail) s_fail = 1;
        __syncthreads();
        fail = s_fail;
        pn = s_pn;
        if (fail) return -1;
        expected += pn - 2;
        if (pn >= 3) {
            if (pn <= CUT_EAR_SM)
                n_cap += cut_ear_clip_cta(C, poly, pn, s_U, s_W, s_prv, s_nxt, cap_out + 3 * n_cap);
            else
                n_cap += cut_ear_clip_cta(C, poly, pn, gU, gU + poly_cap, tmp, tmp + poly_cap, cap_out + 3 * n_cap);
        }
    }
    if (n_cap < expected) return -1;
    return n_cap;
}

// ---------------------------------------------------------------------------
// the CTA cut.  All CUT_NT threads call.  Scratch comes from `arena`; if
// fixed.pv == null the fragments come from `out_arena` (default: `arena`).
// Writes *res.
// ---------------------------------------------------------------------------
static __device__ void cut_cta(const float* __restrict__ verts, int nv, const int* __restrict__ tris, int nt,
                        float pa, float pb, float pc, float pd, Arena* arena, CutFixedOut fixed,
                        CutResult* res, CutShared& sh, Arena* out_arena = nullptr)
{
    const int tid = threadIdx.x, lane = tid & 31;
    Arena* const oarena = out_arena ? out_arena : arena;
    long long tph[5];
    tph[0] = clock64();
    __shared__ int s_err;
    if (tid == 0) s_err = 0;
    __syncthreads();
#define CUT_ALLOC(slot, T, count) do { if (tid == 0) { \
        sh.ptr[slot] = s_err ? nullptr : arena_alloc(arena, sizeof(T) * (unsigned long long)((count) > 0 ? (count) : 1), &s_err); \
        if (!sh.ptr[slot]) s_err |= KERR_PC_SCRATCH_OOM; } } while (0)
    // ---- classify
    CUT_ALLOC(0, signed char, nv);
    __syncthreads();
    if (s_err) goto fail_out;
    {
        signed char* sg = (signed char*)sh.ptr[0];
        for (int v = tid; v < nv; v += CUT_NT) {
            float d = cut_plane_eval(pa, pb, pc, pd, verts + 3 * v);
            sg[v] = (d > CUT_EPS) ? 1 : ((d < -CUT_EPS) ? -1 : 0);
        }
        if (tid < 8) sh.cnt[tid] = 0;
        __syncthreads();
        // count crossing occurrences, and sides present
        int occ = 0, anyp = 0, anyn = 0;
        for (int base = tid; base < nt; base += CUT_ILP * CUT_NT) {
            int ix[CUT_ILP][3], sv[CUT_ILP][3];
            cut_load_tris(tris, sg, nt, base, ix, sv);
            #pragma unroll
            for (int u = 0; u < CUT_ILP; u++) {
                if (base + u * CUT_NT >= nt) continue;
                const int e0 = sv[u][0] >= 0, e1 = sv[u][1] >= 0, e2 = sv[u][2] >= 0;
                occ += (e0 != e1) + (e1 != e2) + (e2 != e0);
            }
        }
        for (int v = tid; v < nv; v += CUT_NT) { anyp |= sg[v] > 0; anyn |= sg[v] < 0; }
        occ = warp_sum_i(occ);
        if (lane == 0) atomicAdd(&sh.cnt[0], occ);
        if (anyp) sh.cnt[1] = 1;
        if (anyn) sh.cnt[2] = 1;
        __syncthreads();
    }
    {
    const signed char* sg = (const signed char*)sh.ptr[0];
    const int n_occ = sh.cnt[0];
    const int any_pos = sh.cnt[1], any_neg = sh.cnt[2];
    if (n_occ == 0) {
        // ---------------- no crossing edge: whole mesh or side split
        if (!any_pos || !any_neg) {
            int to_neg = any_neg && !any_pos;
            // copy whole mesh to one side
            if (tid == 0) {
                float* ov = to_neg ? fixed.nv : fixed.pv; int* ot = to_neg ? fixed.nt : fixed.pt;
                int vc = to_neg ? fixed.nv_cap : fixed.pv_cap, tc = to_neg ? fixed.nt_cap : fixed.pt_cap;
                if (!fixed.pv) {
                    ov = (float*)arena_alloc(oarena, sizeof(float) * 3ull * (nv > 0 ? nv : 1), &s_err);
                    ot = (int*)arena_alloc(oarena, sizeof(int) * 3ull * (nt > 0 ? nt : 1), &s_err);
                    vc = nv; tc = nt;
                }
                if (!ov || !ot || nv > vc || nt > tc) s_err |= KERR_PC_POOL_OOM;
                sh.ptr[1] = ov; sh.ptr[2] = ot; sh.ival[0] = to_neg;
            }
            __syncthreads();
            if (s_err) goto fail_out;
            float* ov = (float*)sh.ptr[1]; int* ot = (int*)sh.ptr[2];
            for (int i = tid; i < 3 * nv; i += CUT_NT) ov[i] = verts[i];
            for (int i = tid; i < 3 * nt; i += CUT_NT) ot[i] = tris[i];
            if (tid == 0) {
                memset(res, 0, sizeof(CutResult));
                if (sh.ival[0]) { res->nv = ov; res->nt = ot; res->nnv = nv; res->nnt = nt; res->n_neg_tris = nt; }
                else            { res->pv = ov; res->pt = ot; res->npv = nv; res->npt = nt; res->n_pos_tris = nt; }
            }
            return;
        }
        // disjoint components on both sides: triangle goes to the negative side
        // if any vertex is negative; vertices renumbered by first use
        CUT_ALLOC(3, int, nv);                 // first use
        __syncthreads();
        if (s_err) goto fail_out;
        int* first = (int*)sh.ptr[3];
        for (int side = 0; side < 2; side++) {
            for (int v = tid; v < nv; v += CUT_NT) first[v] = 0x7fffffff;
            __syncthreads();
            int cnt_t = 0;
            for (int t = tid; t < nt; t += CUT_NT) {
                int i0 = tris[3 * t], i1 = tris[3 * t + 1], i2 = tris[3 * t + 2];
                int isneg = sg[i0] < 0 || sg[i1] < 0 || sg[i2] < 0;
                if (isneg != side) continue;
                cnt_t++;
                atomicMin(&first[i0], 3 * t); atomicMin(&first[i1], 3 * t + 1); atomicMin(&first[i2], 3 * t + 2);
            }
            cnt_t = warp_sum_i(cnt_t);
            if (tid == 0) sh.cnt[3] = 0;
            __syncthreads();
            if (lane == 0) atomicAdd(&sh.cnt[3], cnt_t);
            __syncthreads();
            // rank of each first use among positions 0..3nt-1: flag array over positions
            CUT_ALLOC(4 + side, int, 3 * nt);
            __syncthreads();
            if (s_err) goto fail_out;
            int* rank = (int*)sh.ptr[4 + side];
            for (int p = tid; p < 3 * nt; p += CUT_NT) rank[p] = 0;
            __syncthreads();
            for (int v = tid; v < nv; v += CUT_NT) if (first[v] != 0x7fffffff) rank[first[v]] = 1;
            __syncthreads();
            int nvs = cta_scan_inplace(rank, 3 * nt, sh.scan);
            int nts = sh.cnt[3];
            if (tid == 0) {
                float* ov = side ? fixed.nv : fixed.pv; int* ot = side ? fixed.nt : fixed.pt;
                int vc = side ? fixed.nv_cap : fixed.pv_cap, tc = side ? fixed.nt_cap : fixed.pt_cap;
                if (!fixed.pv) {
                    ov = (float*)arena_alloc(oarena, sizeof(float) * 3ull * (nvs > 0 ? nvs : 1), &s_err);
                    ot = (int*)arena_alloc(oarena, sizeof(int) * 3ull * (nts > 0 ? nts : 1), &s_err);
                    vc = nvs; tc = nts;
                }
                if (!ov || !ot || nvs > vc || nts > tc) s_err |= KERR_PC_POOL_OOM;
                sh.ptr[6 + 2 * side] = ov; sh.ptr[7 + 2 * side] = ot;
                sh.ival[2 + 2 * side] = nvs; sh.ival[3 + 2 * side] = nts;
                sh.cnt[4] = 0;
            }
            __syncthreads();
            if (s_err) goto fail_out;
            float* ov = (float*)sh.ptr[6 + 2 * side]; int* ot = (int*)sh.ptr[7 + 2 * side];
            for (int v = tid; v < nv; v += CUT_NT) {
                if (first[v] == 0x7fffffff) continue;
                int j = rank[first[v]];
                ov[3 * j] = verts[3 * v]; ov[3 * j + 1] = verts[3 * v + 1]; ov[3 * j + 2] = verts[3 * v + 2];
            }
            // triangles of this side in input order: scan over per-triangle flags
            CUT_ALLOC(10 + side, int, nt);
            __syncthreads();
            if (s_err) goto fail_out;
            int* tpos = (int*)sh.ptr[10 + side];
            for (int t = tid; t < nt; t += CUT_NT) {
                int isneg = sg[tris[3 * t]] < 0 || sg[tris[3 * t + 1]] < 0 || sg[tris[3 * t + 2]] < 0;
                tpos[t] = isneg == side;
            }
            __syncthreads();
            cta_scan_inplace(tpos, nt, sh.scan);
            for (int t = tid; t < nt; t += CUT_NT) {
                int i0 = tris[3 * t], i1 = tris[3 * t + 1], i2 = tris[3 * t + 2];
                int isneg = sg[i0] < 0 || sg[i1] < 0 || sg[i2] < 0;
                if (isneg != side) continue;
                int k = tpos[t];
                ot[3 * k] = rank[first[i0]]; ot[3 * k + 1] = rank[first[i1]]; ot[3 * k + 2] = rank[first[i2]];
            }
            __syncthreads();
        }
        if (tid == 0) {
            memset(res, 0, sizeof(CutResult));
            res->pv = (float*)sh.ptr[6]; res->pt = (int*)sh.ptr[7]; res->npv = sh.ival[2]; res->npt = sh.ival[3];
            res->nv = (float*)sh.ptr[8]; res->nt = (int*)sh.ptr[9]; res->nnv = sh.ival[4]; res->nnt = sh.ival[5];
            res->n_pos_tris = res->npt; res->n_neg_tris = res->nnt;
        }
        return;
    }
    // ---------------- crossing edges: collect, sort, dedup
    const int occN = next_pow2_i(n_occ);
    CUT_ALLOC(3, unsigned long long, occN);
    __syncthreads();
    if (s_err) goto fail_out;
    unsigned long long* ce = (unsigned long long*)sh.ptr[3];
    if (tid == 0) sh.cnt[3] = 0;
    __syncthreads();
    // collection order does not matter: the keys are sorted next
    for (int base = 0; base < nt; base += CUT_ILP * CUT_NT) {     // uniform trip count (warp shuffles)
        int ix[CUT_ILP][3], sv[CUT_ILP][3];
        cut_load_tris(tris, sg, nt, base + tid, ix, sv);
        int m = 0;
        #pragma unroll
        for (int u = 0; u < CUT_ILP; u++)
            #pragma unroll
            for (int e = 0; e < 3; e++)
                m += base + tid + u * CUT_NT < nt && (sv[u][e] >= 0) != (sv[u][(e + 1) % 3] >= 0);
        int x = m;                                      // warp inclusive scan of the counts
        #pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(FULL_MASK, x, o);
            if (lane >= o) x += y;
        }
        int wb = 0;
        const int wt = __shfl_sync(FULL_MASK, x, 31);
        if (lane == 31 && wt) wb = atomicAdd(&sh.cnt[3], wt);
        wb = __shfl_sync(FULL_MASK, wb, 31);
        int j = wb + x - m;
        #pragma unroll
        for (int u = 0; u < CUT_ILP; u++)
            #pragma unroll
            for (int e = 0; e < 3; e++) {
                if (base + tid + u * CUT_NT >= nt || (sv[u][e] >= 0) == (sv[u][(e + 1) % 3] >= 0)) continue;
                const int va = ix[u][e], vb = ix[u][(e + 1) % 3];
                const int lo = min(va, vb), hi = max(va, vb);
                ce[j++] = ((unsigned long long)(unsigned)lo << 32) | (unsigned)hi;
            }
    }
    __syncthreads();
    cta_sort_u64(ce, n_occ);
    // unique keys (sorted order) and the intersection vertex of each
    CUT_ALLOC(4, int, n_occ);                  // 1 where a new key starts
    CUT_ALLOC(5, int, n_occ);                  // scanned copy: unique rank
    __syncthreads();
    if (s_err) goto fail_out;
    int* uflag = (int*)sh.ptr[4];
    int* urank = (int*)sh.ptr[5];
    for (int i = tid; i < n_occ; i += CUT_NT) {
        int f = (i == 0 || ce[i] != ce[i - 1]) ? 1 : 0;
        uflag[i] = f; urank[i] = f;
    }
    __syncthreads();
    const int n_u = cta_scan_inplace(urank, n_occ, sh.scan);
    CUT_ALLOC(6, unsigned long long, n_u);     // unique edge keys
    CUT_ALLOC(7, int, n_u);                    // intersection vertex per edge
    CUT_ALLOC(2, int, n_u);                    // new-vertex rank
    __syncthreads();
    if (s_err) goto fail_out;
    unsigned long long* ue = (unsigned long long*)sh.ptr[6];
    int* isect = (int*)sh.ptr[7];
    int* upos = (int*)sh.ptr[2];
    for (int i = tid; i < n_occ; i += CUT_NT) if (uflag[i]) ue[urank[i]] = ce[i];
    __syncthreads();
    for (int i = tid; i < n_u; i += CUT_NT) {
        int va = (int)(ue[i] >> 32), vb = (int)(ue[i] & 0xffffffffu);
        float d0 = cut_plane_eval(pa, pb, pc, pd, verts + 3 * va);
        float d1 = cut_plane_eval(pa, pb, pc, pd, verts + 3 * vb);
        int reuse;
        if (fabsf(d0) <= CUT_EPS && fabsf(d1) > CUT_EPS) reuse = va;
        else if (fabsf(d1) <= CUT_EPS && fabsf(d0) > CUT_EPS) reuse = vb;
        else reuse = -1;
        isect[i] = reuse;
        upos[i] = reuse < 0 ? 1 : 0;
    }
    __syncthreads();
    const int n_new = cta_scan_inplace(upos, n_u, sh.scan);
    const int n_all = nv + n_new;
    CUT_ALLOC(8, float, 3 * n_all);            // all vertices
    __syncthreads();
    if (s_err) goto fail_out;
    float* all = (float*)sh.ptr[8];
    for (int i = tid; i < 3 * nv; i += CUT_NT) all[i] = verts[i];
    for (int i = tid; i < n_u; i += CUT_NT) {
        if (isect[i] >= 0) continue;
        int va = (int)(ue[i] >> 32), vb = (int)(ue[i] & 0xffffffffu);
        float d0 = cut_plane_eval(pa, pb, pc, pd, verts + 3 * va);
        float d1 = cut_plane_eval(pa, pb, pc, pd, verts + 3 * vb);
        float t = d0 / (d0 - d1);
        int ni = nv + upos[i];
        for (int k = 0; k < 3; k++)
            all[3 * ni + k] = fmaf(t, verts[3 * vb + k] - verts[3 * va + k], verts[3 * va + k]);
        isect[i] = ni;
    }
    __syncthreads();
    tph[1] = clock64();
    // ---------------- split: per-triangle piece counts then write in order
    CUT_ALLOC(9, int, nt);     // pos offsets
    CUT_ALLOC(10, int, nt);    // neg offsets
    __syncthreads();
    if (s_err) goto fail_out;
    int* poff = (int*)sh.ptr[9];
    int* noff = (int*)sh.ptr[10];
    auto isect_of = [&](int a, int b) -> int {
        int lo = min(a, b), hi = max(a, b);
        unsigned long long key = ((unsigned long long)(unsigned)lo << 32) | (unsigned)hi;
        int f = lower_bound_u64(ue, n_u, key);
        return (f < n_u && ue[f] == key) ? isect[f] : -1;
    };
    // piece emitter: mode 0 = count, 1 = write
    auto split = [&](int t, int mode, int* pt_, int* nt_, int po, int no) {
        int i0 = tris[3 * t], i1 = tris[3 * t + 1], i2 = tris[3 * t + 2];
        int s0 = sg[i0], s1 = sg[i1], s2 = sg[i2];
        int np_ = 0, nn_ = 0;
        auto P = [&](int x, int y, int z) { if (mode) { pt_[3 * (po + np_)] = x; pt_[3 * (po + np_) + 1] = y; pt_[3 * (po + np_) + 2] = z; } np_++; };
        auto N = [&](int x, int y, int z) { if (mode) { nt_[3 * (no + nn_)] = x; nt_[3 * (no + nn_) + 1] = y; nt_[3 * (no + nn_) + 2] = z; } nn_++; };
        int hp = s0 > 0 || s1 > 0 || s2 > 0, hn = s0 < 0 || s1 < 0 || s2 < 0;
        if (!hp || !hn) {
            if (hn) N(i0, i1, i2);
            else if (hp) P(i0, i1, i2);
            else {
                float e1x = all[3 * i1] - all[3 * i0], e1y = all[3 * i1 + 1] - all[3 * i0 + 1], e1z = all[3 * i1 + 2] - all[3 * i0 + 2];
                float e2x = all[3 * i2] - all[3 * i0], e2y = all[3 * i2 + 1] - all[3 * i0 + 1], e2z = all[3 * i2 + 2] - all[3 * i0 + 2];
                double dot = (double)pa * ((double)e1y * e2z - (double)e1z * e2y)
                           + (double)pb * ((double)e1z * e2x - (double)e1x * e2z)
                           + (double)pc * ((double)e1x * e2y - (double)e1y * e2x);
                if (dot > 0) P(i0, i1, i2); else N(i0, i1, i2);
            }
            return make_int2(np_, nn_);
        }
        int vi[3] = {i0, i1, i2}, si[3] = {s0, s1, s2};
        int on = -1;
        for (int k = 0; k < 3; k++) if (si[k] == 0) { on = k; break; }
        if (on >= 0) {
            int ov = vi[on], a_i = vi[(on + 1) % 3], b_i = vi[(on + 2) % 3], sa = si[(on + 1) % 3], sb = si[(on + 2) % 3];
            if (sa == sb) { if (sa > 0) P(i0, i1, i2); else N(i0, i1, i2); }
            else {
                int nvi = isect_of(a_i, b_i);
                if (nvi >= 0) {
                    if (sa > 0) { P(ov, a_i, nvi); N(ov, nvi, b_i); }
                    else        { N(ov, a_i, nvi); P(ov, nvi, b_i); }
                }
            }
        } else {
            int lone = -1;
            for (int k = 0; k < 3; k++) if (si[k] != si[(k + 1) % 3] && si[k] != si[(k + 2) % 3]) { lone = k; break; }
            if (lone >= 0) {
                int lv = vi[lone], ov1 = vi[(lone + 1) % 3], ov2 = vi[(lone + 2) % 3], lsg = si[lone];
                int nv1 = isect_of(lv, ov1), nv2 = isect_of(lv, ov2);
                if (nv1 >= 0 && nv2 >= 0) {
                    if (lsg > 0) { P(lv, nv1, nv2); N(ov1, nv2, nv1); N(ov1, ov2, nv2); }
                    else         { N(lv, nv1, nv2); P(ov1, nv2, nv1); P(ov1, ov2, nv2); }
                }
            }
        }
        return make_int2(np_, nn_);
    };
    // A triangle with no vertex on the other side and one off the plane is
    // its own single piece (split()'s first case); the batches below handle
    // it inline and leave the rest (crossing or coplanar) to split().
    for (int base = tid; base < nt; base += CUT_ILP * CUT_NT) {
        int ix[CUT_ILP][3], sv[CUT_ILP][3];
        cut_load_tris(tris, sg, nt, base, ix, sv);
        unsigned rare = 0;
        #pragma unroll
        for (int u = 0; u < CUT_ILP; u++) {
            const int t = base + u * CUT_NT;
            if (t >= nt) continue;
            const int side = cut_tri_side(sv[u]);
            if (side == 0) { rare |= 1u << u; continue; }
            poff[t] = side > 0; noff[t] = side < 0;
        }
        #pragma unroll 1
        for (int u = 0; u < CUT_ILP; u++)
            if (rare >> u & 1) {
                const int t = base + u * CUT_NT;
                const int2 c = split(t, 0, nullptr, nullptr, 0, 0);
                poff[t] = c.x; noff[t] = c.y;
            }
    }
    __syncthreads();
    const int n_pos = cta_scan_inplace(poff, nt, sh.scan);
    const int n_neg = cta_scan_inplace(noff, nt, sh.scan);
    CUT_ALLOC(11, int, 3 * n_pos);
    CUT_ALLOC(12, int, 3 * n_neg);
    __syncthreads();
    if (s_err) goto fail_out;
    int* ptri = (int*)sh.ptr[11];
    int* ntri = (int*)sh.ptr[12];
    for (int base = tid; base < nt; base += CUT_ILP * CUT_NT) {
        int ix[CUT_ILP][3], sv[CUT_ILP][3], po[CUT_ILP], no[CUT_ILP];
        #pragma unroll
        for (int u = 0; u < CUT_ILP; u++) {
            const int t = base + u * CUT_NT;
            if (t < nt) { po[u] = poff[t]; no[u] = noff[t]; }
        }
        cut_load_tris(tris, sg, nt, base, ix, sv);
        unsigned rare = 0;
        #pragma unroll
        for (int u = 0; u < CUT_ILP; u++) {
            const int t = base + u * CUT_NT;
            if (t >= nt) continue;
            const int side = cut_tri_side(sv[u]);
            if (side == 0) { rare |= 1u << u; continue; }
            int* dst = side > 0 ? ptri + 3 * po[u] : ntri + 3 * no[u];
            dst[0] = ix[u][0]; dst[1] = ix[u][1]; dst[2] = ix[u][2];
        }
        #pragma unroll 1
        for (int u = 0; u < CUT_ILP; u++)
            if (rare >> u & 1) {
                const int t = base + u * CUT_NT;
                split(t, 1, ptri, ntri, poff[t], noff[t]);
            }
    }
    __syncthreads();
    tph[2] = clock64();
    // ---------------- boundary of the positive side among edges on the cut
    // key = min<<33 | max<<1 | (a > b)
    if (tid == 0) sh.cnt[5] = 0;
    __syncthreads();
    int nbc_local = 0;
    for (int base = tid; base < n_pos; base += CUT_ILP * CUT_NT) {
        int ix[CUT_ILP][3], on[CUT_ILP][3];
        cut_load_on_cut(ptri, sg, nv, n_pos, base, ix, on);
        #pragma unroll
        for (int u = 0; u < CUT_ILP; u++)
            #pragma unroll
            for (int e = 0; e < 3; e++)
                nbc_local += base + u * CUT_NT < n_pos && on[u][e] && on[u][(e + 1) % 3];
    }
    nbc_local = warp_sum_i(nbc_local);
    if (lane == 0) atomicAdd(&sh.cnt[5], nbc_local);
    __syncthreads();
    const int nbc = sh.cnt[5];
    CUT_ALLOC(13, unsigned long long, next_pow2_i(nbc));
    __syncthreads();
    if (s_err) goto fail_out;
    unsigned long long* bk = (unsigned long long*)sh.ptr[13];
    if (tid == 0) sh.cnt[6] = 0;
    __syncthreads();
    for (int base = tid; base < n_pos; base += CUT_ILP * CUT_NT) {
        int ix[CUT_ILP][3], on[CUT_ILP][3];
        cut_load_on_cut(ptri, sg, nv, n_pos, base, ix, on);
        #pragma unroll
        for (int u = 0; u < CUT_ILP; u++)
            #pragma unroll
            for (int e = 0; e < 3; e++) {
                if (base + u * CUT_NT >= n_pos || !on[u][e] || !on[u][(e + 1) % 3]) continue;
                const int a = ix[u][e], b = ix[u][(e + 1) % 3];
                const int lo = min(a, b), hi = max(a, b);
                const int s = atomicAdd(&sh.cnt[6], 1);
                bk[s] = ((unsigned long long)(unsigned)lo << 33) | ((unsigned long long)(unsigned)hi << 1) | (a > b ? 1ull : 0ull);
            }
    }
    __syncthreads();
    cta_sort_u64(bk, nbc);
    // unmatched directed edges -> be (a<<32|b), sorted
    CUT_ALLOC(14, unsigned long long, next_pow2_i(nbc > 0 ? nbc : 1));
    __syncthreads();
    if (s_err) goto fail_out;
    unsigned long long* be = (unsigned long long*)sh.ptr[14];
    if (tid == 0) sh.cnt[7] = 0;
    __syncthreads();
    for (int i = tid; i < nbc; i += CUT_NT) {
        unsigned long long k = bk[i] >> 1;
        bool dup = (i > 0 && (bk[i - 1] >> 1) == k) || (i + 1 < nbc && (bk[i + 1] >> 1) == k);
        if (!dup) {
            int lo = (int)(k >> 32), hi = (int)(k & 0xffffffffu);
            int a = (bk[i] & 1ull) ? hi : lo, b = (bk[i] & 1ull) ? lo : hi;
            int s = atomicAdd(&sh.cnt[7], 1);
            be[s] = ((unsigned long long)(unsigned)a << 32) | (unsigned)b;
        }
    }
    __syncthreads();
    const int nb = sh.cnt[7];
    cta_sort_u64(be, nb);
    tph[3] = clock64();
    // ---------------- caps (whole CTA)
    const int poly_cap = nb * 4 + 64;
    CUT_ALLOC(15, int, 4 * nb + 3 * poly_cap + 3 * poly_cap);
    CUT_ALLOC(13, double, poly_cap > CUT_EAR_SM ? 2 * poly_cap : 1);   // ear-clip coordinates of long polygons
    __syncthreads();
    if (s_err) goto fail_out;
    {
        int* blk = (int*)sh.ptr[15];
        int* used = blk; int* lv = used + nb; int* ls = lv + nb; int* lsz = ls + nb;
        int* poly = lsz + nb; int* tmp = poly + poly_cap; int* capt = tmp + 2 * poly_cap;
        int nl = 0;
        int nc = (nb > 0) ? cut_build_caps(all, n_all, be, nb, pa, pb, pc, used, lv, ls, lsz, poly, tmp,
                                           poly_cap, capt, &nl, (double*)sh.ptr[13]) : 0;
        if (tid == 0) { sh.ival[8] = nc; sh.ival[9] = nl; }
        __syncthreads();
    }
    {
        const int n_cap = sh.ival[8];
        int* capt = (int*)sh.ptr[15] + 4 * nb + 3 * poly_cap;
        if (n_cap < 0) {
            // cap failure: whole mesh on the positive side
            if (tid == 0) {
                float* ov = fixed.pv; int* ot = fixed.pt;
                int vc = fixed.pv_cap, tc = fixed.pt_cap;
                if (!fixed.pv) {
                    ov = (float*)arena_alloc(oarena, sizeof(float) * 3ull * nv, &s_err);
                    ot = (int*)arena_alloc(oarena, sizeof(int) * 3ull * nt, &s_err);
                    vc = nv; tc = nt;
                }
                if (!ov || !ot || nv > vc || nt > tc) s_err |= KERR_PC_POOL_OOM;
                sh.ptr[1] = ov; sh.ptr[2] = ot;
            }
            __syncthreads();
            if (s_err) goto fail_out;
            float* ov = (float*)sh.ptr[1]; int* ot = (int*)sh.ptr[2];
            for (int i = tid; i < 3 * nv; i += CUT_NT) ov[i] = verts[i];
            for (int i = tid; i < 3 * nt; i += CUT_NT) ot[i] = tris[i];
            if (tid == 0) {
                memset(res, 0, sizeof(CutResult));
                res->pv = ov; res->pt = ot; res->npv = nv; res->npt = nt;
                res->n_pos_tris = n_pos; res->n_neg_tris = n_neg; res->cap_failed = 1;
                res->n_loops = sh.ival[9]; res->n_boundary = nb; res->n_cross = n_u;
            }
            return;
        }
        // ---------------- output compaction per side
        int flip;
        {
            float ax = fabsf(pa), ay = fabsf(pb), az = fabsf(pc);
            float n2d[3] = {0.f, 0.f, 0.f};
            if (ax >= ay && ax >= az) n2d[0] = 1.0f;
            else if (ay >= az)        n2d[1] = -1.0f;
            else                      n2d[2] = 1.0f;
            flip = (n2d[0] * (-pa) + n2d[1] * (-pb) + n2d[2] * (-pc) < 0) ? 1 : 0;
        }
        CUT_ALLOC(1, int, n_all);
        __syncthreads();
        if (s_err) goto fail_out;
        int* remap = (int*)sh.ptr[1];
        for (int side = 0; side < 2; side++) {
            const int* st = side == 0 ? ptri : ntri;
            const int ns = side == 0 ? n_pos : n_neg;
            for (int v = tid; v < n_all; v += CUT_NT) remap[v] = 0;
            __syncthreads();
            cut_for_ilp(3 * ns, [&](int i) { return st[i]; }, [&](int, int v) { remap[v] = 1; });
            cut_for_ilp(3 * n_cap, [&](int i) { return capt[i]; }, [&](int, int v) { remap[v] = 1; });
            __syncthreads();
            // remember used flags in the sign bit region: scan destroys them,
            // so mark unused as -1 after the scan by re-deriving from triangles
            CUT_ALLOC(2, int, n_all);
            __syncthreads();
            if (s_err) goto fail_out;
            int* usedf = (int*)sh.ptr[2];
            for (int v = tid; v < n_all; v += CUT_NT) usedf[v] = remap[v];
            __syncthreads();
            const int cnv = cta_scan_inplace(remap, n_all, sh.scan);
            const int cnt_ = ns + n_cap;
            if (tid == 0) {
                float* ov = side ? fixed.nv : fixed.pv; int* ot = side ? fixed.nt : fixed.pt;
                int vc = side ? fixed.nv_cap : fixed.pv_cap, tc = side ? fixed.nt_cap : fixed.pt_cap;
                if (!fixed.pv) {
                    ov = (float*)arena_alloc(oarena, sizeof(float) * 3ull * (cnv > 0 ? cnv : 1), &s_err);
                    ot = (int*)arena_alloc(oarena, sizeof(int) * 3ull * (cnt_ > 0 ? cnt_ : 1), &s_err);
                    vc = cnv; tc = cnt_;
                }
                if (!ov || !ot || cnv > vc || cnt_ > tc) s_err |= KERR_PC_POOL_OOM;
                sh.ptr[6 + 2 * side] = ov; sh.ptr[7 + 2 * side] = ot;
                sh.ival[2 + 2 * side] = cnv; sh.ival[3 + 2 * side] = cnt_;
            }
            __syncthreads();
            if (s_err) goto fail_out;
            float* ov = (float*)sh.ptr[6 + 2 * side]; int* ot = (int*)sh.ptr[7 + 2 * side];
            cut_for_ilp(n_all, [&](int v) { return usedf[v] ? remap[v] : -1; },
                        [&](int v, int j) {
                            if (j >= 0) { ov[3 * j] = all[3 * v]; ov[3 * j + 1] = all[3 * v + 1]; ov[3 * j + 2] = all[3 * v + 2]; }
                        });
            cut_for_ilp(3 * ns, [&](int i) { return remap[st[i]]; }, [&](int i, int j) { ot[i] = j; });
            for (int t = tid; t < n_cap; t += CUT_NT) {
                int v0 = capt[3 * t], v1 = capt[3 * t + 1], v2 = capt[3 * t + 2];
                int o = 3 * (ns + t);
                ot[o] = remap[v0];
                if (side == 0) { ot[o + 1] = flip ? remap[v2] : remap[v1]; ot[o + 2] = flip ? remap[v1] : remap[v2]; }
                else           { ot[o + 1] = flip ? remap[v1] : remap[v2]; ot[o + 2] = flip ? remap[v2] : remap[v1]; }
            }
            __syncthreads();
        }
        if (tid == 0) {
            memset(res, 0, sizeof(CutResult));
            res->pv = (float*)sh.ptr[6]; res->pt = (int*)sh.ptr[7]; res->npv = sh.ival[2]; res->npt = sh.ival[3];
            res->nv = (float*)sh.ptr[8]; res->nt = (int*)sh.ptr[9]; res->nnv = sh.ival[4]; res->nnt = sh.ival[5];
            res->n_pos_tris = n_pos; res->n_neg_tris = n_neg; res->n_cap = n_cap;
            res->n_loops = sh.ival[9]; res->n_boundary = nb; res->n_cross = n_u;
            tph[4] = clock64();
            for (int k = 0; k < 4; k++) res->cyc[k] = (unsigned)((tph[k + 1] - tph[k]) >> 6);
        }
        return;
    }
    }
fail_out:
    __syncthreads();
    if (tid == 0) {
        memset(res, 0, sizeof(CutResult));
        res->err = s_err ? s_err : KERR_PC_SCRATCH_OOM;
    }
#undef CUT_ALLOC
}
