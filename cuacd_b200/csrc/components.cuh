// components.cuh — split a mesh into its vertex-connected components, one
// CTA per mesh (replaces decompose_components_block, cuda/postprocess.cuh:139-527,
// as used by la_decompose_components, cuda/la_lifecycle.cu:310-407).
//
//   1. union-find over triangle edges: a root is always linked under the
//      smaller root with atomicCAS, so the final root of a component is its
//      smallest vertex and the labels do not depend on scheduling;
//   2. components are numbered by their smallest vertex (the reference's
//      sequential numbering, postprocess.cuh:258-270); a mesh with one
//      component is left alone;
//   3. vertices and triangles are written grouped by component, in input
//      order inside each component (a stable partition: per-warp counts, a
//      CTA scan, then warp-match ranks) — the reference scatters with
//      atomics, so its order inside a component is arbitrary;
//   4. each component's signed volume (FP64, anchored at its first vertex);
//      components with negative volume are unreachable inner shells and are
//      dropped when outer shells exist too (postprocess.cuh:449-495).
// Vertices used by no triangle belong to no component and are dropped (the
// reference keeps each as a zero-triangle component).
#pragma once
#include "common.cuh"
#include "cta_util.cuh"

#define CC_BLOCK 256
#define CC_WARPS (CC_BLOCK / 32)
#define CC_MAX_COMP 4096          // more components than this: the mesh stays whole

struct CompMesh { float* v; int* t; int nv, nt; double vol; };

struct CompResult {
    int n;                 // components written (0: the mesh is one component)
    int err;
    CompMesh* comps;       // n entries (output arena)
};

// Scratch bound: two per-vertex arrays + CC_WARPS counters and two starts per component.
__host__ __device__ inline size_t cc_scratch_bytes(int nv)
{
    size_t c = (size_t)(nv < CC_MAX_COMP ? nv : CC_MAX_COMP) + 1;
    return 8 * (size_t)nv + 4 * (CC_WARPS + 2) * c + 8 * 256;
}
// Output bound: component vertices, triangles and descriptors.
__host__ __device__ inline size_t cc_output_bytes(int nv, int nt)
{
    size_t c = (size_t)(nv < CC_MAX_COMP ? nv : CC_MAX_COMP);
    return 12 * (size_t)nv + 12 * (size_t)nt + sizeof(CompMesh) * c + 4 * 256;
}

static __device__ __forceinline__ int cc_find(int* parent, int x)
{
    for (int guard = 0; guard < (1 << 26); guard++) {
        int p = __ldcg(&parent[x]);
        if (p == x) return x;
        int gp = __ldcg(&parent[p]);
        if (gp != p) atomicCAS(&parent[x], p, gp);   // path halving; gp is still an ancestor
        x = p;
    }
    return x;
}

static __device__ __forceinline__ void cc_union(int* parent, int a, int b)
{
    for (int guard = 0; guard < (1 << 26); guard++) {
        a = cc_find(parent, a);
        b = cc_find(parent, b);
        if (a == b) return;
        if (a < b) { int t = a; a = b; b = t; }      // the larger root goes under the smaller
        if (atomicCAS(&parent[a], a, b) == a) return;
    }
}

// Stable partition of [0, n) by key(i) in [-1, C) (-1: dropped): emit(i, k, p)
// receives the position p of i in (key, index) order.  `cnt` holds
// CC_WARPS*C ints, `start` C+1 ints (start[k] = first position of key k).
// Whole CTA.
template <class Key, class Emit>
static __device__ void cc_stable_partition(int n, int C, Key key, Emit emit, int* cnt, int* start, int* sh_scan)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int seg = (n + CC_WARPS - 1) / CC_WARPS;
    const int b = min(n, w * seg), e = min(n, b + seg);
    for (int c = threadIdx.x; c < CC_WARPS * C; c += CC_BLOCK) cnt[c] = 0;
    __syncthreads();
    for (int i = b + lane; i < e; i += 32) {
        int k = key(i);
        if (k >= 0) atomicAdd(&cnt[k * CC_WARPS + w], 1);
    }
    __syncthreads();
    const int total = cta_scan_inplace(cnt, CC_WARPS * C, sh_scan);
    for (int c = threadIdx.x; c < C; c += CC_BLOCK) start[c] = cnt[c * CC_WARPS];
    if (threadIdx.x == 0) start[C] = total;
    __syncthreads();
    for (int base = b; base < e; base += 32) {       // warp-uniform trip count
        const int i = base + lane;
        const int k = i < e ? key(i) : -2;
        const unsigned m = __match_any_sync(0xffffffffu, k);
        const int rank = __popc(m & ((1u << lane) - 1u));
        int p = 0;
        if (k >= 0) p = __ldcg(&cnt[k * CC_WARPS + w]) + rank;
        __syncwarp();
        if (k >= 0 && rank == 0) cnt[k * CC_WARPS + w] += __popc(m);
        __syncwarp();
        if (k >= 0) emit(i, k, p);
    }
    __syncthreads();
}

// All CC_BLOCK threads call.  Scratch from `scr`, components from `out`.
static __device__ void components_cta(const float* __restrict__ v, int nv, const int* __restrict__ t, int nt,
                                      Arena* scr, Arena* out, CompResult* res)
{
    __shared__ int s_err, s_scan[34];
    __shared__ int* s_parent;
    __shared__ int* s_aux;
    __shared__ int* s_cnt;
    __shared__ int* s_vstart;
    __shared__ int* s_tstart;
    __shared__ CompMesh* s_comps;
    __shared__ float* s_ov;
    __shared__ int* s_ot;
    const int tid = threadIdx.x;
    if (nv <= 0 || nt <= 0) {
        if (tid == 0) { res->n = 0; res->err = 0; res->comps = nullptr; }
        return;
    }
    if (tid == 0) {
        s_err = 0;
        s_parent = (int*)arena_alloc(scr, 4ull * nv, &s_err);
        s_aux = (int*)arena_alloc(scr, 4ull * nv, &s_err);
    }
    __syncthreads();
    if (s_err) {
        if (tid == 0) { res->n = 0; res->err = s_err | KERR_DC_OOM; res->comps = nullptr; }
        return;
    }
    int* parent = s_parent;
    int* aux = s_aux;
    for (int i = tid; i < nv; i += CC_BLOCK) { parent[i] = i; aux[i] = 0; }
    __syncthreads();
    for (int i = tid; i < nt; i += CC_BLOCK) {
        const int a = t[3 * i], b = t[3 * i + 1], c = t[3 * i + 2];
        cc_union(parent, a, b);
        cc_union(parent, a, c);
    }
    __syncthreads();
    for (int i = tid; i < nt; i += CC_BLOCK) aux[cc_find(parent, t[3 * i])] = 1;   // roots in use
    __syncthreads();
    for (int i = tid; i < nv; i += CC_BLOCK) parent[i] = cc_find(parent, i);
    __syncthreads();
    const int C = cta_scan_inplace(aux, nv, s_scan);             // aux[root] = component number
    if (C <= 1 || C > CC_MAX_COMP) {
        if (tid == 0) { res->n = 0; res->err = 0; res->comps = nullptr; }
        return;
    }
    // parent[i] <- component of vertex i (-1: used by no triangle)
    for (int i = tid; i < nv; i += CC_BLOCK) {
        const int r = parent[i];
        const int nxt = r + 1 < nv ? aux[r + 1] : C;
        parent[i] = (nxt - aux[r]) ? aux[r] : -1;
    }
    if (tid == 0) {
        s_cnt = (int*)arena_alloc(scr, 4ull * CC_WARPS * C, &s_err);
        s_vstart = (int*)arena_alloc(scr, 4ull * (C + 1), &s_err);
        s_tstart = (int*)arena_alloc(scr, 4ull * (C + 1), &s_err);
        s_comps = (CompMesh*)arena_alloc(out, sizeof(CompMesh) * (unsigned long long)C, &s_err);
        s_ov = (float*)arena_alloc(out, 12ull * nv, &s_err);
        s_ot = (int*)arena_alloc(out, 12ull * nt, &s_err);
    }
    __syncthreads();
    if (s_err) {
        if (tid == 0) { res->n = 0; res->err = s_err | KERR_DC_OOM; res->comps = nullptr; }
        return;
    }
    float* ov = s_ov;
    int* ot = s_ot;
    // vertices: aux[i] <- output position
    cc_stable_partition(nv, C,
        [&](int i) { return parent[i]; },
        [&](int i, int k, int p) {
            ov[3 * p] = v[3 * i]; ov[3 * p + 1] = v[3 * i + 1]; ov[3 * p + 2] = v[3 * i + 2];
            aux[i] = p;
        },
        s_cnt, s_vstart, s_scan);
    const int* vstart = s_vstart;
    cc_stable_partition(nt, C,
        [&](int i) { return parent[t[3 * i]]; },
        [&](int i, int k, int p) {
            const int base = vstart[k];
            ot[3 * p] = aux[t[3 * i]] - base;
            ot[3 * p + 1] = aux[t[3 * i + 1]] - base;
            ot[3 * p + 2] = aux[t[3 * i + 2]] - base;
        },
        s_cnt, s_tstart, s_scan);
    // descriptors and signed volumes (one warp per component)
    const int lane = tid & 31, w = tid >> 5;
    for (int c = w; c < C; c += CC_WARPS) {
        CompMesh m;
        m.v = ov + 3 * (size_t)vstart[c];
        m.t = ot + 3 * (size_t)s_tstart[c];
        m.nv = vstart[c + 1] - vstart[c];
        m.nt = s_tstart[c + 1] - s_tstart[c];
        double acc = 0.0;
        const double ox = m.v[0], oy = m.v[1], oz = m.v[2];
        for (int i = lane; i < m.nt; i += 32) acc += tet6_d(m.v, m.t[3 * i], m.t[3 * i + 1], m.t[3 * i + 2], ox, oy, oz);
        acc = warp_sum_d(acc);
        m.vol = acc / 6.0;
        if (lane == 0) s_comps[c] = m;
    }
    __syncthreads();
    if (tid == 0) {
        int n_inner = 0;
        for (int c = 0; c < C; c++) n_inner += s_comps[c].vol < 0.0;
        const bool drop = n_inner > 0 && n_inner < C;
        int k = 0;
        for (int c = 0; c < C; c++) {
            CompMesh m = s_comps[c];
            if (drop && m.vol < 0.0) continue;
            m.vol = fabs(m.vol);
            s_comps[k++] = m;
        }
        res->n = k; res->err = 0; res->comps = s_comps;
    }
}
