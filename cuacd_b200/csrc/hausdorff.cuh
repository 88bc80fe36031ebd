// hausdorff.cuh — sampled bidirectional Hausdorff distance (sm_100a).
//
// Replaces hausdorff_block (cuda/hausdorff.cuh:271-1478: one 256-thread block
// per pair, thread-0 serial prefix sums, global-memory 4-warp quicksort,
// Karras LBVH with one triangle per leaf, per-thread stack traversal).
//
// Sampling semantics are the reference's: per-surface budget
// res = max(min_samples, (int)(resolution * area)) (:368-397); per-triangle
// count floor(res/area * a_t) with the parity rule for zero counts
// (:433-466); Wang-hash barycentric samples (:517-558); result
// sqrt(max(d_ab^2, d_ba^2)) (:1453).  The area total is summed in 64-bit
// fixed point (2^-36) so every sample is independent of summation order.
//
// B200 layout:
//   prep  (one CTA per surface): areas, budget, sample offsets (CTA scan),
//         Morton order of triangle centroids (CTA bitonic sort), triangles
//         re-laid out in leaf order as 3 float4 (48 B), implicit binary BVH
//         over leaves of HD_LEAF triangles whose internal nodes hold BOTH
//         child boxes (one 64-byte node = two 16-byte box pairs), so a
//         traversal step is one cache line.
//   query (persistent CTAs, device work counter): each chunk of HD_CHUNK
//         samples of one direction; one thread per sample; nearest-triangle
//         search pruned by box distance AND by the pair's running maximum:
//         a sample stops as soon as its best distance is <= the maximum found
//         so far, since it can no longer raise the maximum.  The maximum
//         itself is therefore exact (every sample that could raise it is
//         searched to completion).
#pragma once
#include "common.cuh"
#include "cta_util.cuh"

#define HD_NT     256
#define HD_PREP_NT 1024           // threads of the per-surface prep CTA
#ifndef HD_LEAF
#define HD_LEAF   4               // triangles per BVH leaf
#endif
#define HD_CHUNK  1024
#define HD_STACK  48

struct HDSurf {            // input surface (device pointers, AoS xyz / int3)
    const float* v; const int* t; int nv, nt;
};

struct HDPrep {            // per-surface prep output
    int*    offsets;       // [nt+1] exclusive sample offsets (global scratch)
    float4* tri;           // [3 * nleaf * HD_LEAF] triangles in leaf order
    float4* node;          // [4 * P] child boxes per internal node (lo_l, hi_l, lo_r, hi_r)
    unsigned long long* keys;   // [pow2(nt)] leaf order: (first sample) << 32 | triangle
    int n_samples, res, P, nleaf;
    float area;
    int _pad;
};

static __device__ __forceinline__ unsigned hd_wang(unsigned s)
{
    s = (s ^ 61u) ^ (s >> 16);
    s *= 9u;
    s = s ^ (s >> 4);
    s *= 0x27d4eb2du;
    s = s ^ (s >> 15);
    return s;
}

// FP32 triangle area with the checker's operation order.
static __device__ __forceinline__ float hd_area(const float* v, int a, int b, int c)
{
    float abx = __fsub_rn(v[3 * b], v[3 * a]), aby = __fsub_rn(v[3 * b + 1], v[3 * a + 1]), abz = __fsub_rn(v[3 * b + 2], v[3 * a + 2]);
    float acx = __fsub_rn(v[3 * c], v[3 * a]), acy = __fsub_rn(v[3 * c + 1], v[3 * a + 1]), acz = __fsub_rn(v[3 * c + 2], v[3 * a + 2]);
    float nx = fmaf(aby, acz, -__fmul_rn(abz, acy));
    float ny = fmaf(abz, acx, -__fmul_rn(abx, acz));
    float nz = fmaf(abx, acy, -__fmul_rn(aby, acx));
    float s = fmaf(nz, nz, fmaf(ny, ny, __fmul_rn(nx, nx)));
    return __fmul_rn(0.5f, __fsqrt_rn(s));
}

static __device__ __forceinline__ int hd_tri_count(float at, int t, int nt, int res, float area)
{
    int area_count = (area > 1e-20f) ? __float2int_rz(__fmul_rn(__fdiv_rn((float)res, area), at)) : 0;
    if (nt > res) {
        int step = nt / res;
        return (area_count > 0) ? area_count : ((t % step == 0) ? 1 : 0);
    }
    return (area_count > 0) ? area_count : ((t % 2 == 0) ? 1 : 0);
}

// Sample k of triangle t (checker's exact FP32 sequence).
static __device__ __forceinline__ float3 hd_sample(const float* v, int a, int b, int c, int t, int k)
{
    unsigned ha = hd_wang((unsigned)t * 65537u + (unsigned)k);
    unsigned hb = hd_wang(ha + 0x9e3779b9u);
    float ra = __fdiv_rn((float)(ha & 0xFFFFFFu), (float)0xFFFFFFu);
    float rb = __fdiv_rn((float)(hb & 0xFFFFFFu), (float)0xFFFFFFu);
    float sqa = __fsqrt_rn(ra);
    float w0 = __fsub_rn(1.0f, sqa);
    float w1 = __fmul_rn(sqa, __fsub_rn(1.0f, rb));
    float w2 = __fmul_rn(sqa, rb);
    float3 p;
    p.x = fmaf(w2, v[3 * c],     fmaf(w1, v[3 * b],     __fmul_rn(w0, v[3 * a])));
    p.y = fmaf(w2, v[3 * c + 1], fmaf(w1, v[3 * b + 1], __fmul_rn(w0, v[3 * a + 1])));
    p.z = fmaf(w2, v[3 * c + 2], fmaf(w1, v[3 * b + 2], __fmul_rn(w0, v[3 * a + 2])));
    return p;
}

// Closest-point squared distance from p to triangle (a,b,c) by Voronoi regions.
static __device__ __forceinline__ float hd_pt_tri_d2(float3 p, float3 a, float3 b, float3 c)
{
    float3 ab = make_float3(b.x - a.x, b.y - a.y, b.z - a.z);
    float3 ac = make_float3(c.x - a.x, c.y - a.y, c.z - a.z);
    float3 ap = make_float3(p.x - a.x, p.y - a.y, p.z - a.z);
    float d1 = ab.x * ap.x + ab.y * ap.y + ab.z * ap.z;
    float d2 = ac.x * ap.x + ac.y * ap.y + ac.z * ap.z;
    float3 q;
    if (d1 <= 0.f && d2 <= 0.f) { q = a; goto done; }
    {
        float3 bp = make_float3(p.x - b.x, p.y - b.y, p.z - b.z);
        float d3 = ab.x * bp.x + ab.y * bp.y + ab.z * bp.z;
        float d4 = ac.x * bp.x + ac.y * bp.y + ac.z * bp.z;
        if (d3 >= 0.f && d4 <= d3) { q = b; goto done; }
        float vc = d1 * d4 - d3 * d2;
        if (vc <= 0.f && d1 >= 0.f && d3 <= 0.f) {
            float den = d1 - d3;
            float w = den > 0.f ? d1 / den : 0.f;
            q = make_float3(a.x + w * ab.x, a.y + w * ab.y, a.z + w * ab.z); goto done;
        }
        float3 cp = make_float3(p.x - c.x, p.y - c.y, p.z - c.z);
        float d5 = ab.x * cp.x + ab.y * cp.y + ab.z * cp.z;
        float d6 = ac.x * cp.x + ac.y * cp.y + ac.z * cp.z;
        if (d6 >= 0.f && d5 <= d6) { q = c; goto done; }
        float vb = d5 * d2 - d1 * d6;
        if (vb <= 0.f && d2 >= 0.f && d6 <= 0.f) {
            float den = d2 - d6;
            float w = den > 0.f ? d2 / den : 0.f;
            q = make_float3(a.x + w * ac.x, a.y + w * ac.y, a.z + w * ac.z); goto done;
        }
        float va = d3 * d6 - d5 * d4;
        if (va <= 0.f && (d4 - d3) >= 0.f && (d5 - d6) >= 0.f) {
            float den = (d4 - d3) + (d5 - d6);
            float w = den > 0.f ? (d4 - d3) / den : 0.f;
            q = make_float3(b.x + w * (c.x - b.x), b.y + w * (c.y - b.y), b.z + w * (c.z - b.z)); goto done;
        }
        float den = va + vb + vc;
        if (!(den > 0.f)) {          // degenerate triangle: nearest of its edges
            float best = 3.4e38f;
            float3 e[3][2] = {{a, b}, {b, c}, {c, a}};
            for (int i = 0; i < 3; i++) {
                float3 s0 = e[i][0], s1 = e[i][1];
                float3 d = make_float3(s1.x - s0.x, s1.y - s0.y, s1.z - s0.z);
                float3 w0 = make_float3(p.x - s0.x, p.y - s0.y, p.z - s0.z);
                float dd = d.x * d.x + d.y * d.y + d.z * d.z;
                float t = dd > 1e-30f ? (w0.x * d.x + w0.y * d.y + w0.z * d.z) / dd : 0.f;
                t = fminf(1.f, fmaxf(0.f, t));
                float3 r = make_float3(w0.x - t * d.x, w0.y - t * d.y, w0.z - t * d.z);
                best = fminf(best, r.x * r.x + r.y * r.y + r.z * r.z);
            }
            return best;
        }
        float inv = 1.f / den;
        float v_ = vb * inv, w_ = vc * inv;
        q = make_float3(a.x + ab.x * v_ + ac.x * w_, a.y + ab.y * v_ + ac.y * w_, a.z + ab.z * v_ + ac.z * w_);
    }
done:
    float dx = p.x - q.x, dy = p.y - q.y, dz = p.z - q.z;
    return dx * dx + dy * dy + dz * dz;
}

static __device__ __forceinline__ float hd_box_d2(float3 p, float4 lo, float4 hi)
{
    float dx = fmaxf(fmaxf(lo.x - p.x, 0.f), p.x - hi.x);
    float dy = fmaxf(fmaxf(lo.y - p.y, 0.f), p.y - hi.y);
    float dz = fmaxf(fmaxf(lo.z - p.z, 0.f), p.z - hi.z);
    return dx * dx + dy * dy + dz * dz;
}

static __device__ __forceinline__ unsigned hd_expand10(unsigned v)
{
    v = (v * 0x00010001u) & 0xFF0000FFu;
    v = (v * 0x00000101u) & 0x0F00F00Fu;
    v = (v * 0x00000011u) & 0xC30C30C3u;
    v = (v * 0x00000005u) & 0x49249249u;
    return v;
}

__host__ __device__ inline int hd_nleaf(int nt) { int l = (nt + HD_LEAF - 1) / HD_LEAF; return l < 1 ? 1 : l; }
// Powers of two stop at 2^30: an int shift past it would wrap to zero and the
// loop would never end.  Callers bound nt far below that before sizing.
__host__ __device__ inline int hd_P(int nt) { int l = hd_nleaf(nt); int p = 1; while (p < l && p < (1 << 30)) p <<= 1; return p; }
__host__ __device__ inline int hd_keycap(int nt) { int p = 1; while (p < nt && p < (1 << 30)) p <<= 1; return p; }

// Scratch bytes for one surface's prep.
__host__ __device__ inline size_t hd_prep_bytes(int nt)
{
    size_t b = 0;
    b += ((sizeof(int) * ((size_t)nt + 1)) + 255) & ~(size_t)255;
    b += ((sizeof(float4) * 3 * (size_t)hd_nleaf(nt) * HD_LEAF) + 255) & ~(size_t)255;
    b += ((sizeof(float4) * 4 * (size_t)hd_P(nt)) + 255) & ~(size_t)255;
    b += ((sizeof(unsigned long long) * (size_t)hd_keycap(nt)) + 255) & ~(size_t)255;
    b += ((sizeof(float4) * 2 * (size_t)hd_P(nt)) + 255) & ~(size_t)255;   // leaf boxes (build)
    return b;
}

struct HDShared {
    int scan[34];
    long long fx[HD_PREP_NT / 32];
    float bb[6][HD_PREP_NT / 32];
    float lo[3], hi[3];
    long long fxsum;
    int cnt[256 * (HD_PREP_NT / 32)];     // radix-sort digit counts
};

// Prep one surface.  All HD_PREP_NT threads call.
static __device__ void hd_prep_cta(HDSurf S, char* scratch, float resolution, int min_samples, int total_override,
                            HDPrep* out, HDShared& sh)
{
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int nt = S.nt;
    char* p = scratch;
    HDPrep P;
    P.offsets = (int*)p;   p += ((sizeof(int) * ((size_t)nt + 1)) + 255) & ~(size_t)255;
    P.nleaf = hd_nleaf(nt);
    P.P = hd_P(nt);
    P.tri = (float4*)p;    p += ((sizeof(float4) * 3 * (size_t)P.nleaf * HD_LEAF) + 255) & ~(size_t)255;
    P.node = (float4*)p;   p += ((sizeof(float4) * 4 * (size_t)P.P) + 255) & ~(size_t)255;
    P.keys = (unsigned long long*)p; p += ((sizeof(unsigned long long) * (size_t)hd_keycap(nt)) + 255) & ~(size_t)255;
    float4* lbox = (float4*)p;   // 2 per leaf slot
    if (nt <= 0 || S.nv <= 0) {
        if (tid == 0) { P.n_samples = 0; P.res = 0; P.area = 0.f; *out = P; }
        return;
    }
    // ---- areas (fixed point) and bbox of the triangles' vertices
    long long fx = 0;
    float lo[3] = {3.4e38f, 3.4e38f, 3.4e38f}, hi[3] = {-3.4e38f, -3.4e38f, -3.4e38f};
    for (int t = tid; t < nt; t += HD_PREP_NT) {
        int a = S.t[3 * t], b = S.t[3 * t + 1], c = S.t[3 * t + 2];
        float ar = hd_area(S.v, a, b, c);
        fx += __double2ll_rn(ldexp((double)ar, 36));
        int vv[3] = {a, b, c};
        for (int j = 0; j < 3; j++)
            for (int k = 0; k < 3; k++) { float x = S.v[3 * vv[j] + k]; lo[k] = fminf(lo[k], x); hi[k] = fmaxf(hi[k], x); }
    }
    for (int o = 16; o > 0; o >>= 1) fx += __shfl_xor_sync(FULL_MASK, fx, o);
    for (int k = 0; k < 3; k++) { lo[k] = warp_min(lo[k]); hi[k] = warp_max(hi[k]); }
    if (lane == 0) { sh.fx[w] = fx; for (int k = 0; k < 3; k++) { sh.bb[k][w] = lo[k]; sh.bb[3 + k][w] = hi[k]; } }
    __syncthreads();
    if (tid == 0) {
        long long s = 0;
        for (int i = 0; i < HD_PREP_NT / 32; i++) s += sh.fx[i];
        sh.fxsum = s;
        for (int k = 0; k < 3; k++) {
            float a = 3.4e38f, b = -3.4e38f;
            for (int i = 0; i < HD_PREP_NT / 32; i++) { a = fminf(a, sh.bb[k][i]); b = fmaxf(b, sh.bb[3 + k][i]); }
            sh.lo[k] = a; sh.hi[k] = b;
        }
    }
    __syncthreads();
    double total = ldexp((double)sh.fxsum, -36);
    int res = total_override > 0 ? total_override : (int)((double)resolution * total);
    if (res < min_samples) res = min_samples;
    float area = (float)total;
    // ---- per-triangle counts -> offsets
    for (int t = tid; t < nt; t += HD_PREP_NT) {
        int a = S.t[3 * t], b = S.t[3 * t + 1], c = S.t[3 * t + 2];
        P.offsets[t] = hd_tri_count(hd_area(S.v, a, b, c), t, nt, res, area);
    }
    __syncthreads();
    int n_samples = cta_scan_inplace(P.offsets, nt, sh.scan);
    if (tid == 0) P.offsets[nt] = n_samples;
    // ---- Morton order of centroids
    float ext[3], inv[3];
    for (int k = 0; k < 3; k++) { ext[k] = sh.hi[k] - sh.lo[k]; inv[k] = ext[k] > 0.f ? 1023.0f / ext[k] : 0.f; }
    for (int t = tid; t < nt; t += HD_PREP_NT) {
        int a = S.t[3 * t], b = S.t[3 * t + 1], c = S.t[3 * t + 2];
        unsigned m = 0;
        unsigned q[3];
        for (int k = 0; k < 3; k++) {
            float cen = (S.v[3 * a + k] + S.v[3 * b + k] + S.v[3 * c + k]) * (1.0f / 3.0f);
            float u = (cen - sh.lo[k]) * inv[k];
            q[k] = (unsigned)fminf(fmaxf(u, 0.f), 1023.f);
        }
        m = (hd_expand10(q[0]) << 2) | (hd_expand10(q[1]) << 1) | hd_expand10(q[2]);
        P.keys[t] = ((unsigned long long)m << 32) | (unsigned)t;
    }
    __syncthreads();
    // stable radix sort by the 30-bit code (bits 32..61); the leaf triangle
    // array (48 bytes per slot, written below) is its second buffer
    cta_radix_sort_u64<HD_PREP_NT>(P.keys, (unsigned long long*)P.tri, nt, 32, 30, sh.cnt, sh.scan);
    // ---- triangles in leaf order; empty slots become far-away degenerate points
    const int nslot = P.nleaf * HD_LEAF;
    for (int i = tid; i < nslot; i += HD_PREP_NT) {
        float4 A, B, C;
        if (i < nt) {
            int t = (int)(P.keys[i] & 0xffffffffu);
            int a = S.t[3 * t], b = S.t[3 * t + 1], c = S.t[3 * t + 2];
            A = make_float4(S.v[3 * a], S.v[3 * a + 1], S.v[3 * a + 2], 0.f);
            B = make_float4(S.v[3 * b], S.v[3 * b + 1], S.v[3 * b + 2], 0.f);
            C = make_float4(S.v[3 * c], S.v[3 * c + 1], S.v[3 * c + 2], 0.f);
        } else {
            A = B = C = make_float4(1e30f, 1e30f, 1e30f, 0.f);
        }
        P.tri[3 * i] = A; P.tri[3 * i + 1] = B; P.tri[3 * i + 2] = C;
    }
    __syncthreads();
    // ---- leaf boxes, then internal nodes holding both child boxes
    for (int l = tid; l < P.P; l += HD_PREP_NT) {
        float4 blo = make_float4(3.4e38f, 3.4e38f, 3.4e38f, 0.f), bhi = make_float4(-3.4e38f, -3.4e38f, -3.4e38f, 0.f);
        if (l < P.nleaf) {
            for (int j = 0; j < HD_LEAF; j++) {
                int i = l * HD_LEAF + j;
                if (i >= nt) break;
                for (int k = 0; k < 3; k++) {
                    float4 X = P.tri[3 * i + k];
                    blo.x = fminf(blo.x, X.x); blo.y = fminf(blo.y, X.y); blo.z = fminf(blo.z, X.z);
                    bhi.x = fmaxf(bhi.x, X.x); bhi.y = fmaxf(bhi.y, X.y); bhi.z = fmaxf(bhi.z, X.z);
                }
            }
        }
        lbox[2 * l] = blo; lbox[2 * l + 1] = bhi;
    }
    __syncthreads();
    // node n (1 <= n < P) children 2n, 2n+1; boxes of level below live in
    // lbox (leaves) or in the parents' child slots already written.
    for (int width = P.P >> 1; width >= 1; width >>= 1) {
        for (int j = tid; j < width; j += HD_PREP_NT) {
            int n = width + j;
            int cl = 2 * n, cr = 2 * n + 1;
            float4 llo, lhi, rlo, rhi;
            if (cl >= P.P) {
                llo = lbox[2 * (cl - P.P)]; lhi = lbox[2 * (cl - P.P) + 1];
                rlo = lbox[2 * (cr - P.P)]; rhi = lbox[2 * (cr - P.P) + 1];
            } else {
                float4 a0 = P.node[4 * cl], a1 = P.node[4 * cl + 1], a2 = P.node[4 * cl + 2], a3 = P.node[4 * cl + 3];
                llo = make_float4(fminf(a0.x, a2.x), fminf(a0.y, a2.y), fminf(a0.z, a2.z), 0.f);
                lhi = make_float4(fmaxf(a1.x, a3.x), fmaxf(a1.y, a3.y), fmaxf(a1.z, a3.z), 0.f);
                float4 b0 = P.node[4 * cr], b1 = P.node[4 * cr + 1], b2 = P.node[4 * cr + 2], b3 = P.node[4 * cr + 3];
                rlo = make_float4(fminf(b0.x, b2.x), fminf(b0.y, b2.y), fminf(b0.z, b2.z), 0.f);
                rhi = make_float4(fmaxf(b1.x, b3.x), fmaxf(b1.y, b3.y), fmaxf(b1.z, b3.z), 0.f);
            }
            P.node[4 * n] = llo; P.node[4 * n + 1] = lhi; P.node[4 * n + 2] = rlo; P.node[4 * n + 3] = rhi;
        }
        __syncthreads();
    }
    if (P.P == 1 && tid == 0) {      // single leaf: node 1's "children" are that leaf and an empty box
        P.node[4] = lbox[0]; P.node[5] = lbox[1];
        P.node[6] = make_float4(3.4e38f, 3.4e38f, 3.4e38f, 0.f); P.node[7] = make_float4(-3.4e38f, -3.4e38f, -3.4e38f, 0.f);
    }
    __syncthreads();
    // sample enumeration in leaf (Morton) order, so neighbouring query
    // threads take neighbouring samples: keys[i] <- (first sample of sorted
    // triangle i) << 32 | triangle.  The leaf boxes are dead by now and hold
    // the counts for the scan.
    {
        int* cnt_s = (int*)lbox;
        for (int i = tid; i < nt; i += HD_PREP_NT) {
            const int t = (int)(P.keys[i] & 0xffffffffull);
            cnt_s[i] = P.offsets[t + 1] - P.offsets[t];
        }
        __syncthreads();
        cta_scan_inplace(cnt_s, nt, sh.scan);
        for (int i = tid; i < nt; i += HD_PREP_NT)
            P.keys[i] = ((unsigned long long)(unsigned)cnt_s[i] << 32) | (P.keys[i] & 0xffffffffull);
    }
    if (tid == 0) { P.n_samples = n_samples; P.res = res; P.area = area; *out = P; }
    __syncthreads();
}

// Exact nearest squared distance from q to the surface in `P`, stopping
// early once best <= stop (then the returned value is <= stop).
static __device__ __forceinline__ float hd_nearest(const HDPrep& P, float3 q, float stop)
{
    float best = 3.4e38f;
    int   stk_n[HD_STACK];
    float stk_d[HD_STACK];
    int sp = 0;
    int node = 1;
    if (P.P == 1) {
        // one leaf: test directly
        for (int j = 0; j < HD_LEAF; j++) {
            float4 A = P.tri[3 * j], B = P.tri[3 * j + 1], C = P.tri[3 * j + 2];
            if (A.x >= 1e29f) break;
            best = fminf(best, hd_pt_tri_d2(q, make_float3(A.x, A.y, A.z), make_float3(B.x, B.y, B.z), make_float3(C.x, C.y, C.z)));
        }
        return best;
    }
    for (;;) {
        if (node >= P.P) {
            int base = (node - P.P) * HD_LEAF;
            #pragma unroll
            for (int j = 0; j < HD_LEAF; j++) {
                float4 A = __ldg(&P.tri[3 * (base + j)]), B = __ldg(&P.tri[3 * (base + j) + 1]), C = __ldg(&P.tri[3 * (base + j) + 2]);
                if (A.x < 1e29f)
                    best = fminf(best, hd_pt_tri_d2(q, make_float3(A.x, A.y, A.z), make_float3(B.x, B.y, B.z), make_float3(C.x, C.y, C.z)));
            }
            if (best <= stop) return best;
        } else {
            float4 llo = __ldg(&P.node[4 * node]), lhi = __ldg(&P.node[4 * node + 1]);
            float4 rlo = __ldg(&P.node[4 * node + 2]), rhi = __ldg(&P.node[4 * node + 3]);
            float dl = hd_box_d2(q, llo, lhi), dr = hd_box_d2(q, rlo, rhi);
            bool vl = dl < best && llo.x <= lhi.x, vr = dr < best && rlo.x <= rhi.x;
            if (vl && vr) {
                int nn = dl <= dr ? 2 * node : 2 * node + 1;
                int ff = dl <= dr ? 2 * node + 1 : 2 * node;
                if (sp < HD_STACK) { stk_n[sp] = ff; stk_d[sp] = fmaxf(dl, dr); sp++; }
                node = nn;
                continue;
            }
            if (vl) { node = 2 * node; continue; }
            if (vr) { node = 2 * node + 1; continue; }
        }
        // pop
        bool found = false;
        while (sp > 0) {
            sp--;
            if (stk_d[sp] < best) { node = stk_n[sp]; found = true; break; }
        }
        if (!found) break;
    }
    return best;
}

// One query direction: the samples of surface src against surface dst, for
// pair `pair`; its chunks start at chunk0 of the launch's chunk sequence.
struct HDDir { int src, dst, pair, n_samples, chunk0; };

// Queries.  Each CTA takes chunks of HD_CHUNK samples from the device
// counter; inside a chunk every lane is persistent: it takes the next sample
// from the chunk as soon as its own search ends, so lanes do not wait for
// the warp's longest search.  Each round of a warp walks internal BVH nodes
// until every searching lane stands at a leaf, then tests those leaves
// together.  A search stops once its best distance is <= the pair's running
// maximum (refreshed at every leaf); only finished searches above that
// maximum raise it, so the final maximum is exact, whatever the order.
static __device__ void hd_query_body(const HDSurf* __restrict__ surfs, const HDPrep* __restrict__ preps,
                                     const HDDir* __restrict__ dirs, int n_dirs, const int* total_chunks, int* counter,
                                     float* pair_max)
{
    __shared__ int s_chunk, s_next, s_a0;
    __shared__ int s_pos[HD_CHUNK];              // sorted triangle position of each sample of the chunk
    const int total = *total_chunks;
    for (;;) {
        if (threadIdx.x == 0) { s_chunk = atomicAdd(counter, 1); s_next = 0; }
        __syncthreads();
        const int c = s_chunk;
        if (c >= total) break;
        int lo = 0, hi = n_dirs;                 // last dir with chunk0 <= c
        while (hi - lo > 1) { int m = (lo + hi) >> 1; if (dirs[m].chunk0 <= c) lo = m; else hi = m; }
        while (lo + 1 < n_dirs && dirs[lo + 1].chunk0 <= c && dirs[lo].n_samples == 0) lo++;
        const HDDir D = dirs[lo];
        const HDSurf S = surfs[D.src];
        const HDPrep& PS = preps[D.src];
        const HDPrep PD = preps[D.dst];
        const int s0 = (c - D.chunk0) * HD_CHUNK;
        const int n_chunk = min(HD_CHUNK, D.n_samples - s0);
        volatile float* vmax = pair_max + D.pair;
        // map the chunk's samples to sorted triangle positions: the samples
        // run in leaf order, so the chunk covers a contiguous position range
        // starting at the last position whose first sample is <= s0
        if (threadIdx.x == 0) {
            int a = 0, b = S.nt;
            while (b - a > 1) { int m = (a + b) >> 1; if ((int)(PS.keys[m] >> 32) <= s0) a = m; else b = m; }
            s_a0 = a;
        }
        __syncthreads();
        for (int i = s_a0 + threadIdx.x; i < S.nt; i += HD_NT) {
            const int f = (int)(PS.keys[i] >> 32);
            if (f >= s0 + n_chunk) break;            // first samples grow with i
            const int g = i + 1 < S.nt ? (int)(PS.keys[i + 1] >> 32) : D.n_samples;
            for (int x = max(f, s0); x < min(g, s0 + n_chunk); x++) s_pos[x - s0] = i;
        }
        __syncthreads();
        bool has = false, root_after = false;
        float3 q = make_float3(0.f, 0.f, 0.f);
        float best = 0.f, stop = 0.f;
        int node = 1, sp = 0;
        int bl = -1, last_leaf = -1;                 // leaf of the current / previous best triangle
        // min distance from q to the triangles of leaf l
        auto leaf_d2 = [&](int l) {
            float d = 3.4e38f;
            const int base = l * HD_LEAF;
            #pragma unroll
            for (int jj = 0; jj < HD_LEAF; jj++) {
                float4 A = __ldg(&PD.tri[3 * (base + jj)]), B = __ldg(&PD.tri[3 * (base + jj) + 1]);
                float4 C = __ldg(&PD.tri[3 * (base + jj) + 2]);
                if (A.x < 1e29f)
                    d = fminf(d, hd_pt_tri_d2(q, make_float3(A.x, A.y, A.z), make_float3(B.x, B.y, B.z),
                                              make_float3(C.x, C.y, C.z)));
            }
            return d;
        };
        int   stk_n[HD_STACK];
        float stk_d[HD_STACK];
        // search complete: best is the nearest distance
        auto finish = [&]() {
            if (best > stop) atomic_max_nonneg(pair_max + D.pair, best);
            has = false;
            last_leaf = bl;
        };
        // next node from the stack, or finish
        auto pop = [&]() {
            while (sp > 0) {
                sp--;
                if (stk_d[sp] < best) { node = stk_n[sp]; return; }
            }
            finish();
        };
        for (;;) {
            bool got = false;
            if (!has) {
                const int j = atomicAdd(&s_next, 1);
                if (j < n_chunk) {
                    got = true;
                    const int smp = s0 + j;
                    const unsigned long long kk = PS.keys[s_pos[j]];
                    const int t = (int)(kk & 0xffffffffull);
                    const int k = smp - (int)(kk >> 32);
                    q = hd_sample(S.v, S.t[3 * t], S.t[3 * t + 1], S.t[3 * t + 2], t, k);
                    best = 3.4e38f; stop = *vmax; sp = 0; has = true; bl = -1;
                    // the previous sample's nearest leaf first: its distance
                    // bounds this one's, and usually settles it at once; the
                    // search then starts at the root
                    root_after = last_leaf >= 0 && PD.P > 1;
                    node = root_after ? PD.P + last_leaf : 1;
                }
            }
            // every lane votes once per iteration; the vote is empty only when
            // every idle lane failed to take a sample: the chunk is done
            if (!__any_sync(FULL_MASK, has || got)) break;
            // Every lane, searching or not, goes on to the warp votes below
            // (a lane that skipped them would leave the others waiting in a
            // full-warp vote); PD is the chunk's, so the branch is uniform.
            if (PD.P == 1) {                             // one leaf: test it directly
                if (has) {
                    for (int jj = 0; jj < HD_LEAF; jj++) {
                        float4 A = PD.tri[3 * jj], B = PD.tri[3 * jj + 1], C = PD.tri[3 * jj + 2];
                        if (A.x >= 1e29f) break;
                        best = fminf(best, hd_pt_tri_d2(q, make_float3(A.x, A.y, A.z), make_float3(B.x, B.y, B.z),
                                                        make_float3(C.x, C.y, C.z)));
                    }
                    if (best > stop) atomic_max_nonneg(pair_max + D.pair, best);
                    has = false;
                }
                continue;
            }
            // Internal steps until every searching lane of the warp stands at
            // a leaf (or has finished), then one leaf step by all of them at
            // once: the leaf step -- HD_LEAF point-triangle distances -- is the
            // expensive one, and lanes would otherwise take it one branch
            // apart from the lanes stepping through internal nodes.
            while (__any_sync(FULL_MASK, has && node < PD.P)) {
                if (has && node < PD.P) {
                    float4 llo = __ldg(&PD.node[4 * node]), lhi = __ldg(&PD.node[4 * node + 1]);
                    float4 rlo = __ldg(&PD.node[4 * node + 2]), rhi = __ldg(&PD.node[4 * node + 3]);
                    float dl = hd_box_d2(q, llo, lhi), dr = hd_box_d2(q, rlo, rhi);
                    bool vl = dl < best && llo.x <= lhi.x, vr = dr < best && rlo.x <= rhi.x;
                    if (vl && vr) {
                        int nn = dl <= dr ? 2 * node : 2 * node + 1;
                        int ff = dl <= dr ? 2 * node + 1 : 2 * node;
                        if (sp < HD_STACK) { stk_n[sp] = ff; stk_d[sp] = fmaxf(dl, dr); sp++; }
                        node = nn;
                    } else if (vl) node = 2 * node;
                    else if (vr) node = 2 * node + 1;
                    else pop();
                }
            }
            if (has) {                                   // leaf step
                const float d = leaf_d2(node - PD.P);
                if (d < best) { best = d; bl = node - PD.P; }
                stop = fmaxf(stop, *vmax);
                if (best <= stop) { has = false; last_leaf = bl; }   // cannot raise the maximum
                else if (root_after) { root_after = false; node = 1; }
                else pop();
            }
        }
        __syncthreads();                             // chunk done before s_chunk / s_next change
    }
}
