// concave.cu — candidate planes: concave-edge planes and axis-aligned cuts
// (built with -fmad=false: the plane coefficients must round exactly as the
// checker's).
//
// Concave edges replace la_find_concave_edges (cuda/la_concave.cu:48-363;
// one warp, global-memory quicksort of 3T records, lane-0 consumption):
//   - directed edges as 64-bit keys (lo<<43 | hi<<22 | face), CTA bitonic
//     sort in global memory;
//   - one thread per sorted edge decides "first occurrence of a shared edge
//     whose dihedral exceeds the threshold" (la_concave.cu:160-234), with
//     the dihedral test done on cosines (no acos): valid iff d > 0 and
//     cos < cos(threshold - pi), or d <= 0 and cos > cos(pi - threshold);
//   - the valid edges are compacted in sorted order and fed to the same
//     seeded LCG reservoir (la_concave.cu:40-43,248-273) by one thread;
//   - planes are emitted in reservoir-slot order: face-offset n1, face-offset
//     n0, bisector +eps, bisector -eps (la_concave.cu:285-353).
// Axis cuts replace la_axis_cut_candidate + la_expand's plane placement
// (cuda/la_axis_cut.cuh:10-19, cuda/la_expand.cu:129-199).
#include <cmath>
#include <vector>
#include "context.cuh"
#include "cta_util.cuh"
#include "launch.h"

#define CC_NT 256

static cudaStream_t s_of(gpu_ctx* ctx) { return ctx->stream; }

struct ConcaveParams {
    int K;              // n_concave_edges
    float eps;
    int mode_pos; float cpos;   // d > 0 branch: 0 never, 1 always, 2 compare
    int mode_neg; float cneg;   // d <= 0 branch
};

static ConcaveParams concave_params(int K, float eps, float thr)
{
    ConcaveParams P;
    P.K = K; P.eps = eps;
    const double pi = 3.14159265358979;
    double xp = (double)thr - pi;
    if (xp < 0) P.mode_pos = 1; else if (xp >= pi) P.mode_pos = 0; else { P.mode_pos = 2; P.cpos = (float)cos(xp); }
    double xn = pi - (double)thr;
    if (xn <= 0) P.mode_neg = 0; else if (xn > pi) P.mode_neg = 1; else { P.mode_neg = 2; P.cneg = (float)cos(xn); }
    return P;
}

static __device__ int cc_face_normal(const float* v, const int* t, int f, float* n)
{
    const float* a = v + 3 * t[3 * f]; const float* b = v + 3 * t[3 * f + 1]; const float* c = v + 3 * t[3 * f + 2];
    float e1x = b[0] - a[0], e1y = b[1] - a[1], e1z = b[2] - a[2];
    float e2x = c[0] - a[0], e2y = c[1] - a[1], e2z = c[2] - a[2];
    float nx = fmaf(e1y, e2z, -(e1z * e2y));
    float ny = fmaf(e1z, e2x, -(e1x * e2z));
    float nz = fmaf(e1x, e2y, -(e1y * e2x));
    float len = sqrtf(fmaf(nz, nz, fmaf(ny, ny, nx * nx)));
    if (len < 1e-12f) return 0;
    n[0] = nx / len; n[1] = ny / len; n[2] = nz / len;
    return 1;
}

// One CTA per mesh.  keys, tmp: 3*nt u64 each; flags: 3*nt ints; res: 4*K
// ints.  Writes up to 4K planes and the count.  The directed edges are
// ordered by a stable LSD radix sort of their 64-bit keys (8 passes of 8
// bits; the keys are distinct, so the order is the keys' total order).
static __device__ void concave_cta(const float* __restrict__ v, int nv, const int* __restrict__ t, int nt,
                                   const ConcaveParams& P, unsigned long long* keys, unsigned long long* tmp,
                                   int* flags, int* res, float4* out, int* out_count)
{
    __shared__ int scan[34];
    __shared__ int s_nres;
    __shared__ int cnt[256 * (CC_NT / 32)];
    const int tid = threadIdx.x;
    const int nd = 3 * nt;
    if (nt < 2 || P.K <= 0) { if (tid == 0) *out_count = 0; return; }
    for (int i = tid; i < nd; i += CC_NT) {
        int f = i / 3, k = i % 3;
        int a = t[3 * f + k], b = t[3 * f + (k + 1) % 3];
        unsigned lo = (unsigned)min(a, b), hi = (unsigned)max(a, b);
        keys[i] = ((unsigned long long)lo << 43) | ((unsigned long long)hi << 22) | (unsigned long long)f;
    }
    __syncthreads();
    cta_radix_sort_u64<CC_NT>(keys, tmp, nd, 0, 64, cnt, scan);
    const unsigned long long EDGE = ~((1ull << 22) - 1);
    for (int i = tid; i < nd; i += CC_NT) {
        int valid = 0;
        if (i + 1 < nd) {
            unsigned long long k0 = keys[i], k1 = keys[i + 1];
            bool first = (i == 0) || ((keys[i - 1] & EDGE) != (k0 & EDGE));
            bool shared = ((k0 & EDGE) == (k1 & EDGE)) && ((k0 ^ k1) & ((1ull << 22) - 1));
            if (first && shared) {
                int v0 = (int)(k0 >> 43), v1 = (int)((k0 >> 22) & ((1u << 21) - 1));
                int f0 = (int)(k0 & ((1u << 22) - 1)), f1 = (int)(k1 & ((1u << 22) - 1));
                float n0[3], n1[3];
                if (cc_face_normal(v, t, f0, n0) && cc_face_normal(v, t, f1, n1)) {
                    float c = fmaf(n0[2], n1[2], fmaf(n0[1], n1[1], n0[0] * n1[0]));
                    c = fmaxf(-1.0f, fminf(1.0f, c));
                    int other = -1;
                    for (int k = 0; k < 3; k++) { int vv = t[3 * f0 + k]; if (vv != v0 && vv != v1) { other = vv; break; } }
                    if (other >= 0) {
                        float dx = v[3 * other] - v[3 * v0], dy = v[3 * other + 1] - v[3 * v0 + 1], dz = v[3 * other + 2] - v[3 * v0 + 2];
                        float d = fmaf(dz, n1[2], fmaf(dy, n1[1], dx * n1[0]));
                        if (d > 0.0f) valid = (P.mode_pos == 1) || (P.mode_pos == 2 && c < P.cpos);
                        else          valid = (P.mode_neg == 1) || (P.mode_neg == 2 && c > P.cneg);
                    }
                }
            }
        }
        flags[i] = valid;
    }
    __syncthreads();
    // compact valid positions in sorted order (flags -> exclusive positions)
    int n_valid = cta_scan_inplace(flags, nd, scan);
    // flags now holds positions; the valid ones are where flags[i+1] > flags[i]
    // (or i = nd-1 with flags[i] < n_valid).  Reservoir by one thread.
    if (tid == 0) {
        int n_seen = 0, n_res = 0;
        unsigned rng = 1u;
        for (int i = 0; i < 4 * P.K; i++) res[i] = -1;
        for (int i = 0; i < nd && n_seen < n_valid; i++) {
            int nextpos = (i + 1 < nd) ? flags[i + 1] : n_valid;
            if (nextpos == flags[i]) continue;            // not valid
            unsigned long long k0 = keys[i], k1 = keys[i + 1];
            int v0 = (int)(k0 >> 43), v1 = (int)((k0 >> 22) & ((1u << 21) - 1));
            int f0 = (int)(k0 & ((1u << 22) - 1)), f1 = (int)(k1 & ((1u << 22) - 1));
            n_seen++;
            if (n_res < P.K) {
                int s = n_res++;
                res[4 * s] = v0; res[4 * s + 1] = v1; res[4 * s + 2] = f0; res[4 * s + 3] = f1;
            } else {
                rng = rng * 1664525u + 1013904223u;
                unsigned th = (unsigned)((float)P.K / (float)n_seen * 4294967295.0f);
                if (rng < th) {
                    rng = rng * 1664525u + 1013904223u;
                    int s = (int)(rng % (unsigned)P.K);
                    res[4 * s] = v0; res[4 * s + 1] = v1; res[4 * s + 2] = f0; res[4 * s + 3] = f1;
                }
            }
        }
        s_nres = n_res;
    }
    __syncthreads();
    // planes: slot order; count per slot first (2 or 4), then write
    const int n_res = s_nres;
    __shared__ int s_cnt[1024];
    for (int s = tid; s < n_res; s += CC_NT) {
        int f0 = res[4 * s + 2], f1 = res[4 * s + 3];
        float n0[3], n1[3];
        int c = 0;
        if (cc_face_normal(v, t, f0, n0) && cc_face_normal(v, t, f1, n1)) {
            c = 2;
            float bx = n0[0] + n1[0], by = n0[1] + n1[1], bz = n0[2] + n1[2];
            float bl = sqrtf(fmaf(bz, bz, fmaf(by, by, bx * bx)));
            if (bl >= 1e-4f) c = 4;
        }
        s_cnt[s] = c;
    }
    __syncthreads();
    if (tid == 0) {
        int acc = 0;
        for (int s = 0; s < n_res; s++) { int c = s_cnt[s]; s_cnt[s] = acc; acc += c; }
        *out_count = acc;
    }
    __syncthreads();
    for (int s = tid; s < n_res; s += CC_NT) {
        int v0 = res[4 * s], v1 = res[4 * s + 1], f0 = res[4 * s + 2], f1 = res[4 * s + 3];
        float n0[3], n1[3];
        if (!cc_face_normal(v, t, f0, n0) || !cc_face_normal(v, t, f1, n1)) continue;
        float mx = (v[3 * v0] + v[3 * v1]) * 0.5f, my = (v[3 * v0 + 1] + v[3 * v1 + 1]) * 0.5f, mz = (v[3 * v0 + 2] + v[3 * v1 + 2]) * 0.5f;
        int o = s_cnt[s];
        out[o]     = make_float4(n1[0], n1[1], n1[2], -(fmaf(n1[2], mz, fmaf(n1[1], my, n1[0] * mx)) + P.eps));
        out[o + 1] = make_float4(n0[0], n0[1], n0[2], -(fmaf(n0[2], mz, fmaf(n0[1], my, n0[0] * mx)) + P.eps));
        float bx = n0[0] + n1[0], by = n0[1] + n1[1], bz = n0[2] + n1[2];
        float bl = sqrtf(fmaf(bz, bz, fmaf(by, by, bx * bx)));
        if (bl >= 1e-4f) {
            bx = bx / bl; by = by / bl; bz = bz / bl;
            float bm = fmaf(bz, mz, fmaf(by, my, bx * mx));
            out[o + 2] = make_float4(bx, by, bz, -(bm + P.eps));
            out[o + 3] = make_float4(bx, by, bz, -(bm - P.eps));
        }
    }
    (void)nv;
}

__global__ void __launch_bounds__(CC_NT)
k_concave_planes(const float* __restrict__ v, int nv, const int* __restrict__ t, int nt, ConcaveParams P,
                 unsigned long long* keys, unsigned long long* tmp, int* flags, int* res, float4* out, int* out_count)
{
    concave_cta(v, nv, t, nt, P, keys, tmp, flags, res, out, out_count);
}

// Several meshes, one CTA each (the lookahead's cutting parts).
struct ConcaveJob {
    const float* v; const int* t; int nv, nt;
    unsigned long long* keys; unsigned long long* tmp; int* flags; int* res; float4* out; int* count;
};
__global__ void __launch_bounds__(CC_NT)
k_concave_planes_batch(const ConcaveJob* __restrict__ jobs, int n_jobs, ConcaveParams P)
{
    if ((int)blockIdx.x >= n_jobs) return;
    const ConcaveJob J = jobs[blockIdx.x];
    concave_cta(J.v, J.nv, J.t, J.nt, P, J.keys, J.tmp, J.flags, J.res, J.out, J.count);
}

// Axis cuts: bbox reduction, then plane cut_idx of `width` per thread.
__global__ void __launch_bounds__(CC_NT)
k_axis_planes(const float* __restrict__ v, int nv, int width, float min_edge_dist, float4* out, int* valid)
{
    __shared__ float red[6][CC_NT / 32];
    __shared__ float lo[3], hi[3];
    float l[3] = {1e30f, 1e30f, 1e30f}, h[3] = {-1e30f, -1e30f, -1e30f};
    for (int i = threadIdx.x; i < nv; i += CC_NT)
        for (int k = 0; k < 3; k++) { float x = v[3 * i + k]; l[k] = fminf(l[k], x); h[k] = fmaxf(h[k], x); }
    for (int k = 0; k < 3; k++) { l[k] = warp_min(l[k]); h[k] = warp_max(h[k]); }
    if ((threadIdx.x & 31) == 0) for (int k = 0; k < 3; k++) { red[k][threadIdx.x >> 5] = l[k]; red[3 + k][threadIdx.x >> 5] = h[k]; }
    __syncthreads();
    if (threadIdx.x < 3) {
        int k = threadIdx.x;
        float a = 1e30f, b = -1e30f;
        for (int w = 0; w < CC_NT / 32; w++) { a = fminf(a, red[k][w]); b = fmaxf(b, red[3 + k][w]); }
        lo[k] = a; hi[k] = b;
    }
    __syncthreads();
    for (int ci = threadIdx.x; ci < width; ci += CC_NT) {
        int count = width / 3, rem = width % 3;
        int xc = count + (rem > 0), yc = count + (rem > 1);
        int axis, slice, cpa;
        if (ci < xc) { axis = 0; slice = ci; cpa = xc; }
        else if (ci < xc + yc) { axis = 1; slice = ci - xc; cpa = yc; }
        else { axis = 2; slice = ci - xc - yc; cpa = count; }
        float lv = lo[axis] + min_edge_dist, hv = hi[axis] - min_edge_dist;
        if (lv >= hv) { out[ci] = make_float4(0.f, 0.f, 0.f, 0.f); valid[ci] = 0; continue; }
        float frac = ((float)slice + 1.0f) / ((float)cpa + 1.0f);
        float cut = fmaf(frac, hv - lv, lv);
        out[ci] = make_float4(axis == 0 ? 1.f : 0.f, axis == 1 ? 1.f : 0.f, axis == 2 ? 1.f : 0.f, -cut);
        valid[ci] = 1;
    }
}

extern "C" int cuacd_candidate_planes(gpu_ctx_t ctx, const float* verts, int nv, const int* tris, int nt,
                                      int n_concave_edges, float concave_eps, float concave_threshold,
                                      int width, float min_edge_dist, float* out_planes, int* out_n_concave,
                                      int* out_axis_valid)
{
    if (!ctx) return -1;
    if (nv <= 0 || nt < 0) return ctx_fail(ctx, KERR_MESH_INVALID, "empty mesh");
    if (nv >= (1 << 21) || nt >= (1 << 22)) return ctx_fail(ctx, KERR_MESH_INVALID, "mesh too large for edge keys");
    if (n_concave_edges < 0 || n_concave_edges > 256 || width < 0) return ctx_fail(ctx, KERR_MESH_INVALID, "bad counts");
    for (int i = 0; i < 3 * nt; i++) if (tris[i] < 0 || tris[i] >= nv) return ctx_fail(ctx, KERR_MESH_INVALID, "index out of range");
    CK(cudaSetDevice(ctx->device));
    int nd = 3 * nt;
    int N = nd > 0 ? nd : 1;
    int K = n_concave_edges;
    size_t need = al256(12 * (size_t)nv) + al256(12 * (size_t)(nt > 0 ? nt : 1)) + 2 * al256(8 * (size_t)N)
                + al256(4 * (size_t)(nd > 0 ? nd : 1)) + al256(16 * (size_t)(4 * K + 1)) + al256(16 * (size_t)(4 * K + width + 1))
                + 2 * al256(4 * (size_t)(width + 2));
    int rc = pool_begin(ctx, need);
    if (rc) return rc;
    float* dv = pool_take<float>(ctx, 3 * (size_t)nv);
    int* dt = pool_take<int>(ctx, 3 * (size_t)(nt > 0 ? nt : 1));
    unsigned long long* dk = pool_take<unsigned long long>(ctx, N);
    unsigned long long* dk2 = pool_take<unsigned long long>(ctx, N);
    int* df = pool_take<int>(ctx, nd > 0 ? nd : 1);
    int* dr = pool_take<int>(ctx, 4 * (K + 1));
    float4* dp = pool_take<float4>(ctx, 4 * K + width + 1);
    int* dc = pool_take<int>(ctx, width + 2);
    cudaStream_t s = ctx->stream;
    CK(cudaMemcpyAsync(dv, verts, 12 * (size_t)nv, cudaMemcpyHostToDevice, s));
    if (nt) CK(cudaMemcpyAsync(dt, tris, 12 * (size_t)nt, cudaMemcpyHostToDevice, s));
    CK(cudaMemsetAsync(dc, 0, 4 * (size_t)(width + 2), s));
    ConcaveParams P = concave_params(K, concave_eps, concave_threshold);
    k_concave_planes<<<1, CC_NT, 0, s>>>(dv, nv, dt, nt, P, dk, dk2, df, dr, dp, dc);
    if (width > 0) k_axis_planes<<<1, CC_NT, 0, s>>>(dv, nv, width, min_edge_dist, dp + 4 * K, dc + 1);
    ctx->launches += 1 + (width > 0);
    CK(cudaGetLastError());
    int cnt = 0;
    CK(cudaMemcpyAsync(&cnt, dc, sizeof(int), cudaMemcpyDeviceToHost, s));
    rc = sync_and_check(ctx, "candidate_planes");
    if (rc) return rc;
    if (cnt > 0) CK(cudaMemcpy(out_planes, dp, 16 * (size_t)cnt, cudaMemcpyDeviceToHost));
    if (width > 0) {
        CK(cudaMemcpy(out_planes + 4 * cnt, dp + 4 * K, 16 * (size_t)width, cudaMemcpyDeviceToHost));
        if (out_axis_valid) CK(cudaMemcpy(out_axis_valid, dc + 1, 4 * (size_t)width, cudaMemcpyDeviceToHost));
    }
    *out_n_concave = cnt;
    return 0;
}

// Concave-edge planes of device-resident meshes, one CTA each, scratch
// carved from [scr, scr+cap) (in waves when it does not hold them all); the
// planes (at most 4*K per mesh) land in out[i].  Synchronises the stream.
// Used by the lookahead search for its cutting parts.
int concave_planes_device_batch(gpu_ctx* ctx, int n, const float* const* d_v, const int* nv, const int* const* d_t,
                                const int* nt, int K, float eps, float thr, char* scr, size_t cap,
                                std::vector<std::vector<float4>>& out)
{
    out.assign(n, std::vector<float4>());
    if (K <= 0 || n <= 0) return 0;
    ConcaveParams P = concave_params(K, eps, thr);
    auto part_bytes = [&](int i) -> size_t {
        const size_t nd = 3 * (size_t)(nt[i] > 0 ? nt[i] : 1);
        return 2 * al256(8 * nd) + al256(4 * nd) + al256(4 * (size_t)(4 * (K + 1))) + al256(16 * (size_t)(4 * K + 1))
             + al256(16);
    };
    const size_t job_bytes = al256(sizeof(ConcaveJob) * (size_t)n);
    if (job_bytes >= cap) return ctx_fail(ctx, KERR_HEAP_OOM, "concave planes: scratch too small");
    ConcaveJob* d_jobs = (ConcaveJob*)scr;
    int i0 = 0;
    while (i0 < n) {
        std::vector<ConcaveJob> jobs;
        char* p = scr + job_bytes;
        int i1 = i0;
        while (i1 < n) {
            const size_t b = part_bytes(i1);
            if ((size_t)(p - scr) + b > cap) break;
            ConcaveJob J;
            const size_t nd = 3 * (size_t)(nt[i1] > 0 ? nt[i1] : 1);
            J.v = d_v[i1]; J.t = d_t[i1]; J.nv = nv[i1]; J.nt = nt[i1];
            J.keys = (unsigned long long*)p; p += al256(8 * nd);
            J.tmp = (unsigned long long*)p; p += al256(8 * nd);
            J.flags = (int*)p; p += al256(4 * nd);
            J.res = (int*)p; p += al256(4 * (size_t)(4 * (K + 1)));
            J.out = (float4*)p; p += al256(16 * (size_t)(4 * K + 1));
            J.count = (int*)p; p += al256(16);
            if (nv[i1] >= (1 << 21) || nt[i1] >= (1 << 22))
                return ctx_fail(ctx, KERR_MESH_INVALID, "mesh too large for edge keys");
            jobs.push_back(J);
            i1++;
        }
        if (i1 == i0) return ctx_fail(ctx, KERR_HEAP_OOM, "concave planes need %zu scratch bytes, have %zu",
                                      part_bytes(i0) + job_bytes, cap);
        const int m = i1 - i0;
        CK(cudaMemcpyAsync(d_jobs, jobs.data(), sizeof(ConcaveJob) * m, cudaMemcpyHostToDevice, s_of(ctx)));
        k_concave_planes_batch<<<m, CC_NT, 0, s_of(ctx)>>>(d_jobs, m, P);
        ctx->launches += 1;
        CK(cudaGetLastError());
        std::vector<int> cnt(m);
        for (int k = 0; k < m; k++)
            CK(cudaMemcpyAsync(&cnt[k], jobs[k].count, sizeof(int), cudaMemcpyDeviceToHost, s_of(ctx)));
        CK(cudaStreamSynchronize(s_of(ctx)));
        for (int k = 0; k < m; k++) {
            if (cnt[k] > 4 * K) return ctx_fail(ctx, KERR_MESH_INVALID, "concave plane count %d above %d", cnt[k], 4 * K);
            out[i0 + k].resize(cnt[k]);
            if (cnt[k] > 0)
                CK(cudaMemcpyAsync(out[i0 + k].data(), jobs[k].out, 16 * (size_t)cnt[k], cudaMemcpyDeviceToHost,
                                   s_of(ctx)));
        }
        CK(cudaStreamSynchronize(s_of(ctx)));
        i0 = i1;
    }
    return 0;
}
