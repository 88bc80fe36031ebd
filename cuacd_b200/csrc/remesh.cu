// remesh.cu — remesh front end on the GPU: gpu_preprocess (the reference's
// csrc/preprocess.h:17-24 / csrc/preprocess.c:605-726), a watertight,
// manifold, consistently oriented surface from any triangle soup.
//
// One launch per stage over a resolution-R grid of nodes (x fastest):
//   k_rm_norm        input vertices to grid units (FP64)
//   k_rm_init        distance far, boundary nodes outside, no crossings
//   k_rm_tris        one CTA per triangle: squared distance of the nodes in
//                    its 3-cell band (atomicMin on the float bits; every
//                    value is >= 0, so the bit order is the value order) and
//                    the grid edges it crosses, line by line on each axis
//   k_rm_sweep       one thread per grid line: outside spreads forward and
//                    back along the line through uncrossed edges; the host
//                    repeats the three axes until a round changes nothing
//   k_rm_field       signed, shifted field, in place of the distances
//   k_rm_edge_flags  crossed grid edges -> scan -> vertex ids
//   k_rm_cell_counts triangles and loop centres per cell -> two scans
//   k_rm_edge_verts  / k_rm_cells: vertices and triangles in scan order
// Every per-item computation is in remesh.cuh (shared with the CPU
// emulation test) and is checked value for value against the oracle.  This
// file is built with -fmad=false: every FP64 expression rounds as written.
#include <climits>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include "context.cuh"
#include "cta_util.cuh"
#include "remesh.cuh"

#define RM_NT 256
#define RM_SCAN_NT 512
#define RM_SCAN_PER 16
#define RM_SCAN_TILE (RM_SCAN_NT * RM_SCAN_PER)
#define RM_EINVAL 1                  // CUDA_ERROR_INVALID_VALUE, the reference's code for bad arguments

__constant__ RmTable c_rm_table;

static const RmTable& rm_table()
{
    static const RmTable t = [] { RmTable x; rm_build_table(x); return x; }();
    return t;
}

extern "C" void cuacd_remesh_case_table(int* out)
{
    // per case: nloop, 4 loop lengths, 12 edges (-1 padded) -- host only
    const RmTable& T = rm_table();
    for (int c = 0; c < 256; c++) {
        int* o = out + 17 * c;
        o[0] = T.nloop[c];
        for (int l = 0; l < RM_MAXLOOP; l++) o[1 + l] = T.len[c][l];
        for (int m = 0; m < RM_MAXEDGE; m++) o[5 + m] = T.edge[c][m];
    }
}

__global__ void k_rm_norm(const float* __restrict__ v, int nv, RmParams P, double* __restrict__ u)
{
    const long long n = 3ll * nv;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        u[i] = rm_norm(v[i], (int)(i % 3), P);
}

__global__ void k_rm_init(unsigned* __restrict__ d2, unsigned char* __restrict__ outside,
                          unsigned char* __restrict__ blk, int R)
{
    const long long N = (long long)R * R * R;
    for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < N; n += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(n % R), y = (int)(n / R % R), z = (int)(n / ((long long)R * R));
        d2[n] = RM_FAR;
        outside[n] = (x == 0 || y == 0 || z == 0 || x == R - 1 || y == R - 1 || z == R - 1) ? 1 : 0;
        blk[n] = 0; blk[N + n] = 0; blk[2 * N + n] = 0;
    }
}

__global__ void k_rm_tris(const double* __restrict__ u, const int* __restrict__ tris, int nt, int R,
                          unsigned* __restrict__ d2, unsigned char* __restrict__ blk)
{
    const long long N = (long long)R * R * R;
    for (int t = blockIdx.x; t < nt; t += gridDim.x) {
        double a[3], b[3], c[3];
        for (int k = 0; k < 3; k++) {
            a[k] = u[3ll * tris[3ll * t] + k];
            b[k] = u[3ll * tris[3ll * t + 1] + k];
            c[k] = u[3ll * tris[3ll * t + 2] + k];
        }
        int lo[3], hi[3];
        rm_tri_box(a, b, c, R, lo, hi);
        if (hi[0] >= lo[0] && hi[1] >= lo[1] && hi[2] >= lo[2]) {
            const long long nx = hi[0] - lo[0] + 1, ny = hi[1] - lo[1] + 1, nz = hi[2] - lo[2] + 1;
            const long long vol = nx * ny * nz;
            for (long long q = threadIdx.x; q < vol; q += blockDim.x) {
                const int x = lo[0] + (int)(q % nx), y = lo[1] + (int)(q / nx % ny), z = lo[2] + (int)(q / (nx * ny));
                const double p[3] = {(double)x, (double)y, (double)z};
                const double dd = rm_point_tri_d2(p, a, b, c);
                if (dd <= RM_BAND * RM_BAND) atomicMin(&d2[rm_lin(x, y, z, R)], __float_as_uint((float)dd));
            }
        }
        for (int k = 0; k < 3; k++) {
            if (rm_tri_area2(a, b, c, k) == 0) continue;
            int llo[2], lhi[2];
            rm_tri_lines(a, b, c, k, R, llo, lhi);
            if (lhi[0] < llo[0] || lhi[1] < llo[1]) continue;
            const long long na = lhi[0] - llo[0] + 1, nb = lhi[1] - llo[1] + 1;
            for (long long q = threadIdx.x; q < na * nb; q += blockDim.x) {
                const long long node = rm_line_cross(a, b, c, k, llo[0] + (int)(q % na), llo[1] + (int)(q / na), R);
                if (node >= 0) blk[k * N + node] = 1;
            }
        }
    }
}

__global__ void k_rm_sweep(unsigned char* __restrict__ outside, const unsigned char* __restrict__ blk, int R, int k,
                           int* changed)
{
    const long long line = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (line >= (long long)R * R) return;
    const int i = (k + 1) % 3, j = (k + 2) % 3;
    int q[3];
    q[k] = 0; q[i] = (int)(line % R); q[j] = (int)(line / R);
    const long long base = rm_lin(q[0], q[1], q[2], R);
    const long long st = k == 0 ? 1 : (k == 1 ? R : (long long)R * R);
    const unsigned char* bk = blk + (long long)k * R * R * R;
    bool ch = false;
    unsigned char prev = outside[base];
    for (int c = 1; c < R; c++) {
        const long long idx = base + c * st;
        if (!outside[idx] && prev && !bk[idx - st]) { outside[idx] = 1; ch = true; }
        prev = outside[idx];
    }
    prev = outside[base + (R - 1) * st];
    for (int c = R - 2; c >= 0; c--) {
        const long long idx = base + c * st;
        if (!outside[idx] && prev && !bk[idx]) { outside[idx] = 1; ch = true; }
        prev = outside[idx];
    }
    if (ch) *changed = 1;
}

__global__ void k_rm_field(unsigned* d2, const unsigned char* __restrict__ outside, long long N)
{
    float* sd = (float*)d2;
    for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < N; n += (long long)gridDim.x * blockDim.x)
        sd[n] = rm_field(d2[n], outside[n] != 0);
}

__device__ __forceinline__ bool rm_crossed(const float* sd, long long n, int x, int y, int z, int k, int R)
{
    const int q[3] = {x, y, z};
    if (q[k] > R - 2) return false;
    const long long st = k == 0 ? 1 : (k == 1 ? R : (long long)R * R);
    return (sd[n] < 0.0f) != (sd[n + st] < 0.0f);
}

__global__ void k_rm_edge_flags(const float* __restrict__ sd, int R, int* __restrict__ flag)
{
    const long long N = (long long)R * R * R;
    for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < N; n += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(n % R), y = (int)(n / R % R), z = (int)(n / ((long long)R * R));
        for (int k = 0; k < 3; k++) flag[3 * n + k] = rm_crossed(sd, n, x, y, z, k, R) ? 1 : 0;
    }
}

__global__ void k_rm_cell_counts(const float* __restrict__ sd, int R, int* __restrict__ ntri, int* __restrict__ nctr)
{
    const int Rc = R - 1;
    const long long C = (long long)Rc * Rc * Rc;
    for (long long m = blockIdx.x * (long long)blockDim.x + threadIdx.x; m < C; m += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(m % Rc), y = (int)(m / Rc % Rc), z = (int)(m / ((long long)Rc * Rc));
        const int cs = rm_case(sd, x, y, z, R);
        ntri[m] = c_rm_table.ntri[cs];
        nctr[m] = c_rm_table.nctr[cs];
    }
}

__global__ void k_rm_edge_verts(const float* __restrict__ sd, const int* __restrict__ vid, int R, RmParams P,
                                float* __restrict__ out_v)
{
    const long long N = (long long)R * R * R;
    for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < N; n += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(n % R), y = (int)(n / R % R), z = (int)(n / ((long long)R * R));
        for (int k = 0; k < 3; k++) {
            if (!rm_crossed(sd, n, x, y, z, k, R)) continue;
            double g[3];
            rm_edge_pos(sd, x, y, z, k, R, g);
            const long long v = vid[3 * n + k];
            for (int d = 0; d < 3; d++) out_v[3 * v + d] = rm_denorm(g[d], d, P);
        }
    }
}

__global__ void k_rm_cells(const float* __restrict__ sd, const int* __restrict__ vid, const int* __restrict__ tri_off,
                           const int* __restrict__ ctr_off, int R, RmParams P, int n_edge_verts,
                           float* __restrict__ out_v, int* __restrict__ out_t)
{
    const int Rc = R - 1;
    const long long C = (long long)Rc * Rc * Rc;
    for (long long m = blockIdx.x * (long long)blockDim.x + threadIdx.x; m < C; m += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(m % Rc), y = (int)(m / Rc % Rc), z = (int)(m / ((long long)Rc * Rc));
        rm_cell_emit(c_rm_table, sd, vid, x, y, z, R, P, n_edge_verts, tri_off[m], ctr_off[m], out_v, out_t);
    }
}

// ---- exclusive scan of n ints in place: tiles, then their sums, then add
__global__ void k_rm_scan_tiles(int* data, long long n, int* sums)
{
    __shared__ int sh[34];
    const long long t0 = blockIdx.x * (long long)RM_SCAN_TILE + threadIdx.x * (long long)RM_SCAN_PER;
    int loc[RM_SCAN_PER], s = 0;
    #pragma unroll
    for (int m = 0; m < RM_SCAN_PER; m++) { loc[m] = t0 + m < n ? data[t0 + m] : 0; s += loc[m]; }
    int tot;
    int ex = block_exclusive_scan(s, sh, &tot);
    #pragma unroll
    for (int m = 0; m < RM_SCAN_PER; m++) { if (t0 + m < n) data[t0 + m] = ex; ex += loc[m]; }
    if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

__global__ void k_rm_scan_sums(int* sums, int n, int* total)
{
    __shared__ int sh[34];
    const int t = cta_scan_inplace(sums, n, sh);
    if (threadIdx.x == 0) *total = t;
}

__global__ void k_rm_scan_add(int* data, long long n, const int* __restrict__ sums)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        data[i] += sums[i / RM_SCAN_TILE];
}

static int rm_scan(gpu_ctx* ctx, int* data, long long n, int* sums, int* total, cudaStream_t s, int grid)
{
    const long long tiles = (n + RM_SCAN_TILE - 1) / RM_SCAN_TILE;
    k_rm_scan_tiles<<<(unsigned)tiles, RM_SCAN_NT, 0, s>>>(data, n, sums);
    k_rm_scan_sums<<<1, RM_SCAN_NT, 0, s>>>(sums, (int)tiles, total);
    k_rm_scan_add<<<grid, RM_NT, 0, s>>>(data, n, sums);
    ctx->launches += 3;
    CK(cudaGetLastError());
    return 0;
}

static int rm_grid(const gpu_ctx* ctx, long long n)
{
    const long long want = (n + RM_NT - 1) / RM_NT, cap = (long long)ctx->n_sm * 16;
    return (int)(want < 1 ? 1 : (want < cap ? want : cap));
}

extern "C" int gpu_preprocess(gpu_ctx_t ctx, const float* verts, int nv, const int* tris, int nt, int resolution,
                              float** out_verts, int* out_nv, int** out_tris, int* out_nt)
{
    if (out_verts) *out_verts = nullptr;
    if (out_nv) *out_nv = 0;
    if (out_tris) *out_tris = nullptr;
    if (out_nt) *out_nt = 0;
    if (!ctx) return -1;
    if (!verts || !tris || !out_verts || !out_nv || !out_tris || !out_nt || nv <= 0 || nt <= 0)
        return ctx_fail(ctx, RM_EINVAL, "preprocess: empty mesh or null pointer");
    const int R = resolution;
    if (R < 8 || R > 1024 || (R & (R - 1)))
        return ctx_fail(ctx, RM_EINVAL, "preprocess: resolution %d is not a power of two in [8, 1024]", R);
    for (long long i = 0; i < 3ll * nt; i++)
        if (tris[i] < 0 || tris[i] >= nv)
            return ctx_fail(ctx, RM_EINVAL, "preprocess: triangle index %d outside [0, %d)", tris[i], nv);
    for (long long i = 0; i < 3ll * nv; i++)
        if (!std::isfinite(verts[i]))
            return ctx_fail(ctx, RM_EINVAL, "preprocess: vertex coordinate %lld is not finite", i);
    RmParams P;
    float vmax[3];
    for (int k = 0; k < 3; k++) { P.vmin[k] = verts[k]; vmax[k] = verts[k]; }
    for (long long i = 1; i < nv; i++)
        for (int k = 0; k < 3; k++) {
            const float p = verts[3 * i + k];
            if (p < P.vmin[k]) P.vmin[k] = p;
            if (p > vmax[k]) vmax[k] = p;
        }
    float extent = -1.0f;
    for (int k = 0; k < 3; k++)
        if (vmax[k] - P.vmin[k] > extent) extent = vmax[k] - P.vmin[k];
    if (!(extent > 0.0f) || !(extent < 3.0e38f))
        return ctx_fail(ctx, RM_EINVAL, "preprocess: the mesh has no finite extent");
    P.R = R;
    P.extent = extent;
    P.band = 3.0 / R;
    P.margin = 1.0 + 2.0 * P.band;

    CK(cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->stream;
    const long long N = (long long)R * R * R, C = (long long)(R - 1) * (R - 1) * (R - 1);
    const long long tiles = (3 * N + RM_SCAN_TILE - 1) / RM_SCAN_TILE;
    int rc = pool_begin(ctx, al256(12 * (size_t)nv) + al256(24 * (size_t)nv) + al256(12 * (size_t)nt)
                             + al256(4 * (size_t)N) + al256((size_t)N) + al256(3 * (size_t)N) + al256(12 * (size_t)N)
                             + 2 * al256(4 * (size_t)C) + al256(4 * (size_t)tiles) + al256(64));
    if (rc) return rc;
    float* dv = pool_take<float>(ctx, 3 * (size_t)nv);
    double* du = pool_take<double>(ctx, 3 * (size_t)nv);
    int* dt = pool_take<int>(ctx, 3 * (size_t)nt);
    unsigned* d2 = pool_take<unsigned>(ctx, N);
    unsigned char* outside = pool_take<unsigned char>(ctx, N);
    unsigned char* blk = pool_take<unsigned char>(ctx, 3 * N);
    int* vid = pool_take<int>(ctx, 3 * N);
    int* ctri = pool_take<int>(ctx, C);
    int* cctr = pool_take<int>(ctx, C);
    int* sums = pool_take<int>(ctx, tiles);
    int* misc = pool_take<int>(ctx, 16);        // [0] changed, [1] vertices, [2] triangles, [3] centres
    if (!misc) return ctx_fail(ctx, KERR_HEAP_OOM, "preprocess: device pool carve failed");

    CK(cudaMemcpyToSymbolAsync(c_rm_table, &rm_table(), sizeof(RmTable), 0, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(dv, verts, 12 * (size_t)nv, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(dt, tris, 12 * (size_t)nt, cudaMemcpyHostToDevice, s));
    k_rm_norm<<<rm_grid(ctx, 3ll * nv), RM_NT, 0, s>>>(dv, nv, P, du);
    k_rm_init<<<rm_grid(ctx, N), RM_NT, 0, s>>>(d2, outside, blk, R);
    k_rm_tris<<<(unsigned)(nt < ctx->n_sm * 64 ? nt : ctx->n_sm * 64), RM_NT, 0, s>>>(du, dt, nt, R, d2, blk);
    ctx->launches += 3;
    CK(cudaGetLastError());

    // sign: sweeps until a round of the three axes changes nothing (a round
    // that changes anything adds an outside node, so there are at most N)
    const int line_blocks = (int)(((long long)R * R + RM_NT - 1) / RM_NT);
    for (long long round = 0;; round++) {
        if (round > N) return ctx_fail(ctx, KERR_MESH_INVALID, "preprocess: sign fill did not settle");
        CK(cudaMemsetAsync(misc, 0, sizeof(int), s));
        for (int k = 0; k < 3; k++) k_rm_sweep<<<line_blocks, RM_NT, 0, s>>>(outside, blk, R, k, misc);
        ctx->launches += 3;
        CK(cudaGetLastError());
        int changed = 0;
        CK(cudaMemcpyAsync(&changed, misc, sizeof(int), cudaMemcpyDeviceToHost, s));
        rc = sync_and_check(ctx, "preprocess sign fill");
        if (rc) return rc;
        if (!changed) break;
    }
    k_rm_field<<<rm_grid(ctx, N), RM_NT, 0, s>>>(d2, outside, N);
    const float* sd = (const float*)d2;
    k_rm_edge_flags<<<rm_grid(ctx, N), RM_NT, 0, s>>>(sd, R, vid);
    k_rm_cell_counts<<<rm_grid(ctx, C), RM_NT, 0, s>>>(sd, R, ctri, cctr);
    ctx->launches += 3;
    CK(cudaGetLastError());
    if ((rc = rm_scan(ctx, vid, 3 * N, sums, misc + 1, s, rm_grid(ctx, 3 * N)))) return rc;
    if ((rc = rm_scan(ctx, ctri, C, sums, misc + 2, s, rm_grid(ctx, C)))) return rc;
    if ((rc = rm_scan(ctx, cctr, C, sums, misc + 3, s, rm_grid(ctx, C)))) return rc;
    int cnt[4] = {0, 0, 0, 0};
    CK(cudaMemcpyAsync(cnt, misc, sizeof(cnt), cudaMemcpyDeviceToHost, s));
    rc = sync_and_check(ctx, "preprocess counts");
    if (rc) return rc;
    const long long n_out_v = (long long)cnt[1] + cnt[3], n_out_t = cnt[2];
    if (n_out_v > INT_MAX / 3 || n_out_t > INT_MAX / 3)
        return ctx_fail(ctx, KERR_MESH_INVALID, "preprocess: output too large");

    float* hv = (float*)malloc(12 * (size_t)(n_out_v > 0 ? n_out_v : 1));
    int* ht = (int*)malloc(12 * (size_t)(n_out_t > 0 ? n_out_t : 1));
    if (!hv || !ht) { free(hv); free(ht); return ctx_fail(ctx, KERR_HEAP_OOM, "preprocess: host allocation failed"); }
    if (n_out_t > 0) {
        float* ov = nullptr;
        int* ot = nullptr;
        cudaError_t e = cudaMallocFromPoolAsync((void**)&ov, 12 * (size_t)n_out_v, ctx->parts_pool, s);
        if (e == cudaSuccess) e = cudaMallocFromPoolAsync((void**)&ot, 12 * (size_t)n_out_t, ctx->parts_pool, s);
        if (e == cudaSuccess) {
            k_rm_edge_verts<<<rm_grid(ctx, N), RM_NT, 0, s>>>(sd, vid, R, P, ov);
            k_rm_cells<<<rm_grid(ctx, C), RM_NT, 0, s>>>(sd, vid, ctri, cctr, R, P, cnt[1], ov, ot);
            ctx->launches += 2;
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaMemcpyAsync(hv, ov, 12 * (size_t)n_out_v, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(ht, ot, 12 * (size_t)n_out_t, cudaMemcpyDeviceToHost, s);
        if (ov) cudaFreeAsync(ov, s);
        if (ot) cudaFreeAsync(ot, s);
        if (e == cudaSuccess) {
            rc = sync_and_check(ctx, "preprocess output");
        } else {
            cudaStreamSynchronize(s);
            rc = ctx_fail(ctx, (int)e, "preprocess output: %s", cudaGetErrorString(e));
        }
        if (rc) { free(hv); free(ht); return rc; }
    }
    *out_verts = hv; *out_nv = (int)n_out_v;
    *out_tris = ht; *out_nt = (int)n_out_t;
    return 0;
}
