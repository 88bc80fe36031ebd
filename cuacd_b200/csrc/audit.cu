// audit.cu — topology audit of a triangle mesh (gpu_mesh_audit): degenerate
// triangles, out-of-range indices, open, non-manifold and inconsistently
// oriented edges, as the MAV_* verdict bits of the reference's
// mesh_audit_block (cuda/mesh_audit.cuh:21-26, :92-157).
//
// The reference runs the audit in one 256-thread block with a lock-free
// table of edge records.  Here it is a grid-wide pass: one thread per
// triangle inserts its three undirected edges into an open-addressed table of
// 64-bit keys (lo << 32 | hi) with per-slot incidence and forward counts,
// then one thread per slot classifies the edges.  The table holds at most 3T
// keys at a load of at most 1/2.  The triangle checks follow the reference:
// an index outside [0, nv) marks the triangle bad and skips it; a repeated
// index or an exactly zero FP32 cross product (no contraction: this file is
// built with -fmad=false) marks it degenerate, and its edges still count.
#include <algorithm>
#include <cstdlib>
#include "context.cuh"

#define AUD_NT 256
#define AUD_EMPTY (~0ull)

__device__ __forceinline__ unsigned aud_slot(unsigned long long key, unsigned cap)
{
    return (unsigned)((key * 0x9E3779B97F4A7C15ull) >> 32) & (cap - 1);
}

// Count one traversal of edge a->b; returns false if the table is full.
__device__ __forceinline__ bool aud_add_edge(unsigned long long* keys, unsigned* tot, unsigned* fwd, unsigned cap,
                                             unsigned a, unsigned b)
{
    const unsigned lo = a < b ? a : b, hi = a < b ? b : a;
    const unsigned long long key = ((unsigned long long)lo << 32) | hi;
    unsigned s = aud_slot(key, cap);
    for (unsigned probe = 0; probe < cap; probe++) {
        const unsigned long long prev = atomicCAS(&keys[s], AUD_EMPTY, key);
        if (prev == AUD_EMPTY || prev == key) {
            atomicAdd(&tot[s], 1u);
            if (a < b) atomicAdd(&fwd[s], 1u);
            return true;
        }
        s = (s + 1) & (cap - 1);
    }
    return false;
}

// counters: [0] degenerate, [1] bad index, [2] open, [3] non-manifold,
// [4] flipped, [5] table full
__global__ void __launch_bounds__(AUD_NT)
k_audit_tris(const float* __restrict__ v, int nv, const int* __restrict__ t, int nt, unsigned long long* keys,
             unsigned* tot, unsigned* fwd, unsigned cap, unsigned* counters)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nt) return;
    const int a = t[3 * i], b = t[3 * i + 1], c = t[3 * i + 2];
    if ((unsigned)a >= (unsigned)nv || (unsigned)b >= (unsigned)nv || (unsigned)c >= (unsigned)nv) {
        atomicAdd(&counters[1], 1u);
        return;
    }
    bool degen = a == b || b == c || a == c;
    if (!degen) {
        const float abx = v[3 * b] - v[3 * a], aby = v[3 * b + 1] - v[3 * a + 1], abz = v[3 * b + 2] - v[3 * a + 2];
        const float acx = v[3 * c] - v[3 * a], acy = v[3 * c + 1] - v[3 * a + 1], acz = v[3 * c + 2] - v[3 * a + 2];
        const float nx = aby * acz - abz * acy, ny = abz * acx - abx * acz, nz = abx * acy - aby * acx;
        degen = nx * nx + ny * ny + nz * nz <= 0.0f;
    }
    if (degen) atomicAdd(&counters[0], 1u);
    bool ok = aud_add_edge(keys, tot, fwd, cap, (unsigned)a, (unsigned)b);
    ok &= aud_add_edge(keys, tot, fwd, cap, (unsigned)b, (unsigned)c);
    ok &= aud_add_edge(keys, tot, fwd, cap, (unsigned)c, (unsigned)a);
    if (!ok) atomicAdd(&counters[5], 1u);
}

__global__ void __launch_bounds__(AUD_NT)
k_audit_edges(const unsigned long long* __restrict__ keys, const unsigned* __restrict__ tot,
              const unsigned* __restrict__ fwd, unsigned cap, unsigned* counters)
{
    unsigned open = 0, nonman = 0, flip = 0;
    for (unsigned s = blockIdx.x * blockDim.x + threadIdx.x; s < cap; s += gridDim.x * blockDim.x) {
        if (keys[s] == AUD_EMPTY) continue;
        const unsigned n = tot[s], f = fwd[s];
        if (n == 1) open++;
        else if (n > 2) nonman++;
        else if (n == 2 && (f == 2 || f == 0)) flip++;
    }
    #pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        open += __shfl_xor_sync(FULL_MASK, open, o);
        nonman += __shfl_xor_sync(FULL_MASK, nonman, o);
        flip += __shfl_xor_sync(FULL_MASK, flip, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (open) atomicAdd(&counters[2], open);
        if (nonman) atomicAdd(&counters[3], nonman);
        if (flip) atomicAdd(&counters[4], flip);
    }
}

static unsigned audit_capacity(int nt)
{
    const unsigned long long need = 6ull * (unsigned long long)nt + 1ull;
    unsigned cap = 1024u;
    while (cap < need) cap <<= 1;
    return cap;
}

extern "C" int gpu_mesh_audit(gpu_ctx_t ctx, const float* verts, int n_verts, const int* tris, int n_tris,
                              unsigned int* out_flags)
{
    if (!ctx || !out_flags) return -1;
    *out_flags = 0;
    if (n_verts < 0 || n_tris < 0) return ctx_fail(ctx, KERR_MESH_INVALID, "negative size");
    if ((long long)n_tris * 6 >= (1ll << 31)) return ctx_fail(ctx, KERR_MESH_INVALID, "too many triangles");
    if (n_tris == 0) return 0;
    CK(cudaSetDevice(ctx->device));
    const unsigned cap = audit_capacity(n_tris);
    int rc = pool_begin(ctx, al256(12 * (size_t)n_verts) + al256(12 * (size_t)n_tris) + al256(8 * (size_t)cap)
                             + 2 * al256(4 * (size_t)cap) + al256(64));
    if (rc) return rc;
    float* dv = pool_take<float>(ctx, 3 * (size_t)n_verts);
    int* dt = pool_take<int>(ctx, 3 * (size_t)n_tris);
    unsigned long long* keys = pool_take<unsigned long long>(ctx, cap);
    unsigned* tot = pool_take<unsigned>(ctx, cap);
    unsigned* fwd = pool_take<unsigned>(ctx, cap);
    unsigned* cnt = pool_take<unsigned>(ctx, 16);
    cudaStream_t s = ctx->stream;
    if (n_verts) CK(cudaMemcpyAsync(dv, verts, 12 * (size_t)n_verts, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(dt, tris, 12 * (size_t)n_tris, cudaMemcpyHostToDevice, s));
    CK(cudaMemsetAsync(keys, 0xff, 8 * (size_t)cap, s));
    CK(cudaMemsetAsync(tot, 0, 4 * (size_t)cap, s));
    CK(cudaMemsetAsync(fwd, 0, 4 * (size_t)cap, s));
    CK(cudaMemsetAsync(cnt, 0, 64, s));
    k_audit_tris<<<(n_tris + AUD_NT - 1) / AUD_NT, AUD_NT, 0, s>>>(dv, n_verts, dt, n_tris, keys, tot, fwd, cap, cnt);
    const int eb = (int)std::min<unsigned>((cap + AUD_NT - 1) / AUD_NT, (unsigned)ctx->n_sm * 8);
    k_audit_edges<<<eb, AUD_NT, 0, s>>>(keys, tot, fwd, cap, cnt);
    ctx->launches += 2;
    CK(cudaGetLastError());
    unsigned h[6] = {0, 0, 0, 0, 0, 0};
    CK(cudaMemcpyAsync(h, cnt, sizeof(h), cudaMemcpyDeviceToHost, s));
    rc = sync_and_check(ctx, "mesh_audit");
    if (rc) return rc;
    if (h[5]) return ctx_fail(ctx, KERR_HEAP_OOM, "mesh_audit edge table full");
    unsigned f = CUACD_MAV_OK;
    if (h[0]) f |= CUACD_MAV_DEGEN_TRI;
    if (h[1]) f |= CUACD_MAV_BAD_INDEX;
    if (h[2]) f |= CUACD_MAV_OPEN_EDGE;
    if (h[3]) f |= CUACD_MAV_NONMANIFOLD;
    if (h[4]) f |= CUACD_MAV_FLIPPED;
    *out_flags = f;
    return 0;
}
