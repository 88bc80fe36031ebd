// scorer.cu — learned candidate scorer: per-plane features, a 240-256-256-1
// MLP in BF16 with FP32 accumulation on the 5th-generation tensor cores
// (tcgen05.mma, accumulators in tensor memory), its training (MSE, AdamW) and
// the pruned evaluator that sends
// only the best-predicted planes through the exact evaluator.
//
// Features of plane (n, d) on a part (230 used of SC_K = 240), positions
// relative to the part's vertex centroid c, lengths scaled by R (half the
// bounding-box diagonal):
//   [0..3]    n, d + n.c (offset through the centroid) / R
//   [4..35]   per side (positive, negative): vertex fraction, centroid (3),
//             second moments (xx yy zz xy xz yz) (6), box min (3), max (3)
//   [36..53]  part: centroid (3, absolute), second moments (6), box min (3),
//             max (3), mesh volume, hull volume, rv cost
//   [54..69]  histogram of the vertices' signed distances, 16 bins on [-R, R]
//   [70..229] sketch: 80 vertices (index i*nv/80): signed distance to the
//             plane / R and distance from the line (c, n) / R
#include <vector>
#include <algorithm>
#include <random>
#include <cmath>
#include <cstring>
#include <cuda.h>
#include <cuda_bf16.h>
#include "context.cuh"
#include "launch.h"

#define SC_K      240          // padded feature width
#define SC_NF     230          // features used
#define SC_H      256          // hidden width
#define SC_SKETCH 80
#define SC_TSCALE 10.0f        // targets are scaled by this for the loss

struct PartStats {             // per part, computed on the device
    float c[3];                // vertex centroid
    float m2[6];               // second moments about c
    float lo[3], hi[3];        // box relative to c
    float R;                   // half box diagonal
    float mesh_vol, hull_vol, rv;
};

// ---------------------------------------------------------------------------
// features
// ---------------------------------------------------------------------------
static __device__ __forceinline__ float sc_block_sum(float v, float* sh)
{
    v = warp_sum(v);
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    __syncthreads();
    if (lane == 0) sh[w] = v;
    __syncthreads();
    float t = 0.f;
    for (int i = 0; i < nw; i++) t += sh[i];
    return t;
}
static __device__ __forceinline__ float sc_block_min(float v, float* sh)
{
    v = warp_min(v);
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    __syncthreads();
    if (lane == 0) sh[w] = v;
    __syncthreads();
    float t = 3.4e38f;
    for (int i = 0; i < nw; i++) t = fminf(t, sh[i]);
    return t;
}
static __device__ __forceinline__ float sc_block_max(float v, float* sh)
{
    v = warp_max(v);
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    __syncthreads();
    if (lane == 0) sh[w] = v;
    __syncthreads();
    float t = -3.4e38f;
    for (int i = 0; i < nw; i++) t = fmaxf(t, sh[i]);
    return t;
}

// One CTA: statistics of the part (v, t).
__global__ void __launch_bounds__(256)
k_part_stats(const float* __restrict__ v, int nv, const int* __restrict__ t, int nt, float hull_vol, PartStats* out)
{
    __shared__ float sh[8];
    __shared__ double dsh[33];
    float s[3] = {0.f, 0.f, 0.f};
    for (int i = threadIdx.x; i < nv; i += 256) for (int k = 0; k < 3; k++) s[k] += v[3 * i + k];
    float c[3];
    for (int k = 0; k < 3; k++) c[k] = sc_block_sum(s[k], sh) / (float)(nv > 0 ? nv : 1);
    float m[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f}, lo[3] = {3.4e38f, 3.4e38f, 3.4e38f}, hi[3] = {-3.4e38f, -3.4e38f, -3.4e38f};
    for (int i = threadIdx.x; i < nv; i += 256) {
        float x = v[3 * i] - c[0], y = v[3 * i + 1] - c[1], z = v[3 * i + 2] - c[2];
        m[0] += x * x; m[1] += y * y; m[2] += z * z; m[3] += x * y; m[4] += x * z; m[5] += y * z;
        lo[0] = fminf(lo[0], x); lo[1] = fminf(lo[1], y); lo[2] = fminf(lo[2], z);
        hi[0] = fmaxf(hi[0], x); hi[1] = fmaxf(hi[1], y); hi[2] = fmaxf(hi[2], z);
    }
    PartStats P;
    for (int k = 0; k < 3; k++) P.c[k] = c[k];
    for (int k = 0; k < 6; k++) P.m2[k] = sc_block_sum(m[k], sh) / (float)(nv > 0 ? nv : 1);
    for (int k = 0; k < 3; k++) { P.lo[k] = sc_block_min(lo[k], sh); P.hi[k] = sc_block_max(hi[k], sh); }
    const double mv = fabs(block_mesh_signed_volume(v, nv, t, nt, dsh));
    if (threadIdx.x == 0) {
        float dx = P.hi[0] - P.lo[0], dy = P.hi[1] - P.lo[1], dz = P.hi[2] - P.lo[2];
        P.R = 0.5f * sqrtf(dx * dx + dy * dy + dz * dz);
        if (!(P.R > 0.f)) P.R = 1.f;
        P.mesh_vol = (float)mv; P.hull_vol = hull_vol;
        P.rv = part_cost_rv((double)hull_vol, mv);
        *out = P;
    }
}

// One CTA per plane: the feature row (SC_K floats, zero padded).
__global__ void __launch_bounds__(256)
k_cand_features(const float* __restrict__ v, int nv, const float4* __restrict__ planes, int n_planes,
                const PartStats* __restrict__ stats, float* __restrict__ feat)
{
    __shared__ float sh[8];
    __shared__ float hist[16];
    const int p = blockIdx.x;
    if (p >= n_planes) return;
    const PartStats P = *stats;
    const float4 pl = planes[p];
    const float invR = 1.f / P.R;
    float* f = feat + (size_t)p * SC_K;
    if (threadIdx.x < 16) hist[threadIdx.x] = 0.f;
    // per side: count, sum(3), second moments(6), box(6)
    float cnt[2] = {0.f, 0.f}, sm[2][3] = {{0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}};
    float mm[2][6] = {{0.f, 0.f, 0.f, 0.f, 0.f, 0.f}, {0.f, 0.f, 0.f, 0.f, 0.f, 0.f}};
    float lo[2][3] = {{3.4e38f, 3.4e38f, 3.4e38f}, {3.4e38f, 3.4e38f, 3.4e38f}};
    float hi[2][3] = {{-3.4e38f, -3.4e38f, -3.4e38f}, {-3.4e38f, -3.4e38f, -3.4e38f}};
    __syncthreads();
    for (int i = threadIdx.x; i < nv; i += 256) {
        const float x = v[3 * i] - P.c[0], y = v[3 * i + 1] - P.c[1], z = v[3 * i + 2] - P.c[2];
        const float sd = pl.x * v[3 * i] + pl.y * v[3 * i + 1] + pl.z * v[3 * i + 2] + pl.w;
        int b = (int)floorf((sd * invR + 1.f) * 8.f);
        b = min(15, max(0, b));
        atomicAdd(&hist[b], 1.f);
        if (sd == 0.f) continue;
        const int s = sd > 0.f ? 0 : 1;
        cnt[s] += 1.f; sm[s][0] += x; sm[s][1] += y; sm[s][2] += z;
        mm[s][0] += x * x; mm[s][1] += y * y; mm[s][2] += z * z; mm[s][3] += x * y; mm[s][4] += x * z; mm[s][5] += y * z;
        lo[s][0] = fminf(lo[s][0], x); lo[s][1] = fminf(lo[s][1], y); lo[s][2] = fminf(lo[s][2], z);
        hi[s][0] = fmaxf(hi[s][0], x); hi[s][1] = fmaxf(hi[s][1], y); hi[s][2] = fmaxf(hi[s][2], z);
    }
    const float inv_nv = 1.f / (float)(nv > 0 ? nv : 1);
    for (int s = 0; s < 2; s++) {
        const float c = sc_block_sum(cnt[s], sh);
        const float ic = c > 0.f ? 1.f / c : 0.f;
        float o[16];
        o[0] = c * inv_nv;
        for (int k = 0; k < 3; k++) o[1 + k] = sc_block_sum(sm[s][k], sh) * ic * invR;
        for (int k = 0; k < 6; k++) o[4 + k] = sc_block_sum(mm[s][k], sh) * ic * invR * invR;
        for (int k = 0; k < 3; k++) {
            const float a = sc_block_min(lo[s][k], sh), b = sc_block_max(hi[s][k], sh);
            o[10 + k] = c > 0.f ? a * invR : 0.f;
            o[13 + k] = c > 0.f ? b * invR : 0.f;
        }
        if (threadIdx.x == 0) for (int k = 0; k < 16; k++) f[4 + 16 * s + k] = o[k];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        f[0] = pl.x; f[1] = pl.y; f[2] = pl.z;
        f[3] = (pl.w + pl.x * P.c[0] + pl.y * P.c[1] + pl.z * P.c[2]) * invR;
        for (int k = 0; k < 3; k++) f[36 + k] = P.c[k];
        for (int k = 0; k < 6; k++) f[39 + k] = P.m2[k] * invR * invR;
        for (int k = 0; k < 3; k++) { f[45 + k] = P.lo[k] * invR; f[48 + k] = P.hi[k] * invR; }
        f[51] = P.mesh_vol * invR * invR * invR; f[52] = P.hull_vol * invR * invR * invR; f[53] = P.rv * invR;
        for (int k = 0; k < 16; k++) f[54 + k] = hist[k] * inv_nv;
        for (int k = SC_NF; k < SC_K; k++) f[k] = 0.f;
    }
    if (threadIdx.x < SC_SKETCH) {
        const int i = (int)(((long long)threadIdx.x * nv) / SC_SKETCH);
        float sd = 0.f, rad = 0.f;
        if (i < nv) {
            const float x = v[3 * i] - P.c[0], y = v[3 * i + 1] - P.c[1], z = v[3 * i + 2] - P.c[2];
            sd = pl.x * v[3 * i] + pl.y * v[3 * i + 1] + pl.z * v[3 * i + 2] + pl.w;
            const float along = pl.x * x + pl.y * y + pl.z * z;
            const float r2 = x * x + y * y + z * z - along * along;
            rad = sqrtf(fmaxf(r2, 0.f));
        }
        f[70 + 2 * threadIdx.x] = sd * invR;
        f[71 + 2 * threadIdx.x] = rad * invR;
    }
}

// ---------------------------------------------------------------------------
// GEMM on the 5th-generation tensor cores (tcgen05): C[M x N] = alpha *
// op(A)[M x K] * op(B)[K x N] (+ C if accumulate) (+ bias[j]) (* (mask(i,j) >
// 0)) (relu), BF16 operands, FP32 accumulation in tensor memory.  A(i,k) =
// A[i*ar + k*ac], B(k,j) = B[k*br + j*bc], so transposed operands need no
// copy: the CTA stages each 64-wide K slab of its 128 x 128 output tile into
// shared memory in the K-major core-matrix layout of UMMA (8 rows x 16 bytes
// per core matrix, no swizzle), one elected thread issues four
// tcgen05.mma.cta_group::1.kind::f16 (M 128, N 128, K 16) into a 128-column
// TMEM accumulator and commits them to an mbarrier, and after the last slab
// the four warps read their 32 accumulator lanes each with tcgen05.ld for
// the fused epilogue.  Every wait is bounded: a wait that gives up records
// KERR_TIMEOUT in *err and the CTA still frees its tensor memory.
// ---------------------------------------------------------------------------
#define GM_BM 128
#define GM_BN 128
#define GM_BK 64
#define GM_NT 128
#define GM_STAGES 2
#define GM_DSMEM ((size_t)GM_STAGES * (GM_BM + GM_BN) * GM_BK * 2 + 1024)   // 64 KB of slabs + alignment

struct GemmArgs {
    CUtensorMap tma_a;          // A as a 2D tensor (K inner, M rows) when use_tma_a
    int use_tma_a;
    const __nv_bfloat16* A; long long ar, ac;
    const __nv_bfloat16* B; long long br, bc;
    float* Cf; __nv_bfloat16* Cb; int ldc;
    int M, N, K;
    const float* bias;
    const __nv_bfloat16* mask; int ldm;
    float alpha;
    int relu, accumulate;
    int* err;
};

static __device__ __forceinline__ unsigned smem_addr(const void* p)
{
    return (unsigned)__cvta_generic_to_shared(p);
}

// Shared-memory matrix descriptor of a K-major, unswizzled operand slab
// (tcgen05 descriptor format: start, leading and stride byte offsets in 16 B
// units, version 1 at bits 46-47, layout type 0 = no swizzle).
static __device__ __forceinline__ unsigned long long umma_desc(unsigned addr, unsigned lbo, unsigned sbo)
{
    return (unsigned long long)((addr >> 4) & 0x3FFF) | ((unsigned long long)((lbo >> 4) & 0x3FFF) << 16) |
           ((unsigned long long)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}

// Descriptor of a K-major operand slab written by TMA with the 128-byte
// swizzle: rows of 64 BF16 (128 bytes) whose 16-byte chunks are permuted by
// the row's index mod 8; stride byte offset = 8 rows (1,024 bytes), leading
// offset unused (1), layout type 2 (SWIZZLE_128B) at bits 61-63.  The slab
// must start on a 1,024-byte boundary; the K = 16 steps inside it advance
// the start address by 32 bytes.
static __device__ __forceinline__ unsigned long long umma_desc_sw128(unsigned addr)
{
    return (unsigned long long)((addr >> 4) & 0x3FFF) | (1ull << 16) | ((unsigned long long)(1024 >> 4) << 32) |
           (1ull << 46) | (2ull << 61);
}

// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, A /
// B MN-major when a_mn / b_mn (bits 15 / 16, else K-major), N >> 3 at bits
// 17-22, M >> 4 at bits 24-28.
static __host__ __device__ constexpr unsigned umma_idesc_bf16(int m, int n, int a_mn, int b_mn)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((unsigned)a_mn << 15) | ((unsigned)b_mn << 16) |
           ((unsigned)(n >> 3) << 17) | ((unsigned)(m >> 4) << 24);
}

// Bounded wait for the mbarrier phase `parity`; false when it gave up.
static __device__ __forceinline__ bool mbar_wait(unsigned bar, unsigned parity)
{
    for (int it = 0; it < (1 << 24); it++) {
        unsigned done;
        asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
                     " selp.u32 %0, 1, 0, p;\n}\n" : "=r"(done) : "r"(bar), "r"(parity) : "memory");
        if (done) return true;
    }
    return false;
}

// Element (r, k) of a 128-row, 64-wide slab.  K-major: core matrix
// (k / 8, r / 8) of 128 bytes, row r % 8 at 16 bytes, column k % 8.
// MN-major: the same core matrices, each holding 8 K rows of 8 consecutive
// r.  Either way the leading byte offset (next 8 K) is 16 core matrices and
// the stride byte offset (next 8 rows) one.
static __device__ __forceinline__ int slab_index(int r, int k)
{
    return (((k >> 3) * (GM_BM / 8) + (r >> 3)) << 6) + ((r & 7) << 3) + (k & 7);
}
static __device__ __forceinline__ int slab_index_mn(int r, int k)
{
    return (((k >> 3) * (GM_BM / 8) + (r >> 3)) << 6) + ((k & 7) << 3) + (r & 7);
}

// How an operand X(r, k) = X[r*rs + k*ks] is staged: 2 = MN-major with
// 16-byte loads along r, 1 = K-major with 16-byte loads along k, 0 =
// K-major element by element.
static __host__ __device__ __forceinline__ int stage_mode(long long rs, long long ks, int K)
{
    if (ks == 1 && rs % 8 == 0) return 1;
    if (rs == 1 && (ks % 8 == 0 || K == 1)) return 2;
    return 0;
}

// Stage rows [r0, r0 + 128) x K columns [k0, k0 + 64) of X (R x K, zero
// outside) into a slab (all GM_NT threads).  A slab is 1,024 16-byte chunks
// (8 elements along the contiguous dimension); the eight lanes of each
// quarter warp write the eight chunks of one 128-byte core matrix (no bank
// conflicts), and the four quarters of a warp read 64 contiguous bytes of
// each of eight rows (mode 1) or of each of eight k (mode 2).
static __device__ __forceinline__ void stage_slab(__nv_bfloat16* slab, const __nv_bfloat16* __restrict__ X, long long rs,
                                                  long long ks, int R, int K, int r0, int k0, int mode, int tid)
{
    const __nv_bfloat16 zero = __float2bfloat16(0.f);
    if (mode == 1) {                                       // 8 consecutive k of one row per load
        for (int e = tid; e < GM_BM * (GM_BK / 8); e += GM_NT) {
            // lane bits: r % 8, then k-group % 4; then k-group / 4, row block
            const int r = 8 * (e >> 6) + (e & 7), c = 8 * (4 * ((e >> 5) & 1) + ((e >> 3) & 3));
            const int gr = r0 + r, gk = k0 + c;
            uint4 v;
            if (gr < R && gk + 7 < K) v = *reinterpret_cast<const uint4*>(X + gr * rs + gk);
            else {
                __nv_bfloat16 t[8];
                for (int q = 0; q < 8; q++) t[q] = (gr < R && gk + q < K) ? X[gr * rs + (gk + q)] : zero;
                v = *reinterpret_cast<const uint4*>(t);
            }
            *reinterpret_cast<uint4*>(slab + slab_index(r, c)) = v;
        }
    } else if (mode == 2) {                                // 8 consecutive r of one k per load
        for (int e = tid; e < (GM_BM / 8) * GM_BK; e += GM_NT) {
            // lane bits: k % 8, then row block % 4; then k-group, row block / 4
            const int k = 8 * ((e >> 5) & 7) + (e & 7), r = 8 * (4 * (e >> 8) + ((e >> 3) & 3));
            const int gr = r0 + r, gk = k0 + k;
            uint4 v;
            if (gk < K && gr + 7 < R) v = *reinterpret_cast<const uint4*>(X + gr + gk * ks);
            else {
                __nv_bfloat16 t[8];
                for (int q = 0; q < 8; q++) t[q] = (gk < K && gr + q < R) ? X[(gr + q) + gk * ks] : zero;
                v = *reinterpret_cast<const uint4*>(t);
            }
            *reinterpret_cast<uint4*>(slab + slab_index_mn(r, k)) = v;
        }
    } else {
        for (int e = tid; e < GM_BM * GM_BK; e += GM_NT) {
            const int r = e / GM_BK, c = e % GM_BK;
            const int gr = r0 + r, gk = k0 + c;
            slab[slab_index(r, c)] = (gr < R && gk < K) ? X[gr * rs + gk * ks] : zero;
        }
    }
}

// One 16-byte global -> shared copy (cp.async, L2 only); src_bytes < 16
// zero-fills the rest (0: all zero, src not read).
static __device__ __forceinline__ void cp16(void* dst, const void* src, int src_bytes)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;"
                 :: "r"(smem_addr(dst)), "l"(src), "r"(src_bytes) : "memory");
}

// stage_slab with asynchronous copies (modes 1 and 2: the same chunks in
// the same places; mode 0 stores element by element).  The caller commits
// the group and waits for it before the slab is read.
static __device__ __forceinline__ void stage_slab_async(__nv_bfloat16* slab, const __nv_bfloat16* __restrict__ X,
                                                        long long rs, long long ks, int R, int K, int r0, int k0,
                                                        int mode, int tid)
{
    if (mode == 1) {
        for (int e = tid; e < GM_BM * (GM_BK / 8); e += GM_NT) {
            const int r = 8 * (e >> 6) + (e & 7), c = 8 * (4 * ((e >> 5) & 1) + ((e >> 3) & 3));
            const int gr = r0 + r, gk = k0 + c;
            const int n = (gr < R && gk < K) ? 2 * min(8, K - gk) : 0;
            cp16(slab + slab_index(r, c), n ? (const void*)(X + gr * rs + gk) : (const void*)X, n);
        }
    } else if (mode == 2) {
        for (int e = tid; e < (GM_BM / 8) * GM_BK; e += GM_NT) {
            const int k = 8 * ((e >> 5) & 7) + (e & 7), r = 8 * (4 * (e >> 8) + ((e >> 3) & 3));
            const int gr = r0 + r, gk = k0 + k;
            const int n = (gk < K && gr < R) ? 2 * min(8, R - gr) : 0;
            cp16(slab + slab_index_mn(r, k), n ? (const void*)(X + gr + gk * ks) : (const void*)X, n);
        }
    } else {
        stage_slab(slab, X, rs, ks, R, K, r0, k0, 0, tid);
    }
}

__global__ void __launch_bounds__(GM_NT)
k_gemm_umma(const __grid_constant__ GemmArgs g)
{
    // GM_STAGES slab pairs (dynamic shared memory); after the last MMA the
    // epilogue's transpose tiles
    extern __shared__ __align__(1024) __nv_bfloat16 sm_raw[];
    // the stages start on a 1,024-byte boundary (the 128-byte swizzle of the
    // TMA-written A slabs repeats every 1,024 bytes)
    __nv_bfloat16* const sm = sm_raw + (((1024u - (smem_addr(sm_raw) & 1023u)) & 1023u) >> 1);
    __shared__ __align__(8) unsigned long long s_bar[GM_STAGES];
    __shared__ __align__(8) unsigned long long s_full[GM_STAGES];     // TMA bytes of a stage's A slab landed
    __shared__ unsigned s_tmem;
    __shared__ int s_fail;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int m0 = blockIdx.y * GM_BM, n0 = blockIdx.x * GM_BN;
    if (warp == 0) {                                  // 128 fp32 columns of tensor memory
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     :: "r"(smem_addr(&s_tmem)), "r"(GM_BN) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        s_fail = 0;
        for (int b = 0; b < GM_STAGES; b++) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_addr(&s_bar[b])), "r"(1) : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_addr(&s_full[b])), "r"(1) : "memory");
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const unsigned tmem = s_tmem;
    // A(i, k) = A[i*ar + k*ac]; B as an N x K operand: B(j, k) = B[j*bc + k*br]
    const int amode = stage_mode(g.ar, g.ac, g.K), bmode = stage_mode(g.bc, g.br, g.K);
    const unsigned idesc = umma_idesc_bf16(GM_BM, GM_BN, amode == 2, bmode == 2);
    const int nk = (g.K + GM_BK - 1) / GM_BK;
    // slab pair kt goes to stage kt % 2: its copies are issued while the
    // MMAs of slab kt - 1 run, once those of slab kt - 2 (the stage's last
    // readers) have completed
    unsigned phf[GM_STAGES] = {0u, 0u};
    bool tpend[GM_STAGES] = {false, false};           // thread 0: a TMA copy not yet waited for
    auto stage = [&](int kt) {
        __nv_bfloat16* As = sm + (size_t)(kt & 1) * (GM_BM + GM_BN) * GM_BK;
        if (g.use_tma_a) {
            // one thread: the 128 x 64 box at (k, row) = (kt * 64, m0),
            // zero-filled outside the matrix, into the stage's A slab
            if (tid == 0) {
                const unsigned fb = smem_addr(&s_full[kt & 1]);
                asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
                             :: "r"(fb), "r"(GM_BM * GM_BK * 2) : "memory");
                asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
                             " [%0], [%1, {%2, %3}], [%4];"
                             :: "r"(smem_addr(As)), "l"(reinterpret_cast<unsigned long long>(&g.tma_a)),
                                "r"(kt * GM_BK), "r"(m0), "r"(fb) : "memory");
                tpend[kt & 1] = true;
            }
        } else {
            stage_slab_async(As, g.A, g.ar, g.ac, g.M, g.K, m0, kt * GM_BK, amode, tid);
        }
        stage_slab_async(As + GM_BM * GM_BK, g.B, g.bc, g.br, g.N, g.K, n0, kt * GM_BK, bmode, tid);
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    unsigned ph[GM_STAGES] = {0u, 0u};
    bool pend[GM_STAGES] = {false, false};            // committed MMAs not yet waited for
    // Thread 0 waits for a stage's MMAs and a CTA barrier releases the
    // others (so 127 threads do not poll the mbarrier); a wait that gives up
    // waits once more (bounded) for the MMAs in flight.  pend[] is the same
    // on every thread, so every thread meets the barrier.
    auto wait_stage = [&](int b) {
        const unsigned bar = smem_addr(&s_bar[b]);
        if (tid == 0 && !mbar_wait(bar, ph[b]) && !mbar_wait(bar, ph[b])) atomicOr(&s_fail, 1);
        ph[b] ^= 1u; pend[b] = false;
        __syncthreads();
    };
    if (nk > 0) stage(0);
    for (int kt = 0; kt < nk && !s_fail; kt++) {
        const int b = kt & 1;
        if (kt + 1 < nk) {
            if (pend[(kt + 1) & 1]) wait_stage((kt + 1) & 1);
            stage(kt + 1);
            asm volatile("cp.async.wait_group 1;" ::: "memory");
        } else {
            asm volatile("cp.async.wait_group 0;" ::: "memory");
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");   // copies -> tensor-core reads
        __syncthreads();
        if (tid == 0) {
            // the TMA copy of this stage's A slab (bounded wait)
            if (g.use_tma_a) {
                if (!mbar_wait(smem_addr(&s_full[b]), phf[b])) atomicOr(&s_fail, 1);
                phf[b] ^= 1u; tpend[b] = false;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const unsigned a0 = smem_addr(sm + (size_t)b * (GM_BM + GM_BN) * GM_BK);
            const unsigned b0 = a0 + GM_BM * GM_BK * 2;
            #pragma unroll
            for (int kk = 0; kk < GM_BK / 16; kk++) {
                // K chunk pair (2kk, 2kk+1): leading offset = one chunk of
                // 16 core matrices, stride offset = one core matrix
                const unsigned off = (unsigned)(2 * kk * (GM_BM / 8) * 128);
                const unsigned long long ad = g.use_tma_a ? umma_desc_sw128(a0 + 32u * kk)
                                                          : umma_desc(a0 + off, (GM_BM / 8) * 128, 128);
                const unsigned long long bd = umma_desc(b0 + off, (GM_BN / 8) * 128, 128);
                const unsigned acc = (kt > 0 || kk > 0) ? 1u : 0u;
                asm volatile("{\n .reg .pred p;\n setp.ne.u32 p, %4, 0;\n"
                             " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n"
                             :: "r"(tmem), "l"(ad), "l"(bd), "r"(idesc), "r"(acc) : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                         :: "r"(smem_addr(&s_bar[b])) : "memory");
        }
        pend[b] = true;
    }
    // the last MMAs (and any copies still in flight) before the shared
    // memory and the accumulator are read or released
    for (int b = 0; b < GM_STAGES; b++) if (pend[b]) wait_stage(b);
    asm volatile("cp.async.wait_all;" ::: "memory");
    // a loop stopped early may leave a TMA copy in flight: it lands first
    if (tid == 0)
        for (int b = 0; b < GM_STAGES; b++)
            if (tpend[b] && !mbar_wait(smem_addr(&s_full[b]), phf[b])) atomicOr(&s_fail, 1);
    const bool issued = nk > 0;
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (s_fail) {
        if (tid == 0 && g.err) atomicOr(g.err, KERR_TIMEOUT);
    } else if (issued) {
        // epilogue: warp w owns accumulator lanes (rows) 32w .. 32w + 31.
        // Each 32 x 32 block goes through a padded shared tile so that the
        // lanes then take consecutive columns of one row: coalesced loads of
        // the mask and C, and coalesced stores.
        float* const tile = reinterpret_cast<float*>(sm) + warp * (32 * 33);
        const int c = n0 + lane;
        for (int c0 = 0; c0 < GM_BN; c0 += 32) {
            unsigned v[32];
            const unsigned taddr = tmem + ((unsigned)(32 * warp) << 16) + (unsigned)c0;
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 "
                         "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                         "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                         : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
                           "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
                           "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]),
                           "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]),
                           "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
                         : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            #pragma unroll
            for (int q = 0; q < 32; q++) tile[lane * 33 + q] = __uint_as_float(v[q]);
            __syncwarp();
            const int cc = c + c0;
            const float bias = (g.bias && cc < g.N) ? g.bias[cc] : 0.f;
            for (int rr = 0; rr < 32; rr++) {
                const int r = m0 + 32 * warp + rr;
                if (r >= g.M || cc >= g.N) continue;
                float x = g.alpha * tile[rr * 33 + lane];
                const size_t o = (size_t)r * g.ldc + cc;
                if (g.accumulate && g.Cf) x += g.Cf[o];
                x += bias;
                if (g.mask && !(__bfloat162float(g.mask[(size_t)r * g.ldm + cc]) > 0.f)) x = 0.f;
                if (g.relu) x = fmaxf(x, 0.f);
                if (g.Cf) g.Cf[o] = x;
                if (g.Cb) g.Cb[o] = __float2bfloat16(x);
            }
            __syncwarp();                                  // the tile is rewritten by the next block
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"(GM_BN) : "memory");
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (the
// library links the runtime statically and never the driver library).
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
static EncodeTiledFn encode_tiled()
{
    static EncodeTiledFn fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (EncodeTiledFn)p;
    }
    return fn;
}

// A K-major, contiguous A (A(i, k) = A[i*ar + k]) goes to the tensor core
// through TMA: a 2D map (K inner, M rows, row pitch 2*ar bytes) with
// 128 x 64 boxes and the 128-byte swizzle.  Other operands, or a map the
// driver refuses, are staged with cp.async.
static void gemm_tma_a(GemmArgs& g)
{
    g.use_tma_a = 0;
    if (g.ac != 1 || g.ar % 8 != 0 || g.K % 8 != 0 || g.ar < g.K || ((size_t)g.A & 15)) return;
    EncodeTiledFn fn = encode_tiled();
    if (!fn) return;
    const cuuint64_t dims[2] = {(cuuint64_t)g.K, (cuuint64_t)g.M};
    const cuuint64_t strides[1] = {(cuuint64_t)g.ar * 2};
    const cuuint32_t box[2] = {GM_BK, GM_BM};
    const cuuint32_t estr[2] = {1, 1};
    if (fn(&g.tma_a, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, (void*)g.A, dims, strides, box, estr,
           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS)
        g.use_tma_a = 1;
}

static unsigned long long g_gemm_tma = 0, g_gemm_staged = 0;   // launches by how A was staged

static void gemm(GemmArgs g, int* err, cudaStream_t s)
{
    static bool attr_set[64] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !attr_set[dev]) {
        cudaFuncSetAttribute(k_gemm_umma, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)GM_DSMEM);
        attr_set[dev] = true;
    }
    g.err = err;
    gemm_tma_a(g);
    if (g.M > 0 && g.N > 0) { if (g.use_tma_a) g_gemm_tma++; else g_gemm_staged++; }
    dim3 grid((g.N + GM_BN - 1) / GM_BN, (g.M + GM_BM - 1) / GM_BM);
    if (g.M > 0 && g.N > 0) k_gemm_umma<<<grid, GM_NT, GM_DSMEM, s>>>(g);
}

__global__ void k_f32_to_bf16(const float* in, __nv_bfloat16* out, size_t n)
{
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = __float2bfloat16(in[i]);
}

// Rows idx[0..b) of X (fp32, SC_K wide), standardised by the scorer's
// feature normaliser (nrm[k] = mean, nrm[SC_K + k] = 1 / std), into Xb
// (bf16); targets likewise (scaled).
__global__ void k_gather_rows(const float* X, const float* T, const int* idx, int b, const float* __restrict__ nrm,
                              __nv_bfloat16* Xb, float* Tb)
{
    const int r = blockIdx.x;
    if (r >= b) return;
    const int src = idx ? idx[r] : r;
    for (int k = threadIdx.x; k < SC_K; k += blockDim.x)
        Xb[(size_t)r * SC_K + k] = __float2bfloat16((X[(size_t)src * SC_K + k] - nrm[k]) * nrm[SC_K + k]);
    if (threadIdx.x == 0 && T) Tb[r] = T[src] * SC_TSCALE;
}

// dY = 2 (Y - T) / b (bf16 for the GEMMs, fp32 kept), loss = mean (Y - T)^2.
__global__ void k_mse_grad(const float* Y, const float* T, int b, __nv_bfloat16* dYb, float* dYf, float* loss)
{
    __shared__ float sh[8];
    float l = 0.f;
    for (int i = threadIdx.x; i < b; i += blockDim.x) {
        const float e = Y[i] - T[i];
        l += e * e;
        const float gr = 2.f * e / (float)b;
        dYf[i] = gr;
        dYb[i] = __float2bfloat16(gr);
    }
    l = sc_block_sum(l, sh);
    if (threadIdx.x == 0) *loss = l / (float)b;
}

// Column sums of a b x n fp32 matrix (bias gradients).
__global__ void k_colsum(const float* D, int b, int n, float* out)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    float s = 0.f;
    for (int i = 0; i < b; i++) s += D[(size_t)i * n + j];
    out[j] = s;
}

// AdamW on one flat parameter block (decoupled weight decay where decay=1).
__global__ void k_adamw(float* p, const float* gr, float* m, float* v, __nv_bfloat16* pb, size_t n, float lr,
                        float b1, float b2, float eps, float wd, float c1, float c2, int decay)
{
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float g = gr[i];
    const float mi = b1 * m[i] + (1.f - b1) * g;
    const float vi = b2 * v[i] + (1.f - b2) * g * g;
    m[i] = mi; v[i] = vi;
    float x = p[i];
    if (decay) x -= lr * wd * x;
    x -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    p[i] = x;
    if (pb) pb[i] = __float2bfloat16(x);
}

// ---------------------------------------------------------------------------
// pruning: selection of the planes that go through the exact evaluator
// ---------------------------------------------------------------------------
#define SC_SEL_MAX 1024

// One CTA.  Rank of plane i = number of planes predicted lower (ties: lower
// index first); selected when rank < k or prediction <= k-th + margin.
// Writes the selected planes compacted in index order, pos[i] (slot in the
// compacted list or -1), the count and the predictions in score units.
__global__ void __launch_bounds__(256)
k_select_planes(const float* __restrict__ Y, int n, int k, float margin, const float4* __restrict__ planes,
                float4* __restrict__ sel_planes, int* __restrict__ pos, int* __restrict__ count,
                float* __restrict__ pred)
{
    __shared__ float key[SC_SEL_MAX];
    __shared__ unsigned char fl[SC_SEL_MAX];
    __shared__ float kth;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const float y = Y[i] / SC_TSCALE;
        key[i] = (y == y) ? y : 3.402823466e38f;        // NaN ranks last
        if (pred) pred[i] = y;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const float ki = key[i];
        int r = 0;
        for (int j = 0; j < n; j++) r += (key[j] < ki) || (key[j] == ki && j < i);
        if (r == k - 1) kth = ki;
        fl[i] = r < k;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) fl[i] |= key[i] <= kth + margin;
    __syncthreads();
    if (threadIdx.x == 0) {
        int c = 0;
        for (int i = 0; i < n; i++) {
            if (fl[i]) { sel_planes[c] = planes[i]; pos[i] = c++; }
            else pos[i] = -1;
        }
        *count = c;
    }
}

// out[i] = the exact result of plane i when it was evaluated, else ok = 0
// and FLT_MAX scores.
__global__ void k_scatter_results(const cuacd_cand_result* __restrict__ sub, const int* __restrict__ pos, int n,
                                  cuacd_cand_result* __restrict__ out, int* __restrict__ evaluated)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int j = pos[i];
    cuacd_cand_result r;
    if (j >= 0) r = sub[j];
    else {
        memset(&r, 0, sizeof(r));
        r.score_rv = r.score_full = 3.402823466e38f;
    }
    out[i] = r;
    if (evaluated) evaluated[i] = j >= 0;
}

// ---------------------------------------------------------------------------
// host: the scorer object
// ---------------------------------------------------------------------------
namespace {
const size_t OFF_W1 = 0;
const size_t OFF_B1 = OFF_W1 + (size_t)SC_K * SC_H;
const size_t OFF_W2 = OFF_B1 + SC_H;
const size_t OFF_B2 = OFF_W2 + (size_t)SC_H * SC_H;
const size_t OFF_W3 = OFF_B2 + SC_H;
const size_t OFF_B3 = OFF_W3 + SC_H;
const size_t N_PARAMS = OFF_B3 + 1;
}

struct cuacd_scorer {
    int device;
    float* p32;                  // master parameters (fp32)
    __nv_bfloat16* pb;           // bf16 copies for the GEMMs
    float* g32;                  // gradients
    float* nrm;                  // feature normaliser: mean[SC_K], 1/std[SC_K]
    float* m; float* v;          // AdamW moments
    int step;
    // work buffers for batches of up to cap rows
    int cap;
    float* X; float* T;          // fp32 rows / targets (gathered from)
    int n_rows_cap;
    int* idx;
    __nv_bfloat16 *Xb, *H1, *H2, *dYb, *dH2b, *dH1b;
    float *Tb, *Y, *dYf, *dH2f, *dH1f, *loss;
    int* gerr;                   // error word of the tensor-core GEMMs (KERR_TIMEOUT)
    // pruned-evaluation buffers
    float* mv; int* mt; float4* mp; PartStats* st; float* feat;
    size_t mv_cap, mt_cap, mp_cap;
    char* pr; size_t pr_cap;     // device pruning: selected planes, pos, count, sub-results
    int* h_count;                // pinned
    char* hx; size_t hx_cap;     // host-pointer pruning: staged mesh, planes and results
};

static int sc_fail(gpu_ctx* ctx, int code, const char* msg) { return ctx_fail(ctx, code, "%s", msg); }

#define SCK(call) do { cudaError_t _e = (call); if (_e != cudaSuccess) \
    return ctx_fail(ctx, (int)_e, "%s failed: %s", #call, cudaGetErrorString(_e)); } while (0)

static int sc_reserve(gpu_ctx* ctx, cuacd_scorer* s, int b)
{
    if (b <= s->cap) return 0;
    int c = s->cap > 0 ? s->cap : 1024;
    while (c < b) c *= 2;
    cudaFree(s->idx); cudaFree(s->Xb); cudaFree(s->H1); cudaFree(s->H2); cudaFree(s->dYb); cudaFree(s->dH2b);
    cudaFree(s->dH1b); cudaFree(s->Tb); cudaFree(s->Y); cudaFree(s->dYf); cudaFree(s->dH2f); cudaFree(s->dH1f);
    SCK(cudaMalloc(&s->idx, sizeof(int) * c));
    SCK(cudaMalloc(&s->Xb, sizeof(__nv_bfloat16) * (size_t)c * SC_K));
    SCK(cudaMalloc(&s->H1, sizeof(__nv_bfloat16) * (size_t)c * SC_H));
    SCK(cudaMalloc(&s->H2, sizeof(__nv_bfloat16) * (size_t)c * SC_H));
    SCK(cudaMalloc(&s->dYb, sizeof(__nv_bfloat16) * c));
    SCK(cudaMalloc(&s->dH2b, sizeof(__nv_bfloat16) * (size_t)c * SC_H));
    SCK(cudaMalloc(&s->dH1b, sizeof(__nv_bfloat16) * (size_t)c * SC_H));
    SCK(cudaMalloc(&s->Tb, sizeof(float) * c));
    SCK(cudaMalloc(&s->Y, sizeof(float) * c));
    SCK(cudaMalloc(&s->dYf, sizeof(float) * c));
    SCK(cudaMalloc(&s->dH2f, sizeof(float) * (size_t)c * SC_H));
    SCK(cudaMalloc(&s->dH1f, sizeof(float) * (size_t)c * SC_H));
    s->cap = c;
    return 0;
}

static GemmArgs gargs(const __nv_bfloat16* A, long long ar, long long ac, const __nv_bfloat16* B, long long br,
                      long long bc, int M, int N, int K)
{
    GemmArgs g;
    memset(&g, 0, sizeof(g));
    g.A = A; g.ar = ar; g.ac = ac; g.B = B; g.br = br; g.bc = bc; g.M = M; g.N = N; g.K = K; g.alpha = 1.f;
    return g;
}

// Forward of b gathered rows (s->Xb): H1, H2, Y (Y in target units x SC_TSCALE).
static void sc_forward(cuacd_scorer* s, int b, cudaStream_t st)
{
    GemmArgs g = gargs(s->Xb, SC_K, 1, s->pb + OFF_W1, SC_H, 1, b, SC_H, SC_K);
    g.bias = s->p32 + OFF_B1; g.relu = 1; g.Cb = s->H1; g.ldc = SC_H;
    gemm(g, s->gerr, st);
    g = gargs(s->H1, SC_H, 1, s->pb + OFF_W2, SC_H, 1, b, SC_H, SC_H);
    g.bias = s->p32 + OFF_B2; g.relu = 1; g.Cb = s->H2; g.ldc = SC_H;
    gemm(g, s->gerr, st);
    g = gargs(s->H2, SC_H, 1, s->pb + OFF_W3, 1, 0, b, 1, SC_H);
    g.bias = s->p32 + OFF_B3; g.Cf = s->Y; g.ldc = 1;
    gemm(g, s->gerr, st);
}

// Loss and gradients of the gathered batch into s->g32.
static void sc_backward(cuacd_scorer* s, int b, cudaStream_t st)
{
    k_mse_grad<<<1, 256, 0, st>>>(s->Y, s->Tb, b, s->dYb, s->dYf, s->loss);
    // W3, b3
    GemmArgs g = gargs(s->H2, 1, SC_H, s->dYb, 1, 0, SC_H, 1, b);
    g.Cf = s->g32 + OFF_W3; g.ldc = 1;
    gemm(g, s->gerr, st);
    k_colsum<<<1, 32, 0, st>>>(s->dYf, b, 1, s->g32 + OFF_B3);
    // dH2 = dY W3^T (H2 > 0)
    g = gargs(s->dYb, 1, 0, s->pb + OFF_W3, 0, 1, b, SC_H, 1);
    g.mask = s->H2; g.ldm = SC_H; g.Cf = s->dH2f; g.Cb = s->dH2b; g.ldc = SC_H;
    gemm(g, s->gerr, st);
    // W2, b2
    g = gargs(s->H1, 1, SC_H, s->dH2b, SC_H, 1, SC_H, SC_H, b);
    g.Cf = s->g32 + OFF_W2; g.ldc = SC_H;
    gemm(g, s->gerr, st);
    k_colsum<<<(SC_H + 127) / 128, 128, 0, st>>>(s->dH2f, b, SC_H, s->g32 + OFF_B2);
    // dH1 = dH2 W2^T (H1 > 0)
    g = gargs(s->dH2b, SC_H, 1, s->pb + OFF_W2, 1, SC_H, b, SC_H, SC_H);
    g.mask = s->H1; g.ldm = SC_H; g.Cf = s->dH1f; g.Cb = s->dH1b; g.ldc = SC_H;
    gemm(g, s->gerr, st);
    // W1, b1
    g = gargs(s->Xb, 1, SC_K, s->dH1b, SC_H, 1, SC_K, SC_H, b);
    g.Cf = s->g32 + OFF_W1; g.ldc = SC_H;
    gemm(g, s->gerr, st);
    k_colsum<<<(SC_H + 127) / 128, 128, 0, st>>>(s->dH1f, b, SC_H, s->g32 + OFF_B1);
}

static void sc_adamw(cuacd_scorer* s, float lr, float wd, cudaStream_t st)
{
    s->step++;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const float c1 = 1.f - powf(b1, (float)s->step), c2 = 1.f - powf(b2, (float)s->step);
    const size_t blocks[6][2] = {{OFF_W1, (size_t)SC_K * SC_H}, {OFF_B1, SC_H}, {OFF_W2, (size_t)SC_H * SC_H},
                                 {OFF_B2, SC_H}, {OFF_W3, SC_H}, {OFF_B3, 1}};
    for (int i = 0; i < 6; i++) {
        const size_t o = blocks[i][0], n = blocks[i][1];
        k_adamw<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(s->p32 + o, s->g32 + o, s->m + o, s->v + o, s->pb + o, n,
                                                             lr, b1, b2, eps, wd, c1, c2, (i % 2) == 0);
    }
}

static int sc_upload_rows(gpu_ctx* ctx, cuacd_scorer* s, const float* X, const float* T, int n)
{
    if (n > s->n_rows_cap) {
        cudaFree(s->X); cudaFree(s->T);
        SCK(cudaMalloc(&s->X, sizeof(float) * (size_t)n * SC_K));
        SCK(cudaMalloc(&s->T, sizeof(float) * (size_t)(n > 0 ? n : 1)));
        s->n_rows_cap = n;
    }
    SCK(cudaMemcpyAsync(s->X, X, sizeof(float) * (size_t)n * SC_K, cudaMemcpyHostToDevice, ctx->stream));
    if (T) SCK(cudaMemcpyAsync(s->T, T, sizeof(float) * (size_t)n, cudaMemcpyHostToDevice, ctx->stream));
    return 0;
}

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" int cuacd_scorer_n_params(void) { return (int)N_PARAMS; }

extern "C" void cuacd_scorer_gemm_counts(unsigned long long* tma, unsigned long long* staged)
{
    if (tma) *tma = g_gemm_tma;
    if (staged) *staged = g_gemm_staged;
}
extern "C" int cuacd_scorer_n_features(void) { return SC_K; }

extern "C" int cuacd_scorer_create(gpu_ctx_t ctx, unsigned seed, cuacd_scorer_t* out)
{
    if (!ctx || !out) return -1;
    *out = nullptr;
    SCK(cudaSetDevice(ctx->device));
    cuacd_scorer* s = (cuacd_scorer*)calloc(1, sizeof(cuacd_scorer));
    if (!s) return sc_fail(ctx, -1, "out of host memory");
    s->device = ctx->device;
    cudaError_t e = cudaMalloc(&s->p32, sizeof(float) * N_PARAMS);
    if (!e) e = cudaMalloc(&s->pb, sizeof(__nv_bfloat16) * N_PARAMS);
    if (!e) e = cudaMalloc(&s->g32, sizeof(float) * N_PARAMS);
    if (!e) e = cudaMalloc(&s->m, sizeof(float) * N_PARAMS);
    if (!e) e = cudaMalloc(&s->v, sizeof(float) * N_PARAMS);
    if (!e) e = cudaMalloc(&s->loss, sizeof(float));
    if (!e) e = cudaMalloc(&s->gerr, sizeof(int));
    if (!e) e = cudaMemset(s->gerr, 0, sizeof(int));
    if (!e) e = cudaMalloc(&s->nrm, sizeof(float) * 2 * SC_K);
    if (e) { cuacd_scorer_free(s); return ctx_fail(ctx, (int)e, "scorer allocation failed: %s", cudaGetErrorString(e)); }
    // He-uniform weights, zero biases
    std::vector<float> p(N_PARAMS, 0.f);
    std::mt19937 rng(seed);
    auto fill = [&](size_t off, int fan_in, size_t n) {
        const float a = sqrtf(6.f / (float)fan_in);
        std::uniform_real_distribution<float> U(-a, a);
        for (size_t i = 0; i < n; i++) p[off + i] = U(rng);
    };
    fill(OFF_W1, SC_NF, (size_t)SC_K * SC_H);
    for (int k = SC_NF; k < SC_K; k++) for (int j = 0; j < SC_H; j++) p[OFF_W1 + (size_t)k * SC_H + j] = 0.f;
    fill(OFF_W2, SC_H, (size_t)SC_H * SC_H);
    fill(OFF_W3, SC_H, SC_H);
    *out = s;
    std::vector<float> nrm(2 * SC_K, 0.f);
    for (int k = 0; k < SC_K; k++) nrm[SC_K + k] = 1.f;
    if (cuacd_scorer_set_normalizer(s, nrm.data(), nrm.data() + SC_K)) return ctx_fail(ctx, -1, "scorer set-up failed");
    return cuacd_scorer_set_params(s, p.data());
}

extern "C" int cuacd_scorer_set_normalizer(cuacd_scorer_t s, const float* mean, const float* inv_std)
{
    if (!s || !mean || !inv_std) return -1;
    if (cudaSetDevice(s->device)) return -1;
    if (cudaMemcpy(s->nrm, mean, sizeof(float) * SC_K, cudaMemcpyHostToDevice)) return -1;
    return cudaMemcpy(s->nrm + SC_K, inv_std, sizeof(float) * SC_K, cudaMemcpyHostToDevice) == cudaSuccess ? 0 : -1;
}

extern "C" int cuacd_scorer_get_normalizer(cuacd_scorer_t s, float* mean, float* inv_std)
{
    if (!s || !mean || !inv_std) return -1;
    if (cudaSetDevice(s->device)) return -1;
    if (cudaMemcpy(mean, s->nrm, sizeof(float) * SC_K, cudaMemcpyDeviceToHost)) return -1;
    return cudaMemcpy(inv_std, s->nrm + SC_K, sizeof(float) * SC_K, cudaMemcpyDeviceToHost) == cudaSuccess ? 0 : -1;
}

extern "C" void cuacd_scorer_free(cuacd_scorer_t s)
{
    if (!s) return;
    cudaSetDevice(s->device);
    cudaFree(s->p32); cudaFree(s->pb); cudaFree(s->g32); cudaFree(s->m); cudaFree(s->v); cudaFree(s->loss);
    cudaFree(s->gerr); cudaFree(s->nrm);
    cudaFree(s->X); cudaFree(s->T); cudaFree(s->idx); cudaFree(s->Xb); cudaFree(s->H1); cudaFree(s->H2);
    cudaFree(s->dYb); cudaFree(s->dH2b); cudaFree(s->dH1b); cudaFree(s->Tb); cudaFree(s->Y); cudaFree(s->dYf);
    cudaFree(s->dH2f); cudaFree(s->dH1f); cudaFree(s->mv); cudaFree(s->mt); cudaFree(s->mp); cudaFree(s->st);
    cudaFree(s->pr); cudaFreeHost(s->h_count); cudaFree(s->hx);
    free(s);                     // s->feat points into s->mp
    cudaGetLastError();          // a failed free must not surface in the next call's launch check
}

extern "C" int cuacd_scorer_set_params(cuacd_scorer_t s, const float* params)
{
    if (!s || !params) return -1;
    if (cudaSetDevice(s->device)) return -1;
    if (cudaMemcpy(s->p32, params, sizeof(float) * N_PARAMS, cudaMemcpyHostToDevice)) return -1;
    k_f32_to_bf16<<<(unsigned)((N_PARAMS + 255) / 256), 256>>>(s->p32, s->pb, N_PARAMS);
    if (cudaMemset(s->m, 0, sizeof(float) * N_PARAMS) || cudaMemset(s->v, 0, sizeof(float) * N_PARAMS)) return -1;
    s->step = 0;
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : -1;
}

extern "C" int cuacd_scorer_get_params(cuacd_scorer_t s, float* params)
{
    if (!s || !params) return -1;
    if (cudaSetDevice(s->device)) return -1;
    return cudaMemcpy(params, s->p32, sizeof(float) * N_PARAMS, cudaMemcpyDeviceToHost) == cudaSuccess ? 0 : -1;
}

// Predicted scores of rows already gathered in s->Xb (device), into s->Y.
static void sc_predict_rows(cuacd_scorer* s, int n, cudaStream_t st) { sc_forward(s, n, st); }

static int sc_grow(gpu_ctx* ctx, void** p, size_t& cap, size_t need)
{
    if (need <= cap) return 0;
    cudaFree(*p);
    *p = nullptr;
    cap = 0;
    SCK(cudaMalloc(p, need));
    cap = need;
    return 0;
}

// Room for n planes and their feature rows in s->mp (s->feat follows the planes).
static int sc_feature_buffers(gpu_ctx* ctx, cuacd_scorer* s, int n)
{
    const size_t plane_bytes = (16 * (size_t)n + 255) & ~(size_t)255;
    if (sc_grow(ctx, (void**)&s->mp, s->mp_cap, plane_bytes + sizeof(float) * (size_t)n * SC_K)) return -1;
    if (!s->st) SCK(cudaMalloc(&s->st, sizeof(PartStats)));
    s->feat = (float*)((char*)s->mp + plane_bytes);
    return 0;
}

// Part statistics and the feature rows of n planes (device pointers) into s->feat.
static void sc_launch_features(gpu_ctx* ctx, cuacd_scorer* s, const float* d_v, int nv, const int* d_t, int nt,
                               float hull_vol, const float4* d_planes, int n, cudaStream_t st)
{
    k_part_stats<<<1, 256, 0, st>>>(d_v, nv, d_t, nt, hull_vol, s->st);
    k_cand_features<<<n, 256, 0, st>>>(d_v, nv, d_planes, n, s->st, s->feat);
    ctx->launches += 2;
}

// Features of n planes on one part (host pointers), SC_K floats per plane.
static int sc_features_device(gpu_ctx* ctx, cuacd_scorer* s, const float* verts, int nv, const int* tris, int nt,
                              float hull_vol, const float* planes, int n, cudaStream_t st)
{
    if (sc_grow(ctx, (void**)&s->mv, s->mv_cap, 12 * (size_t)nv)) return -1;
    if (sc_grow(ctx, (void**)&s->mt, s->mt_cap, 12 * (size_t)(nt > 0 ? nt : 1))) return -1;
    if (sc_feature_buffers(ctx, s, n)) return -1;
    SCK(cudaMemcpyAsync(s->mv, verts, 12 * (size_t)nv, cudaMemcpyHostToDevice, st));
    if (nt) SCK(cudaMemcpyAsync(s->mt, tris, 12 * (size_t)nt, cudaMemcpyHostToDevice, st));
    SCK(cudaMemcpyAsync(s->mp, planes, 16 * (size_t)n, cudaMemcpyHostToDevice, st));
    sc_launch_features(ctx, s, s->mv, nv, s->mt, nt, hull_vol, s->mp, n, st);
    SCK(cudaGetLastError());
    return 0;
}

// After a synchronisation: a tensor-core wait of the GEMMs that gave up
// (error word set) fails the call, and the word is cleared.
static int sc_check_gemm(gpu_ctx* ctx, cuacd_scorer* s, cudaStream_t st)
{
    int e = 0;
    SCK(cudaMemcpyAsync(&e, s->gerr, sizeof(int), cudaMemcpyDeviceToHost, st));
    SCK(cudaStreamSynchronize(st));
    if (!e) return 0;
    SCK(cudaMemsetAsync(s->gerr, 0, sizeof(int), st));
    return ctx_fail(ctx, e, "scorer GEMM: a tensor-core wait gave up (0x%x)", e);
}

int scorer_predict_parts(gpu_ctx* ctx, cuacd_scorer* s, const ScorerPart* parts, int n_parts,
                         const float4* d_planes, int n_rows, float* pred, cudaStream_t st)
{
    if (n_rows <= 0) return 0;
    if (sc_feature_buffers(ctx, s, n_rows) || sc_reserve(ctx, s, n_rows)) return -1;
    for (int i = 0; i < n_parts; i++) {
        const ScorerPart& p = parts[i];
        if (p.n <= 0) continue;
        k_part_stats<<<1, 256, 0, st>>>(p.v, p.nv, p.t, p.nt, p.hull_vol, s->st);
        k_cand_features<<<p.n, 256, 0, st>>>(p.v, p.nv, d_planes + p.off, p.n, s->st, s->feat + (size_t)p.off * SC_K);
        ctx->launches += 2;
    }
    k_gather_rows<<<n_rows, 64, 0, st>>>(s->feat, nullptr, nullptr, n_rows, s->nrm, s->Xb, nullptr);
    sc_predict_rows(s, n_rows, st);
    ctx->launches += 4;
    SCK(cudaGetLastError());
    SCK(cudaMemcpyAsync(pred, s->Y, sizeof(float) * (size_t)n_rows, cudaMemcpyDeviceToHost, st));
    SCK(cudaStreamSynchronize(st));
    if (sc_check_gemm(ctx, s, st)) return -1;
    for (int i = 0; i < n_rows; i++) pred[i] /= SC_TSCALE;
    return 0;
}

int scorer_copy_features(gpu_ctx* ctx, cuacd_scorer* s, int n_rows, float* out, cudaStream_t st)
{
    if (n_rows <= 0) return 0;
    SCK(cudaMemcpyAsync(out, s->feat, sizeof(float) * (size_t)n_rows * SC_K, cudaMemcpyDeviceToHost, st));
    SCK(cudaStreamSynchronize(st));
    return 0;
}

int scorer_n_features() { return SC_K; }

extern "C" int cuacd_candidate_features(gpu_ctx_t ctx, cuacd_scorer_t s, const float* verts, int nv, const int* tris,
                                        int nt, float hull_vol, const float* planes, int n, float* out)
{
    if (!ctx || !s || !out) return -1;
    if (n <= 0) return 0;
    if (nv <= 0) return ctx_fail(ctx, KERR_MESH_INVALID, "empty mesh");
    for (int i = 0; i < 3 * nt; i++) if (tris[i] < 0 || tris[i] >= nv) return ctx_fail(ctx, KERR_MESH_INVALID, "index out of range");
    SCK(cudaSetDevice(ctx->device));
    if (sc_features_device(ctx, s, verts, nv, tris, nt, hull_vol, planes, n, ctx->stream)) return -1;
    SCK(cudaMemcpyAsync(out, s->feat, sizeof(float) * (size_t)n * SC_K, cudaMemcpyDeviceToHost, ctx->stream));
    return sync_and_check(ctx, "candidate_features");
}

extern "C" int cuacd_scorer_grad(gpu_ctx_t ctx, cuacd_scorer_t s, const float* X, const float* T, int n,
                                 float* loss, float* grads)
{
    if (!ctx || !s || !X || !T || n <= 0) return -1;
    SCK(cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    if (sc_reserve(ctx, s, n) || sc_upload_rows(ctx, s, X, T, n)) return -1;
    k_gather_rows<<<n, 64, 0, st>>>(s->X, s->T, nullptr, n, s->nrm, s->Xb, s->Tb);
    sc_forward(s, n, st);
    sc_backward(s, n, st);
    ctx->launches += 13;
    SCK(cudaGetLastError());
    if (loss) SCK(cudaMemcpyAsync(loss, s->loss, sizeof(float), cudaMemcpyDeviceToHost, st));
    if (grads) SCK(cudaMemcpyAsync(grads, s->g32, sizeof(float) * N_PARAMS, cudaMemcpyDeviceToHost, st));
    int rc = sync_and_check(ctx, "scorer_grad");
    return rc ? rc : sc_check_gemm(ctx, s, st);
}

extern "C" int cuacd_scorer_train(gpu_ctx_t ctx, cuacd_scorer_t s, const float* X, const float* T, int n, int epochs,
                                  int batch, float lr, float wd, unsigned seed, float* final_loss)
{
    if (!ctx || !s || !X || !T || n <= 0 || epochs <= 0 || batch <= 0) return -1;
    SCK(cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    batch = std::min(batch, n);
    if (sc_reserve(ctx, s, batch) || sc_upload_rows(ctx, s, X, T, n)) return -1;
    std::vector<int> perm(n);
    for (int i = 0; i < n; i++) perm[i] = i;
    std::mt19937 rng(seed);
    int* d_perm = nullptr;
    SCK(cudaMalloc(&d_perm, sizeof(int) * (size_t)n));
    double loss_sum = 0.0; int loss_cnt = 0;
    std::vector<float> losses;
    float* d_losses = nullptr;
    const int steps_per_epoch = n / batch;
    SCK(cudaMalloc(&d_losses, sizeof(float) * (size_t)(steps_per_epoch > 0 ? steps_per_epoch : 1)));
    for (int ep = 0; ep < epochs; ep++) {
        std::shuffle(perm.begin(), perm.end(), rng);
        SCK(cudaMemcpyAsync(d_perm, perm.data(), sizeof(int) * (size_t)n, cudaMemcpyHostToDevice, st));
        for (int b = 0; b < steps_per_epoch; b++) {
            k_gather_rows<<<batch, 64, 0, st>>>(s->X, s->T, d_perm + (size_t)b * batch, batch, s->nrm, s->Xb,
                                                 s->Tb);
            sc_forward(s, batch, st);
            sc_backward(s, batch, st);
            sc_adamw(s, lr, wd, st);
            cudaMemcpyAsync(d_losses + b, s->loss, sizeof(float), cudaMemcpyDeviceToDevice, st);
            ctx->launches += 20;
        }
        if (ep == epochs - 1 && steps_per_epoch > 0) {
            losses.resize(steps_per_epoch);
            SCK(cudaMemcpyAsync(losses.data(), d_losses, sizeof(float) * steps_per_epoch, cudaMemcpyDeviceToHost, st));
        }
    }
    int rc = sync_and_check(ctx, "scorer_train");
    cudaFree(d_perm); cudaFree(d_losses);
    if (!rc) rc = sc_check_gemm(ctx, s, st);
    if (rc) return rc;
    for (float l : losses) { loss_sum += l; loss_cnt++; }
    if (final_loss) *final_loss = loss_cnt ? (float)(loss_sum / loss_cnt) / (SC_TSCALE * SC_TSCALE) : 0.f;
    return 0;
}


extern "C" int cuacd_scorer_predict(gpu_ctx_t ctx, cuacd_scorer_t s, const float* X, int n, float* out)
{
    if (!ctx || !s || !X || !out) return -1;
    if (n <= 0) return 0;
    SCK(cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    if (sc_reserve(ctx, s, n) || sc_upload_rows(ctx, s, X, nullptr, n)) return -1;
    k_gather_rows<<<n, 64, 0, st>>>(s->X, nullptr, nullptr, n, s->nrm, s->Xb, nullptr);
    sc_predict_rows(s, n, st);
    ctx->launches += 4;
    SCK(cudaGetLastError());
    std::vector<float> y(n);
    SCK(cudaMemcpyAsync(y.data(), s->Y, sizeof(float) * (size_t)n, cudaMemcpyDeviceToHost, st));
    int rc = sync_and_check(ctx, "scorer_predict");
    if (!rc) rc = sc_check_gemm(ctx, s, st);
    if (rc) return rc;
    for (int i = 0; i < n; i++) out[i] = y[i] / SC_TSCALE;
    return 0;
}

// Surrogate-pruned evaluation of n planes on one mesh (host pointers; hull_vol
// < 0 computes the part's hull volume here): the
// network predicts every plane's score_full; the top_k lowest predictions,
// plus every plane whose prediction lies within `margin` of the k-th (the
// cases where the ranking is too close to trust), go through the exact
// evaluator.  out[i] is the exact result of an evaluated plane; the others
// get ok = 0 and scores of FLT_MAX.  out_pred (optional) receives the
// predictions, out_evaluated (optional) 1/0 per plane; *out_n_evaluated the
// count.
extern "C" int cuacd_eval_candidates_pruned(gpu_ctx_t ctx, cuacd_scorer_t s, const float* verts, int nv,
                                            const int* tris, int nt, float hull_vol, const float* planes,
                                            int n_planes, int flags,
                                            float hd_resolution, int hd_min_samples, int hd_total, int top_k,
                                            float margin, cuacd_cand_result* out, float* out_pred,
                                            int* out_evaluated, int* out_n_evaluated)
{
    if (!ctx || !s || !out) return -1;
    if (out_n_evaluated) *out_n_evaluated = 0;
    if (n_planes <= 0) return 0;
    if (nv <= 0 || nt <= 0) return ctx_fail(ctx, KERR_MESH_INVALID, "empty mesh");
    for (int i = 0; i < 3 * nt; i++)
        if (tris[i] < 0 || tris[i] >= nv) return ctx_fail(ctx, KERR_MESH_INVALID, "triangle index out of range");
    if (top_k <= 0) top_k = 1;
    SCK(cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    if (hull_vol < 0.f) {       // the exact hull of the part's vertices
        std::vector<float> hv(3 * (size_t)nv);
        std::vector<int> ht(6 * (size_t)nv + 12);
        int hnv = 0, hnt = 0, herr = 0;
        const int off[2] = {0, nv};
        int rc = gpu_kdop_hull(ctx, verts, nv, off, 1, nv, 2 * nv + 4, hv.data(), ht.data(), &hnv, &hnt,
                               &hull_vol, &herr);
        if (rc) return rc;
    }
    // Stage the mesh and planes in the scorer's own device buffers and run
    // the device-pointer form (features, network, selection and the exact
    // evaluation of the kept planes, whose cuts overlap the ranking).
    if (n_planes > SC_SEL_MAX) return ctx_fail(ctx, -1, "pruned evaluation takes at most %d planes", SC_SEL_MAX);
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    const size_t o_t = al(12 * (size_t)nv), o_p = o_t + al(12 * (size_t)nt), o_r = o_p + al(16 * (size_t)n_planes);
    const size_t o_y = o_r + al(sizeof(cuacd_cand_result) * (size_t)n_planes), o_e = o_y + al(4 * (size_t)n_planes);
    if (sc_grow(ctx, (void**)&s->hx, s->hx_cap, o_e + al(4 * (size_t)n_planes))) return -1;
    float* dv = (float*)s->hx;
    int* dt = (int*)(s->hx + o_t);
    float* dp = (float*)(s->hx + o_p);
    cuacd_cand_result* dres = (cuacd_cand_result*)(s->hx + o_r);
    float* dpred = (float*)(s->hx + o_y);
    int* deval = (int*)(s->hx + o_e);
    SCK(cudaMemcpyAsync(dv, verts, 12 * (size_t)nv, cudaMemcpyHostToDevice, st));
    SCK(cudaMemcpyAsync(dt, tris, 12 * (size_t)nt, cudaMemcpyHostToDevice, st));
    SCK(cudaMemcpyAsync(dp, planes, 16 * (size_t)n_planes, cudaMemcpyHostToDevice, st));
    int n_eval = 0;
    int rc = cuacd_eval_candidates_pruned_device(ctx, s, dv, nv, dt, nt, hull_vol, dp, n_planes, flags,
                                                 hd_resolution, hd_min_samples, hd_total, top_k, margin, dres, dpred,
                                                 deval, &n_eval, st);
    if (rc) return rc;
    SCK(cudaMemcpyAsync(out, dres, sizeof(cuacd_cand_result) * (size_t)n_planes, cudaMemcpyDeviceToHost, st));
    if (out_pred) SCK(cudaMemcpyAsync(out_pred, dpred, 4 * (size_t)n_planes, cudaMemcpyDeviceToHost, st));
    std::vector<int> evl(n_planes);
    SCK(cudaMemcpyAsync(evl.data(), deval, 4 * (size_t)n_planes, cudaMemcpyDeviceToHost, st));
    rc = sync_and_check(ctx, "eval_candidates_pruned");
    if (rc) return rc;
    if (out_n_evaluated) *out_n_evaluated = n_eval;
    if (out_evaluated) memcpy(out_evaluated, evl.data(), 4 * (size_t)n_planes);
    // An arena too small for this mesh: evaluate the kept planes again
    // through the host entry point, which grows the pool and retries.
    std::vector<int> kept;
    bool oom = false;
    for (int i = 0; i < n_planes; i++) {
        if (!evl[i]) continue;
        kept.push_back(i);
        if (out[i].err & (KERR_HEAP_OOM | KERR_PC_SCRATCH_OOM | KERR_HD_SCRATCH_OOM)) oom = true;
    }
    if (oom) {
        std::vector<float> sp(4 * kept.size());
        for (size_t j = 0; j < kept.size(); j++) memcpy(&sp[4 * j], planes + 4 * (size_t)kept[j], 16);
        std::vector<cuacd_cand_result> res(kept.size());
        rc = cuacd_eval_candidates(ctx, verts, nv, tris, nt, sp.data(), (int)kept.size(), flags, hd_resolution,
                                   hd_min_samples, hd_total, res.data());
        if (rc) return rc;
        for (size_t j = 0; j < kept.size(); j++) out[kept[j]] = res[j];
    }
    return 0;
}

// Device-pointer form of the pruned evaluation on `stream`: features,
// network, selection and the scatter of results all run on the device; the
// call waits once, for the selected count, before it launches the exact
// evaluator on the selected planes.  hull_vol must be the part's hull volume.
extern "C" int cuacd_eval_candidates_pruned_device(gpu_ctx_t ctx, cuacd_scorer_t s, const float* d_verts, int nv,
                                                   const int* d_tris, int nt, float hull_vol, const float* d_planes,
                                                   int n_planes, int flags, float hd_resolution, int hd_min_samples,
                                                   int hd_total, int top_k, float margin, cuacd_cand_result* d_out,
                                                   float* d_pred, int* d_evaluated, int* out_n_evaluated,
                                                   void* stream)
{
    if (!ctx || !s || !d_out) return -1;
    if (out_n_evaluated) *out_n_evaluated = 0;
    if (n_planes <= 0) return 0;
    if (n_planes > SC_SEL_MAX) return ctx_fail(ctx, -1, "pruned evaluation takes at most %d planes", SC_SEL_MAX);
    if (nv <= 0 || nt <= 0) return ctx_fail(ctx, KERR_MESH_INVALID, "empty mesh");
    if (!(hull_vol >= 0.f)) return ctx_fail(ctx, -1, "hull_vol must be the part's hull volume");
    if (top_k <= 0) top_k = 1;
    const int k = std::min(top_k, n_planes);
    SCK(cudaSetDevice(ctx->device));
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    const size_t o_pos = al(16 * (size_t)n_planes), o_cnt = o_pos + al(4 * (size_t)n_planes), o_sub = o_cnt + 256;
    if (sc_grow(ctx, (void**)&s->pr, s->pr_cap, o_sub + sizeof(cuacd_cand_result) * (size_t)n_planes)) return -1;
    if (!s->h_count) SCK(cudaMallocHost(&s->h_count, sizeof(int)));
    if (sc_feature_buffers(ctx, s, n_planes) || sc_reserve(ctx, s, n_planes)) return -1;
    float4* sel = (float4*)s->pr;
    int* pos = (int*)(s->pr + o_pos);
    int* cnt = (int*)(s->pr + o_cnt);
    cuacd_cand_result* sub = (cuacd_cand_result*)(s->pr + o_sub);
    // Outside stage profiling the cuts of all planes run on a second stream
    // while the network ranks them (the profiled stages stay one serial
    // pipeline, timed per stage).
    const bool overlap = !ctx->profile;
    EvalPrecut P;
    struct Release {                   // the work set of an overlapped evaluation, on every return path
        EvalPrecut& p;
        ~Release() { eval_precut_release(p); }
    } release{P};
    if (overlap) {
        int rc = eval_precut_begin(ctx, d_verts, nv, d_tris, nt, (const float4*)d_planes, n_planes, P, st);
        if (rc) return rc;
    }
    sc_launch_features(ctx, s, d_verts, nv, d_tris, nt, hull_vol, (const float4*)d_planes, n_planes, st);
    k_gather_rows<<<n_planes, 64, 0, st>>>(s->feat, nullptr, nullptr, n_planes, s->nrm, s->Xb, nullptr);
    sc_predict_rows(s, n_planes, st);
    k_select_planes<<<1, 256, 0, st>>>(s->Y, n_planes, k, margin, (const float4*)d_planes, sel, pos, cnt, d_pred);
    ctx->launches += 5;
    SCK(cudaGetLastError());
    SCK(cudaMemcpyAsync(s->h_count, cnt, sizeof(int), cudaMemcpyDeviceToHost, st));
    SCK(cudaStreamSynchronize(st));
    const int n_sel = *s->h_count;
    int rc = overlap ? eval_precut_finish(ctx, P, pos, n_sel, flags, hd_resolution, hd_min_samples, hd_total, sub, st)
                     : cuacd_eval_candidates_device(ctx, d_verts, nv, d_tris, nt, (const float*)sel, n_sel, flags,
                                                    hd_resolution, hd_min_samples, hd_total, sub, st);
    if (rc) return rc;
    k_scatter_results<<<(n_planes + 127) / 128, 128, 0, st>>>(sub, pos, n_planes, d_out, d_evaluated);
    ctx->launches += 1;
    SCK(cudaGetLastError());
    if (out_n_evaluated) *out_n_evaluated = n_sel;
    return 0;
}
