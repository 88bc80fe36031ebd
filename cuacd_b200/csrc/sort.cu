// sort.cu — gpu_test_warp_sort: sort (x,y,z,index) int records by
// (y,x,z,index), one CTA per sub-array (replaces the reference's warp
// quicksort, cuda/warp_sort.cuh:54-250, and its test kernel
// cuda/test_warp_sort.cu:14).  A CTA bitonic network in shared memory for
// sub-arrays up to 4096 records, in global memory beyond.
#include <vector>
#include "context.cuh"

#define SORT_NT 256
#define SORT_SMEM 2048

__device__ __forceinline__ bool rec_less(int4 a, int4 b)
{
    if (a.y != b.y) return a.y < b.y;
    if (a.x != b.x) return a.x < b.x;
    if (a.z != b.z) return a.z < b.z;
    return a.w < b.w;
}

__device__ void bitonic_int4(int4* keys, int n, int N)
{
    for (int i = n + threadIdx.x; i < N; i += SORT_NT) keys[i] = make_int4(0x7fffffff, 0x7fffffff, 0x7fffffff, 0x7fffffff);
    __syncthreads();
    for (int k = 2; k <= N; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = threadIdx.x; i < N; i += SORT_NT) {
                int l = i ^ j;
                if (l > i) {
                    int4 a = keys[i], b = keys[l];
                    bool up = (i & k) == 0;
                    if (rec_less(b, a) == up) { keys[i] = b; keys[l] = a; }
                }
            }
            __syncthreads();
        }
}

__global__ void __launch_bounds__(SORT_NT)
k_sort_records(int4* recs, const int* offsets, int n_arrays, int4* gscratch, const long long* gofs)
{
    __shared__ int4 sm[SORT_SMEM];
    int a = blockIdx.x;
    if (a >= n_arrays) return;
    int lo = offsets[a], n = offsets[a + 1] - lo;
    if (n <= 1) return;
    int N = 1; while (N < n) N <<= 1;
    int4* buf = N <= SORT_SMEM ? sm : gscratch + gofs[a];
    for (int i = threadIdx.x; i < n; i += SORT_NT) buf[i] = recs[lo + i];
    __syncthreads();
    bitonic_int4(buf, n, N);
    for (int i = threadIdx.x; i < n; i += SORT_NT) recs[lo + i] = buf[i];
}

extern "C" int gpu_test_warp_sort(gpu_ctx_t ctx, int* points, int total_pts, const int* offsets, int n_arrays)
{
    if (!ctx) return -1;
    if (n_arrays <= 0) return 0;
    std::vector<long long> gofs(n_arrays);
    long long g = 0;
    for (int i = 0; i < n_arrays; i++) {
        int n = offsets[i + 1] - offsets[i];
        if (n < 0 || offsets[i + 1] > total_pts) return ctx_fail(ctx, KERR_MESH_INVALID, "bad offsets");
        int N = 1; while (N < n) N <<= 1;
        gofs[i] = g;
        if (N > SORT_SMEM) g += N;
    }
    CK(cudaSetDevice(ctx->device));
    size_t need = al256(16 * (size_t)total_pts) + al256(4 * (size_t)(n_arrays + 1)) + al256(8 * (size_t)n_arrays)
                + al256(16 * (size_t)(g > 0 ? g : 1));
    int rc = pool_begin(ctx, need);
    if (rc) return rc;
    int4* d_r = pool_take<int4>(ctx, total_pts);
    int* d_o = pool_take<int>(ctx, n_arrays + 1);
    long long* d_g = pool_take<long long>(ctx, n_arrays);
    int4* d_s = pool_take<int4>(ctx, g > 0 ? g : 1);
    cudaStream_t s = ctx->stream;
    CK(cudaMemcpyAsync(d_r, points, 16 * (size_t)total_pts, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(d_o, offsets, 4 * (size_t)(n_arrays + 1), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(d_g, gofs.data(), 8 * (size_t)n_arrays, cudaMemcpyHostToDevice, s));
    k_sort_records<<<n_arrays, SORT_NT, 0, s>>>(d_r, d_o, n_arrays, d_s, d_g);
    ctx->launches++;
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(points, d_r, 16 * (size_t)total_pts, cudaMemcpyDeviceToHost, s));
    return sync_and_check(ctx, "warp_sort");
}
