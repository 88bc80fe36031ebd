// volume.cuh — batched mesh volume (divergence theorem), sm_100a.
//
// Replaces batch_mesh_volume_kernel / mesh_volume_kernel
// (cuda/test_mesh_volume.cu:13-63, one warp per mesh over
// cuda/mesh_volume.cuh:20-57).  Here the triangles of all meshes are cut into
// fixed tiles of VOL_TILE triangles that never straddle a mesh; each CTA
// reduces its tile in FP64 (signed tets anchored at the mesh's vertex 0), and
// a second pass adds the tile partials of each mesh in tile order, so the
// result does not depend on scheduling.  The grid covers every SM several
// times over, which is what an HBM-bound pass over 12-byte index triples and
// 12-byte vertex gathers needs.
#pragma once
#include "common.cuh"

#define VOL_NT   256
#define VOL_TILE 2048

// tile_mesh[t] = mesh of tile t; tile_first[t] = first triangle (global index)
__global__ void __launch_bounds__(VOL_NT)
k_volume_tiles(const float* __restrict__ verts, const int* __restrict__ tris,
               const int* __restrict__ tri_off, const int* __restrict__ vert_off,
               const int* __restrict__ tile_mesh, const int* __restrict__ tile_first,
               int n_tiles, double* __restrict__ partial)
{
    __shared__ double sh[33];
    int t = blockIdx.x;
    if (t >= n_tiles) return;
    int m = tile_mesh[t];
    int a = tile_first[t];
    int b = min(a + VOL_TILE, tri_off[m + 1]);
    int vo = vert_off ? vert_off[m] : 0;
    const float* v = verts + 3 * (size_t)vo;
    double ox = v[0], oy = v[1], oz = v[2];
    double acc = 0.0;
    for (int i = a + threadIdx.x; i < b; i += VOL_NT) {
        int i0 = __ldg(&tris[3 * (size_t)i]), i1 = __ldg(&tris[3 * (size_t)i + 1]), i2 = __ldg(&tris[3 * (size_t)i + 2]);
        acc += tet6_d(v, i0, i1, i2, ox, oy, oz);
    }
    double s = block_sum_d(acc, sh);
    if (threadIdx.x == 0) partial[t] = s;
}

__global__ void k_volume_reduce(const int* __restrict__ mesh_tile0, const double* __restrict__ partial,
                                int n_meshes, float* __restrict__ out)
{
    int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= n_meshes) return;
    double s = 0.0;
    for (int t = mesh_tile0[m]; t < mesh_tile0[m + 1]; t++) s += partial[t];
    out[m] = (float)fabs(s / 6.0);
}
