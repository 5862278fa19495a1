// Discrete distance queries on an EDT'd DistanceVoxel map.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "gvx_internal.cuh"

namespace gvx {
namespace {

// DistanceVoxel::squaredObstacleDistance (GV/voxel/DistanceVoxel.hpp:40-55).
__device__ __forceinline__ int32_t sqdist_at(uint32_t v, int px, int py, int pz) {
  const int ox = (int)dv_x(v), oy = (int)dv_y(v), oz = (int)dv_z(v);
  if (px == (int)kUninit || py == (int)kUninit || pz == (int)kUninit || ox == (int)kUninit || oy == (int)kUninit ||
      oz == (int)kUninit)
    return kMaxObstacleDistance;
  const int dx = px - ox, dy = py - oy, dz = pz - oz;
  return dx * dx + dy * dy + dz * dz;
}

// getSquaredDistances / SquaredDistanceFunctor (GV/voxelmap/DistanceVoxelMap.hpp:709-752),
// getDistances / DistanceFunctor (:754-797) and gatherVoxelsByIndex
// (GV/voxelmap/TemplateVoxelMap.hpp:381-388), fused: one gather per id, no
// temporary buffer.  mode 0: squared distance, 1: int32(sqrtf), 2: raw voxel.
__global__ void sqdist_kernel(const uint32_t* __restrict__ map, uint32_t X, uint32_t layer, uint64_t nvox,
                              const uint32_t* __restrict__ ids, uint64_t n, int32_t* __restrict__ out, int mode) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const uint32_t id = __ldg(ids + i);
    int32_t r;
    if (id >= nvox) {
      r = (mode == 2) ? (int32_t)kDvUninit : kMaxObstacleDistance;
    } else {
      const uint32_t v = __ldg(map + id);
      if (mode == 2) {
        r = (int32_t)v;
      } else {
        const uint32_t z = id / layer, rem = id - z * layer, y = rem / X, x = rem - y * X;  // mapToVoxels(uint, dims)
        r = sqdist_at(v, (int)x, (int)y, (int)z);
        if (mode == 1) r = (int32_t)sqrtf((float)r);
      }
    }
    out[i] = r;
  }
}

__global__ void sqdist_map_kernel(const uint32_t* __restrict__ map, uint32_t X, uint32_t Y, uint64_t nvox,
                                  int32_t* __restrict__ out) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t layer = (uint64_t)X * Y;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nvox; i += stride) {
    const uint32_t z = (uint32_t)(i / layer), rem = (uint32_t)(i - z * layer), y = rem / X, x = rem - y * X;
    out[i] = sqdist_at(__ldg(map + i), (int)x, (int)y, (int)z);
  }
}

unsigned grid_for(uint64_t n) {
  return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((n + 255) / 256, (uint64_t)device_sms() * 16));
}

}  // namespace

cudaError_t launch_dvm_sqdist(const uint32_t* d_vox, gvx_dims d, const uint32_t* d_ids, uint64_t n, int32_t* d_out,
                              int mode, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  sqdist_kernel<<<grid_for(n), 256, 0, s>>>(d_vox, d.x, d.x * d.y, num_voxels(d), d_ids, n, d_out, mode);
  return cudaGetLastError();
}

cudaError_t launch_dvm_sqdist_map(const uint32_t* d_vox, gvx_dims d, int32_t* d_out, cudaStream_t s) {
  sqdist_map_kernel<<<grid_for(num_voxels(d)), 256, 0, s>>>(d_vox, d.x, d.y, num_voxels(d), d_out);
  return cudaGetLastError();
}

}  // namespace gvx
