// ProbVoxelMap (one int8 log-odds occupancy per voxel) and its merge into a
// DistanceVoxelMap, the producer of EDT obstacles from probabilistic sensor
// fusion in gpu-voxels.
//   insert: kernelInsertGlobalPointCloud<ProbabilisticVoxel>
//           (GV/voxelmap/kernels/VoxelMapOperations.hpp:241-264) with
//           ProbabilisticVoxel::insert / updateOccupancy
//           (GV/voxel/ProbabilisticVoxel.hpp:44-100)
//   merge:  DistanceVoxelMap::mergeOccupied (GV/voxelmap/DistanceVoxelMap.hpp:109-136,
//           operators GV/voxelmap/DistanceVoxelMap.h:92-134)
// The reference updates a voxel with a plain read-modify-write, so points
// that share a voxel within one call can lose updates.  Here every point's
// update is applied (a compare-and-swap on the voxel's 32-bit word): the
// updates of one call are all the same saturating step, so the result does
// not depend on their order.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "gvx_internal.cuh"

namespace gvx {
namespace {

// updateOccupancy for `meaning` (constants GV/helpers/common_defines.h:50-63,154-161).
__device__ __forceinline__ int prob_step(int cur, int mode, int delta) {
  if (mode == 0) return -128;    // eBVM_UNKNOWN / eBVM_UNDEFINED / unused meanings
  if (cur == -128) return delta;  // an unknown voxel starts at probability 0.5
  return min(max(cur + delta, -127), 127);
}

__global__ void pvm_insert_kernel(uint32_t* __restrict__ words, uint32_t X, uint32_t Y, uint32_t Z, float side,
                                  const float* __restrict__ xyz, uint64_t n, int mode, int delta,
                                  uint32_t* __restrict__ outside) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  bool out = false;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const uint32_t x = coord_to_voxel(__ldg(xyz + 3 * i), side), y = coord_to_voxel(__ldg(xyz + 3 * i + 1), side),
                   z = coord_to_voxel(__ldg(xyz + 3 * i + 2), side);
    if (x < X && y < Y && z < Z) {
      const uint64_t id = ((uint64_t)z * Y + y) * X + x;
      uint32_t* w = words + (id >> 2);
      const int sh = (int)(id & 3) * 8;
      uint32_t old = *reinterpret_cast<volatile uint32_t*>(w);
      for (;;) {  // ends: each retry follows another thread's successful swap
        const int cur = (int)(int8_t)(old >> sh);
        const int nxt = prob_step(cur, mode, delta);
        if (nxt == cur) break;
        const uint32_t upd = (old & ~(0xFFu << sh)) | ((uint32_t)(uint8_t)(int8_t)nxt << sh);
        const uint32_t seen = atomicCAS(w, old, upd);
        if (seen == old) break;
        old = seen;
      }
    } else {
      out = true;
    }
  }
  if (outside != nullptr && __any_sync(0xffffffffu, out) && (threadIdx.x & 31) == 0) *outside = 1u;
}

// 16 voxels per thread step: one 16-byte load of occupancies; occupied voxels
// get the site of their own coordinates plus the offset (32-bit wrap, as the
// reference's DistanceVoxel(Vector3ui) constructor, GV/voxel/DistanceVoxel.hpp:61-65).
__global__ void merge_occupied_kernel(uint32_t* __restrict__ dvm, const int8_t* __restrict__ pvm, uint32_t X, uint32_t Y,
                                      uint64_t n, uint32_t ox, uint32_t oy, uint32_t oz, int thr) {
  const uint64_t n16 = n / 16;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  auto put = [&](uint64_t id) {
    const uint32_t x = (uint32_t)(id % X), y = (uint32_t)((id / X) % Y), z = (uint32_t)(id / ((uint64_t)X * Y));
    dvm[id] = (x + ox) | ((y + oy) << 10) | ((z + oz) << 20);
  };
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n16; i += stride) {
    const uint4 q = __ldg(reinterpret_cast<const uint4*>(pvm) + i);
    const uint32_t w[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
    for (int k = 0; k < 16; ++k)
      if ((int)(int8_t)(w[k >> 2] >> ((k & 3) * 8)) > thr) put(i * 16 + k);
  }
  for (uint64_t id = n16 * 16 + (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; id < n; id += stride)
    if ((int)pvm[id] > thr) put(id);
}

unsigned grid_for(uint64_t n, int threads) {
  const int sms = device_sms();
  return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((n + threads - 1) / threads, (uint64_t)sms * 16));
}

}  // namespace

int prob_threshold(float val) {  // ProbabilisticVoxel::floatToProbability, GV/voxel/ProbabilisticVoxel.h:40-45
  float tmp = std::max(std::min(1.0f, val), 0.0f);
  tmp = (tmp * (127.0f - (-127.0f))) + (-127.0f);
  return (int)(int8_t)tmp;
}

cudaError_t launch_pvm_insert(int8_t* d_vox, gvx_dims d, float side, const float* d_xyz, uint64_t n, uint32_t meaning,
                              uint32_t* d_outside, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  int mode = 1, delta = 0;
  if (meaning == 0) delta = -10;                         // eBVM_FREE: sensor model free
  else if (meaning == 1 || meaning == 2) delta = 72;     // eBVM_OCCUPIED, eBVM_COLLISION: sensor model occupied
  else if (meaning >= 4 && meaning <= 254) delta = (int)meaning - 129;  // eBVM_SWEPT_VOLUME range as probability
  else mode = 0;                                         // eBVM_UNKNOWN, eBVM_UNDEFINED
  pvm_insert_kernel<<<grid_for(n, 256), 256, 0, s>>>(reinterpret_cast<uint32_t*>(d_vox), d.x, d.y, d.z, side, d_xyz, n,
                                                     mode, delta, d_outside);
  return cudaGetLastError();
}

cudaError_t launch_merge_occupied(uint32_t* d_dvm, const int8_t* d_pvm, gvx_dims d, const uint32_t off[3], float threshold,
                                  cudaStream_t s) {
  const uint64_t n = num_voxels(d);
  merge_occupied_kernel<<<grid_for(n / 16 + 1, 256), 256, 0, s>>>(d_dvm, d_pvm, d.x, d.y, n, off[0], off[1], off[2],
                                                                   prob_threshold(threshold));
  return cudaGetLastError();
}

}  // namespace gvx
