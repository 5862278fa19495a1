// BitVoxelMap::insertMetaPointCloudWithSelfCollisionCheck
// (GV/voxelmap/BitVoxelMap.hpp:227-341; per sub-cloud kernel
// kernelInsertMetaPointCloudSelfCollCheck, GV/voxelmap/kernels/VoxelMapOperations.hpp:581-631).
//
// Sub-clouds (robot links) go in order.  For sub-cloud k every in-map point
// first checks its voxel as the earlier sub-clouds (and whatever the map held
// before) left it: masked = voxel & mask[k]; if masked has a bit other than
// bit 0 (eBVM_FREE), masked and meaning[k] join the colliding meanings and the
// point is flagged.  Then every in-map point sets meaning[k] in its voxel and
// a flagged point also eBVM_COLLISION.  The reference does check and insert in
// one kernel per sub-cloud; with its default masks (the sub-cloud's own
// meaning and eBVM_COLLISION cleared) the outcome is the same, and the split
// keeps it independent of thread timing for any mask.  The colliding meanings
// are gathered with atomics (the reference ORs them without, so two
// simultaneous hits can drop bits).
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "gvx_internal.cuh"

namespace gvx {
namespace {

struct Mask8 {
  uint32_t w[kBitVoxelWords];
};

__device__ __forceinline__ bool voxel_of(const float* __restrict__ xyz, uint64_t i, float side, uint32_t X, uint32_t Y,
                                         uint32_t Z, uint64_t& id) {
  const uint32_t x = coord_to_voxel(__ldg(xyz + 3 * i), side), y = coord_to_voxel(__ldg(xyz + 3 * i + 1), side),
                 z = coord_to_voxel(__ldg(xyz + 3 * i + 2), side);
  id = (uint64_t)z * X * Y + (uint64_t)y * X + x;
  return x < X && y < Y && z < Z;
}

// Points [begin, end) of one sub-cloud against the map: flags[i - begin] = hit.
__global__ void meta_check_kernel(const uint32_t* __restrict__ map, uint32_t X, uint32_t Y, uint32_t Z, float side,
                                  const float* __restrict__ xyz, uint64_t begin, uint64_t end, Mask8 mask,
                                  uint32_t meaning, uint8_t* __restrict__ flags, uint32_t* __restrict__ colliding,
                                  uint32_t* __restrict__ outside) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  bool out = false;
  for (uint64_t i = begin + (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < end; i += stride) {
    uint64_t id;
    uint8_t hit = 0;
    if (voxel_of(xyz, i, side, X, Y, Z, id)) {
      const uint4* v = reinterpret_cast<const uint4*>(map + id * kBitVoxelWords);
      const uint4 a = v[0], b = v[1];
      const uint32_t m[kBitVoxelWords] = {a.x & mask.w[0], a.y & mask.w[1], a.z & mask.w[2], a.w & mask.w[3],
                                          b.x & mask.w[4], b.y & mask.w[5], b.z & mask.w[6], b.w & mask.w[7]};
      // BitVector::noneButEmpty (GV/helpers/BitVector.h:184-198): bit 0 (eBVM_FREE) does not count
      if ((m[0] & ~1u) | m[1] | m[2] | m[3] | m[4] | m[5] | m[6] | m[7]) {
        hit = 1;
#pragma unroll
        for (int w = 0; w < kBitVoxelWords; ++w)
          if (m[w]) atomicOr(colliding + w, m[w]);
        atomicOr(colliding + (meaning >> 5), 1u << (meaning & 31));
      }
    } else {
      out = true;
    }
    flags[i - begin] = hit;
  }
  if (outside != nullptr && __any_sync(0xffffffffu, out) && (threadIdx.x & 31) == 0) *outside = 1u;
}

// Then the sub-cloud's meaning, and eBVM_COLLISION where the check hit.
__global__ void meta_insert_kernel(uint32_t* __restrict__ map, uint32_t X, uint32_t Y, uint32_t Z, float side,
                                   const float* __restrict__ xyz, uint64_t begin, uint64_t end, uint32_t meaning,
                                   const uint8_t* __restrict__ flags) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = begin + (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < end; i += stride) {
    uint64_t id;
    if (voxel_of(xyz, i, side, X, Y, Z, id)) {
      uint32_t* v = map + id * kBitVoxelWords;
      atomicOr(v + (meaning >> 5), 1u << (meaning & 31));
      if (flags[i - begin]) atomicOr(v + (kEbvmCollision >> 5), 1u << (kEbvmCollision & 31));
    }
  }
}

unsigned grid_for(uint64_t n) {
  const int sms = device_sms();
  const uint64_t want = (n + 255) / 256;
  return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(want, (uint64_t)std::max(sms, 1) * 16));
}

}  // namespace

cudaError_t launch_meta_insert_self_coll(uint8_t* d_vox, gvx_dims d, float side, const float* d_xyz,
                                         const uint64_t* offsets, uint32_t n_clouds, const uint8_t* meanings,
                                         const uint32_t* masks, uint8_t* d_flags, uint32_t* d_colliding,
                                         uint32_t* d_outside, cudaStream_t s) {
  uint32_t* map = reinterpret_cast<uint32_t*>(d_vox);
  cudaError_t e = cudaMemsetAsync(d_colliding, 0, kBitVoxelWords * sizeof(uint32_t), s);
  for (uint32_t k = 0; k < n_clouds && e == cudaSuccess; ++k) {
    const uint64_t begin = offsets[k], end = offsets[k + 1];
    if (end <= begin) continue;
    Mask8 mask;
    for (int w = 0; w < kBitVoxelWords; ++w) mask.w[w] = masks[k * kBitVoxelWords + w];
    const unsigned blocks = grid_for(end - begin);
    meta_check_kernel<<<blocks, 256, 0, s>>>(map, d.x, d.y, d.z, side, d_xyz, begin, end, mask, meanings[k], d_flags,
                                             d_colliding, d_outside);
    if ((e = cudaGetLastError()) != cudaSuccess) break;
    meta_insert_kernel<<<blocks, 256, 0, s>>>(map, d.x, d.y, d.z, side, d_xyz, begin, end, meanings[k], d_flags);
    e = cudaGetLastError();
  }
  return e;
}

}  // namespace gvx
