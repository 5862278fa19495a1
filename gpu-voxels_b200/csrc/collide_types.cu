// Typed collisions: which swept-volume / meaning bits collide, not only how
// many voxels.
//   map vs map:  BitVoxelMap::collideWithTypes(BitVectorVoxelMap*) (GV/voxelmap/BitVoxelMap.hpp:212-217)
//                -> kernelCollideVoxelMapsBitvector (GV/voxelmap/kernels/VoxelMapOperations.hpp:187-239)
//                with SVCollider at window 0 (GV/voxel/SVCollider.hpp:90-96,
//                bitMarginCollisionCheck GV/helpers/BitVector.h:415-470): the
//                types of voxel i are self & other on the swept-volume bits.
//   map vs prob: collideWithTypes(ProbVoxelMap*) (BitVoxelMap.hpp:219-224), SVCollider.hpp:98-108.
//   list vs map / prob / mask: BitVoxelList::collideWithTypes, collideWithTypeMask
//                (GV/voxellist/BitVoxelList.hpp:120-246) -> kernelCollideWithVoxelMap[BitMask]
//                (GV/voxellist/kernels/VoxelListOperations.hpp:204-260,282-325).
//   list vs list: collideWithTypes(BitVectorVoxelList*) (BitVoxelList.hpp:94-118).
// Thread per voxel / entry with two 16-byte loads; the types are OR-reduced
// per warp and merged with one atomicOr per word per warp, the count with
// one atomic per block.  Colliding voxels / entries get eBVM_COLLISION.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "gvx_internal.cuh"

namespace gvx {
namespace {

constexpr unsigned kAll = 0xffffffffu;

struct Bits8 {
  uint32_t w[8];
};

// A voxel the kernel only reads (the other map, the mask): read-only cache.
__device__ __forceinline__ Bits8 load_voxel(const uint32_t* v) {
  const uint4 a = __ldg(reinterpret_cast<const uint4*>(v));
  const uint4 b = __ldg(reinterpret_cast<const uint4*>(v) + 1);
  return Bits8{{a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w}};
}

// A voxel the kernel may mark afterwards (this map, the list): a plain load,
// since the read-only cache is only for data no thread writes during the kernel.
__device__ __forceinline__ Bits8 load_voxel_rw(const uint32_t* v) {
  const uint4 a = *reinterpret_cast<const uint4*>(v);
  const uint4 b = *(reinterpret_cast<const uint4*>(v) + 1);
  return Bits8{{a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w}};
}

__device__ __forceinline__ bool any_but_free(const Bits8& v) {  // !noneButEmpty
  return ((v.w[0] & ~1u) | v.w[1] | v.w[2] | v.w[3] | v.w[4] | v.w[5] | v.w[6] | v.w[7]) != 0u;
}

// Merge this thread's hit count and types into the outputs.
__device__ __forceinline__ void flush(unsigned hits, const Bits8& t, unsigned long long* count, uint32_t* types) {
  __shared__ unsigned long long s_sum;
  if (threadIdx.x == 0) s_sum = 0ull;
  __syncthreads();
  const unsigned h = __reduce_add_sync(kAll, hits);
  if (types != nullptr) {
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const uint32_t o = __reduce_or_sync(kAll, t.w[k]);
      if ((threadIdx.x & 31) == 0 && o) atomicOr(types + k, o);
    }
  }
  if ((threadIdx.x & 31) == 0 && h) atomicAdd(&s_sum, (unsigned long long)h);
  __syncthreads();
  if (threadIdx.x == 0 && s_sum) atomicAdd(count, s_sum);
}

__device__ __forceinline__ void mark_collision(uint32_t* v) { atomicOr(v, 1u << kEbvmCollision); }

// mode 0: other is a BitVoxel map (SV-bit intersection); 1: int8 occupancy >= thr
__global__ void __launch_bounds__(256) bvm_types_kernel(uint32_t* __restrict__ self, const void* __restrict__ other,
                                                        uint64_t n, int mode, int thr, unsigned long long* count,
                                                        uint32_t* types) {
  Bits8 acc{{0, 0, 0, 0, 0, 0, 0, 0}};
  unsigned hits = 0;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    uint32_t* sv = self + i * kBitVoxelWords;
    const Bits8 a = load_voxel_rw(sv);
    Bits8 t;
    bool hit;
    if (mode == 0) {
      const Bits8 b = load_voxel(reinterpret_cast<const uint32_t*>(other) + i * kBitVoxelWords);
      uint32_t any = 0;
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        t.w[k] = a.w[k] & (k == 0 ? (b.w[0] & ~0xFu) : b.w[k]);  // bits 0..3 are not swept-volume ids
        any |= t.w[k];
      }
      hit = any != 0u;
    } else {
      t = a;
      hit = (int)reinterpret_cast<const int8_t*>(other)[i] >= thr && any_but_free(a);
    }
    if (hit) {
      ++hits;
#pragma unroll
      for (int k = 0; k < 8; ++k) acc.w[k] |= t.w[k];
      mark_collision(sv);
    }
  }
  flush(hits, acc, count, types);
}

// kind 0: BitVoxel map, 1: int8 occupancy compared (as float) with fthr
__global__ void __launch_bounds__(256) list_types_kernel(const uint32_t* __restrict__ ids, uint32_t* __restrict__ lvox,
                                                         uint64_t n, const void* __restrict__ map, uint64_t map_n,
                                                         int kind, float fthr, int64_t off, const uint32_t* mask,
                                                         unsigned long long* count, uint32_t* types) {
  Bits8 acc{{0, 0, 0, 0, 0, 0, 0, 0}};
  Bits8 mk{{0, 0, 0, 0, 0, 0, 0, 0}};
  if (mask != nullptr) mk = load_voxel(mask);
  unsigned hits = 0;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const int64_t j = (int64_t)__ldg(ids + i) + off;
    if (j < 0 || j >= (int64_t)map_n) continue;
    const bool occ = kind == 0 ? any_but_free(load_voxel(reinterpret_cast<const uint32_t*>(map) + (uint64_t)j * kBitVoxelWords))
                               : ((float)reinterpret_cast<const int8_t*>(map)[j] >= fthr);
    if (!occ) continue;
    uint32_t* lv = lvox + i * kBitVoxelWords;
    const Bits8 a = load_voxel_rw(lv);
    if (mask != nullptr) {
      uint32_t meet = 0;
#pragma unroll
      for (int k = 0; k < 8; ++k) meet |= a.w[k] & mk.w[k];
      if (!meet) continue;
    }
    ++hits;
#pragma unroll
    for (int k = 0; k < 8; ++k) acc.w[k] |= a.w[k];
    mark_collision(lv);
  }
  flush(hits, acc, count, types);
}

// ids of list a present in sorted list b (binary search): types |= a | b
__global__ void __launch_bounds__(256) list_list_types_kernel(const uint32_t* __restrict__ ids_a,
                                                              const uint32_t* __restrict__ vox_a, uint64_t na,
                                                              const uint32_t* __restrict__ ids_b,
                                                              const uint32_t* __restrict__ vox_b, uint64_t nb,
                                                              unsigned long long* count, uint32_t* types) {
  Bits8 acc{{0, 0, 0, 0, 0, 0, 0, 0}};
  unsigned hits = 0;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < na; i += stride) {
    const uint32_t id = __ldg(ids_a + i);
    uint64_t lo = 0, hi = nb;
    while (lo < hi) {
      const uint64_t mid = (lo + hi) >> 1;
      if (__ldg(ids_b + mid) < id) lo = mid + 1; else hi = mid;
    }
    if (lo < nb && __ldg(ids_b + lo) == id) {
      ++hits;
      const Bits8 a = load_voxel(vox_a + i * kBitVoxelWords), b = load_voxel(vox_b + lo * kBitVoxelWords);
#pragma unroll
      for (int k = 0; k < 8; ++k) acc.w[k] |= a.w[k] | b.w[k];
    }
  }
  flush(hits, acc, count, types);
}

unsigned grid_for(uint64_t n) {
  const int sms = device_sms();
  return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((n + 255) / 256, (uint64_t)sms * 8));
}

cudaError_t zero_outputs(unsigned long long* d_count, uint32_t* d_types, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(d_count, 0, sizeof(unsigned long long), s);
  if (e == cudaSuccess && d_types != nullptr) e = cudaMemsetAsync(d_types, 0, kBitVoxelBytes, s);
  return e;
}

}  // namespace

int sv_threshold(float val) {  // SVCollider::floatToProbability (GV/voxel/SVCollider.hpp:144-148), no clamping
  return (int)(int8_t)((val * (127.0f - (-127.0f))) + (-127.0f));
}

cudaError_t launch_bvm_collide_types(uint8_t* d_self, const void* d_other, uint64_t n, int mode, float threshold,
                                     unsigned long long* d_count, uint32_t* d_types, cudaStream_t s) {
  cudaError_t e = zero_outputs(d_count, d_types, s);
  if (e != cudaSuccess || n == 0) return e;
  bvm_types_kernel<<<grid_for(n), 256, 0, s>>>(reinterpret_cast<uint32_t*>(d_self), d_other, n, mode,
                                               sv_threshold(threshold), d_count, d_types);
  return cudaGetLastError();
}

cudaError_t launch_list_collide_types(const uint32_t* d_ids, uint8_t* d_lvox, uint64_t n, const void* d_map,
                                      uint64_t map_n, int kind, float threshold, int64_t off, const uint8_t* d_mask,
                                      unsigned long long* d_count, uint32_t* d_types, cudaStream_t s) {
  cudaError_t e = zero_outputs(d_count, d_types, s);
  if (e != cudaSuccess || n == 0) return e;
  list_types_kernel<<<grid_for(n), 256, 0, s>>>(d_ids, reinterpret_cast<uint32_t*>(d_lvox), n, d_map, map_n, kind,
                                                threshold, off, reinterpret_cast<const uint32_t*>(d_mask), d_count,
                                                d_types);
  return cudaGetLastError();
}

cudaError_t launch_list_list_types(const uint32_t* d_ids_a, const uint8_t* d_vox_a, uint64_t na, const uint32_t* d_ids_b,
                                   const uint8_t* d_vox_b, uint64_t nb, unsigned long long* d_count, uint32_t* d_types,
                                   cudaStream_t s) {
  cudaError_t e = zero_outputs(d_count, d_types, s);
  if (e != cudaSuccess || na == 0 || nb == 0) return e;
  list_list_types_kernel<<<grid_for(na), 256, 0, s>>>(d_ids_a, reinterpret_cast<const uint32_t*>(d_vox_a), na, d_ids_b,
                                                      reinterpret_cast<const uint32_t*>(d_vox_b), nb, d_count, d_types);
  return cudaGetLastError();
}

}  // namespace gvx
