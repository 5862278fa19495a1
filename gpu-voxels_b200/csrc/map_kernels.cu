// Map fill and point-cloud voxelisation kernels.
#include <cuda_runtime.h>

#include <atomic>
#include <stdint.h>

#include <algorithm>

#include "gvx_internal.cuh"

namespace gvx {
namespace {


// clearMap for DistanceVoxel (GV/voxelmap/TemplateVoxelMap.hpp:244-271):
// 16-byte stores of the uninitialised value; the map base is 256-B aligned.
__global__ void dvm_fill_kernel(uint4* __restrict__ v4, uint64_t n4, uint32_t* __restrict__ tail, uint32_t ntail) {
  const uint4 u = make_uint4(kDvUninit, kDvUninit, kDvUninit, kDvUninit);
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += stride) __stcs(v4 + i, u);
  if (blockIdx.x == 0 && threadIdx.x < ntail) tail[threadIdx.x] = kDvUninit;
}

// kernelInsertGlobalPointCloud<DistanceVoxel> (GV/voxelmap/kernels/VoxelMapOperations.hpp:266-300):
// every point in a voxel writes the voxel's own coordinate, so the scatter
// needs no atomics (DistanceVoxel::insert, GV/voxel/DistanceVoxel.hpp:125-138).
__global__ void dvm_insert_kernel(uint32_t* __restrict__ map, uint32_t X, uint32_t Y, uint32_t Z, float side,
                                  const float* __restrict__ xyz, uint64_t n, uint32_t* __restrict__ outside) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  bool out = false;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const float px = __ldg(xyz + 3 * i), py = __ldg(xyz + 3 * i + 1), pz = __ldg(xyz + 3 * i + 2);
    const uint32_t x = coord_to_voxel(px, side), y = coord_to_voxel(py, side), z = coord_to_voxel(pz, side);
    if (x < X && y < Y && z < Z) {
      map[z * X * Y + y * X + x] = dv_pack(x, y, z);
    } else {
      out = true;
    }
  }
  if (outside != nullptr && __any_sync(0xffffffffu, out) && (threadIdx.x & 31) == 0) *outside = 1u;
}

// kernelInsertGlobalPointCloud<BitVoxel> (VoxelMapOperations.hpp:241-264).  The
// reference ORs the byte without an atomic; a 32-bit atomicOr gives the same
// result and stays correct when different meanings hit one voxel at once.
__global__ void bvm_insert_kernel(uint32_t* __restrict__ map, uint32_t X, uint32_t Y, uint32_t Z, float side,
                                  const float* __restrict__ xyz, uint64_t n, uint32_t meaning,
                                  uint32_t* __restrict__ outside) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  const uint32_t word = meaning >> 5, bit = 1u << (meaning & 31);
  bool out = false;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const float px = __ldg(xyz + 3 * i), py = __ldg(xyz + 3 * i + 1), pz = __ldg(xyz + 3 * i + 2);
    const uint32_t x = coord_to_voxel(px, side), y = coord_to_voxel(py, side), z = coord_to_voxel(pz, side);
    if (x < X && y < Y && z < Z) {
      const uint64_t id = (uint64_t)z * X * Y + (uint64_t)y * X + x;
      atomicOr(map + id * kBitVoxelWords + word, bit);
    } else {
      out = true;
    }
  }
  if (outside != nullptr && __any_sync(0xffffffffu, out) && (threadIdx.x & 31) == 0) *outside = 1u;
}

// kernelClearVoxelMap(BitVoxel*, size, BitVector bits) (VoxelMapOperations.hpp:57-71):
// clears `bits` in every voxel (clearBit / clearBitVoxelMeaning use one bit).
__global__ void bvm_clear_bits_kernel(uint4* __restrict__ vox, uint64_t n, uint4 lo, uint4 hi) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    uint4 a = vox[2 * i], b = vox[2 * i + 1];
    a.x &= ~lo.x; a.y &= ~lo.y; a.z &= ~lo.z; a.w &= ~lo.w;
    b.x &= ~hi.x; b.y &= ~hi.y; b.z &= ~hi.z; b.w &= ~hi.w;
    vox[2 * i] = a;
    vox[2 * i + 1] = b;
  }
}

// kernelShiftBitVector / performLeftShift (VoxelMapOperations.hpp:813-820,
// GV/helpers/BitVector.h:355-402): every voxel's 256 bits move down by
// `shift` (<= 56) bit positions -- swept-volume meaning k becomes k - shift --
// and the four meanings below eBVM_SWEPT_VOLUME_START are cleared.
__global__ void bvm_shift_kernel(uint32_t* __restrict__ vox, uint64_t n, uint32_t shift) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  const uint32_t ws = shift >> 5, bs = shift & 31;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    uint32_t* v = vox + i * kBitVoxelWords;
    uint32_t in[kBitVoxelWords + 2];
#pragma unroll
    for (int w = 0; w < (int)kBitVoxelWords; ++w) in[w] = v[w];
    in[kBitVoxelWords] = in[kBitVoxelWords + 1] = 0u;
    uint32_t out[kBitVoxelWords];
#pragma unroll
    for (int w = 0; w < (int)kBitVoxelWords; ++w) {
      const uint32_t lo = w + ws < kBitVoxelWords + 2 ? in[w + ws] : 0u;
      const uint32_t hi = w + ws + 1 < kBitVoxelWords + 2 ? in[w + ws + 1] : 0u;
      out[w] = (uint32_t)((((uint64_t)hi << 32) | lo) >> bs);
    }
    out[0] &= ~0xFu;
#pragma unroll
    for (int w = 0; w < (int)kBitVoxelWords; ++w) v[w] = out[w];
  }
}

unsigned grid_for(uint64_t n, int threads) {
  const uint64_t want = (n + threads - 1) / threads;
  const uint64_t cap = (uint64_t)device_sms() * 16;
  return (unsigned)std::max<uint64_t>(1, std::min(want, cap));
}

}  // namespace

namespace {
constexpr int kSmsDevices = 64;
std::atomic<int> g_sms_of[kSmsDevices];
}  // namespace

int device_sms() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 1;
  if (dev >= 0 && dev < kSmsDevices) {
    const int cached = g_sms_of[dev].load(std::memory_order_relaxed);
    if (cached > 0) return cached;
  }
  int sms = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms < 1) return 1;
  if (dev >= 0 && dev < kSmsDevices) g_sms_of[dev].store(sms, std::memory_order_relaxed);
  return sms;
}

cudaError_t launch_dvm_clear(uint32_t* d_vox, uint64_t n, cudaStream_t s) {
  const uint64_t n4 = n / 4;
  const uint32_t ntail = (uint32_t)(n - n4 * 4);
  dvm_fill_kernel<<<grid_for(std::max<uint64_t>(n4, 1), 256), 256, 0, s>>>(reinterpret_cast<uint4*>(d_vox), n4,
                                                                          d_vox + n4 * 4, ntail);
  return cudaGetLastError();
}

cudaError_t launch_dvm_insert(uint32_t* d_vox, gvx_dims d, float side, const float* d_xyz, uint64_t n,
                              uint32_t* d_outside, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  dvm_insert_kernel<<<grid_for(n, 256), 256, 0, s>>>(d_vox, d.x, d.y, d.z, side, d_xyz, n, d_outside);
  return cudaGetLastError();
}

cudaError_t launch_bvm_insert(uint8_t* d_vox, gvx_dims d, float side, const float* d_xyz, uint64_t n, uint32_t meaning,
                              uint32_t* d_outside, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  bvm_insert_kernel<<<grid_for(n, 256), 256, 0, s>>>(reinterpret_cast<uint32_t*>(d_vox), d.x, d.y, d.z, side, d_xyz, n,
                                                     meaning, d_outside);
  return cudaGetLastError();
}

cudaError_t launch_bvm_clear_bits(uint8_t* d_vox, gvx_dims d, const uint32_t bits[8], cudaStream_t s) {
  const uint64_t n = (uint64_t)d.x * d.y * d.z;
  bvm_clear_bits_kernel<<<grid_for(n, 256), 256, 0, s>>>(reinterpret_cast<uint4*>(d_vox), n,
                                                         make_uint4(bits[0], bits[1], bits[2], bits[3]),
                                                         make_uint4(bits[4], bits[5], bits[6], bits[7]));
  return cudaGetLastError();
}

cudaError_t launch_bvm_shift(uint8_t* d_vox, gvx_dims d, uint32_t shift, cudaStream_t s) {
  const uint64_t n = (uint64_t)d.x * d.y * d.z;
  bvm_shift_kernel<<<grid_for(n, 256), 256, 0, s>>>(reinterpret_cast<uint32_t*>(d_vox), n, shift);
  return cudaGetLastError();
}

}  // namespace gvx
