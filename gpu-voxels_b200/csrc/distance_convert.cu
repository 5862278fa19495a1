// Consumers of an EDT'd DistanceVoxelMap: the free-space byte map, the
// flood-fill initialisation and the conversion of a distance band into a
// BitVectorVoxelList.
//   extract_distances: DistanceVoxelMap::extract_distances
//                      (GV/voxelmap/DistanceVoxelMap.hpp:676-688) with
//                      DistanceVoxel::extract_byte_distance (GV/voxel/DistanceVoxel.h:144-199)
//   init_floodfill:    DistanceVoxelMap::init_floodfill (DistanceVoxelMap.hpp:658-674) with
//                      DistanceVoxel::init_floodfill_distance (DistanceVoxel.h:201-215)
//   extract_given_distances: GV/helpers_highlevel/DistanceMapConverter.cu:156-196
//                      (transform_to_bitvoxel :103-154)
// The byte is recomputed from the map where needed instead of stored.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "gvx_internal.cuh"

namespace gvx {
namespace {

constexpr int kTile = 4096;  // voxels per compaction tile (16 per thread of a 256-thread block)

__device__ __forceinline__ int8_t free_space_byte(uint32_t v, int x, int y, int z, int X, int Y, int Z, int r) {
  if (x > X - r) return (int8_t)(X - x < 0 ? 0 : X - x);
  if (y > Y - r) return (int8_t)(Y - y < 0 ? 0 : Y - y);
  if (z > Z - r) return (int8_t)(Z - z < 0 ? 0 : Z - z);
  if (x < r) return (int8_t)(x < 0 ? 0 : x);
  if (y < r) return (int8_t)(y < 0 ? 0 : y);
  if (z < r) return (int8_t)(z < 0 ? 0 : z);
  const int ox = (int)dv_x(v), oy = (int)dv_y(v), oz = (int)dv_z(v);
  int32_t sq = kMaxObstacleDistance;  // DistanceVoxel::squaredObstacleDistance
  if (ox != (int)kUninit && oy != (int)kUninit && oz != (int)kUninit) {
    const int dx = x - ox, dy = y - oy, dz = z - oz;
    sq = dx * dx + dy * dy + dz * dz;
  }
  const int fs = (int)sqrtf((float)sq);
  return (int8_t)(fs > 127 ? 127 : fs);
}

__device__ __forceinline__ int8_t byte_at(const uint32_t* __restrict__ vox, uint64_t i, uint32_t X, uint32_t Y,
                                          uint32_t Z, int r) {
  const uint64_t layer = (uint64_t)X * Y;
  const int z = (int)(i / layer), y = (int)((i % layer) / X), x = (int)(i % X);
  return free_space_byte(__ldg(vox + i), x, y, z, (int)X, (int)Y, (int)Z, r);
}

__global__ void extract_distances_kernel(const uint32_t* __restrict__ vox, uint32_t X, uint32_t Y, uint32_t Z, int r,
                                         int8_t* __restrict__ out) {
  const uint64_t n = (uint64_t)X * Y * Z;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = byte_at(vox, i, X, Y, Z, r);
}

__global__ void init_floodfill_kernel(const int8_t* __restrict__ in, int16_t* __restrict__ out, uint64_t n, int r) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = (int16_t)((int)in[i] <= r ? kManhattanTooClose : kManhattanUninitialized);
}

// Matching voxels of one tile as a bit mask per thread: thread t tests the
// stripe of voxels 16t .. 16t + 15 of the tile, in id order.
__device__ __forceinline__ uint32_t tile_mask(const uint32_t* vox, uint64_t base, uint64_t n, uint32_t X, uint32_t Y,
                                              uint32_t Z, int mn, int mx) {
  uint32_t m = 0;
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    const uint64_t i = base + (uint64_t)threadIdx.x * 16 + k;
    if (i < n) {
      const int b = byte_at(vox, i, X, Y, Z, 0);
      if (b >= mn && b <= mx) m |= 1u << k;
    }
  }
  return m;
}

__global__ void __launch_bounds__(256) band_count_kernel(const uint32_t* __restrict__ vox, uint32_t X, uint32_t Y,
                                                         uint32_t Z, int mn, int mx, uint32_t* __restrict__ tile_count) {
  __shared__ uint32_t warp_sum[8];
  const uint64_t n = (uint64_t)X * Y * Z;
  const uint64_t base = (uint64_t)blockIdx.x * kTile;
  uint32_t c = __popc(tile_mask(vox, base, n, X, Y, Z, mn, mx));
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0) warp_sum[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t t = 0;
    for (int w = 0; w < 8; ++w) t += warp_sum[w];
    tile_count[blockIdx.x] = t;
  }
}

// Exclusive prefix over the tile counts in one block; total at [n_tiles].
__global__ void __launch_bounds__(1024) tile_scan_kernel(uint32_t* __restrict__ counts, uint32_t n_tiles) {
  __shared__ uint32_t part[1024];
  const uint32_t per = (n_tiles + 1023) / 1024;
  const uint32_t lo = threadIdx.x * per, hi = min(lo + per, n_tiles);
  uint32_t s = 0;
  for (uint32_t i = lo; i < hi; ++i) s += counts[i];
  part[threadIdx.x] = s;
  __syncthreads();
  for (int off = 1; off < 1024; off <<= 1) {  // inclusive scan of the 1024 partial sums
    const uint32_t v = threadIdx.x >= (unsigned)off ? part[threadIdx.x - off] : 0u;
    __syncthreads();
    part[threadIdx.x] += v;
    __syncthreads();
  }
  uint32_t run = threadIdx.x ? part[threadIdx.x - 1] : 0u;
  for (uint32_t i = lo; i < hi; ++i) {
    const uint32_t c = counts[i];
    counts[i] = run;
    run += c;
  }
  if (threadIdx.x == 1023) counts[n_tiles] = part[1023];
}

// Write the tile's matches in id order: thread t's stripe precedes thread t+1's.
__global__ void __launch_bounds__(256) band_write_kernel(const uint32_t* __restrict__ vox, uint32_t X, uint32_t Y,
                                                         uint32_t Z, int mn, int mx, const uint32_t* __restrict__ tile_off,
                                                         uint32_t* __restrict__ ids, uint8_t* __restrict__ out_vox) {
  __shared__ uint32_t warp_pre[8];
  const uint64_t n = (uint64_t)X * Y * Z;
  const uint64_t base = (uint64_t)blockIdx.x * kTile;
  const uint32_t m = tile_mask(vox, base, n, X, Y, Z, mn, mx);
  const uint32_t c = __popc(m);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t inc = c;  // inclusive warp scan
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t v = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += v;
  }
  if (lane == 31) warp_pre[warp] = inc;
  __syncthreads();
  uint32_t before = 0;
  for (int w = 0; w < warp; ++w) before += warp_pre[w];
  uint64_t k = (uint64_t)tile_off[blockIdx.x] + before + inc - c;
  for (uint32_t mm = m; mm; mm &= mm - 1, ++k) {
    const int j = __ffs(mm) - 1;
    const uint64_t i = base + (uint64_t)threadIdx.x * 16 + j;
    const int b = byte_at(vox, i, X, Y, Z, 0);
    ids[k] = (uint32_t)i;
    // transform_to_bitvoxel: eBVM_OCCUPIED, swept-volume bits 4 .. 4 + b - 1
    uint32_t w[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    w[0] = 1u << 1;
    unsigned fs = (uint16_t)b + 4u;
    if (fs > 255u) {
      w[7] |= 0x80000000u;
      fs = 255u;
    }
    for (unsigned s = 4; s < fs; ++s) w[s >> 5] |= 1u << (s & 31);
    uint4* dst = reinterpret_cast<uint4*>(out_vox + k * kBitVoxelBytes);
    dst[0] = make_uint4(w[0], w[1], w[2], w[3]);
    dst[1] = make_uint4(w[4], w[5], w[6], w[7]);
  }
}

unsigned grid_for(uint64_t n) {
  const int sms = device_sms();
  return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((n + 255) / 256, (uint64_t)sms * 16));
}

}  // namespace

cudaError_t launch_extract_distances(const uint32_t* d_vox, gvx_dims d, int robot_radius, int8_t* d_out, cudaStream_t s) {
  extract_distances_kernel<<<grid_for(num_voxels(d)), 256, 0, s>>>(d_vox, d.x, d.y, d.z, robot_radius, d_out);
  return cudaGetLastError();
}

cudaError_t launch_init_floodfill(const int8_t* d_in, int16_t* d_out, uint64_t n, int robot_radius, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  init_floodfill_kernel<<<grid_for(n), 256, 0, s>>>(d_in, d_out, n, robot_radius);
  return cudaGetLastError();
}

uint64_t band_tiles(gvx_dims d) { return (num_voxels(d) + kTile - 1) / kTile; }

cudaError_t launch_band_count(const uint32_t* d_vox, gvx_dims d, int mn, int mx, uint32_t* d_tiles, cudaStream_t s) {
  const uint64_t nt = band_tiles(d);
  band_count_kernel<<<(unsigned)nt, 256, 0, s>>>(d_vox, d.x, d.y, d.z, mn, mx, d_tiles);
  tile_scan_kernel<<<1, 1024, 0, s>>>(d_tiles, (uint32_t)nt);
  return cudaGetLastError();
}

cudaError_t launch_band_write(const uint32_t* d_vox, gvx_dims d, int mn, int mx, const uint32_t* d_tiles, uint32_t* d_ids,
                              uint8_t* d_lvox, cudaStream_t s) {
  band_write_kernel<<<(unsigned)band_tiles(d), 256, 0, s>>>(d_vox, d.x, d.y, d.z, mn, mx, d_tiles, d_ids, d_lvox);
  return cudaGetLastError();
}

}  // namespace gvx
