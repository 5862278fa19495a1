// Exact 3D Euclidean distance transform on a DistanceVoxel map, in place.
//
// Result: bit-identical to DistanceVoxelMap::parallelBanding3D(1,1,1)
// (GV/voxelmap/DistanceVoxelMap.hpp:284-645) -- every voxel holds the same
// nearest site, including the reference's tie-breaking -- for any dims in
// [1,1023]^3 (the reference itself needs x == y and x % 64 == 0).
//
// Three sweeps, one kernel each:
//   pass Z : phase 1 (kernelPBAphase1FloodZ, VoxelMapOperationsPBA.hpp:63-124)
//            per (x,y) column.
//   pass Y : phase 2 + 3 (kernelPBAphase2ProximateBackpointers :289-379,
//            kernelPBAphase3Distances :604-703) per (x,z) column along y.
//   pass X : the same sweep per (y,z) row along x.  The reference transposes
//            the map (kernelPBA3DTransposeXY :825-888) and sweeps along y
//            again; sweeping x directly in the original frame is the same
//            computation with the roles of the site's x and y fields swapped.
//
// Passes Y and X: one thread per column, a warp owns 32 adjacent columns.
// The columns stream through shared memory in 32-row chunks (cp.async,
// double buffered; pass X transposes each 32x32 chunk on the way in), the
// proximate-site stack of phases 2/3 is the reference's positional stack,
// kept in a per-map scratch buffer laid out [slice][block][row][lane] so the
// lanes of a warp push and pop the same row with one 128-byte access, and
// phase 3 writes each row of the warp's 32 columns with one coalesced store
// (pass X through a 32x33 staging tile).  The sweep is a chain of dependent
// steps per column, so the design goal is many columns in flight per SM.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "gvx_internal.cuh"

namespace gvx {
namespace {

constexpr int kChunk = 32;        // rows staged per step
constexpr int kSweepWarps = 8;    // warps per CTA in passes Y and X
constexpr int kTileWords = 32 * 33;

__device__ __forceinline__ void cp_async4(uint32_t* smem_dst, const uint32_t* gmem_src) {
  unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async16(uint32_t* smem_dst, const uint32_t* gmem_src) {
  unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// devicePBAintersection3DY (VoxelMapOperationsPBA.hpp:265-276) in a column
// frame: sites (a, row, c), column at (a0, c0).  Halving is exact, so the
// reference's "/ 2.0f" is a multiply by 0.5; the products and sums are exact
// for coordinates below 1024, so only the IEEE divide and the final add
// round.  The _rn intrinsics forbid any contraction.
__device__ __forceinline__ float pba_isect(int a1, int r1, int c1, int a2, int r2, int c2, int a0, int c0) {
  const float aM = __fmul_rn((float)(a1 + a2), 0.5f);
  const float rM = __fmul_rn((float)(r1 + r2), 0.5f);
  const float cM = __fmul_rn((float)(c1 + c2), 0.5f);
  const float na = (float)(a2 - a1);
  const float nr = (float)(r2 - r1);
  const float nc = (float)(c2 - c1);
  const float num = __fadd_rn(__fmul_rn(na, __fsub_rn(aM, (float)a0)), __fmul_rn(nc, __fsub_rn(cM, (float)c0)));
  return __fadd_rn(rM, __fdiv_rn(num, nr));
}

// Stack entry: a | backptr<<10 | c<<20, the reference's packing.
struct Site {
  uint32_t a, b, c;
};
__device__ __forceinline__ Site unpack(uint32_t e) { return Site{e & 0x3ffu, (e >> 10) & 0x3ffu, e >> 20}; }

// ---------------------------------------------------------------------------
// pass Z: phase 1 per (x, y) column, m1 = 1; the whole column in shared memory.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) edt_pass_z(uint32_t* __restrict__ map, int X, int Y, int Z, int warps_per_cta) {
  extern __shared__ __align__(16) uint32_t smem[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nxb = (X + 31) >> 5;
  const long long item = (long long)blockIdx.x * warps_per_cta + warp;
  if (item >= (long long)nxb * Y) return;
  const int xb = (int)(item % nxb), y = (int)(item / nxb);
  const int x0 = xb * 32, valid_cols = min(32, X - x0);
  const uint64_t layer = (uint64_t)X * Y;
  uint32_t* tile = smem + (size_t)warp * Z * 32;
  const uint32_t* src = map + (uint64_t)y * X + x0;
  if (valid_cols == 32 && (X & 3) == 0) {
    const int part = lane & 7;
    for (int r = lane >> 3; r < Z; r += 4) cp_async16(tile + r * 32 + part * 4, src + (uint64_t)r * layer + part * 4);
  } else if (lane < valid_cols) {
    for (int r = 0; r < Z; ++r) cp_async4(tile + r * 32 + lane, src + (uint64_t)r * layer + lane);
  } else {
    for (int r = 0; r < Z; ++r) tile[r * 32 + lane] = kDvUninit;
  }
  cp_async_wait_all();
  __syncwarp();

  // flood forward (in shared memory)
  uint32_t obstacle = kDvUninit;
#pragma unroll 8
  for (int z = 0; z < Z; ++z) {
    const uint32_t cur = tile[z * 32 + lane];
    if ((cur >> 20) != kUninit) obstacle = cur;
    tile[z * 32 + lane] = obstacle;
  }
  // flood backward; ties keep the lower z (<=, VoxelMapOperationsPBA.hpp:118)
  obstacle = kDvUninit;
  uint32_t* dst = map + (uint64_t)y * X + x0 + lane;
  const bool store = lane < valid_cols;
#pragma unroll 8
  for (int z = Z - 1; z >= 0; --z) {
    const int dist_prev = abs((int)(obstacle >> 20) - z);
    const uint32_t next = tile[z * 32 + lane];
    const int dist_next = abs(z - (int)(next >> 20));
    if (dist_next <= dist_prev) obstacle = next;
    if (store) dst[(uint64_t)z * layer] = obstacle;
  }
}

// ---------------------------------------------------------------------------
// passes Y and X
// ---------------------------------------------------------------------------

// Geometry of one warp's work item.
struct Sweep {
  int L;             // column length (rows)
  int a0_base;       // column coordinate of lane 0 (x0 for pass Y, y0 for pass X)
  int c0;            // slice (z)
  int valid;         // valid lanes
  uint32_t* slice;   // map + z * layer
  int X;             // map row length
};

// Issue the cp.async copies of chunk `c` into `tile`.
template <bool kXPass>
__device__ __forceinline__ void stage_chunk(uint32_t* tile, const Sweep& s, int c, bool vec16) {
  const int lane = threadIdx.x & 31;
  const int r0 = c * kChunk;
  const int rows = min(kChunk, s.L - r0);
  if (!kXPass) {
    // rows r0.. of columns a0_base..a0_base+31: tile[r*32 + lane]
    const uint32_t* src = s.slice + (uint64_t)r0 * s.X + s.a0_base;
    if (vec16) {
      const int part = lane & 7;
      for (int r = lane >> 3; r < rows; r += 4) cp_async16(tile + r * 32 + part * 4, src + (uint64_t)r * s.X + part * 4);
    } else if (lane < s.valid) {
      for (int r = 0; r < rows; ++r) cp_async4(tile + r * 32 + lane, src + (uint64_t)r * s.X + lane);
    } else {
      for (int r = 0; r < rows; ++r) tile[r * 32 + lane] = kDvUninit;
    }
  } else {
    // x positions r0+lane of rows a0_base+t, transposed: tile[(x - r0) * 33 + t]
    const uint32_t* src = s.slice + (uint64_t)s.a0_base * s.X + r0 + lane;
    const bool in_row = lane < rows;
    for (int t = 0; t < 32; ++t) {
      if (!in_row) continue;
      if (t < s.valid) cp_async4(tile + lane * 33 + t, src + (uint64_t)t * s.X);
      else tile[lane * 33 + t] = kDvUninit;
    }
  }
}

template <bool kXPass>
__device__ __forceinline__ uint32_t tile_at(const uint32_t* tile, int r) {
  const int lane = threadIdx.x & 31;
  return kXPass ? tile[r * 33 + lane] : tile[r * 32 + lane];
}

template <bool kXPass>
__global__ void __launch_bounds__(kSweepWarps * 32, 3) edt_sweep(uint32_t* __restrict__ map, uint32_t* __restrict__ scratch,
                                                                 int X, int Y, int Z) {
  extern __shared__ __align__(16) uint32_t s_tiles[];  // [kSweepWarps][2][kTileWords]
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int cols = kXPass ? Y : X;  // columns per slice
  const int L = kXPass ? X : Y;
  const int nblk = (cols + 31) >> 5;
  const long long item = (long long)blockIdx.x * kSweepWarps + warp;
  if (item >= (long long)nblk * Z) return;
  const int blk = (int)(item % nblk), z = (int)(item / nblk);
  Sweep s;
  s.L = L;
  s.a0_base = blk * 32;
  s.c0 = z;
  s.valid = min(32, cols - s.a0_base);
  s.slice = map + (uint64_t)z * X * Y;
  s.X = X;
  const bool vec16 = !kXPass && s.valid == 32 && (X & 3) == 0;
  uint32_t* tiles[2] = {s_tiles + (2 * warp) * kTileWords, s_tiles + (2 * warp + 1) * kTileWords};
  uint32_t* stk = scratch + ((uint64_t)item * L) * 32 + lane;  // entry of row p: stk[p * 32]
  const int a0 = s.a0_base + lane;
  const int c0 = z;
  const int nchunks = (L + kChunk - 1) / kChunk;

  // ---- phase 2: proximate sites, positional stack with back-pointers ----
  stage_chunk<kXPass>(tiles[0], s, 0, vec16);
  cp_async_commit();
  if (nchunks > 1) stage_chunk<kXPass>(tiles[1], s, 1, vec16);
  cp_async_commit();

  int last_y = (int)kUninit;  // row of the stack top, UNINIT when empty
  Site top{kUninit, kUninit, kUninit}, second{kUninit, kUninit, kUninit};
  float i_top = 0.0f;  // intersection of (second, top); valid when top.b != UNINIT
  uint32_t cur_a = kUninit;
  for (int c = 0; c < nchunks; ++c) {
    cp_async_wait1();
    __syncwarp();
    const uint32_t* tile = tiles[c & 1];
    const int r0 = c * kChunk;
    const int rows = min(kChunk, L - r0);
    for (int r = 0; r < rows; ++r) {
      const int ty = r0 + r;
      const uint32_t v = tile_at<kXPass>(tile, r);
      cur_a = kXPass ? ((v >> 10) & 0x3ffu) : (v & 0x3ffu);
      if (cur_a != kUninit) {
        const uint32_t cur_c = v >> 20;
        float i2 = 0.0f;
        bool have_i2 = false;
        while (top.b != kUninit) {
          i2 = pba_isect((int)top.a, last_y, (int)top.c, (int)cur_a, ty, (int)cur_c, a0, c0);
          have_i2 = true;
          if (i_top < i2) break;
          last_y = (int)top.b;  // pop
          top = second;
          have_i2 = false;
          if (top.b != kUninit) {
            second = unpack(stk[(int)top.b * 32]);
            i_top = pba_isect((int)second.a, (int)top.b, (int)second.c, (int)top.a, last_y, (int)top.c, a0, c0);
          }
        }
        if (last_y != (int)kUninit)
          i_top = have_i2 ? i2 : pba_isect((int)top.a, last_y, (int)top.c, (int)cur_a, ty, (int)cur_c, a0, c0);
        second = top;
        top = Site{cur_a, (uint32_t)last_y, cur_c};
        last_y = ty;
        stk[ty * 32] = dv_pack(top.a, top.b, top.c);
      }
    }
    __syncwarp();
    if (c + 2 < nchunks) stage_chunk<kXPass>(tiles[c & 1], s, c + 2, vec16);
    cp_async_commit();
  }
  cp_async_wait_all();
  if (cur_a == kUninit) stk[(L - 1) * 32] = dv_pack(kUninit, (uint32_t)last_y, kUninit);  // tail pointer

  // ---- phase 3: walk rows downward, popping sites that fall behind ----
  float inter = 0.0f;
  last_y = L - 1;
  top = unpack(stk[last_y * 32]);
  if (top.a == kUninit) {
    last_y = (int)top.b;
    if (last_y != (int)kUninit) top = unpack(stk[last_y * 32]);
  }
  if (top.b != kUninit) {
    second = unpack(stk[(int)top.b * 32]);
    inter = pba_isect((int)second.a, (int)top.b, (int)second.c, (int)top.a, last_y, (int)top.c, a0, c0);
  }
  uint32_t* stage = tiles[0];
  for (int ty = L - 1; ty >= 0; --ty) {
    while (top.b != kUninit) {
      if ((float)ty > inter) break;
      last_y = (int)top.b;
      top = second;
      if (top.b != kUninit) {
        second = unpack(stk[(int)top.b * 32]);
        inter = pba_isect((int)second.a, (int)top.b, (int)second.c, (int)top.a, last_y, (int)top.c, a0, c0);
      }
    }
    if (!kXPass) {
      if (lane < s.valid) s.slice[(uint64_t)ty * X + s.a0_base + lane] = dv_pack(top.a, (uint32_t)last_y, top.c);
    } else {
      // original frame: x-field = row of the site, y-field = a
      stage[(ty & 31) * 33 + lane] = dv_pack((uint32_t)last_y, top.a, top.c);
      if ((ty & 31) == 0) {
        __syncwarp();
        if (ty + lane < X) {
          for (int r = 0; r < s.valid; ++r) s.slice[(uint64_t)(s.a0_base + r) * X + ty + lane] = stage[lane * 33 + r];
        }
        __syncwarp();
      }
    }
  }
}

int g_smem_optin = -1;

int max_smem_optin() {
  if (g_smem_optin < 0) {
    int dev = 0, v = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    g_smem_optin = v;
  }
  return g_smem_optin;
}

cudaError_t launch_pass_z(uint32_t* map, gvx_dims d, cudaStream_t s) {
  const size_t per_warp = (size_t)d.z * 32 * 4;
  int w = (int)std::max<size_t>(1, std::min<size_t>(8, 98304 / per_warp));
  const size_t smem = per_warp * w;
  if ((int)smem > max_smem_optin()) return cudaErrorInvalidConfiguration;
  cudaError_t e = cudaFuncSetAttribute(edt_pass_z, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(edt_pass_z, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
  if (e != cudaSuccess) return e;
  const long long items = (long long)((d.x + 31) / 32) * d.y;
  edt_pass_z<<<(unsigned)((items + w - 1) / w), 32 * w, smem, s>>>(map, (int)d.x, (int)d.y, (int)d.z, w);
  return cudaGetLastError();
}

template <bool kXPass>
cudaError_t launch_sweep(uint32_t* map, uint32_t* scratch, gvx_dims d, cudaStream_t s) {
  const long long cols = kXPass ? d.y : d.x;
  const long long items = ((cols + 31) / 32) * d.z;
  const int smem = kSweepWarps * 2 * kTileWords * 4;
  cudaError_t e = cudaFuncSetAttribute(edt_sweep<kXPass>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(edt_sweep<kXPass>, cudaFuncAttributePreferredSharedMemoryCarveout,
                             cudaSharedmemCarveoutMaxShared);
  if (e != cudaSuccess) return e;
  edt_sweep<kXPass><<<(unsigned)((items + kSweepWarps - 1) / kSweepWarps), kSweepWarps * 32, smem, s>>>(
      map, scratch, (int)d.x, (int)d.y, (int)d.z);
  return cudaGetLastError();
}

}  // namespace

uint64_t edt_scratch_words(gvx_dims d) {
  const uint64_t y_pass = (uint64_t)((d.x + 31) / 32) * 32 * d.y * d.z;
  const uint64_t x_pass = (uint64_t)((d.y + 31) / 32) * 32 * d.x * d.z;
  return std::max(y_pass, x_pass);
}

cudaError_t launch_edt_pass(uint32_t* d_vox, uint32_t* d_scratch, gvx_dims d, int pass, cudaStream_t s) {
  switch (pass) {
    case 0: return launch_pass_z(d_vox, d, s);
    case 1: return launch_sweep<false>(d_vox, d_scratch, d, s);
    case 2: return launch_sweep<true>(d_vox, d_scratch, d, s);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_edt(uint32_t* d_vox, uint32_t* d_scratch, gvx_dims d, cudaStream_t s) {
  for (int pass = 0; pass < 3; ++pass) {
    cudaError_t e = launch_edt_pass(d_vox, d_scratch, d, pass, s);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

}  // namespace gvx
