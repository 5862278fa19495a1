// Exact 3D Euclidean distance transform on a DistanceVoxel map, in place.
//
// Result: bit-identical to DistanceVoxelMap::parallelBanding3D(1,1,1)
// (GV/voxelmap/DistanceVoxelMap.hpp:284-645) -- every voxel holds the same
// nearest site, including the reference's tie-breaking -- for any dims in
// [1,1023]^3 (the reference itself needs x == y and x % 64 == 0).
//
// Three sweeps, each one kernel that reads and writes every voxel once:
//   pass Z : phase 1 (kernelPBAphase1FloodZ, VoxelMapOperationsPBA.hpp:63-124)
//            per (x,y) column.
//   pass Y : phase 2 + 3 (kernelPBAphase2ProximateBackpointers :289-379,
//            kernelPBAphase3Distances :604-703) per (x,z) column along y.
//   pass X : the same sweep per (y,z) row along x.  The reference transposes
//            the map (kernelPBA3DTransposeXY :825-888) and sweeps along y
//            again; sweeping x directly in the original frame is the same
//            computation with the roles of the site's x and y fields swapped.
//
// Layout: one warp owns 32 adjacent columns and stages them in shared memory
// (cp.async), so the column walk and the positional proximate-site stack of
// phases 2/3 live on chip.  Column element (row r, lane l) sits at
// tile[r * pitch + l]; with pitch % 32 == 0 (passes Z, Y) or pitch == 33
// (pass X, transposed on load) the sequential walk is bank-conflict free.
// Each voxel costs 4 B of HBM read + 4 B of write per pass (24 B per EDT).
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "gvx_internal.cuh"

namespace gvx {
namespace {

__device__ __forceinline__ void cp_async4(uint32_t* smem_dst, const uint32_t* gmem_src) {
  unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async16(uint32_t* smem_dst, const uint32_t* gmem_src) {
  unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// devicePBAintersection3DY (VoxelMapOperationsPBA.hpp:265-276) in a column
// frame: sites (a, row, c), column at (a0, c0).  Same operation order; the
// products and sums are exact for coordinates below 1024, so only the IEEE
// divide and the final add round.  Explicit _rn intrinsics forbid contraction.
__device__ __forceinline__ float pba_isect(int a1, int r1, int c1, int a2, int r2, int c2, int a0, int c0) {
  const float aM = __fdiv_rn((float)(a1 + a2), 2.0f);
  const float rM = __fdiv_rn((float)(r1 + r2), 2.0f);
  const float cM = __fdiv_rn((float)(c1 + c2), 2.0f);
  const float na = (float)(a2 - a1);
  const float nr = (float)(r2 - r1);
  const float nc = (float)(c2 - c1);
  const float num = __fadd_rn(__fmul_rn(na, __fsub_rn(aM, (float)a0)), __fmul_rn(nc, __fsub_rn(cM, (float)c0)));
  return __fadd_rn(rM, __fdiv_rn(num, nr));
}

// Stack entry (internal): a | backptr<<10 | c<<20, the reference's packing.
struct Site {
  uint32_t a, b, c;  // a-field, back-pointer (or row for the input), c-field
};
__device__ __forceinline__ Site unpack(uint32_t e) { return Site{e & 0x3ffu, (e >> 10) & 0x3ffu, e >> 20}; }

// The a-field of an input value: x for pass Y, y for pass X (the transposed frame).
template <bool kXPass>
__device__ __forceinline__ uint32_t field_a(uint32_t v) {
  return kXPass ? ((v >> 10) & 0x3ffu) : (v & 0x3ffu);
}

// Phase 2 for one column held in shared memory (element r at col[r * pitch]).
// In place: each row is read before its stack entry overwrites it and
// back-pointers only reach rows already overwritten, exactly the reference's
// positional stack (there held in a separate initial_map buffer).
template <bool kXPass>
__device__ __forceinline__ void column_phase2(uint32_t* col, int pitch, int L, int a0, int c0) {
  int last_y = (int)kUninit;  // row of the stack top, UNINIT when empty
  Site top{kUninit, kUninit, kUninit}, second{kUninit, kUninit, kUninit};
  float i_top = 0.0f;  // intersection of (second, top); valid when top.b != UNINIT
  uint32_t cur_a = kUninit;
  for (int ty = 0; ty < L; ++ty) {
    const uint32_t v = col[ty * pitch];
    cur_a = field_a<kXPass>(v);
    if (cur_a != kUninit) {
      const uint32_t cur_c = v >> 20;
      float i2 = 0.0f;
      bool have_i2 = false;
      while (top.b != kUninit) {
        i2 = pba_isect((int)top.a, last_y, (int)top.c, (int)cur_a, ty, (int)cur_c, a0, c0);
        have_i2 = true;
        if (i_top < i2) break;
        last_y = (int)top.b;  // pop: top <- second, second <- *(second.backpointer)
        top = second;
        have_i2 = false;
        if (top.b != kUninit) {
          second = unpack(col[(int)top.b * pitch]);
          i_top = pba_isect((int)second.a, (int)top.b, (int)second.c, (int)top.a, last_y, (int)top.c, a0, c0);
        }
      }
      if (last_y != (int)kUninit) {  // the new pair (old top, current) gets its intersection
        i_top = have_i2 ? i2 : pba_isect((int)top.a, last_y, (int)top.c, (int)cur_a, ty, (int)cur_c, a0, c0);
      }
      second = top;
      top = Site{cur_a, (uint32_t)last_y, cur_c};
      last_y = ty;
      col[ty * pitch] = dv_pack(top.a, top.b, top.c);
    }
  }
  if (cur_a == kUninit) col[(L - 1) * pitch] = dv_pack(kUninit, (uint32_t)last_y, kUninit);  // tail pointer
}

// Phase 3 walk: calls emit(ty, site_a, site_row, site_c) for ty = L-1 .. 0.
template <class Emit>
__device__ __forceinline__ void column_phase3(const uint32_t* col, int pitch, int L, int a0, int c0, Emit&& emit) {
  int last_y = L - 1;
  Site top = unpack(col[last_y * pitch]);
  Site second{kUninit, kUninit, kUninit};
  float inter = 0.0f;
  if (top.a == kUninit) {  // tail pointer
    last_y = (int)top.b;
    if (last_y != (int)kUninit) top = unpack(col[last_y * pitch]);
  }
  if (top.b != kUninit) {
    second = unpack(col[(int)top.b * pitch]);
    inter = pba_isect((int)second.a, (int)top.b, (int)second.c, (int)top.a, last_y, (int)top.c, a0, c0);
  }
  for (int ty = L - 1; ty >= 0; --ty) {
    while (top.b != kUninit) {
      if ((float)ty > inter) break;
      last_y = (int)top.b;
      top = second;
      if (top.b != kUninit) {
        second = unpack(col[(int)top.b * pitch]);
        inter = pba_isect((int)second.a, (int)top.b, (int)second.c, (int)top.a, last_y, (int)top.c, a0, c0);
      }
    }
    emit(ty, top.a, (uint32_t)last_y, top.c);
  }
}

// Stage 32 adjacent columns (x0 .. x0+31) of `rows` rows into tile[r*32 + lane].
// Row r starts at src + r * stride.  Lanes past the map edge get UNINIT.
__device__ __forceinline__ void stage_rows32(uint32_t* tile, const uint32_t* src, uint64_t stride, int rows,
                                             int valid_cols, bool vec16) {
  const int lane = threadIdx.x & 31;
  if (vec16) {
    // 8 chunks of 16 B per row; lane covers chunk (lane & 7) of rows (lane >> 3) + 4k.
    const int part = lane & 7;
    for (int r = lane >> 3; r < rows; r += 4) cp_async16(tile + r * 32 + part * 4, src + (uint64_t)r * stride + part * 4);
  } else if (lane < valid_cols) {
    for (int r = 0; r < rows; ++r) cp_async4(tile + r * 32 + lane, src + (uint64_t)r * stride + lane);
  } else {
    for (int r = 0; r < rows; ++r) tile[r * 32 + lane] = kDvUninit;
  }
  cp_async_wait_all();
  __syncwarp();
}

// ---------------------------------------------------------------------------
// pass Z: phase 1 per (x, y) column, m1 = 1.
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
  const bool vec16 = (valid_cols == 32) && ((X & 3) == 0);
  stage_rows32(tile, src, layer, Z, valid_cols, vec16);

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
// pass Y: phases 2 + 3 per (x, z) column along y.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) edt_pass_y(uint32_t* __restrict__ map, int X, int Y, int Z, int warps_per_cta) {
  extern __shared__ __align__(16) uint32_t smem[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nxb = (X + 31) >> 5;
  const long long item = (long long)blockIdx.x * warps_per_cta + warp;
  if (item >= (long long)nxb * Z) return;
  const int xb = (int)(item % nxb), z = (int)(item / nxb);
  const int x0 = xb * 32, valid_cols = min(32, X - x0);
  const uint64_t layer = (uint64_t)X * Y;
  uint32_t* tile = smem + (size_t)warp * Y * 32;
  uint32_t* slice = map + (uint64_t)z * layer + x0;
  const bool vec16 = (valid_cols == 32) && ((X & 3) == 0);
  stage_rows32(tile, slice, (uint64_t)X, Y, valid_cols, vec16);

  const int tx = x0 + lane;
  uint32_t* col = tile + lane;
  column_phase2<false>(col, 32, Y, tx, z);
  const bool store = lane < valid_cols;
  column_phase3(col, 32, Y, tx, z, [&](int ty, uint32_t a, uint32_t row, uint32_t c) {
    if (store) slice[(uint64_t)ty * X + lane] = dv_pack(a, row, c);
  });
}

// ---------------------------------------------------------------------------
// pass X: phases 2 + 3 per (y, z) row along x, in the original frame.
// Lane l owns row y0 + l; the rows are staged transposed (tile[x*33 + l]) and
// the results leave through a 32x33 per-warp buffer so stores stay coalesced.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) edt_pass_x(uint32_t* __restrict__ map, int X, int Y, int Z, int warps_per_cta) {
  extern __shared__ __align__(16) uint32_t smem[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nyb = (Y + 31) >> 5;
  const long long item = (long long)blockIdx.x * warps_per_cta + warp;
  if (item >= (long long)nyb * Z) return;
  const int yb = (int)(item % nyb), z = (int)(item / nyb);
  const int y0 = yb * 32, valid_rows = min(32, Y - y0);
  const uint64_t layer = (uint64_t)X * Y;
  const int per_warp = X * 33 + 32 * 33;
  uint32_t* tile = smem + (size_t)warp * per_warp;
  uint32_t* stage = tile + X * 33;
  uint32_t* slice = map + (uint64_t)z * layer + (uint64_t)y0 * X;

  for (int r = 0; r < 32; ++r) {
    if (r < valid_rows) {
      for (int x = lane; x < X; x += 32) cp_async4(tile + x * 33 + r, slice + (uint64_t)r * X + x);
    } else {
      for (int x = lane; x < X; x += 32) tile[x * 33 + r] = kDvUninit;
    }
  }
  cp_async_wait_all();
  __syncwarp();

  const int ty0 = y0 + lane;
  uint32_t* col = tile + lane;
  column_phase2<true>(col, 33, X, ty0, z);
  column_phase3(col, 33, X, ty0, z, [&](int tx, uint32_t a, uint32_t row, uint32_t c) {
    // output in the original frame: x-field = row of the site, y-field = a
    stage[(tx & 31) * 33 + lane] = dv_pack(row, a, c);
    if ((tx & 31) == 0) {
      __syncwarp();
      const int xb = tx;  // chunk [xb, xb + 31]
      if (xb + lane < X) {
        for (int r = 0; r < valid_rows; ++r) slice[(uint64_t)r * X + xb + lane] = stage[lane * 33 + r];
      }
      __syncwarp();
    }
  });
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

// Warps per CTA: as many as fit a ~96 KB CTA budget, at most 8.
int pick_warps(size_t bytes_per_warp) {
  int w = (int)(98304 / bytes_per_warp);
  return std::max(1, std::min(8, w));
}

template <typename K>
cudaError_t launch_pass(K kernel, uint32_t* map, gvx_dims d, long long items, size_t bytes_per_warp, cudaStream_t s) {
  const int w = pick_warps(bytes_per_warp);
  const size_t smem = bytes_per_warp * w;
  if ((int)smem > max_smem_optin()) return cudaErrorInvalidConfiguration;
  cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const long long blocks = (items + w - 1) / w;
  kernel<<<(unsigned)blocks, 32 * w, smem, s>>>(map, (int)d.x, (int)d.y, (int)d.z, w);
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_edt_pass(uint32_t* d_vox, gvx_dims d, int pass, cudaStream_t s) {
  const long long nxb = (d.x + 31) / 32, nyb = (d.y + 31) / 32;
  switch (pass) {
    case 0: return launch_pass(edt_pass_z, d_vox, d, nxb * d.y, (size_t)d.z * 32 * 4, s);
    case 1: return launch_pass(edt_pass_y, d_vox, d, nxb * d.z, (size_t)d.y * 32 * 4, s);
    case 2: return launch_pass(edt_pass_x, d_vox, d, nyb * d.z, ((size_t)d.x * 33 + 32 * 33) * 4, s);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_edt(uint32_t* d_vox, gvx_dims d, cudaStream_t s) {
  for (int pass = 0; pass < 3; ++pass) {
    cudaError_t e = launch_edt_pass(d_vox, d, pass, s);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

}  // namespace gvx
