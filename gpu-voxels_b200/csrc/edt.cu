// Exact 3D Euclidean distance transform on a DistanceVoxel map, in place.
//
// Result: bit-identical to DistanceVoxelMap::parallelBanding3D(1,1,1)
// (GV/voxelmap/DistanceVoxelMap.hpp:284-645) -- every voxel holds the same
// nearest site, including the reference's tie-breaking -- for any dims in
// [1,1023]^3 (the reference itself needs x == y and x % 64 == 0).
//
// Three sweeps (pass Z one launch, passes Y and X one fused launch):
//   pass Z : phase 1 (kernelPBAphase1FloodZ, VoxelMapOperationsPBA.hpp:63-124)
//            per (x,y) column.
//   pass Y : phase 2 + 3 (kernelPBAphase2ProximateBackpointers :289-379,
//            kernelPBAphase3Distances :604-703) per (x,z) column along y.
//   pass X : the same sweep per (y,z) row along x.  The reference transposes
//            the map (kernelPBA3DTransposeXY :825-888) and sweeps along y
//            again; sweeping x directly in the original frame is the same
//            computation with the roles of the site's x and y fields swapped.
//
// Passes Y and X: one thread per column, a warp owns 32 consecutive columns
// (numbered slice by slice, so an item may span slices) and streams them
// through shared memory in chunks of rows (cp.async, double buffered; pass X
// transposes each chunk on the way in and out).  Within a chunk the rows
// advance in lockstep and only the stack pops a row triggers run divergently;
// a lane with a long run of pops hands it to the whole warp, which tests 31
// stack entries per round.  The proximate-site stack is compact
// (depth-indexed, each entry carries its row): its top lives in an on-chip
// ring per lane together with each entry's bisector, an entry reaches the
// map's workspace only when the ring evicts it, and phase 3 streams the stack
// back top-down through a prefetched on-chip window.  Stack order, tests and
// tie rules are the reference's; the bisector's quotient is rounded exactly
// as the IEEE divide rounds it (quotient_rn).
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cstdlib>
#include <mutex>

#include "gvx_internal.cuh"

namespace gvx {
namespace {

constexpr unsigned kFullMask = 0xffffffffu;

__device__ __forceinline__ void cp_async4(uint32_t* smem_dst, const uint32_t* gmem_src) {
  unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async8(void* smem_dst, const void* gmem_src) {
  unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async16(uint32_t* smem_dst, const uint32_t* gmem_src) {
  unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// ---------------------------------------------------------------------------
// pass Z: phase 1 per (x, y) column, m1 = 1.
// The forward flood only changes value at rows whose input holds a site, so
// the forward scan records those (value, row) pairs -- the column's site list
// -- in an on-chip ring, and the backward flood walks the list downward.
// Each lane also stores its forward-flood value at the end of every chunk
// (the chunk's carry) to the workspace.  A warp in which some column has more
// sites than the ring holds walks back chunk by chunk instead: it restages
// the (still unmodified) input of each chunk, rebuilds the chunk's forward
// flood from the carry of the chunk below, and floods backward from that.
// Every row is a fixed, lockstep step.
// ---------------------------------------------------------------------------
constexpr int kZChunk = 16;
constexpr int kZRing = 16;
constexpr int kZWarps = 8;
// Pass Z from occupancy bits keeps two words per lane and 32-row chunk (the
// chunk's mask and the last site below it); up to 32 chunks (Z <= 1024).
__host__ __device__ constexpr int z_bits_words(int Z) { return 32 * ((Z + 31) >> 5); }
constexpr int kZBitsSmemMax = kZWarps * 2 * z_bits_words(1024) * 4;
constexpr int kZWarpWords = 2 * kZChunk * 32 + 2 * kZRing * 32;

// Words of the EDT workspace's counter area (Z slice counters, queue head,
// error word, pass Z's other-sites flag, padded to 32).
__host__ __device__ __forceinline__ uint64_t edt_sync_words(int Z) { return ((uint64_t)Z + 3 + 31) / 32 * 32; }

// Workspace words of pass Z's chunk carries for a map: per warp item
// (32 columns) one word per lane and chunk.
__host__ __device__ __forceinline__ uint64_t zcarry_item_words(int Z) { return (uint64_t)((Z + kZChunk - 1) / kZChunk) * 32; }

// Pass Z items: the (x, y) columns numbered f = y * X + x, 32 consecutive
// ones per warp item (an item may span rows of the layer, so no lane idles).
__host__ __device__ __forceinline__ uint64_t z_items(int X, int Y) { return ((uint64_t)X * Y + 31) / 32; }

// One warp item of pass Z (columns f0 .. f0 + 31); wbase = the warp's
// kZWarpWords of shared memory; carry = the item's zcarry_item_words(Z) words.
// The sites carry their own coordinates, so the columns' (x, y) are not needed.
__device__ __forceinline__ void pass_z_item(uint32_t* __restrict__ map, int X, int Y, int Z, long long item,
                                            uint32_t* wbase, uint32_t* __restrict__ carry) {
  const int lane = threadIdx.x & 31;
  const uint64_t layer = (uint64_t)X * Y;
  const uint64_t f0 = (uint64_t)item * 32;
  const int valid_cols = layer - f0 < 32 ? (int)(layer - f0) : 32;
  uint32_t* const tile0 = wbase;
  uint32_t* const tile1 = wbase + kZChunk * 32;
  uint32_t* ringV = wbase + 2 * kZChunk * 32 + lane;  // slot k: ringV[k * 32]
  uint32_t* ringR = ringV + kZRing * 32;
  const uint32_t* src = map + f0;
  const bool vec16 = valid_cols == 32 && (layer & 3) == 0;  // f0 is a multiple of 32
  const int nchunks = (Z + kZChunk - 1) / kZChunk;
  auto stage = [&](uint32_t* tile, int c) {
    const int r0 = c * kZChunk, rows = min(kZChunk, Z - r0);
    const uint32_t* s0 = src + (uint64_t)r0 * layer;
    if (vec16) {
      const int part = lane & 7;
      for (int r = lane >> 3; r < rows; r += 4) cp_async16(tile + r * 32 + part * 4, s0 + (uint64_t)r * layer + part * 4);
    } else if (lane < valid_cols) {
      for (int r = 0; r < rows; ++r) cp_async4(tile + r * 32 + lane, s0 + (uint64_t)r * layer + lane);
    } else {
      for (int r = 0; r < rows; ++r) tile[r * 32 + lane] = kDvUninit;
    }
  };

  // forward: record the sites of the column and each chunk's carry
  stage(tile0, 0);
  cp_async_commit();
  if (nchunks > 1) stage(tile1, 1);
  cp_async_commit();
  int m = 0;                 // sites seen
  uint32_t flood = kDvUninit;  // forward-flood value
  // This lane's column as a DistanceVoxel without z (idle lanes: unused).
  uint32_t xy;
  {
    const uint32_t f = (uint32_t)(f0 + lane < layer ? f0 + lane : layer - 1), y = f / (uint32_t)X;
    xy = (f - y * (uint32_t)X) | (y << 10);
  }
  bool self = true;  // every site of the column holds its own voxel (as after insertPointCloud)
  for (int c = 0; c < nchunks; ++c) {
    cp_async_wait1();
    __syncwarp();
    const uint32_t* tile = (c & 1) ? tile1 : tile0;
    const int r0 = c * kZChunk, rows = min(kZChunk, Z - r0);
    for (int r = 0; r < rows; ++r) {
      const uint32_t v = tile[r * 32 + lane];
      if ((v >> 20) != kUninit) {
        ringV[(m % kZRing) * 32] = v;
        ringR[(m % kZRing) * 32] = (uint32_t)(r0 + r);
        ++m;
        flood = v;
        self = self && v == (xy | ((uint32_t)(r0 + r) << 20));
      }
    }
    carry[c * 32 + lane] = flood;
    __syncwarp();
    if (c + 2 < nchunks) stage((c & 1) ? tile1 : tile0, c + 2);
    cp_async_commit();
  }
  cp_async_wait_all();
  __syncwarp();

  // backward: obstacle(z) from the forward value fwd(z) = last site at or below z;
  // ties keep the lower z (<=, VoxelMapOperationsPBA.hpp:112-122)
  uint32_t obstacle = kDvUninit;
  uint32_t* dst = map + f0 + lane;
  const bool live = lane < valid_cols;
  if (__all_sync(kFullMask, self && m <= kZRing)) {
    // Every site holds its own voxel and the ring holds them all: the closed
    // form of the backward rule (the occupancy-bit pass, pass_z_bits_item):
    // between consecutive site rows s1 < s2 (s2 = 1023 above the highest,
    // s1 = 1023 below the lowest) rows z <= (s1 + s2) / 2 take s1, the rest s2.
    auto enc = [&](int o) -> uint32_t { return o == 1023 ? kDvUninit : xy | ((uint32_t)o << 20); };
    int j = m - 1;  // ring index of s1
    int s1 = j >= 0 ? (int)ringR[(j % kZRing) * 32] : 1023, s2 = 1023, sw;
    uint32_t v1, v2;
    auto set_pair = [&]() {
      sw = s1 == 1023 ? -1 : (s1 + s2) >> 1;
      v1 = enc(s1);
      v2 = enc(s2);
    };
    set_pair();
    int z = Z - 1;
    for (; z >= 0 && ((z + 1) & 31); --z) {  // down to a multiple of 32 rows, row by row
      if (s1 != 1023 && z < s1) {
        s2 = s1;
        --j;
        s1 = j >= 0 ? (int)ringR[(j % kZRing) * 32] : 1023;
        set_pair();
      }
      if (live) dst[(uint64_t)z * layer] = z <= sw ? v1 : v2;
    }
    for (int zc = z - 31; zc >= 0; zc -= 32) {  // 32-row chunks
      uint32_t* d = dst + (uint64_t)(zc + 31) * layer;
      if (__all_sync(kFullMask, s1 == 1023 || s1 < zc)) {  // no lane passes a site here
#pragma unroll
        for (int l = 31; l >= 0; --l) {
          if (live) *d = zc + l <= sw ? v1 : v2;
          d -= layer;
        }
      } else {
#pragma unroll
        for (int l = 31; l >= 0; --l) {
          if (s1 != 1023 && zc + l < s1) {
            s2 = s1;
            --j;
            s1 = j >= 0 ? (int)ringR[(j % kZRing) * 32] : 1023;
            set_pair();
          }
          if (live) *d = zc + l <= sw ? v1 : v2;
          d -= layer;
        }
      }
    }
    return;
  }
  if (!__any_sync(kFullMask, m > kZRing)) {
    int j = m - 1;  // index of the site fwd(z)
    uint32_t fwdV = kDvUninit;
    int fwdRow = -1;
    if (j >= 0) {
      fwdV = ringV[(j % kZRing) * 32];
      fwdRow = (int)ringR[(j % kZRing) * 32];
    }
    for (int z = Z - 1; z >= 0; --z) {
      while (fwdRow > z) {  // step to the previous site (all in the ring)
        --j;
        if (j < 0) {
          fwdV = kDvUninit;
          fwdRow = -1;
        } else {
          fwdV = ringV[(j % kZRing) * 32];
          fwdRow = (int)ringR[(j % kZRing) * 32];
        }
      }
      const int dist_prev = abs((int)(obstacle >> 20) - z);
      const int dist_next = abs(z - (int)(fwdV >> 20));
      if (dist_next <= dist_prev) obstacle = fwdV;
      if (live) dst[(uint64_t)z * layer] = obstacle;
    }
    return;
  }
  // chunk by chunk: restage the input (descending, double buffered), rebuild
  // the chunk's forward flood in place from the carry below, flood backward
  __syncwarp();  // the carries of all lanes
  stage(tile0, nchunks - 1);
  cp_async_commit();
  if (nchunks > 1) stage(tile1, nchunks - 2);
  cp_async_commit();
  for (int c = nchunks - 1, k = 0; c >= 0; --c, ++k) {
    cp_async_wait1();
    __syncwarp();
    uint32_t* tile = (k & 1) ? tile1 : tile0;
    const int r0 = c * kZChunk, rows = min(kZChunk, Z - r0);
    uint32_t f = c > 0 ? carry[(c - 1) * 32 + lane] : kDvUninit;
    for (int r = 0; r < rows; ++r) {
      const uint32_t v = tile[r * 32 + lane];
      if ((v >> 20) != kUninit) f = v;
      tile[r * 32 + lane] = f;
    }
    for (int r = rows - 1; r >= 0; --r) {
      const int z = r0 + r;
      const uint32_t fwdV = tile[r * 32 + lane];
      const int dist_prev = abs((int)(obstacle >> 20) - z);
      const int dist_next = abs(z - (int)(fwdV >> 20));
      if (dist_next <= dist_prev) obstacle = fwdV;
      if (live) dst[(uint64_t)z * layer] = obstacle;
    }
    __syncwarp();
    if (c - 2 >= 0) stage(tile, c - 2);
    cp_async_commit();
  }
  cp_async_wait_all();
}

// ---------------------------------------------------------------------------
// Voxelisation fused with pass Z.  After clearMap + insertPointCloud a
// DistanceVoxelMap holds each occupied voxel's own coordinate and UNINIT
// elsewhere, so it is fully described by one occupancy bit per voxel.  The
// fused path records those bits (word (f / 32) * Z + z, bit f % 32, f = y * X + x)
// in the workspace instead of clearing and scattering the map, and pass Z
// reads the bits: the map is written once, by pass Z.  The flood arithmetic
// is phase 1's (the same values, the same ties, UNINIT's z read as 1023).
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ uint64_t occ_words(int X, int Y, int Z) { return z_items(X, Y) * Z; }

__device__ __forceinline__ void occ_set(uint32_t* bits, int X, int Z, uint32_t x, uint32_t y, uint32_t z) {
  const uint32_t f = y * (uint32_t)X + x;
  atomicOr(bits + (uint64_t)(f >> 5) * Z + z, 1u << (f & 31));
}

// insertPointCloud into the occupancy bits (coordinates as
// kernelInsertGlobalPointCloud, GV/voxelmap/kernels/VoxelMapOperations.hpp:266-300).
__global__ void occ_insert_kernel(uint32_t* __restrict__ bits, int X, int Y, int Z, float side,
                                  const float* __restrict__ xyz, uint64_t n, uint32_t* __restrict__ outside) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  bool out = false;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const uint32_t x = coord_to_voxel(__ldg(xyz + 3 * i), side), y = coord_to_voxel(__ldg(xyz + 3 * i + 1), side),
                   z = coord_to_voxel(__ldg(xyz + 3 * i + 2), side);
    if (x < (uint32_t)X && y < (uint32_t)Y && z < (uint32_t)Z) occ_set(bits, X, Z, x, y, z);
    else out = true;
  }
  if (outside != nullptr && __any_sync(kFullMask, out) && (threadIdx.x & 31) == 0) *outside = 1u;
}

// Pass Z of one warp item (32 consecutive columns f = y * X + x) from occupancy bits.
// The item's Z words are read 32 at a time and bit-transposed across the warp
// into one 32-row mask per lane; an ascending pass keeps, per 32-row chunk, each lane's
// mask and the last occupied z below the chunk (smem), and the backward flood
// reads the forward value of every row from them.  wbase: 2 * zw words, zw =
// 32 * (chunks of the tallest map of the launch) (z_bits_words).
__device__ __forceinline__ void pass_z_bits_item(uint32_t* __restrict__ map, const uint32_t* __restrict__ bits, int X,
                                                 int Y, int Z, long long item, uint32_t* wbase, int zw) {
  const int lane = threadIdx.x & 31;
  const uint32_t f = (uint32_t)item * 32u + (uint32_t)lane;  // this lane's column y * X + x
  const uint32_t* wcol = bits + (uint64_t)item * Z;
  uint32_t* mk = wbase + lane;         // chunk c: mk[c * 32]
  uint32_t* lb = wbase + zw + lane;  // chunk c: lb[c * 32], 1023 = none
  const int nch = (Z + 31) >> 5;
  // All of the column's occupancy words in flight at once (word z of chunk c
  // lands in mk[c * 32] of lane z & 31), then transposed in place: a lane
  // reads its word, the butterfly exchanges registers, and the lane writes
  // its mask back to the same slot.
  for (int c = 0; c < nch; ++c) {
    const int z = c * 32 + lane;
    if (z < Z) cp_async4(mk + c * 32, wcol + z);
    else mk[c * 32] = 0u;
  }
  cp_async_commit();
  cp_async_wait_all();
  __syncwarp();
  uint32_t last = 1023u;
  for (int c = 0; c < nch; ++c) {
    // 32 x 32 bit transpose across the warp (lane l holds row c*32 + l, bit j
    // = column j): five butterfly stages, each swapping the off-diagonal
    // s x s blocks between lanes l and l ^ s.
    uint32_t mine = mk[c * 32];
#pragma unroll
    for (int sft = 16; sft >= 1; sft >>= 1) {
      const uint32_t hi = sft == 16 ? 0xFFFF0000u : sft == 8 ? 0xFF00FF00u : sft == 4 ? 0xF0F0F0F0u
                        : sft == 2 ? 0xCCCCCCCCu : 0xAAAAAAAAu;  // columns j with j & sft
      const uint32_t t = __shfl_xor_sync(kFullMask, mine, sft);
      mine = (lane & sft) ? (mine & hi) | ((t & hi) >> sft) : (mine & ~hi) | ((t & ~hi) << sft);
    }
    mk[c * 32] = mine;
    lb[c * 32] = last;
    if (mine) last = (uint32_t)(c * 32 + 31 - __clz(mine));
  }
  __syncwarp();
  const uint64_t layer = (uint64_t)X * Y;
  uint32_t* const col = map + f;  // dereferenced only when live
  const bool live = f < layer;
  const uint32_t fl = min(f, (uint32_t)layer - 1u);
  const uint32_t y = fl / (uint32_t)X;
  const uint32_t base = (fl - y * (uint32_t)X) | (y << 10);
  auto enc = [&](int o) -> uint32_t { return o == 1023 ? kDvUninit : base | ((uint32_t)o << 20); };
  // kernelPBAphase1FloodZ's backward loop keeps the forward-flood value fz
  // (the highest site at or below z) when |z - fz| <= |obst - z|.  Between
  // consecutive sites s1 < s2 of a column (s2 = 1023 above the highest
  // site, s1 = 1023 below the lowest) that recurrence gives s1 on the rows
  // z <= (s1 + s2) / 2 and s2 above (with s1 = 1023: s2 everywhere), the
  // reference's UNINIT-as-1023 arithmetic included.  So a row is one compare
  // and select; the pair (s1, s2) moves down only when the scan passes s1.
  int s2 = 1023, s1, sw;
  uint32_t v1, v2;
  auto set_pair = [&]() {
    sw = s1 == 1023 ? -1 : (s1 + s2) >> 1;
    v1 = enc(s1);
    v2 = enc(s2);
  };
  {
    const int c = nch - 1;
    const uint32_t mm = mk[c * 32] & ((2u << ((Z - 1) & 31)) - 1u);
    s1 = mm ? c * 32 + 31 - __clz(mm) : (int)lb[c * 32];
  }
  set_pair();
  for (int c = nch - 1; c >= 0; --c) {
    const int zc = c * 32;
    const uint32_t mfull = mk[c * 32];
    const int lbc = (int)lb[c * 32];
    const int top = min(31, Z - 1 - zc);
    uint32_t* dst = col + (uint64_t)(zc + top) * layer;
    auto row = [&](int l) {
      const int z = zc + l;
      if (s1 != 1023 && z < s1) {  // the scan passed s1: the pair moves down
        s2 = s1;
        const uint32_t mm = mfull & ((2u << l) - 1u);
        s1 = mm ? zc + 31 - __clz(mm) : lbc;
        set_pair();
      }
      if (live) *dst = z <= sw ? v1 : v2;
      dst -= layer;
    };
    if (top == 31 && __all_sync(kFullMask, s1 == 1023 || s1 < zc)) {
      // no lane passes a site in this chunk (none in it, none above s1)
#pragma unroll
      for (int l = 31; l >= 0; --l) {
        if (live) *dst = zc + l <= sw ? v1 : v2;
        dst -= layer;
      }
    } else if (top == 31) {
#pragma unroll
      for (int l = 31; l >= 0; --l) row(l);
    } else {
      for (int l = top; l >= 0; --l) row(l);
    }
  }
}

// skip (optional): the flag occ_from_map_kernel sets when the general pass Z
// has to run instead.
__global__ void __launch_bounds__(kZWarps * 32) edt_pass_z_bits(uint32_t* __restrict__ map,
                                                                 const uint32_t* __restrict__ bits, int X, int Y, int Z,
                                                                 const uint32_t* __restrict__ skip) {
  extern __shared__ __align__(16) uint32_t s_z[];  // [kZWarps][2 * zw]
  if (skip != nullptr && *skip != 0u) return;
  const int warp = threadIdx.x >> 5;
  const long long item = (long long)blockIdx.x * kZWarps + warp;
  if (item >= (long long)z_items(X, Y)) return;
  const int zw = z_bits_words(Z);
  pass_z_bits_item(map, bits, X, Y, Z, item, s_z + (size_t)warp * 2 * zw, zw);
}

// ---------------------------------------------------------------------------
// passes Y and X
// ---------------------------------------------------------------------------

// Exact small-integer -> float conversions on the ALU/FMA pipes (the
// converter sits on the narrow XU pipe, which the reciprocal also needs):
// for 0 <= v < 2^22 the bit pattern 0x4B400000 | v is the float
// kBias + v with kBias = 2^23 + 2^22, and a difference of two such floats is
// exact.  A column coordinate is kept biased (kBias + a0, exact below 2^24).
constexpr float kBias = 12582912.0f;
__device__ __forceinline__ float biased(uint32_t v) { return __uint_as_float(0x4B400000u | v); }
__device__ __forceinline__ float small_to_float(int v) { return biased((uint32_t)v) - kBias; }

// a - b per component in one packed instruction: fma(b, -1, a) rounds once,
// the same as the scalar subtraction.
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.f, -1.f), a); }


// A site in the column frame: packed entry (a | row << 10 | c << 20) plus
// twice its row and its squared offset from the column as exact floats
// (offset < 2^21).  A0, C0: the column's coordinates, biased.
//
// kOwn: pass Z took the occupancy-bit route (every input voxel UNINIT or its
// own site), so every site pass Y reads shares its voxel's x and y, and every
// site pass X reads shares its voxel's x.  The map's own entries then serve as
// stack entries: pass Y's frame order is the map order, its site's row field
// already equals the row and its a offset is 0 (the squared offset is dc^2
// alone, the same float); pass X keeps map order (row = x in bits 0-9, a = y
// in bits 10-19), so its sites go back to the map unchanged.
struct Col {
  uint32_t e;
  float r2, d;
};

template <bool kXPass, bool kOwn>
__device__ __forceinline__ Col make_col(uint32_t e, float A0, float C0) {
  constexpr bool kMapX = kXPass && kOwn;
  Col s;
  s.e = e;
  s.r2 = biased(kMapX ? ((e << 1) & 0x7feu) : ((e >> 9) & 0x7feu)) - kBias;  // 2 * row
  if (!kXPass && kOwn) {
    const float dc = biased(e >> 20) - C0;
    s.d = __fmul_rn(dc, dc);
  } else {
    const float2 dd =
        sub2(make_float2(biased(kMapX ? ((e >> 10) & 0x3ffu) : (e & 0x3ffu)), biased(e >> 20)), make_float2(A0, C0));
    s.d = __fmaf_rn(dd.x, dd.x, __fmul_rn(dd.y, dd.y));  // exact: integers below 2^21
  }
  return s;
}

// devicePBAintersection3DY (VoxelMapOperationsPBA.hpp:265-276) is
//   yM + (nx*(xM-x0) + nz*(zM-z0)) / ny.
// For integer coordinates below 1024 its numerator is exact in float and
// equals (d2 - d1) / 2, d = squared offset of a site from the column, so the
// value is fl(0.5*(r1 + r2) + fl((d2 - d1) / (2*(r2 - r1)))) with every operand
// exact: bit for bit the reference's float.  With r2 = 2 * row the divisor is
// r2' - r2 (never 0: stacked sites have distinct rows) and the midpoint
// 0.25 * (r2 + r2'), both exact.
//
// The quotient is rounded to nearest without the general divide: num is an
// integer with |num| < 2^21 and den an even integer in [2, 2046] (rows below
// 1024, the later site second).  Markstein's correction (P. Markstein,
// "Computation of elementary functions on the IBM RISC System/6000
// processor", IBM J. Res. Develop. 34(1), 1990): with q0 close to Q = num/den
// the residual r = num - q0*den is exact in one fma, and fma(r, y, q0) with
// y ~ 1/den is Q plus (Q - q0) * (y*den - 1).  Here y is the hardware's
// approximate reciprocal alone (relative error about 2^-23) and q0 = num*y,
// so |Q - q0| < 2^-22 |Q| and the fma's exact value is within 2^-21 ulp of
// Q.  Q is never that close to a rounding midpoint: num has at most 21
// significant bits, so Q is not a 25-bit binary fraction (no ties), and a
// midpoint m = (2k+1) 2^(e-24) differs from num/den by a nonzero multiple of
// 2^(e-24)/den, at least 2^-12 ulp for den <= 2046.  The fma therefore rounds
// to RN(Q).  gvx_check_bisector_quotient compares every (num, den) of the
// domain with the IEEE divide on the device.
__device__ __forceinline__ float quotient_rn(float num, float den) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(den));
  const float q0 = __fmul_rn(num, y);
  const float r = __fmaf_rn(-q0, den, num);
  return __fmaf_rn(r, y, q0);
}

__device__ __forceinline__ float bisect(const Col& s1, const Col& s2) {
  const float2 df = sub2(make_float2(s2.d, s2.r2), make_float2(s1.d, s1.r2));
  const float q = quotient_rn(df.x, df.y);
  return __fadd_rn(__fmul_rn(__fadd_rn(s1.r2, s2.r2), 0.25f), q);
}

// Geometry of one warp's work item.
// The columns of a pass are numbered slice by slice (f = z * cols + a, cols =
// X for pass Y, Y for pass X) and an item is 32 consecutive ones, so no lane
// idles when cols is not a multiple of 32: such an item spans two (or, with
// cols < 32, more) slices.
struct Sweep {
  int L;             // column length (rows)
  int valid;         // valid lanes (a prefix of the warp)
  bool one_slice;    // every valid lane in one slice (warp-uniform)
  uint32_t* map;
  int X;             // map row length
  uint32_t col;      // this lane's column start (element index; pass Y: row stride X, pass X: contiguous)
  uint32_t col0;     // lane 0's column start
  int a, z;          // this lane's column coordinate (x for pass Y, y for pass X) and slice
};

// Column start of row t of an X-pass item spanning slices: lane t's `col`
// (all lanes take part).
__device__ __forceinline__ uint32_t row_start(const Sweep& s, int t) {
  return __shfl_sync(0xffffffffu, s.col, t & 31);
}

template <int kRows>
struct SweepCfg {
  static constexpr int kWarps = 8;                       // warps per CTA
  static constexpr int kTileWords = kRows * 33;          // one staging tile
  static constexpr int kRing = 16;                       // ring slots per lane (a power of two)
  static constexpr int kPhase2Words = 2 * kTileWords + 2 * kRing * 32;
  // Phase 3: pass X stages kStageRows output rows (pitch 36) before its
  // transposed flush; pass Y stores rows directly.  The stack window (kWin
  // (site, bisector) pairs per lane) follows the staging rows.
  static constexpr int kStageRows = 8;
  static constexpr int kStagePitch = 36;
  static constexpr int kStageWords = kStageRows * kStagePitch;
  static constexpr int kWin = 32;
  static constexpr int kPhase3Words = kStageWords + kWin * 64;
  static constexpr int kWarpWords = kPhase2Words > kPhase3Words ? kPhase2Words : kPhase3Words;
  static_assert((kWin & (kWin - 1)) == 0, "window slots are depth mod kWin");
  static_assert((kRing & (kRing - 1)) == 0, "ring slots are depth mod kRing");
  static_assert(kTileWords % 4 == 0, "the second tile and the ring take 16-byte copies and 8-byte slots");
  static_assert(kStageWords % 2 == 0 && kWarpWords % 2 == 0, "8-byte window entries need even offsets");
};

// Finish the pops of lane `o` with the whole warp.  The stack entries of a
// column are e_0 .. e_{n-1} with I_j = bisect(e_{j-1}, e_j); the sequential
// loop pops e_j while !(I_j < bisect(e_j, cur)) and stops at j = 0.  Each
// test depends only on e_j, I_j and cur, so lane t tests depth start - t and
// the first kept depth (lowest t) is exactly where the sequential loop stops.
// Lane 31 only supplies the entry below lane 30's, so a round covers 31
// depths.  All 32 lanes call this; only lane o's state changes.  Pass Y
// only.
template <class Cfg, bool kOwnA>
__device__ __forceinline__ void coop_pops(int o, float A0, float C0, uint2* ring_base, const uint2* gstk_base, int L,
                                          int& n, int& lo, const Col& cur, Col& top, float& top_i, float& i2) {
  const int lane = threadIdx.x & 31;
  const int on = __shfl_sync(kFullMask, n, o);
  const int olo = __shfl_sync(kFullMask, lo, o);
  const uint32_t ce = __shfl_sync(kFullMask, cur.e, o);
  const float oA0 = __shfl_sync(kFullMask, A0, o);  // lane o's column, biased
  const float oC0 = __shfl_sync(kFullMask, C0, o);
  const Col oc = make_col<false, kOwnA>(ce, oA0, oC0);
  uint2* ring = ring_base + o;
  const uint2* gstk = gstk_base + (size_t)o * L;
  for (int start = on - 1;; start -= 31) {
    const int j = start - lane;
    const int jc = max(j, 0);
    // the ring slot, replaced by the workspace entry below the ring (a
    // predicated load, so one decode and no divergent branch)
    const uint2 rq = ring[(jc & (Cfg::kRing - 1)) * 32];
    uint32_t e = rq.x;
    float I = __uint_as_float(rq.y);
    if (jc < olo) {
      const uint2 p = gstk[jc];
      e = p.x;
      I = __uint_as_float(p.y);
    }
    const Col ec = make_col<false, kOwnA>(e, oA0, oC0);
    const float b = bisect(ec, oc);
    const bool keep = j <= 0 || I < b;
    const unsigned kb = __ballot_sync(kFullMask, keep) & 0x7fffffffu;
    if (kb) {
      const int t = __ffs(kb) - 1;
      // Refill lane o's ring with the tested entries from the kept depth
      // down (their slots belong to popped depths), so its next pops stay on
      // chip: after the push the ring holds depths >= new_lo.
      const int u_last = min(t + Cfg::kRing - 2, 31);
      const int new_lo = max(start - u_last, 0);
      if (lane >= t && lane <= u_last && j >= 0 && jc < olo) {
        ring[(jc & (Cfg::kRing - 1)) * 32] = make_uint2(e, __float_as_uint(I));
      }
      const uint32_t e_top = __shfl_sync(kFullMask, e, t);
      const float i_top = __shfl_sync(kFullMask, I, t);
      const float b_top = __shfl_sync(kFullMask, b, t);
      if (lane == o) {
        n = start - t + 1;
        lo = min(lo, new_lo);
        top = make_col<false, kOwnA>(e_top, oA0, oC0);
        top_i = i_top;
        i2 = b_top;
      }
      __syncwarp();  // the refill before lane o's next ring access
      return;
    }
  }
}

// Issue the cp.async copies of chunk `c` (rows c*kRows ..) into `tile`.
// Pass Y: tile[r*32 + lane] = row r of column lane.  Pass X: the chunk holds
// x positions, transposed: tile[(x - r0)*33 + t] = element x of row t.
template <bool kXPass, int kRows>
__device__ __forceinline__ void stage_chunk(uint32_t* tile, const Sweep& s, int c, bool vec16) {
  const int lane = threadIdx.x & 31;
  const int r0 = c * kRows;
  const int rows = min(kRows, s.L - r0);
  if (!kXPass) {
    if (vec16) {  // one slice, 32 lanes, 16-byte aligned: 8 lanes per row
      const uint32_t* src = s.map + s.col0 + (uint64_t)r0 * s.X;
      const int part = lane & 7;
      if (rows == kRows) {  // a whole chunk: the copies unrolled
#pragma unroll
        for (int k = 0; k < kRows / 4; ++k) {
          const int r = (lane >> 3) + 4 * k;
          cp_async16(tile + r * 32 + part * 4, src + (uint64_t)r * s.X + part * 4);
        }
      } else {
        for (int r = lane >> 3; r < rows; r += 4) cp_async16(tile + r * 32 + part * 4, src + (uint64_t)r * s.X + part * 4);
      }
    } else if (lane < s.valid) {
      const uint32_t* src = s.map + s.col + (uint64_t)r0 * s.X;
      for (int r = 0; r < rows; ++r) cp_async4(tile + r * 32 + lane, src + (uint64_t)r * s.X);
    } else {
      for (int r = 0; r < rows; ++r) tile[r * 32 + lane] = kDvUninit;
    }
  } else {
    const int xl = lane % kRows;  // x within the chunk
    const int t0 = lane / kRows;
    if (s.one_slice) {  // rows t are X apart
      if (xl < rows) {
        const uint32_t* src = s.map + s.col0 + r0 + xl;
        if (s.valid == 32) {  // every column live: the copies unrolled
#pragma unroll
          for (int k = 0; k < kRows; ++k) {
            const int t = t0 + k * (32 / kRows);
            cp_async4(tile + xl * 33 + t, src + (uint64_t)t * s.X);
          }
        } else {
          for (int t = t0; t < 32; t += 32 / kRows) {
            if (t < s.valid) cp_async4(tile + xl * 33 + t, src + (uint64_t)t * s.X);
            else tile[xl * 33 + t] = kDvUninit;
          }
        }
      }
    } else {
      for (int t = t0; t < 32; t += 32 / kRows) {  // the same trip count on every lane (row_start shuffles)
        const uint32_t rs = row_start(s, t);
        if (xl < rows) {
          if (t < s.valid) cp_async4(tile + xl * 33 + t, s.map + rs + r0 + xl);
          else tile[xl * 33 + t] = kDvUninit;
        }
      }
    }
  }
}

// One warp item of pass Y (kXPass false) or X: 32 consecutive columns (see
// Sweep); wbase = the warp's kWarpWords of shared memory; stack = L * 64
// words of workspace: entry d of lane l is the pair (site, bisector with the
// entry below) at ((uint2*)stack)[l * L + d] -- each lane's stack contiguous,
// so its spills, refills and window reads fill whole sectors.  kOwnA: pass Z
// took the occupancy-bit route (make_col's kOwn).
template <bool kXPass, int kRows, bool kOwnA = false>
__device__ __forceinline__ void sweep_item(uint32_t* __restrict__ map, uint32_t* __restrict__ stack, int X, int Y,
                                           int Z, long long item, uint32_t* wbase) {
  using Cfg = SweepCfg<kRows>;
  const int lane = threadIdx.x & 31;
  const unsigned cols = kXPass ? Y : X;  // columns per slice
  const int L = kXPass ? X : Y;
  const unsigned total = cols * (unsigned)Z;  // below 2^30
  const unsigned f0 = (unsigned)item * 32u;
  Sweep s;
  s.L = L;
  s.X = X;
  s.map = map;
  s.valid = (int)min(32u, total - f0);
  {
    const unsigned f = min(f0 + (unsigned)lane, total - 1u);  // idle lanes mirror the last column
    s.z = (int)(f / cols);
    s.a = (int)(f - (unsigned)s.z * cols);
    const unsigned layer = (unsigned)X * (unsigned)Y;
    s.col = (unsigned)s.z * layer + (kXPass ? (unsigned)s.a * (unsigned)X : (unsigned)s.a);
    const unsigned z0 = f0 / cols;
    s.col0 = z0 * layer + (kXPass ? (f0 - z0 * cols) * (unsigned)X : f0 - z0 * cols);
    s.one_slice = (f0 + (unsigned)s.valid - 1u) / cols == z0;
  }
  // lane 0's column is a multiple of 4 when X is (f0 is a multiple of 32)
  const bool vec16 = !kXPass && s.one_slice && s.valid == 32 && (X & 3) == 0;
  uint32_t* tile0 = wbase;
  uint32_t* tile1 = wbase + Cfg::kTileWords;
  // the ring: slot k of this lane = (site, bisector) at ring[k * 32]
  uint2* ring = reinterpret_cast<uint2*>(wbase + 2 * Cfg::kTileWords) + lane;
  uint2* gstk = reinterpret_cast<uint2*>(stack) + (size_t)lane * L;  // this lane's stack, depth d: gstk[d]
  const float A0 = biased((uint32_t)s.a);  // this lane's column coordinate, biased
  const float C0 = biased((uint32_t)s.z);
  const int nchunks = (L + kRows - 1) / kRows;
  const int tpitch = kXPass ? 33 : 32;
  // Pops a lane runs alone per row before the warp takes over.  Pass Y (input:
  // the nearest site per z column) has rare, long pop runs; in pass X nearly
  // every row pushes and runs stay short, so there the warp never takes over
  // (0) -- measured faster at 512^3.
  constexpr int kSoloPops = kXPass ? 0 : 2;

  // ---- phase 2: proximate sites ------------------------------------------
  // Rows advance in lockstep (the per-row work runs on all 32 lanes); the pops
  // a row triggers run as a loop over just the lanes that need them.  The ring
  // keeps each entry's bisector with the entry below, so a pop reads the new
  // top's (site, bisector) pair instead of recomputing the bisector.
  stage_chunk<kXPass, kRows>(tile0, s, 0, vec16);
  cp_async_commit();
  if (nchunks > 1) stage_chunk<kXPass, kRows>(tile1, s, 1, vec16);
  cp_async_commit();

  // The stack lives in the ring (depths [lo, n)) and in the workspace
  // (depths [0, spill)); lo <= spill always (so a depth below the ring has its
  // workspace copy, and the eviction test needs only spill).  An entry
  // is written to the workspace only when a push evicts it from the ring (and
  // the ring's remainder once phase 2 ends), so entries pushed and popped
  // within the ring's reach never leave the chip.
  int n = 0;      // stack depth
  int lo = 0;     // lowest depth in the ring
  int spill = 0;  // depths below it have their workspace copy
  // The top decoded, with top_i = bisector(second, top); a pop reads the new
  // top (site, bisector) from the ring, or below the ring from the workspace.
  Col top{0u, 0.f, 0.f};
  float top_i = 0.f;
  for (int c = 0; c < nchunks; ++c) {
    cp_async_wait1();
    __syncwarp();
    const uint32_t* tile = (c & 1) ? tile1 : tile0;
    const int r0 = c * kRows;
    const int rows = min(kRows, L - r0);
    float row2f = small_to_float(2 * r0);  // 2 * row, exact
    for (int r = 0; r < rows; ++r, row2f += 2.0f) {
      const uint32_t v = tile[r * tpitch + lane];
      const uint32_t a = kXPass ? ((v >> 10) & 0x3ffu) : (v & 0x3ffu);
      const bool has = a != kUninit;
      Col cur;
      cur.e = kOwnA ? v : (a | ((uint32_t)(r0 + r) << 10) | (v & 0xFFF00000u));
      cur.r2 = row2f;
      {
        if (!kXPass && kOwnA) {
          const float dc = biased(v >> 20) - C0;
          cur.d = __fmul_rn(dc, dc);
        } else {
          const float2 dd = sub2(make_float2(biased(a), biased(v >> 20)), make_float2(A0, C0));
          cur.d = __fmaf_rn(dd.x, dd.x, __fmul_rn(dd.y, dd.y));
        }
      }
      // Before a row's pops the top is the site of the last earlier row that
      // had one, so this bisector does not wait for the pops of earlier rows;
      // computed for every lane (used only when the stack is not empty).
      float i2 = bisect(top, cur);
      {
        bool deep = false;
        if (has) {
          for (int p = 0; n >= 2 && !(top_i < i2); ++p) {  // top is dominated by (second, current): pop
            if (kSoloPops > 0 && p == kSoloPops) {
              deep = true;
              break;
            }
            --n;
            // the new top: its ring slot, or below the ring the workspace (a
            // predicated load; no divergent branch)
            const int d = n - 1;
            uint2 q = ring[(d & (Cfg::kRing - 1)) * 32];
            if (d < lo) q = gstk[d];
            top = make_col<kXPass, kOwnA>(q.x, A0, C0);
            top_i = __uint_as_float(q.y);
            i2 = bisect(top, cur);
          }
        }
        // Long pop runs: the warp tests 31 entries of one lane's stack per round.
        if constexpr (kSoloPops > 0) {
          unsigned deep_lanes = __ballot_sync(kFullMask, deep);
          if (deep_lanes) __syncwarp();  // the owners' ring and workspace writes
          while (deep_lanes) {
            const int o = __ffs(deep_lanes) - 1;
            deep_lanes &= deep_lanes - 1;
            coop_pops<Cfg, kOwnA>(o, A0, C0, reinterpret_cast<uint2*>(wbase + 2 * Cfg::kTileWords),
                                  gstk - (size_t)lane * L, L, n, lo, cur, top, top_i, i2);
          }
        }
        if (has) {
          // (the bottom entry's bisector is never read: phase 2 pops need two
          // entries, phase 3 and the warp pops never test depth 0)
          spill = min(spill, n);  // workspace copies at or above n are stale
          lo = min(lo, n);
          const int slot = (n & (Cfg::kRing - 1)) * 32;  // push the current site
          const int ev = n - Cfg::kRing;             // the depth this slot held
          if (ev >= spill) {  // evicted before it reached the workspace (spill >= lo always)
            gstk[ev] = ring[slot];
            spill = ev + 1;
          }
          ring[slot] = make_uint2(cur.e, __float_as_uint(i2));
          lo = max(lo, ev + 1);
          ++n;
          top = cur;
          top_i = i2;
        }
      }
    }
    __syncwarp();
    if (c + 2 < nchunks) stage_chunk<kXPass, kRows>((c & 1) ? tile1 : tile0, s, c + 2, vec16);
    cp_async_commit();
  }
  // the ring's entries that never reached the workspace
  spill = min(spill, n);
  for (int d = spill; d < n; ++d) gstk[d] = ring[(d & (Cfg::kRing - 1)) * 32];
  cp_async_wait_all();
  __syncwarp();

  // ---- phase 3: rows downward, popping sites that fall behind ----
  // Each stack entry carries its bisector with the entry below, so a pop is
  // one read.  The stack streams back from the workspace through a kWin-entry
  // window per lane (slot = depth mod kWin).  At each chunk start every lane
  // requests the entries down to kWin below its top (cp.async), so the pops
  // of the following chunks find them on chip; a lane that pops past what
  // has landed waits for its request or reads the workspace directly.
  constexpr int kWin = Cfg::kWin;
  constexpr int kP3Rows = kXPass ? Cfg::kStageRows : kRows;
  uint32_t* xstage = wbase;  // pass X: kStageRows x kStagePitch
  uint2* win = reinterpret_cast<uint2*>(wbase + (kXPass ? Cfg::kStageWords : 0)) + lane;  // depth d: win[(d % kWin) * 32]
  int k = n - 1;    // index of the current top
  int flo = n;      // lowest depth requested into the window
  int safe_lo = n;  // depths >= safe_lo have landed
  // Copy depths [new_lo, hi) into the window.  hi never exceeds the lowest
  // depth already requested nor, after the first request, the top (depths
  // at or above it are dead); requests are waited for before the next one,
  // so one request spans at most kWin depths and no two copies in flight
  // target the same slot.
  auto request = [&](int hi, int new_lo) {
    for (int d = hi - 1; d >= new_lo; --d) cp_async8(win + (d & (kWin - 1)) * 32, gstk + d);
    cp_async_commit();
    flo = min(flo, new_lo);
  };
  auto entry = [&](int d) -> uint2 {
    if (d < safe_lo) {
      cp_async_wait_all();
      safe_lo = flo;
      if (d < flo) return gstk[d];
    }
    return win[(d & (kWin - 1)) * 32];
  };
  // The voxel value a top entry gives, in map order (pass X in its general
  // form swaps the entry's first two fields back).
  auto out_of = [](uint32_t te) -> uint32_t {
    return (kXPass && !kOwnA) ? (((te >> 10) & 0x3ffu) | ((te & 0x3ffu) << 10) | (te & 0xFFF00000u)) : te;
  };
  uint32_t out = kDvUninit;
  float top_b = 0.f;  // bisector of the top with the entry below
  if (n > 0) {
    request(n, max(0, n - kWin));
    cp_async_wait_all();
    safe_lo = flo;
    const uint2 t = entry(k);
    out = out_of(t.x);
    top_b = __uint_as_float(t.y);
  }
  uint32_t* col_out = map + s.col;  // pass Y: this lane's column, row stride X
  const bool live = lane < s.valid;
  for (int c = (L + kP3Rows - 1) / kP3Rows - 1; c >= 0; --c) {
    const int r0 = c * kP3Rows;
    const int rows = min(kP3Rows, L - r0);
    cp_async_wait_all();  // the previous chunk's request
    safe_lo = flo;
    if (k >= 1) request(min(flo, k), max(0, k - kWin));
    float tyf = small_to_float(r0 + rows - 1);
#pragma unroll 4  // fewer loop-carried moves and branches (measured 1.88 -> 1.87 ms at 512^3)
    for (int r = rows - 1; r >= 0; --r, tyf -= 1.0f) {
      while (k >= 1 && tyf <= top_b) {  // pop
        --k;
        const uint2 t = entry(k);
        out = out_of(t.x);
        top_b = __uint_as_float(t.y);
      }
      if (kXPass) xstage[r * Cfg::kStagePitch + lane] = out;
      else if (live) col_out[(uint64_t)(r0 + r) * X] = out;
    }
    if (kXPass) {  // transposed flush: 4 rows of the map x 8 consecutive x per store
      __syncwarp();
      const int xl = lane >> 2, t0 = lane & 3;
      if (s.one_slice) {  // rows t are X apart
        if (xl < rows) {
          uint32_t* dst = map + (uint64_t)s.col0 + r0 + xl;
          if (s.valid == 32) {
#pragma unroll
            for (int k = 0; k < 8; ++k) dst[(uint64_t)(t0 + 4 * k) * X] = xstage[xl * Cfg::kStagePitch + t0 + 4 * k];
          } else {
            for (int t = t0; t < s.valid; t += 4) dst[(uint64_t)t * X] = xstage[xl * Cfg::kStagePitch + t];
          }
        }
      } else {
        for (int t = t0; t < 32; t += 4) {  // the same trip count on every lane (row_start shuffles)
          const uint32_t rs = row_start(s, t);
          if (xl < rows && t < s.valid) map[(uint64_t)rs + r0 + xl] = xstage[xl * Cfg::kStagePitch + t];
        }
      }
      __syncwarp();
    }
  }
  cp_async_wait_all();
}

// A map's other-sites flag in a batch: word Z + 2 of its workspace, as for one map.
__device__ __forceinline__ uint32_t* batch_other(const BatchMap& m) { return m.scratch + m.Z + 2; }

// Map owning warp item g of a batch pass: last k with prefix[k] <= g.
__device__ __forceinline__ uint32_t batch_owner(const long long* __restrict__ prefix, uint32_t n, long long g) {
  uint32_t lo = 0, hi = n;
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (__ldg(prefix + mid) <= g) lo = mid; else hi = mid;
  }
  return lo;
}

// carries: the map's workspace past its counters (zcarry_item_words per item)
// run_if (optional): runs only when this flag is set (occ_from_map_kernel).
__global__ void __launch_bounds__(kZWarps * 32, 3) edt_pass_z(uint32_t* __restrict__ map, uint32_t* __restrict__ carries,
                                                               int X, int Y, int Z, const uint32_t* __restrict__ run_if) {
  extern __shared__ __align__(16) uint32_t s_z[];  // [kZWarps][kZWarpWords]
  if (run_if != nullptr && *run_if == 0u) return;
  const int warp = threadIdx.x >> 5;
  const long long item = (long long)blockIdx.x * kZWarps + warp;
  if (item >= (long long)z_items(X, Y)) return;
  pass_z_item(map, X, Y, Z, item, s_z + (size_t)warp * kZWarpWords, carries + (uint64_t)item * zcarry_item_words(Z));
}

// Pass Z over every map of a batch: persistent warps stride over the items of
// all maps.
__global__ void __launch_bounds__(kZWarps * 32, 3) edt_pass_z_batch(const BatchMap* __restrict__ maps,
                                                                     const long long* __restrict__ prefix,
                                                                     uint32_t n_maps, long long total) {
  extern __shared__ __align__(16) uint32_t s_z[];
  const int warp = threadIdx.x >> 5;
  for (long long g = (long long)blockIdx.x * kZWarps + warp; g < total; g += (long long)gridDim.x * kZWarps) {
    const uint32_t k = batch_owner(prefix, n_maps, g);
    const BatchMap m = maps[k];
    if (*batch_other(m) == 0u) continue;  // the bits pass took this map
    const long long item = g - __ldg(prefix + k);
    pass_z_item(m.vox, m.X, m.Y, m.Z, item, s_z + (size_t)warp * kZWarpWords,
                m.scratch + edt_sync_words(m.Z) + (uint64_t)item * zcarry_item_words(m.Z));
    __syncwarp();
  }
}

// Words of stack one warp needs for a map (a pair per row per lane).
__host__ __device__ __forceinline__ uint64_t warp_stack_words(int X, int Y) { return (uint64_t)max(X, Y) * 64; }

// The fused voxelisation for every map of a batch: each map's occupancy
// bits sit in its own workspace past the counters.
__device__ __forceinline__ uint32_t* batch_occ(const BatchMap& m) { return m.scratch + edt_sync_words(m.Z); }

__global__ void occ_clear_batch_kernel(const BatchMap* __restrict__ maps) {
  const BatchMap m = maps[blockIdx.y];
  if (blockIdx.x == 0 && threadIdx.x == 0) *batch_other(m) = 0u;  // every site will be its own
  uint32_t* bits = batch_occ(m);
  const uint64_t n = occ_words(m.X, m.Y, m.Z);
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    bits[i] = 0u;
}

// point i belongs to map k with offsets[k] <= i < offsets[k + 1]
__global__ void occ_insert_batch_kernel(const BatchMap* __restrict__ maps, uint32_t n_maps, const float* __restrict__ xyz,
                                        const uint64_t* __restrict__ offsets, uint64_t n) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    uint32_t lo = 0, hi = n_maps;
    while (hi - lo > 1) {
      const uint32_t mid = (lo + hi) >> 1;
      if (__ldg(offsets + mid) <= i) lo = mid; else hi = mid;
    }
    const BatchMap m = maps[lo];
    const uint32_t x = coord_to_voxel(__ldg(xyz + 3 * i), m.side), y = coord_to_voxel(__ldg(xyz + 3 * i + 1), m.side),
                   z = coord_to_voxel(__ldg(xyz + 3 * i + 2), m.side);
    if (x < (uint32_t)m.X && y < (uint32_t)m.Y && z < (uint32_t)m.Z) occ_set(batch_occ(m), m.X, m.Z, x, y, z);
  }
}

// Occupancy bits of a filled map for the bits pass Z.  After clearMap and
// insertPointCloud every voxel is UNINIT or holds its own coordinates, and
// kernelPBAphase1FloodZ (GV/voxelmap/kernels/VoxelMapOperationsPBA.hpp:63-124)
// then depends only on which voxels are sites.  A voxel holding any other
// site (a map transformed before, sites moved by mergeOccupied's offset,
// caller-written data) sets *other_sites, and the general pass Z runs instead.
// One warp task = one item (32 columns) x 32 rows.  Lane L reads columns
// 4 * (L & 7) .. + 3 of rows zc + (L >> 3) + 4 j, j = 0..7 (one 16-byte load
// each when vec), so a load instruction covers 4 whole rows of the item; the
// 8 lanes of a row OR their 4-bit pieces into the row's occupancy word
// (bit k = column k) with three xor shuffles, and lane L stores the word of
// row (L >> 3) + 4 (L & 7): the warp's 32 words as one 128-byte store.
// Consecutive warps take consecutive items of the same rows.  vec: map and
// rows 16-byte aligned.
// One task of occ_from_map: returns whether this lane saw another site.
__device__ __forceinline__ bool occ_from_map_task(const uint32_t* __restrict__ map, uint32_t* __restrict__ bits, int X,
                                                  int Y, int Z, long long t, long long items, bool vec) {
  const int lane = threadIdx.x & 31;
  const int g = lane >> 3, q = lane & 7;
  const uint32_t layer = (uint32_t)X * (uint32_t)Y;
  const bool x_aligned = (X & 31) == 0;  // an item's 32 columns lie in one y row
  bool other = false;
  {
    const int chunk = (int)(t / items);
    const uint32_t item = (uint32_t)(t - (long long)chunk * items);
    const int zc = chunk * 32;
    const uint32_t f = item * 32u + 4u * (uint32_t)q;  // this lane's first column
    const int ncols = (int)min(32u, layer - item * 32u);
    const uint32_t y0 = f / (uint32_t)X, x0 = f - y0 * (uint32_t)X;  // f < layer when 4q < ncols
    // all eight row pieces in flight before any is used
    uint32_t vv[8][4];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int z = zc + g + 4 * j;
#pragma unroll
      for (int i = 0; i < 4; ++i) vv[j][i] = kDvUninit;
      if (z < Z) {
        const uint32_t* row = map + (uint64_t)z * layer + f;
        if (vec && ncols == 32) {
          const uint4 w = __ldg(reinterpret_cast<const uint4*>(row));
          vv[j][0] = w.x;
          vv[j][1] = w.y;
          vv[j][2] = w.z;
          vv[j][3] = w.w;
        } else {
#pragma unroll
          for (int i = 0; i < 4; ++i)
            if (4 * q + i < ncols) vv[j][i] = __ldg(row + i);
        }
      }
    }
    uint32_t word = 0u;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int z = zc + g + 4 * j;
      const uint32_t* v = vv[j];
      uint32_t piece = 0u;
      if (x_aligned) {
        const uint32_t c0 = (x0 | (y0 << 10)) + ((uint32_t)z << 20);
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          piece |= (uint32_t)(v[i] != kDvUninit) << i;
          other |= v[i] != kDvUninit && v[i] != c0 + (uint32_t)i;
        }
      } else {
        uint32_t x = x0, y = y0;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          piece |= (uint32_t)(v[i] != kDvUninit) << i;
          other |= v[i] != kDvUninit && v[i] != (x | (y << 10) | ((uint32_t)z << 20));
          if (++x == (uint32_t)X) {
            x = 0u;
            ++y;
          }
        }
      }
      uint32_t rw = piece << (4 * q);
      rw |= __shfl_xor_sync(kFullMask, rw, 1);
      rw |= __shfl_xor_sync(kFullMask, rw, 2);
      rw |= __shfl_xor_sync(kFullMask, rw, 4);
      if (j == q) word = rw;  // row g + 4 q
    }
    const int zs = zc + g + 4 * q;
    if (zs < Z) bits[(uint64_t)item * Z + zs] = word;
  }
  return other;
}

__global__ void __launch_bounds__(256) occ_from_map_kernel(const uint32_t* __restrict__ map, uint32_t* __restrict__ bits,
                                                           int X, int Y, int Z, uint32_t* __restrict__ other_sites,
                                                           int vec) {
  const long long items = (long long)z_items(X, Y);
  const long long tasks = items * ((Z + 31) >> 5);
  const long long warps = ((long long)gridDim.x * blockDim.x) >> 5;
  bool other = false;
  for (long long t = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < tasks; t += warps)
    other |= occ_from_map_task(map, bits, X, Y, Z, t, items, vec != 0);
  if (__any_sync(kFullMask, other) && (threadIdx.x & 31) == 0) atomicOr(other_sites, 1u);
}

// The same over every map of a batch: map k owns tasks [prefix[k],
// prefix[k+1]); its bits go to its own workspace past the counters, its
// other-sites flag to word Z + 2 of its workspace (cleared by
// batch_flags_clear_kernel before).
__global__ void __launch_bounds__(256) occ_from_map_batch_kernel(const BatchMap* __restrict__ maps,
                                                                 const long long* __restrict__ prefix,
                                                                 uint32_t n_maps, long long total) {
  const long long warps = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long g = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; g < total; g += warps) {
    const uint32_t k = batch_owner(prefix, n_maps, g);
    const BatchMap m = maps[k];
    const bool vec = (reinterpret_cast<uintptr_t>(m.vox) & 15u) == 0 && ((uint64_t)m.X * m.Y) % 4 == 0;
    const bool other =
        occ_from_map_task(m.vox, batch_occ(m), m.X, m.Y, m.Z, g - __ldg(prefix + k), (long long)z_items(m.X, m.Y), vec);
    if (__any_sync(kFullMask, other) && (threadIdx.x & 31) == 0) atomicOr(batch_other(m), 1u);
  }
}

__global__ void batch_flags_clear_kernel(const BatchMap* __restrict__ maps, uint32_t n_maps) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n_maps) *batch_other(maps[k]) = 0u;
}

__global__ void __launch_bounds__(kZWarps * 32) edt_pass_z_bits_batch(const BatchMap* __restrict__ maps,
                                                                       const long long* __restrict__ prefix,
                                                                       uint32_t n_maps, long long total, int zw,
                                                                       int skip_other) {
  extern __shared__ __align__(16) uint32_t s_z[];  // [kZWarps][2 * zw]
  const int warp = threadIdx.x >> 5;
  for (long long g = (long long)blockIdx.x * kZWarps + warp; g < total; g += (long long)gridDim.x * kZWarps) {
    const uint32_t k = batch_owner(prefix, n_maps, g);
    const BatchMap m = maps[k];
    if (skip_other && *batch_other(m) != 0u) continue;  // the general pass takes this map
    pass_z_bits_item(m.vox, batch_occ(m), m.X, m.Y, m.Z, g - __ldg(prefix + k), s_z + (size_t)warp * 2 * zw, zw);
    __syncwarp();
  }
}

// One pass (Y or X) on its own (per-pass timing and the fallback of the fused
// schedule below): persistent warps stride over the items, one stack each.
template <bool kXPass, int kRows>
__global__ void __launch_bounds__(SweepCfg<kRows>::kWarps * 32, 3)
    edt_sweep(uint32_t* __restrict__ map, uint32_t* __restrict__ stacks, int X, int Y, int Z) {
  using Cfg = SweepCfg<kRows>;
  extern __shared__ __align__(16) uint32_t s_sweep[];  // [kWarps][kWarpWords]
  const int warp = threadIdx.x >> 5;
  const long long gw = (long long)blockIdx.x * Cfg::kWarps + warp;
  uint32_t* stack = stacks + (uint64_t)gw * warp_stack_words(X, Y);
  const long long items = ((long long)(kXPass ? Y : X) * Z + 31) / 32;
  for (long long item = gw; item < items; item += (long long)gridDim.x * Cfg::kWarps) {
    sweep_item<kXPass, kRows>(map, stack, X, Y, Z, item, s_sweep + (size_t)warp * Cfg::kWarpWords);
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------
// Fused Y -> X schedule.  Pass X on slice z reads only what pass Y wrote to
// slice z, so one persistent launch runs both: warps take items from a queue
// (all Y items in z order, then all X items in z order), a Y item bumps the
// completion counter of each slice it touches, and an X item first waits
// until each of its slices counts all the Y items touching it.  Every item a
// wait depends on
// sits earlier in the queue and was taken by a running warp that waits on
// nothing, so the waits end; they are bounded all the same (kSpinLimit
// sleeps, then the error word is set and the item is skipped).  The tail of
// pass Y overlaps the start of pass X, and no warp idles while its block's
// other warps finish.  Stacks are per resident warp (a warp's items run one
// after the other).
// ---------------------------------------------------------------------------
constexpr unsigned kSpinLimit = 1u << 24;  // x ~128 ns sleeps: seconds

__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Slices za..zb that item g of a pass with `cols` columns per slice touches
// (at most 32: an item is 32 consecutive columns).
__device__ __forceinline__ void item_slices(unsigned g, unsigned cols, unsigned Z, unsigned& za, unsigned& zb) {
  const unsigned f0 = g * 32u;
  za = f0 / cols;
  zb = min(f0 + 31u, cols * Z - 1u) / cols;
}

// Y items that touch slice z (its columns z*X .. z*X + X - 1).
__device__ __forceinline__ unsigned y_items_of_slice(unsigned z, unsigned X) {
  return ((z + 1u) * X - 1u) / 32u - (z * X) / 32u + 1u;
}

// After a Y item: its output stores, then the counter of every slice it
// touched (lane j bumps slice za + j).
__device__ __forceinline__ void publish_slices(unsigned* done, unsigned za, unsigned zb) {
  __threadfence();
  __syncwarp();
  const unsigned lane = threadIdx.x & 31;
  if (lane <= zb - za) {
    __threadfence();
    atomicAdd(done + za + lane, 1u);
  }
}

// Before an X item: wait (bounded) until every slice it reads has all its Y
// items done (lane j waits for slice za + j).
__device__ __forceinline__ bool wait_slices(const unsigned* done, unsigned za, unsigned zb, unsigned X, unsigned* err) {
  const unsigned lane = threadIdx.x & 31;
  int ok = 1;
  if (lane <= zb - za) {
    const unsigned need = y_items_of_slice(za + lane, X);
    unsigned spins = 0;
    while (ld_acquire_gpu(done + za + lane) < need) {
      if (++spins > kSpinLimit) {
        atomicOr(err, 1u);
        ok = 0;
        break;
      }
      __nanosleep(128);
    }
  }
  __syncwarp();  // orders the waiting lanes' acquires before every lane's loads
  ok = __all_sync(kFullMask, ok);
  __threadfence();
  return ok != 0;
}

__device__ __forceinline__ unsigned next_item(unsigned* head) {
  unsigned g = 0;
  if ((threadIdx.x & 31) == 0) g = atomicAdd(head, 1u);
  return __shfl_sync(kFullMask, g, 0);
}

// sync = [done: Z words][head][err][pass Z's other-sites flag]; done, head
// and err zeroed before the launch.  A zero flag means every site lies in its
// own z column, and both passes take the map's entries as stack entries
// (sweep_item's kOwnA).
template <int kRows>
__global__ void __launch_bounds__(SweepCfg<kRows>::kWarps * 32, 3)
    edt_sweep_yx(uint32_t* __restrict__ map, uint32_t* __restrict__ stacks, unsigned* __restrict__ sync, int X, int Y,
                 int Z) {
  using Cfg = SweepCfg<kRows>;
  extern __shared__ __align__(16) uint32_t s_sweep[];
  const int warp = threadIdx.x >> 5;
  uint32_t* wbase = s_sweep + (size_t)warp * Cfg::kWarpWords;
  uint32_t* stack = stacks + ((uint64_t)blockIdx.x * Cfg::kWarps + warp) * warp_stack_words(X, Y);
  unsigned* done = sync;
  unsigned* head = sync + Z;
  unsigned* err = head + 1;
  const bool own = sync[Z + 2] == 0u;
  const unsigned ny = ((unsigned)X * Z + 31u) / 32u, nall = ny + ((unsigned)Y * Z + 31u) / 32u;
  for (unsigned g = next_item(head); g < nall; g = next_item(head)) {
    unsigned za, zb;
    if (g < ny) {
      if (own) sweep_item<false, kRows, true>(map, stack, X, Y, Z, g, wbase);
      else sweep_item<false, kRows, false>(map, stack, X, Y, Z, g, wbase);
      item_slices(g, X, Z, za, zb);
      publish_slices(done, za, zb);
    } else {
      const unsigned item = g - ny;
      item_slices(item, Y, Z, za, zb);
      if (wait_slices(done, za, zb, X, err)) {
        if (own) sweep_item<true, kRows, true>(map, stack, X, Y, Z, item, wbase);
        else sweep_item<true, kRows, false>(map, stack, X, Y, Z, item, wbase);
      }
    }
    __syncwarp();
  }
}

// The same schedule over every map of a batch: the queue holds all maps' Y
// items, then all maps' X items.  maps[k].sync_off locates map k's slice
// counters in `sync`; the queue head and error word follow them.  Both passes
// of a map whose pass Z took the occupancy-bit route (its other-sites flag
// clear) run sweep_item's kOwnA form.
template <int kRows>
__global__ void __launch_bounds__(SweepCfg<kRows>::kWarps * 32, 3)
    edt_sweep_yx_batch(const BatchMap* __restrict__ maps, const long long* __restrict__ prefix_y,
                       const long long* __restrict__ prefix_x, uint32_t n_maps, unsigned total_y, unsigned total_x,
                       uint32_t* __restrict__ stacks, uint32_t stack_len, unsigned* __restrict__ sync,
                       unsigned sync_words) {
  using Cfg = SweepCfg<kRows>;
  extern __shared__ __align__(16) uint32_t s_sweep[];
  const int warp = threadIdx.x >> 5;
  uint32_t* wbase = s_sweep + (size_t)warp * Cfg::kWarpWords;
  uint32_t* stack = stacks + ((uint64_t)blockIdx.x * Cfg::kWarps + warp) * (uint64_t)stack_len * 64;
  unsigned* head = sync + sync_words;
  unsigned* err = head + 1;
  const unsigned nall = total_y + total_x;
  for (unsigned g = next_item(head); g < nall; g = next_item(head)) {
    const bool x_item = g >= total_y;
    const long long q = x_item ? (long long)(g - total_y) : (long long)g;
    const long long* prefix = x_item ? prefix_x : prefix_y;
    const uint32_t k = batch_owner(prefix, n_maps, q);
    const BatchMap m = maps[k];
    const unsigned item = (unsigned)(q - __ldg(prefix + k));
    unsigned* done = sync + m.sync_off;
    unsigned za, zb;
    if (!x_item) {
      if (*batch_other(m) == 0u) sweep_item<false, kRows, true>(m.vox, stack, m.X, m.Y, m.Z, item, wbase);
      else sweep_item<false, kRows, false>(m.vox, stack, m.X, m.Y, m.Z, item, wbase);
      item_slices(item, m.X, m.Z, za, zb);
      publish_slices(done, za, zb);
    } else {
      item_slices(item, m.Y, m.Z, za, zb);
      if (wait_slices(done, za, zb, m.X, err)) {
        if (*batch_other(m) == 0u) sweep_item<true, kRows, true>(m.vox, stack, m.X, m.Y, m.Z, item, wbase);
        else sweep_item<true, kRows, false>(m.vox, stack, m.X, m.Y, m.Z, item, wbase);
      }
    }
    __syncwarp();
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

// Per-kernel launch set-up, done once per device: the dynamic shared memory
// attribute and the number of resident blocks on the whole device (the
// queries cost microseconds, which small maps would pay on every call).
constexpr int kMaxDevices = 64;
struct KernelSetup {
  std::once_flag once[kMaxDevices];
  cudaError_t err[kMaxDevices] = {};
  long long blocks[kMaxDevices] = {};
};

template <auto kKernel>
cudaError_t kernel_setup(int threads, int smem, long long* resident) {
  static KernelSetup st;  // one per kernel
  const auto kern = kKernel;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::call_once(st.once[dev], [&] {
    cudaError_t r = smem > max_smem_optin() ? cudaErrorInvalidConfiguration : cudaSuccess;
    if (r == cudaSuccess) r = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (r == cudaSuccess)
      r = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
    int per_sm = 0, sm = 0;
    if (r == cudaSuccess) r = cudaDeviceGetAttribute(&sm, cudaDevAttrMultiProcessorCount, dev);
    if (r == cudaSuccess) r = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem);
    st.err[dev] = r;
    st.blocks[dev] = (long long)std::max(per_sm, 1) * std::max(sm, 1);
  });
  if (resident) *resident = st.blocks[dev];
  return st.err[dev];
}

// Pass Z of a filled map: occupancy bits from the map, then the bits pass;
// when some voxel holds another site than its own, the bits pass skips and
// the general pass runs (both are launched; the flag picks on the device).
// The bits and the general pass's chunk carries share the workspace area
// after the counters.
cudaError_t launch_pass_z(uint32_t* map, uint32_t* scratch, gvx_dims d, cudaStream_t s) {
  const int X = (int)d.x, Y = (int)d.y, Z = (int)d.z;
  uint32_t* other = scratch + (uint64_t)Z + 2;
  uint32_t* area = scratch + edt_sync_words(Z);
  cudaError_t e = cudaMemsetAsync(other, 0, sizeof(uint32_t), s);
  if (e != cudaSuccess) return e;
  int dev = 0, sm = 0;
  if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
  if ((e = cudaDeviceGetAttribute(&sm, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
  int per_sm = 0;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, occ_from_map_kernel, 256, 0)) != cudaSuccess) return e;
  const long long tasks = (long long)z_items(X, Y) * ((Z + 31) >> 5);  // one per warp, 8 warps per block
  const long long occ_blocks =
      std::max<long long>(1, std::min<long long>((tasks + 7) / 8, (long long)std::max(sm, 1) * std::max(per_sm, 1)));
  const int vec = ((reinterpret_cast<uintptr_t>(map) & 15u) == 0 && ((uint64_t)X * Y) % 4 == 0) ? 1 : 0;
  occ_from_map_kernel<<<(unsigned)occ_blocks, 256, 0, s>>>(map, area, X, Y, Z, other, vec);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  const long long items = (long long)z_items(X, Y);
  const unsigned z_blocks = (unsigned)((items + kZWarps - 1) / kZWarps);
  if ((e = kernel_setup<edt_pass_z_bits>(kZWarps * 32, kZBitsSmemMax, nullptr)) != cudaSuccess) return e;
  edt_pass_z_bits<<<z_blocks, kZWarps * 32, kZWarps * 2 * z_bits_words(Z) * 4, s>>>(map, area, X, Y, Z, other);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  const int smem = kZWarps * kZWarpWords * 4;
  if ((e = kernel_setup<edt_pass_z>(kZWarps * 32, smem, nullptr)) != cudaSuccess) return e;
  edt_pass_z<<<z_blocks, kZWarps * 32, smem, s>>>(map, area, X, Y, Z, other);
  return cudaGetLastError();
}

// Workspace layout: [slice counters, queue head, error word: sync_words(d)]
// [stack area: one stack of warp_stack_words per launched warp; before the
// sweeps, pass Z keeps its chunk carries there].
uint64_t sync_words(gvx_dims d) { return edt_sync_words((int)d.z); }
uint64_t zcarry_words(gvx_dims d) { return z_items((int)d.x, (int)d.y) * zcarry_item_words((int)d.z); }

// Blocks for a persistent sweep launch: resident, fitting the stack area, and
// no more than the items need (0 when the area holds no block's stacks).
long long sweep_blocks(long long resident, uint64_t stack_area, gvx_dims d, int warps, long long items) {
  const uint64_t per_block = (uint64_t)warps * warp_stack_words((int)d.x, (int)d.y);
  return std::min<long long>({resident, (long long)(stack_area / per_block), (items + warps - 1) / warps});
}

template <bool kXPass, int kRows>
cudaError_t launch_sweep(uint32_t* map, uint32_t* scratch, uint64_t scratch_words, gvx_dims d, cudaStream_t s) {
  using Cfg = SweepCfg<kRows>;
  const long long items = edt_pass_items(d, kXPass ? 2 : 1);
  const int smem = Cfg::kWarps * Cfg::kWarpWords * 4;
  long long blocks = 0;
  cudaError_t e = kernel_setup<edt_sweep<kXPass, kRows>>(Cfg::kWarps * 32, smem, &blocks);
  if (e != cudaSuccess) return e;
  blocks = sweep_blocks(blocks, scratch_words - sync_words(d), d, Cfg::kWarps, items);
  if (blocks < 1) return cudaErrorInvalidValue;
  edt_sweep<kXPass, kRows><<<(unsigned)blocks, Cfg::kWarps * 32, smem, s>>>(map, scratch + sync_words(d), (int)d.x,
                                                                             (int)d.y, (int)d.z);
  return cudaGetLastError();
}

// Stack area that lets the fused launch run one warp per item, up to
// kFusedWarpCap warps (more than a B200 keeps resident).
constexpr uint64_t kFusedWarpCap = 4096;
uint64_t fused_stack_words(gvx_dims d) {
  const uint64_t items = (uint64_t)(edt_pass_items(d, 1) + edt_pass_items(d, 2));
  const uint64_t warps = std::min<uint64_t>((items + 7) / 8 * 8, kFusedWarpCap);
  return warps * warp_stack_words((int)d.x, (int)d.y);
}

// Fused Y -> X launch for one map: as many blocks as are resident, as the
// stack area holds and as there are items.
template <int kRows>
cudaError_t launch_sweep_yx(uint32_t* map, uint32_t* scratch, uint64_t scratch_words, gvx_dims d, cudaStream_t s) {
  using Cfg = SweepCfg<kRows>;
  const int smem = Cfg::kWarps * Cfg::kWarpWords * 4;
  long long blocks = 0;
  cudaError_t e = kernel_setup<edt_sweep_yx<kRows>>(Cfg::kWarps * 32, smem, &blocks);
  if (e != cudaSuccess) return e;
  const long long items = edt_pass_items(d, 1) + edt_pass_items(d, 2);
  blocks = sweep_blocks(blocks, scratch_words - sync_words(d), d, Cfg::kWarps, items);
  if (blocks < 1) return cudaErrorInvalidValue;
  unsigned* sync = scratch;
  e = cudaMemsetAsync(sync, 0, (d.z + 2) * sizeof(unsigned), s);
  if (e != cudaSuccess) return e;
  edt_sweep_yx<kRows><<<(unsigned)blocks, Cfg::kWarps * 32, smem, s>>>(map, scratch + sync_words(d), sync, (int)d.x,
                                                                       (int)d.y, (int)d.z);
  return cudaGetLastError();
}

// Rows per staging chunk of the sweeps: 16 unless the environment variable
// GVX_EDT_SWEEP_ROWS or set_edt_sweep_rows picks 32.
int g_sweep_rows = -1;

int sweep_rows() {
  if (g_sweep_rows < 0) {
    const char* env = getenv("GVX_EDT_SWEEP_ROWS");
    g_sweep_rows = (env && atoi(env) == 32) ? 32 : 16;
  }
  return g_sweep_rows;
}

template <int kRows>
cudaError_t launch_yx_batch(const BatchMap* d_table, const BatchItems& it, cudaStream_t s) {
  using Cfg = SweepCfg<kRows>;
  const int smem = Cfg::kWarps * Cfg::kWarpWords * 4;
  auto kern = edt_sweep_yx_batch<kRows>;
  long long blocks = 0;
  cudaError_t e = kernel_setup<edt_sweep_yx_batch<kRows>>(Cfg::kWarps * 32, smem, &blocks);
  if (e != cudaSuccess) return e;
  blocks = std::min<long long>(blocks, it.stack_warps / Cfg::kWarps);
  blocks = std::min<long long>(blocks, (it.total[1] + it.total[2] + Cfg::kWarps - 1) / Cfg::kWarps);
  if (blocks < 1) return cudaErrorInvalidConfiguration;
  e = cudaMemsetAsync(it.d_sync, 0, (it.sync_words + 2) * sizeof(unsigned), s);
  if (e != cudaSuccess) return e;
  kern<<<(unsigned)blocks, Cfg::kWarps * 32, smem, s>>>(d_table, it.d_prefix[1], it.d_prefix[2], it.n_maps,
                                                        (unsigned)it.total[1], (unsigned)it.total[2], it.d_stacks,
                                                        it.stack_len, it.d_sync, it.sync_words);
  return cudaGetLastError();
}

template <int kRows>
long long batch_stack_warps() {
  using Cfg = SweepCfg<kRows>;
  const int smem = Cfg::kWarps * Cfg::kWarpWords * 4;
  long long blocks = 0;
  if (kernel_setup<edt_sweep_yx_batch<kRows>>(Cfg::kWarps * 32, smem, &blocks) != cudaSuccess) return -1;
  return blocks * Cfg::kWarps;
}

// Every (num, den) of the bisector domain: den = 2 * (blockIdx.y + 1), num
// over (-2^21, 2^21); counts quotients whose bits differ from the IEEE divide.
__global__ void quotient_check_kernel(unsigned long long* __restrict__ mismatches) {
  const float den = (float)(2 * (blockIdx.y + 1));
  constexpr int kHalf = (1 << 21) - 1;
  unsigned long long bad = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i <= 2 * kHalf; i += gridDim.x * blockDim.x) {
    const float num = (float)(i - kHalf);
    bad += __float_as_uint(quotient_rn(num, den)) != __float_as_uint(__fdiv_rn(num, den));
  }
  if (bad) atomicAdd(mismatches, bad);
}

}  // namespace

cudaError_t check_bisector_quotient(unsigned long long* d_mismatches, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(d_mismatches, 0, sizeof(unsigned long long), s);
  if (e != cudaSuccess) return e;
  quotient_check_kernel<<<dim3(64, 1023), 256, 0, s>>>(d_mismatches);
  return cudaGetLastError();
}

void set_edt_sweep_rows(int rows) { g_sweep_rows = rows == 32 ? 32 : 16; }

uint64_t edt_scratch_words_min(gvx_dims d) {
  return sync_words(d) + std::max<uint64_t>({SweepCfg<32>::kWarps * warp_stack_words((int)d.x, (int)d.y),
                                             zcarry_words(d), occ_words((int)d.x, (int)d.y, (int)d.z)});
}
uint64_t edt_scratch_words(gvx_dims d) {
  return std::max(sync_words(d) + fused_stack_words(d), edt_scratch_words_min(d));
}

cudaError_t launch_edt_pass(uint32_t* d_vox, uint32_t* d_scratch, uint64_t scratch_words, gvx_dims d, int pass,
                            cudaStream_t s, int rows) {
  if (scratch_words < edt_scratch_words_min(d)) return cudaErrorInvalidValue;
  const bool big = (rows == 0 ? sweep_rows() : rows) == 32;
  switch (pass) {
    case 0: return launch_pass_z(d_vox, d_scratch, d, s);
    case 1:
      return big ? launch_sweep<false, 32>(d_vox, d_scratch, scratch_words, d, s)
                 : launch_sweep<false, 16>(d_vox, d_scratch, scratch_words, d, s);
    case 2:
      return big ? launch_sweep<true, 32>(d_vox, d_scratch, scratch_words, d, s)
                 : launch_sweep<true, 16>(d_vox, d_scratch, scratch_words, d, s);
    case 3:
      return big ? launch_sweep_yx<32>(d_vox, d_scratch, scratch_words, d, s)
                 : launch_sweep_yx<16>(d_vox, d_scratch, scratch_words, d, s);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_edt(uint32_t* d_vox, uint32_t* d_scratch, uint64_t scratch_words, gvx_dims d, cudaStream_t s,
                       const EdtConfig& cfg) {
  cudaError_t e = launch_edt_pass(d_vox, d_scratch, scratch_words, d, 0, s, cfg.rows);
  if (e != cudaSuccess || cfg.fused) return e == cudaSuccess ? launch_edt_pass(d_vox, d_scratch, scratch_words, d, 3, s, cfg.rows) : e;
  e = launch_edt_pass(d_vox, d_scratch, scratch_words, d, 1, s, cfg.rows);
  return e == cudaSuccess ? launch_edt_pass(d_vox, d_scratch, scratch_words, d, 2, s, cfg.rows) : e;
}

cudaError_t edt_read_error(const uint32_t* d_scratch, gvx_dims d, uint32_t* flag) {
  return cudaMemcpy(flag, d_scratch + d.z + 1, sizeof(uint32_t), cudaMemcpyDeviceToHost);
}

long long edt_pass_items(gvx_dims d, int pass) {
  switch (pass) {
    case 0: return (long long)z_items((int)d.x, (int)d.y);
    case 1: return ((long long)d.x * d.z + 31) / 32;  // pass Y: columns numbered slice by slice
    default: return ((long long)d.y * d.z + 31) / 32;
  }
}

long long edt_batch_stack_warps() {
  return std::max(batch_stack_warps<16>(), batch_stack_warps<32>());
}

cudaError_t launch_voxelize_edt(uint32_t* d_vox, uint32_t* d_scratch, uint64_t scratch_words, gvx_dims d, float side,
                                const float* d_xyz, uint64_t n, uint32_t* d_outside, cudaStream_t s,
                                const EdtConfig& cfg) {
  if (scratch_words < edt_scratch_words_min(d)) return cudaErrorInvalidValue;
  uint32_t* bits = d_scratch + edt_sync_words((int)d.z);
  // the occupancy bits and, in the same memset, pass Z's other-sites flag
  // (every site is its own: the fused sweep's pass Y may skip the x offset)
  uint32_t* other = d_scratch + d.z + 2;
  cudaError_t e = cudaMemsetAsync(other, 0, (bits - other + occ_words((int)d.x, (int)d.y, (int)d.z)) * sizeof(uint32_t), s);
  if (e != cudaSuccess) return e;
  if (n > 0) {
    const unsigned blocks = (unsigned)std::min<uint64_t>((n + 255) / 256, (uint64_t)device_sms() * 16);
    occ_insert_kernel<<<blocks, 256, 0, s>>>(bits, (int)d.x, (int)d.y, (int)d.z, side, d_xyz, n, d_outside);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  e = kernel_setup<edt_pass_z_bits>(kZWarps * 32, kZBitsSmemMax, nullptr);
  if (e != cudaSuccess) return e;
  const int smem = kZWarps * 2 * z_bits_words((int)d.z) * 4;  // sized by Z: more resident warps
  const long long items = (long long)z_items((int)d.x, (int)d.y);
  edt_pass_z_bits<<<(unsigned)((items + kZWarps - 1) / kZWarps), kZWarps * 32, smem, s>>>(d_vox, bits, (int)d.x,
                                                                                         (int)d.y, (int)d.z, nullptr);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if (cfg.fused) return launch_edt_pass(d_vox, d_scratch, scratch_words, d, 3, s, cfg.rows);
  e = launch_edt_pass(d_vox, d_scratch, scratch_words, d, 1, s, cfg.rows);
  return e == cudaSuccess ? launch_edt_pass(d_vox, d_scratch, scratch_words, d, 2, s, cfg.rows) : e;
}

// The occupancy-bit pass Z over a batch (one persistent launch); skip_other:
// leave maps whose other-sites flag is set to the general pass.
cudaError_t launch_z_bits_batch(const BatchMap* d_table, const BatchItems& it, cudaStream_t s, int skip_other) {
  cudaError_t e;
  e = kernel_setup<edt_pass_z_bits_batch>(kZWarps * 32, kZBitsSmemMax, nullptr);
  if (e != cudaSuccess) return e;
  const int zw = z_bits_words((int)it.z_max);
  const int smem = kZWarps * 2 * zw * 4;  // sized by the tallest map: more resident warps
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, edt_pass_z_bits_batch, kZWarps * 32, smem);
  if (e != cudaSuccess) return e;
  int dev = 0, sm = 0;
  if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
  if ((e = cudaDeviceGetAttribute(&sm, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
  long long blocks = (long long)std::max(per_sm, 1) * std::max(sm, 1);
  blocks = std::max<long long>(1, std::min<long long>(blocks, (it.total[0] + kZWarps - 1) / kZWarps));
  edt_pass_z_bits_batch<<<(unsigned)blocks, kZWarps * 32, smem, s>>>(d_table, it.d_prefix[0], it.n_maps, it.total[0], zw,
                                                                      skip_other);
  return cudaGetLastError();
}

cudaError_t launch_voxelize_edt_batch(const BatchMap* d_table, const BatchItems& it, const float* d_xyz,
                                      const uint64_t* d_offsets, uint64_t n_total, cudaStream_t s, int rows) {
  occ_clear_batch_kernel<<<dim3(64, it.n_maps), 256, 0, s>>>(d_table);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  if (n_total > 0) {
    const unsigned blocks = (unsigned)std::min<uint64_t>((n_total + 255) / 256, (uint64_t)device_sms() * 16);
    occ_insert_batch_kernel<<<blocks, 256, 0, s>>>(d_table, it.n_maps, d_xyz, d_offsets, n_total);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  if ((e = launch_z_bits_batch(d_table, it, s, 0)) != cudaSuccess) return e;
  return (rows == 0 ? sweep_rows() : rows) == 32 ? launch_yx_batch<32>(d_table, it, s)
                                                 : launch_yx_batch<16>(d_table, it, s);
}

// Batched EDT of filled maps.  Pass Z as for one map: each map's occupancy
// bits and other-sites flag from its voxels, then the bits pass for the maps
// whose voxels are all UNINIT or their own sites and the general pass for the
// others (each launch skips the other maps).
cudaError_t launch_edt_batch(const BatchMap* d_table, const BatchItems& it, cudaStream_t s, int rows) {
  batch_flags_clear_kernel<<<(it.n_maps + 255) / 256, 256, 0, s>>>(d_table, it.n_maps);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, occ_from_map_batch_kernel, 256, 0)) != cudaSuccess)
    return e;
  const long long occ_blocks = std::max<long long>(
      1, std::min<long long>((it.total[3] + 7) / 8, (long long)device_sms() * std::max(per_sm, 1)));
  occ_from_map_batch_kernel<<<(unsigned)occ_blocks, 256, 0, s>>>(d_table, it.d_prefix[3], it.n_maps, it.total[3]);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if ((e = launch_z_bits_batch(d_table, it, s, 1)) != cudaSuccess) return e;
  const int smem = kZWarps * kZWarpWords * 4;
  long long blocks = 0;
  if ((e = kernel_setup<edt_pass_z_batch>(kZWarps * 32, smem, &blocks)) != cudaSuccess) return e;
  blocks = std::max<long long>(1, std::min<long long>(blocks, (it.total[0] + kZWarps - 1) / kZWarps));
  edt_pass_z_batch<<<(unsigned)blocks, kZWarps * 32, smem, s>>>(d_table, it.d_prefix[0], it.n_maps, it.total[0]);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  return (rows == 0 ? sweep_rows() : rows) == 32 ? launch_yx_batch<32>(d_table, it, s)
                                                 : launch_yx_batch<16>(d_table, it, s);
}

}  // namespace gvx
