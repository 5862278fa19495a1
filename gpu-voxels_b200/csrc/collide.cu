// BitVoxel collision counting: map vs map, list vs map (single and batched),
// list vs list.
//
// A BitVoxel<256> is 32 bytes.  Two adjacent lanes share one voxel, each
// loading one 16-byte half, so a warp instruction reads 512 contiguous bytes.
// DefaultCollider::collide(BitVoxel, BitVoxel) (GV/voxel/DefaultCollider.hpp:76-81)
// is "both voxels hold a meaning other than eBVM_FREE" (BitVector::noneButEmpty,
// GV/helpers/BitVector.h:184-198): OR the 8 words with bit 0 masked.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <atomic>
#include <climits>

#include "gvx_internal.cuh"

namespace gvx {
namespace {

constexpr unsigned kFull = 0xffffffffu;

int sms() { return device_sms(); }

// Non-empty test of one 16-byte half; `low` marks the half holding bit 0.
__device__ __forceinline__ uint32_t half_bits(uint4 v, bool low) {
  return ((low ? (v.x & ~1u) : v.x) | v.y | v.z | v.w);
}

__device__ __forceinline__ void block_count_add(unsigned long long local, unsigned long long* dst) {
  __shared__ unsigned long long s_sum;
  if (threadIdx.x == 0) s_sum = 0ull;
  __syncthreads();
  local = __reduce_add_sync(kFull, (unsigned)local);
  if ((threadIdx.x & 31) == 0 && local) atomicAdd(&s_sum, local);
  __syncthreads();
  if (threadIdx.x == 0 && s_sum) atomicAdd(dst, s_sum);
}

// kernelCollideVoxelMapsDebug (GV/voxelmap/kernels/VoxelMapOperations.hpp:129-184):
// count i where self[i+off] and other[i] collide; mark self with eBVM_COLLISION.
__global__ void __launch_bounds__(256) bvm_collide_kernel(uint32_t* __restrict__ self, const uint32_t* __restrict__ other,
                                                          uint64_t n, int64_t off, int mark,
                                                          unsigned long long* __restrict__ count) {
  const int lane = threadIdx.x & 31;
  const bool low = (lane & 1) == 0;
  const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
  const uint64_t gw = (uint64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  unsigned long long hits = 0;
  constexpr int kUnroll = 4;
  for (uint64_t base = gw * 16 * kUnroll; base < n; base += warps * 16 * kUnroll) {
    uint4 a[kUnroll], b[kUnroll];
    bool ok[kUnroll];
    int64_t j[kUnroll];
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
      const uint64_t i = base + u * 16 + (lane >> 1);
      j[u] = (int64_t)i + off;
      ok[u] = i < n && j[u] >= 0 && j[u] < (int64_t)n;
      a[u] = make_uint4(0, 0, 0, 0);
      b[u] = make_uint4(0, 0, 0, 0);
      if (ok[u]) {
        a[u] = __ldcs(reinterpret_cast<const uint4*>(self + (uint64_t)j[u] * kBitVoxelWords) + (lane & 1));
        b[u] = __ldcs(reinterpret_cast<const uint4*>(other + i * kBitVoxelWords) + (lane & 1));
      }
    }
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
      uint32_t ma = half_bits(a[u], low), mb = half_bits(b[u], low);
      ma |= __shfl_xor_sync(kFull, ma, 1);
      mb |= __shfl_xor_sync(kFull, mb, 1);
      const bool hit = ok[u] && ma != 0u && mb != 0u;
      if (hit && low) {
        ++hits;
        if (mark) self[(uint64_t)j[u] * kBitVoxelWords] = a[u].x | (1u << kCollisionBit);
      }
    }
  }
  block_count_add(hits, count);
}

// kernelCollideWithVoxelMap (GV/voxellist/kernels/VoxelListOperations.hpp:146-197):
// list entry k collides with map voxel ids[k] + off when that lies in the map.
__global__ void __launch_bounds__(256) list_collide_map_kernel(const uint32_t* __restrict__ ids, uint32_t* __restrict__ lvox,
                                                               uint64_t n, const uint32_t* __restrict__ map,
                                                               uint64_t map_n, int64_t off, int mark,
                                                               unsigned long long* __restrict__ count) {
  const int lane = threadIdx.x & 31;
  const bool low = (lane & 1) == 0;
  const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
  const uint64_t gw = (uint64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  unsigned long long hits = 0;
  for (uint64_t base = gw * 16; base < n; base += warps * 16) {
    const uint64_t k = base + (lane >> 1);
    bool ok = k < n;
    int64_t j = 0;
    uint4 a = make_uint4(0, 0, 0, 0), b = make_uint4(0, 0, 0, 0);
    if (ok) {
      j = (int64_t)__ldg(ids + k) + off;
      ok = j >= 0 && j < (int64_t)map_n;
    }
    if (ok) {
      a = *(reinterpret_cast<const uint4*>(lvox + k * kBitVoxelWords) + (lane & 1));
      b = __ldg(reinterpret_cast<const uint4*>(map + (uint64_t)j * kBitVoxelWords) + (lane & 1));
    }
    uint32_t ma = half_bits(a, low), mb = half_bits(b, low);
    ma |= __shfl_xor_sync(kFull, ma, 1);
    mb |= __shfl_xor_sync(kFull, mb, 1);
    const bool hit = ok && ma != 0u && mb != 0u;
    if (hit && low) {
      ++hits;
      if (mark) lvox[k * kBitVoxelWords] = a.x | (1u << kCollisionBit);
    }
  }
  block_count_add(hits, count);
}

// Batched form: many CSR lists in one launch, per-list counts.  A warp walks
// 16 entries per group (lane pairs share an entry, as above) and owns a
// contiguous range of groups, so the list of its first entry is found by one
// binary search and the lists of later entries by a monotone advance; four
// groups' gathers are issued before any is used.  Hits are aggregated per
// list per warp with __match_any_sync before the atomic.
__global__ void __launch_bounds__(256) lists_collide_map_kernel(const uint32_t* __restrict__ ids, uint32_t* __restrict__ lvox,
                                                                const uint64_t* __restrict__ offsets, uint32_t n_lists,
                                                                uint64_t n_total, const uint32_t* __restrict__ map,
                                                                uint64_t map_n, int mark,
                                                                unsigned long long* __restrict__ counts) {
  constexpr int kU = 4;
  const int lane = threadIdx.x & 31;
  const bool low = (lane & 1) == 0;
  const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
  const uint64_t gw = (uint64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const uint64_t groups = (n_total + 15) / 16;
  const uint64_t per = (groups + warps - 1) / warps;
  const uint64_t g_begin = gw * per, g_end = min(groups, g_begin + per);
  if (g_begin >= g_end) return;
  // the list of the warp's first entry: last k with offsets[k] <= entry
  uint32_t list = 0;
  {
    uint32_t lo = 0, hi = n_lists;
    const uint64_t first = g_begin * 16;
    while (hi - lo > 1) {
      const uint32_t mid = (lo + hi) >> 1;
      if (__ldg(offsets + mid) <= first) lo = mid; else hi = mid;
    }
    list = lo;
  }
  for (uint64_t g = g_begin; g < g_end; g += kU) {
    uint4 a[kU], b[kU];
    bool ok[kU];
    uint64_t k[kU];
#pragma unroll
    for (int u = 0; u < kU; ++u) {
      k[u] = (g + u) * 16 + (lane >> 1);
      ok[u] = g + u < g_end && k[u] < n_total;
      a[u] = make_uint4(0, 0, 0, 0);
      b[u] = make_uint4(0, 0, 0, 0);
      if (ok[u]) {
        const uint64_t j = __ldg(ids + k[u]);
        ok[u] = j < map_n;
        a[u] = *(reinterpret_cast<const uint4*>(lvox + k[u] * kBitVoxelWords) + (lane & 1));
        if (ok[u]) b[u] = __ldg(reinterpret_cast<const uint4*>(map + j * kBitVoxelWords) + (lane & 1));
      }
    }
#pragma unroll
    for (int u = 0; u < kU; ++u) {
      // this lane's list: at or after the list of the warp's previous entries
      uint32_t my = list;
      const uint64_t kk = min(k[u], n_total - 1);
      while (my + 1 < n_lists && __ldg(offsets + my + 1) <= kk) ++my;
      list = __shfl_sync(kFull, my, 30);  // the group's last entry: a lower bound for the next group
      uint32_t ma = half_bits(a[u], low), mb = half_bits(b[u], low);
      ma |= __shfl_xor_sync(kFull, ma, 1);
      mb |= __shfl_xor_sync(kFull, mb, 1);
      const bool hit = ok[u] && ma != 0u && mb != 0u && low;
      if (hit && mark) lvox[k[u] * kBitVoxelWords] = a[u].x | (1u << kCollisionBit);
      const unsigned hit_mask = __ballot_sync(kFull, hit);
      if (hit_mask) {
        const unsigned same = __match_any_sync(kFull, my);
        const unsigned mine = same & hit_mask;
        if (hit && (__ffs(mine) - 1) == lane) atomicAdd(counts + my, (unsigned long long)__popc(mine));
      }
    }
  }
}

// Bits at the even positions of x, packed into the low 16 bits.
__device__ __forceinline__ uint32_t even_bits(uint32_t x) {
  x &= 0x55555555u;
  x = (x | (x >> 1)) & 0x33333333u;
  x = (x | (x >> 2)) & 0x0F0F0F0Fu;
  x = (x | (x >> 4)) & 0x00FF00FFu;
  return (x | (x >> 8)) & 0x0000FFFFu;
}

// One bit per map voxel: set where the voxel holds a meaning other than
// eBVM_FREE (DefaultCollider's test on that side, GV/voxel/DefaultCollider.hpp:
// 76-81).  A warp reduces 32 voxels (1 KB, two 512-byte load instructions of
// lane pairs) to one word; four words in flight per warp.
__global__ void __launch_bounds__(256) bvm_occ_bits_kernel(const uint32_t* __restrict__ map, uint64_t n,
                                                           uint32_t* __restrict__ bits) {
  constexpr int kU = 4;
  const int lane = threadIdx.x & 31;
  const bool low = (lane & 1) == 0;
  const uint64_t words = (n + 31) / 32;
  const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
  const uint64_t gw = (uint64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  for (uint64_t w0 = gw * kU; w0 < words; w0 += warps * kU) {
    uint4 h[kU][2];
#pragma unroll
    for (int u = 0; u < kU; ++u) {
#pragma unroll
      for (int half = 0; half < 2; ++half) {
        const uint64_t v = (w0 + u) * 32 + half * 16 + (lane >> 1);  // voxel of this lane pair
        h[u][half] = v < n ? __ldcs(reinterpret_cast<const uint4*>(map + v * kBitVoxelWords) + (lane & 1))
                           : make_uint4(0, 0, 0, 0);
      }
    }
#pragma unroll
    for (int u = 0; u < kU; ++u) {
      uint32_t word = 0;
#pragma unroll
      for (int half = 0; half < 2; ++half) {
        uint32_t m = half_bits(h[u][half], low);
        m |= __shfl_xor_sync(kFull, m, 1);
        word |= even_bits(__ballot_sync(kFull, m != 0u)) << (16 * half);
      }
      if (lane == 0 && w0 + u < words) bits[w0 + u] = word;
    }
  }
}

// The batched form against those bits.  Each lane takes 4 consecutive
// entries (one 16-byte id load when the ids are 16-byte aligned), a warp 128
// per group, over a contiguous range of groups.  An entry can collide only
// where its map bit is set, so the main loop reads just the ids (prefetched
// one step ahead) and their bits (the bit array stays in L2); the entries
// whose bit is set go to a per-warp queue in shared memory with a lower bound
// of their list, and 32 at a time the warp reads their 32-byte voxels, marks
// and counts the hits (list found by a short advance from the bound).
constexpr int kListQueue = 64;  // per-warp candidate queue (two rounds of 32)

__device__ __forceinline__ void flush_candidates(const uint64_t* __restrict__ cand_k, const uint32_t* __restrict__ cand_lb,
                                                 int count, uint32_t* __restrict__ lvox,
                                                 const uint64_t* __restrict__ offsets, uint32_t n_lists, int mark,
                                                 unsigned long long* __restrict__ counts) {
  const int lane = threadIdx.x & 31;
  bool hit = false;
  uint32_t my = 0;
  if (lane < count) {
    const uint64_t k = cand_k[lane];
    my = cand_lb[lane];
    while (my + 1 < n_lists && __ldg(offsets + my + 1) <= k) ++my;
    uint32_t* v = lvox + k * kBitVoxelWords;
    const uint4 lo4 = *reinterpret_cast<const uint4*>(v);
    const uint4 hi4 = *(reinterpret_cast<const uint4*>(v) + 1);
    hit = ((lo4.x & ~1u) | lo4.y | lo4.z | lo4.w | hi4.x | hi4.y | hi4.z | hi4.w) != 0u;
    if (hit && mark) v[0] = lo4.x | (1u << kCollisionBit);
  }
  const unsigned hit_mask = __ballot_sync(kFull, hit);
  if (hit_mask) {
    const unsigned same = __match_any_sync(kFull, my);
    const unsigned mine = same & hit_mask;
    if (hit && (__ffs(mine) - 1) == lane) atomicAdd(counts + my, (unsigned long long)__popc(mine));
  }
}

__global__ void __launch_bounds__(256) lists_collide_bits_kernel(const uint32_t* __restrict__ ids,
                                                                 uint32_t* __restrict__ lvox,
                                                                 const uint64_t* __restrict__ offsets, uint32_t n_lists,
                                                                 uint64_t n_total, const uint32_t* __restrict__ bits,
                                                                 uint64_t map_n, int mark,
                                                                 unsigned long long* __restrict__ counts) {
  constexpr int kE = 4;       // entries per lane and group
  constexpr int kG = 32 * kE;
  __shared__ uint64_t s_k[8][kListQueue];
  __shared__ uint32_t s_lb[8][kListQueue];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint64_t* cand_k = s_k[warp];
  uint32_t* cand_lb = s_lb[warp];
  const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
  const uint64_t gw = (uint64_t)blockIdx.x * (blockDim.x >> 5) + warp;
  const uint64_t groups = (n_total + kG - 1) / kG;
  const uint64_t per = (groups + warps - 1) / warps;
  const uint64_t g_begin = gw * per, g_end = min(groups, g_begin + per);
  if (g_begin >= g_end) return;
  // list of the warp's first entry: last k with offsets[k] <= entry
  uint32_t list = 0;
  {
    uint32_t lo = 0, hi = n_lists;
    const uint64_t first = g_begin * kG;
    while (hi - lo > 1) {
      const uint32_t mid = (lo + hi) >> 1;
      if (__ldg(offsets + mid) <= first) lo = mid; else hi = mid;
    }
    list = lo;
  }
  // Entry e of lane l in group g is g * kG + e * 32 + l: each load covers 32
  // consecutive entries of a sorted list, so its bit lookups fall in few lines.
  auto load_ids = [&](uint64_t g, uint32_t (&j)[kE]) {
    const uint64_t k0 = g * kG + (uint64_t)lane;
#pragma unroll
    for (int e = 0; e < kE; ++e) j[e] = (g < g_end && k0 + e * 32 < n_total) ? __ldg(ids + k0 + e * 32) : 0xFFFFFFFFu;
  };
  int queued = 0;  // warp-uniform
  uint32_t jn[kE];
  load_ids(g_begin, jn);
  for (uint64_t g = g_begin; g < g_end; ++g) {
    uint32_t j[kE];
#pragma unroll
    for (int e = 0; e < kE; ++e) j[e] = jn[e];
    load_ids(g + 1, jn);  // the next group's ids in flight while this one is tested
    unsigned occ = 0;
#pragma unroll
    for (int e = 0; e < kE; ++e)
      occ |= (unsigned)(j[e] < map_n && ((__ldg(bits + (j[e] >> 5)) >> (j[e] & 31)) & 1u)) << e;
    const uint64_t k0 = g * kG + (uint64_t)lane;
#pragma unroll
    for (int e = 0; e < kE; ++e) {
      const bool c = (occ >> e) & 1u;
      const unsigned cm = __ballot_sync(kFull, c);
      if (cm) {  // append this round's candidates to the queue
        if (c) {
          const int slot = queued + __popc(cm & ((1u << lane) - 1u));
          cand_k[slot] = k0 + e * 32;
          cand_lb[slot] = list;
        }
        queued += __popc(cm);
        __syncwarp();
        if (queued >= 32) {
          flush_candidates(cand_k, cand_lb, 32, lvox, offsets, n_lists, mark, counts);
          __syncwarp();
          queued -= 32;
          if (lane < queued) {  // the remainder moves to the front
            cand_k[lane] = cand_k[32 + lane];
            cand_lb[lane] = cand_lb[32 + lane];
          }
          __syncwarp();
        }
      }
    }
    // the bound for the next group: the list of its first entry
    const uint64_t next = min((g + 1) * kG, n_total - 1);
    while (list + 1 < n_lists && __ldg(offsets + list + 1) <= next) ++list;
  }
  if (queued > 0) flush_candidates(cand_k, cand_lb, queued, lvox, offsets, n_lists, mark, counts);
}

// BitVoxel test of a whole 32-byte voxel: a meaning other than eBVM_FREE.
// A plain (coherent) load: the kernels below may mark this voxel afterwards,
// so it is not read-only for the kernel's duration.
__device__ __forceinline__ bool bitvoxel_occupied(const uint32_t* v) {
  const uint4 lo = *reinterpret_cast<const uint4*>(v);
  const uint4 hi = *(reinterpret_cast<const uint4*>(v) + 1);
  return ((lo.x & ~1u) | lo.y | lo.z | lo.w | hi.x | hi.y | hi.z | hi.w) != 0u;
}

// kernelCollideVoxelMapsDebug with DefaultCollider::collide(BitVoxel,
// ProbabilisticVoxel) (GV/voxelmap/kernels/VoxelMapOperations.hpp:129-184,
// GV/voxel/DefaultCollider.hpp:68-73): count i where other[i]'s occupancy
// reaches `thr` and self[i+off] holds a meaning other than eBVM_FREE; mark
// self with eBVM_COLLISION.  A thread takes 4 consecutive occupancy bytes
// (one 4-byte load, a warp reads 128 contiguous bytes) and loads the 32-byte
// BitVoxel only where the occupancy passes.
__global__ void __launch_bounds__(256) bvm_collide_pvm_kernel(uint32_t* __restrict__ self, const int8_t* __restrict__ other,
                                                              uint64_t n, int64_t off, int thr, int mark,
                                                              unsigned long long* __restrict__ count) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  unsigned long long hits = 0;
  for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t * 4 < n; t += stride) {
    const uint64_t i0 = t * 4;
    int p[4];
    if (i0 + 4 <= n) {
      const char4 c = __ldcs(reinterpret_cast<const char4*>(other) + t);
      p[0] = c.x; p[1] = c.y; p[2] = c.z; p[3] = c.w;
    } else {
#pragma unroll
      for (int k = 0; k < 4; ++k) p[k] = i0 + k < n ? (int)other[i0 + k] : INT_MIN;
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int64_t j = (int64_t)(i0 + k) + off;
      if (p[k] >= thr && j >= 0 && j < (int64_t)n) {
        uint32_t* v = self + (uint64_t)j * kBitVoxelWords;
        if (bitvoxel_occupied(v)) {
          ++hits;
          if (mark) v[0] |= 1u << kCollisionBit;
        }
      }
    }
  }
  block_count_add(hits, count);
}

// kernelCollideWithVoxelMap with DefaultCollider::collide(BitVoxel,
// ProbabilisticVoxel) (GV/voxellist/kernels/VoxelListOperations.hpp:146-197):
// entry k collides when map voxel ids[k] + off lies in the map, its occupancy
// reaches `thr` and the entry holds a meaning other than eBVM_FREE.
__global__ void __launch_bounds__(256) list_collide_pvm_kernel(const uint32_t* __restrict__ ids, uint32_t* __restrict__ lvox,
                                                               uint64_t n, const int8_t* __restrict__ map, uint64_t map_n,
                                                               int64_t off, int thr, int mark,
                                                               unsigned long long* __restrict__ count) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  unsigned long long hits = 0;
  for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += stride) {
    const int64_t j = (int64_t)__ldg(ids + k) + off;
    if (j < 0 || j >= (int64_t)map_n || (int)__ldg(map + j) < thr) continue;
    uint32_t* v = lvox + k * kBitVoxelWords;
    if (bitvoxel_occupied(v)) {
      ++hits;
      if (mark) v[0] |= 1u << kCollisionBit;
    }
  }
  block_count_add(hits, count);
}

// collideVoxellists (GV/voxellist/TemplateVoxelList.hpp:231-289): count of ids
// of `a` found in the sorted list `b` (thrust::binary_search semantics).
__global__ void __launch_bounds__(256) list_collide_list_kernel(const uint32_t* __restrict__ a, uint64_t na,
                                                                const uint32_t* __restrict__ b, uint64_t nb,
                                                                unsigned long long* __restrict__ count) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  unsigned long long hits = 0;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < na; i += stride) {
    const uint32_t key = __ldg(a + i);
    uint64_t lo = 0, hi = nb;
    while (lo < hi) {
      const uint64_t mid = lo + ((hi - lo) >> 1);
      if (__ldg(b + mid) < key) lo = mid + 1; else hi = mid;
    }
    hits += (lo < nb && __ldg(b + lo) == key);
  }
  block_count_add(hits, count);
}

// Blocks of `kernel` (256 threads) resident on the device at once, queried once
// per kernel: kernels whose warps own contiguous ranges must not run in waves.
template <auto kKernel>
unsigned resident_blocks() {
  static std::atomic<int> per_sm{0};  // one cache per kernel
  int v = per_sm.load(std::memory_order_relaxed);
  if (v == 0) {
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, kKernel, 256, 0) != cudaSuccess || v < 1) v = 1;
    per_sm.store(v, std::memory_order_relaxed);
  }
  return (unsigned)(v * sms());
}

unsigned grid_cap(uint64_t work_items, int per_block) {
  const uint64_t want = (work_items + per_block - 1) / per_block;
  return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(want, (uint64_t)sms() * 8));
}

}  // namespace

cudaError_t launch_bvm_collide(uint8_t* d_self, const uint8_t* d_other, uint64_t n, int64_t off, int mark,
                               unsigned long long* d_count, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(d_count, 0, sizeof(unsigned long long), s);
  if (e != cudaSuccess || n == 0) return e;
  bvm_collide_kernel<<<grid_cap(n, 8 * 16 * 4), 256, 0, s>>>(reinterpret_cast<uint32_t*>(d_self),
                                                             reinterpret_cast<const uint32_t*>(d_other), n, off, mark,
                                                             d_count);
  return cudaGetLastError();
}

cudaError_t launch_list_collide_map(const uint32_t* d_ids, uint8_t* d_list_vox, uint64_t n, const uint8_t* d_map,
                                    uint64_t map_n, int64_t off, int mark, unsigned long long* d_count, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(d_count, 0, sizeof(unsigned long long), s);
  if (e != cudaSuccess || n == 0) return e;
  list_collide_map_kernel<<<grid_cap(n, 8 * 16), 256, 0, s>>>(d_ids, reinterpret_cast<uint32_t*>(d_list_vox), n,
                                                              reinterpret_cast<const uint32_t*>(d_map), map_n, off,
                                                              mark, d_count);
  return cudaGetLastError();
}

cudaError_t launch_lists_collide_map(const uint32_t* d_ids, uint8_t* d_vox, const uint64_t* d_offsets, uint32_t n_lists,
                                     uint64_t n_total, const uint8_t* d_map, uint64_t map_n, int mark,
                                     unsigned long long* d_counts, cudaStream_t s, uint32_t* d_occ) {
  cudaError_t e = cudaMemsetAsync(d_counts, 0, sizeof(unsigned long long) * n_lists, s);
  if (e != cudaSuccess || n_total == 0 || n_lists == 0) return e;
  if (d_occ != nullptr && 2 * n_total >= map_n) {
    // many entries per voxel: one streaming read of the map beats a 32-byte
    // random gather per entry
    bvm_occ_bits_kernel<<<grid_cap((map_n + 31) / 32, 8 * 4), 256, 0, s>>>(reinterpret_cast<const uint32_t*>(d_map),
                                                                           map_n, d_occ);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    const unsigned grid = std::min(grid_cap(n_total, 8 * 128), resident_blocks<lists_collide_bits_kernel>());
    lists_collide_bits_kernel<<<grid, 256, 0, s>>>(d_ids, reinterpret_cast<uint32_t*>(d_vox), d_offsets, n_lists,
                                                   n_total, d_occ, map_n, mark, d_counts);
    return cudaGetLastError();
  }
  const unsigned grid = std::min(grid_cap(n_total, 8 * 16), resident_blocks<lists_collide_map_kernel>());
  lists_collide_map_kernel<<<grid, 256, 0, s>>>(
      d_ids, reinterpret_cast<uint32_t*>(d_vox), d_offsets, n_lists, n_total, reinterpret_cast<const uint32_t*>(d_map),
      map_n, mark, d_counts);
  return cudaGetLastError();
}

cudaError_t launch_bvm_collide_pvm(uint8_t* d_self, const int8_t* d_other, uint64_t n, int64_t off, int thr, int mark,
                                   unsigned long long* d_count, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(d_count, 0, sizeof(unsigned long long), s);
  if (e != cudaSuccess || n == 0) return e;
  bvm_collide_pvm_kernel<<<grid_cap((n + 3) / 4, 256), 256, 0, s>>>(reinterpret_cast<uint32_t*>(d_self), d_other, n, off,
                                                                    thr, mark, d_count);
  return cudaGetLastError();
}

cudaError_t launch_list_collide_pvm(const uint32_t* d_ids, uint8_t* d_list_vox, uint64_t n, const int8_t* d_map,
                                    uint64_t map_n, int64_t off, int thr, int mark, unsigned long long* d_count,
                                    cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(d_count, 0, sizeof(unsigned long long), s);
  if (e != cudaSuccess || n == 0) return e;
  list_collide_pvm_kernel<<<grid_cap(n, 256), 256, 0, s>>>(d_ids, reinterpret_cast<uint32_t*>(d_list_vox), n, d_map,
                                                           map_n, off, thr, mark, d_count);
  return cudaGetLastError();
}

cudaError_t launch_list_collide_list(const uint32_t* d_a, uint64_t na, const uint32_t* d_b, uint64_t nb,
                                     unsigned long long* d_count, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(d_count, 0, sizeof(unsigned long long), s);
  if (e != cudaSuccess || na == 0 || nb == 0) return e;
  list_collide_list_kernel<<<grid_cap(na, 256), 256, 0, s>>>(d_a, na, d_b, nb, d_count);
  return cudaGetLastError();
}

}  // namespace gvx
