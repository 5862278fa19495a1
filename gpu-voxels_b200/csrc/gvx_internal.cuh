// Internal definitions shared by the gvx CUDA translation units.
//
// Value formats follow gpu-voxels (GV = packages/gpu_voxels/src/gpu_voxels/):
//   DistanceVoxel  x | y<<10 | z<<20, uninitialised coordinate 1023
//                  (GV/voxel/DistanceVoxel.hpp:31-65, GV/helpers/common_defines.h:113-131)
//   BitVoxel<256>  32 bytes, bit k = meaning k (GV/helpers/BitVector.h:349-350)
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "../../include/gvx.h"

namespace gvx {

constexpr uint32_t kUninit = 1023u;              // PBA_UNINITIALISED_COORD
constexpr uint32_t kDvUninit = 0x3FFFFFFFu;      // all three coordinates uninitialised
constexpr int32_t kMaxObstacleDistance = 2147483647;  // MAX_OBSTACLE_DISTANCE
constexpr uint32_t kBitVoxelBytes = 32;
constexpr int16_t kManhattanUninitialized = 32767;  // MANHATTAN_DISTANCE_UNINITIALIZED (common_defines.h:117)
constexpr int16_t kManhattanTooClose = 32765;       // MANHATTAN_DISTANCE_TOO_CLOSE (:119)
constexpr uint32_t kBitVoxelWords = 8;
constexpr uint32_t kEbvmCollision = 2;  // eBVM_COLLISION (GV/helpers/common_defines.h:55)
constexpr uint32_t kCollisionBit = 2;            // eBVM_COLLISION
constexpr uint32_t kMaxDim = 1023;

__host__ __device__ __forceinline__ uint32_t dv_pack(uint32_t x, uint32_t y, uint32_t z) {
  return x | (y << 10) | (z << 20);
}
__host__ __device__ __forceinline__ uint32_t dv_x(uint32_t v) { return v & 0x3ffu; }
__host__ __device__ __forceinline__ uint32_t dv_y(uint32_t v) { return (v >> 10) & 0x3ffu; }
__host__ __device__ __forceinline__ uint32_t dv_z(uint32_t v) { return v >> 20; }

// mapToVoxels(float, Vector3f) (GV/voxelmap/kernels/VoxelMapOperations.h:121-131):
// IEEE divide, floor, saturating float->u32 convert (negative and NaN -> 0).
__device__ __forceinline__ uint32_t coord_to_voxel(float c, float side) {
  return __float2uint_rz(floorf(__fdiv_rn(c, side)));
}

}  // namespace gvx

// Opaque handle definitions (C ABI types).
struct gvx_dvm {
  gvx_dims dims;
  float side;
  uint32_t* d_vox;
  bool owns;
  uint32_t* d_scratch;  // EDT workspace (proximate-site stacks, slice counters), owned
  uint64_t scratch_words;
  int edt_rows;   // EDT sweep configuration (0 = library default), set by the autotuner
  int edt_fused;
};

struct gvx_bvm {
  gvx_dims dims;
  float side;
  uint8_t* d_vox;
  // insertMetaPointCloudWithSelfCollisionCheck: per-point hit flags of the
  // largest sub-cloud so far, and the colliding meanings (8 words)
  uint8_t* d_flags = nullptr;
  uint64_t flags_cap = 0;
  uint32_t* d_colliding = nullptr;
  // batched list collisions: one bit per voxel, set where the voxel holds a
  // meaning other than eBVM_FREE (refilled from the map by every such call)
  uint32_t* d_occ = nullptr;
};

struct gvx_pvm {
  gvx_dims dims;
  float side;
  int8_t* d_vox;  // one occupancy byte per voxel, allocation rounded up to 16 bytes
};

struct gvx_blist {
  gvx_dims ref;
  float side;
  uint32_t* d_ids;
  uint8_t* d_vox;
  uint64_t n;
  uint64_t cap;
  // insertPointCloud's device buffers, kept with the list and grown only
  // when a call needs more: the sort/scan work area and the spare storage
  // the merged list is written to (then swapped with d_ids / d_vox).
  void* d_work = nullptr;
  size_t work_bytes = 0;
  uint32_t* d_ids2 = nullptr;
  uint8_t* d_vox2 = nullptr;
  uint64_t cap2 = 0;
};

namespace gvx {

// One map of a batch, as the batched kernels see it.
struct BatchMap {
  uint32_t* vox;
  uint32_t* scratch;
  int X, Y, Z;
  float side;
  uint64_t nvox;
  uint32_t sync_off;  // first of this map's Z slice counters in BatchItems::d_sync
};

// Work-item layout of the batched EDT: for pass p, map k owns warp items
// [prefix[p][k], prefix[p][k+1]); prefix[3] numbers the occupancy-bit tasks
// of pass Z on filled maps (32 columns x 32 rows each).  The fused Y -> X launch keeps one stack of
// stack_len rows (64 words each) per resident warp in d_stacks and its slice
// counters, queue head and error word in d_sync (sync_words + 2 words).
struct BatchItems {
  long long* d_prefix[4];
  long long total[4];
  uint32_t n_maps;
  uint32_t* d_stacks;
  long long stack_warps;
  uint32_t stack_len;
  unsigned* d_sync;
  unsigned sync_words;
  uint32_t z_max;  // the tallest map's Z
};

// Error reporting shared by the ABI units.
void set_error(const std::string& msg);
// Streaming multiprocessors of the current device (cudaDevAttrMultiProcessorCount,
// cached per device; 1 if the query fails), for grid sizing.
int device_sms();
gvx_status cuda_status(cudaError_t e, const char* what);

inline uint64_t num_voxels(const gvx_dims& d) { return (uint64_t)d.x * d.y * d.z; }
inline cudaStream_t as_stream(gvx_stream s) { return reinterpret_cast<cudaStream_t>(s); }

// Launchers implemented in the kernel translation units.  They check only
// what the kernels need; argument validation happens in the ABI layer.
cudaError_t launch_dvm_clear(uint32_t* d_vox, uint64_t n, cudaStream_t s);
cudaError_t launch_dvm_insert(uint32_t* d_vox, gvx_dims d, float side, const float* d_xyz, uint64_t n,
                              uint32_t* d_outside, cudaStream_t s);
cudaError_t launch_bvm_insert(uint8_t* d_vox, gvx_dims d, float side, const float* d_xyz, uint64_t n, uint32_t meaning,
                              uint32_t* d_outside, cudaStream_t s);
// EDT workspace: the Z slice counters, queue head and error word of the
// fused Y -> X launch, then the proximate-site stacks.  edt_scratch_words is
// the size that lets the fused launch use every resident warp;
// edt_scratch_words_min the least any launch needs.
uint64_t edt_scratch_words(gvx_dims d);
uint64_t edt_scratch_words_min(gvx_dims d);
// EDT launch configuration: rows per staging chunk of the sweeps (16 or 32;
// 0 = library default) and whether the y and x sweeps run as one fused launch.
struct EdtConfig {
  int rows = 0;
  int fused = 1;
};
cudaError_t launch_edt(uint32_t* d_vox, uint32_t* d_scratch, uint64_t scratch_words, gvx_dims d, cudaStream_t s,
                       const EdtConfig& cfg = EdtConfig{});
// pass 0 = Z (occupancy bits from the map, the bits pass, and the general
// pass when a voxel holds another site), 1 = Y, 2 = X, 3 = fused Y -> X
cudaError_t launch_edt_pass(uint32_t* d_vox, uint32_t* d_scratch, uint64_t scratch_words, gvx_dims d, int pass,
                            cudaStream_t s, int rows = 0);
// Synchronous read of the error word the last fused launch left (0 = ok).
cudaError_t edt_read_error(const uint32_t* d_scratch, gvx_dims d, uint32_t* flag);
// BitVoxelMap bit maintenance: clear `bits` (8 words) in every voxel; move
// every voxel's bits down by `shift` (<= 56) and clear meanings 0..3.
cudaError_t launch_bvm_clear_bits(uint8_t* d_vox, gvx_dims d, const uint32_t bits[8], cudaStream_t s);
cudaError_t launch_bvm_shift(uint8_t* d_vox, gvx_dims d, uint32_t shift, cudaStream_t s);
// Sub-clouds in order (points offsets[k] .. offsets[k+1] of d_xyz, host
// offsets): check against the map, then insert meaning[k] (+ eBVM_COLLISION
// where hit); masks: 8 words per sub-cloud (host); d_flags: at least the
// largest sub-cloud's points; d_colliding: 8 words, zeroed here.
cudaError_t launch_meta_insert_self_coll(uint8_t* d_vox, gvx_dims d, float side, const float* d_xyz,
                                         const uint64_t* offsets, uint32_t n_clouds, const uint8_t* meanings,
                                         const uint32_t* masks, uint8_t* d_flags, uint32_t* d_colliding,
                                         uint32_t* d_outside, cudaStream_t s);
// Counts the quotients of the EDT bisector domain whose bits differ from the
// IEEE divide (every numerator and divisor the sweeps can meet).
cudaError_t check_bisector_quotient(unsigned long long* d_mismatches, cudaStream_t s);
// Resident warps of the fused batch launch (size of the batch stack pool).
long long edt_batch_stack_warps();
// Rows per staging chunk of the sweeps (16 or 32).
void set_edt_sweep_rows(int rows);
// Warp work items of one EDT pass for a map of dims d.
long long edt_pass_items(gvx_dims d, int pass);
// All maps of a batch, one persistent launch per pass.
cudaError_t launch_edt_batch(const BatchMap* d_table, const BatchItems& items, cudaStream_t s, int rows = 0);
// clearMap + insertPointCloud + EDT in one pass: occupancy bits in the
// workspace, pass Z reads them (the map is written once).
cudaError_t launch_voxelize_edt(uint32_t* d_vox, uint32_t* d_scratch, uint64_t scratch_words, gvx_dims d, float side,
                                const float* d_xyz, uint64_t n, uint32_t* d_outside, cudaStream_t s,
                                const EdtConfig& cfg = EdtConfig{});
cudaError_t launch_voxelize_edt_batch(const BatchMap* d_table, const BatchItems& items, const float* d_xyz,
                                      const uint64_t* d_offsets, uint64_t n_total, cudaStream_t s, int rows = 0);
// Launch shape of the trilinear query kernels (every shape gives the same
// results): threads per block and the grid cap in blocks per SM.  Per process,
// picked by gvx_query_autotune or set with gvx_set_query_config.
struct QueryConfig {
  int threads = 256;
  int blocks_per_sm = 16;
};
QueryConfig query_config();
void set_query_config(const QueryConfig& c);
// Trilinear distance queries and their adjoint (continuous.cu), in that shape.
cudaError_t launch_trilinear(const gvx_dvm* m, const float* d_xyz, uint64_t n, float* d_dist, float* d_grad, cudaStream_t s);
cudaError_t launch_trilinear_bwd(const gvx_dvm* m, const float* d_xyz, uint64_t n, const float* d_gout, float* d_gxyz,
                                 cudaStream_t s);
// Autotuner cache (tune.cu): the best configuration recorded for `key` on the
// current device, from memory or the file named by GVX_TUNE_CACHE.
bool tune_lookup(const std::string& key, EdtConfig* cfg, float* ms);
void tune_store(const std::string& key, const EdtConfig& cfg, float ms);
std::string tune_device_name();
cudaError_t launch_pvm_insert(int8_t* d_vox, gvx_dims d, float side, const float* d_xyz, uint64_t n, uint32_t meaning,
                              uint32_t* d_outside, cudaStream_t s);
cudaError_t launch_merge_occupied(uint32_t* d_dvm, const int8_t* d_pvm, gvx_dims d, const uint32_t off[3], float threshold,
                                  cudaStream_t s);
int prob_threshold(float val);
// Typed collisions (collide_types.cu).  mode / kind 0: the other map is a
// BitVoxel map; 1: an int8 ProbVoxelMap.  d_count (uint64) and d_types (32 B)
// are overwritten with this call's count and OR of colliding types.
cudaError_t launch_bvm_collide_types(uint8_t* d_self, const void* d_other, uint64_t n, int mode, float threshold,
                                     unsigned long long* d_count, uint32_t* d_types, cudaStream_t s);
cudaError_t launch_list_collide_types(const uint32_t* d_ids, uint8_t* d_lvox, uint64_t n, const void* d_map,
                                      uint64_t map_n, int kind, float threshold, int64_t off, const uint8_t* d_mask,
                                      unsigned long long* d_count, uint32_t* d_types, cudaStream_t s);
cudaError_t launch_list_list_types(const uint32_t* d_ids_a, const uint8_t* d_vox_a, uint64_t na, const uint32_t* d_ids_b,
                                   const uint8_t* d_vox_b, uint64_t nb, unsigned long long* d_count, uint32_t* d_types,
                                   cudaStream_t s);
cudaError_t launch_extract_distances(const uint32_t* d_vox, gvx_dims d, int robot_radius, int8_t* d_out, cudaStream_t s);
cudaError_t launch_init_floodfill(const int8_t* d_in, int16_t* d_out, uint64_t n, int robot_radius, cudaStream_t s);
// Distance band -> list: per-tile counts, exclusive tile offsets (+ total at
// [band_tiles]), then ids and voxels written in id order.
uint64_t band_tiles(gvx_dims d);
cudaError_t launch_band_count(const uint32_t* d_vox, gvx_dims d, int mn, int mx, uint32_t* d_tiles, cudaStream_t s);
cudaError_t launch_band_write(const uint32_t* d_vox, gvx_dims d, int mn, int mx, const uint32_t* d_tiles, uint32_t* d_ids,
                              uint8_t* d_lvox, cudaStream_t s);
cudaError_t launch_dvm_sqdist(const uint32_t* d_vox, gvx_dims d, const uint32_t* d_ids, uint64_t n, int32_t* d_out,
                              int mode, cudaStream_t s);
cudaError_t launch_dvm_sqdist_map(const uint32_t* d_vox, gvx_dims d, int32_t* d_out, cudaStream_t s);
cudaError_t launch_bvm_collide(uint8_t* d_self, const uint8_t* d_other, uint64_t n, int64_t off, int mark,
                               unsigned long long* d_count, cudaStream_t s);
// ProbVoxelMap forms of collideWith (DefaultCollider): thr is the occupancy
// threshold as a Probability (floatToProbability, clamped).
cudaError_t launch_bvm_collide_pvm(uint8_t* d_self, const int8_t* d_other, uint64_t n, int64_t off, int thr, int mark,
                                   unsigned long long* d_count, cudaStream_t s);
cudaError_t launch_list_collide_pvm(const uint32_t* d_ids, uint8_t* d_list_vox, uint64_t n, const int8_t* d_map,
                                    uint64_t map_n, int64_t off, int thr, int mark, unsigned long long* d_count,
                                    cudaStream_t s);
cudaError_t launch_list_collide_map(const uint32_t* d_ids, uint8_t* d_list_vox, uint64_t n, const uint8_t* d_map,
                                    uint64_t map_n, int64_t off, int mark, unsigned long long* d_count, cudaStream_t s);
// d_occ (optional, (map_n + 31) / 32 words): when given and the lists hold at
// least half as many entries as the map has voxels, the map is first reduced to
// one occupancy bit per voxel and the entries test those bits.
cudaError_t launch_lists_collide_map(const uint32_t* d_ids, uint8_t* d_vox, const uint64_t* d_offsets, uint32_t n_lists,
                                     uint64_t n_total, const uint8_t* d_map, uint64_t map_n, int mark,
                                     unsigned long long* d_counts, cudaStream_t s, uint32_t* d_occ = nullptr);
cudaError_t launch_list_collide_list(const uint32_t* d_a, uint64_t na, const uint32_t* d_b, uint64_t nb,
                                     unsigned long long* d_count, cudaStream_t s);

}  // namespace gvx
