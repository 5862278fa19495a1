// C ABI of the engine (include/gvx.h): argument checks, handle lifetime and
// dispatch to the kernels.  No exception crosses this boundary; failures
// return a gvx_status and leave a message in gvx_last_error().
#include <cuda_runtime.h>
#include <stdint.h>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "gvx_internal.cuh"

namespace gvx {

cudaError_t launch_sphere_clearance(const gvx_dvm* m, const gvx_arm& arm, const float* d_q, uint64_t n_cfg, float* d_out,
                                    cudaStream_t s);
cudaError_t launch_traj_cost(const gvx_dvm* m, const gvx_arm& arm, const float* d_q, uint64_t n_traj, uint32_t n_wp,
                             float margin, float* d_cost, cudaStream_t s);
cudaError_t launch_traj_cost_bwd(const gvx_dvm* m, const gvx_arm& arm, const float* d_q, uint64_t n_traj, uint32_t n_wp,
                                 float margin, const float* d_gcost, float* d_gq, cudaStream_t s);

namespace {
thread_local std::string t_last_error;
}

void set_error(const std::string& msg) { t_last_error = msg; }

gvx_status cuda_status(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return GVX_OK;
  set_error(std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")");
  if (e == cudaErrorMemoryAllocation) return GVX_ERR_OOM;
  return GVX_ERR_CUDA;
}

namespace {

gvx_status fail(gvx_status st, const std::string& msg) {
  set_error(msg);
  return st;
}

gvx_status check_dims(const gvx_dims* d) {
  if (d == nullptr) return fail(GVX_ERR_INVALID_ARG, "dims is null");
  if (d->x < 1 || d->y < 1 || d->z < 1 || d->x > kMaxDim || d->y > kMaxDim || d->z > kMaxDim)
    return fail(GVX_ERR_OUT_OF_DOMAIN, "every map axis must be in [1, 1023] (10-bit DistanceVoxel coordinates)");
  return GVX_OK;
}

bool same_dims(const gvx_dims& a, const gvx_dims& b) { return a.x == b.x && a.y == b.y && a.z == b.z; }

int64_t linear_offset(const gvx_dims& d, const int32_t* off) {
  if (off == nullptr) return 0;
  // getVoxelIndexSigned (GV/voxelmap/kernels/VoxelMapOperations.h:63-75)
  return (int64_t)off[2] * (int64_t)d.x * (int64_t)d.y + (int64_t)off[1] * (int64_t)d.x + (int64_t)off[0];
}

}  // namespace
}  // namespace gvx

using namespace gvx;

extern "C" {

const char* gvx_last_error(void) { return t_last_error.c_str(); }

const char* gvx_version(void) { return "gvx 0.1.0 (sm_100a)"; }

gvx_status gvx_init_device(int device) {
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0) return fail(GVX_ERR_NO_DEVICE, "no CUDA device visible");
  if (device < 0 || device >= count) return fail(GVX_ERR_INVALID_ARG, "device index out of range");
  cudaDeviceProp p;
  e = cudaGetDeviceProperties(&p, device);
  if (e != cudaSuccess) return cuda_status(e, "cudaGetDeviceProperties");
  if (p.major != 10) return fail(GVX_ERR_NO_DEVICE, std::string("device is not compute capability 10.x: ") + p.name);
  return cuda_status(cudaSetDevice(device), "cudaSetDevice");
}

/* ---- DistanceVoxelMap -------------------------------------------------- */

gvx_status gvx_dvm_create(const gvx_dims* dims, float voxel_side, gvx_dvm** out) {
  if (out == nullptr) return fail(GVX_ERR_INVALID_ARG, "out is null");
  *out = nullptr;
  gvx_status st = check_dims(dims);
  if (st != GVX_OK) return st;
  if (!(voxel_side > 0.0f)) return fail(GVX_ERR_INVALID_ARG, "voxel side must be > 0");
  gvx_dvm* m = new (std::nothrow) gvx_dvm{*dims, voxel_side, nullptr, true, nullptr, edt_scratch_words(*dims), 0, 1};
  if (m == nullptr) return fail(GVX_ERR_OOM, "host allocation failed");
  const uint64_t n = num_voxels(*dims);
  cudaError_t e = cudaMalloc(&m->d_vox, n * sizeof(uint32_t) + 16);
  if (e == cudaSuccess) e = cudaMalloc(&m->d_scratch, m->scratch_words * sizeof(uint32_t));
  if (e != cudaSuccess) {
    if (m->d_vox) cudaFree(m->d_vox);
    delete m;
    return cuda_status(e, "cudaMalloc(DistanceVoxelMap)");
  }
  e = launch_dvm_clear(m->d_vox, n, 0);
  if (e == cudaSuccess) e = cudaStreamSynchronize(0);
  if (e != cudaSuccess) {
    cudaFree(m->d_vox);
    cudaFree(m->d_scratch);
    delete m;
    return cuda_status(e, "clear new DistanceVoxelMap");
  }
  *out = m;
  return GVX_OK;
}

gvx_status gvx_dvm_wrap(const gvx_dims* dims, float voxel_side, uint32_t* d_voxels, gvx_dvm** out) {
  if (out == nullptr || d_voxels == nullptr) return fail(GVX_ERR_INVALID_ARG, "null argument");
  *out = nullptr;
  gvx_status st = check_dims(dims);
  if (st != GVX_OK) return st;
  if (!(voxel_side > 0.0f)) return fail(GVX_ERR_INVALID_ARG, "voxel side must be > 0");
  if (reinterpret_cast<uintptr_t>(d_voxels) % 16 != 0) return fail(GVX_ERR_INVALID_ARG, "voxel buffer must be 16-byte aligned");
  gvx_dvm* m = new (std::nothrow) gvx_dvm{*dims, voxel_side, d_voxels, false, nullptr, edt_scratch_words(*dims), 0, 1};
  if (m == nullptr) return fail(GVX_ERR_OOM, "host allocation failed");
  cudaError_t e = cudaMalloc(&m->d_scratch, m->scratch_words * sizeof(uint32_t));
  if (e != cudaSuccess) {
    delete m;
    return cuda_status(e, "cudaMalloc(EDT workspace)");
  }
  *out = m;
  return GVX_OK;
}

gvx_status gvx_dvm_destroy(gvx_dvm* m) {
  if (m == nullptr) return GVX_OK;
  cudaError_t e = cudaSuccess;
  if (m->owns && m->d_vox) e = cudaFree(m->d_vox);
  if (m->d_scratch) {
    cudaError_t e2 = cudaFree(m->d_scratch);
    if (e == cudaSuccess) e = e2;
  }
  delete m;
  return cuda_status(e, "cudaFree(DistanceVoxelMap)");
}

gvx_status gvx_dvm_info(const gvx_dvm* m, gvx_dims* dims, float* voxel_side, uint32_t** d_voxels) {
  if (m == nullptr) return fail(GVX_ERR_INVALID_ARG, "map is null");
  if (dims) *dims = m->dims;
  if (voxel_side) *voxel_side = m->side;
  if (d_voxels) *d_voxels = m->d_vox;
  return GVX_OK;
}

gvx_status gvx_dvm_clear(gvx_dvm* m, gvx_stream stream) {
  if (m == nullptr) return fail(GVX_ERR_INVALID_ARG, "map is null");
  return cuda_status(launch_dvm_clear(m->d_vox, num_voxels(m->dims), as_stream(stream)), "clearMap");
}

gvx_status gvx_dvm_insert_points(gvx_dvm* m, const float* d_xyz, uint64_t n, uint32_t* d_outside, gvx_stream stream) {
  if (m == nullptr || (n > 0 && d_xyz == nullptr)) return fail(GVX_ERR_INVALID_ARG, "null argument");
  return cuda_status(launch_dvm_insert(m->d_vox, m->dims, m->side, d_xyz, n, d_outside, as_stream(stream)),
                     "insertPointCloud(DistanceVoxelMap)");
}

gvx_status gvx_dvm_edt(gvx_dvm* m, uint32_t m1, uint32_t m2, uint32_t m3, gvx_stream stream) {
  (void)m1; (void)m2; (void)m3;
  if (m == nullptr) return fail(GVX_ERR_INVALID_ARG, "map is null");
  return cuda_status(launch_edt(m->d_vox, m->d_scratch, m->scratch_words, m->dims, as_stream(stream), EdtConfig{m->edt_rows, m->edt_fused}), "parallelBanding3D");
}

gvx_status gvx_dvm_voxelize_edt(gvx_dvm* m, const float* d_xyz, uint64_t n, uint32_t* d_outside, gvx_stream stream) {
  if (m == nullptr || (n > 0 && d_xyz == nullptr)) return fail(GVX_ERR_INVALID_ARG, "null argument");
  return cuda_status(launch_voxelize_edt(m->d_vox, m->d_scratch, m->scratch_words, m->dims, m->side, d_xyz, n, d_outside,
                                         as_stream(stream), EdtConfig{m->edt_rows, m->edt_fused}),
                     "voxelize + EDT");
}

gvx_status gvx_dvm_edt_pass(gvx_dvm* m, int pass, gvx_stream stream) {
  if (m == nullptr || pass < 0 || pass > 3) return fail(GVX_ERR_INVALID_ARG, "map is null or pass not in {0,1,2,3}");
  return cuda_status(launch_edt_pass(m->d_vox, m->d_scratch, m->scratch_words, m->dims, pass, as_stream(stream), m->edt_rows), "EDT pass");
}

gvx_status gvx_dvm_edt_check(gvx_dvm* m, uint32_t* flags) {
  if (m == nullptr || flags == nullptr) return fail(GVX_ERR_INVALID_ARG, "null argument");
  cudaError_t e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = edt_read_error(m->d_scratch, m->dims, flags);
  if (e != cudaSuccess) return cuda_status(e, "EDT check");
  if (*flags != 0) return fail(GVX_ERR_TIMEOUT, "EDT: a slice wait of the fused y->x sweep gave up (results invalid)");
  return GVX_OK;
}

gvx_status gvx_check_bisector_quotient(uint64_t* mismatches) {
  if (mismatches == nullptr) return fail(GVX_ERR_INVALID_ARG, "null argument");
  unsigned long long* d = nullptr;
  cudaError_t e = cudaMalloc(&d, sizeof(unsigned long long));
  if (e != cudaSuccess) return cuda_status(e, "bisector check");
  unsigned long long h = 0;
  e = check_bisector_quotient(d, nullptr);
  if (e == cudaSuccess) e = cudaMemcpy(&h, d, sizeof(h), cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) return cuda_status(e, "bisector check");
  *mismatches = h;
  return GVX_OK;
}

gvx_status gvx_dvm_sqdist(const gvx_dvm* m, const uint32_t* d_ids, uint64_t n, int32_t* d_out, gvx_stream stream) {
  if (m == nullptr || (n > 0 && (d_ids == nullptr || d_out == nullptr))) return fail(GVX_ERR_INVALID_ARG, "null argument");
  return cuda_status(launch_dvm_sqdist(m->d_vox, m->dims, d_ids, n, d_out, 0, as_stream(stream)), "getSquaredDistances");
}

gvx_status gvx_dvm_dist(const gvx_dvm* m, const uint32_t* d_ids, uint64_t n, int32_t* d_out, gvx_stream stream) {
  if (m == nullptr || (n > 0 && (d_ids == nullptr || d_out == nullptr))) return fail(GVX_ERR_INVALID_ARG, "null argument");
  return cuda_status(launch_dvm_sqdist(m->d_vox, m->dims, d_ids, n, d_out, 1, as_stream(stream)), "getDistances");
}

gvx_status gvx_dvm_gather(const gvx_dvm* m, const uint32_t* d_ids, uint64_t n, uint32_t* d_out, gvx_stream stream) {
  if (m == nullptr || (n > 0 && (d_ids == nullptr || d_out == nullptr))) return fail(GVX_ERR_INVALID_ARG, "null argument");
  return cuda_status(
      launch_dvm_sqdist(m->d_vox, m->dims, d_ids, n, reinterpret_cast<int32_t*>(d_out), 2, as_stream(stream)),
      "gatherVoxelsByIndex");
}

gvx_status gvx_dvm_sqdist_map(const gvx_dvm* m, int32_t* d_out, gvx_stream stream) {
  if (m == nullptr || d_out == nullptr) return fail(GVX_ERR_INVALID_ARG, "null argument");
  return cuda_status(launch_dvm_sqdist_map(m->d_vox, m->dims, d_out, as_stream(stream)), "sqdist_map");
}

/* ---- continuous queries ------------------------------------------------ */

gvx_status gvx_query_trilinear(const gvx_dvm* m, const float* d_xyz, uint64_t n, float* d_dist, float* d_grad,
                               gvx_stream stream) {
  if (m == nullptr || (n > 0 && (d_xyz == nullptr || d_dist == nullptr))) return fail(GVX_ERR_INVALID_ARG, "null argument");
  return cuda_status(launch_trilinear(m, d_xyz, n, d_dist, d_grad, as_stream(stream)), "trilinear query");
}

gvx_status gvx_query_trilinear_bwd(const gvx_dvm* m, const float* d_xyz, uint64_t n, const float* d_grad_dist,
                                   float* d_grad_xyz, gvx_stream stream) {
  if (m == nullptr || (n > 0 && (d_xyz == nullptr || d_grad_dist == nullptr || d_grad_xyz == nullptr)))
    return fail(GVX_ERR_INVALID_ARG, "null argument");
  return cuda_status(launch_trilinear_bwd(m, d_xyz, n, d_grad_dist, d_grad_xyz, as_stream(stream)), "trilinear adjoint");
}

static gvx_status check_arm(const gvx_arm* arm) {
  if (arm == nullptr) return fail(GVX_ERR_INVALID_ARG, "arm is null");
  if (arm->n_joints < 1 || arm->n_joints > GVX_MAX_JOINTS) return fail(GVX_ERR_INVALID_ARG, "n_joints out of [1,16]");
  if (arm->n_spheres < 1 || arm->n_spheres > GVX_MAX_SPHERES) return fail(GVX_ERR_INVALID_ARG, "n_spheres out of [1,256]");
  for (int s = 0; s < arm->n_spheres; ++s)
    if (arm->link[s] < 0 || arm->link[s] >= arm->n_joints) return fail(GVX_ERR_INVALID_ARG, "sphere link out of range");
  return GVX_OK;
}

gvx_status gvx_sphere_clearance(const gvx_dvm* m, const gvx_arm* arm, const float* d_q, uint64_t n_cfg, float* d_out,
                                gvx_stream stream) {
  if (m == nullptr || (n_cfg > 0 && (d_q == nullptr || d_out == nullptr))) return fail(GVX_ERR_INVALID_ARG, "null argument");
  gvx_status st = check_arm(arm);
  if (st != GVX_OK) return st;
  return cuda_status(launch_sphere_clearance(m, *arm, d_q, n_cfg, d_out, as_stream(stream)), "sphere clearance");
}

gvx_status gvx_traj_cost(const gvx_dvm* m, const gvx_arm* arm, const float* d_q, uint64_t n_traj, uint32_t n_wp,
                         float margin, float* d_cost, gvx_stream stream) {
  if (m == nullptr || (n_traj > 0 && (d_q == nullptr || d_cost == nullptr))) return fail(GVX_ERR_INVALID_ARG, "null argument");
  gvx_status st = check_arm(arm);
  if (st != GVX_OK) return st;
  return cuda_status(launch_traj_cost(m, *arm, d_q, n_traj, n_wp, margin, d_cost, as_stream(stream)), "trajectory cost");
}

gvx_status gvx_traj_cost_bwd(const gvx_dvm* m, const gvx_arm* arm, const float* d_q, uint64_t n_traj, uint32_t n_wp,
                             float margin, const float* d_grad_cost, float* d_grad_q, gvx_stream stream) {
  if (m == nullptr || (n_traj > 0 && (d_q == nullptr || d_grad_cost == nullptr || d_grad_q == nullptr)))
    return fail(GVX_ERR_INVALID_ARG, "null argument");
  gvx_status st = check_arm(arm);
  if (st != GVX_OK) return st;
  return cuda_status(launch_traj_cost_bwd(m, *arm, d_q, n_traj, n_wp, margin, d_grad_cost, d_grad_q, as_stream(stream)),
                     "trajectory cost adjoint");
}

/* ---- BitVectorVoxelMap ------------------------------------------------- */

gvx_status gvx_bvm_create(const gvx_dims* dims, float voxel_side, gvx_bvm** out) {
  if (out == nullptr) return fail(GVX_ERR_INVALID_ARG, "out is null");
  *out = nullptr;
  gvx_status st = check_dims(dims);
  if (st != GVX_OK) return st;
  if (!(voxel_side > 0.0f)) return fail(GVX_ERR_INVALID_ARG, "voxel side must be > 0");
  gvx_bvm* m = new (std::nothrow) gvx_bvm{*dims, voxel_side, nullptr};
  if (m == nullptr) return fail(GVX_ERR_OOM, "host allocation failed");
  const uint64_t bytes = num_voxels(*dims) * kBitVoxelBytes;
  cudaError_t e = cudaMalloc(&m->d_vox, bytes);
  if (e == cudaSuccess) e = cudaMemset(m->d_vox, 0, bytes);
  if (e == cudaSuccess) e = cudaMalloc(&m->d_occ, (num_voxels(*dims) + 31) / 32 * sizeof(uint32_t));
  if (e != cudaSuccess) {
    if (m->d_vox) cudaFree(m->d_vox);
    if (m->d_occ) cudaFree(m->d_occ);
    delete m;
    return cuda_status(e, "cudaMalloc(BitVectorVoxelMap)");
  }
  *out = m;
  return GVX_OK;
}

gvx_status gvx_bvm_destroy(gvx_bvm* m) {
  if (m == nullptr) return GVX_OK;
  cudaError_t e = m->d_vox ? cudaFree(m->d_vox) : cudaSuccess;
  if (m->d_flags) cudaFree(m->d_flags);
  if (m->d_colliding) cudaFree(m->d_colliding);
  if (m->d_occ) cudaFree(m->d_occ);
  delete m;
  return cuda_status(e, "cudaFree(BitVectorVoxelMap)");
}

gvx_status gvx_bvm_info(const gvx_bvm* m, gvx_dims* dims, float* voxel_side, uint8_t** d_voxels) {
  if (m == nullptr) return fail(GVX_ERR_INVALID_ARG, "map is null");
  if (dims) *dims = m->dims;
  if (voxel_side) *voxel_side = m->side;
  if (d_voxels) *d_voxels = m->d_vox;
  return GVX_OK;
}

gvx_status gvx_bvm_clear(gvx_bvm* m, gvx_stream stream) {
  if (m == nullptr) return fail(GVX_ERR_INVALID_ARG, "map is null");
  return cuda_status(cudaMemsetAsync(m->d_vox, 0, num_voxels(m->dims) * kBitVoxelBytes, as_stream(stream)), "clearMap(BitVoxelMap)");
}

gvx_status gvx_bvm_insert_points(gvx_bvm* m, const float* d_xyz, uint64_t n, uint32_t meaning, uint32_t* d_outside,
                                 gvx_stream stream) {
  if (m == nullptr || (n > 0 && d_xyz == nullptr)) return fail(GVX_ERR_INVALID_ARG, "null argument");
  if (meaning > 255) return fail(GVX_ERR_INVALID_ARG, "meaning must be in [0, 255]");
  return cuda_status(launch_bvm_insert(m->d_vox, m->dims, m->side, d_xyz, n, meaning, d_outside, as_stream(stream)),
                     "insertPointCloud(BitVoxelMap)");
}

gvx_status gvx_bvm_clear_bits(gvx_bvm* m, const uint8_t* bits, gvx_stream stream) {
  if (m == nullptr || bits == nullptr) return fail(GVX_ERR_INVALID_ARG, "null argument");
  uint32_t w[kBitVoxelWords];
  memcpy(w, bits, kBitVoxelBytes);
  return cuda_status(launch_bvm_clear_bits(m->d_vox, m->dims, w, as_stream(stream)), "clearBits(BitVoxelMap)");
}

gvx_status gvx_bvm_shift_swept_volume_ids(gvx_bvm* m, uint32_t shift, gvx_stream stream) {
  if (m == nullptr) return fail(GVX_ERR_INVALID_ARG, "map is null");
  if (shift > 56) return fail(GVX_ERR_INVALID_ARG, "maximum shift size is 56");
  return cuda_status(launch_bvm_shift(m->d_vox, m->dims, shift, as_stream(stream)), "shiftLeftSweptVolumeIDs");
}

gvx_status gvx_blist_clear_bits(gvx_blist* l, const uint8_t* bits, gvx_stream stream) {
  if (l == nullptr || bits == nullptr) return fail(GVX_ERR_INVALID_ARG, "null argument");
  if (l->n == 0) return GVX_OK;
  uint32_t w[kBitVoxelWords];
  memcpy(w, bits, kBitVoxelBytes);
  return cuda_status(launch_bvm_clear_bits(l->d_vox, gvx_dims{(uint32_t)l->n, 1u, 1u}, w, as_stream(stream)),
                     "clearBits(BitVoxelList)");
}

gvx_status gvx_blist_shift_swept_volume_ids(gvx_blist* l, uint32_t shift, gvx_stream stream) {
  if (l == nullptr) return fail(GVX_ERR_INVALID_ARG, "list is null");
  if (shift > 56) return fail(GVX_ERR_INVALID_ARG, "maximum shift size is 56");
  if (l->n == 0) return GVX_OK;
  return cuda_status(launch_bvm_shift(l->d_vox, gvx_dims{(uint32_t)l->n, 1u, 1u}, shift, as_stream(stream)),
                     "shiftLeftSweptVolumeIDs(BitVoxelList)");
}

gvx_status gvx_bvm_insert_meta_points_self_coll(gvx_bvm* m, const float* d_xyz, const uint64_t* offsets,
                                                uint32_t n_clouds, const uint8_t* meanings, const uint8_t* masks,
                                                uint8_t* colliding, int* any, uint32_t* d_outside, gvx_stream stream) {
  if (m == nullptr || offsets == nullptr || n_clouds == 0) return fail(GVX_ERR_INVALID_ARG, "need a map and at least one sub-cloud");
  uint64_t largest = 0;
  for (uint32_t k = 0; k < n_clouds; ++k) {
    if (offsets[k + 1] < offsets[k]) return fail(GVX_ERR_INVALID_ARG, "sub-cloud offsets must not decrease");
    largest = std::max<uint64_t>(largest, offsets[k + 1] - offsets[k]);
  }
  if (offsets[n_clouds] > offsets[0] && d_xyz == nullptr) return fail(GVX_ERR_INVALID_ARG, "points are null");
  // default meanings eBVM_SWEPT_VOLUME_START + k (4 .. 254) and masks: every
  // bit but eBVM_COLLISION and the sub-cloud's own meaning (BitVoxelMap.hpp:262-293)
  constexpr uint32_t kSweptStart = 4, kSweptEnd = 254;
  if (meanings == nullptr && n_clouds > kSweptEnd - kSweptStart + 1)
    return fail(GVX_ERR_INVALID_ARG, "more sub-clouds than swept-volume meanings; pass meanings");
  std::vector<uint8_t> mean(n_clouds);
  std::vector<uint32_t> mask((size_t)n_clouds * kBitVoxelWords);
  for (uint32_t k = 0; k < n_clouds; ++k) {
    mean[k] = meanings ? meanings[k] : (uint8_t)(kSweptStart + k);
    uint32_t* mk = mask.data() + (size_t)k * kBitVoxelWords;
    if (masks) {
      memcpy(mk, masks + (size_t)k * kBitVoxelBytes, kBitVoxelBytes);
    } else {
      for (uint32_t w = 0; w < kBitVoxelWords; ++w) mk[w] = 0xFFFFFFFFu;
      mk[kEbvmCollision >> 5] &= ~(1u << (kEbvmCollision & 31));
      mk[mean[k] >> 5] &= ~(1u << (mean[k] & 31));
    }
  }
  cudaError_t e = cudaSuccess;
  if (m->d_colliding == nullptr) e = cudaMalloc(&m->d_colliding, kBitVoxelBytes);
  if (e == cudaSuccess && largest > m->flags_cap) {  // grows with the largest sub-cloud seen
    if (m->d_flags) cudaFree(m->d_flags);
    m->d_flags = nullptr;
    m->flags_cap = 0;
    e = cudaMalloc(&m->d_flags, largest);
    if (e == cudaSuccess) m->flags_cap = largest;
  }
  if (e != cudaSuccess) return cuda_status(e, "insertMetaPointCloudWithSelfCollisionCheck workspace");
  cudaStream_t s = as_stream(stream);
  e = launch_meta_insert_self_coll(m->d_vox, m->dims, m->side, d_xyz, offsets, n_clouds, mean.data(), mask.data(),
                                   m->d_flags, m->d_colliding, d_outside, s);
  uint32_t host[kBitVoxelWords] = {};
  if (e == cudaSuccess) e = cudaMemcpyAsync(host, m->d_colliding, kBitVoxelBytes, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_status(e, "insertMetaPointCloudWithSelfCollisionCheck");
  if (colliding) memcpy(colliding, host, kBitVoxelBytes);
  if (any) {
    uint32_t o = 0;
    for (uint32_t w = 0; w < kBitVoxelWords; ++w) o |= host[w];
    *any = o != 0;
  }
  return GVX_OK;
}

gvx_status gvx_bvm_collide(gvx_bvm* self, const gvx_bvm* other, const int32_t offset[3], int mark, uint64_t* d_count,
                           gvx_stream stream) {
  if (self == nullptr || other == nullptr || d_count == nullptr) return fail(GVX_ERR_INVALID_ARG, "null argument");
  if (!same_dims(self->dims, other->dims)) return fail(GVX_ERR_INVALID_ARG, "maps differ in dimensions");
  return cuda_status(launch_bvm_collide(self->d_vox, other->d_vox, num_voxels(self->dims), linear_offset(self->dims, offset),
                                        mark, reinterpret_cast<unsigned long long*>(d_count), as_stream(stream)),
                     "collideWith(BitVectorVoxelMap)");
}

gvx_status gvx_bvm_collide_pvm(gvx_bvm* self, const gvx_pvm* other, float coll_threshold, const int32_t offset[3],
                               int mark, uint64_t* d_count, gvx_stream stream) {
  if (self == nullptr || other == nullptr || d_count == nullptr) return fail(GVX_ERR_INVALID_ARG, "null argument");
  if (!same_dims(self->dims, other->dims)) return fail(GVX_ERR_INVALID_ARG, "maps differ in dimensions");
  return cuda_status(launch_bvm_collide_pvm(self->d_vox, other->d_vox, num_voxels(self->dims),
                                            linear_offset(self->dims, offset), prob_threshold(coll_threshold), mark,
                                            reinterpret_cast<unsigned long long*>(d_count), as_stream(stream)),
                     "collideWith(ProbVoxelMap)");
}

/* ---- typed collisions ---------------------------------------------------- */

gvx_status gvx_bvm_collide_types(gvx_bvm* self, const gvx_bvm* other, uint64_t* d_count, uint8_t* d_types,
                                 gvx_stream stream) {
  if (self == nullptr || other == nullptr || d_count == nullptr) return fail(GVX_ERR_INVALID_ARG, "null argument");
  if (!same_dims(self->dims, other->dims)) return fail(GVX_ERR_INVALID_ARG, "maps differ in dimensions");
  return cuda_status(launch_bvm_collide_types(self->d_vox, other->d_vox, num_voxels(self->dims), 0, 0.f,
                                              reinterpret_cast<unsigned long long*>(d_count),
                                              reinterpret_cast<uint32_t*>(d_types), as_stream(stream)),
                     "collideWithTypes(BitVectorVoxelMap)");
}

gvx_status gvx_bvm_collide_types_pvm(gvx_bvm* self, const gvx_pvm* other, float coll_threshold, uint64_t* d_count,
                                     uint8_t* d_types, gvx_stream stream) {
  if (self == nullptr || other == nullptr || d_count == nullptr) return fail(GVX_ERR_INVALID_ARG, "null argument");
  if (!same_dims(self->dims, other->dims)) return fail(GVX_ERR_INVALID_ARG, "maps differ in dimensions");
  return cuda_status(launch_bvm_collide_types(self->d_vox, other->d_vox, num_voxels(self->dims), 1, coll_threshold,
                                              reinterpret_cast<unsigned long long*>(d_count),
                                              reinterpret_cast<uint32_t*>(d_types), as_stream(stream)),
                     "collideWithTypes(ProbVoxelMap)");
}

/* ---- ProbVoxelMap ------------------------------------------------------ */

gvx_status gvx_pvm_create(const gvx_dims* dims, float voxel_side, gvx_pvm** out) {
  if (out == nullptr) return fail(GVX_ERR_INVALID_ARG, "out is null");
  *out = nullptr;
  gvx_status st = check_dims(dims);
  if (st != GVX_OK) return st;
  if (!(voxel_side > 0.0f)) return fail(GVX_ERR_INVALID_ARG, "voxel side must be > 0");
  gvx_pvm* m = new (std::nothrow) gvx_pvm{*dims, voxel_side, nullptr};
  if (m == nullptr) return fail(GVX_ERR_OOM, "host allocation failed");
  const uint64_t bytes = (num_voxels(*dims) + 15) / 16 * 16;
  cudaError_t e = cudaMalloc(&m->d_vox, bytes);
  if (e == cudaSuccess) e = cudaMemset(m->d_vox, 0x80, bytes);  // UNKNOWN_PROBABILITY
  if (e != cudaSuccess) {
    if (m->d_vox) cudaFree(m->d_vox);
    delete m;
    return cuda_status(e, "cudaMalloc(ProbVoxelMap)");
  }
  *out = m;
  return GVX_OK;
}

gvx_status gvx_pvm_destroy(gvx_pvm* m) {
  if (m == nullptr) return GVX_OK;
  cudaError_t e = m->d_vox ? cudaFree(m->d_vox) : cudaSuccess;
  delete m;
  return cuda_status(e, "cudaFree(ProbVoxelMap)");
}

gvx_status gvx_pvm_info(const gvx_pvm* m, gvx_dims* dims, float* voxel_side, int8_t** d_voxels) {
  if (m == nullptr) return fail(GVX_ERR_INVALID_ARG, "map is null");
  if (dims) *dims = m->dims;
  if (voxel_side) *voxel_side = m->side;
  if (d_voxels) *d_voxels = m->d_vox;
  return GVX_OK;
}

gvx_status gvx_pvm_clear(gvx_pvm* m, gvx_stream stream) {
  if (m == nullptr) return fail(GVX_ERR_INVALID_ARG, "map is null");
  return cuda_status(cudaMemsetAsync(m->d_vox, 0x80, num_voxels(m->dims), as_stream(stream)), "clearMap(ProbVoxelMap)");
}

gvx_status gvx_pvm_insert_points(gvx_pvm* m, const float* d_xyz, uint64_t n, uint32_t meaning, uint32_t* d_outside,
                                 gvx_stream stream) {
  if (m == nullptr || (n > 0 && d_xyz == nullptr)) return fail(GVX_ERR_INVALID_ARG, "null argument");
  if (meaning > 255) return fail(GVX_ERR_INVALID_ARG, "meaning must be in [0, 255]");
  return cuda_status(launch_pvm_insert(m->d_vox, m->dims, m->side, d_xyz, n, meaning, d_outside, as_stream(stream)),
                     "insertPointCloud(ProbVoxelMap)");
}

gvx_status gvx_dvm_merge_occupied(gvx_dvm* m, const gvx_pvm* other, const uint32_t offset[3], float occupancy_threshold,
                                  gvx_stream stream) {
  if (m == nullptr || other == nullptr) return fail(GVX_ERR_INVALID_ARG, "null argument");
  if (!same_dims(m->dims, other->dims)) return fail(GVX_ERR_INVALID_ARG, "maps differ in dimensions");
  const uint32_t zero[3] = {0, 0, 0};
  return cuda_status(launch_merge_occupied(m->d_vox, other->d_vox, m->dims, offset ? offset : zero, occupancy_threshold,
                                           as_stream(stream)),
                     "mergeOccupied");
}

/* ---- BitVectorVoxelList ------------------------------------------------ */

gvx_status gvx_blist_create(const gvx_dims* ref_dims, float voxel_side, gvx_blist** out) {
  if (out == nullptr) return fail(GVX_ERR_INVALID_ARG, "out is null");
  *out = nullptr;
  gvx_status st = check_dims(ref_dims);
  if (st != GVX_OK) return st;
  if (!(voxel_side > 0.0f)) return fail(GVX_ERR_INVALID_ARG, "voxel side must be > 0");
  gvx_blist* l = new (std::nothrow) gvx_blist{*ref_dims, voxel_side, nullptr, nullptr, 0, 0};
  if (l == nullptr) return fail(GVX_ERR_OOM, "host allocation failed");
  *out = l;
  return GVX_OK;
}

gvx_status gvx_blist_destroy(gvx_blist* l) {
  if (l == nullptr) return GVX_OK;
  if (l->d_ids) cudaFree(l->d_ids);
  if (l->d_vox) cudaFree(l->d_vox);
  if (l->d_ids2) cudaFree(l->d_ids2);
  if (l->d_vox2) cudaFree(l->d_vox2);
  if (l->d_work) cudaFree(l->d_work);
  delete l;
  return GVX_OK;
}

gvx_status gvx_blist_size(const gvx_blist* l, uint64_t* n) {
  if (l == nullptr || n == nullptr) return fail(GVX_ERR_INVALID_ARG, "null argument");
  *n = l->n;
  return GVX_OK;
}

gvx_status gvx_blist_data(const gvx_blist* l, uint32_t** d_ids, uint8_t** d_voxels) {
  if (l == nullptr) return fail(GVX_ERR_INVALID_ARG, "list is null");
  if (d_ids) *d_ids = l->d_ids;
  if (d_voxels) *d_voxels = l->d_vox;
  return GVX_OK;
}

gvx_status gvx_blist_clear(gvx_blist* l) {
  if (l == nullptr) return fail(GVX_ERR_INVALID_ARG, "list is null");
  l->n = 0;
  return GVX_OK;
}

}  // extern "C"

namespace gvx {
namespace {

// Grow the list's storage to hold `cap` entries, keeping the first l->n.
cudaError_t blist_reserve(gvx_blist* l, uint64_t cap, cudaStream_t s) {
  if (cap <= l->cap) return cudaSuccess;
  uint32_t* ids = nullptr;
  uint8_t* vox = nullptr;
  cudaError_t e = cudaMalloc(&ids, cap * sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaMalloc(&vox, cap * kBitVoxelBytes);
  if (e == cudaSuccess && l->n) e = cudaMemcpyAsync(ids, l->d_ids, l->n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s);
  if (e == cudaSuccess && l->n) e = cudaMemcpyAsync(vox, l->d_vox, l->n * kBitVoxelBytes, cudaMemcpyDeviceToDevice, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    if (ids) cudaFree(ids);
    if (vox) cudaFree(vox);
    return e;
  }
  if (l->d_ids) cudaFree(l->d_ids);
  if (l->d_vox) cudaFree(l->d_vox);
  l->d_ids = ids;
  l->d_vox = vox;
  l->cap = cap;
  return cudaSuccess;
}

constexpr uint32_t kNoId = 0xFFFFFFFFu;

// Voxelise points into (id, source index) pairs for the list; out-of-bounds
// points get kNoId (remove_out_of_bounds, GV/voxellist/TemplateVoxelList.hpp:318-341).
__global__ void list_keys_kernel(const float* __restrict__ xyz, uint64_t n, gvx_dims d, float side, const uint32_t* old_ids,
                                 uint64_t n_old, uint32_t* __restrict__ keys, uint32_t* __restrict__ vals) {
  const uint64_t total = n_old + n;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t id;
    if (i < n_old) {
      id = old_ids[i];
    } else {
      const uint64_t p = i - n_old;
      const uint32_t x = coord_to_voxel(xyz[3 * p], side), y = coord_to_voxel(xyz[3 * p + 1], side),
                     z = coord_to_voxel(xyz[3 * p + 2], side);
      id = (x < d.x && y < d.y && z < d.z) ? z * d.x * d.y + y * d.x + x : kNoId;
    }
    keys[i] = id;
    vals[i] = (uint32_t)i;
  }
}

// make_unique (TemplateVoxelList.hpp:143-212): heads of equal-id runs.
__global__ void list_heads_kernel(const uint32_t* __restrict__ keys, uint64_t n, uint32_t* __restrict__ head) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    head[i] = (keys[i] != kNoId && (i == 0 || keys[i] != keys[i - 1])) ? 1u : 0u;
}

// OR-merge every run into one entry.  Source voxels: old entries (index <
// n_old) come from old_vox, new points carry only bit `meaning`.
__global__ void list_merge_kernel(const uint32_t* __restrict__ keys, const uint32_t* __restrict__ vals, uint64_t n,
                                  const uint32_t* __restrict__ head, const uint32_t* __restrict__ pos,
                                  const uint32_t* __restrict__ old_vox, uint64_t n_old, uint32_t meaning,
                                  uint32_t* __restrict__ out_ids, uint32_t* __restrict__ out_vox) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    if (!head[i]) continue;
    uint32_t acc[kBitVoxelWords] = {0, 0, 0, 0, 0, 0, 0, 0};
    const uint32_t key = keys[i];
    for (uint64_t k = i; k < n && keys[k] == key; ++k) {
      const uint32_t src = vals[k];
      if (src < n_old) {
        for (int w = 0; w < (int)kBitVoxelWords; ++w) acc[w] |= old_vox[(uint64_t)src * kBitVoxelWords + w];
      } else {
        acc[meaning >> 5] |= 1u << (meaning & 31);
      }
    }
    const uint32_t o = pos[i];
    out_ids[o] = key;
    for (int w = 0; w < (int)kBitVoxelWords; ++w) out_vox[(uint64_t)o * kBitVoxelWords + w] = acc[w];
  }
}

// Grow-only device buffer: reallocated (contents dropped) only when `need`
// exceeds what it holds, then with headroom so slowly growing inputs
// reallocate rarely.  cudaFree waits for work still using the old buffer.
cudaError_t grow(void** p, size_t* have, size_t need) {
  if (need <= *have && *p != nullptr) return cudaSuccess;
  if (*p) cudaFree(*p);
  *p = nullptr;
  *have = 0;
  const size_t bytes = std::max<size_t>(need + need / 4, 4096);
  cudaError_t e = cudaMalloc(p, bytes);
  if (e == cudaSuccess) *have = bytes;
  return e;
}

// Spare list storage for at least `cap` entries (the merged list's target).
cudaError_t blist_spare(gvx_blist* l, uint64_t cap) {
  if (cap <= l->cap2 && l->d_ids2 != nullptr) return cudaSuccess;
  size_t have_i = 0, have_v = 0;
  void* ids = l->d_ids2;
  void* vox = l->d_vox2;
  cudaError_t e = grow(&ids, &have_i, cap * sizeof(uint32_t));
  if (e == cudaSuccess) e = grow(&vox, &have_v, cap * kBitVoxelBytes);
  l->d_ids2 = static_cast<uint32_t*>(ids);
  l->d_vox2 = static_cast<uint8_t*>(vox);
  l->cap2 = e == cudaSuccess ? std::min<uint64_t>(have_i / sizeof(uint32_t), have_v / kBitVoxelBytes) : 0;
  return e;
}

inline size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

}  // namespace
}  // namespace gvx

extern "C" {

gvx_status gvx_blist_insert_points(gvx_blist* l, const float* d_xyz, uint64_t n, uint32_t meaning, gvx_stream stream) {
  if (l == nullptr || (n > 0 && d_xyz == nullptr)) return fail(GVX_ERR_INVALID_ARG, "null argument");
  if (meaning > 255) return fail(GVX_ERR_INVALID_ARG, "meaning must be in [0, 255]");
  if (n == 0) return GVX_OK;
  cudaStream_t s = as_stream(stream);
  const uint64_t total = l->n + n;
  if (total >= 0xFFFFFFFFull) return fail(GVX_ERR_OUT_OF_DOMAIN, "list too long");
  // work area: keys, vals, sorted keys, sorted vals, run heads, run positions
  // (total words each), then CUB's temporary storage
  size_t sort_bytes = 0, scan_bytes = 0;
  cudaError_t e = cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, (uint32_t*)nullptr, (uint32_t*)nullptr,
                                                  (uint32_t*)nullptr, (uint32_t*)nullptr, (int64_t)total, 0, 32, s);
  if (e == cudaSuccess)
    e = cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, (uint32_t*)nullptr, (uint32_t*)nullptr, (int64_t)total, s);
  if (e != cudaSuccess) return cuda_status(e, "list sort sizing");
  const size_t arr = align256(total * 4);
  if ((e = grow(&l->d_work, &l->work_bytes, 6 * arr + align256(std::max(sort_bytes, scan_bytes)))) != cudaSuccess)
    return cuda_status(e, "list insert buffers");
  char* w = static_cast<char*>(l->d_work);
  uint32_t* keys = reinterpret_cast<uint32_t*>(w);
  uint32_t* vals = reinterpret_cast<uint32_t*>(w + arr);
  uint32_t* keys2 = reinterpret_cast<uint32_t*>(w + 2 * arr);
  uint32_t* vals2 = reinterpret_cast<uint32_t*>(w + 3 * arr);
  uint32_t* head = reinterpret_cast<uint32_t*>(w + 4 * arr);
  uint32_t* pos = reinterpret_cast<uint32_t*>(w + 5 * arr);
  void* tmp = w + 6 * arr;
  const unsigned blocks = (unsigned)std::min<uint64_t>((total + 255) / 256, 4096);
  list_keys_kernel<<<blocks, 256, 0, s>>>(d_xyz, n, l->ref, l->side, l->d_ids, l->n, keys, vals);
  e = cub::DeviceRadixSort::SortPairs(tmp, sort_bytes, keys, keys2, vals, vals2, (int64_t)total, 0, 32, s);
  if (e != cudaSuccess) return cuda_status(e, "list sort");
  list_heads_kernel<<<blocks, 256, 0, s>>>(keys2, total, head);
  e = cub::DeviceScan::ExclusiveSum(tmp, scan_bytes, head, pos, (int64_t)total, s);
  uint32_t last_head = 0, last_pos = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&last_head, head + total - 1, 4, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&last_pos, pos + total - 1, 4, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);  // the merged list's length sizes its storage
  if (e != cudaSuccess) return cuda_status(e, "list scan");
  const uint64_t n_out = (uint64_t)last_pos + last_head;
  if ((e = blist_spare(l, n_out)) != cudaSuccess) return cuda_status(e, "list output");
  list_merge_kernel<<<blocks, 256, 0, s>>>(keys2, vals2, total, head, pos, reinterpret_cast<const uint32_t*>(l->d_vox),
                                           l->n, meaning, l->d_ids2, reinterpret_cast<uint32_t*>(l->d_vox2));
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);  // blocking, as the reference's insert
  if (e != cudaSuccess) return cuda_status(e, "list merge");
  // the merged list becomes the list; the old storage is the next call's spare
  std::swap(l->d_ids, l->d_ids2);
  std::swap(l->d_vox, l->d_vox2);
  std::swap(l->cap, l->cap2);
  l->n = n_out;
  return GVX_OK;
}

gvx_status gvx_blist_set(gvx_blist* l, const uint32_t* d_ids, const uint8_t* d_voxels, uint64_t n, uint32_t meaning,
                         gvx_stream stream) {
  if (l == nullptr || (n > 0 && d_ids == nullptr)) return fail(GVX_ERR_INVALID_ARG, "null argument");
  if (meaning > 255) return fail(GVX_ERR_INVALID_ARG, "meaning must be in [0, 255]");
  cudaStream_t s = as_stream(stream);
  l->n = 0;
  cudaError_t e = blist_reserve(l, n, s);
  if (e != cudaSuccess) return cuda_status(e, "list storage");
  if (n == 0) return GVX_OK;
  e = cudaMemcpyAsync(l->d_ids, d_ids, n * 4, cudaMemcpyDeviceToDevice, s);
  if (e == cudaSuccess) {
    if (d_voxels) {
      e = cudaMemcpyAsync(l->d_vox, d_voxels, n * kBitVoxelBytes, cudaMemcpyDeviceToDevice, s);
    } else {
      // every voxel gets bit `meaning`: byte pattern written with a 2D memset per byte column
      e = cudaMemsetAsync(l->d_vox, 0, n * kBitVoxelBytes, s);
      if (e == cudaSuccess)
        e = cudaMemset2DAsync(l->d_vox + (meaning >> 3), kBitVoxelBytes, (int)(1u << (meaning & 7)), 1, n, s);
    }
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_status(e, "list set");
  l->n = n;
  return GVX_OK;
}

gvx_status gvx_blist_collide_types_bvm(gvx_blist* l, const gvx_bvm* map, const int32_t offset[3], uint64_t* d_count,
                                       uint8_t* d_types, gvx_stream stream) {
  if (l == nullptr || map == nullptr || d_count == nullptr) return fail(GVX_ERR_INVALID_ARG, "null argument");
  if (!same_dims(l->ref, map->dims)) return fail(GVX_ERR_INVALID_ARG, "the list's reference dims differ from the map's");
  return cuda_status(launch_list_collide_types(l->d_ids, l->d_vox, l->n, map->d_vox, num_voxels(map->dims), 0, 0.f,
                                               linear_offset(map->dims, offset), nullptr,
                                               reinterpret_cast<unsigned long long*>(d_count),
                                               reinterpret_cast<uint32_t*>(d_types), as_stream(stream)),
                     "collideWithTypes(list, BitVectorVoxelMap)");
}

gvx_status gvx_blist_collide_types_pvm(gvx_blist* l, const gvx_pvm* map, float coll_threshold, const int32_t offset[3],
                                       uint64_t* d_count, uint8_t* d_types, gvx_stream stream) {
  if (l == nullptr || map == nullptr || d_count == nullptr) return fail(GVX_ERR_INVALID_ARG, "null argument");
  if (!same_dims(l->ref, map->dims)) return fail(GVX_ERR_INVALID_ARG, "the list's reference dims differ from the map's");
  return cuda_status(launch_list_collide_types(l->d_ids, l->d_vox, l->n, map->d_vox, num_voxels(map->dims), 1,
                                               coll_threshold, linear_offset(map->dims, offset), nullptr,
                                               reinterpret_cast<unsigned long long*>(d_count),
                                               reinterpret_cast<uint32_t*>(d_types), as_stream(stream)),
                     "collideWithTypes(list, ProbVoxelMap)");
}

gvx_status gvx_blist_collide_type_mask_bvm(gvx_blist* l, const gvx_bvm* map, const uint8_t* d_mask, const int32_t offset[3],
                                           uint64_t* d_count, gvx_stream stream) {
  if (l == nullptr || map == nullptr || d_mask == nullptr || d_count == nullptr)
    return fail(GVX_ERR_INVALID_ARG, "null argument");
  if (!same_dims(l->ref, map->dims)) return fail(GVX_ERR_INVALID_ARG, "the list's reference dims differ from the map's");
  return cuda_status(launch_list_collide_types(l->d_ids, l->d_vox, l->n, map->d_vox, num_voxels(map->dims), 0, 0.f,
                                               linear_offset(map->dims, offset), d_mask,
                                               reinterpret_cast<unsigned long long*>(d_count), nullptr,
                                               as_stream(stream)),
                     "collideWithTypeMask");
}

gvx_status gvx_blist_collide_types_blist(const gvx_blist* l, const gvx_blist* other, uint64_t* d_count, uint8_t* d_types,
                                         gvx_stream stream) {
  if (l == nullptr || other == nullptr || d_count == nullptr) return fail(GVX_ERR_INVALID_ARG, "null argument");
  return cuda_status(launch_list_list_types(l->d_ids, l->d_vox, l->n, other->d_ids, other->d_vox, other->n,
                                            reinterpret_cast<unsigned long long*>(d_count),
                                            reinterpret_cast<uint32_t*>(d_types), as_stream(stream)),
                     "collideWithTypes(list, list)");
}

gvx_status gvx_dvm_extract_distances(const gvx_dvm* m, int8_t* d_out, int robot_radius, gvx_stream stream) {
  if (m == nullptr || d_out == nullptr) return fail(GVX_ERR_INVALID_ARG, "null argument");
  return cuda_status(launch_extract_distances(m->d_vox, m->dims, robot_radius, d_out, as_stream(stream)), "extract_distances");
}

gvx_status gvx_dvm_init_floodfill(const gvx_dvm* m, const int8_t* d_distances, int16_t* d_manhattan, int robot_radius,
                                  gvx_stream stream) {
  if (m == nullptr || d_distances == nullptr || d_manhattan == nullptr) return fail(GVX_ERR_INVALID_ARG, "null argument");
  return cuda_status(launch_init_floodfill(d_distances, d_manhattan, num_voxels(m->dims), robot_radius, as_stream(stream)),
                     "init_floodfill");
}

gvx_status gvx_extract_given_distances(const gvx_dvm* m, int min_dist, int max_dist, gvx_blist* result, uint64_t* n_out,
                                       gvx_stream stream) {
  if (m == nullptr || result == nullptr) return fail(GVX_ERR_INVALID_ARG, "null argument");
  if (!same_dims(m->dims, result->ref)) return fail(GVX_ERR_INVALID_ARG, "the list's reference dims differ from the map's");
  if (min_dist < -128 || min_dist > 127 || max_dist < -128 || max_dist > 127)
    return fail(GVX_ERR_OUT_OF_DOMAIN, "distance bounds are free_space_t (int8) values");
  cudaStream_t s = as_stream(stream);
  const uint64_t nt = band_tiles(m->dims);
  uint32_t* tiles = nullptr;
  cudaError_t e = cudaMalloc(&tiles, (nt + 1) * sizeof(uint32_t));
  if (e == cudaSuccess) e = launch_band_count(m->d_vox, m->dims, min_dist, max_dist, tiles, s);
  uint32_t total = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&total, tiles + nt, sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  result->n = 0;
  if (e == cudaSuccess) e = blist_reserve(result, total, s);
  if (e == cudaSuccess && total > 0) e = launch_band_write(m->d_vox, m->dims, min_dist, max_dist, tiles, result->d_ids,
                                                           result->d_vox, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (tiles) cudaFree(tiles);
  if (e != cudaSuccess) return cuda_status(e, "extract_given_distances");
  result->n = total;
  if (n_out) *n_out = total;
  return GVX_OK;
}

gvx_status gvx_blist_collide_bvm(gvx_blist* l, const gvx_bvm* map, const int32_t offset[3], int mark, uint64_t* d_count,
                                 gvx_stream stream) {
  if (l == nullptr || map == nullptr || d_count == nullptr) return fail(GVX_ERR_INVALID_ARG, "null argument");
  if (!same_dims(l->ref, map->dims))
    return fail(GVX_ERR_INVALID_ARG, "the list's reference map dimensions differ from the colliding map's");
  return cuda_status(launch_list_collide_map(l->d_ids, l->d_vox, l->n, map->d_vox, num_voxels(map->dims),
                                             linear_offset(map->dims, offset), mark,
                                             reinterpret_cast<unsigned long long*>(d_count), as_stream(stream)),
                     "collideWith(BitVoxelList, BitVectorVoxelMap)");
}

gvx_status gvx_blist_collide_pvm(gvx_blist* l, const gvx_pvm* map, float coll_threshold, const int32_t offset[3],
                                 int mark, uint64_t* d_count, gvx_stream stream) {
  if (l == nullptr || map == nullptr || d_count == nullptr) return fail(GVX_ERR_INVALID_ARG, "null argument");
  if (!same_dims(l->ref, map->dims))
    return fail(GVX_ERR_INVALID_ARG, "the list's reference map dimensions differ from the colliding map's");
  return cuda_status(launch_list_collide_pvm(l->d_ids, l->d_vox, l->n, map->d_vox, num_voxels(map->dims),
                                             linear_offset(map->dims, offset), prob_threshold(coll_threshold), mark,
                                             reinterpret_cast<unsigned long long*>(d_count), as_stream(stream)),
                     "collideWith(BitVoxelList, ProbVoxelMap)");
}

gvx_status gvx_blist_collide_blist(const gvx_blist* l, const gvx_blist* other, const int32_t offset[3], uint64_t* d_count,
                                   gvx_stream stream) {
  if (l == nullptr || other == nullptr || d_count == nullptr) return fail(GVX_ERR_INVALID_ARG, "null argument");
  if (offset != nullptr && (offset[0] != 0 || offset[1] != 0 || offset[2] != 0))
    return fail(GVX_ERR_INVALID_ARG, "offset for voxel-list collision is not supported");
  return cuda_status(launch_list_collide_list(l->d_ids, l->n, other->d_ids, other->n,
                                              reinterpret_cast<unsigned long long*>(d_count), as_stream(stream)),
                     "collideWith(BitVoxelList, BitVoxelList)");
}

gvx_status gvx_lists_collide_bvm(const uint32_t* d_ids, uint8_t* d_voxels, const uint64_t* d_offsets, uint32_t n_lists,
                                 uint64_t n_total, const gvx_bvm* map, int mark, uint64_t* d_counts, gvx_stream stream) {
  if (map == nullptr || d_offsets == nullptr || d_counts == nullptr || (n_total > 0 && (d_ids == nullptr || d_voxels == nullptr)))
    return fail(GVX_ERR_INVALID_ARG, "null argument");
  if (n_lists == 0) return GVX_OK;
  return cuda_status(launch_lists_collide_map(d_ids, d_voxels, d_offsets, n_lists, n_total, map->d_vox,
                                              num_voxels(map->dims), mark,
                                              reinterpret_cast<unsigned long long*>(d_counts), as_stream(stream),
                                              map->d_occ),
                     "batched list collision");
}

}  // extern "C"
