// TEST INFRASTRUCTURE ONLY -- builds oracle/_ref/libgvref.so.
//
// Runs gpu-voxels' OWN CUDA kernels (included from the reference source tree
// at build time, never copied) so that the CPU oracle and the product can be
// checked against the reference's actual output on the same B200.  This file
// only restates the host-side launch sequences, with the reference's own
// launch shapes:
//   DistanceVoxelMap::parallelBanding3D   GV/voxelmap/DistanceVoxelMap.hpp:284-645
//   TemplateVoxelMap::insertPointCloud    GV/voxelmap/TemplateVoxelMap.hpp:689-709
//   collisionCheckWithCounterRelativeTransform  GV/voxelmap/TemplateVoxelMap.hpp:588-621
//   collisionCheckWithCollider (list)     GV/voxellist/TemplateVoxelList.hpp:1170-1213
//   computeLinearLoad                     GV/helpers/MathHelpers.cpp:29-83
// (GV = packages/gpu_voxels/src/gpu_voxels/).  Built by oracle/Makefile `ref`.
#include <gpu_voxels/voxelmap/kernels/VoxelMapOperationsPBA.hpp>
#include <gpu_voxels/voxel/DefaultCollider.hpp>
// The list kernel names voxelmap::getHighestVoxelPtr unqualified; the
// reference's own translation units see it through their using-directives.
#include <gpu_voxels/voxelmap/kernels/VoxelMapOperations.h>
namespace gpu_voxels { namespace voxellist { using voxelmap::getHighestVoxelPtr; } }
#include <gpu_voxels/voxellist/kernels/VoxelListOperations.hpp>

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstring>
#include <vector>

using namespace gpu_voxels;
using namespace gpu_voxels::voxelmap;

namespace {

// computeLinearLoad (GV/helpers/MathHelpers.cpp:29-83), restated: 1024
// threads per block, at most cMAX_NR_OF_BLOCKS blocks (kernels grid-stride).
void linear_load(uint32_t n, uint32_t* blocks, uint32_t* threads) {
  if (n == 0) { *blocks = 1; *threads = 1; return; }
  *threads = cMAX_THREADS_PER_BLOCK;
  if (n <= cMAX_NR_OF_BLOCKS * cMAX_THREADS_PER_BLOCK) *blocks = (n + cMAX_THREADS_PER_BLOCK - 1) / cMAX_THREADS_PER_BLOCK;
  else *blocks = cMAX_NR_OF_BLOCKS;
}

int check(cudaError_t e) { return e == cudaSuccess ? 0 : (int)e; }

// The launch sequence of parallelBanding3D on device buffers.
int pba_device(DistanceVoxel* map, DistanceVoxel* initial, Vector3ui dim, uint32_t m1, uint32_t m2, uint32_t m3,
               cudaStream_t s, cudaEvent_t* ev_begin, cudaEvent_t* ev_end) {
  const uint32_t bs1 = PBA_DEFAULT_M1_BLOCK_SIZE, bs2 = PBA_DEFAULT_M2_BLOCK_SIZE, bs3 = PBA_DEFAULT_M3_BLOCK_SIZE;
  m1 = std::max(1u, std::min(m1, dim.z));
  m2 = std::max(1u, std::min(m2, dim.y));
  m3 = std::max(1u, std::min(m3, dim.y));
  if (dim.z % m1) m1 = 1;
  if ((dim.x % m2) || (dim.y % m2)) m2 = 1;
  if ((dim.x % m3) || (dim.y % m3)) m3 = 1;
  const size_t n = (size_t)dim.x * dim.y * dim.z;
  if (ev_begin) cudaEventRecord(*ev_begin, s);
  // thrust::device_vector initial_map(original) -- a device copy (:342)
  cudaMemcpyAsync(initial, map, n * sizeof(DistanceVoxel), cudaMemcpyDeviceToDevice, s);
  thrust::device_ptr<DistanceVoxel> dmap(map), dinit(initial);
  dim3 m1_block(std::min(bs1, dim.x));
  dim3 m1_grid(dim.x / m1_block.x, dim.y, m1);
  kernelPBAphase1FloodZ<<<m1_grid, m1_block, 0, s>>>(dmap, dmap, dim, dim.z / m1);
  if (m1 > 1) {
    kernelPBAphase1PropagateInterband<<<m1_grid, m1_block, 0, s>>>(dmap, dinit, dim, dim.z / m1);
    kernelPBAphase1Update<<<m1_grid, m1_block, 0, s>>>(dinit, dmap, dim, dim.z / m1);
  }
  dim3 m2_block(std::min(bs2, std::min(dim.x, dim.y)));
  dim3 m2_grid(dim.x / m2_block.x, m2, dim.z);
  thrust::device_ptr<pba_fw_ptr_t> fw((pba_fw_ptr_t*)map);
  cudaResourceDesc rd;
  memset(&rd, 0, sizeof(rd));
  rd.resType = cudaResourceTypeLinear;
  rd.res.linear.devPtr = initial;
  rd.res.linear.sizeInBytes = n * sizeof(int);
  rd.res.linear.desc.f = cudaChannelFormatKindSigned;
  rd.res.linear.desc.x = 32;
  cudaTextureDesc td;
  memset(&td, 0, sizeof(td));
  td.addressMode[0] = cudaAddressModeClamp;
  td.filterMode = cudaFilterModePoint;
  td.readMode = cudaReadModeElementType;
  td.normalizedCoords = 0;
  cudaTextureObject_t tex = 0;
  cudaError_t e = cudaCreateTextureObject(&tex, &rd, &td, nullptr);
  if (e != cudaSuccess) return check(e);
  dim3 m3_block(std::min(bs3, std::min(dim.x, dim.y)), m3);
  dim3 m3_grid(dim.x / m3_block.x, 1, dim.z);
  dim3 tr_block(PBA_TILE_DIM, PBA_TILE_DIM);
  dim3 tr_grid(dim.x / tr_block.x, dim.y / tr_block.y, dim.z);
  for (int pass = 0; pass < 2; ++pass) {
    kernelPBAphase2ProximateBackpointers<<<m2_grid, m2_block, 0, s>>>(dmap, dinit, dim, dim.y / m2);
    if (m2 > 1) kernelPBAphase2CreateForwardPointers<<<m2_grid, m2_block, 0, s>>>(dinit, fw, dim, dim.y / m2);
    for (uint32_t bc = m2; bc > 1; bc /= 2) {
      dim3 mg(dim.x / m2_block.x, bc / 2, dim.z);
      kernelPBAphase2MergeBands<<<mg, m2_block, 0, s>>>(dinit, fw, dim, dim.y / bc);
    }
    kernelPBAphase3Distances<<<m3_grid, m3_block, 0, s>>>(tex, dmap, dim);
    kernelPBA3DTransposeXY<<<tr_grid, tr_block, 0, s>>>(dmap);
  }
  if (ev_end) cudaEventRecord(*ev_end, s);
  e = cudaStreamSynchronize(s);
  cudaDestroyTextureObject(tex);
  if (e != cudaSuccess) return check(e);
  return check(cudaGetLastError());
}

}  // namespace

extern "C" {

int ref_available(void) {
  int n = 0;
  return cudaGetDeviceCount(&n) == cudaSuccess && n > 0;
}

// Reference EDT on a host map (uint32 DistanceVoxels, modified in place).
int ref_pba(uint32_t* h_map, const uint32_t dims[3], uint32_t m1, uint32_t m2, uint32_t m3) {
  const Vector3ui dim(dims[0], dims[1], dims[2]);
  const size_t n = (size_t)dims[0] * dims[1] * dims[2];
  DistanceVoxel *map = nullptr, *init = nullptr;
  if (cudaMalloc(&map, n * 4) != cudaSuccess) return -1;
  if (cudaMalloc(&init, n * 4) != cudaSuccess) { cudaFree(map); return -1; }
  int rc = check(cudaMemcpy(map, h_map, n * 4, cudaMemcpyHostToDevice));
  if (!rc) rc = pba_device(map, init, dim, m1, m2, m3, 0, nullptr, nullptr);
  if (!rc) rc = check(cudaMemcpy(h_map, map, n * 4, cudaMemcpyDeviceToHost));
  cudaFree(map);
  cudaFree(init);
  return rc;
}

// Reference EDT timing: `iters` runs on a device copy of h_map (the map is
// re-uploaded before each run); returns the mean milliseconds per EDT.
int ref_pba_time(const uint32_t* h_map, const uint32_t dims[3], int iters, float* ms_out) {
  const Vector3ui dim(dims[0], dims[1], dims[2]);
  const size_t n = (size_t)dims[0] * dims[1] * dims[2];
  DistanceVoxel *src = nullptr, *map = nullptr, *init = nullptr;
  if (cudaMalloc(&src, n * 4) || cudaMalloc(&map, n * 4) || cudaMalloc(&init, n * 4)) return -1;
  int rc = check(cudaMemcpy(src, h_map, n * 4, cudaMemcpyHostToDevice));
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  float total = 0.f;
  for (int it = 0; it < iters + 1 && !rc; ++it) {
    cudaMemcpy(map, src, n * 4, cudaMemcpyDeviceToDevice);
    rc = pba_device(map, init, dim, 1, 1, 1, 0, &a, &b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    if (it > 0) total += ms;  // first run is a warm-up
  }
  *ms_out = iters > 0 ? total / iters : 0.f;
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(src);
  cudaFree(map);
  cudaFree(init);
  return rc;
}

// kernelInsertGlobalPointCloud<DistanceVoxel> with the reference's launch sizing.
int ref_dvm_insert(uint32_t* h_map, const uint32_t dims[3], float side, const float* h_xyz, uint32_t n, int* outside) {
  const Vector3ui dim(dims[0], dims[1], dims[2]);
  const size_t nv = (size_t)dims[0] * dims[1] * dims[2];
  DistanceVoxel* map = nullptr;
  Vector3f* pts = nullptr;
  bool* flag = nullptr;
  if (cudaMalloc(&map, nv * 4) || cudaMalloc(&pts, (size_t)n * sizeof(Vector3f) + 4) || cudaMalloc(&flag, 1)) return -1;
  cudaMemcpy(map, h_map, nv * 4, cudaMemcpyHostToDevice);
  cudaMemcpy(pts, h_xyz, (size_t)n * 12, cudaMemcpyHostToDevice);
  cudaMemset(flag, 0, 1);
  uint32_t blocks, threads;
  linear_load(n, &blocks, &threads);
  kernelInsertGlobalPointCloud<<<blocks, threads>>>(map, dim, side, pts, n, eBVM_OCCUPIED, flag);
  int rc = check(cudaDeviceSynchronize());
  bool f = false;
  cudaMemcpy(&f, flag, 1, cudaMemcpyDeviceToHost);
  *outside = f ? 1 : 0;
  if (!rc) rc = check(cudaMemcpy(h_map, map, nv * 4, cudaMemcpyDeviceToHost));
  cudaFree(map);
  cudaFree(pts);
  cudaFree(flag);
  return rc;
}

// kernelCollideVoxelMapsDebug with DefaultCollider on two BitVectorVoxel maps
// (host arrays of 32-byte voxels); `self` receives the collision marks.
// Zero offset only: the reference shifts the base pointer without a bounds
// check (TemplateVoxelMap.hpp:596-600), which this driver never exercises.
int ref_bvm_collide(uint8_t* h_self, const uint8_t* h_other, uint32_t nvox, uint64_t* count) {
  BitVectorVoxel *a = nullptr, *b = nullptr;
  uint16_t* res = nullptr;
  const size_t bytes = (size_t)nvox * sizeof(BitVectorVoxel);
  if (cudaMalloc(&a, bytes) || cudaMalloc(&b, bytes) || cudaMalloc(&res, cMAX_NR_OF_BLOCKS * sizeof(uint16_t))) return -1;
  cudaMemcpy(a, h_self, bytes, cudaMemcpyHostToDevice);
  cudaMemcpy(b, h_other, bytes, cudaMemcpyHostToDevice);
  cudaMemset(res, 0, cMAX_NR_OF_BLOCKS * sizeof(uint16_t));
  uint32_t blocks, threads;
  linear_load(nvox, &blocks, &threads);
  DefaultCollider collider(1.0f);
  kernelCollideVoxelMapsDebug<<<blocks, threads>>>(a, nvox, b, collider, res);
  int rc = check(cudaDeviceSynchronize());
  std::vector<uint16_t> h(cMAX_NR_OF_BLOCKS);
  cudaMemcpy(h.data(), res, cMAX_NR_OF_BLOCKS * sizeof(uint16_t), cudaMemcpyDeviceToHost);
  uint64_t c = 0;
  for (uint32_t i = 0; i < blocks; ++i) c += h[i];
  *count = c;
  if (!rc) rc = check(cudaMemcpy(h_self, a, bytes, cudaMemcpyDeviceToHost));
  cudaFree(a);
  cudaFree(b);
  cudaFree(res);
  return rc;
}

// kernelCollideVoxelMapsDebug with DefaultCollider(coll_threshold) on a
// BitVectorVoxel map (self, marked) against a ProbVoxelMap (one int8
// occupancy per voxel), as BitVoxelMap::collideWith(const ProbVoxelMap*)
// (GV/voxelmap/BitVoxelMap.hpp:205-210) launches it; zero offset.
int ref_bvm_collide_pvm(uint8_t* h_self, const int8_t* h_other, uint32_t nvox, float coll_threshold, uint64_t* count) {
  static_assert(sizeof(ProbabilisticVoxel) == 1, "one occupancy byte per voxel");
  BitVectorVoxel* a = nullptr;
  ProbabilisticVoxel* b = nullptr;
  uint16_t* res = nullptr;
  const size_t bytes = (size_t)nvox * sizeof(BitVectorVoxel);
  if (cudaMalloc(&a, bytes) || cudaMalloc(&b, nvox) || cudaMalloc(&res, cMAX_NR_OF_BLOCKS * sizeof(uint16_t))) return -1;
  cudaMemcpy(a, h_self, bytes, cudaMemcpyHostToDevice);
  cudaMemcpy(b, h_other, nvox, cudaMemcpyHostToDevice);
  cudaMemset(res, 0, cMAX_NR_OF_BLOCKS * sizeof(uint16_t));
  uint32_t blocks, threads;
  linear_load(nvox, &blocks, &threads);
  DefaultCollider collider(coll_threshold);
  kernelCollideVoxelMapsDebug<<<blocks, threads>>>(a, nvox, b, collider, res);
  int rc = check(cudaDeviceSynchronize());
  std::vector<uint16_t> h(cMAX_NR_OF_BLOCKS);
  cudaMemcpy(h.data(), res, cMAX_NR_OF_BLOCKS * sizeof(uint16_t), cudaMemcpyDeviceToHost);
  uint64_t c = 0;
  for (uint32_t i = 0; i < blocks; ++i) c += h[i];
  *count = c;
  if (!rc) rc = check(cudaMemcpy(h_self, a, bytes, cudaMemcpyDeviceToHost));
  cudaFree(a);
  cudaFree(b);
  cudaFree(res);
  return rc;
}

// kernelCollideWithVoxelMap<BitVectorVoxel, ProbabilisticVoxel, DefaultCollider>
// for one list, as BitVoxelList::collideWith(const ProbVoxelMap*)
// (GV/voxellist/BitVoxelList.hpp:63-69 -> TemplateVoxelList.hpp:1170-1213)
// launches it; the list voxels receive the marks.
int ref_list_collide_pvm(const uint32_t* h_ids, uint8_t* h_list_vox, uint32_t n, const int8_t* h_map,
                         const uint32_t dims[3], const int32_t offset[3], float coll_threshold, uint64_t* h_count) {
  const Vector3ui dim(dims[0], dims[1], dims[2]);
  const Vector3i off(offset[0], offset[1], offset[2]);
  const uint64_t nvox = (uint64_t)dims[0] * dims[1] * dims[2];
  ProbabilisticVoxel* map = nullptr;
  BitVectorVoxel* lvox = nullptr;
  MapVoxelID* ids = nullptr;
  uint16_t* res = nullptr;
  if (cudaMalloc(&map, nvox) || cudaMalloc(&lvox, ((size_t)n + 1) * sizeof(BitVectorVoxel)) ||
      cudaMalloc(&ids, ((size_t)n + 1) * sizeof(MapVoxelID)) || cudaMalloc(&res, cMAX_NR_OF_BLOCKS * sizeof(uint16_t))) {
    cudaFree(map); cudaFree(lvox); cudaFree(ids); cudaFree(res);
    return -1;
  }
  int rc = check(cudaMemcpy(map, h_map, nvox, cudaMemcpyHostToDevice));
  if (!rc) rc = check(cudaMemcpy(lvox, h_list_vox, (size_t)n * sizeof(BitVectorVoxel), cudaMemcpyHostToDevice));
  if (!rc) rc = check(cudaMemcpy(ids, h_ids, (size_t)n * sizeof(MapVoxelID), cudaMemcpyHostToDevice));
  uint32_t blocks, threads;
  linear_load(n, &blocks, &threads);
  DefaultCollider collider(coll_threshold);
  if (!rc) {
    voxellist::kernelCollideWithVoxelMap<<<blocks, threads, sizeof(BitVectorVoxel) * cMAX_THREADS_PER_BLOCK>>>(
        ids, lvox, n, map, dim, collider, off, res);
    rc = check(cudaDeviceSynchronize());
  }
  std::vector<uint16_t> h(cMAX_NR_OF_BLOCKS);
  if (!rc) rc = check(cudaMemcpy(h.data(), res, blocks * sizeof(uint16_t), cudaMemcpyDeviceToHost));
  uint64_t c = 0;
  for (uint32_t i = 0; i < blocks && !rc; ++i) c += h[i];
  *h_count = c;
  if (!rc) rc = check(cudaMemcpy(h_list_vox, lvox, (size_t)n * sizeof(BitVectorVoxel), cudaMemcpyDeviceToHost));
  cudaFree(map);
  cudaFree(lvox);
  cudaFree(ids);
  cudaFree(res);
  return rc;
}

// kernelCollideWithVoxelMap<BitVectorVoxel, BitVectorVoxel, DefaultCollider>
// (GV/voxellist/kernels/VoxelListOperations.hpp:146-197) over many lists
// against one BitVectorVoxelMap, one launch per list with the launch sizing of
// TemplateVoxelList::collisionCheckWithCollider (TemplateVoxelList.hpp:
// 1170-1213): computeLinearLoad(list size), cMAX_THREADS_PER_BLOCK BitVectorVoxels
// of dynamic shared memory, per-block uint16 counts summed on the host.
// Lists are CSR on the host (ids, 32-byte voxels, offsets[n_lists + 1]); the
// list voxels receive the reference's collision marks.  `offset` is the
// relative map offset in voxels (x, y, z).
int ref_lists_collide_map(const uint32_t* h_ids, uint8_t* h_list_vox, const uint64_t* h_offsets, uint32_t n_lists,
                          const uint8_t* h_map, const uint32_t dims[3], const int32_t offset[3], uint64_t* h_counts) {
  const Vector3ui dim(dims[0], dims[1], dims[2]);
  const Vector3i off(offset[0], offset[1], offset[2]);
  const uint64_t nvox = (uint64_t)dims[0] * dims[1] * dims[2];
  const uint64_t n_ids = h_offsets[n_lists];
  BitVectorVoxel *map = nullptr, *lvox = nullptr;
  MapVoxelID* ids = nullptr;
  uint16_t* res = nullptr;
  if (cudaMalloc(&map, nvox * sizeof(BitVectorVoxel)) || cudaMalloc(&lvox, (n_ids + 1) * sizeof(BitVectorVoxel)) ||
      cudaMalloc(&ids, (n_ids + 1) * sizeof(MapVoxelID)) ||
      cudaMalloc(&res, cMAX_NR_OF_BLOCKS * sizeof(uint16_t))) {
    cudaFree(map); cudaFree(lvox); cudaFree(ids); cudaFree(res);
    return -1;
  }
  int rc = check(cudaMemcpy(map, h_map, nvox * sizeof(BitVectorVoxel), cudaMemcpyHostToDevice));
  if (!rc) rc = check(cudaMemcpy(lvox, h_list_vox, n_ids * sizeof(BitVectorVoxel), cudaMemcpyHostToDevice));
  if (!rc) rc = check(cudaMemcpy(ids, h_ids, n_ids * sizeof(MapVoxelID), cudaMemcpyHostToDevice));
  std::vector<uint16_t> h(cMAX_NR_OF_BLOCKS);
  DefaultCollider collider(1.0f);
  const size_t dyn_smem = sizeof(BitVectorVoxel) * cMAX_THREADS_PER_BLOCK;
  for (uint32_t l = 0; l < n_lists && !rc; ++l) {
    const uint32_t n = (uint32_t)(h_offsets[l + 1] - h_offsets[l]);
    uint32_t blocks, threads;
    linear_load(n, &blocks, &threads);
    voxellist::kernelCollideWithVoxelMap<<<blocks, threads, dyn_smem>>>(ids + h_offsets[l], lvox + h_offsets[l], n, map,
                                                                        dim, collider, off, res);
    rc = check(cudaDeviceSynchronize());
    if (!rc) rc = check(cudaMemcpy(h.data(), res, blocks * sizeof(uint16_t), cudaMemcpyDeviceToHost));
    uint64_t c = 0;
    for (uint32_t i = 0; i < blocks; ++i) c += h[i];
    h_counts[l] = c;
  }
  if (!rc) rc = check(cudaMemcpy(h_list_vox, lvox, n_ids * sizeof(BitVectorVoxel), cudaMemcpyDeviceToHost));
  cudaFree(map);
  cudaFree(lvox);
  cudaFree(ids);
  cudaFree(res);
  return rc;
}

}  // extern "C"
