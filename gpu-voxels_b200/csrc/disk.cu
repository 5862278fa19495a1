// The voxel maps' on-disk format, as TemplateVoxelMap::writeToDisk /
// readFromDisk (GV/voxelmap/TemplateVoxelMap.hpp:906-1039) write and read it
// in binary mode: int32 MapType (getTemplateType: BitVectorVoxelMap 0,
// ProbVoxelMap 4, DistanceVoxelMap 9), float voxel side, uint32 x, y, z, then
// the device voxel array byte for byte.  Reading checks the type and the
// dims (a mismatch fails), a different voxel side only warns, as in the
// reference.  Maps of 4 GiB and more are written in full (the reference's
// 32-bit buffer size truncates them).  Host code; the data streams through a
// bounded host buffer.
#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <string>
#include <vector>

#include "gvx_internal.cuh"

namespace gvx {
namespace {

constexpr uint64_t kChunk = 64ull << 20;

gvx_status disk_fail(gvx_status st, const std::string& msg) {
  set_error(msg);
  return st;
}

struct File {
  FILE* f = nullptr;
  File(const char* path, const char* mode) : f(std::fopen(path, mode)) {}
  ~File() {
    if (f) std::fclose(f);
  }
};

gvx_status write_map(const char* path, int32_t type, float side, const gvx_dims& d, const void* d_data, uint64_t bytes) {
  if (path == nullptr) return disk_fail(GVX_ERR_INVALID_ARG, "path is null");
  File out(path, "wb");
  if (!out.f) return disk_fail(GVX_ERR_INVALID_ARG, std::string("cannot open for writing: ") + path);
  const uint32_t dims[3] = {d.x, d.y, d.z};
  bool ok = std::fwrite(&type, 4, 1, out.f) == 1 && std::fwrite(&side, 4, 1, out.f) == 1 &&
            std::fwrite(dims, 4, 3, out.f) == 3;
  std::vector<char> buf((size_t)std::min(bytes, kChunk));
  for (uint64_t off = 0; ok && off < bytes; off += kChunk) {
    const size_t n = (size_t)std::min(kChunk, bytes - off);
    cudaError_t e = cudaMemcpy(buf.data(), static_cast<const char*>(d_data) + off, n, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_status(e, "writeToDisk");
    ok = std::fwrite(buf.data(), 1, n, out.f) == n;
  }
  if (!ok) return disk_fail(GVX_ERR_INVALID_ARG, std::string("write failed: ") + path);
  return GVX_OK;
}

gvx_status read_map(const char* path, int32_t type, float side, const gvx_dims& d, void* d_data, uint64_t bytes) {
  if (path == nullptr) return disk_fail(GVX_ERR_INVALID_ARG, "path is null");
  File in(path, "rb");
  if (!in.f) return disk_fail(GVX_ERR_INVALID_ARG, std::string("cannot open for reading: ") + path);
  int32_t t = -1;
  float s = 0.f;
  uint32_t dims[3] = {0, 0, 0};
  if (std::fread(&t, 4, 1, in.f) != 1 || std::fread(&s, 4, 1, in.f) != 1 || std::fread(dims, 4, 3, in.f) != 3)
    return disk_fail(GVX_ERR_INVALID_ARG, "file too short for the map header");
  if (t != type) return disk_fail(GVX_ERR_INVALID_ARG, "voxel map type does not match");
  if (dims[0] != d.x || dims[1] != d.y || dims[2] != d.z)
    return disk_fail(GVX_ERR_INVALID_ARG, "map dimensions in the file do not match the map");
  if (s != side)
    std::fprintf(stderr, "gvx: readFromDisk: voxel side %g in the file differs from the map's %g; continuing\n", s, side);
  std::vector<char> buf((size_t)std::min(bytes, kChunk));
  for (uint64_t off = 0; off < bytes; off += kChunk) {
    const size_t n = (size_t)std::min(kChunk, bytes - off);
    if (std::fread(buf.data(), 1, n, in.f) != n) return disk_fail(GVX_ERR_INVALID_ARG, "file shorter than the map");
    cudaError_t e = cudaMemcpy(static_cast<char*>(d_data) + off, buf.data(), n, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_status(e, "readFromDisk");
  }
  return GVX_OK;
}

constexpr int32_t kTypeBitVectorVoxelMap = 0, kTypeProbVoxelMap = 4, kTypeDistanceVoxelMap = 9;

}  // namespace
}  // namespace gvx

using namespace gvx;

extern "C" {

gvx_status gvx_dvm_write_to_disk(const gvx_dvm* m, const char* path) {
  if (m == nullptr) return disk_fail(GVX_ERR_INVALID_ARG, "map is null");
  if (cudaDeviceSynchronize() != cudaSuccess) return cuda_status(cudaGetLastError(), "writeToDisk");
  return write_map(path, kTypeDistanceVoxelMap, m->side, m->dims, m->d_vox, num_voxels(m->dims) * 4);
}
gvx_status gvx_dvm_read_from_disk(gvx_dvm* m, const char* path) {
  if (m == nullptr) return disk_fail(GVX_ERR_INVALID_ARG, "map is null");
  if (cudaDeviceSynchronize() != cudaSuccess) return cuda_status(cudaGetLastError(), "readFromDisk");
  return read_map(path, kTypeDistanceVoxelMap, m->side, m->dims, m->d_vox, num_voxels(m->dims) * 4);
}
gvx_status gvx_bvm_write_to_disk(const gvx_bvm* m, const char* path) {
  if (m == nullptr) return disk_fail(GVX_ERR_INVALID_ARG, "map is null");
  if (cudaDeviceSynchronize() != cudaSuccess) return cuda_status(cudaGetLastError(), "writeToDisk");
  return write_map(path, kTypeBitVectorVoxelMap, m->side, m->dims, m->d_vox, num_voxels(m->dims) * kBitVoxelBytes);
}
gvx_status gvx_bvm_read_from_disk(gvx_bvm* m, const char* path) {
  if (m == nullptr) return disk_fail(GVX_ERR_INVALID_ARG, "map is null");
  if (cudaDeviceSynchronize() != cudaSuccess) return cuda_status(cudaGetLastError(), "readFromDisk");
  return read_map(path, kTypeBitVectorVoxelMap, m->side, m->dims, m->d_vox, num_voxels(m->dims) * kBitVoxelBytes);
}
gvx_status gvx_pvm_write_to_disk(const gvx_pvm* m, const char* path) {
  if (m == nullptr) return disk_fail(GVX_ERR_INVALID_ARG, "map is null");
  if (cudaDeviceSynchronize() != cudaSuccess) return cuda_status(cudaGetLastError(), "writeToDisk");
  return write_map(path, kTypeProbVoxelMap, m->side, m->dims, m->d_vox, num_voxels(m->dims));
}
gvx_status gvx_pvm_read_from_disk(gvx_pvm* m, const char* path) {
  if (m == nullptr) return disk_fail(GVX_ERR_INVALID_ARG, "map is null");
  if (cudaDeviceSynchronize() != cudaSuccess) return cuda_status(cudaGetLastError(), "readFromDisk");
  return read_map(path, kTypeProbVoxelMap, m->side, m->dims, m->d_vox, num_voxels(m->dims));
}

}  // extern "C"
