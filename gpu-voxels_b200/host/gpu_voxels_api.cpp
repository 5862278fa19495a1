// Implementation of the gpu_voxels C++ API (include/gpu_voxels/*.h) over the
// gvx C ABI (include/gvx.h).  Every map operation takes the map's recursive
// timed mutex, like the reference (GV/GpuVoxelsMap.h:289); calls the
// reference makes blocking (host-vector queries, collideWith counts) block
// here too, the rest are stream-ordered on the default stream.  Errors are
// reported as the reference does: a message on stderr and a neutral return
// value (SSIZE_MAX for a dimension mismatch in list collisions).
#include <cuda_runtime.h>
#include <stdint.h>

#include <climits>
#include <cstdio>
#include <stdexcept>
#include <string>

#include "../../include/gpu_voxels/GpuVoxels.h"
#include "../../include/gpu_voxels/helpers_highlevel/DistanceMapConverter.h"
#include "../../include/gvx.h"

namespace gpu_voxels {
namespace {

void report(const char* what) { std::fprintf(stderr, "gpu_voxels: %s: %s\n", what, gvx_last_error()); }

bool ok(gvx_status st, const char* what) {
  if (st == GVX_OK) return true;
  report(what);
  return false;
}

void require(gvx_status st, const char* what) {
  if (st != GVX_OK) throw std::runtime_error(std::string("gpu_voxels: ") + what + ": " + gvx_last_error());
}

gvx_dims to_dims(const Vector3ui& d) { return gvx_dims{d.x, d.y, d.z}; }


// TemplateVoxelMap::clone (GV/voxelmap/TemplateVoxelMap.hpp:1101-1120).
void clone_voxels(GpuVoxelsMap& self, const GpuVoxelsMap& other, void* dst, const void* src, size_t bytes) {
  if (self.getVoxelSideLength() != other.getVoxelSideLength() || !(self.getDimensions() == other.getDimensions())) {
    std::fprintf(stderr, "gpu_voxels: clone: map dimensions or voxel side length differ; not cloned\n");
    return;
  }
  if (&self == &other) return;
  std::unique_lock<std::recursive_timed_mutex> a(self.mutexRef(), std::defer_lock);
  std::unique_lock<std::recursive_timed_mutex> b(other.mutexRef(), std::defer_lock);
  std::lock(a, b);
  cudaDeviceSynchronize();
  if (cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToDevice) != cudaSuccess)
    std::fprintf(stderr, "gpu_voxels: clone: device copy failed\n");
  cudaDeviceSynchronize();
}

}  // namespace

// ---------------------------------------------------------------------------
// GpuVoxelsMap: the staging area of the host-vector overloads
// ---------------------------------------------------------------------------
GpuVoxelsMap::~GpuVoxelsMap() {
  if (m_staging) cudaFree(m_staging);
}

void* GpuVoxelsMap::stagingBuffer(size_t bytes) const {
  if (bytes <= m_staging_bytes && m_staging != nullptr) return m_staging;
  if (m_staging) cudaFree(m_staging);  // waits for work still reading it
  m_staging = nullptr;
  m_staging_bytes = 0;
  const size_t cap = std::max<size_t>(bytes + bytes / 4, 1 << 16);
  if (cudaMalloc(&m_staging, cap) != cudaSuccess) {
    m_staging = nullptr;
    throw std::runtime_error("gpu_voxels: cudaMalloc of the staging area failed");
  }
  m_staging_bytes = cap;
  return m_staging;
}

const Vector3f* GpuVoxelsMap::stagePoints(const std::vector<Vector3f>& points) const {
  if (points.empty()) return nullptr;
  void* d = stagingBuffer(points.size() * sizeof(Vector3f));
  // synchronous copy on the legacy default stream: ordered after earlier
  // default-stream work that read the area
  if (cudaMemcpy(d, points.data(), points.size() * sizeof(Vector3f), cudaMemcpyHostToDevice) != cudaSuccess)
    throw std::runtime_error("gpu_voxels: point cloud upload failed");
  return static_cast<const Vector3f*>(d);
}

// ---------------------------------------------------------------------------
// MetaPointCloud and the maps' generic insertMetaPointCloud
// ---------------------------------------------------------------------------
MetaPointCloud::MetaPointCloud(const std::vector<uint32_t>& sizes) {
  for (uint32_t n : sizes) addCloud(n);
}

MetaPointCloud::MetaPointCloud(const std::vector<std::vector<Vector3f> >& clouds) {
  for (const auto& c : clouds) addCloud(c);
}

MetaPointCloud::MetaPointCloud(const MetaPointCloud& other) : m_clouds(other.m_clouds), m_sizes(other.m_sizes) {}

MetaPointCloud& MetaPointCloud::operator=(const MetaPointCloud& other) {
  if (this != &other) {
    m_clouds = other.m_clouds;
    m_sizes = other.m_sizes;
    m_dirty = true;
  }
  return *this;
}

MetaPointCloud::~MetaPointCloud() {
  if (m_dev_xyz) cudaFree(m_dev_xyz);
}

void MetaPointCloud::addCloud(uint32_t cloud_size) {
  m_clouds.emplace_back(cloud_size, Vector3f());
  m_sizes.push_back(cloud_size);
  m_dirty = true;
}

void MetaPointCloud::addCloud(const std::vector<Vector3f>& cloud, bool sync) {
  m_clouds.push_back(cloud);
  m_sizes.push_back((uint32_t)cloud.size());
  m_dirty = true;
  if (sync) syncToDevice();
}

void MetaPointCloud::updatePointCloud(uint16_t cloud, const std::vector<Vector3f>& pointcloud, bool sync) {
  m_clouds.at(cloud) = pointcloud;
  m_sizes.at(cloud) = (uint32_t)pointcloud.size();
  m_dirty = true;
  if (sync) syncToDevice();
}

uint32_t MetaPointCloud::getAccumulatedPointcloudSize() const {
  uint64_t n = 0;
  for (uint32_t s : m_sizes) n += s;
  return (uint32_t)n;
}

std::vector<uint64_t> MetaPointCloud::cloudOffsets() const {
  std::vector<uint64_t> off(m_sizes.size() + 1, 0);
  for (size_t k = 0; k < m_sizes.size(); ++k) off[k + 1] = off[k] + m_sizes[k];
  return off;
}

void MetaPointCloud::syncToDevice() const {
  const uint64_t n = getAccumulatedPointcloudSize();
  if (n > m_dev_capacity) {
    if (m_dev_xyz) cudaFree(m_dev_xyz);
    m_dev_xyz = nullptr;
    m_dev_capacity = 0;
    if (cudaMalloc(&m_dev_xyz, n * sizeof(Vector3f)) != cudaSuccess) throw std::runtime_error("cudaMalloc failed");
    m_dev_capacity = n;
  }
  uint64_t at = 0;
  for (const auto& c : m_clouds) {
    if (!c.empty())
      cudaMemcpy(m_dev_xyz + 3 * at, c.data(), c.size() * sizeof(Vector3f), cudaMemcpyHostToDevice);
    at += c.size();
  }
  m_dirty = false;
}

const float* MetaPointCloud::deviceXYZ() const {
  if (m_dirty) syncToDevice();
  return m_dev_xyz;
}

void GpuVoxelsMap::insertMetaPointCloud(const MetaPointCloud& meta_point_cloud,
                                        const std::vector<BitVoxelMeaning>& voxel_meanings) {
  if (voxel_meanings.size() != meta_point_cloud.getNumberOfPointclouds())
    throw std::invalid_argument("gpu_voxels: insertMetaPointCloud needs one meaning per sub-cloud");
  for (uint16_t k = 0; k < meta_point_cloud.getNumberOfPointclouds(); ++k) {
    const Vector3f* p = meta_point_cloud.getPointCloud(k);
    insertPointCloud(std::vector<Vector3f>(p, p + meta_point_cloud.getPointcloudSize(k)), voxel_meanings[k]);
  }
}

// ---------------------------------------------------------------------------
// DistanceVoxelMap
// ---------------------------------------------------------------------------
namespace voxelmap {

ProbVoxelMap::ProbVoxelMap(const Vector3ui dim, const float voxel_side_length, const MapType map_type)
    : GpuVoxelsMap(map_type, dim, voxel_side_length) {
  gvx_dims d = to_dims(dim);
  require(gvx_pvm_create(&d, voxel_side_length, &m_handle), "ProbVoxelMap");
}

ProbVoxelMap::~ProbVoxelMap() { gvx_pvm_destroy(m_handle); }

void ProbVoxelMap::clearMap() {
  lock_guard g(m_mutex);
  ok(gvx_pvm_clear(m_handle, nullptr), "clearMap");
  cudaDeviceSynchronize();
}

void ProbVoxelMap::insertPointCloud(const std::vector<Vector3f>& points, BitVoxelMeaning voxel_meaning) {
  lock_guard g(m_mutex);
  insertPointCloud(stagePoints(points), (uint32_t)points.size(), voxel_meaning);
  cudaDeviceSynchronize();
}

void ProbVoxelMap::insertPointCloud(const Vector3f* d_points, uint32_t size, BitVoxelMeaning voxel_meaning) {
  lock_guard g(m_mutex);
  ok(gvx_pvm_insert_points(m_handle, reinterpret_cast<const float*>(d_points), size, (uint32_t)voxel_meaning, nullptr,
                           nullptr),
     "insertPointCloud");
}

size_t ProbVoxelMap::getMemoryUsage() const { return getVoxelMapSize(); }

bool ProbVoxelMap::writeToDisk(const std::string path) {
  lock_guard g(m_mutex);
  return ok(gvx_pvm_write_to_disk(m_handle, path.c_str()), "writeToDisk");
}

bool ProbVoxelMap::readFromDisk(const std::string path) {
  lock_guard g(m_mutex);
  return ok(gvx_pvm_read_from_disk(m_handle, path.c_str()), "readFromDisk");
}

void ProbVoxelMap::clone(const ProbVoxelMap& other) {
  int8_t* src = nullptr;
  gvx_pvm_info(other.handle(), nullptr, nullptr, &src);
  clone_voxels(*this, other, getDeviceDataPtr(), src, getVoxelMapSize());
}

Probability* ProbVoxelMap::getDeviceDataPtr() {
  int8_t* p = nullptr;
  gvx_pvm_info(m_handle, nullptr, nullptr, &p);
  return p;
}

DistanceVoxelMap::DistanceVoxelMap(const Vector3ui dim, const float voxel_side_length, const MapType map_type)
    : GpuVoxelsMap(map_type, dim, voxel_side_length) {
  gvx_dims d = to_dims(dim);
  require(gvx_dvm_create(&d, voxel_side_length, &m_handle), "DistanceVoxelMap");
}

DistanceVoxelMap::DistanceVoxelMap(Voxel* dev_data, const Vector3ui dim, const float voxel_side_length,
                                   const MapType map_type)
    : GpuVoxelsMap(map_type, dim, voxel_side_length) {
  gvx_dims d = to_dims(dim);
  require(gvx_dvm_wrap(&d, voxel_side_length, reinterpret_cast<uint32_t*>(dev_data), &m_handle), "DistanceVoxelMap");
}

DistanceVoxelMap::~DistanceVoxelMap() { gvx_dvm_destroy(m_handle); }

void DistanceVoxelMap::clearMap() {
  lock_guard g(m_mutex);
  ok(gvx_dvm_clear(m_handle, nullptr), "clearMap");
}

void DistanceVoxelMap::insertPointCloud(const std::vector<Vector3f>& points, BitVoxelMeaning voxel_meaning) {
  lock_guard g(m_mutex);
  insertPointCloud(stagePoints(points), (uint32_t)points.size(), voxel_meaning);
  cudaDeviceSynchronize();
}

void DistanceVoxelMap::insertPointCloud(const Vector3f* d_points, uint32_t size, BitVoxelMeaning voxel_meaning) {
  lock_guard g(m_mutex);
  if (voxel_meaning != eBVM_OCCUPIED) {
    // DistanceVoxel::insert only knows eBVM_OCCUPIED (GV/voxel/DistanceVoxel.hpp:125-138)
    std::fprintf(stderr, "gpu_voxels: DistanceVoxelMap only supports eBVM_OCCUPIED; use clearMap to free voxels\n");
    return;
  }
  ok(gvx_dvm_insert_points(m_handle, reinterpret_cast<const float*>(d_points), size, nullptr, nullptr), "insertPointCloud");
}

size_t DistanceVoxelMap::getMemoryUsage() const { return getVoxelMapSize() * sizeof(Voxel); }

bool DistanceVoxelMap::writeToDisk(const std::string path) {
  lock_guard g(m_mutex);
  return ok(gvx_dvm_write_to_disk(m_handle, path.c_str()), "writeToDisk");
}

bool DistanceVoxelMap::readFromDisk(const std::string path) {
  lock_guard g(m_mutex);
  return ok(gvx_dvm_read_from_disk(m_handle, path.c_str()), "readFromDisk");
}

void DistanceVoxelMap::parallelBanding3D(uint32_t m1, uint32_t m2, uint32_t m3, uint32_t, uint32_t, uint32_t, bool) {
  lock_guard g(m_mutex);
  ok(gvx_dvm_edt(m_handle, m1, m2, m3, nullptr), "parallelBanding3D");
  cudaDeviceSynchronize();  // the reference returns with the EDT complete
}

void DistanceVoxelMap::voxelizeAndTransform(const std::vector<Vector3f>& points) {
  lock_guard g(m_mutex);
  voxelizeAndTransform(stagePoints(points), (uint32_t)points.size());
}

void DistanceVoxelMap::voxelizeAndTransform(const Vector3f* d_points, uint32_t size) {
  lock_guard g(m_mutex);
  ok(gvx_dvm_voxelize_edt(m_handle, reinterpret_cast<const float*>(d_points), size, nullptr, nullptr),
     "voxelizeAndTransform");
  cudaDeviceSynchronize();
}

void DistanceVoxelMap::jumpFlood3D(int, int, bool) { parallelBanding3D(); }

void DistanceVoxelMap::exactDistances3D(std::vector<Vector3f>& points) { voxelizeAndTransform(points); }

void DistanceVoxelMap::fill_pba_uninit() { fill_pba_uninit(*this); }

void DistanceVoxelMap::fill_pba_uninit(DistanceVoxelMap& other) {
  lock_guard g(other.m_mutex);
  ok(gvx_dvm_clear(other.m_handle, nullptr), "fill_pba_uninit");
  cudaDeviceSynchronize();
}

size_t DistanceVoxelMap::collideWithTypes(const GpuVoxelsMapSharedPtr, BitVectorVoxel&, float, const Vector3ui&) {
  return 0;
}

void DistanceVoxelMap::clearBitVoxelMeaning(BitVoxelMeaning) {}

bool DistanceVoxelMap::insertMetaPointCloudWithSelfCollisionCheck(const MetaPointCloud*,
                                                                  const std::vector<BitVoxelMeaning>&,
                                                                  const std::vector<BitVector<BIT_VECTOR_LENGTH> >&,
                                                                  BitVector<BIT_VECTOR_LENGTH>*) {
  std::fprintf(stderr, "gpu_voxels: insertMetaPointCloudWithSelfCollisionCheck: operation not supported by a DistanceVoxelMap\n");
  return true;
}

void DistanceVoxelMap::extract_distances(free_space_t* dev_distances, int robot_radius) const {
  lock_guard g(m_mutex);
  ok(gvx_dvm_extract_distances(m_handle, dev_distances, robot_radius, nullptr), "extract_distances");
  cudaDeviceSynchronize();
}

void DistanceVoxelMap::init_floodfill(free_space_t* dev_distances, manhattan_dist_t* dev_manhattan_distances,
                                      uint32_t robot_radius) {
  lock_guard g(m_mutex);
  ok(gvx_dvm_init_floodfill(m_handle, dev_distances, dev_manhattan_distances, (int)robot_radius, nullptr),
     "init_floodfill");
  cudaDeviceSynchronize();
}

bool DistanceVoxelMap::mergeOccupied(const std::shared_ptr<ProbVoxelMap> other, const Vector3ui& voxel_offset,
                                     float occupancy_threshold) {
  if (!other) return false;
  std::lock(m_mutex, other->mutexRef());
  lock_guard g1(m_mutex, std::adopt_lock);
  std::lock_guard<std::recursive_timed_mutex> g2(other->mutexRef(), std::adopt_lock);
  const uint32_t off[3] = {voxel_offset.x, voxel_offset.y, voxel_offset.z};
  const bool r = ok(gvx_dvm_merge_occupied(m_handle, other->handle(), off, occupancy_threshold, nullptr), "mergeOccupied");
  cudaDeviceSynchronize();
  return r;
}

void DistanceVoxelMap::getSquaredDistances(const uint32_t* b, const uint32_t* e, int32_t* out) {
  lock_guard g(m_mutex);
  ok(gvx_dvm_sqdist(m_handle, b, (uint64_t)(e - b), out, nullptr), "getSquaredDistances");
}

void DistanceVoxelMap::getDistances(const uint32_t* b, const uint32_t* e, int32_t* out) {
  lock_guard g(m_mutex);
  ok(gvx_dvm_dist(m_handle, b, (uint64_t)(e - b), out, nullptr), "getDistances");
}

void DistanceVoxelMap::gatherVoxelsByIndex(const uint32_t* b, const uint32_t* e, Voxel* out) {
  lock_guard g(m_mutex);
  ok(gvx_dvm_gather(m_handle, b, (uint64_t)(e - b), reinterpret_cast<uint32_t*>(out), nullptr), "gatherVoxelsByIndex");
}

// Host-vector queries: ids and results share the map's staging area.
static void host_query(gvx_dvm* h, void* stage, std::vector<uint32_t>& idx, std::vector<int32_t>& out, bool squared) {
  out.resize(idx.size());
  if (idx.empty()) return;
  uint32_t* di = static_cast<uint32_t*>(stage);
  int32_t* dout = reinterpret_cast<int32_t*>(static_cast<char*>(stage) + ((idx.size() * 4 + 255) & ~(size_t)255));
  cudaMemcpy(di, idx.data(), idx.size() * 4, cudaMemcpyHostToDevice);
  gvx_status st = squared ? gvx_dvm_sqdist(h, di, idx.size(), dout, nullptr) : gvx_dvm_dist(h, di, idx.size(), dout, nullptr);
  if (ok(st, squared ? "getSquaredDistancesToHost" : "getDistancesToHost"))
    cudaMemcpy(out.data(), dout, idx.size() * 4, cudaMemcpyDeviceToHost);
}

void DistanceVoxelMap::getSquaredDistancesToHost(std::vector<uint32_t>& indices, std::vector<int32_t>& output) {
  lock_guard g(m_mutex);
  host_query(m_handle, stagingBuffer(2 * ((indices.size() * 4 + 255) & ~(size_t)255) + 256), indices, output, true);
}

void DistanceVoxelMap::getDistancesToHost(std::vector<uint32_t>& indices, std::vector<int32_t>& output) {
  lock_guard g(m_mutex);
  host_query(m_handle, stagingBuffer(2 * ((indices.size() * 4 + 255) & ~(size_t)255) + 256), indices, output, false);
}

DistanceVoxel::pba_dist_t DistanceVoxelMap::getSquaredObstacleDistance(uint32_t x, uint32_t y, uint32_t z) {
  std::vector<uint32_t> idx(1, (z * m_dim.y + y) * m_dim.x + x);
  std::vector<int32_t> out;
  getSquaredDistancesToHost(idx, out);
  return out.empty() ? MAX_OBSTACLE_DISTANCE : out[0];
}

DistanceVoxel::pba_dist_t DistanceVoxelMap::getSquaredObstacleDistance(const Vector3ui& p) {
  return getSquaredObstacleDistance(p.x, p.y, p.z);
}

DistanceVoxel::pba_dist_t DistanceVoxelMap::getObstacleDistance(uint32_t x, uint32_t y, uint32_t z) {
  std::vector<uint32_t> idx(1, (z * m_dim.y + y) * m_dim.x + x);
  std::vector<int32_t> out;
  getDistancesToHost(idx, out);
  return out.empty() ? MAX_OBSTACLE_DISTANCE : out[0];
}

DistanceVoxel::pba_dist_t DistanceVoxelMap::getObstacleDistance(const Vector3ui& p) { return getObstacleDistance(p.x, p.y, p.z); }

void DistanceVoxelMap::clone(const DistanceVoxelMap& other) {
  uint32_t* src = nullptr;
  gvx_dvm_info(other.handle(), nullptr, nullptr, &src);
  clone_voxels(*this, other, getDeviceDataPtr(), src, getVoxelMapSize() * sizeof(DistanceVoxel));
}

DistanceVoxel* DistanceVoxelMap::getDeviceDataPtr() {
  uint32_t* p = nullptr;
  gvx_dvm_info(m_handle, nullptr, nullptr, &p);
  return reinterpret_cast<DistanceVoxel*>(p);
}

const DistanceVoxel* DistanceVoxelMap::getConstDeviceDataPtr() const {
  uint32_t* p = nullptr;
  gvx_dvm_info(m_handle, nullptr, nullptr, &p);
  return reinterpret_cast<const DistanceVoxel*>(p);
}

// ---------------------------------------------------------------------------
// BitVoxelMap<256>
// ---------------------------------------------------------------------------

template <size_t length>
BitVoxelMap<length>::BitVoxelMap(const Vector3ui dim, const float voxel_side_length, const MapType map_type)
    : GpuVoxelsMap(map_type, dim, voxel_side_length) {
  gvx_dims d = to_dims(dim);
  require(gvx_bvm_create(&d, voxel_side_length, &m_handle), "BitVoxelMap");
  if (cudaMalloc(&m_dev_count, sizeof(uint64_t)) != cudaSuccess || cudaMalloc(&m_dev_types, 32) != cudaSuccess)
    throw std::runtime_error("cudaMalloc failed");
}

template <size_t length>
BitVoxelMap<length>::~BitVoxelMap() {
  gvx_bvm_destroy(m_handle);
  if (m_dev_count) cudaFree(m_dev_count);
  if (m_dev_types) cudaFree(m_dev_types);
}

template <size_t length>
void BitVoxelMap<length>::clearMap() {
  lock_guard g(m_mutex);
  ok(gvx_bvm_clear(m_handle, nullptr), "clearMap");
}

template <size_t length>
void BitVoxelMap<length>::insertPointCloud(const std::vector<Vector3f>& points, BitVoxelMeaning voxel_meaning) {
  lock_guard g(m_mutex);
  insertPointCloud(stagePoints(points), (uint32_t)points.size(), voxel_meaning);
  cudaDeviceSynchronize();
}

template <size_t length>
void BitVoxelMap<length>::insertPointCloud(const Vector3f* d_points, uint32_t size, BitVoxelMeaning voxel_meaning) {
  lock_guard g(m_mutex);
  ok(gvx_bvm_insert_points(m_handle, reinterpret_cast<const float*>(d_points), size, (uint32_t)voxel_meaning, nullptr,
                           nullptr),
     "insertPointCloud");
}

template <size_t length>
size_t BitVoxelMap<length>::getMemoryUsage() const {
  return getVoxelMapSize() * (length / 8);
}

template <size_t length>
size_t BitVoxelMap<length>::collideWith(const BitVoxelMap<length>* map, float, const Vector3i& offset) {
  std::lock(m_mutex, map->m_mutex);
  std::lock_guard<std::recursive_timed_mutex> g1(m_mutex, std::adopt_lock);
  std::lock_guard<std::recursive_timed_mutex> g2(map->m_mutex, std::adopt_lock);
  const int32_t off[3] = {offset.x, offset.y, offset.z};
  if (!ok(gvx_bvm_collide(m_handle, map->m_handle, off, 1, m_dev_count, nullptr), "collideWith")) return 0;
  uint64_t count = 0;
  cudaMemcpy(&count, m_dev_count, sizeof(count), cudaMemcpyDeviceToHost);
  return (size_t)count;
}

template <size_t length>
size_t BitVoxelMap<length>::collideWith(const ProbVoxelMap* map, float coll_threshold, const Vector3i& offset) {
  std::lock(m_mutex, map->mutexRef());
  std::lock_guard<std::recursive_timed_mutex> g1(m_mutex, std::adopt_lock);
  std::lock_guard<std::recursive_timed_mutex> g2(map->mutexRef(), std::adopt_lock);
  const int32_t off[3] = {offset.x, offset.y, offset.z};
  if (!ok(gvx_bvm_collide_pvm(m_handle, map->handle(), coll_threshold, off, 1, m_dev_count, nullptr), "collideWith"))
    return 0;
  uint64_t count = 0;
  cudaMemcpy(&count, m_dev_count, sizeof(count), cudaMemcpyDeviceToHost);
  return (size_t)count;
}

// The count and types a typed-collision call left on the device.
static size_t read_types(const uint64_t* d_count, const uint8_t* d_types, BitVectorVoxel* types, bool accumulate) {
  uint64_t count = 0;
  BitVectorVoxel t;
  cudaMemcpy(&count, d_count, sizeof(count), cudaMemcpyDeviceToHost);
  cudaMemcpy(t.bitVector().data(), d_types, 32, cudaMemcpyDeviceToHost);
  if (accumulate) types->bitVector() |= t.bitVector();
  else *types = t;
  return (size_t)count;
}

template <size_t length>
size_t BitVoxelMap<length>::collideWithTypes(const BitVoxelMap<length>* map, BitVectorVoxel& types, float,
                                             const Vector3i&) {
  std::lock(m_mutex, map->m_mutex);
  std::lock_guard<std::recursive_timed_mutex> g1(m_mutex, std::adopt_lock);
  std::lock_guard<std::recursive_timed_mutex> g2(map->m_mutex, std::adopt_lock);
  if (!ok(gvx_bvm_collide_types(m_handle, map->m_handle, m_dev_count, m_dev_types, nullptr), "collideWithTypes")) return 0;
  return read_types(m_dev_count, m_dev_types, &types, true);  // the reference ORs into the caller's set
}

template <size_t length>
size_t BitVoxelMap<length>::collideWithTypes(const ProbVoxelMap* map, BitVectorVoxel& types, float coll_threshold,
                                             const Vector3i&) {
  std::lock(m_mutex, map->mutexRef());
  std::lock_guard<std::recursive_timed_mutex> g1(m_mutex, std::adopt_lock);
  std::lock_guard<std::recursive_timed_mutex> g2(map->mutexRef(), std::adopt_lock);
  if (!ok(gvx_bvm_collide_types_pvm(m_handle, map->handle(), coll_threshold, m_dev_count, m_dev_types, nullptr),
          "collideWithTypes"))
    return 0;
  return read_types(m_dev_count, m_dev_types, &types, true);
}

template <size_t length>
void BitVoxelMap<length>::clearBits(BitVector<length> bits) {
  std::lock_guard<std::recursive_timed_mutex> guard(m_mutex);
  ok(gvx_bvm_clear_bits(m_handle, bits.data(), nullptr), "clearBits");
  cudaDeviceSynchronize();
}

template <size_t length>
void BitVoxelMap<length>::clearBit(const uint32_t bit_index) {
  BitVector<length> b;
  b.setBit(bit_index);
  clearBits(b);
}

template <size_t length>
void BitVoxelMap<length>::clearBitVoxelMeaning(BitVoxelMeaning voxel_meaning) {
  clearBit(uint32_t(voxel_meaning));
}

template <size_t length>
void BitVoxelMap<length>::shiftLeftSweptVolumeIDs(uint8_t shift_size) {
  std::lock_guard<std::recursive_timed_mutex> guard(m_mutex);
  ok(gvx_bvm_shift_swept_volume_ids(m_handle, shift_size, nullptr), "shiftLeftSweptVolumeIDs");
  cudaDeviceSynchronize();
}

template <size_t length>
bool BitVoxelMap<length>::insertMetaPointCloudWithSelfCollisionCheck(const MetaPointCloud* robot_links,
                                                                     const std::vector<BitVoxelMeaning>& voxel_meanings,
                                                                     const std::vector<BitVector<length> >& collision_masks,
                                                                     BitVector<length>* colliding_meanings) {
  std::lock_guard<std::recursive_timed_mutex> guard(m_mutex);
  if (robot_links == nullptr || robot_links->getNumberOfPointclouds() == 0) return false;
  const uint32_t n = robot_links->getNumberOfPointclouds();
  if ((!voxel_meanings.empty() && voxel_meanings.size() != n) || (!collision_masks.empty() && collision_masks.size() != n))
    throw std::invalid_argument("gpu_voxels: one meaning and one collision mask per sub-cloud (or none)");
  std::vector<uint8_t> meanings(voxel_meanings.begin(), voxel_meanings.end());
  std::vector<uint8_t> masks;
  for (const auto& m : collision_masks) masks.insert(masks.end(), m.data(), m.data() + BitVector<length>::m_size);
  const std::vector<uint64_t> offsets = robot_links->cloudOffsets();
  BitVector<length> colliding;
  int any = 0;
  if (!ok(gvx_bvm_insert_meta_points_self_coll(m_handle, robot_links->deviceXYZ(), offsets.data(), n,
                                               meanings.empty() ? nullptr : meanings.data(),
                                               masks.empty() ? nullptr : masks.data(), colliding.data(), &any, nullptr,
                                               nullptr),
          "insertMetaPointCloudWithSelfCollisionCheck"))
    return false;
  if (colliding_meanings) *colliding_meanings = colliding;
  return any != 0;
}

template <size_t length>
bool BitVoxelMap<length>::writeToDisk(const std::string path) {
  lock_guard g(m_mutex);
  return ok(gvx_bvm_write_to_disk(m_handle, path.c_str()), "writeToDisk");
}

template <size_t length>
bool BitVoxelMap<length>::readFromDisk(const std::string path) {
  lock_guard g(m_mutex);
  return ok(gvx_bvm_read_from_disk(m_handle, path.c_str()), "readFromDisk");
}

template <size_t length>
uint8_t* BitVoxelMap<length>::getDeviceDataPtr() {
  uint8_t* p = nullptr;
  gvx_bvm_info(m_handle, nullptr, nullptr, &p);
  return p;
}

template <size_t length>
void BitVoxelMap<length>::clone(const BitVoxelMap& other) {
  uint8_t* src = nullptr;
  gvx_bvm_info(other.handle(), nullptr, nullptr, &src);
  clone_voxels(*this, other, getDeviceDataPtr(), src, getVoxelMapSize() * 32);
}

template class BitVoxelMap<BIT_VECTOR_LENGTH>;

}  // namespace voxelmap

// ---------------------------------------------------------------------------
// BitVoxelList<256, uint32>
// ---------------------------------------------------------------------------
namespace voxellist {

template <size_t length, class ID>
BitVoxelList<length, ID>::BitVoxelList(const Vector3ui ref_map_dim, const float voxel_side_length, const MapType map_type)
    : GpuVoxelsMap(map_type, ref_map_dim, voxel_side_length) {
  gvx_dims d = to_dims(ref_map_dim);
  require(gvx_blist_create(&d, voxel_side_length, &m_handle), "BitVoxelList");
  if (cudaMalloc(&m_dev_count, sizeof(uint64_t)) != cudaSuccess || cudaMalloc(&m_dev_types, 64) != cudaSuccess)
    throw std::runtime_error("cudaMalloc failed");
}

template <size_t length, class ID>
BitVoxelList<length, ID>::~BitVoxelList() {
  gvx_blist_destroy(m_handle);
  if (m_dev_count) cudaFree(m_dev_count);
  if (m_dev_types) cudaFree(m_dev_types);
}

template <size_t length, class ID>
void BitVoxelList<length, ID>::clearMap() {
  lock_guard g(m_mutex);
  ok(gvx_blist_clear(m_handle), "clearMap");
}

template <size_t length, class ID>
void BitVoxelList<length, ID>::insertPointCloud(const std::vector<Vector3f>& points, BitVoxelMeaning voxel_meaning) {
  lock_guard g(m_mutex);
  insertPointCloud(stagePoints(points), (uint32_t)points.size(), voxel_meaning);
}

template <size_t length, class ID>
void BitVoxelList<length, ID>::insertPointCloud(const Vector3f* d_points, uint32_t size, BitVoxelMeaning voxel_meaning) {
  lock_guard g(m_mutex);
  ok(gvx_blist_insert_points(m_handle, reinterpret_cast<const float*>(d_points), size, (uint32_t)voxel_meaning, nullptr),
     "insertPointCloud");
}

template <size_t length, class ID>
size_t BitVoxelList<length, ID>::getMemoryUsage() const {
  uint64_t n = 0;
  gvx_blist_size(m_handle, &n);
  return (size_t)n * (sizeof(ID) + length / 8);
}

template <size_t length, class ID>
Vector3ui BitVoxelList<length, ID>::getDimensions() const {
  uint64_t n = 0;
  gvx_blist_size(m_handle, &n);
  return Vector3ui((uint32_t)n, 1, 1);
}

template <size_t length, class ID>
size_t BitVoxelList<length, ID>::collideWith(const voxelmap::BitVoxelMap<length>* map, float, const Vector3i& offset) {
  if (map->getDimensions() != m_dim) {
    std::fprintf(stderr, "gpu_voxels: list reference dims differ from the map's; not checking collisions\n");
    return SSIZE_MAX;
  }
  lock_guard g(m_mutex);
  const int32_t off[3] = {offset.x, offset.y, offset.z};
  if (!ok(gvx_blist_collide_bvm(m_handle, map->handle(), off, 1, m_dev_count, nullptr), "collideWith")) return 0;
  uint64_t count = 0;
  cudaMemcpy(&count, m_dev_count, sizeof(count), cudaMemcpyDeviceToHost);
  return (size_t)count;
}

template <size_t length, class ID>
size_t BitVoxelList<length, ID>::collideWith(const voxelmap::ProbVoxelMap* map, float coll_threshold,
                                             const Vector3i& offset) {
  if (map->getDimensions() != m_dim) {
    std::fprintf(stderr, "gpu_voxels: list reference dims differ from the map's; not checking collisions\n");
    return SSIZE_MAX;
  }
  lock_guard g(m_mutex);
  const int32_t off[3] = {offset.x, offset.y, offset.z};
  if (!ok(gvx_blist_collide_pvm(m_handle, map->handle(), coll_threshold, off, 1, m_dev_count, nullptr), "collideWith"))
    return 0;
  uint64_t count = 0;
  cudaMemcpy(&count, m_dev_count, sizeof(count), cudaMemcpyDeviceToHost);
  return (size_t)count;
}

template <size_t length, class ID>
size_t BitVoxelList<length, ID>::collideWith(const BitVoxelList<length, ID>* other, float, const Vector3i& offset) {
  if (offset != Vector3i()) {
    std::fprintf(stderr, "gpu_voxels: offset for voxel-list collision not supported\n");
    return 0;
  }
  lock_guard g(m_mutex);
  const int32_t off[3] = {0, 0, 0};
  if (!ok(gvx_blist_collide_blist(m_handle, other->m_handle, off, m_dev_count, nullptr), "collideWith")) return 0;
  uint64_t count = 0;
  cudaMemcpy(&count, m_dev_count, sizeof(count), cudaMemcpyDeviceToHost);
  return (size_t)count;
}

template <size_t length, class ID>
size_t BitVoxelList<length, ID>::collideWithTypes(const voxelmap::BitVoxelMap<length>* map, BitVectorVoxel& types, float,
                                                  const Vector3i& offset) {
  if (map->getDimensions() != m_dim) {
    std::fprintf(stderr, "gpu_voxels: list reference dims differ from the map's; not checking collisions\n");
    return SSIZE_MAX;
  }
  lock_guard g(m_mutex);
  const int32_t off[3] = {offset.x, offset.y, offset.z};
  if (!ok(gvx_blist_collide_types_bvm(m_handle, map->handle(), off, m_dev_count, m_dev_types, nullptr), "collideWithTypes"))
    return 0;
  return voxelmap::read_types(m_dev_count, m_dev_types, &types, false);  // the reference clears the set first
}

template <size_t length, class ID>
size_t BitVoxelList<length, ID>::collideWithTypes(const voxelmap::ProbVoxelMap* map, BitVectorVoxel& types,
                                                  float coll_threshold, const Vector3i& offset) {
  if (map->getDimensions() != m_dim) {
    std::fprintf(stderr, "gpu_voxels: list reference dims differ from the map's; not checking collisions\n");
    return SSIZE_MAX;
  }
  lock_guard g(m_mutex);
  const int32_t off[3] = {offset.x, offset.y, offset.z};
  if (!ok(gvx_blist_collide_types_pvm(m_handle, map->handle(), coll_threshold, off, m_dev_count, m_dev_types, nullptr),
          "collideWithTypes"))
    return 0;
  return voxelmap::read_types(m_dev_count, m_dev_types, &types, false);
}

template <size_t length, class ID>
size_t BitVoxelList<length, ID>::collideWithTypes(const BitVoxelList<length, ID>* other, BitVectorVoxel& types, float,
                                                  const Vector3i& offset) {
  if (offset != Vector3i()) {
    std::fprintf(stderr, "gpu_voxels: offset for voxel-list collision not supported\n");
    types = BitVectorVoxel();
    return 0;
  }
  lock_guard g(m_mutex);
  if (!ok(gvx_blist_collide_types_blist(m_handle, other->m_handle, m_dev_count, m_dev_types, nullptr), "collideWithTypes"))
    return 0;
  return voxelmap::read_types(m_dev_count, m_dev_types, &types, false);
}

template <size_t length, class ID>
size_t BitVoxelList<length, ID>::collideWithTypeMask(const voxelmap::BitVoxelMap<length>* map,
                                                     const BitVectorVoxel& types_to_check, float, const Vector3i& offset) {
  if (map->getDimensions() != m_dim) {
    std::fprintf(stderr, "gpu_voxels: list reference dims differ from the map's; not checking collisions\n");
    return SSIZE_MAX;
  }
  lock_guard g(m_mutex);
  cudaMemcpy(m_dev_types + 32, types_to_check.bitVector().data(), 32, cudaMemcpyHostToDevice);
  const int32_t off[3] = {offset.x, offset.y, offset.z};
  if (!ok(gvx_blist_collide_type_mask_bvm(m_handle, map->handle(), m_dev_types + 32, off, m_dev_count, nullptr),
          "collideWithTypeMask"))
    return 0;
  uint64_t count = 0;
  cudaMemcpy(&count, m_dev_count, sizeof(count), cudaMemcpyDeviceToHost);
  return (size_t)count;
}

template <size_t length, class ID>
void BitVoxelList<length, ID>::insertCoordinateList(const std::vector<Vector3ui>& coordinates,
                                                    const BitVoxelMeaning voxel_meaning) {
  std::vector<Vector3f> pts;
  pts.reserve(coordinates.size());
  const float s = m_voxel_side_length;
  for (const Vector3ui& c : coordinates)  // voxel centres land in their own voxel
    if (c.x < m_dim.x && c.y < m_dim.y && c.z < m_dim.z)
      pts.push_back(Vector3f((c.x + 0.5f) * s, (c.y + 0.5f) * s, (c.z + 0.5f) * s));
  insertPointCloud(pts, voxel_meaning);
}

template <size_t length, class ID>
void BitVoxelList<length, ID>::insertCoordinateList(const Vector3ui* d_coordinates, uint32_t size,
                                                    const BitVoxelMeaning voxel_meaning) {
  std::vector<Vector3ui> host(size);
  if (size) cudaMemcpy(host.data(), d_coordinates, size * sizeof(Vector3ui), cudaMemcpyDeviceToHost);
  insertCoordinateList(host, voxel_meaning);
}

template <size_t length, class ID>
void BitVoxelList<length, ID>::copyCoordsToHost(std::vector<Vector3ui>& host_vec) const {
  std::vector<ID> ids;
  copyIdsToHost(ids);
  host_vec.resize(ids.size());
  const uint64_t layer = (uint64_t)m_dim.x * m_dim.y;
  for (size_t i = 0; i < ids.size(); ++i)
    host_vec[i] = Vector3ui((uint32_t)(ids[i] % m_dim.x), (uint32_t)((ids[i] / m_dim.x) % m_dim.y),
                            (uint32_t)(ids[i] / layer));
}

template <size_t length, class ID>
void BitVoxelList<length, ID>::shiftLeftSweptVolumeIDs(uint8_t shift_size) {
  lock_guard g(m_mutex);
  ok(gvx_blist_shift_swept_volume_ids(m_handle, shift_size, nullptr), "shiftLeftSweptVolumeIDs");
  cudaDeviceSynchronize();
}

template <size_t length, class ID>
void BitVoxelList<length, ID>::clearBitVoxelMeaning(BitVoxelMeaning voxel_meaning) {
  lock_guard g(m_mutex);
  BitVector<length> b;
  b.setBit(uint32_t(voxel_meaning));
  ok(gvx_blist_clear_bits(m_handle, b.data(), nullptr), "clearBitVoxelMeaning");
  cudaDeviceSynchronize();
}

template <size_t length, class ID>
void BitVoxelList<length, ID>::copyIdsToHost(std::vector<ID>& ids) const {
  uint64_t n = 0;
  uint32_t* d = nullptr;
  gvx_blist_size(m_handle, &n);
  gvx_blist_data(m_handle, &d, nullptr);
  ids.resize(n);
  if (n) cudaMemcpy(ids.data(), d, n * sizeof(ID), cudaMemcpyDeviceToHost);
}

template <size_t length, class ID>
void BitVoxelList<length, ID>::copyVoxelsToHost(std::vector<uint8_t>& voxels) const {
  uint64_t n = 0;
  uint8_t* d = nullptr;
  gvx_blist_size(m_handle, &n);
  gvx_blist_data(m_handle, nullptr, &d);
  voxels.resize(n * (length / 8));
  if (n) cudaMemcpy(voxels.data(), d, voxels.size(), cudaMemcpyDeviceToHost);
}

template class BitVoxelList<BIT_VECTOR_LENGTH, MapVoxelID>;

}  // namespace voxellist

// ---------------------------------------------------------------------------
// GpuVoxels facade
// ---------------------------------------------------------------------------

std::mutex GpuVoxels::s_instance_mutex;
GpuVoxelsSharedPtr GpuVoxels::s_instance;

GpuVoxels::GpuVoxels() {
  int dev = 0;
  cudaGetDevice(&dev);
  if (gvx_init_device(dev) != GVX_OK) {
    // the reference exits with code 123 when no suitable GPU is found (GV/GpuVoxels.cpp:33-42)
    std::fprintf(stderr, "gpu_voxels: %s\n", gvx_last_error());
  }
}

GpuVoxels::~GpuVoxels() { m_managed_maps.clear(); }

GpuVoxelsSharedPtr GpuVoxels::getInstance() {
  std::lock_guard<std::mutex> g(s_instance_mutex);
  if (!s_instance) s_instance.reset(new GpuVoxels());
  return s_instance;
}

void GpuVoxels::initialize(uint32_t dim_x, uint32_t dim_y, uint32_t dim_z, float voxel_side_length) {
  std::lock_guard<std::recursive_mutex> g(m_mutex);
  m_dim = Vector3ui(dim_x, dim_y, dim_z);
  m_voxel_side_length = voxel_side_length;
}

GpuVoxelsMapSharedPtr GpuVoxels::addMap(const MapType map_type, const std::string& map_name) {
  std::lock_guard<std::recursive_mutex> g(m_mutex);
  if (m_managed_maps.count(map_name)) {
    std::fprintf(stderr, "gpu_voxels: a map named '%s' exists already\n", map_name.c_str());
    return GpuVoxelsMapSharedPtr();
  }
  GpuVoxelsMapSharedPtr map;
  try {
    switch (map_type) {
      case MT_DISTANCE_VOXELMAP: map.reset(new voxelmap::DistanceVoxelMap(m_dim, m_voxel_side_length, map_type)); break;
      case MT_BITVECTOR_VOXELMAP: map.reset(new BitVectorVoxelMap(m_dim, m_voxel_side_length, map_type)); break;
      case MT_BITVECTOR_VOXELLIST: map.reset(new BitVectorVoxelList(m_dim, m_voxel_side_length, map_type)); break;
      case MT_PROBAB_VOXELMAP: map.reset(new voxelmap::ProbVoxelMap(m_dim, m_voxel_side_length, map_type)); break;
      default:
        std::fprintf(stderr, "gpu_voxels: map type %d is outside the distance-field collision path\n", (int)map_type);
        return GpuVoxelsMapSharedPtr();
    }
  } catch (const std::exception& e) {
    std::fprintf(stderr, "%s\n", e.what());
    return GpuVoxelsMapSharedPtr();
  }
  m_managed_maps[map_name] = map;
  return map;
}

bool GpuVoxels::visualizeMap(const std::string& map_name, const bool /*force_repaint*/) {
  if (!getMap(map_name)) {
    std::fprintf(stderr, "gpu_voxels: Map with name '%s' not found.\n", map_name.c_str());
    return false;
  }
  return false;  // no viewer
}

bool GpuVoxels::delMap(const std::string& map_name) {
  std::lock_guard<std::recursive_mutex> g(m_mutex);
  return m_managed_maps.erase(map_name) > 0;
}

GpuVoxelsMapSharedPtr GpuVoxels::getMap(const std::string& map_name) {
  std::lock_guard<std::recursive_mutex> g(m_mutex);
  auto it = m_managed_maps.find(map_name);
  return it == m_managed_maps.end() ? GpuVoxelsMapSharedPtr() : it->second;
}

bool GpuVoxels::clearMap(const std::string& map_name) {
  GpuVoxelsMapSharedPtr m = getMap(map_name);
  if (!m) return false;
  m->clearMap();
  return true;
}

bool GpuVoxels::insertPointCloudIntoMap(const std::vector<Vector3f>& point_cloud, std::string map_name,
                                        const BitVoxelMeaning voxel_meaning) {
  GpuVoxelsMapSharedPtr m = getMap(map_name);
  if (!m) return false;
  m->insertPointCloud(point_cloud, voxel_meaning);
  return true;
}

void GpuVoxels::getDimensions(uint32_t& dim_x, uint32_t& dim_y, uint32_t& dim_z) const {
  dim_x = m_dim.x;
  dim_y = m_dim.y;
  dim_z = m_dim.z;
}

void GpuVoxels::getDimensions(Vector3ui& dim) const { dim = m_dim; }

void GpuVoxels::getVoxelSideLength(float& voxel_side_length) const { voxel_side_length = m_voxel_side_length; }

}  // namespace gpu_voxels

// ---------------------------------------------------------------------------
// distance_map_converter
// ---------------------------------------------------------------------------
namespace gpu_voxels {
namespace distance_map_converter {

size_t extract_given_distances(const voxelmap::DistanceVoxelMap& dist_map, free_space_t min_dist, free_space_t max_dist,
                               BitVectorVoxelList& result) {
  uint64_t n = 0;
  ok(gvx_extract_given_distances(dist_map.handle(), min_dist, max_dist, result.handle(), &n, nullptr),
     "extract_given_distances");
  return (size_t)n;
}

}  // namespace distance_map_converter
}  // namespace gpu_voxels
