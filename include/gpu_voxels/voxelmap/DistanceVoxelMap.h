// DistanceVoxelMap of the gpu_voxels C++ API (gpu-voxels
// GV/voxelmap/DistanceVoxelMap.h:55-140) over the gvx C ABI.  Voxels are
// uint32 DistanceVoxels (x | y<<10 | z<<20); parallelBanding3D computes the
// exact EDT in place with the results of the reference's (1,1,1) banding.
#pragma once

#include <stdint.h>

#include <vector>

#if __has_include(<thrust/device_ptr.h>)
#include <thrust/device_ptr.h>
#define GVX_HAVE_THRUST_DEVICE_PTR 1
#endif

#include "../GpuVoxelsMap.h"
#include "ProbVoxelMap.h"

struct gvx_dvm;

namespace gpu_voxels {

// Host-side view of one DistanceVoxel (GV/voxel/DistanceVoxel.h:51-120).
class DistanceVoxel {
 public:
  typedef int32_t pba_dist_t;
  typedef uint32_t pba_voxel_t;
  DistanceVoxel() : m_obstacle(0x3FFFFFFFu) {}
  explicit DistanceVoxel(pba_voxel_t v) : m_obstacle(v) {}
  DistanceVoxel(uint32_t x, uint32_t y, uint32_t z) : m_obstacle(x | (y << 10) | (z << 20)) {}
  Vector3ui getObstacle() const { return Vector3ui(m_obstacle & 0x3ffu, (m_obstacle >> 10) & 0x3ffu, m_obstacle >> 20); }
  // squaredObstacleDistance (GV/voxel/DistanceVoxel.hpp:40-55)
  pba_dist_t squaredObstacleDistance(const Vector3i& p) const {
    const Vector3ui o = getObstacle();
    if (p.x == PBA_UNINITIALISED_COORD || p.y == PBA_UNINITIALISED_COORD || p.z == PBA_UNINITIALISED_COORD ||
        (int32_t)o.x == PBA_UNINITIALISED_COORD || (int32_t)o.y == PBA_UNINITIALISED_COORD ||
        (int32_t)o.z == PBA_UNINITIALISED_COORD)
      return MAX_OBSTACLE_DISTANCE;
    const int32_t dx = p.x - (int32_t)o.x, dy = p.y - (int32_t)o.y, dz = p.z - (int32_t)o.z;
    return dx * dx + dy * dy + dz * dz;
  }
  pba_voxel_t raw() const { return m_obstacle; }

 private:
  pba_voxel_t m_obstacle;
};
static_assert(sizeof(DistanceVoxel) == 4, "DistanceVoxel is 4 bytes");

namespace voxelmap {

class DistanceVoxelMap : public GpuVoxelsMap {
 public:
  typedef DistanceVoxel Voxel;

  DistanceVoxelMap(const Vector3ui dim, const float voxel_side_length, const MapType map_type = MT_DISTANCE_VOXELMAP);
  // Non-owning: wraps caller-owned device memory of dim.x*dim.y*dim.z voxels.
  DistanceVoxelMap(Voxel* dev_data, const Vector3ui dim, const float voxel_side_length,
                   const MapType map_type = MT_DISTANCE_VOXELMAP);
  ~DistanceVoxelMap() override;

  void clearMap() override;
  void insertPointCloud(const std::vector<Vector3f>& points, BitVoxelMeaning voxel_meaning) override;
  void insertPointCloud(const Vector3f* d_points, uint32_t size, BitVoxelMeaning voxel_meaning) override;
  size_t getMemoryUsage() const override;
  bool writeToDisk(const std::string path) override;
  bool readFromDisk(const std::string path) override;

  // Exact EDT (GV/voxelmap/DistanceVoxelMap.hpp:284-645).  Band counts and
  // block sizes are accepted for source compatibility; the result is always
  // the reference's (1,1,1) result.
  void parallelBanding3D(uint32_t m1 = 1, uint32_t m2 = 1, uint32_t m3 = 1,
                         uint32_t m1_blocksize = PBA_DEFAULT_M1_BLOCK_SIZE,
                         uint32_t m2_blocksize = PBA_DEFAULT_M2_BLOCK_SIZE,
                         uint32_t m3_blocksize = PBA_DEFAULT_M3_BLOCK_SIZE, bool detailtimer = false);

  // gvx extension (no reference counterpart): clearMap + insertPointCloud +
  // parallelBanding3D in one call, the same result, without writing the
  // inserted map first (the fastest form for a per-frame sensor loop).
  void voxelizeAndTransform(const std::vector<Vector3f>& points);
  void voxelizeAndTransform(const Vector3f* d_points, uint32_t size);

  // The reference's other two EDTs, kept for source compatibility.  Both
  // compute the exact transform of parallelBanding3D: jumpFlood3D
  // (DistanceVoxelMap.hpp:141-206) is an approximation in the reference, and
  // exactDistances3D (DistanceVoxelMap.hpp:208-251: brute force over `points`,
  // every voxel written) gives the same squared distances; a voxel equally
  // near two obstacles may name the other one as its site.
  void jumpFlood3D(int block_size = 1024, int debug = 0, bool logging_reinit = false);
  void exactDistances3D(std::vector<Vector3f>& points);
  // fill_pba_uninit (DistanceVoxelMap.hpp:647-657): every voxel of `other`
  // (of this map) set to the uninitialised DistanceVoxel.
  void fill_pba_uninit();
  void fill_pba_uninit(DistanceVoxelMap& other);
  // No-ops in the reference for a DistanceVoxelMap (DistanceVoxelMap.hpp:85-107):
  // collideWithTypes returns 0, clearBitVoxelMeaning does nothing, and the
  // self-collision insert reports the operation as unsupported and returns true.
  size_t collideWithTypes(const GpuVoxelsMapSharedPtr other, BitVectorVoxel& meanings_in_collision,
                          float coll_threshold = 1.0, const Vector3ui& offset = Vector3ui());
  void clearBitVoxelMeaning(BitVoxelMeaning voxel_meaning);
  bool insertMetaPointCloudWithSelfCollisionCheck(
      const MetaPointCloud* robot_links,
      const std::vector<BitVoxelMeaning>& voxel_meanings = std::vector<BitVoxelMeaning>(),
      const std::vector<BitVector<BIT_VECTOR_LENGTH> >& collision_masks = std::vector<BitVector<BIT_VECTOR_LENGTH> >(),
      BitVector<BIT_VECTOR_LENGTH>* colliding_meanings = NULL) override;

  // mergeOccupied (GV/voxelmap/DistanceVoxelMap.hpp:109-136): voxels of `other`
  // whose occupancy exceeds the threshold become sites (own coordinates +
  // voxel_offset).  Returns false when the maps' dims differ.
  bool mergeOccupied(const std::shared_ptr<ProbVoxelMap> other, const Vector3ui& voxel_offset = Vector3ui(),
                     float occupancy_threshold = 0.5f);

  // extract_distances (GV/voxelmap/DistanceVoxelMap.hpp:676-688): one
  // free-space byte per voxel into dev_distances (device, getVoxelMapSize()).
  void extract_distances(free_space_t* dev_distances, int robot_radius) const;
  // init_floodfill (DistanceVoxelMap.hpp:658-674): dev_manhattan_distances[i] =
  // MANHATTAN_DISTANCE_TOO_CLOSE where dev_distances[i] <= robot_radius, else
  // MANHATTAN_DISTANCE_UNINITIALIZED.
  void init_floodfill(free_space_t* dev_distances, manhattan_dist_t* dev_manhattan_distances, uint32_t robot_radius);

  // Queries at linear voxel ids (device pointers; [begin, end) ids -> out).
  void getSquaredDistances(const uint32_t* dev_indices_begin, const uint32_t* dev_indices_end, int32_t* dev_output);
  void getDistances(const uint32_t* dev_indices_begin, const uint32_t* dev_indices_end, int32_t* dev_output);
  void gatherVoxelsByIndex(const uint32_t* dev_indices_begin, const uint32_t* dev_indices_end, Voxel* dev_output);
#ifdef GVX_HAVE_THRUST_DEVICE_PTR
  // The thrust::device_ptr forms the reference declares
  // (GV/voxelmap/DistanceVoxelMap.h:81,84; GV/voxelmap/TemplateVoxelMap.h:111).
  void getSquaredDistances(thrust::device_ptr<uint32_t> dev_indices_begin, thrust::device_ptr<uint32_t> dev_indices_end,
                           thrust::device_ptr<int32_t> dev_output) {
    getSquaredDistances(dev_indices_begin.get(), dev_indices_end.get(), dev_output.get());
  }
  void getDistances(thrust::device_ptr<uint32_t> dev_indices_begin, thrust::device_ptr<uint32_t> dev_indices_end,
                    thrust::device_ptr<int32_t> dev_output) {
    getDistances(dev_indices_begin.get(), dev_indices_end.get(), dev_output.get());
  }
  void gatherVoxelsByIndex(thrust::device_ptr<uint32_t> dev_indices_begin, thrust::device_ptr<uint32_t> dev_indices_end,
                           thrust::device_ptr<Voxel> dev_output_begin) {
    gatherVoxelsByIndex(dev_indices_begin.get(), dev_indices_end.get(), dev_output_begin.get());
  }
#endif
  // Host vectors; blocking (GV/voxelmap/DistanceVoxelMap.hpp:726-739,771-784).
  void getSquaredDistancesToHost(std::vector<uint32_t>& indices, std::vector<int32_t>& output);
  void getDistancesToHost(std::vector<uint32_t>& indices, std::vector<int32_t>& output);
  DistanceVoxel::pba_dist_t getSquaredObstacleDistance(const Vector3ui& pos);
  DistanceVoxel::pba_dist_t getSquaredObstacleDistance(uint32_t x, uint32_t y, uint32_t z);
  DistanceVoxel::pba_dist_t getObstacleDistance(const Vector3ui& pos);
  DistanceVoxel::pba_dist_t getObstacleDistance(uint32_t x, uint32_t y, uint32_t z);

  // TemplateVoxelMap::clone (GV/voxelmap/TemplateVoxelMap.hpp:1101-1120): copies
  // the other map's voxels when dims and voxel side length match; otherwise an
  // error message and no change.  Blocking.
  void clone(const DistanceVoxelMap& other);

  Voxel* getDeviceDataPtr();
  const Voxel* getConstDeviceDataPtr() const;
  size_t getVoxelMapSize() const { return (size_t)m_dim.x * m_dim.y * m_dim.z; }
  gvx_dvm* handle() const { return m_handle; }

 private:
  gvx_dvm* m_handle = nullptr;
};

}  // namespace voxelmap

typedef std::shared_ptr<voxelmap::DistanceVoxelMap> DistanceVoxelMapSharedPtr;

}  // namespace gpu_voxels
