// Abstract map of the gpu_voxels C++ API (gpu-voxels GV/GpuVoxelsMap.h:49-290):
// every map has a type, dimensions, a voxel side length and a recursive timed
// mutex that each operation takes, like the reference's
// boost::recursive_timed_mutex (std:: in place of boost::).
#pragma once

#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "helpers/common_defines.h"
#include "helpers/cuda_datatypes.h"
#include "voxel/BitVoxel.h"

namespace gpu_voxels {

class MetaPointCloud;

class GpuVoxelsMap {
 public:
  GpuVoxelsMap(MapType type, const Vector3ui& dims, float voxel_side_length)
      : m_map_type(type), m_dim(dims), m_voxel_side_length(voxel_side_length) {}
  virtual ~GpuVoxelsMap();

  GpuVoxelsMap(const GpuVoxelsMap&) = delete;
  GpuVoxelsMap& operator=(const GpuVoxelsMap&) = delete;

  // Down-cast, as GpuVoxelsMap::as<T>() (GV/GpuVoxelsMap.h:70-87).
  template <class T>
  T* as() { return dynamic_cast<T*>(this); }
  template <class T>
  const T* as() const { return dynamic_cast<const T*>(this); }

  MapType getMapType() const { return m_map_type; }
  virtual Vector3ui getDimensions() const { return m_dim; }
  float getVoxelSideLength() const { return m_voxel_side_length; }

  virtual void clearMap() = 0;
  virtual void insertPointCloud(const std::vector<Vector3f>& points, BitVoxelMeaning voxel_meaning) = 0;
  // Device-resident points (n packed Vector3f on the current device).
  virtual void insertPointCloud(const Vector3f* d_points, uint32_t size, BitVoxelMeaning voxel_meaning) = 0;
  // Number of bytes of device memory held by the map.
  virtual size_t getMemoryUsage() const = 0;
  // TemplateVoxelMap::writeToDisk / readFromDisk (GV/voxelmap/TemplateVoxelMap.hpp:906-1039):
  // the reference's binary map file; false on I/O errors or (reading) another
  // map type or dims.  Maps without a file form return false.
  virtual bool writeToDisk(const std::string path) { (void)path; return false; }
  virtual bool readFromDisk(const std::string path) { (void)path; return false; }

  // insertMetaPointCloud (GV/GpuVoxelsMap.h:138): sub-cloud k is inserted with
  // voxel_meanings[k] (one meaning per sub-cloud).
  virtual void insertMetaPointCloud(const MetaPointCloud& meta_point_cloud,
                                    const std::vector<BitVoxelMeaning>& voxel_meanings);
  // insertMetaPointCloudWithSelfCollisionCheck (GV/GpuVoxelsMap.h:141-153):
  // inserts the sub-clouds in order, each checked against what the earlier
  // ones (and the map before) hold; true if any sub-cloud collided.  Empty
  // meanings / masks select the defaults (eBVM_SWEPT_VOLUME_START + k; every
  // bit but eBVM_COLLISION and the own meaning).  Provided by BitVoxelMap;
  // other maps return false, as the reference's DistanceVoxelMap does.
  virtual bool insertMetaPointCloudWithSelfCollisionCheck(
      const MetaPointCloud* robot_links,
      const std::vector<BitVoxelMeaning>& voxel_meanings = std::vector<BitVoxelMeaning>(),
      const std::vector<BitVector<BIT_VECTOR_LENGTH> >& collision_masks = std::vector<BitVector<BIT_VECTOR_LENGTH> >(),
      BitVector<BIT_VECTOR_LENGTH>* colliding_meanings = NULL) {
    (void)robot_links;
    (void)voxel_meanings;
    (void)collision_masks;
    (void)colliding_meanings;
    return false;
  }
  // The map's lock, for operations that lock two maps together.
  std::recursive_timed_mutex& mutexRef() const { return m_mutex; }

 protected:
  typedef std::lock_guard<std::recursive_timed_mutex> lock_guard;
  // Device staging area of the host-vector overloads (point clouds, query
  // ids and results): enlarged when a call needs more than it holds and
  // otherwise reused, so repeated calls allocate no device memory.  Freed
  // with the map.  Callers hold the map's mutex.
  void* stagingBuffer(size_t bytes) const;
  // A host point cloud copied into the staging area (nullptr when empty).
  const Vector3f* stagePoints(const std::vector<Vector3f>& points) const;
  MapType m_map_type;
  Vector3ui m_dim;
  float m_voxel_side_length;
  mutable std::recursive_timed_mutex m_mutex;

 private:
  mutable void* m_staging = nullptr;
  mutable size_t m_staging_bytes = 0;
};

typedef std::shared_ptr<GpuVoxelsMap> GpuVoxelsMapSharedPtr;

}  // namespace gpu_voxels
