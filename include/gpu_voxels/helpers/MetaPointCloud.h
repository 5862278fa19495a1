// MetaPointCloud of the gpu_voxels C++ API (gpu-voxels GV/helpers/MetaPointCloud.h:40-230):
// an ordered set of point clouds (typically one per robot link) kept on the
// host and mirrored to one contiguous device array when a map reads it.
// Provided: the constructors from sizes and from point vectors, addCloud,
// updatePointCloud, syncToDevice and the size and host accessors.  Not
// provided: file loading and the transform* members (robot kinematics is not
// part of this library).
#pragma once

#include <stdint.h>

#include <vector>

#include "cuda_datatypes.h"

namespace gpu_voxels {

class MetaPointCloud {
 public:
  MetaPointCloud() = default;
  explicit MetaPointCloud(const std::vector<uint32_t>& point_cloud_sizes);
  explicit MetaPointCloud(const std::vector<std::vector<Vector3f> >& point_clouds);
  MetaPointCloud(const MetaPointCloud& other);
  MetaPointCloud& operator=(const MetaPointCloud& other);
  ~MetaPointCloud();

  void addCloud(uint32_t cloud_size);
  void addCloud(const std::vector<Vector3f>& cloud, bool sync = false);
  // Replaces cloud `cloud` (its size may change).
  void updatePointCloud(uint16_t cloud, const std::vector<Vector3f>& pointcloud, bool sync = false);
  // Copies every cloud to the device array (done on demand by the maps).
  void syncToDevice() const;

  uint16_t getNumberOfPointclouds() const { return (uint16_t)m_clouds.size(); }
  uint32_t getPointcloudSize(uint16_t cloud = 0) const { return (uint32_t)m_clouds.at(cloud).size(); }
  uint32_t getAccumulatedPointcloudSize() const;
  const std::vector<uint32_t>& getPointcloudSizes() const { return m_sizes; }
  const Vector3f* getPointCloud(uint16_t cloud) const { return m_clouds.at(cloud).data(); }

  // gvx: the device copy (all clouds back to back, xyz floats) and the
  // first-point offsets of every cloud plus the total.
  const float* deviceXYZ() const;
  std::vector<uint64_t> cloudOffsets() const;

 private:
  std::vector<std::vector<Vector3f> > m_clouds;
  std::vector<uint32_t> m_sizes;
  mutable float* m_dev_xyz = nullptr;
  mutable uint64_t m_dev_capacity = 0;  // points
  mutable bool m_dirty = true;
};

}  // namespace gpu_voxels
