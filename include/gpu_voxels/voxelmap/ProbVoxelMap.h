// ProbVoxelMap of the gpu_voxels C++ API (gpu-voxels GV/voxelmap/ProbVoxelMap.h:36-90)
// over the gvx C ABI: one int8 occupancy per voxel (ProbabilisticVoxel,
// GV/voxel/ProbabilisticVoxel.h), UNKNOWN (-128) after creation and clearMap.
// It is the input of DistanceVoxelMap::mergeOccupied.
#pragma once

#include <stdint.h>

#include <vector>

#include "../GpuVoxelsMap.h"

struct gvx_pvm;

namespace gpu_voxels {

typedef int8_t Probability;
static const Probability UNKNOWN_PROBABILITY = Probability(-128);
static const Probability MIN_PROBABILITY = Probability(-127);
static const Probability MAX_PROBABILITY = Probability(127);

namespace voxelmap {

class ProbVoxelMap : public GpuVoxelsMap {
 public:
  ProbVoxelMap(const Vector3ui dim, const float voxel_side_length, const MapType map_type = MT_PROBAB_VOXELMAP);
  ~ProbVoxelMap() override;

  void clearMap() override;
  // ProbabilisticVoxel::insert per point (GV/voxel/ProbabilisticVoxel.hpp:78-100).
  void insertPointCloud(const std::vector<Vector3f>& points, BitVoxelMeaning voxel_meaning) override;
  void insertPointCloud(const Vector3f* d_points, uint32_t size, BitVoxelMeaning voxel_meaning) override;
  size_t getMemoryUsage() const override;
  bool writeToDisk(const std::string path) override;
  bool readFromDisk(const std::string path) override;

  // TemplateVoxelMap::clone (GV/voxelmap/TemplateVoxelMap.hpp:1101-1120): copies
  // the other map's voxels when dims and voxel side length match; otherwise an
  // error message and no change.  Blocking.
  void clone(const ProbVoxelMap& other);

  Probability* getDeviceDataPtr();
  size_t getVoxelMapSize() const { return (size_t)m_dim.x * m_dim.y * m_dim.z; }
  gvx_pvm* handle() const { return m_handle; }

 private:
  gvx_pvm* m_handle = nullptr;
};

}  // namespace voxelmap

typedef std::shared_ptr<voxelmap::ProbVoxelMap> ProbVoxelMapSharedPtr;

}  // namespace gpu_voxels
