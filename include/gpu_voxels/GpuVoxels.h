// Facade of the gpu_voxels C++ API (gpu-voxels GV/GpuVoxels.h:60-340): a
// process-wide registry of named maps sharing one set of dimensions and one
// voxel side length.  Map types on the distance-field collision path are
// supported: MT_DISTANCE_VOXELMAP, MT_BITVECTOR_VOXELMAP, MT_BITVECTOR_VOXELLIST.
#pragma once

#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "GpuVoxelsMap.h"
#include "helpers/common_defines.h"
#include "helpers/cuda_datatypes.h"
#include "voxellist/BitVoxelList.h"
#include "voxelmap/BitVoxelMap.h"
#include "voxelmap/DistanceVoxelMap.h"
#include "voxelmap/ProbVoxelMap.h"

namespace gpu_voxels {

class GpuVoxels;
typedef std::shared_ptr<GpuVoxels> GpuVoxelsSharedPtr;

class GpuVoxels {
 public:
  // getInstance (GV/GpuVoxels.cpp:69-78); the first call selects and checks the device.
  static GpuVoxelsSharedPtr getInstance();
  ~GpuVoxels();

  void initialize(uint32_t dim_x, uint32_t dim_y, uint32_t dim_z, float voxel_side_length);
  // addMap (GV/GpuVoxels.cpp:164-302): the new map, or an empty pointer for
  // a duplicate name or a type outside this library (the reference returns
  // an empty pointer for both too).
  GpuVoxelsMapSharedPtr addMap(const MapType map_type, const std::string& map_name);
  bool delMap(const std::string& map_name);
  GpuVoxelsMapSharedPtr getMap(const std::string& map_name);
  bool clearMap(const std::string& map_name);
  // insertPointCloudIntoMap (GV/GpuVoxels.cpp:443-469)
  bool insertPointCloudIntoMap(const std::vector<Vector3f>& point_cloud, std::string map_name,
                               const BitVoxelMeaning voxel_meaning);
  void getDimensions(uint32_t& dim_x, uint32_t& dim_y, uint32_t& dim_z) const;
  void getDimensions(Vector3ui& dim) const;
  void getVoxelSideLength(float& voxel_side_length) const;
  // visualizeMap (GV/GpuVoxels.cpp:585-594) hands the map to the separate
  // shared-memory viewer program, which this library does not provide: false
  // always, with the reference's message for an unknown map name.
  bool visualizeMap(const std::string& map_name, const bool force_repaint = true);

 private:
  GpuVoxels();
  static std::mutex s_instance_mutex;
  static GpuVoxelsSharedPtr s_instance;
  Vector3ui m_dim;
  float m_voxel_side_length = 0.f;
  std::map<std::string, GpuVoxelsMapSharedPtr> m_managed_maps;
  mutable std::recursive_mutex m_mutex;
};

}  // namespace gpu_voxels
