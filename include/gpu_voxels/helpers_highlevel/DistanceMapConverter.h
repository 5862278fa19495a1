// distance_map_converter of the gpu_voxels C++ API
// (gpu-voxels GV/helpers_highlevel/DistanceMapConverter.h:27-72) over the gvx C ABI.
#pragma once

#include <stddef.h>

#include "../voxellist/BitVoxelList.h"
#include "../voxelmap/DistanceVoxelMap.h"

namespace gpu_voxels {
namespace distance_map_converter {

// Voxels whose free-space byte (DistanceVoxelMap::extract_distances at robot
// radius 0) lies in [min_dist, max_dist] become `result`, in id order, each
// voxel with eBVM_OCCUPIED and swept-volume bits 4 .. 4 + byte - 1
// (DistanceMapConverter.cu:156-196).  Returns the number of entries.
size_t extract_given_distances(const voxelmap::DistanceVoxelMap& dist_map, free_space_t min_dist,
                               free_space_t max_dist, BitVectorVoxelList& result);

}  // namespace distance_map_converter
}  // namespace gpu_voxels
