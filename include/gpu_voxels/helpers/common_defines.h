// Enumerations and constants of the gpu_voxels C++ API, with the values of
// gpu-voxels' GV/helpers/common_defines.h (MapType :153-172, BitVoxelMeaning
// :51-64, PBA constants :111-139) so existing call sites compile unchanged.
#pragma once

#include <stddef.h>
#include <stdint.h>

namespace gpu_voxels {

static const size_t BIT_VECTOR_LENGTH = 256;

enum BitVoxelMeaning {
  eBVM_FREE = 0,
  eBVM_OCCUPIED = 1,
  eBVM_COLLISION = 2,
  eBVM_UNKNOWN = 3,
  eBVM_SWEPT_VOLUME_START = 4,
  eBVM_SWEPT_VOLUME_END = 254,
  // the swept-volume range read as occupancy probabilities by ProbVoxelMap
  eBVM_MAX_FREE_PROB = 4,
  eBVM_UNCERTAIN_OCC_PROB = 129,
  eBVM_MAX_OCC_PROB = 254,
  eBVM_UNDEFINED = 255
};

enum MapType {
  MT_BITVECTOR_VOXELMAP,
  MT_BITVECTOR_VOXELLIST,
  MT_BITVECTOR_OCTREE,
  MT_BITVECTOR_MORTON_VOXELLIST,
  MT_PROBAB_VOXELMAP,
  MT_PROBAB_VOXELLIST,
  MT_PROBAB_OCTREE,
  MT_PROBAB_MORTON_VOXELLIST,
  MT_COUNTING_VOXELLIST,
  MT_DISTANCE_VOXELMAP
};

static const int32_t PBA_UNINITIALISED_COORD = 1023;
static const int32_t MAX_OBSTACLE_DISTANCE = 2147483647;
static const uint32_t PBA_DEFAULT_M1_BLOCK_SIZE = 64;
static const uint32_t PBA_DEFAULT_M2_BLOCK_SIZE = 64;
static const uint32_t PBA_DEFAULT_M3_BLOCK_SIZE = 16;

typedef uint32_t MapVoxelID;
// free-space byte and flood-fill distance types (GV/voxel/DistanceVoxel.h:149,203)
typedef int8_t free_space_t;
typedef int16_t manhattan_dist_t;
static const int MANHATTAN_DISTANCE_UNINITIALIZED = 32767;  // SHRT_MAX
static const int MANHATTAN_DISTANCE_START = MANHATTAN_DISTANCE_UNINITIALIZED - 1;
static const int MANHATTAN_DISTANCE_TOO_CLOSE = MANHATTAN_DISTANCE_UNINITIALIZED - 2;

namespace voxelmap {
class DistanceVoxelMap;
template <size_t length>
class BitVoxelMap;
}  // namespace voxelmap
namespace voxellist {
template <size_t length, class VoxelIDType>
class BitVoxelList;
}  // namespace voxellist

typedef voxelmap::BitVoxelMap<BIT_VECTOR_LENGTH> BitVectorVoxelMap;
typedef voxellist::BitVoxelList<BIT_VECTOR_LENGTH, MapVoxelID> BitVectorVoxelList;

}  // namespace gpu_voxels
