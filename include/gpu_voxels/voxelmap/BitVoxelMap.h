// BitVoxelMap<256> of the gpu_voxels C++ API (gpu-voxels
// GV/voxelmap/BitVoxelMap.h:40-120) over the gvx C ABI: 32-byte bit-vector
// voxels, point insertion with a meaning, and the collideWith counts.
#pragma once

#include <stdint.h>

#include <vector>

#include "../GpuVoxelsMap.h"
#include "../helpers/MetaPointCloud.h"
#include "../voxel/BitVoxel.h"
#include "ProbVoxelMap.h"

struct gvx_bvm;

namespace gpu_voxels {
namespace voxelmap {

template <size_t length>
class BitVoxelMap : public GpuVoxelsMap {
  static_assert(length == BIT_VECTOR_LENGTH, "only BitVoxelMap<256> is provided");

 public:
  BitVoxelMap(const Vector3ui dim, const float voxel_side_length, const MapType map_type = MT_BITVECTOR_VOXELMAP);
  ~BitVoxelMap() override;

  void clearMap() override;
  void insertPointCloud(const std::vector<Vector3f>& points, BitVoxelMeaning voxel_meaning) override;
  void insertPointCloud(const Vector3f* d_points, uint32_t size, BitVoxelMeaning voxel_meaning) override;
  size_t getMemoryUsage() const override;
  bool writeToDisk(const std::string path) override;
  bool readFromDisk(const std::string path) override;

  // collideWith(const BitVectorVoxelMap*, float, const Vector3i&) (GV/voxelmap/BitVoxelMap.hpp:198-203):
  // voxels where both maps hold a meaning other than eBVM_FREE, this map
  // shifted by `offset`; colliding voxels of this map get eBVM_COLLISION.
  size_t collideWith(const BitVoxelMap<length>* map, float coll_threshold = 1.0, const Vector3i& offset = Vector3i());
  // collideWith(const ProbVoxelMap*, float, const Vector3i&) (GV/voxelmap/BitVoxelMap.hpp:205-210,
  // DefaultCollider GV/voxel/DefaultCollider.hpp:68-73): voxels where the
  // ProbVoxelMap's occupancy reaches floatToProbability(coll_threshold) and
  // this map (shifted by `offset`) holds a meaning other than eBVM_FREE;
  // colliding voxels of this map get eBVM_COLLISION.
  size_t collideWith(const ProbVoxelMap* map, float coll_threshold = 1.0, const Vector3i& offset = Vector3i());

  // collideWithTypes (GV/voxelmap/BitVoxelMap.hpp:212-224): the swept-volume
  // types colliding with `map` (with a ProbVoxelMap: this map's types where
  // its occupancy reaches the threshold) are OR-ed into types_in_collision;
  // colliding voxels get eBVM_COLLISION.  `offset` is ignored, as in the reference.
  size_t collideWithTypes(const BitVoxelMap<length>* map, BitVectorVoxel& types_in_collision,
                          float coll_threshold = 1.0, const Vector3i& offset = Vector3i());
  size_t collideWithTypes(const ProbVoxelMap* map, BitVectorVoxel& types_in_collision, float coll_threshold = 1.0,
                          const Vector3i& offset = Vector3i());

  // clearBit / clearBits / clearBitVoxelMeaning (GV/voxelmap/BitVoxelMap.hpp:63-88,343-347):
  // the given bit(s) cleared in every voxel.
  void clearBit(const uint32_t bit_index);
  void clearBits(BitVector<length> bits);
  void clearBitVoxelMeaning(BitVoxelMeaning voxel_meaning);
  // shiftLeftSweptVolumeIDs (BitVoxelMap.hpp:349-361): swept-volume meaning k
  // becomes k - shift_size in every voxel, meanings 0..3 are cleared; shifts
  // above 56 are refused (message, no change), as in the reference.
  void shiftLeftSweptVolumeIDs(uint8_t shift_size);

  // insertMetaPointCloudWithSelfCollisionCheck (GV/voxelmap/BitVoxelMap.hpp:227-341):
  // sub-cloud k goes in after sub-clouds 0 .. k-1; a point hits when its
  // voxel & collision_masks[k] holds a meaning other than eBVM_FREE; the hit
  // meanings and the sub-cloud's own meaning go to colliding_meanings and the
  // voxel gets eBVM_COLLISION.  Returns whether any sub-cloud hit.
  bool insertMetaPointCloudWithSelfCollisionCheck(
      const MetaPointCloud* robot_links,
      const std::vector<BitVoxelMeaning>& voxel_meanings = std::vector<BitVoxelMeaning>(),
      const std::vector<BitVector<length> >& collision_masks = std::vector<BitVector<length> >(),
      BitVector<length>* colliding_meanings = NULL) override;

  // TemplateVoxelMap::clone (GV/voxelmap/TemplateVoxelMap.hpp:1101-1120): copies
  // the other map's voxels when dims and voxel side length match; otherwise an
  // error message and no change.  Blocking.
  void clone(const BitVoxelMap& other);

  // Raw 32-byte voxels on the device.
  uint8_t* getDeviceDataPtr();
  size_t getVoxelMapSize() const { return (size_t)m_dim.x * m_dim.y * m_dim.z; }
  gvx_bvm* handle() const { return m_handle; }

 private:
  gvx_bvm* m_handle = nullptr;
  uint64_t* m_dev_count = nullptr;
  uint8_t* m_dev_types = nullptr;
};

extern template class BitVoxelMap<BIT_VECTOR_LENGTH>;

}  // namespace voxelmap
}  // namespace gpu_voxels
