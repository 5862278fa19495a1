// BitVoxelList<256, MapVoxelID> of the gpu_voxels C++ API (gpu-voxels
// GV/voxellist/BitVoxelList.h:40-170) over the gvx C ABI: a sorted list of
// unique voxel ids with 32-byte bit vectors, tied to a reference map's dims.
#pragma once

#include <stdint.h>

#include <vector>

#include "../GpuVoxelsMap.h"
#include "../voxelmap/BitVoxelMap.h"

struct gvx_blist;

namespace gpu_voxels {
namespace voxellist {

template <size_t length, class VoxelIDType>
class BitVoxelList : public GpuVoxelsMap {
  static_assert(length == BIT_VECTOR_LENGTH, "only BitVoxelList<256, uint32> is provided");

 public:
  BitVoxelList(const Vector3ui ref_map_dim, const float voxel_side_length, const MapType map_type = MT_BITVECTOR_VOXELLIST);
  ~BitVoxelList() override;

  void clearMap() override;
  void insertPointCloud(const std::vector<Vector3f>& points, BitVoxelMeaning voxel_meaning) override;
  void insertPointCloud(const Vector3f* d_points, uint32_t size, BitVoxelMeaning voxel_meaning) override;
  size_t getMemoryUsage() const override;
  // As in the reference, a list's "dimensions" are its length in x.
  Vector3ui getDimensions() const override;

  // collideWith(const BitVectorVoxelMap*) (GV/voxellist/BitVoxelList.hpp:71-77).
  // Returns SSIZE_MAX when the map's dims differ from the list's reference dims.
  size_t collideWith(const voxelmap::BitVoxelMap<length>* map, float coll_threshold = 1.0,
                     const Vector3i& offset = Vector3i());
  // collideWith(const ProbVoxelMap*) (GV/voxellist/BitVoxelList.hpp:63-69,
  // DefaultCollider GV/voxel/DefaultCollider.hpp:68-73): entries whose map
  // voxel (id + offset, inside the map) has an occupancy reaching
  // floatToProbability(coll_threshold) and that hold a meaning other than
  // eBVM_FREE; they get eBVM_COLLISION.  SSIZE_MAX when the map's dims
  // differ from the list's reference dims.
  size_t collideWith(const voxelmap::ProbVoxelMap* map, float coll_threshold = 1.0,
                     const Vector3i& offset = Vector3i());
  // collideWith(const BitVectorVoxelList*) (GV/voxellist/BitVoxelList.hpp:79-92):
  // number of this list's ids present in `other`; offsets are not supported (returns 0).
  size_t collideWith(const BitVoxelList<length, VoxelIDType>* other, float coll_threshold = 1.0,
                     const Vector3i& offset = Vector3i());

  // collideWithTypes / collideWithTypeMask (GV/voxellist/BitVoxelList.hpp:94-246):
  // types_in_collision receives the OR of the colliding entries' types (for a
  // list: of both lists' entries at the common ids); against maps colliding
  // entries get eBVM_COLLISION.  SSIZE_MAX when a map's dims differ from the
  // list's reference dims; list vs list with an offset returns 0.
  size_t collideWithTypes(const voxelmap::BitVoxelMap<length>* map, BitVectorVoxel& types_in_collision,
                          float coll_threshold = 1.0, const Vector3i& offset = Vector3i());
  size_t collideWithTypes(const voxelmap::ProbVoxelMap* map, BitVectorVoxel& types_in_collision,
                          float coll_threshold = 1.0, const Vector3i& offset = Vector3i());
  size_t collideWithTypes(const BitVoxelList<length, VoxelIDType>* other, BitVectorVoxel& types_in_collision,
                          float coll_threshold = 1.0, const Vector3i& offset = Vector3i());
  size_t collideWithTypeMask(const voxelmap::BitVoxelMap<length>* map, const BitVectorVoxel& types_to_check,
                             float coll_threshold = 1.0, const Vector3i& offset = Vector3i());

  // insertCoordinateList (GV/voxellist/TemplateVoxelList.hpp:396-438): voxel
  // coordinates (host or device) inserted with `voxel_meaning`, as points at
  // the voxel centres; coordinates outside the reference dims are dropped.
  void insertCoordinateList(const std::vector<Vector3ui>& coordinates, const BitVoxelMeaning voxel_meaning);
  void insertCoordinateList(const Vector3ui* d_coordinates, uint32_t size, const BitVoxelMeaning voxel_meaning);
  // copyCoordsToHost (TemplateVoxelList.hpp:292-299): the entries' voxel
  // coordinates, in id order.
  void copyCoordsToHost(std::vector<Vector3ui>& host_vec) const;
  // shiftLeftSweptVolumeIDs (GV/voxellist/BitVoxelList.hpp:641-664): meaning k
  // of every entry becomes k - shift_size (<= 56), meanings 0..3 cleared.
  void shiftLeftSweptVolumeIDs(uint8_t shift_size);
  // clearBitVoxelMeaning: the meaning's bit cleared in every entry (the
  // reference's list reports this as not yet supported).
  void clearBitVoxelMeaning(BitVoxelMeaning voxel_meaning);

  // Host copies of the ids and the 32-byte voxels.
  void copyIdsToHost(std::vector<VoxelIDType>& ids) const;
  void copyVoxelsToHost(std::vector<uint8_t>& voxels) const;
  gvx_blist* handle() const { return m_handle; }

 private:
  gvx_blist* m_handle = nullptr;
  uint64_t* m_dev_count = nullptr;
  uint8_t* m_dev_types = nullptr;  // 32 B result + 32 B mask
};

extern template class BitVoxelList<BIT_VECTOR_LENGTH, MapVoxelID>;

}  // namespace voxellist
}  // namespace gpu_voxels
