// Host-side BitVector<N> / BitVoxel<N> of the gpu_voxels C++ API (gpu-voxels
// GV/helpers/BitVector.h:44-300, GV/voxel/BitVoxel.h:40-110): N bits as N/8
// bytes, bit k in byte k >> 3 at position k & 7 -- the layout of the 32-byte
// voxels on the device.  Used to pass and return meaning sets (for example
// the types in collision).
#pragma once

#include <stdint.h>
#include <string.h>

#include "../helpers/common_defines.h"

namespace gpu_voxels {

template <size_t num_bits>
class BitVector {
  static_assert(num_bits % 32 == 0, "BitVector length must be a multiple of 32");

 public:
  typedef uint8_t item_type;
  static const size_t m_size = num_bits / 8;

  BitVector() { clear(); }
  void clear() { memset(m_bytes, 0, m_size); }
  bool isZero() const {
    for (size_t i = 0; i < m_size; ++i)
      if (m_bytes[i]) return false;
    return true;
  }
  // All bits but bit 0 (eBVM_FREE) clear (BitVector.h:184-198).
  bool noneButEmpty() const {
    if (m_bytes[0] & 0xFE) return false;
    for (size_t i = 1; i < m_size; ++i)
      if (m_bytes[i]) return false;
    return true;
  }
  bool getBit(uint32_t index) const { return (m_bytes[index >> 3] >> (index & 7)) & 1u; }
  void setBit(uint32_t index) { m_bytes[index >> 3] |= item_type(1u << (index & 7)); }
  void clearBit(uint32_t index) { m_bytes[index >> 3] &= item_type(~(1u << (index & 7))); }
  // The byte holding the bit at `index` (given in bits).
  item_type getByte(uint32_t index, uint8_t = 0) const { return m_bytes[index >> 3]; }
  void setByte(uint32_t index, item_type data) { m_bytes[index >> 3] = data; }
  BitVector operator|(const BitVector& o) const {
    BitVector r;
    for (size_t i = 0; i < m_size; ++i) r.m_bytes[i] = m_bytes[i] | o.m_bytes[i];
    return r;
  }
  BitVector operator&(const BitVector& o) const {
    BitVector r;
    for (size_t i = 0; i < m_size; ++i) r.m_bytes[i] = m_bytes[i] & o.m_bytes[i];
    return r;
  }
  BitVector operator~() const {
    BitVector r;
    for (size_t i = 0; i < m_size; ++i) r.m_bytes[i] = item_type(~m_bytes[i]);
    return r;
  }
  BitVector& operator|=(const BitVector& o) {
    for (size_t i = 0; i < m_size; ++i) m_bytes[i] |= o.m_bytes[i];
    return *this;
  }
  bool operator==(const BitVector& o) const { return memcmp(m_bytes, o.m_bytes, m_size) == 0; }
  item_type* data() { return m_bytes; }
  const item_type* data() const { return m_bytes; }

 private:
  item_type m_bytes[m_size];
};

template <size_t length>
class BitVoxel {
 public:
  BitVector<length>& bitVector() { return m_bit_vector; }
  const BitVector<length>& bitVector() const { return m_bit_vector; }
  // BitVoxel::insert: sets the meaning's bit.
  void insert(BitVoxelMeaning voxel_meaning) { m_bit_vector.setBit((uint32_t)voxel_meaning); }
  bool isOccupied(float) const { return !m_bit_vector.noneButEmpty(); }

 private:
  BitVector<length> m_bit_vector;
};

typedef BitVoxel<BIT_VECTOR_LENGTH> BitVectorVoxel;
static_assert(sizeof(BitVectorVoxel) == 32, "a BitVoxel<256> is 32 bytes");

}  // namespace gpu_voxels
