// Vector types of the gpu_voxels C++ API (same names, members and layout as
// gpu-voxels' Vector3f / Vector3ui / Vector3i, GV/helpers/cuda_vectors.h:40-210,
// so point clouds pass through unchanged: Vector3f is 3 packed floats).
#pragma once

#include <stdint.h>

#include <ostream>

namespace gpu_voxels {

struct Vector3ui {
  uint32_t x, y, z;
  Vector3ui() : x(0), y(0), z(0) {}
  explicit Vector3ui(uint32_t v) : x(v), y(v), z(v) {}
  Vector3ui(uint32_t x_, uint32_t y_, uint32_t z_) : x(x_), y(y_), z(z_) {}
  bool operator==(const Vector3ui& o) const { return x == o.x && y == o.y && z == o.z; }
  bool operator!=(const Vector3ui& o) const { return !(*this == o); }
};

struct Vector3i {
  int32_t x, y, z;
  Vector3i() : x(0), y(0), z(0) {}
  explicit Vector3i(int32_t v) : x(v), y(v), z(v) {}
  Vector3i(int32_t x_, int32_t y_, int32_t z_) : x(x_), y(y_), z(z_) {}
  bool operator==(const Vector3i& o) const { return x == o.x && y == o.y && z == o.z; }
  bool operator!=(const Vector3i& o) const { return !(*this == o); }
};

struct Vector3f {
  float x, y, z;
  Vector3f() : x(0.f), y(0.f), z(0.f) {}
  explicit Vector3f(float v) : x(v), y(v), z(v) {}
  Vector3f(float x_, float y_, float z_) : x(x_), y(y_), z(z_) {}
};
static_assert(sizeof(Vector3f) == 12, "Vector3f must be three packed floats");

inline std::ostream& operator<<(std::ostream& o, const Vector3ui& v) { return o << "(" << v.x << ", " << v.y << ", " << v.z << ")"; }
inline std::ostream& operator<<(std::ostream& o, const Vector3i& v) { return o << "(" << v.x << ", " << v.y << ", " << v.z << ")"; }
inline std::ostream& operator<<(std::ostream& o, const Vector3f& v) { return o << "(" << v.x << ", " << v.y << ", " << v.z << ")"; }

}  // namespace gpu_voxels
