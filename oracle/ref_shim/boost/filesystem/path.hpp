// Minimal stand-in for boost::filesystem::path so that gpu-voxels'
// common_defines.h compiles without Boost (used only by the oracle/_ref build).
#pragma once
#include <string>
namespace boost {
namespace filesystem {
struct path {
  std::string s;
  path() {}
  path(const char* c) : s(c) {}
  path(const std::string& c) : s(c) {}
  path operator/(const path& o) const { return path(s + "/" + o.s); }
  std::string string() const { return s; }
};
}  // namespace filesystem
}  // namespace boost
