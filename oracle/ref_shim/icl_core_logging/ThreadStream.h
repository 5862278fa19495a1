// No-op stand-in for icl_core's log stream (oracle/_ref build only).
#pragma once
#include <cstdint>
#include <iostream>
namespace icl_core {
namespace logging {
struct ThreadStream {
  template <class T>
  ThreadStream& operator<<(const T&) { return *this; }
  ThreadStream& operator<<(std::ostream& (*)(std::ostream&)) { return *this; }
};
inline std::ostream& endl(std::ostream& o) { return o; }
}  // namespace logging
}  // namespace icl_core
