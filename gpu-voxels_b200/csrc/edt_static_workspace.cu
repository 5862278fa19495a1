// EDT entry point that allocates no device memory.
//
// Who needs it: callers that must not call cudaMalloc once they are running.
// A real-time robot control loop typically forbids device allocation after
// start-up (an allocation can block for milliseconds and may fail on a busy
// GPU), and code embedded in a host application that owns all device memory
// through its own pool (a ROS node, a motion-planning plugin, a sensor
// pipeline) is handed device buffers but has no say over allocations.  The
// regular path allocates the EDT workspace when a map handle is created;
// this entry point takes only the caller's voxel buffer and uses a workspace
// that is part of the library image instead.
//
// The workspace is a file-scope __device__ array of kStaticWorkspaceWords
// 32-bit words: 64 MiB of stack area plus 8 KiB for the EDT's per-slice
// counters.  This file is its own device module (the library is built
// without relocatable device code), so when the array is placed on a GPU
// follows CUDA's module loading: under lazy loading (CUDA_MODULE_LOADING=LAZY,
// the default) at the first call on that device, under eager loading in
// every device context the process creates.  Either way it stays there until
// the process exits.  Maps whose EDT workspace would exceed it (more than
// 16,777,216 voxels once x and y are rounded up to multiples of 32; 256^3
// fits) are rejected with GVX_ERR_OUT_OF_DOMAIN.
//
// The fused y -> x sweep's bounded waits report a give-up in an error word
// inside this workspace (word dims.z + 1, zeroed by every call), which
// gvx_dvm_edt_static_workspace_check reads without a map handle.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <mutex>

#include "gvx_internal.cuh"

namespace gvx {
namespace {

constexpr uint64_t kStaticWorkspaceWords = 16ull * 1024 * 1024 + 2048;  // 64 MiB + 8 KiB
constexpr uint64_t kStaticStackVoxels = 16ull * 1024 * 1024;               // the size limit callers see
constexpr int kMaxDevices = 64;

static __device__ __align__(256) uint32_t g_edt_workspace[kStaticWorkspaceWords];

std::mutex g_setup_mutex;
uint32_t* g_workspace_addr[kMaxDevices] = {};

// Device address of the workspace on the current device.  In host code the
// array's name is only a host-side stand-in, so the address is looked up once
// per device with cudaGetSymbolAddress (with that device current) and cached
// for the life of the process.  The cache does not survive cudaDeviceReset
// (or any other teardown of the device's primary context): the module, and
// with it the array, is then placed anew at another address.
gvx_status workspace_address(uint32_t** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_status(e, "cudaGetDevice");
  if (dev < 0 || dev >= kMaxDevices) {
    set_error("device index beyond the static workspace table");
    return GVX_ERR_INVALID_ARG;
  }
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (g_workspace_addr[dev] == nullptr) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_edt_workspace);
    if (e != cudaSuccess) return cuda_status(e, "cudaGetSymbolAddress(static EDT workspace)");
    g_workspace_addr[dev] = static_cast<uint32_t*>(p);
  }
  *out = g_workspace_addr[dev];
  return GVX_OK;
}

}  // namespace
}  // namespace gvx

extern "C" gvx_status gvx_dvm_edt_static_workspace(uint32_t* d_voxels, const gvx_dims* dims, gvx_stream stream) {
  using namespace gvx;
  if (d_voxels == nullptr || dims == nullptr) {
    set_error("null argument");
    return GVX_ERR_INVALID_ARG;
  }
  if (dims->x < 1 || dims->y < 1 || dims->z < 1 || dims->x > kMaxDim || dims->y > kMaxDim || dims->z > kMaxDim) {
    set_error("every map axis must be in [1, 1023] (10-bit DistanceVoxel coordinates)");
    return GVX_ERR_OUT_OF_DOMAIN;
  }
  if (reinterpret_cast<uintptr_t>(d_voxels) % 16 != 0) {
    set_error("voxel buffer must be 16-byte aligned");
    return GVX_ERR_INVALID_ARG;
  }
  const uint64_t x32 = (dims->x + 31) / 32 * 32, y32 = (dims->y + 31) / 32 * 32;
  const uint64_t padded = std::max(x32 * dims->y, (uint64_t)dims->x * y32) * dims->z;
  if (padded > kStaticStackVoxels || edt_scratch_words_min(*dims) > kStaticWorkspaceWords) {
    set_error("map too large for the static EDT workspace: needs more than 16,777,216 voxels "
              "(x and y rounded up to multiples of 32); use gvx_dvm_create + gvx_dvm_edt");
    return GVX_ERR_OUT_OF_DOMAIN;
  }
  uint32_t* workspace = nullptr;
  gvx_status st = workspace_address(&workspace);
  if (st != GVX_OK) return st;
  return cuda_status(launch_edt(d_voxels, workspace, kStaticWorkspaceWords, *dims, as_stream(stream)), "EDT (static workspace)");
}

extern "C" gvx_status gvx_dvm_edt_static_workspace_check(const gvx_dims* dims, uint32_t* flags) {
  using namespace gvx;
  if (dims == nullptr || flags == nullptr) {
    set_error("null argument");
    return GVX_ERR_INVALID_ARG;
  }
  if (dims->z < 1 || dims->z > kMaxDim) {
    set_error("every map axis must be in [1, 1023] (10-bit DistanceVoxel coordinates)");
    return GVX_ERR_OUT_OF_DOMAIN;
  }
  // The counter area is [slice counters: z][queue head][error word]; a copy
  // from the symbol needs no device address and allocates nothing.
  cudaError_t e = cudaDeviceSynchronize();
  if (e == cudaSuccess)
    e = cudaMemcpyFromSymbol(flags, g_edt_workspace, sizeof(uint32_t), (size_t)(dims->z + 1) * sizeof(uint32_t),
                             cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_status(e, "static-workspace EDT check");
  if (*flags != 0) {
    set_error("EDT (static workspace): a slice wait of the fused y->x sweep gave up (results invalid)");
    return GVX_ERR_TIMEOUT;
  }
  return GVX_OK;
}
