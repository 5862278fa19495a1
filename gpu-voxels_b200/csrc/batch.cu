// Batched processing of many DistanceVoxelMaps of uneven dims (no
// counterpart in gpu-voxels, which handles one map per call with a device
// synchronisation after every step).
//
// A gvx_batch holds a device table of map descriptors.  Clear, voxelisation
// and trilinear queries run as one launch each over all maps; the EDT runs
// its three passes over all maps; the whole step (clear -> insert -> EDT ->
// queries) can be recorded once as a CUDA graph and replayed with a single
// launch call.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <new>
#include <string>
#include <vector>

#include "gvx_internal.cuh"
#include "trilinear.cuh"

namespace gvx {
namespace {

// clearMap for every map: CTA row y clears map y.
__global__ void batch_clear_kernel(const BatchMap* __restrict__ maps) {
  const BatchMap m = maps[blockIdx.y];
  const uint64_t n4 = m.nvox / 4;
  const uint4 u = make_uint4(kDvUninit, kDvUninit, kDvUninit, kDvUninit);
  uint4* v4 = reinterpret_cast<uint4*>(m.vox);
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += stride) __stcs(v4 + i, u);
  if (blockIdx.x == 0 && threadIdx.x < (m.nvox & 3)) m.vox[n4 * 4 + threadIdx.x] = kDvUninit;
}

// Map owning item i of a CSR layout: last k with offsets[k] <= i.
__device__ __forceinline__ uint32_t owner(const uint64_t* __restrict__ offsets, uint32_t n, uint64_t i) {
  uint32_t lo = 0, hi = n;
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (__ldg(offsets + mid) <= i) lo = mid; else hi = mid;
  }
  return lo;
}

// kernelInsertGlobalPointCloud<DistanceVoxel> for every map at once: point i
// belongs to map owner(offsets, i).
__global__ void batch_insert_kernel(const BatchMap* __restrict__ maps, uint32_t n_maps, const float* __restrict__ xyz,
                                    const uint64_t* __restrict__ offsets, uint64_t n) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const BatchMap m = maps[owner(offsets, n_maps, i)];
    const uint32_t x = coord_to_voxel(__ldg(xyz + 3 * i), m.side), y = coord_to_voxel(__ldg(xyz + 3 * i + 1), m.side),
                   z = coord_to_voxel(__ldg(xyz + 3 * i + 2), m.side);
    if (x < (uint32_t)m.X && y < (uint32_t)m.Y && z < (uint32_t)m.Z)
      m.vox[((uint64_t)z * m.Y + y) * m.X + x] = dv_pack(x, y, z);
  }
}

// Trilinear distance (+ gradient) for queries of many maps: query i reads map map_of[i].
__global__ void batch_trilinear_kernel(const BatchMap* __restrict__ maps, const float* __restrict__ xyz,
                                       const uint32_t* __restrict__ map_of, uint64_t n, float* __restrict__ dist,
                                       float* __restrict__ grad) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const BatchMap bm = maps[__ldg(map_of + i)];
    const MapView m{bm.vox, bm.X, bm.Y, bm.Z, bm.side, (reinterpret_cast<uintptr_t>(bm.vox) & 15u) == 0,
                    (uint64_t)bm.X * bm.Y * bm.Z};
    const Tri t = trilinear(m, __ldg(xyz + 3 * i), __ldg(xyz + 3 * i + 1), __ldg(xyz + 3 * i + 2));
    dist[i] = t.d * m.side;
    if (grad != nullptr) {
      grad[3 * i] = t.gx;
      grad[3 * i + 1] = t.gy;
      grad[3 * i + 2] = t.gz;
    }
  }
}

int sms() { return device_sms(); }

gvx_status fail(gvx_status st, const char* msg) {
  set_error(msg);
  return st;
}

}  // namespace
}  // namespace gvx

struct gvx_batch {
  std::vector<gvx_dvm*> maps;
  gvx::BatchMap* d_table = nullptr;
  gvx::BatchItems items{};
  long long* d_prefix = nullptr;  // 3 x (n_maps + 1)
  uint32_t* d_stacks = nullptr;   // fused Y -> X: one stack per resident warp
  unsigned* d_sync = nullptr;     // slice counters of all maps, queue head, error word
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int edt_rows = 0;  // sweep rows per staging chunk (0 = library default), set by the autotuner
};

using namespace gvx;

extern "C" {

gvx_status gvx_batch_create(gvx_dvm* const* maps, uint32_t n_maps, gvx_batch** out) {
  if (out == nullptr || maps == nullptr || n_maps == 0) return fail(GVX_ERR_INVALID_ARG, "need at least one map");
  *out = nullptr;
  std::vector<BatchMap> table(n_maps);
  uint32_t sync_words = 0, stack_len = 1, z_max = 1;
  for (uint32_t k = 0; k < n_maps; ++k) {
    if (maps[k] == nullptr) return fail(GVX_ERR_INVALID_ARG, "null map in batch");
    const gvx_dvm* m = maps[k];
    table[k] = BatchMap{m->d_vox,  m->d_scratch, (int)m->dims.x,     (int)m->dims.y,
                        (int)m->dims.z, m->side, num_voxels(m->dims), sync_words};
    sync_words += m->dims.z;
    stack_len = std::max(stack_len, std::max(m->dims.x, m->dims.y));
    z_max = std::max(z_max, m->dims.z);
  }
  const long long stack_warps = edt_batch_stack_warps();
  if (stack_warps <= 0) return fail(GVX_ERR_CUDA, "occupancy query for the batched EDT failed");
  gvx_batch* b = new (std::nothrow) gvx_batch();
  if (b == nullptr) return fail(GVX_ERR_OOM, "host allocation failed");
  b->maps.assign(maps, maps + n_maps);
  std::vector<long long> prefix(4 * (size_t)(n_maps + 1), 0);
  for (int p = 0; p < 4; ++p) {
    for (uint32_t k = 0; k < n_maps; ++k) {
      const gvx_dims& d = maps[k]->dims;
      const long long items = p < 3 ? edt_pass_items(d, p)  // occupancy tasks: z items x 32-row chunks
                                    : edt_pass_items(d, 0) * (long long)((d.z + 31) / 32);
      prefix[p * (n_maps + 1) + k + 1] = prefix[p * (n_maps + 1) + k] + items;
    }
    b->items.total[p] = prefix[p * (n_maps + 1) + n_maps];
  }
  b->items.n_maps = n_maps;
  cudaError_t e = cudaMalloc(&b->d_table, n_maps * sizeof(BatchMap));
  if (e == cudaSuccess) e = cudaMemcpy(b->d_table, table.data(), n_maps * sizeof(BatchMap), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMalloc(&b->d_prefix, prefix.size() * sizeof(long long));
  if (e == cudaSuccess) e = cudaMemcpy(b->d_prefix, prefix.data(), prefix.size() * sizeof(long long), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMalloc(&b->d_stacks, (size_t)stack_warps * stack_len * 64 * sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaMalloc(&b->d_sync, (sync_words + 2) * sizeof(unsigned));
  if (e == cudaSuccess) e = cudaMemset(b->d_sync, 0, (sync_words + 2) * sizeof(unsigned));
  if (e != cudaSuccess) {
    if (b->d_table) cudaFree(b->d_table);
    if (b->d_prefix) cudaFree(b->d_prefix);
    if (b->d_stacks) cudaFree(b->d_stacks);
    if (b->d_sync) cudaFree(b->d_sync);
    delete b;
    return cuda_status(e, "batch table");
  }
  for (int p = 0; p < 4; ++p) b->items.d_prefix[p] = b->d_prefix + p * (size_t)(n_maps + 1);
  b->items.d_stacks = b->d_stacks;
  b->items.stack_warps = stack_warps;
  b->items.stack_len = stack_len;
  b->items.d_sync = b->d_sync;
  b->items.sync_words = sync_words;
  b->items.z_max = z_max;
  *out = b;
  return GVX_OK;
}

gvx_status gvx_batch_destroy(gvx_batch* b) {
  if (b == nullptr) return GVX_OK;
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  if (b->d_table) cudaFree(b->d_table);
  if (b->d_prefix) cudaFree(b->d_prefix);
  if (b->d_stacks) cudaFree(b->d_stacks);
  if (b->d_sync) cudaFree(b->d_sync);
  delete b;
  return GVX_OK;
}

gvx_status gvx_batch_clear(gvx_batch* b, gvx_stream stream) {
  if (b == nullptr) return fail(GVX_ERR_INVALID_ARG, "batch is null");
  dim3 grid((unsigned)std::max(1, sms() * 4 / (int)std::min<size_t>(b->maps.size(), 64)), (unsigned)b->maps.size());
  batch_clear_kernel<<<grid, 256, 0, as_stream(stream)>>>(b->d_table);
  return cuda_status(cudaGetLastError(), "batch clear");
}

gvx_status gvx_batch_insert_points(gvx_batch* b, const float* d_xyz, const uint64_t* d_offsets, uint64_t n_total,
                                   gvx_stream stream) {
  if (b == nullptr || d_offsets == nullptr || (n_total > 0 && d_xyz == nullptr)) return fail(GVX_ERR_INVALID_ARG, "null argument");
  if (n_total == 0) return GVX_OK;
  const unsigned blocks = (unsigned)std::min<uint64_t>((n_total + 255) / 256, (uint64_t)sms() * 16);
  batch_insert_kernel<<<blocks, 256, 0, as_stream(stream)>>>(b->d_table, (uint32_t)b->maps.size(), d_xyz, d_offsets,
                                                             n_total);
  return cuda_status(cudaGetLastError(), "batch insert");
}

gvx_status gvx_batch_edt(gvx_batch* b, gvx_stream stream) {
  if (b == nullptr) return fail(GVX_ERR_INVALID_ARG, "batch is null");
  return cuda_status(launch_edt_batch(b->d_table, b->items, as_stream(stream), b->edt_rows), "batch EDT");
}

gvx_status gvx_batch_voxelize_edt(gvx_batch* b, const float* d_xyz, const uint64_t* d_offsets, uint64_t n_total,
                                  gvx_stream stream) {
  if (b == nullptr || d_offsets == nullptr || (n_total > 0 && d_xyz == nullptr)) return fail(GVX_ERR_INVALID_ARG, "null argument");
  return cuda_status(launch_voxelize_edt_batch(b->d_table, b->items, d_xyz, d_offsets, n_total, as_stream(stream), b->edt_rows),
                     "batch voxelize + EDT");
}

gvx_status gvx_batch_edt_check(gvx_batch* b, uint32_t* flags) {
  if (b == nullptr || flags == nullptr) return fail(GVX_ERR_INVALID_ARG, "null argument");
  cudaError_t e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaMemcpy(flags, b->d_sync + b->items.sync_words + 1, sizeof(uint32_t), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_status(e, "batch EDT check");
  if (*flags != 0) return fail(GVX_ERR_TIMEOUT, "batched EDT: a slice wait gave up (results invalid)");
  return GVX_OK;
}

gvx_status gvx_batch_autotune(gvx_batch* b, int force, gvx_edt_config* out, gvx_stream stream) {
  if (b == nullptr) return fail(GVX_ERR_INVALID_ARG, "batch is null");
  std::string key = tune_device_name() + "|batch|" + std::to_string(b->maps.size());
  uint64_t h = 1469598103934665603ull;  // FNV-1a over the dims of all maps
  for (const gvx_dvm* m : b->maps)
    for (uint32_t v : {m->dims.x, m->dims.y, m->dims.z}) h = (h ^ v) * 1099511628211ull;
  key += "|" + std::to_string(h);
  EdtConfig best;
  float best_ms = 0.f;
  if (force || !tune_lookup(key, &best, &best_ms)) {
    cudaStream_t s = as_stream(stream);
    uint64_t total = 0;
    for (const gvx_dvm* m : b->maps) total += num_voxels(m->dims);
    uint32_t* save = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaError_t e = cudaMalloc(&save, total * sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    auto copy_all = [&](bool to_save) {
      uint64_t off = 0;
      cudaError_t r = cudaSuccess;
      for (const gvx_dvm* m : b->maps) {
        const uint64_t n = num_voxels(m->dims);
        if (r == cudaSuccess)
          r = cudaMemcpyAsync(to_save ? save + off : m->d_vox, to_save ? m->d_vox : save + off, n * sizeof(uint32_t),
                              cudaMemcpyDeviceToDevice, s);
        off += n;
      }
      return r;
    };
    if (e == cudaSuccess) e = copy_all(true);
    best_ms = 1e30f;
    for (int rows : {16, 32}) {
      float t_min = 1e30f;
      for (int rep = 0; rep < 4 && e == cudaSuccess; ++rep) {  // first run warms up
        e = copy_all(false);
        if (e == cudaSuccess) e = cudaEventRecord(e0, s);
        if (e == cudaSuccess) e = launch_edt_batch(b->d_table, b->items, s, rows);
        if (e == cudaSuccess) e = cudaEventRecord(e1, s);
        if (e == cudaSuccess) e = cudaEventSynchronize(e1);
        float ms = 0.f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
        if (e == cudaSuccess && rep > 0) t_min = std::min(t_min, ms);
      }
      if (e == cudaSuccess && t_min < best_ms) {
        best_ms = t_min;
        best = EdtConfig{rows, 1};
      }
    }
    if (e == cudaSuccess) e = copy_all(false);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (save) cudaFree(save);
    if (e != cudaSuccess) return cuda_status(e, "batch autotune");
    uint32_t flag = 0;
    e = cudaMemcpy(&flag, b->d_sync + b->items.sync_words + 1, sizeof(uint32_t), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_status(e, "batch autotune");
    if (flag) return fail(GVX_ERR_TIMEOUT, "batch autotune: a bounded wait gave up");
    tune_store(key, best, best_ms);
  }
  b->edt_rows = best.rows;
  if (out) *out = gvx_edt_config{(uint32_t)best.rows, 1u, best_ms};
  return GVX_OK;
}

gvx_status gvx_batch_query_trilinear(gvx_batch* b, const float* d_xyz, const uint32_t* d_map, uint64_t n, float* d_dist,
                                     float* d_grad, gvx_stream stream) {
  if (b == nullptr || (n > 0 && (d_xyz == nullptr || d_map == nullptr || d_dist == nullptr)))
    return fail(GVX_ERR_INVALID_ARG, "null argument");
  if (n == 0) return GVX_OK;
  const QueryConfig q = query_config();
  const unsigned blocks = (unsigned)std::max<uint64_t>(
      1, std::min<uint64_t>((n + q.threads - 1) / q.threads, (uint64_t)sms() * q.blocks_per_sm));
  batch_trilinear_kernel<<<blocks, q.threads, 0, as_stream(stream)>>>(b->d_table, d_xyz, d_map, n, d_dist, d_grad);
  return cuda_status(cudaGetLastError(), "batch trilinear");
}

gvx_status gvx_batch_graph_capture(gvx_batch* b, const float* d_xyz, const uint64_t* d_offsets, uint64_t n_total,
                                   const float* d_qxyz, const uint32_t* d_qmap, uint64_t n_q, float* d_dist, float* d_grad,
                                   gvx_stream stream) {
  if (b == nullptr) return fail(GVX_ERR_INVALID_ARG, "batch is null");
  cudaStream_t s = nullptr;
  cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
  if (e != cudaSuccess) return cuda_status(e, "capture stream");
  // one plain run first: it sets every kernel attribute outside the capture
  gvx_status st = gvx_batch_voxelize_edt(b, d_xyz, d_offsets, n_total, s);
  if (st == GVX_OK) st = gvx_batch_query_trilinear(b, d_qxyz, d_qmap, n_q, d_dist, d_grad, s);
  if (st == GVX_OK) st = cuda_status(cudaStreamSynchronize(s), "batch warm-up");
  if (st != GVX_OK) {
    cudaStreamDestroy(s);
    return st;
  }
  if (b->exec) { cudaGraphExecDestroy(b->exec); b->exec = nullptr; }
  if (b->graph) { cudaGraphDestroy(b->graph); b->graph = nullptr; }
  e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    st = gvx_batch_voxelize_edt(b, d_xyz, d_offsets, n_total, s);
    if (st == GVX_OK) st = gvx_batch_query_trilinear(b, d_qxyz, d_qmap, n_q, d_dist, d_grad, s);
    cudaGraph_t g = nullptr;
    cudaError_t e2 = cudaStreamEndCapture(s, &g);
    if (st == GVX_OK && e2 == cudaSuccess) {
      b->graph = g;
      e2 = cudaGraphInstantiate(&b->exec, g, 0);
      if (e2 != cudaSuccess) st = cuda_status(e2, "graph instantiate");
    } else if (st == GVX_OK) {
      st = cuda_status(e2, "end capture");
    }
  } else {
    st = cuda_status(e, "begin capture");
  }
  cudaStreamDestroy(s);
  (void)stream;
  return st;
}

gvx_status gvx_batch_graph_launch(gvx_batch* b, gvx_stream stream) {
  if (b == nullptr || b->exec == nullptr) return fail(GVX_ERR_INVALID_ARG, "no captured graph");
  return cuda_status(cudaGraphLaunch(b->exec, as_stream(stream)), "graph launch");
}

}  // extern "C"
