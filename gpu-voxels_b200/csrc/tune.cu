// EDT autotuner: picks the sweep configuration (rows per staging chunk, fused
// or separate y/x launches) by timing every candidate on a copy of the map's
// current content.  Results are bit-identical for every candidate; only the
// speed differs.  Choices are cached per (device, dims) in memory and, when
// the environment variable GVX_TUNE_CACHE names a file, in that file (one
// line per entry: key rows fused ms), so later processes skip the timing.
// No counterpart in the reference, whose band counts are fixed by the caller.
#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>
#include <string>

#include "gvx_internal.cuh"

namespace gvx {
namespace {

std::mutex g_tune_mutex;
std::map<std::string, std::pair<EdtConfig, float>> g_tune_cache;
bool g_tune_file_loaded = false;

void load_file_locked() {
  if (g_tune_file_loaded) return;
  g_tune_file_loaded = true;
  const char* path = getenv("GVX_TUNE_CACHE");
  if (path == nullptr || *path == 0) return;
  std::ifstream f(path);
  std::string line;
  while (std::getline(f, line)) {
    std::istringstream is(line);
    std::string key;
    EdtConfig c;
    float ms = 0.f;
    if (is >> key >> c.rows >> c.fused >> ms && (c.rows == 16 || c.rows == 32) && (c.fused == 0 || c.fused == 1))
      g_tune_cache[key] = {c, ms};
  }
}

}  // namespace

std::string tune_device_name() {
  int dev = 0;
  cudaDeviceProp p{};
  if (cudaGetDevice(&dev) != cudaSuccess || cudaGetDeviceProperties(&p, dev) != cudaSuccess) return "unknown";
  std::string name = p.name;
  for (char& ch : name)
    if (ch == ' ' || ch == '|') ch = '_';
  return name + "_sm" + std::to_string(p.multiProcessorCount);
}

QueryConfig g_query;  // guarded by g_tune_mutex
std::map<std::string, std::pair<QueryConfig, float>> g_query_cache;

QueryConfig query_config() {
  std::lock_guard<std::mutex> lock(g_tune_mutex);
  return g_query;
}

void set_query_config(const QueryConfig& c) {
  std::lock_guard<std::mutex> lock(g_tune_mutex);
  g_query = c;
}

bool tune_lookup(const std::string& key, EdtConfig* cfg, float* ms) {
  std::lock_guard<std::mutex> lock(g_tune_mutex);
  load_file_locked();
  auto it = g_tune_cache.find(key);
  if (it == g_tune_cache.end()) return false;
  *cfg = it->second.first;
  *ms = it->second.second;
  return true;
}

void tune_store(const std::string& key, const EdtConfig& cfg, float ms) {
  std::lock_guard<std::mutex> lock(g_tune_mutex);
  load_file_locked();
  g_tune_cache[key] = {cfg, ms};
  const char* path = getenv("GVX_TUNE_CACHE");
  if (path == nullptr || *path == 0) return;
  std::ofstream f(path, std::ios::app);
  f << key << ' ' << cfg.rows << ' ' << cfg.fused << ' ' << ms << '\n';
}

}  // namespace gvx

using namespace gvx;

namespace {

gvx_status tune_fail(gvx_status st, const char* msg) {
  set_error(msg);
  return st;
}

std::string map_key(const gvx_dims& d) {
  return tune_device_name() + "|map|" + std::to_string(d.x) + "x" + std::to_string(d.y) + "x" + std::to_string(d.z);
}

}  // namespace

extern "C" {

gvx_status gvx_set_query_config(const gvx_query_config* cfg) {
  if (cfg == nullptr) return tune_fail(GVX_ERR_INVALID_ARG, "null argument");
  if (!(cfg->threads == 64 || cfg->threads == 128 || cfg->threads == 256 || cfg->threads == 512) ||
      cfg->blocks_per_sm < 1 || cfg->blocks_per_sm > 64)
    return tune_fail(GVX_ERR_INVALID_ARG, "threads must be 64, 128, 256 or 512 and blocks_per_sm in [1, 64]");
  set_query_config(QueryConfig{(int)cfg->threads, (int)cfg->blocks_per_sm});
  return GVX_OK;
}

gvx_status gvx_query_autotune(const gvx_dvm* m, const float* d_xyz, uint64_t n, float* d_dist, float* d_grad, int force,
                              gvx_query_config* out, gvx_stream stream) {
  if (m == nullptr || n == 0 || d_xyz == nullptr || d_dist == nullptr)
    return tune_fail(GVX_ERR_INVALID_ARG, "need a map, points and a distance buffer");
  const std::string key = tune_device_name() + "|query";
  float best_ms = 0.f;
  QueryConfig best;
  bool cached = false;
  {
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    auto it = g_query_cache.find(key);
    if (!force && it != g_query_cache.end()) {
      best = it->second.first;
      best_ms = it->second.second;
      cached = true;
    }
  }
  if (!cached) {
    cudaStream_t s = as_stream(stream);
    cudaEvent_t a, b;
    if (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess)
      return tune_fail(GVX_ERR_CUDA, "query autotune: event creation failed");
    const QueryConfig before = query_config();
    best_ms = -1.f;
    cudaError_t e = cudaSuccess;
    for (int threads : {64, 128, 256, 512}) {
      for (int cap : {8, 16, 32}) {
        set_query_config(QueryConfig{threads, cap});
        float total = 0.f;
        for (int rep = 0; rep < 4 && e == cudaSuccess; ++rep) {  // the first is a warm-up
          e = cudaEventRecord(a, s);
          if (e == cudaSuccess) e = launch_trilinear(m, d_xyz, n, d_dist, d_grad, s);
          if (e == cudaSuccess) e = cudaEventRecord(b, s);
          if (e == cudaSuccess) e = cudaEventSynchronize(b);
          float ms = 0.f;
          if (e == cudaSuccess) cudaEventElapsedTime(&ms, a, b);
          if (rep > 0) total += ms;
        }
        if (e != cudaSuccess) break;
        if (best_ms < 0.f || total / 3 < best_ms) {
          best_ms = total / 3;
          best = QueryConfig{threads, cap};
        }
      }
      if (e != cudaSuccess) break;
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (e != cudaSuccess) {
      set_query_config(before);
      return cuda_status(e, "query autotune");
    }
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    g_query_cache[key] = {best, best_ms};
  }
  set_query_config(best);
  if (out) *out = gvx_query_config{(uint32_t)best.threads, (uint32_t)best.blocks_per_sm, best_ms};
  return GVX_OK;
}

gvx_status gvx_dvm_set_edt_config(gvx_dvm* m, const gvx_edt_config* cfg) {
  if (m == nullptr || cfg == nullptr) return tune_fail(GVX_ERR_INVALID_ARG, "null argument");
  if (!(cfg->rows == 0 || cfg->rows == 16 || cfg->rows == 32) || cfg->fused > 1)
    return tune_fail(GVX_ERR_INVALID_ARG, "rows must be 0, 16 or 32 and fused 0 or 1");
  m->edt_rows = (int)cfg->rows;
  m->edt_fused = (int)cfg->fused;
  return GVX_OK;
}

gvx_status gvx_dvm_autotune(gvx_dvm* m, int force, gvx_edt_config* out, gvx_stream stream) {
  if (m == nullptr) return tune_fail(GVX_ERR_INVALID_ARG, "map is null");
  const std::string key = map_key(m->dims);
  EdtConfig best;
  float best_ms = 0.f;
  if (force || !tune_lookup(key, &best, &best_ms)) {
    cudaStream_t s = as_stream(stream);
    const uint64_t n = num_voxels(m->dims);
    uint32_t* tmp = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaError_t e = cudaMalloc(&tmp, n * sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    const EdtConfig cands[4] = {{16, 1}, {32, 1}, {16, 0}, {32, 0}};
    best_ms = 1e30f;
    for (int c = 0; c < 4 && e == cudaSuccess; ++c) {
      float t_min = 1e30f;
      for (int rep = 0; rep < 4 && e == cudaSuccess; ++rep) {  // first run warms up
        e = cudaMemcpyAsync(tmp, m->d_vox, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s);
        if (e == cudaSuccess) e = cudaEventRecord(e0, s);
        if (e == cudaSuccess) e = launch_edt(tmp, m->d_scratch, m->scratch_words, m->dims, s, cands[c]);
        if (e == cudaSuccess) e = cudaEventRecord(e1, s);
        if (e == cudaSuccess) e = cudaEventSynchronize(e1);
        float ms = 0.f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
        if (e == cudaSuccess && rep > 0) t_min = std::min(t_min, ms);
      }
      if (e == cudaSuccess && t_min < best_ms) {
        best_ms = t_min;
        best = cands[c];
      }
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (tmp) cudaFree(tmp);
    if (e != cudaSuccess) return cuda_status(e, "EDT autotune");
    uint32_t flag = 0;
    e = edt_read_error(m->d_scratch, m->dims, &flag);
    if (e != cudaSuccess) return cuda_status(e, "EDT autotune");
    if (flag) return tune_fail(GVX_ERR_TIMEOUT, "EDT autotune: a bounded wait gave up");
    tune_store(key, best, best_ms);
  }
  m->edt_rows = best.rows;
  m->edt_fused = best.fused;
  if (out) *out = gvx_edt_config{(uint32_t)best.rows, (uint32_t)best.fused, best_ms};
  return GVX_OK;
}

}  // extern "C"
