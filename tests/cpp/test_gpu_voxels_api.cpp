// The reference's own test scenarios, written against the gpu_voxels C++ API
// of this library (include/gpu_voxels/*.h) the way gpu-voxels' Boost tests
// are written (GV/test/testing_distance.cu, testing_voxelmap.cu,
// testing_voxellist.cu).  Prints one line per case; exit code = failures.
#include <cuda_runtime.h>
#include <limits.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <vector>

#include "../../include/gpu_voxels/GpuVoxels.h"
#include "../../include/gpu_voxels/helpers_highlevel/DistanceMapConverter.h"

using namespace gpu_voxels;

static int g_failures = 0;
#define CHECK(cond, name)                                            \
  do {                                                               \
    const bool _ok = static_cast<bool>(cond);                        \
    std::printf("%s %s\n", _ok ? "PASS" : "FAIL", name);             \
    if (!_ok) ++g_failures;                                          \
  } while (0)

// createBoxOfPoints (GV/helpers/GeometryGeneration.cpp:90-107), float accumulation.
static std::vector<Vector3f> box_of_points(Vector3f lo, Vector3f hi, float delta) {
  std::vector<Vector3f> out;
  for (float x = lo.x; x <= hi.x; x += delta)
    for (float y = lo.y; y <= hi.y; y += delta)
      for (float z = lo.z; z <= hi.z; z += delta) out.push_back(Vector3f(x, y, z));
  return out;
}

// createEquidistantPointsInBox (GV/helpers/GeometryGeneration.cpp:237-264).
static std::vector<Vector3f> equidistant(size_t max_points, Vector3ui dims, float s) {
  std::vector<Vector3f> out;
  for (uint32_t i = 0; i < (dims.x - 1) / 2; i++)
    for (uint32_t j = 0; j < (dims.y - 1) / 2; j++)
      for (uint32_t k = 0; k < (dims.z - 1) / 2; k++) {
        if (out.size() >= max_points) return out;
        out.push_back(Vector3f(i * 2 * s + s / 2.0, j * 2 * s + s / 2.0, k * 2 * s + s / 2.0));
      }
  return out;
}

static void distance_extraction() {
  // GV/test/testing_distance.cu:129-220
  const Vector3ui dims(64, 64, 64);
  voxelmap::DistanceVoxelMap map(dims, 1.f);
  std::vector<uint32_t> idx = {0, 10, 100, 1000, 10000};
  std::vector<Vector3f> obstacles;
  for (uint32_t id : idx)
    obstacles.push_back(Vector3f((float)(id % 64), (float)((id / 64) % 64), (float)(id / 4096)));
  map.clearMap();
  map.insertPointCloud(obstacles, eBVM_OCCUPIED);
  std::vector<DistanceVoxel> gathered(idx.size());
  {
    uint32_t* d_idx = nullptr;
    DistanceVoxel* d_out = nullptr;
    cudaMalloc(&d_idx, idx.size() * 4);
    cudaMalloc(&d_out, idx.size() * 4);
    cudaMemcpy(d_idx, idx.data(), idx.size() * 4, cudaMemcpyHostToDevice);
    // the thrust::device_ptr form, as the reference's test calls it
    map.gatherVoxelsByIndex(thrust::device_ptr<uint32_t>(d_idx), thrust::device_ptr<uint32_t>(d_idx + idx.size()),
                            thrust::device_ptr<DistanceVoxel>(d_out));
    cudaMemcpy(gathered.data(), d_out, idx.size() * 4, cudaMemcpyDeviceToHost);
    cudaFree(d_idx);
    cudaFree(d_out);
  }
  bool own = true;
  for (size_t i = 0; i < idx.size(); ++i)
    own &= gathered[i].getObstacle() == Vector3ui(idx[i] % 64, (idx[i] / 64) % 64, idx[i] / 4096);
  CHECK(own, "distance_extraction: gatherVoxelsByIndex returns own coordinates");
  std::vector<int32_t> sq, d, dn;
  map.getSquaredDistancesToHost(idx, sq);
  map.getDistancesToHost(idx, d);
  std::vector<uint32_t> nb(idx);
  for (auto& v : nb) ++v;
  map.parallelBanding3D(1, 1, 1);
  map.getDistancesToHost(nb, dn);
  bool zero = true, differ = true;
  for (size_t i = 0; i < idx.size(); ++i) {
    zero &= sq[i] == 0 && d[i] == 0;
    differ &= d[i] != dn[i];
  }
  CHECK(zero, "distance_extraction: zero distance at obstacles");
  CHECK(differ, "distance_extraction: neighbour distance differs");
  // device-pointer queries (raw and thrust::device_ptr) agree with the host form
  std::vector<int32_t> sq_host, sq_raw(nb.size()), sq_thrust(nb.size()), d_host, d_thrust(nb.size());
  map.getSquaredDistancesToHost(nb, sq_host);
  map.getDistancesToHost(nb, d_host);
  {
    uint32_t* d_idx = nullptr;
    int32_t* d_out = nullptr;
    cudaMalloc(&d_idx, nb.size() * 4);
    cudaMalloc(&d_out, nb.size() * 4);
    cudaMemcpy(d_idx, nb.data(), nb.size() * 4, cudaMemcpyHostToDevice);
    map.getSquaredDistances(d_idx, d_idx + nb.size(), d_out);
    cudaMemcpy(sq_raw.data(), d_out, nb.size() * 4, cudaMemcpyDeviceToHost);
    thrust::device_ptr<uint32_t> b(d_idx), e(d_idx + nb.size());
    thrust::device_ptr<int32_t> o(d_out);
    map.getSquaredDistances(b, e, o);
    cudaMemcpy(sq_thrust.data(), d_out, nb.size() * 4, cudaMemcpyDeviceToHost);
    map.getDistances(b, e, o);
    cudaMemcpy(d_thrust.data(), d_out, nb.size() * 4, cudaMemcpyDeviceToHost);
    cudaFree(d_idx);
    cudaFree(d_out);
  }
  CHECK(sq_raw == sq_host && sq_thrust == sq_host && d_thrust == d_host,
        "distance_extraction: device-pointer queries equal the host queries");
}

static void distance_correctness() {
  // GV/test/testing_distance.cu:39-127, PBA against brute force on the lattice
  const Vector3ui dims(128, 128, 131);
  voxelmap::DistanceVoxelMap map(dims, 1.f);
  std::vector<Vector3f> pts = equidistant(10000, dims, 1.f);
  map.insertPointCloud(pts, eBVM_OCCUPIED);
  map.parallelBanding3D();
  // brute force on a sample of voxels
  std::vector<uint32_t> idx;
  for (uint32_t i = 0; i < dims.x * dims.y * dims.z; i += 997) idx.push_back(i);
  std::vector<int32_t> sq;
  map.getSquaredDistancesToHost(idx, sq);
  double maxerr = 0;
  for (size_t k = 0; k < idx.size(); ++k) {
    const int x = idx[k] % dims.x, y = (idx[k] / dims.x) % dims.y, z = idx[k] / (dims.x * dims.y);
    int64_t best = INT64_MAX;
    for (const Vector3f& p : pts) {
      const int64_t dx = x - (int)p.x, dy = y - (int)p.y, dz = z - (int)p.z;
      best = std::min(best, dx * dx + dy * dy + dz * dz);
    }
    maxerr = std::max(maxerr, std::fabs(std::sqrt((double)best) - std::sqrt((double)sq[k])));
  }
  CHECK(maxerr < 0.01, "distance_correctness: PBA vs brute force maxerr < 0.01");
}

static void collisions() {
  // GV/test/testing_voxelmap.cu:96-168 with BitVectorVoxelMaps, default dims 89x123x74
  GpuVoxels::getInstance()->initialize(89, 123, 74, 1.f);
  GpuVoxelsSharedPtr gvl = GpuVoxels::getInstance();
  gvl->addMap(MT_BITVECTOR_VOXELMAP, "a");
  gvl->addMap(MT_BITVECTOR_VOXELMAP, "b");
  BitVectorVoxelMap* a = gvl->getMap("a")->as<BitVectorVoxelMap>();
  BitVectorVoxelMap* b = gvl->getMap("b")->as<BitVectorVoxelMap>();
  std::vector<Vector3f> pts = equidistant(10000, Vector3ui(89, 123, 74), 1.f);
  gvl->insertPointCloudIntoMap(pts, "a", eBVM_OCCUPIED);
  gvl->insertPointCloudIntoMap(pts, "b", eBVM_OCCUPIED);
  CHECK(a->collideWith(b, 0.1f) == 10000, "collision: all points collide");
  a->clearMap();
  b->clearMap();
  a->insertPointCloud(box_of_points(Vector3f(2.1f, 2.1f, 2.1f), Vector3f(4.1f, 4.1f, 4.1f), 0.5f), eBVM_OCCUPIED);
  b->insertPointCloud(box_of_points(Vector3f(3.1f, 3.1f, 3.1f), Vector3f(5.1f, 5.1f, 5.1f), 0.5f), eBVM_OCCUPIED);
  CHECK(a->collideWith(b, 0.1f) == 8, "collision_with_offset: 8 without offset");
  CHECK(a->collideWith(b, 0.1f, Vector3i(-1, 0, -1)) == 18, "collision_with_offset: 18 with negative offset");
  CHECK(b->collideWith(a, 0.1f, Vector3i(1, 0, 1)) == 18, "collision_with_offset: 18 with positive offset");

  BitVectorVoxelList list(Vector3ui(89, 123, 74), 1.f);
  list.insertPointCloud(box_of_points(Vector3f(1.1f, 1.1f, 1.1f), Vector3f(3.9f, 3.9f, 3.9f), 0.1f), BitVoxelMeaning(11));
  list.insertPointCloud(box_of_points(Vector3f(2.1f, 2.1f, 2.1f), Vector3f(4.9f, 4.9f, 4.9f), 0.1f), BitVoxelMeaning(12));
  CHECK(list.getDimensions().x == 46, "bitvoxellist: 46 unique voxels");
  BitVectorVoxelMap m(Vector3ui(89, 123, 74), 1.f);
  m.insertPointCloud(box_of_points(Vector3f(1.1f, 1.1f, 1.1f), Vector3f(3.9f, 3.9f, 3.9f), 0.1f), eBVM_OCCUPIED);
  m.insertPointCloud(box_of_points(Vector3f(2.1f, 2.1f, 2.1f), Vector3f(4.9f, 4.9f, 4.9f), 0.1f), eBVM_OCCUPIED);
  CHECK(list.collideWith(&m, 1.0f) == 46, "collide_bitvoxellist_with_bitvoxelmap: 46");
  CHECK(list.collideWith(&list, 1.0f) == 46, "bitvoxellist vs bitvoxellist: 46");
  BitVectorVoxelList one(Vector3ui(89, 123, 74), 1.f);
  std::vector<Vector3f> box = box_of_points(Vector3f(1.1f, 1.1f, 1.1f), Vector3f(3.9f, 3.9f, 3.9f), 0.1f);
  one.insertPointCloud(box, eBVM_OCCUPIED);
  BitVectorVoxelMap m2(Vector3ui(89, 123, 74), 1.f);
  m2.insertPointCloud(box, eBVM_OCCUPIED);
  const size_t want[] = {27, 27, 18, 18, 9, 9, 0, 0};
  bool shift_ok = true;
  int k = 0;
  for (float shift = 0.0f; shift < 4.0f; shift += 0.5f) shift_ok &= one.collideWith(&m2, 1.0f, Vector3i(shift, 0, 0)) == want[k++];
  CHECK(shift_ok, "collide_bitvoxellist_with_voxelmap_shifting: 27/18/9/0");
  BitVectorVoxelMap wrong(Vector3ui(10, 10, 10), 1.f);
  CHECK(one.collideWith(&wrong, 1.0f) == (size_t)SSIZE_MAX, "list vs map with other dims: SSIZE_MAX");
  gvl->delMap("a");
  gvl->delMap("b");
}

// The reference's ProbMap2DistMap example (EX/ProbMap2DistMap.cpp:60-95): two
// overlapping cubes inserted into a ProbVoxelMap with maximal occupied and
// free probability; voxels above 0.55 merged into a DistanceVoxelMap.
static void prob_map_to_distance_map() {
  GpuVoxelsSharedPtr gvl = GpuVoxels::getInstance();
  gvl->initialize(128, 128, 128, 1.0f);
  CHECK(gvl->addMap(MT_PROBAB_VOXELMAP, "myProbVoxelMap"), "addMap(MT_PROBAB_VOXELMAP)");
  gvl->addMap(MT_DISTANCE_VOXELMAP, "myDistanceMap");
  ProbVoxelMapSharedPtr prob(gvl->getMap("myProbVoxelMap"), gvl->getMap("myProbVoxelMap")->as<voxelmap::ProbVoxelMap>());
  DistanceVoxelMapSharedPtr dist(gvl->getMap("myDistanceMap"),
                                 gvl->getMap("myDistanceMap")->as<voxelmap::DistanceVoxelMap>());
  prob->insertPointCloud(box_of_points(Vector3f(40, 40, 40), Vector3f(60, 60, 60), 0.9f), eBVM_MAX_OCC_PROB);
  prob->insertPointCloud(box_of_points(Vector3f(50, 50, 50), Vector3f(70, 70, 70), 0.9f), eBVM_MAX_FREE_PROB);
  CHECK(dist->mergeOccupied(prob, Vector3ui(0, 0, 0), 0.55f), "mergeOccupied");
  std::vector<DistanceVoxel> host(dist->getVoxelMapSize());
  cudaMemcpy(host.data(), dist->getDeviceDataPtr(), host.size() * sizeof(DistanceVoxel), cudaMemcpyDeviceToHost);
  size_t sites = 0;
  for (const DistanceVoxel& v : host) sites += v.raw() != 0x3FFFFFFFu;
  CHECK(sites == 20 * 20 * 20 - 10 * 10 * 10, "mergeOccupied: box 1 minus the overlap (7000 sites)");
  dist->parallelBanding3D();
  // the voxel at (30,30,30) is nearest to the cube's corner (40,40,40): 3 * 10^2
  CHECK(dist->getSquaredObstacleDistance(30, 30, 30) == 300, "EDT after mergeOccupied: corner distance 300");
  const std::string file = "/tmp/gvx_test_dist_map.gvm";
  CHECK(dist->writeToDisk(file), "writeToDisk");
  voxelmap::DistanceVoxelMap loaded(Vector3ui(128, 128, 128), 1.0f);
  CHECK(loaded.readFromDisk(file) && loaded.getSquaredObstacleDistance(30, 30, 30) == 300, "readFromDisk round trip");
  voxelmap::DistanceVoxelMap other(Vector3ui(64, 64, 64), 1.0f);
  CHECK(!other.readFromDisk(file), "readFromDisk rejects other dims");
  std::remove(file.c_str());
  gvl->delMap("myProbVoxelMap");
  gvl->delMap("myDistanceMap");
}

// addMap returning the map (GV/GpuVoxels.cpp:164-302) and collideWith
// against a ProbVoxelMap (BitVoxelMap.hpp:205-210, BitVoxelList.hpp:63-69):
// the expected counts are recomputed on the host from the maps' contents
// with DefaultCollider's rule (occupancy >= floatToProbability(threshold)
// and a BitVoxel meaning other than eBVM_FREE).
static void prob_map_collisions() {
  GpuVoxelsSharedPtr gvl = GpuVoxels::getInstance();
  gvl->initialize(96, 80, 72, 1.0f);
  voxelmap::ProbVoxelMap* env = gvl->addMap(MT_PROBAB_VOXELMAP, "env")->as<voxelmap::ProbVoxelMap>();
  BitVectorVoxelMap* robot = gvl->addMap(MT_BITVECTOR_VOXELMAP, "robot")->as<BitVectorVoxelMap>();
  BitVectorVoxelList* robot_list = gvl->addMap(MT_BITVECTOR_VOXELLIST, "robot_list")->as<BitVectorVoxelList>();
  CHECK(env && robot && robot_list, "addMap(...)->as<T>() returns the new maps");
  CHECK(!gvl->addMap(MT_PROBAB_VOXELMAP, "env"), "addMap with a taken name: empty pointer");
  CHECK(!gvl->addMap(MT_BITVECTOR_OCTREE, "tree"), "addMap of a type outside the library: empty pointer");
  env->insertPointCloud(box_of_points(Vector3f(20, 20, 20), Vector3f(40, 40, 40), 0.9f), eBVM_MAX_OCC_PROB);
  env->insertPointCloud(box_of_points(Vector3f(30, 30, 30), Vector3f(50, 50, 50), 0.9f), eBVM_MAX_FREE_PROB);
  const std::vector<Vector3f> arm = box_of_points(Vector3f(25, 25, 25), Vector3f(45, 45, 45), 0.9f);
  robot->insertPointCloud(arm, BitVoxelMeaning(7));
  robot_list->insertPointCloud(arm, BitVoxelMeaning(7));
  const size_t n = robot->getVoxelMapSize();
  std::vector<int8_t> occ(n);
  cudaMemcpy(occ.data(), env->getDeviceDataPtr(), n, cudaMemcpyDeviceToHost);
  std::vector<uint8_t> bits(n * 32);
  cudaMemcpy(bits.data(), robot->getDeviceDataPtr(), n * 32, cudaMemcpyDeviceToHost);
  auto expect = [&](float thr, int dx) {
    float t = std::max(std::min(1.0f, thr), 0.0f);
    const int p = (int)(int8_t)(t * (127.0f - (-127.0f)) + (-127.0f));
    size_t c = 0;
    for (size_t i = 0; i < n; ++i) {
      const int64_t j = (int64_t)i + dx;
      if (j < 0 || j >= (int64_t)n || occ[i] < p) continue;
      const uint8_t* v = &bits[(size_t)j * 32];
      bool any = (v[0] & ~1u) != 0;
      for (int k = 1; k < 32; ++k) any = any || v[k] != 0;
      c += any;
    }
    return c;
  };
  // list entry at id meets map voxel id + dx
  auto expect_list = [&](float thr, int dx) {
    float t = std::max(std::min(1.0f, thr), 0.0f);
    const int p = (int)(int8_t)(t * (127.0f - (-127.0f)) + (-127.0f));
    size_t c = 0;
    for (size_t id = 0; id < n; ++id) {
      const uint8_t* v = &bits[id * 32];
      bool any = (v[0] & ~1u) != 0;
      for (int k = 1; k < 32; ++k) any = any || v[k] != 0;
      const int64_t j = (int64_t)id + dx;
      c += any && j >= 0 && j < (int64_t)n && occ[(size_t)j] >= p;
    }
    return c;
  };
  const size_t want = expect(0.55f, 0);
  CHECK(want > 0 && want == expect_list(0.55f, 0), "prob-map collision scene overlaps");
  CHECK(robot_list->collideWith(env, 0.55f) == want, "BitVoxelList::collideWith(ProbVoxelMap*)");
  CHECK(robot_list->collideWith(env, 0.55f, Vector3i(-2, 1, 0)) == expect_list(0.55f, -2 + 96),
        "BitVoxelList::collideWith(ProbVoxelMap*) with an offset");
  CHECK(robot->collideWith(env, 0.55f, Vector3i(3, 0, 0)) == expect(0.55f, 3), "BitVoxelMap::collideWith(ProbVoxelMap*) offset 3");
  CHECK(robot->collideWith(env, 2.0f) == expect(2.0f, 0), "BitVoxelMap::collideWith(ProbVoxelMap*) threshold clamped to 1");
  CHECK(robot->collideWith(env, 0.55f) == want, "BitVoxelMap::collideWith(ProbVoxelMap*)");
  voxelmap::ProbVoxelMap small(Vector3ui(8, 8, 8), 1.0f);
  CHECK(robot_list->collideWith(&small, 0.55f) == (size_t)SSIZE_MAX, "list vs ProbVoxelMap with other dims: SSIZE_MAX");
  gvl->delMap("env");
  gvl->delMap("robot");
  gvl->delMap("robot_list");
}

// Free-space bytes and the distance band -> BitVoxelList conversion
// (DistanceVoxelMap::extract_distances, distance_map_converter) on one site.
static void distance_consumers() {
  voxelmap::DistanceVoxelMap dist(Vector3ui(8, 8, 8), 1.0f);
  dist.insertPointCloud(std::vector<Vector3f>{Vector3f(3.5f, 3.5f, 3.5f)}, eBVM_OCCUPIED);
  dist.parallelBanding3D();
  free_space_t* d_bytes = nullptr;
  manhattan_dist_t* d_flood = nullptr;
  cudaMalloc(&d_bytes, 512);
  cudaMalloc(&d_flood, 512 * sizeof(manhattan_dist_t));
  dist.extract_distances(d_bytes, 0);
  std::vector<free_space_t> bytes(512);
  cudaMemcpy(bytes.data(), d_bytes, 512, cudaMemcpyDeviceToHost);
  CHECK(bytes[7 + 8 * 7 + 64 * 7] == 6 && bytes[3 + 8 * 3 + 64 * 3] == 0, "extract_distances: int(sqrt(48)) = 6, site 0");
  dist.init_floodfill(d_bytes, d_flood, 2);
  std::vector<manhattan_dist_t> flood(512);
  cudaMemcpy(flood.data(), d_flood, 512 * sizeof(manhattan_dist_t), cudaMemcpyDeviceToHost);
  bool flood_ok = true;
  for (int i = 0; i < 512; ++i)
    flood_ok &= flood[i] == (bytes[i] <= 2 ? MANHATTAN_DISTANCE_TOO_CLOSE : MANHATTAN_DISTANCE_UNINITIALIZED);
  CHECK(flood_ok, "init_floodfill");
  BitVectorVoxelList band(Vector3ui(8, 8, 8), 1.0f);
  CHECK(distance_map_converter::extract_given_distances(dist, 1, 1, band) == 26, "extract_given_distances(1,1): 26 voxels");
  cudaFree(d_bytes);
  cudaFree(d_flood);
}

// collideWithTypes: two swept volumes (meanings 10 and 20) against a map and a
// list holding meaning 10 in an overlapping box.
static void typed_collisions() {
  const Vector3ui dim(32, 32, 32);
  BitVectorVoxelMap sv(dim, 1.0f), obstacle(dim, 1.0f);
  sv.insertPointCloud(box_of_points(Vector3f(2.5f, 2.5f, 2.5f), Vector3f(5.5f, 5.5f, 5.5f), 1.0f), BitVoxelMeaning(10));
  sv.insertPointCloud(box_of_points(Vector3f(20.5f, 20.5f, 20.5f), Vector3f(22.5f, 22.5f, 22.5f), 1.0f),
                      BitVoxelMeaning(20));
  obstacle.insertPointCloud(box_of_points(Vector3f(4.5f, 4.5f, 4.5f), Vector3f(8.5f, 8.5f, 8.5f), 1.0f),
                            BitVoxelMeaning(10));
  BitVectorVoxel types;
  const size_t n = sv.collideWithTypes(&obstacle, types);
  CHECK(n == 8 && types.bitVector().getBit(10) && !types.bitVector().getBit(20), "collideWithTypes map: 8 voxels of type 10");
  BitVectorVoxelList list(dim, 1.0f);
  list.insertPointCloud(box_of_points(Vector3f(4.5f, 4.5f, 4.5f), Vector3f(6.5f, 6.5f, 6.5f), 1.0f), BitVoxelMeaning(30));
  BitVectorVoxel ltypes;
  const size_t ln = list.collideWithTypes(&obstacle, ltypes);
  CHECK(ln == 27 && ltypes.bitVector().getBit(30), "collideWithTypes list vs map: 27 entries of type 30");
  BitVectorVoxel mask;
  mask.bitVector().setBit(31);
  CHECK(list.collideWithTypeMask(&obstacle, mask) == 0, "collideWithTypeMask with a disjoint mask: 0");
}

// selfcollision_metapointcloud (GV/test/testing_voxelmap.cu), default fixture dims 89 x 123 x 74.
static void selfcollision_metapointcloud() {
  for (int j = 2; j < 11; j += 8) {
    BitVectorVoxelMap map(Vector3ui(89, 123, 74), 1.f, MT_BITVECTOR_VOXELMAP);
    const float d = 1.0f / j;
    std::vector<std::vector<Vector3f> > colliding = {
        box_of_points(Vector3f(2.1f, 2.1f, 2.1f), Vector3f(5.1f, 5.1f, 5.1f), d),
        box_of_points(Vector3f(4.1f, 4.1f, 4.1f), Vector3f(7.1f, 7.1f, 7.1f), d),
        box_of_points(Vector3f(6.1f, 6.1f, 6.1f), Vector3f(9.1f, 9.1f, 9.1f), d),
        box_of_points(Vector3f(10.1f, 10.1f, 10.1f), Vector3f(12.1f, 12.1f, 12.1f), d)};
    std::vector<std::vector<Vector3f> > separate = {
        box_of_points(Vector3f(30.1f, 30.1f, 30.1f), Vector3f(32.1f, 32.1f, 32.1f), d),
        box_of_points(Vector3f(40.1f, 40.1f, 40.1f), Vector3f(43.1f, 43.1f, 43.1f), d),
        box_of_points(Vector3f(60.1f, 60.1f, 60.1f), Vector3f(64.1f, 64.1f, 64.1f), d),
        box_of_points(Vector3f(65.1f, 65.1f, 65.1f), Vector3f(68.1f, 68.1f, 68.1f), d)};
    MetaPointCloud mc(colliding), ms(separate);
    CHECK(map.insertMetaPointCloudWithSelfCollisionCheck(&mc), "selfcollision: default masks, overlapping boxes");
    CHECK(!map.insertMetaPointCloudWithSelfCollisionCheck(&ms), "selfcollision: default masks, separate boxes");
    map.clearMap();
    std::vector<BitVoxelMeaning> meanings = {BitVoxelMeaning(51), BitVoxelMeaning(52), BitVoxelMeaning(53),
                                             BitVoxelMeaning(54)};
    BitVector<BIT_VECTOR_LENGTH> all;
    all = ~all;
    all.clearBit(eBVM_COLLISION);
    std::vector<BitVector<BIT_VECTOR_LENGTH> > masks(4, all);
    masks[0].clearBit(52);
    masks[1].clearBit(51);
    for (int k = 0; k < 4; ++k) masks[k].clearBit(51 + k);
    BitVector<BIT_VECTOR_LENGTH> hit;
    bool self = map.insertMetaPointCloudWithSelfCollisionCheck(&mc, meanings, masks, &hit);
    const bool bits_ok = !hit.getBit(51) && hit.getBit(52) && hit.getBit(53) && !hit.getBit(54);
    hit.clearBit(52);
    hit.clearBit(53);
    CHECK(self && bits_ok && hit.isZero(), "selfcollision: masks, meanings 52 and 53 only");
    for (int k = 0; k < 4; ++k) {
      masks[k] = all;
      masks[k].clearBit(51 + k);
    }
    hit.clear();
    self = map.insertMetaPointCloudWithSelfCollisionCheck(&ms, meanings, masks, &hit);
    CHECK(!self && hit.isZero(), "selfcollision: masks, separate boxes");
  }
}

// The reference's other EDT entry points give parallelBanding3D's squared distances.
static void other_edt_entry_points() {
  const Vector3ui dims(40, 36, 30);
  std::vector<Vector3f> pts = equidistant(60, dims, 1.f);
  voxelmap::DistanceVoxelMap a(dims, 1.f), b(dims, 1.f), c(dims, 1.f);
  a.insertPointCloud(pts, eBVM_OCCUPIED);
  a.parallelBanding3D();
  b.insertPointCloud(pts, eBVM_OCCUPIED);
  b.jumpFlood3D();
  c.insertPointCloud(std::vector<Vector3f>(1, Vector3f(1.5f, 1.5f, 1.5f)), eBVM_OCCUPIED);  // replaced below
  c.exactDistances3D(pts);
  bool same = true;
  for (uint32_t z = 0; z < dims.z; z += 3)
    for (uint32_t y = 0; y < dims.y; y += 5)
      for (uint32_t x = 0; x < dims.x; x += 7) {
        const int32_t d = a.getSquaredObstacleDistance(x, y, z);
        same = same && b.getSquaredObstacleDistance(x, y, z) == d && c.getSquaredObstacleDistance(x, y, z) == d;
      }
  CHECK(same, "jumpFlood3D / exactDistances3D: parallelBanding3D's squared distances");
  voxelmap::DistanceVoxelMap e(dims, 1.f);
  e.insertPointCloud(std::vector<Vector3f>(1, Vector3f(3.5f, 3.5f, 3.5f)), eBVM_OCCUPIED);  // replaced below
  e.voxelizeAndTransform(pts);
  std::vector<uint32_t> all(a.getVoxelMapSize());
  for (uint32_t i = 0; i < all.size(); ++i) all[i] = i;
  std::vector<int32_t> da, de;
  a.getSquaredDistancesToHost(all, da);
  e.getSquaredDistancesToHost(all, de);
  CHECK(da == de, "voxelizeAndTransform: clearMap + insertPointCloud + parallelBanding3D");
  a.fill_pba_uninit();
  CHECK(a.getSquaredObstacleDistance(3, 3, 3) == INT32_MAX, "fill_pba_uninit: no sites left");
}

// clone (TemplateVoxelMap.hpp:1101-1120) of each map type; a map of other dims is left alone;
// visualizeMap has no viewer to hand to.
static void clone_maps() {
  const Vector3ui dims(30, 26, 22);
  std::vector<Vector3f> pts = equidistant(40, dims, 1.f);
  voxelmap::DistanceVoxelMap a(dims, 1.f), b(dims, 1.f), other(Vector3ui(30, 26, 21), 1.f);
  a.insertPointCloud(pts, eBVM_OCCUPIED);
  a.parallelBanding3D();
  b.clone(a);
  other.clone(a);  // message, no change
  std::vector<uint32_t> all(a.getVoxelMapSize());
  for (uint32_t i = 0; i < all.size(); ++i) all[i] = i;
  std::vector<int32_t> da, db;
  a.getSquaredDistancesToHost(all, da);
  b.getSquaredDistancesToHost(all, db);
  CHECK(da == db, "clone: DistanceVoxelMap copy has the same distances");
  CHECK(other.getSquaredObstacleDistance(0, 0, 0) == INT32_MAX, "clone: other dims refused, map unchanged");
  BitVectorVoxelMap ba(dims, 1.f, MT_BITVECTOR_VOXELMAP), bb(dims, 1.f, MT_BITVECTOR_VOXELMAP),
      bs(dims, 0.5f, MT_BITVECTOR_VOXELMAP);
  ba.insertPointCloud(pts, eBVM_OCCUPIED);
  bb.clone(ba);
  bs.clone(ba);  // other side length: refused
  CHECK(bb.collideWith(&ba) == pts.size() && bs.collideWith(&ba) == 0, "clone: BitVectorVoxelMap");
  voxelmap::ProbVoxelMap pa(dims, 1.f), pb(dims, 1.f);
  pa.insertPointCloud(pts, eBVM_OCCUPIED);
  pb.clone(pa);
  std::vector<int8_t> ha(pa.getVoxelMapSize()), hb(pb.getVoxelMapSize());
  cudaMemcpy(ha.data(), pa.getDeviceDataPtr(), ha.size(), cudaMemcpyDeviceToHost);
  cudaMemcpy(hb.data(), pb.getDeviceDataPtr(), hb.size(), cudaMemcpyDeviceToHost);
  CHECK(ha == hb, "clone: ProbVoxelMap");
  GpuVoxelsSharedPtr gvl = GpuVoxels::getInstance();
  CHECK(!gvl->visualizeMap("no such map"), "visualizeMap: unknown map -> false");
}

// insertCoordinateList / copyCoordsToHost round trip; out-of-map coordinates are dropped.
static void list_coordinates() {
  BitVectorVoxelList list(Vector3ui(50, 40, 30), 0.01f, MT_BITVECTOR_VOXELLIST);
  std::vector<Vector3ui> coords = {Vector3ui(49, 39, 29), Vector3ui(0, 0, 0), Vector3ui(7, 8, 9), Vector3ui(7, 8, 9),
                                   Vector3ui(50, 1, 1)};
  list.insertCoordinateList(coords, BitVoxelMeaning(20));
  std::vector<Vector3ui> back;
  list.copyCoordsToHost(back);
  CHECK(back.size() == 3 && back[0] == Vector3ui(0, 0, 0) && back[1] == Vector3ui(7, 8, 9) &&
            back[2] == Vector3ui(49, 39, 29),
        "insertCoordinateList / copyCoordsToHost: 3 unique in-map voxels in id order");
}

int main() {
  GpuVoxels::getInstance();
  list_coordinates();
  clone_maps();
  other_edt_entry_points();
  selfcollision_metapointcloud();
  distance_consumers();
  typed_collisions();
  distance_extraction();
  distance_correctness();
  collisions();
  prob_map_to_distance_map();
  prob_map_collisions();
  std::printf("%d failure(s)\n", g_failures);
  return g_failures;
}
