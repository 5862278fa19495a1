/*
 * gvx_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C, single-file CPU restatement of gpu-voxels' distance-field
 * collision path.  It is the checker for the CUDA product: only the test
 * suite, the smoke entry and the benchmark's CPU-baseline leg load it.  The
 * product library never links or calls it.
 *
 * Every routine cites the reference function it restates (paths are within
 * the gpu-voxels project; GV = packages/gpu_voxels/src/gpu_voxels/).
 *
 * Parity pin: the restatement is checked against (1) the known answers of the
 * reference's own Boost tests (GV/test/testing_distance.cu,
 * GV/test/testing_voxelmap.cu, GV/test/testing_voxellist.cu) and (2) golden
 * maps produced by the reference's own PBA kernels compiled for sm_100a
 * (oracle/ref_pba_driver.cu, tests/golden/).
 *
 * Floating point: the only FP32 arithmetic on the integer path is the PBA
 * bisector test and the voxelisation divide.  Both are written with the same
 * operation order as the reference; build with -ffp-contract=off and without
 * -ffast-math (SSE float arithmetic is IEEE round-to-nearest).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define UNINIT 1023u          /* PBA_UNINITIALISED_COORD, GV/helpers/common_defines.h:113,123 */
#define DV_UNINIT 0x3FFFFFFFu /* DistanceVoxel with all three coordinates uninitialised */
#define MAX_OBSTACLE_DISTANCE 2147483647 /* GV/helpers/common_defines.h:131 */
#define BITVOXEL_BYTES 32     /* BitVoxel<256>, GV/helpers/common_defines.h:47 */
#define EBVM_COLLISION 2      /* GV/helpers/common_defines.h:55 */

typedef struct { uint32_t x, y, z; } u3;

/* DistanceVoxel decode: GV/voxel/DistanceVoxel.hpp:31-37 (z keeps the top 12 bits) */
static inline u3 dv_dec(uint32_t v) { u3 r = {v & 0x3ffu, (v >> 10) & 0x3ffu, v >> 20}; return r; }
/* DistanceVoxel encode: GV/voxel/DistanceVoxel.hpp:61-65 (no masking, uint32 wrap) */
static inline uint32_t dv_enc(uint32_t x, uint32_t y, uint32_t z) { return x | (y << 10) | (z << 20); }

int orc_version(void) { return 3; }

int orc_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/* ------------------------------------------------------------------------ */
/* Voxelisation                                                              */
/* ------------------------------------------------------------------------ */

/* mapToVoxels(float, Vector3f), GV/voxelmap/kernels/VoxelMapOperations.h:121-131:
 * static_cast<uint32_t>(floor(c / s)).  On the device the float->u32 convert
 * saturates (negative and NaN -> 0, >= 2^32 -> UINT32_MAX); the host cast is
 * undefined, so the saturation is spelled out. */
uint32_t orc_coord_to_voxel(float c, float s) {
  float q = c / s;
  float f = floorf(q);
  if (!(f > 0.0f)) return 0u; /* NaN, -0, negatives */
  if (f >= 4294967296.0f) return 0xFFFFFFFFu;
  return (uint32_t)f;
}

/* clearMap for DistanceVoxel, GV/voxelmap/TemplateVoxelMap.hpp:244-271 */
void orc_dvm_clear(uint32_t *map, uint64_t n) {
  for (uint64_t i = 0; i < n; ++i) map[i] = DV_UNINIT;
}

/* kernelInsertGlobalPointCloud<DistanceVoxel>, GV/voxelmap/kernels/VoxelMapOperations.hpp:266-300,
 * with DistanceVoxel::insert(pos, eBVM_OCCUPIED), GV/voxel/DistanceVoxel.hpp:125-138.
 * Returns 1 when any point fell outside the map (the points_outside_map flag). */
int orc_dvm_insert(uint32_t *map, const uint32_t dims[3], float side, const float *xyz, uint64_t n) {
  int outside = 0;
  for (uint64_t i = 0; i < n; ++i) {
    uint32_t x = orc_coord_to_voxel(xyz[3 * i + 0], side);
    uint32_t y = orc_coord_to_voxel(xyz[3 * i + 1], side);
    uint32_t z = orc_coord_to_voxel(xyz[3 * i + 2], side);
    if (x < dims[0] && y < dims[1] && z < dims[2]) {
      uint32_t id = z * dims[0] * dims[1] + y * dims[0] + x; /* getVoxelIndexUnsigned, VoxelMapOperations.h:44-49 */
      map[id] = dv_enc(x, y, z);
    } else {
      outside = 1;
    }
  }
  return outside;
}

/* ------------------------------------------------------------------------ */
/* PBA, band counts m1 = m2 = m3 = 1                                         */
/* ------------------------------------------------------------------------ */

/* devicePBAintersection3DY, GV/voxelmap/kernels/VoxelMapOperationsPBA.hpp:265-276.
 * Same operation order; every product and sum is exact for coordinates
 * below 1024, only the divide and the final add round. */
static inline float pba_isect(int x1, int y1, int z1, int x2, int y2, int z2, int x0, int z0) {
  float xM = (x1 + x2) / 2.0f;
  float yM = (y1 + y2) / 2.0f;
  float zM = (z1 + z2) / 2.0f;
  float nx = (float)(x2 - x1);
  float ny = (float)(y2 - y1);
  float nz = (float)(z2 - z1);
  return yM + (nx * (xM - (float)x0) + nz * (zM - (float)z0)) / ny;
}

float orc_pba_isect(int x1, int y1, int z1, int x2, int y2, int z2, int x0, int z0) {
  return pba_isect(x1, y1, z1, x2, y2, z2, x0, z0);
}

/* kernelPBAphase1FloodZ with m1 = 1, GV/voxelmap/kernels/VoxelMapOperationsPBA.hpp:63-124.
 * One (x,y) column; `col` is the column with element stride `st`, in place
 * (the reference passes the same buffer as input and output, DistanceVoxelMap.hpp:396-398). */
static void pba_phase1_column(uint32_t *col, uint64_t st, int Z) {
  uint32_t obstacle = DV_UNINIT;
  for (int i = 0; i < Z; ++i) { /* flood forward */
    uint32_t cur = col[(uint64_t)i * st];
    if ((cur >> 20) != UNINIT) obstacle = cur;
    col[(uint64_t)i * st] = obstacle;
  }
  obstacle = DV_UNINIT; /* flood backward; ties keep the lower z (<=, :118) */
  const int tz_top = Z - 1;
  for (int i = 0; i < Z; ++i) {
    uint64_t id = (uint64_t)(tz_top - i) * st;
    int dist_prev = abs((int)(obstacle >> 20) - (tz_top - i));
    uint32_t next = col[id];
    int dist_next = abs((tz_top - i) - (int)(next >> 20));
    if (dist_next <= dist_prev) obstacle = next;
    col[id] = obstacle;
  }
}

/*
 * One PBA column sweep (phase 2 + phase 3 with m2 = m3 = 1) in the
 * reference's own (possibly transposed) frame.
 *   kernelPBAphase2ProximateBackpointers, VoxelMapOperationsPBA.hpp:289-379
 *   kernelPBAphase3Distances,             VoxelMapOperationsPBA.hpp:604-703
 * `in`/`out` are the column (stride `st`), `stk` a positional scratch column
 * of length Y (the reference's initial_map slice), tx/tz the column position.
 * Sites use the stored x and z fields; their y is the row index.
 */
static void pba_phase23_column(const uint32_t *in, uint32_t *out, uint64_t st, uint32_t *stk, int Y, int tx, int tz) {
  /* phase 2 */
  int last_y = (int)UNINIT;
  u3 top = {UNINIT, UNINIT, UNINIT}, second = {UNINIT, UNINIT, UNINIT};
  u3 cur = {UNINIT, UNINIT, UNINIT};
  for (int ty = 0; ty < Y; ++ty) {
    cur = dv_dec(in[(uint64_t)ty * st]);
    if (cur.x != UNINIT) {
      while (top.y != UNINIT) {
        float i1 = pba_isect((int)second.x, (int)top.y, (int)second.z, (int)top.x, last_y, (int)top.z, tx, tz);
        float i2 = pba_isect((int)top.x, last_y, (int)top.z, (int)cur.x, ty, (int)cur.z, tx, tz);
        if (i1 < i2) break;
        last_y = (int)top.y;
        top = second;
        if (top.y != UNINIT) second = dv_dec(stk[top.y]);
      }
      second = top;
      top.x = cur.x; top.y = (uint32_t)last_y; top.z = cur.z;
      last_y = ty;
      stk[ty] = dv_enc(top.x, top.y, top.z);
    }
  }
  if (cur.x == UNINIT) stk[Y - 1] = dv_enc(UNINIT, (uint32_t)last_y, UNINIT); /* tail pointer */

  /* phase 3 */
  float inter = 0.0f;
  last_y = Y - 1;
  top = dv_dec(stk[last_y]);
  if (top.x == UNINIT) {
    last_y = (int)top.y;
    if (last_y != (int)UNINIT) top = dv_dec(stk[last_y]);
  }
  if (top.y != UNINIT) {
    second = dv_dec(stk[top.y]);
    inter = pba_isect((int)second.x, (int)top.y, (int)second.z, (int)top.x, last_y, (int)top.z, tx, tz);
  }
  for (int ty = Y - 1; ty >= 0; --ty) {
    while (top.y != UNINIT) {
      if ((float)ty > inter) break;
      last_y = (int)top.y;
      top = second;
      if (top.y != UNINIT) {
        second = dv_dec(stk[top.y]);
        inter = pba_isect((int)second.x, (int)top.y, (int)second.z, (int)top.x, last_y, (int)top.z, tx, tz);
      }
    }
    out[(uint64_t)ty * st] = dv_enc(top.x, (uint32_t)last_y, top.z);
  }
}

/* kernelPBA3DTransposeXY, VoxelMapOperationsPBA.hpp:825-888 (square XY only):
 * voxel (x,y,z) <- voxel (y,x,z) with the site's x and y swapped. */
static void pba_transpose_xy(uint32_t *map, int N, int Z) {
  const uint64_t layer = (uint64_t)N * N;
#pragma omp parallel for schedule(static)
  for (int z = 0; z < Z; ++z) {
    uint32_t *L = map + (uint64_t)z * layer;
    for (int y = 0; y < N; ++y) {
      for (int x = y; x < N; ++x) {
        u3 a = dv_dec(L[(uint64_t)y * N + x]);
        u3 b = dv_dec(L[(uint64_t)x * N + y]);
        L[(uint64_t)x * N + y] = dv_enc(a.y, a.x, a.z);
        L[(uint64_t)y * N + x] = dv_enc(b.y, b.x, b.z);
      }
    }
  }
}

/* Phase 1 over the whole map (all (x,y) columns). */
static void pba_phase1(uint32_t *map, const uint32_t d[3]) {
  const uint64_t layer = (uint64_t)d[0] * d[1];
#pragma omp parallel for schedule(static)
  for (int64_t c = 0; c < (int64_t)layer; ++c) pba_phase1_column(map + c, layer, (int)d[2]);
}

/*
 * Literal restatement of DistanceVoxelMap::parallelBanding3D(1,1,1),
 * GV/voxelmap/DistanceVoxelMap.hpp:284-645, launch order :396-626:
 *   phase 1; initial_map = copy; phase 2 + 3 along y; transpose XY;
 *   phase 2 + 3 along y; transpose XY.
 * Requires dims x == y (the reference's own domain).  Returns -1 otherwise.
 */
int orc_pba_reference_order(uint32_t *map, const uint32_t d[3]) {
  if (d[0] != d[1]) return -1;
  const int N = (int)d[0], Z = (int)d[2];
  const uint64_t layer = (uint64_t)N * N, n = layer * (uint64_t)Z;
  uint32_t *stk = (uint32_t *)malloc(n * sizeof(uint32_t));
  if (!stk) return -2;
  memcpy(stk, map, n * sizeof(uint32_t)); /* initial_map copy, :342 (before phase 1) */
  pba_phase1(map, d);
  for (int pass = 0; pass < 2; ++pass) {
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < (int64_t)N * Z; ++c) {
      int tx = (int)(c % N), tz = (int)(c / N);
      uint64_t base = (uint64_t)tz * layer + (uint64_t)tx;
      /* stk holds the column at the same positions as the map (positional stack) */
      uint32_t *scol = (uint32_t *)malloc((size_t)N * sizeof(uint32_t));
      for (int y = 0; y < N; ++y) scol[y] = stk[base + (uint64_t)y * N];
      pba_phase23_column(map + base, map + base, (uint64_t)N, scol, N, tx, tz);
      for (int y = 0; y < N; ++y) stk[base + (uint64_t)y * N] = scol[y];
      free(scol);
    }
    pba_transpose_xy(map, N, Z);
  }
  free(stk);
  return 0;
}

/*
 * The same algorithm for any dims (x != y allowed): the second sweep runs
 * along x in the original frame instead of transposing.  Reading the
 * transposed frame back: a site's stored y field plays the role of "x", the
 * column's y position plays the role of tx, and the output packs
 * (row, y-field, z-field).  For x == y it reproduces orc_pba_reference_order
 * bit for bit (checked by the tests).
 */
static void pba_sweep_x_row(uint32_t *row, uint32_t *stk, uint32_t *tmp_in, int X, int y0, int z0) {
  /* Express the row in the transposed frame, run the column sweep, map back. */
  for (int x = 0; x < X; ++x) {
    u3 v = dv_dec(row[x]);
    tmp_in[x] = dv_enc(v.y, v.x, v.z);
  }
  pba_phase23_column(tmp_in, tmp_in, 1, stk, X, y0, z0);
  for (int x = 0; x < X; ++x) {
    u3 v = dv_dec(tmp_in[x]);
    row[x] = dv_enc(v.y, v.x, v.z);
  }
}

int orc_pba(uint32_t *map, const uint32_t d[3]) {
  const int X = (int)d[0], Y = (int)d[1], Z = (int)d[2];
  if (X < 1 || Y < 1 || Z < 1 || X > 1023 || Y > 1023 || Z > 1023) return -1;
  const uint64_t layer = (uint64_t)X * Y;
  pba_phase1(map, d);
  /* sweep along y for every (x, z) */
#pragma omp parallel
  {
    uint32_t *stk = (uint32_t *)malloc((size_t)Y * sizeof(uint32_t));
#pragma omp for schedule(static)
    for (int64_t c = 0; c < (int64_t)X * Z; ++c) {
      int tx = (int)(c % X), tz = (int)(c / X);
      uint32_t *col = map + (uint64_t)tz * layer + (uint64_t)tx;
      pba_phase23_column(col, col, (uint64_t)X, stk, Y, tx, tz);
    }
    free(stk);
  }
  /* sweep along x for every (y, z) */
#pragma omp parallel
  {
    uint32_t *stk = (uint32_t *)malloc((size_t)X * sizeof(uint32_t));
    uint32_t *tmp = (uint32_t *)malloc((size_t)X * sizeof(uint32_t));
#pragma omp for schedule(static)
    for (int64_t r = 0; r < (int64_t)Y * Z; ++r) {
      int ty = (int)(r % Y), tz = (int)(r / Y);
      pba_sweep_x_row(map + (uint64_t)tz * layer + (uint64_t)ty * X, stk, tmp, X, ty, tz);
    }
    free(stk);
    free(tmp);
  }
  return 0;
}

/* Phase 1 alone (exposed for per-pass tests). */
void orc_pba_phase1(uint32_t *map, const uint32_t d[3]) { pba_phase1(map, d); }

/* ------------------------------------------------------------------------ */
/* Distance queries                                                          */
/* ------------------------------------------------------------------------ */

/* DistanceVoxel::squaredObstacleDistance, GV/voxel/DistanceVoxel.hpp:40-55 */
static inline int32_t dv_sqdist(uint32_t v, int px, int py, int pz) {
  u3 o = dv_dec(v);
  if (px == (int)UNINIT || py == (int)UNINIT || pz == (int)UNINIT || o.x == UNINIT || o.y == UNINIT || o.z == UNINIT)
    return MAX_OBSTACLE_DISTANCE;
  int dx = px - (int)o.x, dy = py - (int)o.y, dz = pz - (int)o.z;
  return dx * dx + dy * dy + dz * dz;
}

/* getSquaredDistances / SquaredDistanceFunctor, GV/voxelmap/DistanceVoxelMap.hpp:709-752:
 * gather the voxel at each linear id, decode the id (mapToVoxels(uint, dims),
 * VoxelMapOperations.h:159-167), return the squared distance. */
void orc_sqdist(const uint32_t *map, const uint32_t d[3], const uint32_t *ids, uint64_t n, int32_t *out) {
  const uint32_t layer = d[0] * d[1];
  for (uint64_t i = 0; i < n; ++i) {
    uint32_t id = ids[i];
    uint32_t z = id / layer, rem = id - z * layer, y = rem / d[0], x = rem - y * d[0];
    out[i] = dv_sqdist(map[id], (int)x, (int)y, (int)z);
  }
}

/* getDistances / DistanceFunctor, DistanceVoxelMap.hpp:754-797:
 * sqrtf of the squared distance, stored in int32 (truncation). */
void orc_dist(const uint32_t *map, const uint32_t d[3], const uint32_t *ids, uint64_t n, int32_t *out) {
  orc_sqdist(map, d, ids, n, out);
  for (uint64_t i = 0; i < n; ++i) out[i] = (int32_t)sqrtf((float)out[i]);
}

/* Squared distance of every voxel to its stored site (whole map). */
void orc_sqdist_map(const uint32_t *map, const uint32_t d[3], int32_t *out) {
  const uint64_t layer = (uint64_t)d[0] * d[1];
#pragma omp parallel for schedule(static)
  for (int64_t z = 0; z < (int64_t)d[2]; ++z)
    for (uint32_t y = 0; y < d[1]; ++y)
      for (uint32_t x = 0; x < d[0]; ++x) {
        uint64_t id = (uint64_t)z * layer + (uint64_t)y * d[0] + x;
        out[id] = dv_sqdist(map[id], (int)x, (int)y, (int)z);
      }
}

/* Exhaustive exact squared EDT against the obstacle voxels of an inserted
 * map: the role of kernelExactDistances3D, VoxelMapOperations.hpp:896-990.
 * Output is the squared distance (INT_MAX when the map has no obstacle). */
void orc_brute_sqdist(const uint32_t *inserted, const uint32_t d[3], int32_t *out) {
  const uint64_t layer = (uint64_t)d[0] * d[1], n = layer * d[2];
  uint64_t k = 0;
  for (uint64_t i = 0; i < n; ++i) k += (inserted[i] != DV_UNINIT);
  int32_t *site = (int32_t *)malloc((k ? k : 1) * 3 * sizeof(int32_t));
  k = 0;
  for (uint64_t i = 0; i < n; ++i)
    if (inserted[i] != DV_UNINIT) {
      u3 o = dv_dec(inserted[i]);
      site[3 * k] = (int32_t)o.x; site[3 * k + 1] = (int32_t)o.y; site[3 * k + 2] = (int32_t)o.z; ++k;
    }
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t i = 0; i < (int64_t)n; ++i) {
    int z = (int)(i / layer), rem = (int)(i % layer), y = rem / (int)d[0], x = rem % (int)d[0];
    int64_t best = MAX_OBSTACLE_DISTANCE;
    for (uint64_t j = 0; j < k; ++j) {
      int64_t dx = x - site[3 * j], dy = y - site[3 * j + 1], dz = z - site[3 * j + 2];
      int64_t s = dx * dx + dy * dy + dz * dz;
      if (s < best) best = s;
    }
    out[i] = (int32_t)best;
  }
  free(site);
}

/* ------------------------------------------------------------------------ */
/* BitVoxel maps and lists                                                  */
/* ------------------------------------------------------------------------ */

/* BitVector<256>::noneButEmpty, GV/helpers/BitVector.h:184-198 */
static inline int bv_none_but_empty(const uint8_t *b) {
  if (b[0] & 0xFE) return 0;
  for (int i = 1; i < BITVOXEL_BYTES; ++i)
    if (b[i]) return 0;
  return 1;
}

/* kernelInsertGlobalPointCloud<BitVoxel>, VoxelMapOperations.hpp:241-264;
 * BitVoxel::insert -> BitVector::setBit, GV/helpers/BitVector.h:224-228. */
int orc_bvm_insert(uint8_t *map, const uint32_t d[3], float side, const float *xyz, uint64_t n, uint32_t meaning) {
  int outside = 0;
  for (uint64_t i = 0; i < n; ++i) {
    uint32_t x = orc_coord_to_voxel(xyz[3 * i + 0], side);
    uint32_t y = orc_coord_to_voxel(xyz[3 * i + 1], side);
    uint32_t z = orc_coord_to_voxel(xyz[3 * i + 2], side);
    if (x < d[0] && y < d[1] && z < d[2]) {
      uint64_t id = (uint64_t)z * d[0] * d[1] + (uint64_t)y * d[0] + x;
      map[id * BITVOXEL_BYTES + (meaning >> 3)] |= (uint8_t)(1u << (meaning & 7));
    } else {
      outside = 1;
    }
  }
  return outside;
}

/* kernelClearVoxelMap(BitVoxel*, size, BitVector bits), GV/voxelmap/kernels/VoxelMapOperations.hpp:57-71:
 * a voxel holding any of `bits` keeps only its other bits. */
void orc_bvm_clear_bits(uint8_t *map, uint64_t n, const uint8_t *bits) {
  for (uint64_t i = 0; i < n; ++i) {
    uint8_t *v = map + i * BITVOXEL_BYTES;
    int any = 0;
    for (int b = 0; b < BITVOXEL_BYTES; ++b) any |= v[b] & bits[b];
    if (any)
      for (int b = 0; b < BITVOXEL_BYTES; ++b) v[b] &= (uint8_t)~bits[b];
  }
}

/* performLeftShift, GV/helpers/BitVector.h:355-402, on every voxel
 * (kernelShiftBitVector, VoxelMapOperations.hpp:813-820): a 64-bit buffer
 * holds eight input bytes; each output byte is the buffer shifted right by
 * `shift`, the buffer then moves on by one byte and takes in the byte eight
 * further on; output byte 0 keeps only its upper four bits. */
void orc_bvm_shift(uint8_t *map, uint64_t n, uint32_t shift) {
  for (uint64_t i = 0; i < n; ++i) {
    uint8_t *v = map + i * BITVOXEL_BYTES;
    uint64_t buffer = 0;
    for (uint32_t b = 0; b < 8; ++b) buffer += (uint64_t)v[b] << (b * 8);
    for (uint32_t b = 0; b < BITVOXEL_BYTES; ++b) {
      uint8_t out = (uint8_t)(buffer >> shift);
      if (b == 0) out &= 0xF0;
      v[b] = out;
      buffer >>= 8;
      if (b + 8 < BITVOXEL_BYTES) buffer += (uint64_t)v[b + 8] << 56;
    }
  }
}

/*
 * BitVoxelMap::insertMetaPointCloudWithSelfCollisionCheck, GV/voxelmap/BitVoxelMap.hpp:227-341,
 * with kernelInsertMetaPointCloudSelfCollCheck, GV/voxelmap/kernels/VoxelMapOperations.hpp:581-631,
 * run one sub-cloud after the other (the reference synchronises after each)
 * and, inside a sub-cloud, one point after the other: masked = voxel & mask;
 * if masked has a bit but bit 0, colliding |= masked, colliding gets the
 * sub-cloud's meaning and the voxel eBVM_COLLISION; then the voxel gets the
 * meaning.  (With masks that keep the sub-cloud's own meaning or
 * eBVM_COLLISION the reference's result depends on its threads' timing; the
 * reference's defaults clear both.)  Returns the outside flag.
 */
int orc_bvm_insert_meta_self_coll(uint8_t *map, const uint32_t d[3], float side, const float *xyz,
                                  const uint64_t *offsets, uint32_t n_clouds, const uint8_t *meanings,
                                  const uint8_t *masks, uint8_t *colliding) {
  int outside = 0;
  memset(colliding, 0, BITVOXEL_BYTES);
  for (uint32_t k = 0; k < n_clouds; ++k) {
    const uint8_t *mask = masks + (size_t)k * BITVOXEL_BYTES;
    const uint32_t meaning = meanings[k];
    for (uint64_t i = offsets[k]; i < offsets[k + 1]; ++i) {
      uint32_t x = orc_coord_to_voxel(xyz[3 * i + 0], side);
      uint32_t y = orc_coord_to_voxel(xyz[3 * i + 1], side);
      uint32_t z = orc_coord_to_voxel(xyz[3 * i + 2], side);
      if (!(x < d[0] && y < d[1] && z < d[2])) {
        outside = 1;
        continue;
      }
      uint8_t *v = map + ((uint64_t)z * d[0] * d[1] + (uint64_t)y * d[0] + x) * BITVOXEL_BYTES;
      uint8_t masked[BITVOXEL_BYTES];
      for (int b = 0; b < BITVOXEL_BYTES; ++b) masked[b] = v[b] & mask[b];
      if (!bv_none_but_empty(masked)) {
        for (int b = 0; b < BITVOXEL_BYTES; ++b) colliding[b] |= masked[b];
        colliding[meaning >> 3] |= (uint8_t)(1u << (meaning & 7));
        v[EBVM_COLLISION >> 3] |= (uint8_t)(1u << (EBVM_COLLISION & 7));
      }
      v[meaning >> 3] |= (uint8_t)(1u << (meaning & 7));
    }
  }
  return outside;
}

/*
 * BitVoxelMap::collideWith(BitVectorVoxelMap*), GV/voxelmap/BitVoxelMap.hpp:198-203
 *  -> collisionCheckWithCounterRelativeTransform, GV/voxelmap/TemplateVoxelMap.hpp:588-621
 *  -> kernelCollideVoxelMapsDebug, GV/voxelmap/kernels/VoxelMapOperations.hpp:129-184
 *  with DefaultCollider::collide(BitVoxel, BitVoxel), GV/voxel/DefaultCollider.hpp:76-81.
 * Voxel i of `other` is tested against voxel i + offset_linear of `self`
 * (the reference shifts this map's base pointer by the linear offset,
 * getVoxelPtrSignedOffset, VoxelMapOperations.h:84-97); pairs whose shifted
 * index leaves the map are skipped.  Colliding voxels of `self` get
 * eBVM_COLLISION when `mark` is set.
 */
uint64_t orc_bvm_collide(uint8_t *self, const uint8_t *other, uint64_t n, int64_t offset_linear, int mark) {
  uint64_t count = 0;
  for (uint64_t i = 0; i < n; ++i) {
    int64_t j = (int64_t)i + offset_linear;
    if (j < 0 || j >= (int64_t)n) continue;
    uint8_t *a = self + (uint64_t)j * BITVOXEL_BYTES;
    const uint8_t *b = other + i * BITVOXEL_BYTES;
    if (!bv_none_but_empty(a) && !bv_none_but_empty(b)) {
      ++count;
      if (mark) a[EBVM_COLLISION >> 3] |= (uint8_t)(1u << (EBVM_COLLISION & 7));
    }
  }
  return count;
}

/* Parallel count for the CPU baseline (no marking). */
uint64_t orc_bvm_collide_count_omp(const uint8_t *self, const uint8_t *other, uint64_t n) {
  uint64_t count = 0;
#pragma omp parallel for reduction(+ : count) schedule(static)
  for (int64_t i = 0; i < (int64_t)n; ++i) {
    const uint64_t *a = (const uint64_t *)(self + (uint64_t)i * BITVOXEL_BYTES);
    const uint64_t *b = (const uint64_t *)(other + (uint64_t)i * BITVOXEL_BYTES);
    uint64_t ma = (a[0] & ~(uint64_t)1) | a[1] | a[2] | a[3];
    uint64_t mb = (b[0] & ~(uint64_t)1) | b[1] | b[2] | b[3];
    count += (ma != 0) & (mb != 0);
  }
  return count;
}

/*
 * BitVoxelList::collideWith(BitVectorVoxelMap*), GV/voxellist/BitVoxelList.hpp:71-77
 *  -> TemplateVoxelList::collisionCheckWithCollider, GV/voxellist/TemplateVoxelList.hpp:1170-1213
 *  -> kernelCollideWithVoxelMap, GV/voxellist/kernels/VoxelListOperations.hpp:146-197.
 * For list entry i, the map voxel at ids[i] + offset_linear is tested when it
 * lies inside the map; colliding list voxels get eBVM_COLLISION when `mark`.
 */
uint64_t orc_list_collide_map(const uint32_t *ids, uint8_t *list_voxels, uint64_t n, const uint8_t *map, uint64_t map_n,
                              int64_t offset_linear, int mark) {
  uint64_t count = 0;
  for (uint64_t i = 0; i < n; ++i) {
    int64_t j = (int64_t)ids[i] + offset_linear;
    if (j < 0 || j >= (int64_t)map_n) continue;
    uint8_t *a = list_voxels + i * BITVOXEL_BYTES;
    if (!bv_none_but_empty(a) && !bv_none_but_empty(map + (uint64_t)j * BITVOXEL_BYTES)) {
      ++count;
      if (mark) a[EBVM_COLLISION >> 3] |= (uint8_t)(1u << (EBVM_COLLISION & 7));
    }
  }
  return count;
}

/* Parallel count over many lists (CPU baseline of the batched form). */
void orc_lists_collide_map_omp(const uint32_t *ids, const uint8_t *list_voxels, const uint64_t *offsets, uint64_t nlists,
                               const uint8_t *map, uint64_t map_n, uint64_t *counts) {
#pragma omp parallel for schedule(dynamic, 1)
  for (int64_t l = 0; l < (int64_t)nlists; ++l) {
    uint64_t c = 0;
    for (uint64_t i = offsets[l]; i < offsets[l + 1]; ++i) {
      uint64_t j = ids[i];
      if (j >= map_n) continue;
      const uint64_t *a = (const uint64_t *)(list_voxels + i * BITVOXEL_BYTES);
      const uint64_t *b = (const uint64_t *)(map + j * BITVOXEL_BYTES);
      uint64_t ma = (a[0] & ~(uint64_t)1) | a[1] | a[2] | a[3];
      uint64_t mb = (b[0] & ~(uint64_t)1) | b[1] | b[2] | b[3];
      c += (ma != 0) & (mb != 0);
    }
    counts[l] = c;
  }
}

/* BitVoxelMap::collideWith(const ProbVoxelMap*), GV/voxelmap/BitVoxelMap.hpp:205-210
 * -> collisionCheckWithCounterRelativeTransform (TemplateVoxelMap.hpp:588-621)
 * -> kernelCollideVoxelMapsDebug (VoxelMapOperations.hpp:129-184) with
 * DefaultCollider::collide(BitVoxel v1, ProbabilisticVoxel v2)
 * (GV/voxel/DefaultCollider.hpp:68-73): v2.occupancy >= thr && !v1.noneButEmpty;
 * v1 = self[i + offset], v2 = other[i]; thr = floatToProbability(coll_threshold). */
uint64_t orc_bvm_collide_pvm(uint8_t *self, const int8_t *other, uint64_t n, int64_t offset_linear, int thr, int mark) {
  uint64_t count = 0;
  for (uint64_t i = 0; i < n; ++i) {
    int64_t j = (int64_t)i + offset_linear;
    if (j < 0 || j >= (int64_t)n) continue;
    uint8_t *a = self + (uint64_t)j * BITVOXEL_BYTES;
    if ((int)other[i] >= thr && !bv_none_but_empty(a)) {
      ++count;
      if (mark) a[EBVM_COLLISION >> 3] |= (uint8_t)(1u << (EBVM_COLLISION & 7));
    }
  }
  return count;
}

/* BitVoxelList::collideWith(const ProbVoxelMap*), GV/voxellist/BitVoxelList.hpp:63-69
 * -> collisionCheckWithCollider (TemplateVoxelList.hpp:1170-1213) ->
 * kernelCollideWithVoxelMap (VoxelListOperations.hpp:146-197), same collider:
 * entry i meets map voxel ids[i] + offset when that lies in the map. */
uint64_t orc_list_collide_pvm(const uint32_t *ids, uint8_t *list_voxels, uint64_t n, const int8_t *map, uint64_t map_n,
                              int64_t offset_linear, int thr, int mark) {
  uint64_t count = 0;
  for (uint64_t i = 0; i < n; ++i) {
    int64_t j = (int64_t)ids[i] + offset_linear;
    if (j < 0 || j >= (int64_t)map_n) continue;
    uint8_t *a = list_voxels + i * BITVOXEL_BYTES;
    if ((int)map[j] >= thr && !bv_none_but_empty(a)) {
      ++count;
      if (mark) a[EBVM_COLLISION >> 3] |= (uint8_t)(1u << (EBVM_COLLISION & 7));
    }
  }
  return count;
}

/* BitVoxelList::collideWith(BitVectorVoxelList*) -> collideVoxellists,
 * GV/voxellist/TemplateVoxelList.hpp:231-289: number of this list's ids
 * present in the other (sorted) list, thrust::binary_search semantics. */
uint64_t orc_list_collide_list(const uint32_t *ids_a, uint64_t na, const uint32_t *ids_b, uint64_t nb) {
  uint64_t count = 0;
  for (uint64_t i = 0; i < na; ++i) {
    uint64_t lo = 0, hi = nb;
    while (lo < hi) {
      uint64_t mid = lo + (hi - lo) / 2;
      if (ids_b[mid] < ids_a[i]) lo = mid + 1; else hi = mid;
    }
    count += (lo < nb && ids_b[lo] == ids_a[i]);
  }
  return count;
}

/*
 * TemplateVoxelList::insertPointCloud, GV/voxellist/TemplateVoxelList.hpp:363-393:
 * voxelise each point (kernelInsertGlobalPointCloud for lists,
 * VoxelListOperations.hpp:43-61), drop out-of-bounds entries
 * (remove_out_of_bounds, :318-341), sort by id and OR-merge duplicates
 * (make_unique, :143-212).  `ids_io`/`voxels_io` hold `*n_io` existing sorted
 * entries and room for `*n_io + npts`; on return `*n_io` is the new length.
 */
static int cmp_u64(const void *a, const void *b) {
  uint64_t x = *(const uint64_t *)a, y = *(const uint64_t *)b;
  return (x > y) - (x < y);
}

void orc_list_insert(uint32_t *ids_io, uint8_t *voxels_io, uint64_t *n_io, const uint32_t d[3], float side, const float *xyz,
                     uint64_t npts, uint32_t meaning) {
  uint64_t n0 = *n_io, m = n0;
  uint64_t *keys = (uint64_t *)malloc((n0 + npts + 1) * sizeof(uint64_t)); /* (id << 32) | source index */
  uint8_t *vox = (uint8_t *)malloc((n0 + npts + 1) * BITVOXEL_BYTES);
  for (uint64_t i = 0; i < n0; ++i) {
    keys[i] = ((uint64_t)ids_io[i] << 32) | i;
    memcpy(vox + i * BITVOXEL_BYTES, voxels_io + i * BITVOXEL_BYTES, BITVOXEL_BYTES);
  }
  for (uint64_t i = 0; i < npts; ++i) {
    uint32_t x = orc_coord_to_voxel(xyz[3 * i], side), y = orc_coord_to_voxel(xyz[3 * i + 1], side),
             z = orc_coord_to_voxel(xyz[3 * i + 2], side);
    if (x >= d[0] || y >= d[1] || z >= d[2]) continue;
    uint32_t id = z * d[0] * d[1] + y * d[0] + x;
    keys[m] = ((uint64_t)id << 32) | m;
    memset(vox + m * BITVOXEL_BYTES, 0, BITVOXEL_BYTES);
    vox[m * BITVOXEL_BYTES + (meaning >> 3)] |= (uint8_t)(1u << (meaning & 7));
    ++m;
  }
  qsort(keys, m, sizeof(uint64_t), cmp_u64);
  uint64_t out = 0;
  for (uint64_t i = 0; i < m;) {
    uint32_t id = (uint32_t)(keys[i] >> 32);
    uint8_t acc[BITVOXEL_BYTES];
    memset(acc, 0, sizeof(acc));
    while (i < m && (uint32_t)(keys[i] >> 32) == id) {
      const uint8_t *src = vox + (keys[i] & 0xFFFFFFFFu) * BITVOXEL_BYTES;
      for (int b = 0; b < BITVOXEL_BYTES; ++b) acc[b] |= src[b];
      ++i;
    }
    ids_io[out] = id;
    memcpy(voxels_io + out * BITVOXEL_BYTES, acc, BITVOXEL_BYTES);
    ++out;
  }
  *n_io = out;
  free(keys);
  free(vox);
}

/* ------------------------------------------------------------------------ */
/* ProbVoxelMap and DistanceVoxelMap::mergeOccupied                          */
/* ------------------------------------------------------------------------ */

/* ProbabilisticVoxel::insert -> updateOccupancy, GV/voxel/ProbabilisticVoxel.hpp:44-100,
 * constants GV/helpers/common_defines.h:154-161 (UNKNOWN -128, MIN -127,
 * MAX 127, sensor model free -10 / occupied 72) and the meaning ranges
 * GV/helpers/common_defines.h:50-63. */
static int8_t prob_update(int8_t cur, uint32_t meaning) {
  int delta;
  switch (meaning) {
    case 0: delta = -10; break;          /* eBVM_FREE */
    case 1: case 2: delta = 72; break;   /* eBVM_OCCUPIED, eBVM_COLLISION */
    case 3: case 255: return -128;       /* eBVM_UNKNOWN, eBVM_UNDEFINED */
    default:
      if (meaning >= 4 && meaning <= 254) { delta = (int)meaning - 129; break; }
      return -128;
  }
  if (cur == -128) return (int8_t)delta;
  int v = (int)cur + delta;
  if (v < -127) v = -127;
  if (v > 127) v = 127;
  return (int8_t)v;
}

/* kernelInsertGlobalPointCloud<ProbabilisticVoxel>, GV/voxelmap/kernels/VoxelMapOperations.hpp:241-264:
 * every point applies its update to its voxel, one after the other (the
 * reference's device update is not atomic and can lose updates when points
 * share a voxel; all updates of one call are the same monotone saturating
 * step, so applying each of them gives one order-independent result). */
int orc_pvm_insert(int8_t *map, const uint32_t d[3], float side, const float *xyz, uint64_t n, uint32_t meaning) {
  int outside = 0;
  for (uint64_t i = 0; i < n; ++i) {
    uint32_t x = orc_coord_to_voxel(xyz[3 * i + 0], side);
    uint32_t y = orc_coord_to_voxel(xyz[3 * i + 1], side);
    uint32_t z = orc_coord_to_voxel(xyz[3 * i + 2], side);
    if (x < d[0] && y < d[1] && z < d[2]) {
      uint64_t id = (uint64_t)z * d[0] * d[1] + (uint64_t)y * d[0] + x;
      map[id] = prob_update(map[id], meaning);
    } else {
      outside = 1;
    }
  }
  return outside;
}

/* ProbabilisticVoxel::floatToProbability, GV/voxel/ProbabilisticVoxel.h:40-45 */
int orc_float_to_probability(float val) {
  float tmp = val < 1.0f ? val : 1.0f;
  tmp = tmp > 0.0f ? tmp : 0.0f;
  tmp = (tmp * (127.0f - (-127.0f))) + (-127.0f);
  return (int)(int8_t)tmp;
}

/* DistanceVoxelMap::mergeOccupied, GV/voxelmap/DistanceVoxelMap.hpp:109-136 with
 * mergeOccupiedOperator / probVoxelOccupied, GV/voxelmap/DistanceVoxelMap.h:92-134:
 * voxel i whose occupancy exceeds the threshold gets the site of its own
 * coordinates plus the offset, packed with 32-bit wrap-around. */
void orc_dvm_merge_occupied(uint32_t *dvm, const int8_t *pvm, const uint32_t d[3], const uint32_t off[3], float thr) {
  const int t = orc_float_to_probability(thr);
  const uint64_t n = (uint64_t)d[0] * d[1] * d[2];
  for (uint64_t i = 0; i < n; ++i) {
    if ((int)pvm[i] <= t) continue;
    uint32_t x = (uint32_t)(i % d[0]), y = (uint32_t)((i / d[0]) % d[1]), z = (uint32_t)(i / ((uint64_t)d[0] * d[1]));
    dvm[i] = (x + off[0]) | ((y + off[1]) << 10) | ((z + off[2]) << 20);
  }
}

/* ------------------------------------------------------------------------ */
/* Distance-map consumers                                                    */
/* ------------------------------------------------------------------------ */

/* DistanceVoxel::extract_byte_distance, GV/voxel/DistanceVoxel.h:144-199, as
 * applied by DistanceVoxelMap::extract_distances (GV/voxelmap/DistanceVoxelMap.hpp:676-688):
 * voxels within robot_radius of the map border get their border distance;
 * the rest int(sqrtf(squared distance)) capped at SCHAR_MAX; int8 result. */
static int8_t free_space_byte(uint32_t v, int x, int y, int z, int X, int Y, int Z, int r) {
  if (x > X - r) return (int8_t)(X - x < 0 ? 0 : X - x);
  if (y > Y - r) return (int8_t)(Y - y < 0 ? 0 : Y - y);
  if (z > Z - r) return (int8_t)(Z - z < 0 ? 0 : Z - z);
  if (x < r) return (int8_t)(x < 0 ? 0 : x);
  if (y < r) return (int8_t)(y < 0 ? 0 : y);
  if (z < r) return (int8_t)(z < 0 ? 0 : z);
  int fs = (int)sqrtf((float)dv_sqdist(v, x, y, z));
  return (int8_t)(fs > 127 ? 127 : fs);
}

void orc_extract_distances(const uint32_t *map, const uint32_t d[3], int r, int8_t *out) {
  const uint64_t layer = (uint64_t)d[0] * d[1], n = layer * d[2];
  for (uint64_t i = 0; i < n; ++i) {
    int z = (int)(i / layer), y = (int)((i % layer) / d[0]), x = (int)(i % d[0]);
    out[i] = free_space_byte(map[i], x, y, z, (int)d[0], (int)d[1], (int)d[2], r);
  }
}

/* DistanceVoxel::init_floodfill_distance, GV/voxel/DistanceVoxel.h:201-215
 * (MANHATTAN_DISTANCE_* constants, GV/helpers/common_defines.h:117-119). */
void orc_init_floodfill(const int8_t *in, int16_t *out, uint64_t n, int r) {
  for (uint64_t i = 0; i < n; ++i) out[i] = (int16_t)((int)in[i] <= r ? 32765 : 32767);
}

/* distance_map_converter::extract_given_distances,
 * GV/helpers_highlevel/DistanceMapConverter.cu:156-196 with transform_to_bitvoxel (:103-154):
 * free-space bytes at robot radius 0; voxels with min <= byte <= max, in id
 * order, become list entries whose voxel has eBVM_OCCUPIED and the
 * swept-volume bits 4 .. 4 + byte - 1 set (UNDEFINED and a cap above 255).
 * Returns the count; ids / voxels (32 B each) may be NULL to count only. */
uint64_t orc_extract_given_distances(const uint32_t *map, const uint32_t d[3], int mn, int mx, uint32_t *ids,
                                     uint8_t *vox) {
  const uint64_t layer = (uint64_t)d[0] * d[1], n = layer * d[2];
  uint64_t k = 0;
  for (uint64_t i = 0; i < n; ++i) {
    int z = (int)(i / layer), y = (int)((i % layer) / d[0]), x = (int)(i % d[0]);
    int8_t b = free_space_byte(map[i], x, y, z, (int)d[0], (int)d[1], (int)d[2], 0);
    if (b < mn || b > mx) continue;
    if (ids) ids[k] = (uint32_t)i;
    if (vox) {
      uint8_t *v = vox + k * BITVOXEL_BYTES;
      memset(v, 0, BITVOXEL_BYTES);
      v[0] |= 1u << 1; /* eBVM_OCCUPIED */
      unsigned fs = (uint16_t)(int)b + 4u;
      if (fs > 255u) { v[31] |= 0x80u; fs = 255u; }
      for (unsigned s = 4; s < fs; ++s) v[s >> 3] |= (uint8_t)(1u << (s & 7));
    }
    ++k;
  }
  return k;
}

/* ------------------------------------------------------------------------ */
/* Typed collisions                                                          */
/* ------------------------------------------------------------------------ */

/* BitVoxelMap::collideWithTypes(BitVectorVoxelMap*) (GV/voxelmap/BitVoxelMap.hpp:212-217)
 * -> collisionCheckBitvector (:91-143) -> kernelCollideVoxelMapsBitvector
 * (GV/voxelmap/kernels/VoxelMapOperations.hpp:187-239) with SVCollider
 * (GV/voxel/SVCollider.hpp:90-96) and bitMarginCollisionCheck at window 0
 * and bit offset 0 (GV/helpers/BitVector.h:415-470): the colliding types of
 * voxel i are self[i] & other[i] restricted to the swept-volume bits (bits
 * 0..3 of `other` masked out); a voxel with any collides, is counted, marks
 * self with eBVM_COLLISION and adds its types to `types` (32 bytes, OR). */
uint64_t orc_bvm_collide_types(uint8_t *self, const uint8_t *other, uint64_t n, uint8_t *types) {
  uint64_t count = 0;
  for (uint64_t i = 0; i < n; ++i) {
    uint8_t *a = self + i * BITVOXEL_BYTES;
    const uint8_t *b = other + i * BITVOXEL_BYTES;
    uint8_t t[BITVOXEL_BYTES];
    int any = 0;
    for (int k = 0; k < BITVOXEL_BYTES; ++k) {
      t[k] = (uint8_t)(a[k] & (k == 0 ? (b[k] & 0xF0) : b[k]));
      any |= t[k];
    }
    if (!any) continue;
    ++count;
    for (int k = 0; k < BITVOXEL_BYTES; ++k) types[k] |= t[k];
    a[EBVM_COLLISION >> 3] |= (uint8_t)(1u << (EBVM_COLLISION & 7));
  }
  return count;
}

/* SVCollider::floatToProbability (GV/voxel/SVCollider.hpp:144-148): no clamping. */
static int sv_threshold(float val) { return (int)(int8_t)((val * (127.0f - (-127.0f))) + (-127.0f)); }

/* BitVoxelMap::collideWithTypes(ProbVoxelMap*) (BitVoxelMap.hpp:219-224) with
 * SVCollider::collide(BitVoxel, ProbabilisticVoxel, ...) (SVCollider.hpp:98-108):
 * occupancy >= threshold and self not empty -> all of self's bits are types. */
uint64_t orc_bvm_collide_types_pvm(uint8_t *self, const int8_t *other, uint64_t n, float thr, uint8_t *types) {
  const int t = sv_threshold(thr);
  uint64_t count = 0;
  for (uint64_t i = 0; i < n; ++i) {
    uint8_t *a = self + i * BITVOXEL_BYTES;
    if (!((int)other[i] >= t && !bv_none_but_empty(a))) continue;
    ++count;
    for (int k = 0; k < BITVOXEL_BYTES; ++k) types[k] |= a[k];
    a[EBVM_COLLISION >> 3] |= (uint8_t)(1u << (EBVM_COLLISION & 7));
  }
  return count;
}

/* BitVoxelList::collideWithTypes(BitVectorVoxelMap*) / (ProbVoxelMap*) and
 * collideWithTypeMask (GV/voxellist/BitVoxelList.hpp:120-246) ->
 * kernelCollideWithVoxelMap / kernelCollideWithVoxelMapBitMask
 * (GV/voxellist/kernels/VoxelListOperations.hpp:204-260,282-325): entry i meets
 * map voxel ids[i] + offset (skipped outside the map); it collides when that
 * voxel is occupied -- BitVoxel: not noneButEmpty; ProbabilisticVoxel:
 * occupancy >= threshold as a float -- and, with a mask, when its own bits
 * meet the mask.  Colliding entries are counted, add their bits (before the
 * mark) to `types` and get eBVM_COLLISION.  map_kind 0: BitVoxel map, 1: int8. */
uint64_t orc_list_collide_types_map(const uint32_t *ids, uint8_t *list_voxels, uint64_t n, const void *map,
                                    uint64_t map_n, int map_kind, float thr, int64_t offset_linear, const uint8_t *mask,
                                    uint8_t *types) {
  uint64_t count = 0;
  for (uint64_t i = 0; i < n; ++i) {
    int64_t j = (int64_t)ids[i] + offset_linear;
    if (j < 0 || j >= (int64_t)map_n) continue;
    int occ = map_kind == 0 ? !bv_none_but_empty((const uint8_t *)map + (uint64_t)j * BITVOXEL_BYTES)
                            : ((float)((const int8_t *)map)[j] >= thr);
    if (!occ) continue;
    uint8_t *a = list_voxels + i * BITVOXEL_BYTES;
    if (mask) {
      int meet = 0;
      for (int k = 0; k < BITVOXEL_BYTES; ++k) meet |= a[k] & mask[k];
      if (!meet) continue;
    }
    ++count;
    if (types)
      for (int k = 0; k < BITVOXEL_BYTES; ++k) types[k] |= a[k];
    a[EBVM_COLLISION >> 3] |= (uint8_t)(1u << (EBVM_COLLISION & 7));
  }
  return count;
}

/* BitVoxelList::collideWithTypes(BitVectorVoxelList*) (BitVoxelList.hpp:94-118):
 * the ids present in both sorted lists; types = OR over them of both voxels. */
uint64_t orc_list_collide_types_list(const uint32_t *ids_a, const uint8_t *vox_a, uint64_t na, const uint32_t *ids_b,
                                     const uint8_t *vox_b, uint64_t nb, uint8_t *types) {
  uint64_t i = 0, j = 0, count = 0;
  while (i < na && j < nb) {
    if (ids_a[i] < ids_b[j]) { ++i; continue; }
    if (ids_b[j] < ids_a[i]) { ++j; continue; }
    for (int k = 0; k < BITVOXEL_BYTES; ++k) types[k] |= vox_a[i * BITVOXEL_BYTES + k] | vox_b[j * BITVOXEL_BYTES + k];
    ++count; ++i; ++j;
  }
  return count;
}
