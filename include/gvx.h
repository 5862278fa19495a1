/*
 * gvx.h -- C ABI of the B200 distance-field collision engine.
 *
 * Plain pointers and sizes only.  Every call returns a gvx_status; a
 * non-zero status leaves a message in gvx_last_error() (per thread).
 * Device pointers (d_*) are caller-owned device memory; host pointers (h_*)
 * are caller-owned host memory.  Calls taking a `stream` are stream-ordered
 * and asynchronous unless their comment says otherwise; pass 0 for the
 * legacy default stream.
 *
 * Each entry point names the reference interface it replaces
 * (GV = packages/gpu_voxels/src/gpu_voxels/ in gpu-voxels).
 *
 * Value formats (identical to the reference):
 *   DistanceVoxel : uint32  x | y<<10 | z<<20, 0x3FFFFFFF = uninitialised
 *                   (GV/voxel/DistanceVoxel.hpp:31-65, GV/helpers/common_defines.h:113-131)
 *   BitVoxel<256> : 32 bytes, bit k = BitVoxelMeaning k (GV/helpers/BitVector.h:349-350)
 *   linear id     : z*X*Y + y*X + x (GV/voxelmap/kernels/VoxelMapOperations.h:44-49)
 *   points        : float32 xyz triples in metres (Vector3f, GV/helpers/cuda_vectors.h:192-203)
 */
#ifndef GVX_H_
#define GVX_H_

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define GVX_API __attribute__((visibility("default")))
#else
#define GVX_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum gvx_status {
  GVX_OK = 0,
  GVX_ERR_INVALID_ARG = 1,  /* null pointer, bad enum, mismatched dims */
  GVX_ERR_OUT_OF_DOMAIN = 2,/* dims outside [1,1023] per axis, too many voxels */
  GVX_ERR_OOM = 3,          /* device allocation failed */
  GVX_ERR_CUDA = 4,         /* a CUDA runtime call failed */
  GVX_ERR_TIMEOUT = 5,      /* a bounded device-side wait gave up */
  GVX_ERR_NO_DEVICE = 6     /* no CUDA device with compute capability 10.x */
} gvx_status;

typedef struct gvx_dims { uint32_t x, y, z; } gvx_dims;

/* Opaque handles. */
typedef struct gvx_dvm gvx_dvm;   /* DistanceVoxelMap */
typedef struct gvx_bvm gvx_bvm;   /* BitVectorVoxelMap (BitVoxelMap<256>) */
typedef struct gvx_pvm gvx_pvm;   /* ProbVoxelMap (int8 occupancy per voxel) */
typedef struct gvx_blist gvx_blist; /* BitVectorVoxelList */

typedef void *gvx_stream; /* cudaStream_t */

/* ---- library ----------------------------------------------------------- */
GVX_API const char *gvx_last_error(void);
GVX_API const char *gvx_version(void);
/* Replaces cuTestAndInitDevice (GV/helpers/cuda_handling.cu:102-130): select
 * the device, check it is a compute-capability-10 part. */
GVX_API gvx_status gvx_init_device(int device);

/* ---- DistanceVoxelMap (GV/voxelmap/DistanceVoxelMap.h) ------------------ */

/* Replaces DistanceVoxelMap(dim, side, MT_DISTANCE_VOXELMAP) ->
 * TemplateVoxelMap ctor (GV/voxelmap/TemplateVoxelMap.hpp:62-144).  The map
 * is cleared (all voxels uninitialised).  Dims must be in [1,1023] per axis. */
GVX_API gvx_status gvx_dvm_create(const gvx_dims *dims, float voxel_side, gvx_dvm **out);
/* Wraps caller-owned device memory, like the non-owning ctor
 * TemplateVoxelMap(Voxel* dev_data, ...) (TemplateVoxelMap.hpp:145-154). */
GVX_API gvx_status gvx_dvm_wrap(const gvx_dims *dims, float voxel_side, uint32_t *d_voxels, gvx_dvm **out);
GVX_API gvx_status gvx_dvm_destroy(gvx_dvm *m);
GVX_API gvx_status gvx_dvm_info(const gvx_dvm *m, gvx_dims *dims, float *voxel_side, uint32_t **d_voxels);

/* Replaces TemplateVoxelMap<DistanceVoxel>::clearMap (TemplateVoxelMap.hpp:244-271). */
GVX_API gvx_status gvx_dvm_clear(gvx_dvm *m, gvx_stream stream);

/* Replaces TemplateVoxelMap::insertPointCloud(const Vector3f*, uint32_t, eBVM_OCCUPIED)
 * (TemplateVoxelMap.hpp:689-709) with kernelInsertGlobalPointCloud<DistanceVoxel>
 * (GV/voxelmap/kernels/VoxelMapOperations.hpp:266-300).  d_xyz: n float triples
 * on the device.  d_outside (optional, device uint32): set to 1 when a point
 * fell outside the map (the reference's points_outside_map flag). */
GVX_API gvx_status gvx_dvm_insert_points(gvx_dvm *m, const float *d_xyz, uint64_t n, uint32_t *d_outside, gvx_stream stream);

/* Replaces DistanceVoxelMap::parallelBanding3D(m1,m2,m3,...)
 * (GV/voxelmap/DistanceVoxelMap.hpp:284-645).  Exact EDT in place: every
 * voxel ends up holding its nearest obstacle site, bit-identical to the
 * reference with band counts (1,1,1).  The band counts are accepted for
 * API compatibility; results never depend on them. */
GVX_API gvx_status gvx_dvm_edt(gvx_dvm *m, uint32_t m1, uint32_t m2, uint32_t m3, gvx_stream stream);
/* clearMap + insertPointCloud + parallelBanding3D in one call, with the same
 * result (and the same outside flag) as the three calls in a row
 * (TemplateVoxelMap.hpp:244-271, :665-709; DistanceVoxelMap.hpp:284-645).
 * The points are recorded as occupancy bits in the map's workspace and the
 * z sweep builds the map from them, so the map is written once instead of
 * cleared, scattered and re-read.  No counterpart in the reference. */
GVX_API gvx_status gvx_dvm_voxelize_edt(gvx_dvm *m, const float *d_xyz, uint64_t n, uint32_t *d_outside,
                                        gvx_stream stream);
/* One stage of the EDT, for per-pass timing and tests: 0 = the z sweep (when
 * every voxel is UNINIT or its own site: occupancy bits read from the map,
 * then the sweep over the bits; otherwise the general sweep), 1 = the y sweep,
 * 2 = the x sweep (one launch each), 3 = the y and x sweeps
 * as the single fused launch gvx_dvm_edt uses, which takes pass 0's output
 * and its record of the route it took (0 then 3 == gvx_dvm_edt;
 * 0, 1, 2 gives the same result).  Pass 0 alone equals the reference's
 * phase 1 (kernelPBAphase1FloodZ, GV/voxelmap/kernels/VoxelMapOperationsPBA.hpp:63-124). */
GVX_API gvx_status gvx_dvm_edt_pass(gvx_dvm *m, int pass, gvx_stream stream);
/* EDT launch configuration chosen by the autotuner: rows per staging chunk of
 * the sweeps (16 or 32; 0 = library default), whether the y and x sweeps run
 * as one fused launch (1) or two (0), and the time measured for it. */
typedef struct {
  uint32_t rows;
  uint32_t fused;
  float ms;
} gvx_edt_config;
/* Project-written autotuner (no counterpart in the reference, whose PBA band
 * counts are fixed by the caller): times every configuration on a copy of
 * the map's current content (allocated for the call and freed; the map is
 * not modified), keeps the fastest for this map's later EDTs and returns it.
 * Choices are cached per device and dims in memory and, if the environment
 * variable GVX_TUNE_CACHE names a file, across processes; force = 1 re-times.
 * Synchronises the stream.  Every configuration gives bit-identical results. */
GVX_API gvx_status gvx_dvm_autotune(gvx_dvm *m, int force, gvx_edt_config *out, gvx_stream stream);
/* Sets the configuration explicitly (ms is ignored). */
GVX_API gvx_status gvx_dvm_set_edt_config(gvx_dvm *m, const gvx_edt_config *cfg);
/* Synchronises the device and reads the error word of the last EDT on this
 * map: *flags = 0 when every bounded wait of the fused y -> x sweep ended in
 * time, else non-zero with GVX_ERR_TIMEOUT (the map's content is then
 * invalid).  No counterpart in the reference, whose EDT has no waits. */
GVX_API gvx_status gvx_dvm_edt_check(gvx_dvm *m, uint32_t *flags);
/* Self-check of the EDT's bisector arithmetic on this device: the sweeps
 * round the quotient of devicePBAintersection3DY (VoxelMapOperationsPBA.hpp:
 * 265-276) without the general divide.  Compares it, bit for bit, with the
 * IEEE divide for every numerator (|num| < 2^21) and divisor (even, 2..2046)
 * the sweeps can meet; *mismatches = 0 when all agree.  Synchronous. */
GVX_API gvx_status gvx_check_bisector_quotient(uint64_t *mismatches);

/* No counterpart in the reference.  The same EDT as gvx_dvm_edt, in place on
 * caller-owned device voxels (uint32 DistanceVoxels, x fastest, 16-byte
 * aligned), for callers that may not allocate device memory once running
 * (real-time control loops, plugins inside a host that owns all device
 * memory).  It calls no cudaMalloc/cudaFree and no allocating library
 * routine: its workspace is a 64 MiB array built into the library.  Under
 * CUDA's default lazy module loading the array is committed on a device at
 * this entry point's first call there; under eager loading
 * (CUDA_MODULE_LOADING=EAGER) in every device context the process creates.
 * It stays committed until the process exits.
 * Limit: the map must need at most 16,777,216 workspace words, i.e. at most
 * 16,777,216 voxels with x and y rounded up to multiples of 32 (256^3 fits);
 * larger maps return GVX_ERR_OUT_OF_DOMAIN and are left untouched.
 * The first call on each device looks up the workspace's device address
 * (cudaGetSymbolAddress) and caches it; make that first call before any
 * stream capture.  The cached address does not survive cudaDeviceReset.
 * All calls share the one workspace and no part of it has to start at zero,
 * but calls that overlap on the GPU (other streams, other threads) race on
 * it: order them on one stream or synchronise between them. */
GVX_API gvx_status gvx_dvm_edt_static_workspace(uint32_t *d_voxels, const gvx_dims *dims, gvx_stream stream);
/* No counterpart in the reference.  The handle-free form of gvx_dvm_edt_check
 * for gvx_dvm_edt_static_workspace: synchronises the device and reads the
 * error word of the last static-workspace EDT (the one with these dims):
 * *flags = 0 when every bounded wait of its fused y -> x sweep ended in
 * time, else non-zero with GVX_ERR_TIMEOUT (that map's content is then
 * invalid).  Allocates nothing. */
GVX_API gvx_status gvx_dvm_edt_static_workspace_check(const gvx_dims *dims, uint32_t *flags);

/* Replaces DistanceVoxelMap::getSquaredDistances(device_ptr<uint> b, e, device_ptr<int32_t> out)
 * (DistanceVoxelMap.hpp:741-752): squared voxel distance to the nearest site
 * at each linear id; INT32_MAX when the map has no site or the id is out of range. */
GVX_API gvx_status gvx_dvm_sqdist(const gvx_dvm *m, const uint32_t *d_ids, uint64_t n, int32_t *d_out, gvx_stream stream);
/* Replaces DistanceVoxelMap::getDistances (DistanceVoxelMap.hpp:786-797): int32(sqrtf(sqdist)). */
GVX_API gvx_status gvx_dvm_dist(const gvx_dvm *m, const uint32_t *d_ids, uint64_t n, int32_t *d_out, gvx_stream stream);
/* Replaces TemplateVoxelMap::gatherVoxelsByIndex (TemplateVoxelMap.hpp:381-388). */
GVX_API gvx_status gvx_dvm_gather(const gvx_dvm *m, const uint32_t *d_ids, uint64_t n, uint32_t *d_out, gvx_stream stream);
/* Whole-map squared distances (the voxel-wise form of SquaredDistanceFunctor). */
GVX_API gvx_status gvx_dvm_sqdist_map(const gvx_dvm *m, int32_t *d_out, gvx_stream stream);

/* ---- continuous queries (no reference counterpart; new in this library) -- */

/* Trilinear distance (metres) at continuous points (metres) and its spatial
 * gradient.  Voxel i's centre is (i + 0.5) * side (getVoxelCenter,
 * GV/voxelmap/kernels/VoxelMapOperations.h:175-182); corner distances are
 * sqrt(sqdist) * side; points are clamped to the centre lattice.
 * d_grad (optional): n*3 floats. */
GVX_API gvx_status gvx_query_trilinear(const gvx_dvm *m, const float *d_xyz, uint64_t n, float *d_dist, float *d_grad,
                               gvx_stream stream);
/* Adjoint: d_grad_xyz[i] = d_grad_dist[i] * grad d(x_i); recomputes the gathers. */
GVX_API gvx_status gvx_query_trilinear_bwd(const gvx_dvm *m, const float *d_xyz, uint64_t n, const float *d_grad_dist,
                                   float *d_grad_xyz, gvx_stream stream);
/* Launch shape of the trilinear query kernels (gvx_query_trilinear, its
 * adjoint and gvx_batch_query_trilinear): threads per block (64, 128, 256 or
 * 512) and the grid cap in blocks per SM (1..64; the kernels stride over the
 * points).  One setting per process; default 256 x 16.  Every shape gives
 * bit-identical results, only the speed changes. */
typedef struct {
  uint32_t threads;
  uint32_t blocks_per_sm;
  float ms;
} gvx_query_config;
/* Project-written query autotuner: times gvx_query_trilinear on the caller's
 * points and output buffers (which it overwrites) for threads {64, 128, 256,
 * 512} x caps {8, 16, 32} blocks per SM, sets the fastest and returns it in
 * *out (optional).  The choice is cached per device for the process; force = 1
 * re-times.  Synchronises the stream.  d_grad may be NULL. */
GVX_API gvx_status gvx_query_autotune(const gvx_dvm *m, const float *d_xyz, uint64_t n, float *d_dist, float *d_grad,
                                      int force, gvx_query_config *out, gvx_stream stream);
/* Sets the shape explicitly (ms is ignored); GVX_ERR_INVALID_ARG outside the ranges above. */
GVX_API gvx_status gvx_set_query_config(const gvx_query_config *cfg);

/* Serial-chain arm in the reference's DH convention
 * (KinematicLink::convertDHtoM, GV/robot/dh_robot/KinematicLink.cu:24-79):
 * T_j = Rz(theta_j + q_j) Tz(d_j) Tx(a_j) Rx(alpha_j).  Spheres sit on links:
 * sphere s lies on link link[s] at fraction t[s] of the segment from the
 * link's start frame origin to its end frame origin, radius r[s]. */
#define GVX_MAX_JOINTS 16
#define GVX_MAX_SPHERES 256
typedef struct gvx_arm {
  int32_t n_joints;
  int32_t n_spheres;
  float base[16];                 /* row-major 4x4 base transform */
  float theta[GVX_MAX_JOINTS], d[GVX_MAX_JOINTS], a[GVX_MAX_JOINTS], alpha[GVX_MAX_JOINTS];
  int32_t link[GVX_MAX_SPHERES];
  float t[GVX_MAX_SPHERES], r[GVX_MAX_SPHERES];
} gvx_arm;

/* Per configuration: min over spheres of (trilinear distance at the centre - radius).
 * d_q: n_cfg * n_joints floats.  d_out: n_cfg floats. */
GVX_API gvx_status gvx_sphere_clearance(const gvx_dvm *m, const gvx_arm *arm, const float *d_q, uint64_t n_cfg, float *d_out,
                                gvx_stream stream);
/* Hinge cost per trajectory: sum over waypoints and spheres of
 * max(0, margin - (d(centre) - r)).  d_q: n_traj * n_wp * n_joints.
 * d_cost: n_traj floats. */
GVX_API gvx_status gvx_traj_cost(const gvx_dvm *m, const gvx_arm *arm, const float *d_q, uint64_t n_traj, uint32_t n_wp,
                         float margin, float *d_cost, gvx_stream stream);
/* Adjoint of gvx_traj_cost: d_grad_q = d_grad_cost[traj] * dcost/dq, with the
 * forward kinematics recomputed (nothing is stored by the forward). */
GVX_API gvx_status gvx_traj_cost_bwd(const gvx_dvm *m, const gvx_arm *arm, const float *d_q, uint64_t n_traj, uint32_t n_wp,
                             float margin, const float *d_grad_cost, float *d_grad_q, gvx_stream stream);

/* ---- batches of maps (no reference counterpart) ------------------------- */

/* Many DistanceVoxelMaps of uneven dims processed together.  The reference
 * runs one map per call with device synchronisations in between
 * (DistanceVoxelMap.hpp:284-645); a batch runs clear, voxelisation, the EDT
 * passes and trilinear queries as one launch each over all maps, and can
 * record the whole step as a CUDA graph.  The maps stay owned by the caller
 * and must outlive the batch. */
typedef struct gvx_batch gvx_batch;
GVX_API gvx_status gvx_batch_create(gvx_dvm *const *maps, uint32_t n_maps, gvx_batch **out);
GVX_API gvx_status gvx_batch_destroy(gvx_batch *b);
GVX_API gvx_status gvx_batch_clear(gvx_batch *b, gvx_stream stream);
/* Points of all maps concatenated; map k owns points [d_offsets[k], d_offsets[k+1]). */
GVX_API gvx_status gvx_batch_insert_points(gvx_batch *b, const float *d_xyz, const uint64_t *d_offsets, uint64_t n_total,
                                           gvx_stream stream);
/* EDT of every map, bit-identical to gvx_dvm_edt per map: one launch for the
 * z sweeps of all maps, one fused launch for their y and x sweeps. */
GVX_API gvx_status gvx_batch_edt(gvx_batch *b, gvx_stream stream);
/* gvx_batch_clear + gvx_batch_insert_points + gvx_batch_edt in one call, as
 * gvx_dvm_voxelize_edt per map (this is what a captured graph records). */
GVX_API gvx_status gvx_batch_voxelize_edt(gvx_batch *b, const float *d_xyz, const uint64_t *d_offsets,
                                          uint64_t n_total, gvx_stream stream);
/* As gvx_dvm_edt_check, for the last gvx_batch_edt. */
GVX_API gvx_status gvx_batch_edt_check(gvx_batch *b, uint32_t *flags);
/* As gvx_dvm_autotune for the batched EDT (rows per staging chunk; the batch
 * always fuses).  The maps' content is saved to a temporary buffer before the
 * timing runs and restored after them.  Re-capture a graph after tuning. */
GVX_API gvx_status gvx_batch_autotune(gvx_batch *b, int force, gvx_edt_config *out, gvx_stream stream);
/* Query i is answered on map d_map[i]; d_grad optional. */
GVX_API gvx_status gvx_batch_query_trilinear(gvx_batch *b, const float *d_xyz, const uint32_t *d_map, uint64_t n,
                                             float *d_dist, float *d_grad, gvx_stream stream);
/* Record clear -> insert -> EDT -> queries on the given device buffers as one
 * CUDA graph (runs the step once outside the capture first); replay it with
 * gvx_batch_graph_launch.  Blocking. */
GVX_API gvx_status gvx_batch_graph_capture(gvx_batch *b, const float *d_xyz, const uint64_t *d_offsets, uint64_t n_total,
                                           const float *d_qxyz, const uint32_t *d_qmap, uint64_t n_q, float *d_dist,
                                           float *d_grad, gvx_stream stream);
GVX_API gvx_status gvx_batch_graph_launch(gvx_batch *b, gvx_stream stream);

/* ---- BitVectorVoxelMap (GV/voxelmap/BitVoxelMap.h) ---------------------- */

/* Replaces BitVoxelMap<256>(dim, side, MT_BITVECTOR_VOXELMAP).  Unlike the
 * reference (32-bit byte limit, TemplateVoxelMap.hpp:71-81) a 512^3 map is allowed. */
GVX_API gvx_status gvx_bvm_create(const gvx_dims *dims, float voxel_side, gvx_bvm **out);
GVX_API gvx_status gvx_bvm_destroy(gvx_bvm *m);
GVX_API gvx_status gvx_bvm_info(const gvx_bvm *m, gvx_dims *dims, float *voxel_side, uint8_t **d_voxels);
/* Replaces TemplateVoxelMap<BitVectorVoxel>::clearMap. */
GVX_API gvx_status gvx_bvm_clear(gvx_bvm *m, gvx_stream stream);
/* Replaces insertPointCloud with kernelInsertGlobalPointCloud<BitVoxel>
 * (VoxelMapOperations.hpp:241-264): sets bit `meaning` (0..255). */
GVX_API gvx_status gvx_bvm_insert_points(gvx_bvm *m, const float *d_xyz, uint64_t n, uint32_t meaning, uint32_t *d_outside,
                                 gvx_stream stream);
/* Replaces BitVoxelMap::clearBits / clearBit / clearBitVoxelMeaning
 * (GV/voxelmap/BitVoxelMap.hpp:63-88,343-347; kernelClearVoxelMap,
 * VoxelMapOperations.hpp:45-71): clears the set bits of `bits` (host, 32
 * bytes, BitVector<256> layout) in every voxel. */
GVX_API gvx_status gvx_bvm_clear_bits(gvx_bvm *m, const uint8_t *bits, gvx_stream stream);
/* Replaces BitVoxelMap::shiftLeftSweptVolumeIDs (BitVoxelMap.hpp:349-361;
 * performLeftShift, GV/helpers/BitVector.h:355-402): every voxel's meaning k
 * becomes k - shift (lower ones drop out) and meanings 0..3 are cleared.
 * shift <= 56, else GVX_ERR_INVALID_ARG and nothing changes. */
GVX_API gvx_status gvx_bvm_shift_swept_volume_ids(gvx_bvm *m, uint32_t shift, gvx_stream stream);
/* Replaces BitVoxelMap::insertMetaPointCloudWithSelfCollisionCheck
 * (GV/voxelmap/BitVoxelMap.hpp:227-341; kernel kernelInsertMetaPointCloudSelfCollCheck,
 * VoxelMapOperations.hpp:581-631).  Sub-cloud k (a robot link) is d_xyz points
 * offsets[k] .. offsets[k+1] (host array of n_clouds + 1 entries).  Sub-clouds
 * go in order; each first checks its voxels against the map as the earlier
 * ones left it (voxel bits & masks[k]; a hit is any masked bit but bit 0),
 * then sets meanings[k] in its voxels and eBVM_COLLISION where it hit.
 * meanings: n_clouds bytes (host), NULL = eBVM_SWEPT_VOLUME_START + k.
 * masks: n_clouds BitVectors of 32 bytes (host), NULL = every bit but
 * eBVM_COLLISION and the sub-cloud's own meaning.  colliding (host, 32 bytes,
 * may be NULL) receives the OR of the masked bits of every hit plus the
 * meanings of the sub-clouds that hit; *any (may be NULL) = colliding != 0,
 * the reference's return value.  *d_outside = 1 if a point lies outside the
 * map.  Synchronises the stream. */
GVX_API gvx_status gvx_bvm_insert_meta_points_self_coll(gvx_bvm *m, const float *d_xyz, const uint64_t *offsets,
                                                        uint32_t n_clouds, const uint8_t *meanings, const uint8_t *masks,
                                                        uint8_t *colliding, int *any, uint32_t *d_outside,
                                                        gvx_stream stream);
/* Replaces BitVoxelMap::collideWith(const BitVectorVoxelMap*, thr, offset)
 * (GV/voxelmap/BitVoxelMap.hpp:198-203 -> TemplateVoxelMap.hpp:588-621 ->
 * kernelCollideVoxelMapsDebug, VoxelMapOperations.hpp:129-184, DefaultCollider
 * GV/voxel/DefaultCollider.hpp:76-81).  Counts voxels i where self[i+off] and
 * other[i] both hold a meaning other than eBVM_FREE; off is the linear form of
 * `offset`; pairs whose shifted index leaves the map are skipped.  With
 * mark != 0 colliding self voxels get eBVM_COLLISION.  *d_count (device
 * uint64) receives the count. */
GVX_API gvx_status gvx_bvm_collide(gvx_bvm *self, const gvx_bvm *other, const int32_t offset[3], int mark, uint64_t *d_count,
                           gvx_stream stream);

/* Replaces BitVoxelMap::collideWith(const ProbVoxelMap*, coll_threshold, offset)
 * (GV/voxelmap/BitVoxelMap.hpp:205-210 -> TemplateVoxelMap.hpp:588-621 ->
 * kernelCollideVoxelMapsDebug, DefaultCollider::collide(BitVoxel,
 * ProbabilisticVoxel), GV/voxel/DefaultCollider.hpp:68-73).  Counts voxels i
 * where other[i]'s occupancy reaches floatToProbability(coll_threshold)
 * (clamped to [0, 1], GV/voxel/ProbabilisticVoxel.h:40-45) and self[i+off]
 * holds a meaning other than eBVM_FREE; pairs whose shifted index leaves the
 * map are skipped; with mark != 0 colliding self voxels get eBVM_COLLISION.
 * *d_count (device uint64) receives the count. */
GVX_API gvx_status gvx_bvm_collide_pvm(gvx_bvm *self, const gvx_pvm *other, float coll_threshold,
                                       const int32_t offset[3], int mark, uint64_t *d_count, gvx_stream stream);

/* ---- Typed collisions ------------------------------------------------------ */
/* Every call overwrites *d_count (device uint64) with the number of colliding
 * voxels / entries and, where given, d_types (device, 32 bytes = one
 * BitVector<256>) with the OR of the colliding types; colliding voxels of
 * `self` / entries of the list get eBVM_COLLISION. */

/* Replaces BitVoxelMap::collideWithTypes(const BitVectorVoxelMap*, BitVectorVoxel&, thr, offset)
 * (GV/voxelmap/BitVoxelMap.hpp:212-217 -> kernelCollideVoxelMapsBitvector,
 * GV/voxelmap/kernels/VoxelMapOperations.hpp:187-239, SVCollider window 0,
 * GV/voxel/SVCollider.hpp:90-96, GV/helpers/BitVector.h:415-470): the types of
 * voxel i are self[i] & other[i] on the swept-volume bits (4..255).  The
 * reference ignores the offset and threshold here; so does this entry. */
GVX_API gvx_status gvx_bvm_collide_types(gvx_bvm *self, const gvx_bvm *other, uint64_t *d_count, uint8_t *d_types,
                                         gvx_stream stream);
/* Replaces collideWithTypes(const ProbVoxelMap*, ...) (BitVoxelMap.hpp:219-224,
 * SVCollider.hpp:98-108): occupancy >= SVCollider's threshold (thr*254-127,
 * not clamped) and self not empty; the types are all of self's bits. */
GVX_API gvx_status gvx_bvm_collide_types_pvm(gvx_bvm *self, const gvx_pvm *other, float coll_threshold,
                                             uint64_t *d_count, uint8_t *d_types, gvx_stream stream);

/* ---- ProbVoxelMap (GV/voxelmap/ProbVoxelMap.h) and mergeOccupied -------- */

/* Replaces ProbVoxelMap(dim, side, MT_PROBAB_VOXELMAP) (GV/voxelmap/ProbVoxelMap.hpp:35-39):
 * one int8 occupancy per voxel (ProbabilisticVoxel, GV/voxel/ProbabilisticVoxel.h),
 * created UNKNOWN (-128). */
GVX_API gvx_status gvx_pvm_create(const gvx_dims *dims, float voxel_side, gvx_pvm **out);
GVX_API gvx_status gvx_pvm_destroy(gvx_pvm *m);
GVX_API gvx_status gvx_pvm_info(const gvx_pvm *m, gvx_dims *dims, float *voxel_side, int8_t **d_voxels);
/* Replaces TemplateVoxelMap<ProbabilisticVoxel>::clearMap (GV/voxelmap/TemplateVoxelMap.hpp:222-238). */
GVX_API gvx_status gvx_pvm_clear(gvx_pvm *m, gvx_stream stream);
/* Replaces insertPointCloud -> kernelInsertGlobalPointCloud<ProbabilisticVoxel>
 * (GV/voxelmap/kernels/VoxelMapOperations.hpp:241-264) with
 * ProbabilisticVoxel::insert (GV/voxel/ProbabilisticVoxel.hpp:44-100): eBVM_FREE
 * adds -10, eBVM_OCCUPIED/COLLISION +72, meanings 4..254 add meaning - 129,
 * UNKNOWN/UNDEFINED reset to -128; an UNKNOWN voxel starts from 0; sums
 * saturate at [-127, 127].  Every point's update is applied (the reference's
 * non-atomic update can drop some when points share a voxel). */
GVX_API gvx_status gvx_pvm_insert_points(gvx_pvm *m, const float *d_xyz, uint64_t n, uint32_t meaning,
                                         uint32_t *d_outside, gvx_stream stream);
/* Replaces DistanceVoxelMap::mergeOccupied(prob_map, offset, threshold)
 * (GV/voxelmap/DistanceVoxelMap.hpp:109-136, GV/voxelmap/DistanceVoxelMap.h:92-134):
 * every voxel whose occupancy exceeds floatToProbability(threshold) gets the
 * site of its own coordinates plus `offset` (NULL = 0); other voxels keep
 * their value.  The maps must have equal dims (the reference does not check). */
GVX_API gvx_status gvx_dvm_merge_occupied(gvx_dvm *m, const gvx_pvm *other, const uint32_t offset[3],
                                          float occupancy_threshold, gvx_stream stream);

/* ---- On-disk format ------------------------------------------------------- */
/* Replace TemplateVoxelMap::writeToDisk / readFromDisk (GV/voxelmap/TemplateVoxelMap.hpp:906-1039),
 * binary mode: int32 MapType (BitVectorVoxelMap 0, ProbVoxelMap 4,
 * DistanceVoxelMap 9), float voxel side, uint32 x, y, z, then the voxels byte
 * for byte -- files interchange with the reference's.  Blocking (the device
 * is synchronised first).  Reading fails on a different type or dims and
 * only warns on a different voxel side, as the reference does. */
GVX_API gvx_status gvx_dvm_write_to_disk(const gvx_dvm *m, const char *path);
GVX_API gvx_status gvx_dvm_read_from_disk(gvx_dvm *m, const char *path);
GVX_API gvx_status gvx_bvm_write_to_disk(const gvx_bvm *m, const char *path);
GVX_API gvx_status gvx_bvm_read_from_disk(gvx_bvm *m, const char *path);
GVX_API gvx_status gvx_pvm_write_to_disk(const gvx_pvm *m, const char *path);
GVX_API gvx_status gvx_pvm_read_from_disk(gvx_pvm *m, const char *path);

/* ---- Consumers of the distance field ------------------------------------- */

/* Replaces DistanceVoxelMap::extract_distances(free_space_t*, robot_radius)
 * (GV/voxelmap/DistanceVoxelMap.hpp:676-688, DistanceVoxel::extract_byte_distance
 * GV/voxel/DistanceVoxel.h:144-199): one int8 per voxel -- the distance to the
 * map border for voxels within robot_radius of it, else int(sqrtf(squared
 * obstacle distance)) capped at 127. */
GVX_API gvx_status gvx_dvm_extract_distances(const gvx_dvm *m, int8_t *d_out, int robot_radius, gvx_stream stream);
/* Replaces DistanceVoxelMap::init_floodfill (DistanceVoxelMap.hpp:658-674,
 * DistanceVoxel::init_floodfill_distance DistanceVoxel.h:201-215): int16 per
 * voxel, 32765 (too close) where the byte <= robot_radius, else 32767. */
GVX_API gvx_status gvx_dvm_init_floodfill(const gvx_dvm *m, const int8_t *d_distances, int16_t *d_manhattan,
                                          int robot_radius, gvx_stream stream);

/* ---- BitVectorVoxelList (GV/voxellist/BitVoxelList.h) ------------------- */

/* Replaces BitVoxelList<256,uint32>(dim, side, MT_BITVECTOR_VOXELLIST). */
GVX_API gvx_status gvx_blist_create(const gvx_dims *ref_dims, float voxel_side, gvx_blist **out);
GVX_API gvx_status gvx_blist_destroy(gvx_blist *l);
/* Number of (unique) entries; synchronises the list's last update. */
GVX_API gvx_status gvx_blist_size(const gvx_blist *l, uint64_t *n);
GVX_API gvx_status gvx_blist_data(const gvx_blist *l, uint32_t **d_ids, uint8_t **d_voxels);
GVX_API gvx_status gvx_blist_clear(gvx_blist *l);
/* Replaces TemplateVoxelList::insertPointCloud (GV/voxellist/TemplateVoxelList.hpp:363-393):
 * voxelise, drop out-of-bounds, sort and merge duplicates (make_unique, :143-212).
 * Blocking. */
GVX_API gvx_status gvx_blist_insert_points(gvx_blist *l, const float *d_xyz, uint64_t n, uint32_t meaning, gvx_stream stream);
/* BitVoxelList::shiftLeftSweptVolumeIDs (GV/voxellist/BitVoxelList.hpp:641-664):
 * performLeftShift on every entry's voxel (as gvx_bvm_shift_swept_volume_ids;
 * entries stay even when their voxel becomes empty).  shift <= 56. */
GVX_API gvx_status gvx_blist_shift_swept_volume_ids(gvx_blist *l, uint32_t shift, gvx_stream stream);
/* Clears the set bits of `bits` (host, 32 bytes) in every entry's voxel; the
 * C++ BitVoxelList::clearBitVoxelMeaning uses it (the reference's list
 * reports that operation as not yet supported, BitVoxelList.hpp:57-61). */
GVX_API gvx_status gvx_blist_clear_bits(gvx_blist *l, const uint8_t *bits, gvx_stream stream);
/* Replaces BitVoxelList::collideWithTypes(const BitVectorVoxelMap*, ...) and
 * (const ProbVoxelMap*, ...) (GV/voxellist/BitVoxelList.hpp:120-201 ->
 * kernelCollideWithVoxelMap, GV/voxellist/kernels/VoxelListOperations.hpp:204-260):
 * entry i meets map voxel ids[i] + offset (skipped outside the map) and
 * collides when that voxel is occupied (BitVoxel: not noneButEmpty;
 * ProbVoxelMap: occupancy >= coll_threshold compared as float); its bits
 * (before the mark) are the types. */
GVX_API gvx_status gvx_blist_collide_types_bvm(gvx_blist *l, const gvx_bvm *map, const int32_t offset[3],
                                               uint64_t *d_count, uint8_t *d_types, gvx_stream stream);
GVX_API gvx_status gvx_blist_collide_types_pvm(gvx_blist *l, const gvx_pvm *map, float coll_threshold,
                                               const int32_t offset[3], uint64_t *d_count, uint8_t *d_types,
                                               gvx_stream stream);
/* Replaces BitVoxelList::collideWithTypeMask(map, types_to_check, ...)
 * (BitVoxelList.hpp:203-246, kernelCollideWithVoxelMapBitMask
 * VoxelListOperations.hpp:282-325): as above, counting only entries whose
 * bits meet the mask (d_mask: device, 32 bytes). */
GVX_API gvx_status gvx_blist_collide_type_mask_bvm(gvx_blist *l, const gvx_bvm *map, const uint8_t *d_mask,
                                                   const int32_t offset[3], uint64_t *d_count, gvx_stream stream);
/* Replaces BitVoxelList::collideWithTypes(const BitVectorVoxelList*, ...)
 * (BitVoxelList.hpp:94-118): ids present in both lists; types = OR of both
 * entries' bits.  Offsets are unsupported there and not taken here. */
GVX_API gvx_status gvx_blist_collide_types_blist(const gvx_blist *l, const gvx_blist *other, uint64_t *d_count,
                                                 uint8_t *d_types, gvx_stream stream);
/* Replaces distance_map_converter::extract_given_distances
 * (GV/helpers_highlevel/DistanceMapConverter.cu:156-196): the voxels whose
 * free-space byte (extract_distances at robot radius 0) lies in
 * [min_dist, max_dist] become the list `result` (its reference dims must be
 * the map's), in id order, each voxel with eBVM_OCCUPIED and swept-volume
 * bits 4 .. 4 + byte - 1 (transform_to_bitvoxel, :103-154).  Blocking;
 * *n_out = the number of entries. */
GVX_API gvx_status gvx_extract_given_distances(const gvx_dvm *m, int min_dist, int max_dist, gvx_blist *result,
                                               uint64_t *n_out, gvx_stream stream);
/* Set the list to already-sorted unique ids with their voxels (device
 * arrays, copied).  n_voxels == 0 means every voxel gets bit `meaning`. */
GVX_API gvx_status gvx_blist_set(gvx_blist *l, const uint32_t *d_ids, const uint8_t *d_voxels, uint64_t n, uint32_t meaning,
                         gvx_stream stream);
/* Replaces BitVoxelList::collideWith(const BitVectorVoxelMap*, thr, offset)
 * (BitVoxelList.hpp:71-77 -> TemplateVoxelList.hpp:1170-1213 ->
 * kernelCollideWithVoxelMap, GV/voxellist/kernels/VoxelListOperations.hpp:146-197).
 * Returns GVX_ERR_INVALID_ARG when the map's dims differ from the list's
 * reference dims (the reference returns SSIZE_MAX). */
GVX_API gvx_status gvx_blist_collide_bvm(gvx_blist *l, const gvx_bvm *map, const int32_t offset[3], int mark, uint64_t *d_count,
                                 gvx_stream stream);
/* Replaces BitVoxelList::collideWith(const ProbVoxelMap*, coll_threshold, offset)
 * (GV/voxellist/BitVoxelList.hpp:63-69 -> TemplateVoxelList.hpp:1170-1213 ->
 * kernelCollideWithVoxelMap, VoxelListOperations.hpp:146-197, DefaultCollider
 * GV/voxel/DefaultCollider.hpp:68-73): entry i collides when map voxel
 * ids[i] + offset lies in the map, its occupancy reaches
 * floatToProbability(coll_threshold) and the entry holds a meaning other
 * than eBVM_FREE; with mark != 0 colliding entries get eBVM_COLLISION.
 * GVX_ERR_INVALID_ARG when the map's dims differ from the list's reference dims. */
GVX_API gvx_status gvx_blist_collide_pvm(gvx_blist *l, const gvx_pvm *map, float coll_threshold,
                                         const int32_t offset[3], int mark, uint64_t *d_count, gvx_stream stream);
/* Replaces BitVoxelList::collideWith(const BitVectorVoxelList*, thr, offset)
 * (BitVoxelList.hpp:79-92 -> collideVoxellists, TemplateVoxelList.hpp:231-289):
 * number of this list's ids present in `other`.  Non-zero offsets are
 * rejected, as in the reference (:248-251). */
GVX_API gvx_status gvx_blist_collide_blist(const gvx_blist *l, const gvx_blist *other, const int32_t offset[3],
                                   uint64_t *d_count, gvx_stream stream);

/* Batched list-vs-map collision (no reference counterpart; the reference
 * runs one launch per list): n_lists CSR lists over concatenated arrays,
 * list k = entries [d_offsets[k], d_offsets[k+1]).  Ids must be < the map's
 * voxel count to be tested.  d_counts: n_lists uint64, overwritten.  One
 * launch; when the lists hold at least half as many entries as the map has
 * voxels, two: the map is first reduced to one occupancy bit per voxel (a
 * buffer of voxels / 8 bytes kept with the map handle) and the entries test
 * those bits, so calls on one map must not overlap on the GPU. */
GVX_API gvx_status gvx_lists_collide_bvm(const uint32_t *d_ids, uint8_t *d_voxels, const uint64_t *d_offsets, uint32_t n_lists,
                                 uint64_t n_total, const gvx_bvm *map, int mark, uint64_t *d_counts, gvx_stream stream);

#ifdef __cplusplus
}
#endif
#endif /* GVX_H_ */
