// Continuous distance queries on an EDT'd DistanceVoxel map (no counterpart
// in gpu-voxels, whose queries stop at integer voxel distances): trilinear
// distance + spatial gradient and its adjoint, sphere-model clearance per arm
// configuration, and a hinge trajectory cost with a hand-written adjoint that
// recomputes the forward kinematics.
//
// Distance field: corner value D(i,j,k) = sqrt(squaredObstacleDistance) in
// voxel units at voxel centres (i + 0.5) * side (getVoxelCenter,
// GV/voxelmap/kernels/VoxelMapOperations.h:175-182); D = sqrt(INT32_MAX) where
// the map holds no site.  The interpolant is trilinear on the centre lattice,
// points are clamped to it (zero gradient along a clamped axis).
//
// Kinematics: the reference's DH convention (DHParameters::convertDHtoM,
// GV/robot/dh_robot/KinematicLink.cu:24-79) chained as
// KinematicChain::setConfiguration (GV/robot/dh_robot/KinematicChain.cu:104-124).
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "gvx_internal.cuh"
#include "trilinear.cuh"

namespace gvx {
namespace {

constexpr unsigned kFull = 0xffffffffu;

__global__ void trilinear_kernel(MapView m, const float* __restrict__ xyz, uint64_t n, float* __restrict__ dist,
                                 float* __restrict__ grad) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const Tri t = trilinear(m, __ldg(xyz + 3 * i), __ldg(xyz + 3 * i + 1), __ldg(xyz + 3 * i + 2));
    dist[i] = t.d * m.side;
    if (grad != nullptr) {
      grad[3 * i] = t.gx;
      grad[3 * i + 1] = t.gy;
      grad[3 * i + 2] = t.gz;
    }
  }
}

__global__ void trilinear_bwd_kernel(MapView m, const float* __restrict__ xyz, uint64_t n,
                                     const float* __restrict__ gout, float* __restrict__ gxyz) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const Tri t = trilinear(m, __ldg(xyz + 3 * i), __ldg(xyz + 3 * i + 1), __ldg(xyz + 3 * i + 2));
    const float g = __ldg(gout + i);
    gxyz[3 * i] = g * t.gx;
    gxyz[3 * i + 1] = g * t.gy;
    gxyz[3 * i + 2] = g * t.gz;
  }
}

// ---------------------------------------------------------------------------
// Forward kinematics: frames F_0 = base, F_{j+1} = F_j * A_j(q_j),
// A_j = Rz(theta_j + q_j) Tz(d_j) Tx(a_j) Rx(alpha_j).  Link j spans origin
// o_j -> o_{j+1}; joint j turns about z_j (third column of F_j) through o_j.
// The chain runs once per configuration (one lane) in FP64, and sphere
// centres are formed in FP64 and rounded once to FP32: an FP32 chain of
// seven frames alone puts the centres ~1e-6 m off, 1e-4 voxel at 1 cm.  The
// distance queries themselves stay FP32.
// ---------------------------------------------------------------------------
struct Frame {
  double r[9];  // row-major rotation
  double o[3];
};

__device__ __forceinline__ Frame base_frame(const gvx_arm& arm) {
  Frame f;
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 3; ++j) f.r[3 * i + j] = arm.base[4 * i + j];
    f.o[i] = arm.base[4 * i + 3];
  }
  return f;
}

__device__ __forceinline__ Frame dh_step(const Frame& F, const gvx_arm& arm, int j, float q) {
  double st, ct, sa, ca;
  sincos((double)arm.theta[j] + (double)q, &st, &ct);
  sincos((double)arm.alpha[j], &sa, &ca);
  const double A[9] = {ct, -st * ca, st * sa, st, ct * ca, -ct * sa, 0.0, sa, ca};
  const double t[3] = {(double)arm.a[j] * ct, (double)arm.a[j] * st, (double)arm.d[j]};
  Frame G;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
#pragma unroll
    for (int k = 0; k < 3; ++k)
      G.r[3 * i + k] = F.r[3 * i] * A[k] + F.r[3 * i + 1] * A[3 + k] + F.r[3 * i + 2] * A[6 + k];
    G.o[i] = F.r[3 * i] * t[0] + F.r[3 * i + 1] * t[1] + F.r[3 * i + 2] * t[2] + F.o[i];
  }
  return G;
}

// Per-warp FK into shared memory: origins o[0..J] and joint axes z[0..J-1].
struct WarpFK {
  double o[GVX_MAX_JOINTS + 1][3];
  double z[GVX_MAX_JOINTS][3];
};

__device__ __forceinline__ void warp_fk(const gvx_arm& arm, const float* q, WarpFK& fk) {
  const int lane = threadIdx.x & 31;
  if (lane == 0) {
    Frame F = base_frame(arm);
    for (int j = 0; j < arm.n_joints; ++j) {
      fk.o[j][0] = F.o[0]; fk.o[j][1] = F.o[1]; fk.o[j][2] = F.o[2];
      fk.z[j][0] = F.r[2]; fk.z[j][1] = F.r[5]; fk.z[j][2] = F.r[8];
      F = dh_step(F, arm, j, __ldg(q + j));
    }
    fk.o[arm.n_joints][0] = F.o[0]; fk.o[arm.n_joints][1] = F.o[1]; fk.o[arm.n_joints][2] = F.o[2];
  }
  __syncwarp();
}

// Sphere centre in FP64 (the distance query splits it into cell and fraction
// in double, and the adjoint's moment arms use it as it is).
__device__ __forceinline__ void sphere_centre(const gvx_arm& arm, const WarpFK& fk, int s, double c[3]) {
  const int j = arm.link[s];
  const double t = arm.t[s];
#pragma unroll
  for (int i = 0; i < 3; ++i) c[i] = fma(t, fk.o[j + 1][i] - fk.o[j][i], fk.o[j][i]);
}

constexpr int kWarpsPerBlock = 8;

// Min clearance per configuration; one warp per configuration, lanes over spheres.
__global__ void __launch_bounds__(kWarpsPerBlock * 32) sphere_clearance_kernel(MapView m, gvx_arm arm,
                                                                              const float* __restrict__ q, uint64_t n_cfg,
                                                                              float* __restrict__ out) {
  __shared__ WarpFK s_fk[kWarpsPerBlock];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint64_t total_warps = (uint64_t)gridDim.x * kWarpsPerBlock;
  for (uint64_t cfg = (uint64_t)blockIdx.x * kWarpsPerBlock + warp; cfg < n_cfg; cfg += total_warps) {
    warp_fk(arm, q + cfg * arm.n_joints, s_fk[warp]);
    float best = __int_as_float(0x7f800000);  // +inf
    for (int s = lane; s < arm.n_spheres; s += 32) {
      double c[3];
      sphere_centre(arm, s_fk[warp], s, c);
      const Tri t = trilinear(m, c[0], c[1], c[2]);
      best = fminf(best, t.d * m.side - arm.r[s]);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) best = fminf(best, __shfl_xor_sync(kFull, best, o));
    if (lane == 0) out[cfg] = best;
    __syncwarp();
  }
}

// Hinge cost: one block per trajectory, warp w takes waypoints w, w+8, ...;
// fixed-order reductions keep the result deterministic.
__global__ void __launch_bounds__(kWarpsPerBlock * 32) traj_cost_kernel(MapView m, gvx_arm arm, const float* __restrict__ q,
                                                                       uint64_t n_traj, uint32_t n_wp, float margin,
                                                                       float* __restrict__ cost) {
  __shared__ WarpFK s_fk[kWarpsPerBlock];
  __shared__ float s_part[kWarpsPerBlock];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (uint64_t traj = blockIdx.x; traj < n_traj; traj += gridDim.x) {
    float acc = 0.0f;
    for (uint32_t w = warp; w < n_wp; w += kWarpsPerBlock) {
      warp_fk(arm, q + (traj * n_wp + w) * arm.n_joints, s_fk[warp]);
      for (int s = lane; s < arm.n_spheres; s += 32) {
        double c[3];
        sphere_centre(arm, s_fk[warp], s, c);
        const Tri t = trilinear(m, c[0], c[1], c[2]);
        acc += fmaxf(0.0f, margin - (t.d * m.side - arm.r[s]));
      }
      __syncwarp();
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(kFull, acc, o);
    if (lane == 0) s_part[warp] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
      float sum = 0.0f;
      for (int i = 0; i < kWarpsPerBlock; ++i) sum += s_part[i];
      cost[traj] = sum;
    }
    __syncthreads();
  }
}

// Adjoint of the hinge cost.  For an active sphere s on link j,
//   d cost / d q_k = -grad d(c_s) . (z_k x (c_s - o_k))   for k <= j.
// One warp per waypoint, FK recomputed: each lane evaluates its spheres once
// and adds every joint's term to a per-joint accumulator in FP64 (the moment
// arm c_s - o_k formed in double, so nothing large cancels); the spatial
// gradient g_s stays FP32 (the trilinear query's own precision).  A fixed xor
// butterfly sums the accumulators over the warp, so the result is
// deterministic.
__global__ void __launch_bounds__(kWarpsPerBlock * 32) traj_cost_bwd_kernel(MapView m, gvx_arm arm,
                                                                           const float* __restrict__ q, uint64_t n_traj,
                                                                           uint32_t n_wp, float margin,
                                                                           const float* __restrict__ gcost,
                                                                           float* __restrict__ gq) {
  __shared__ WarpFK s_fk[kWarpsPerBlock];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int J = arm.n_joints;
  const uint64_t n_items = n_traj * n_wp;
  const uint64_t total_warps = (uint64_t)gridDim.x * kWarpsPerBlock;
  for (uint64_t item = (uint64_t)blockIdx.x * kWarpsPerBlock + warp; item < n_items; item += total_warps) {
    const uint64_t traj = item / n_wp;
    warp_fk(arm, q + item * J, s_fk[warp]);
    double acc[GVX_MAX_JOINTS];
#pragma unroll
    for (int k = 0; k < GVX_MAX_JOINTS; ++k) acc[k] = 0.0;
    for (int s = lane; s < arm.n_spheres; s += 32) {
      double c[3];
      sphere_centre(arm, s_fk[warp], s, c);
      const Tri t = trilinear(m, c[0], c[1], c[2]);
      if (margin - (t.d * m.side - arm.r[s]) > 0.0f) {
        const int js = arm.link[s];
        const double gx = t.gx, gy = t.gy, gz = t.gz;
#pragma unroll
        for (int k = 0; k < GVX_MAX_JOINTS; ++k) {
          if (k > js) break;  // joints beyond the sphere's link do not move it
          const double* o = s_fk[warp].o[k];
          const double* z = s_fk[warp].z[k];
          const double lx = c[0] - o[0], ly = c[1] - o[1], lz = c[2] - o[2];
          acc[k] -= gx * (z[1] * lz - z[2] * ly) + gy * (z[2] * lx - z[0] * lz) + gz * (z[0] * ly - z[1] * lx);
        }
      }
    }
#pragma unroll
    for (int k = 0; k < GVX_MAX_JOINTS; ++k) {
      if (k >= J) break;  // warp-uniform
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) acc[k] += __shfl_xor_sync(kFull, acc[k], o);
    }
    if (lane == 0) {
      const double g = __ldg(gcost + traj);
#pragma unroll
      for (int k = 0; k < GVX_MAX_JOINTS; ++k)
        if (k < J) gq[item * J + k] = (float)(g * acc[k]);
    }
    __syncwarp();
  }
}

int sms() { return device_sms(); }

unsigned blocks_for(uint64_t items, uint64_t per_block, uint64_t cap_per_sm) {
  return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((items + per_block - 1) / per_block, (uint64_t)sms() * cap_per_sm));
}

MapView view(const gvx_dvm* m) {
  return MapView{m->d_vox, (int)m->dims.x, (int)m->dims.y, (int)m->dims.z, m->side,
                 (reinterpret_cast<uintptr_t>(m->d_vox) & 15u) == 0, num_voxels(m->dims)};
}

}  // namespace

cudaError_t launch_trilinear(const gvx_dvm* m, const float* d_xyz, uint64_t n, float* d_dist, float* d_grad, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  const QueryConfig q = query_config();
  trilinear_kernel<<<blocks_for(n, q.threads, q.blocks_per_sm), q.threads, 0, s>>>(view(m), d_xyz, n, d_dist, d_grad);
  return cudaGetLastError();
}

cudaError_t launch_trilinear_bwd(const gvx_dvm* m, const float* d_xyz, uint64_t n, const float* d_gout, float* d_gxyz,
                                 cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  const QueryConfig q = query_config();
  trilinear_bwd_kernel<<<blocks_for(n, q.threads, q.blocks_per_sm), q.threads, 0, s>>>(view(m), d_xyz, n, d_gout, d_gxyz);
  return cudaGetLastError();
}

cudaError_t launch_sphere_clearance(const gvx_dvm* m, const gvx_arm& arm, const float* d_q, uint64_t n_cfg, float* d_out,
                                    cudaStream_t s) {
  if (n_cfg == 0) return cudaSuccess;
  sphere_clearance_kernel<<<blocks_for(n_cfg, kWarpsPerBlock, 8), kWarpsPerBlock * 32, 0, s>>>(view(m), arm, d_q, n_cfg,
                                                                                              d_out);
  return cudaGetLastError();
}

cudaError_t launch_traj_cost(const gvx_dvm* m, const gvx_arm& arm, const float* d_q, uint64_t n_traj, uint32_t n_wp,
                             float margin, float* d_cost, cudaStream_t s) {
  if (n_traj == 0) return cudaSuccess;
  traj_cost_kernel<<<(unsigned)std::min<uint64_t>(n_traj, (uint64_t)sms() * 32), kWarpsPerBlock * 32, 0, s>>>(
      view(m), arm, d_q, n_traj, n_wp, margin, d_cost);
  return cudaGetLastError();
}

cudaError_t launch_traj_cost_bwd(const gvx_dvm* m, const gvx_arm& arm, const float* d_q, uint64_t n_traj, uint32_t n_wp,
                                 float margin, const float* d_gcost, float* d_gq, cudaStream_t s) {
  if (n_traj == 0 || n_wp == 0) return cudaSuccess;
  traj_cost_bwd_kernel<<<blocks_for(n_traj * n_wp, kWarpsPerBlock, 8), kWarpsPerBlock * 32, 0, s>>>(
      view(m), arm, d_q, n_traj, n_wp, margin, d_gcost, d_gq);
  return cudaGetLastError();
}

}  // namespace gvx
