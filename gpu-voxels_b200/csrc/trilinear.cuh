// Trilinear distance field over an EDT'd DistanceVoxel map (device helpers
// shared by the continuous-query kernels and the batched schedule).
//
// Corner value D(i,j,k) = sqrt(squaredObstacleDistance) in voxel units at
// voxel centres (i + 0.5) * side (getVoxelCenter,
// GV/voxelmap/kernels/VoxelMapOperations.h:175-182); D = sqrt(INT32_MAX) where
// the map holds no site.  The interpolant is trilinear on the centre lattice,
// points are clamped to it (zero gradient along a clamped axis).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "gvx_internal.cuh"

namespace gvx {

struct MapView {
  const uint32_t* vox;
  int X, Y, Z;
  float side;
  bool aligned16;  // vox on a 16-byte boundary (the corner-pair loads below need it)
  uint64_t n;      // voxels in the map (a 16-byte word is read only when it lies inside)
};

// Distance (voxel units) from lattice point (i, j, k) to the site `v` holds.
__device__ __forceinline__ float corner_value(uint32_t v, int i, int j, int k) {
  const int ox = (int)dv_x(v), oy = (int)dv_y(v), oz = (int)dv_z(v);
  if (ox == (int)kUninit || oy == (int)kUninit || oz == (int)kUninit) return sqrtf((float)kMaxObstacleDistance);
  const int dx = i - ox, dy = j - oy, dz = k - oz;
  return sqrtf((float)(dx * dx + dy * dy + dz * dz));
}

// The two corners (i0, j, k) and (i1, j, k) of a cell edge along x.  They
// are neighbours in memory (i1 = i0 + 1, or i1 = i0 on a one-voxel axis);
// when both lie in one aligned 16-byte word (3 of 4 positions) a single
// 16-byte load fetches them, so a random-order query touches about 5 L1
// lines per point instead of 8 -- the queries are bound by those gathers.
__device__ __forceinline__ void corner_pair(const MapView& m, int i0, int i1, int j, int k, float& d0, float& d1) {
  const uint64_t idx = ((uint64_t)k * m.Y + j) * m.X + i0;
  const int o = (int)(idx & 3u);
  uint32_t v0, v1;
  if (m.aligned16 && i1 == i0 + 1 && o != 3 && idx - o + 4 <= m.n) {
    const uint4 q = __ldg(reinterpret_cast<const uint4*>(m.vox + (idx - o)));
    v0 = o == 0 ? q.x : (o == 1 ? q.y : q.z);
    v1 = o == 0 ? q.y : (o == 1 ? q.z : q.w);
  } else {
    v0 = __ldg(m.vox + idx);
    v1 = __ldg(m.vox + idx + (uint64_t)(i1 - i0));
  }
  d0 = corner_value(v0, i0, j, k);
  d1 = corner_value(v1, i1, j, k);
}

// Lattice coordinate along one axis: u = p/side - 0.5 clamped to [0, n-1];
// returns the lower corner, the fraction and whether the axis is free.  The
// fraction is taken from the residual p - (i0 + 0.5) * side (one fused
// rounding) rather than from u, which keeps it accurate far from the origin.
__device__ __forceinline__ void axis_setup(float p, float side, int n, int& i0, int& i1, float& f, bool& free_axis) {
  const float u = __fsub_rn(__fdiv_rn(p, side), 0.5f);
  const float hi = (float)(n - 1);
  free_axis = (u >= 0.0f) && (u <= hi);
  const float uc = fminf(fmaxf(u, 0.0f), hi);  // NaN -> 0
  i0 = (int)floorf(uc);
  if (free_axis) {
    // choose the cell by the sign of the exact residual, not the rounded u
    if (i0 > 0 && fmaf(-((float)i0 + 0.5f), side, p) < 0.0f) --i0;
    else if (i0 < n - 1 && fmaf(-((float)i0 + 1.5f), side, p) >= 0.0f) ++i0;
  }
  i0 = min(i0, max(n - 2, 0));
  i1 = min(i0 + 1, n - 1);
  if (free_axis) {
    f = __fdiv_rn(fmaf(-((float)i0 + 0.5f), side, p), side);
    f = fminf(fmaxf(f, 0.0f), 1.0f);
  } else {
    f = uc - (float)i0;
  }
}

// The same split of an FP64 position (sphere centres from the FP64 forward
// kinematics): cell and fraction come from p / side - 0.5 in double, so only
// the fraction (in [0, 1]) is rounded to float -- an FP32 position alone would
// carry up to half an ulp of p (1.2e-5 voxel at 2.56 m with 1 cm voxels).
__device__ __forceinline__ void axis_setup(double p, float side, int n, int& i0, int& i1, float& f, bool& free_axis) {
  const double u = p / (double)side - 0.5;
  const double hi = (double)(n - 1);
  free_axis = (u >= 0.0) && (u <= hi);
  const double uc = fmin(fmax(u, 0.0), hi);  // NaN -> 0
  i0 = min((int)floor(uc), max(n - 2, 0));
  i1 = min(i0 + 1, n - 1);
  f = (float)(uc - (double)i0);
}

struct Tri {
  float d;           // voxel units
  float gx, gy, gz;  // d(distance)/d(position), dimensionless
};

// Trilinear distance and gradient at a position given in float or double.
template <class Real>
__device__ __forceinline__ Tri trilinear(const MapView& m, Real px, Real py, Real pz) {
  int i0, i1, j0, j1, k0, k1;
  float fx, fy, fz;
  bool ax, ay, az;
  axis_setup(px, m.side, m.X, i0, i1, fx, ax);
  axis_setup(py, m.side, m.Y, j0, j1, fy, ay);
  axis_setup(pz, m.side, m.Z, k0, k1, fz, az);
  float d000, d100, d010, d110, d001, d101, d011, d111;
  corner_pair(m, i0, i1, j0, k0, d000, d100);
  corner_pair(m, i0, i1, j1, k0, d010, d110);
  corner_pair(m, i0, i1, j0, k1, d001, d101);
  corner_pair(m, i0, i1, j1, k1, d011, d111);
  // interpolate along x, then y, then z
  const float e00 = fmaf(fx, d100 - d000, d000), e10 = fmaf(fx, d110 - d010, d010);
  const float e01 = fmaf(fx, d101 - d001, d001), e11 = fmaf(fx, d111 - d011, d011);
  const float g0 = fmaf(fy, e10 - e00, e00), g1 = fmaf(fy, e11 - e01, e01);
  Tri t;
  t.d = fmaf(fz, g1 - g0, g0);
  // partial derivatives of the interpolant in lattice units
  const float sx0 = fmaf(fy, (d110 - d010) - (d100 - d000), d100 - d000);
  const float sx1 = fmaf(fy, (d111 - d011) - (d101 - d001), d101 - d001);
  t.gx = ax ? fmaf(fz, sx1 - sx0, sx0) : 0.0f;
  const float sy0 = e10 - e00, sy1 = e11 - e01;
  t.gy = ay ? fmaf(fz, sy1 - sy0, sy0) : 0.0f;
  t.gz = az ? (g1 - g0) : 0.0f;
  return t;
}

}  // namespace gvx
