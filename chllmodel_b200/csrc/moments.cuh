// FP64 moments of one lattice site, shared by the observables kernel
// (observables.cu) and the batched kernel's measurements (batched.cu).
//
// Per site (FP64 arithmetic on the FP32 state), added into acc[0..8]:
//   acc[0] total energy with the lattice's boundary, each bond once
//          (+x, +y, +z) plus the field term;
//   acc[1] the reference etot() sum (chll_mod.f90:414-456): x and y
//          periodic, z open, and the +y dot product's x component read from
//          the diagonal neighbour (ip1,jp1,k) exactly as chll_mod.f90:438;
//   acc[2] s;  acc[3..8] nx*nx, ny*ny, nz*nz, nx*ny, nx*nz, ny*nz.
#pragma once
#include <cmath>

#include "chll_common.cuh"

namespace chll {

// Slots of one colour are < 2^31 (a lattice has < 2^32 sites), so all the
// index arithmetic below is 32-bit.
__device__ __forceinline__ float4 site_at(const LatticeView& L, int i, int j, int k) {
  return colour_array(L, (i + j + k) & 1)[((uint32_t)k * (uint32_t)L.nj + (uint32_t)j) *
                                              (uint32_t)L.hx +
                                          ((uint32_t)i >> 1)];
}

// Slot -> (row, plane) divisions of one lattice, built on the host.  For a
// z-slab (zhalo = 1) the view's planes are global planes kglob0.. of a
// lattice of nkg planes, and the plane after the view's last one is its halo:
// the +z bond of the last plane reads it, and exists unless the global
// lattice ends there (open boundary).
struct MomentGeom {
  uint32_t per_colour;  // hx * nj * nk
  FastDiv by_hx, by_nj;
  int zhalo, kglob0, nkg;
};

__host__ inline MomentGeom make_moment_geom(const LatticeView& L) {
  MomentGeom M;
  M.per_colour = (uint32_t)L.hx * (uint32_t)L.nj * (uint32_t)L.nk;
  M.by_hx = FastDiv((uint32_t)L.hx);
  M.by_nj = FastDiv((uint32_t)L.nj);
  M.zhalo = 0;
  M.kglob0 = 0;
  M.nkg = L.nk;
  return M;
}

__host__ inline MomentGeom make_slab_moment_geom(const LatticeView& L, int kglob0, int nkg) {
  MomentGeom M = make_moment_geom(L);
  M.zhalo = 1;
  M.kglob0 = kglob0;
  M.nkg = nkg;
  return M;
}

// eps*(1 - dot^2) - K*dot*cross*sfac for a forward bond.
__device__ __forceinline__ double fwd_bond(double eps, double K, double dot, double cross,
                                           double si, double sj) {
  return eps * (1.0 - dot * dot) - K * dot * cross * (0.5 * (si + sj));
}

// Storage slot e of the concatenated colour arrays (colour = e >= per_colour).
// REF_ETOT: also the reference etot() column acc[1] (measurement rows); the
// batched moments leave it out.
template <bool REF_ETOT>
__device__ __forceinline__ void site_moments(const LatticeView& L, const MomentGeom& M,
                                             const CouplingD& cp, uint32_t e,
                                             double acc[kObsMoments]) {
  const double eps = cp.eps, K = cp.K, g = cp.g;
  const int c = e >= M.per_colour;
  const uint32_t t = e - (c ? M.per_colour : 0u);
  const uint32_t r = M.by_hx.div(t);
  const int h = (int)(t - r * (uint32_t)L.hx);
  const int k = (int)M.by_nj.div(r);
  const int j = (int)(r - (uint32_t)k * (uint32_t)L.nj);
  const int i = 2 * h + ((c + j + k) & 1);
  if (i >= L.ni) return;
  const float4 nf = colour_array(L, c)[t];
  const double nx = nf.x, ny = nf.y, nz = nf.z, s = nf.w;
  const int ip = (i + 1 == L.ni) ? 0 : i + 1;
  const int jp = (j + 1 == L.nj) ? 0 : j + 1;
  const int kp = (k + 1 == L.nk && !M.zhalo) ? 0 : k + 1;
  const float4 X = site_at(L, ip, j, k);
  const float4 Y = site_at(L, i, jp, k);
  const float4 Z = site_at(L, i, j, kp);

  const double dx = nx * X.x + ny * X.y + nz * X.z;
  const double cx = ny * X.z - nz * X.y;
  const double bx = fwd_bond(eps, K, dx, cx, s, X.w);
  const double dy = nx * Y.x + ny * Y.y + nz * Y.z;
  const double cy = nz * Y.x - nx * Y.z;
  const double by = fwd_bond(eps, K, dy, cy, s, Y.w);
  const double dz = nx * Z.x + ny * Z.y + nz * Z.z;
  const double cz = nx * Z.y - ny * Z.x;
  const double bz = fwd_bond(eps, K, dz, cz, s, Z.w);

  const bool has_xp = L.periodic || (i + 1 < L.ni);
  const bool has_yp = L.periodic || (j + 1 < L.nj);
  const bool ref_zp = M.kglob0 + k + 1 < M.nkg;  // z is open in etot
  const bool has_zp = L.periodic || ref_zp;
  acc[0] += (has_xp ? bx : 0.0) + (has_yp ? by : 0.0) + (has_zp ? bz : 0.0) - g * s;

  if (REF_ETOT) {
    const float4 T = site_at(L, ip, jp, k);  // diagonal read of chll_mod.f90:438
    const double dyt = nx * (double)T.x + ny * Y.y + nz * Y.z;
    const double byt = fwd_bond(eps, K, dyt, cy, s, Y.w);
    acc[1] += bx + byt + (ref_zp ? bz : 0.0) - g * s;
  }

  acc[2] += s;
  acc[3] += nx * nx;
  acc[4] += ny * ny;
  acc[5] += nz * nz;
  acc[6] += nx * ny;
  acc[7] += nx * nz;
  acc[8] += ny * nz;
}

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Largest eigenvalue of a symmetric 3x3 matrix (Smith, "Eigenvalues of a
// symmetric 3x3 matrix", CACM 4(4):168, 1961): trigonometric solution of the
// characteristic cubic.
__host__ __device__ inline double sym3_max_eig(double a11, double a22, double a33, double a12,
                                               double a13, double a23) {
  const double p1 = a12 * a12 + a13 * a13 + a23 * a23;
  const double q = (a11 + a22 + a33) / 3.0;
  const double b11 = a11 - q, b22 = a22 - q, b33 = a33 - q;
  const double p2 = b11 * b11 + b22 * b22 + b33 * b33 + 2.0 * p1;
  if (p2 <= 0.0) return q;
  const double p = sqrt(p2 / 6.0);
  const double c11 = b11 / p, c22 = b22 / p, c33 = b33 / p;
  const double c12 = a12 / p, c13 = a13 / p, c23 = a23 / p;
  const double det = c11 * (c22 * c33 - c23 * c23) - c12 * (c12 * c33 - c23 * c13) +
                     c13 * (c12 * c23 - c22 * c13);
  double r = det / 2.0;
  r = r < -1.0 ? -1.0 : (r > 1.0 ? 1.0 : r);
  const double phi = acos(r) / 3.0;
  return q + 2.0 * p * cos(phi);
}

}  // namespace chll
