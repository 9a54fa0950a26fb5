// Per-site trial arithmetic shared by the plain and batched sweep kernels.
// All FP32.  The reference (chll_mod.f90:117-245) evaluates the full local
// energy twice per trial; here the trial is decided on the energy difference,
// which needs only the products that change.
#pragma once
#include "chll_common.cuh"

namespace chll {

// Neighbours of one site in the order +x, -x, +y, -y, +z, -z.  A missing
// neighbour (open boundary) is the zero vector with s = 0: every term of an
// energy difference is a product with the neighbour, so it contributes 0.
struct Nbrs {
  float4 b[6];
};

// (v x b) . e_axis for axis 0,1,2 (chll_mod.f90:373,387,401).
template <int AXIS>
__device__ __forceinline__ float cross_axis(float vx, float vy, float vz, float4 b) {
  if (AXIS == 0) return vy * b.z - vz * b.y;
  if (AXIS == 1) return vz * b.x - vx * b.z;
  return vx * b.y - vy * b.x;
}

// Director proposal of chll_mod.f90:149-182: rotate n in its tangent plane by
// amplitude d at angle phi = 2*pi*u, then renormalise.  |nz| > 0.999 (FP64 in
// the reference) is exactly |nz| >= 0.999f for an FP32 nz.
// The angle is taken as psi = 2*pi*(u - 1/2) in [-pi, pi), where the hardware
// sine/cosine have absolute error <= 2^-21.4, and sin(phi) = -sin(psi),
// cos(phi) = -cos(psi); u - 1/2 is exact for a 24-bit uniform.
__device__ __forceinline__ void propose_director(float nx, float ny, float nz, float d, float u,
                                                 float& mx, float& my, float& mz) {
  float sn, cs;
  __sincosf(6.28318530717958647692f * (u - 0.5f), &sn, &cs);
  sn = -sn;
  cs = -cs;
  float x, y, z;
  if (fabsf(nz) >= 0.999f) {
    x = nx + d * cs;
    y = ny + d * sn;
    z = nz;
  } else {
    const float ru = rsqrtf(nx * nx + ny * ny);
    const float ux = -ny * ru, uy = nx * ru;
    float vx = -nz * nx, vy = -nz * ny, vz = nx * nx + ny * ny;
    const float rv = rsqrtf(vx * vx + vy * vy + vz * vz);
    vx *= rv;
    vy *= rv;
    vz *= rv;
    const float a = d * cs, bb = d * sn;
    x = nx + a * ux + bb * vx;
    y = ny + a * uy + bb * vy;
    z = nz + bb * vz;
  }
  const float r = rsqrtf(x * x + y * y + z * z);
  mx = x * r;
  my = y * r;
  mz = z * r;
}

// One bond's contribution to E(m) - E(n) for a director trial n -> m: the
// nematic part into dn, and (s + s_b)*(dot_m*x_m - dot_o*x_o) into the
// accumulator of its direction (+axis bonds carry sigma = -1, -axis +1).
template <int AXIS>
__device__ __forceinline__ void dir_bond(float nx, float ny, float nz, float mx, float my,
                                         float mz, float s, float4 b, float& dn, float& dc) {
  const float d_o = nx * b.x + ny * b.y + nz * b.z;
  const float d_m = mx * b.x + my * b.y + mz * b.z;
  const float x_o = cross_axis<AXIS>(nx, ny, nz, b);
  const float x_m = cross_axis<AXIS>(mx, my, mz, b);
  dn = fmaf(d_o, d_o, dn);
  dn = fmaf(-d_m, d_m, dn);
  dc = fmaf(s + b.w, fmaf(d_m, x_m, -d_o * x_o), dc);
}

// Energy difference of the director trial: eps*sum(dot_o^2 - dot_m^2) +
// K*sum(sigma*sfac*(dot_m*x_m - dot_o*x_o)), sfac = (s + s_b)/2.
__device__ __forceinline__ float director_dE(const float4& n, float mx, float my, float mz,
                                             const Nbrs& nb, const Coupling& cp) {
  float dn = 0.f, dplus = 0.f, dminus = 0.f;
  dir_bond<0>(n.x, n.y, n.z, mx, my, mz, n.w, nb.b[0], dn, dplus);
  dir_bond<0>(n.x, n.y, n.z, mx, my, mz, n.w, nb.b[1], dn, dminus);
  dir_bond<1>(n.x, n.y, n.z, mx, my, mz, n.w, nb.b[2], dn, dplus);
  dir_bond<1>(n.x, n.y, n.z, mx, my, mz, n.w, nb.b[3], dn, dminus);
  dir_bond<2>(n.x, n.y, n.z, mx, my, mz, n.w, nb.b[4], dn, dplus);
  dir_bond<2>(n.x, n.y, n.z, mx, my, mz, n.w, nb.b[5], dn, dminus);
  return fmaf(cp.eps, dn, 0.5f * cp.K * (dminus - dplus));
}

template <int AXIS, int SIGMA>
__device__ __forceinline__ float chiral_bond(const float4& n, float4 b) {
  const float dt = n.x * b.x + n.y * b.y + n.z * b.z;
  return (float)SIGMA * dt * cross_axis<AXIS>(n.x, n.y, n.z, b);
}

// Energy difference of the chirality flip s -> -s (chll_mod.f90:226-233):
// the nematic terms cancel and (snew + s_b)/2 - (s + s_b)/2 = -s, so
//   dE = -s*K*sum(sigma*dot*cross) + 2*g*s.
__device__ __forceinline__ float spin_dE(const float4& n, const Nbrs& nb, const Coupling& cp) {
  float c = chiral_bond<0, -1>(n, nb.b[0]);
  c += chiral_bond<0, +1>(n, nb.b[1]);
  c += chiral_bond<1, -1>(n, nb.b[2]);
  c += chiral_bond<1, +1>(n, nb.b[3]);
  c += chiral_bond<2, -1>(n, nb.b[4]);
  c += chiral_bond<2, +1>(n, nb.b[5]);
  return n.w * fmaf(-cp.K, c, 2.0f * cp.g);
}

// Metropolis rule of chll_mod.f90:188-200: accept if dE < 0, else if
// u <= exp(-dE/kT).  At kT = 0 this gives exp(-inf) = 0 for dE > 0 and NaN
// (reject) for dE = 0, as the reference's division does.
__device__ __forceinline__ bool metropolis(float dE, float u, float inv_kT) {
  return (dE < 0.f) || (u <= __expf(-dE * inv_kT));
}

}  // namespace chll
