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

// 1/sqrt(x) by the hardware approximation (PTX rsqrt.approx, subnormals
// flushed).  Its two uses below only see normal inputs (rho^2 >= 1 - 0.999^2
// away from the poles, |m|^2 near 1), so flushing never applies.  Measured
// against rsqrtf: the chains of three test lattices came out bit-identical
// and the 480^3 passes 5% faster.
__device__ __forceinline__ float rsqrt_approx(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// Director proposal of chll_mod.f90:149-182: rotate n in its tangent plane by
// amplitude d at angle phi = 2*pi*u, then renormalise.  |nz| > 0.999 (FP64 in
// the reference) is exactly |nz| >= 0.999f for an FP32 nz.
// The angle is taken as psi = 2*pi*(u - 1/2) in [-pi, pi), where the hardware
// sine/cosine have absolute error <= 2^-21.4, and sin(phi) = -sin(psi),
// cos(phi) = -cos(psi).  uc = u - 1/2 (UnitRandoms.ang) is exact for the
// 16-bit angle uniform.
__device__ __forceinline__ void propose_director(float nx, float ny, float nz, float d, float uc,
                                                 float& mx, float& my, float& mz) {
  float sn, cs;
  __sincosf(__fmul_rn(6.28318530717958647692f, uc), &sn, &cs);
  const float a = -__fmul_rn(d, cs), bb = -__fmul_rn(d, sn);  // d cos(phi), d sin(phi)
  float x, y, z;
  if (fabsf(nz) >= 0.999f) {
    x = __fadd_rn(nx, a);
    y = __fadd_rn(ny, bb);
    z = nz;
  } else {
    // u = (-ny, nx, 0)/rho and v = (-nz nx, -nz ny, rho^2)/rho: for a unit
    // director |v| = rho |n| = rho, so one 1/rho scales both
    const float rho2 = fmaf(ny, ny, __fmul_rn(nx, nx));
    const float ru = rsqrt_approx(rho2);
    const float ar = __fmul_rn(a, ru), br = __fmul_rn(bb, ru);
    const float bnz = __fmul_rn(br, nz);
    x = fmaf(-bnz, nx, fmaf(-ar, ny, nx));
    y = fmaf(-bnz, ny, fmaf(ar, nx, ny));
    z = fmaf(br, rho2, nz);
  }
  const float r = rsqrt_approx(fmaf(z, z, fmaf(y, y, __fmul_rn(x, x))));
  mx = __fmul_rn(x, r);
  my = __fmul_rn(y, r);
  mz = __fmul_rn(z, r);
}

// Every product and sum below is an explicit fmaf / __fmul_rn / __fadd_rn, so
// the compiler cannot contract it differently in different kernels: the
// plain, fused, staged and batched sweeps compute identical bits.

// v . b
__device__ __forceinline__ float dot3(float vx, float vy, float vz, float4 b) {
  return fmaf(vz, b.z, fmaf(vy, b.y, __fmul_rn(vx, b.x)));
}

// (v x b) . e_axis for axis 0,1,2 (chll_mod.f90:373,387,401).
template <int AXIS>
__device__ __forceinline__ float cross_axis(float vx, float vy, float vz, float4 b) {
  if (AXIS == 0) return fmaf(vy, b.z, -__fmul_rn(vz, b.y));
  if (AXIS == 1) return fmaf(vz, b.x, -__fmul_rn(vx, b.z));
  return fmaf(vx, b.y, -__fmul_rn(vy, b.x));
}

// Bond sums of one director v over its six neighbours b, with
// p_b = (v.b) * ((v x b).e_b) and sigma_b = -1 for +axis, +1 for -axis:
//   q = sum (v.b)^2,   c = sum sigma_b p_b,   w = sum sigma_b s_b p_b.
// The local energy (chll_mod.f90:363-412) is then
//   E(v, s) = sum_b eps (1 - (v.b)^2) + (K/2) (s c + w) - g s,
// so a director trial and a chirality flip both follow from q, c, w of the
// current and the trial director.
struct BondSums {
  float q, c, w;
};

template <int AXIS, int SIGMA>
__device__ __forceinline__ void bond_acc(float vx, float vy, float vz, float4 b, BondSums& S) {
  const float dt = dot3(vx, vy, vz, b);
  const float p = __fmul_rn(dt, cross_axis<AXIS>(vx, vy, vz, b));
  S.q = fmaf(dt, dt, S.q);
  S.c = SIGMA > 0 ? __fadd_rn(S.c, p) : __fsub_rn(S.c, p);
  S.w = fmaf(SIGMA > 0 ? b.w : -b.w, p, S.w);
}

__device__ __forceinline__ BondSums bond_sums(float vx, float vy, float vz, const Nbrs& nb) {
  BondSums S = {0.f, 0.f, 0.f};
  bond_acc<0, -1>(vx, vy, vz, nb.b[0], S);
  bond_acc<0, +1>(vx, vy, vz, nb.b[1], S);
  bond_acc<1, -1>(vx, vy, vz, nb.b[2], S);
  bond_acc<1, +1>(vx, vy, vz, nb.b[3], S);
  bond_acc<2, -1>(vx, vy, vz, nb.b[4], S);
  bond_acc<2, +1>(vx, vy, vz, nb.b[5], S);
  return S;
}

// The bond sums of two directors against the same six neighbours as FP32x2
// pairs (sm_100 packed FP32 fma/mul): lane x the current director, lane y the
// trial.  Each lane performs exactly the scalar bond_acc operations in the
// same order, so the sums are bit-identical to two bond_sums calls, in about
// half the FP32 instructions (measured on the 480^3 passes: 31% fewer FMA-pipe
// instructions, 15% fewer in all; the batched grid 11% faster).
struct BondSums2 {
  float2 q, c, w;
};

__device__ __forceinline__ float2 bcast(float v) { return make_float2(v, v); }

template <int AXIS, int SIGMA>
__device__ __forceinline__ void bond_acc2(float2 vx, float2 vy, float2 vz, float4 b,
                                          BondSums2& S) {
  const float2 bx = bcast(b.x), by = bcast(b.y), bz = bcast(b.z);
  const float2 dt = __ffma2_rn(vz, bz, __ffma2_rn(vy, by, __fmul2_rn(vx, bx)));
  float2 cr;
  if (AXIS == 0) cr = __ffma2_rn(vy, bz, __fmul2_rn(vz, bcast(-b.y)));
  else if (AXIS == 1) cr = __ffma2_rn(vz, bx, __fmul2_rn(vx, bcast(-b.z)));
  else cr = __ffma2_rn(vx, by, __fmul2_rn(vy, bcast(-b.x)));
  const float2 p = __fmul2_rn(dt, cr);
  S.q = __ffma2_rn(dt, dt, S.q);
  S.c = __ffma2_rn(p, bcast(SIGMA > 0 ? 1.f : -1.f), S.c);
  S.w = __ffma2_rn(bcast(SIGMA > 0 ? b.w : -b.w), p, S.w);
}

__device__ __forceinline__ void bond_sums2(float nx, float ny, float nz, float mx, float my,
                                           float mz, const Nbrs& nb, BondSums& o, BondSums& m) {
  const float2 vx = make_float2(nx, mx), vy = make_float2(ny, my), vz = make_float2(nz, mz);
  BondSums2 S = {bcast(0.f), bcast(0.f), bcast(0.f)};
  bond_acc2<0, -1>(vx, vy, vz, nb.b[0], S);
  bond_acc2<0, +1>(vx, vy, vz, nb.b[1], S);
  bond_acc2<1, -1>(vx, vy, vz, nb.b[2], S);
  bond_acc2<1, +1>(vx, vy, vz, nb.b[3], S);
  bond_acc2<2, -1>(vx, vy, vz, nb.b[4], S);
  bond_acc2<2, +1>(vx, vy, vz, nb.b[5], S);
  o = {S.q.x, S.c.x, S.w.x};
  m = {S.q.y, S.c.y, S.w.y};
}

// E(m, s) - E(n, s) = eps (q_n - q_m) + (K/2) (s (c_m - c_n) + (w_m - w_n)).
__device__ __forceinline__ float director_dE(const BondSums& o, const BondSums& m, float s,
                                             const Coupling& cp) {
  const float chi = fmaf(s, __fsub_rn(m.c, o.c), __fsub_rn(m.w, o.w));
  return fmaf(cp.eps, __fsub_rn(o.q, m.q), __fmul_rn(__fmul_rn(0.5f, cp.K), chi));
}

// E(n, -s) - E(n, s) = s (2 g - K c) (chll_mod.f90:226-233): the flip does not
// depend on the neighbours' chiralities, only on c of the current director.
__device__ __forceinline__ float flip_dE(float c, float s, const Coupling& cp) {
  return __fmul_rn(s, fmaf(-cp.K, c, __fmul_rn(2.0f, cp.g)));
}

// 2^x by the hardware approximation (PTX ex2.approx, subnormals flushed).
__device__ __forceinline__ float ex2_approx(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// Metropolis rule of chll_mod.f90:188-200: accept if dE < 0, else if
// u <= exp(-dE/kT), evaluated as 2^(dE c) with c = -log2(e)/kT (the identity
// exp(x) = 2^(x log2 e); c is the same for every trial of a launch, so the
// compiler computes it once).  At kT = 0, c = -inf gives 2^-inf = 0 for
// dE > 0 and NaN (reject) for dE = 0, as the reference's division does.
// Flushing subnormals changes nothing: the smallest nonzero uniform is 2^-24.
__device__ __forceinline__ bool metropolis(float dE, float u, float inv_kT) {
  const float c = __fmul_rn(-inv_kT, 1.4426950408889634f);  // -log2(e)/kT
  return (dE < 0.f) || (u <= ex2_approx(__fmul_rn(dE, c)));
}

// Both sites of unit g of colour C (sites present: v0, v1), with the block's
// one random call for this pass (chll_common.cuh: {g, step, replica, C}, or
// step + 1 for a pass of colour-0 flips alone, the four half-sweep form's
// flip pass).  Trials in chain order: the flip left over from the previous
// sweep, the director trial, this sweep's flip.  The bond sums of the
// current director serve the flip and the director trial; after an accepted
// trial those of the trial director serve the second flip, exactly as a
// separate flip pass would recompute them.  The two sites' trials are written
// side by side and only their acceptance depends on v0, v1, so the two
// independent chains interleave; a missing (padding) site's arithmetic is
// discarded.
template <int C, bool FLIP_BEFORE, bool DIR, bool FLIP_AFTER, class KEY>
__device__ __forceinline__ void unit_trials(float4& n0, float4& n1, const Nbrs& nb0,
                                            const Nbrs& nb1, bool v0, bool v1, uint32_t g,
                                            uint32_t step, float d, const Coupling& cp,
                                            const KEY& key, uint32_t replica,
                                            unsigned int& nacc, unsigned int& nflip) {
  constexpr bool kNextStep = FLIP_AFTER && !DIR && C == 0;
  const UnitRandoms u = unit_randoms(
      philox4x32_10({{g, kNextStep ? step + 1u : step, replica, (uint32_t)C}}, key));
  // The trial directors depend only on n's direction, which the flips before
  // them leave alone, so both bond sums of a site come from one paired pass.
  float mx0, my0, mz0, mx1, my1, mz1;
  BondSums o0, o1, m0, m1;
  if (DIR) {
    propose_director(n0.x, n0.y, n0.z, d, u.ang[0], mx0, my0, mz0);
    propose_director(n1.x, n1.y, n1.z, d, u.ang[1], mx1, my1, mz1);
    bond_sums2(n0.x, n0.y, n0.z, mx0, my0, mz0, nb0, o0, m0);
    bond_sums2(n1.x, n1.y, n1.z, mx1, my1, mz1, nb1, o1, m1);
  } else {
    o0 = bond_sums(n0.x, n0.y, n0.z, nb0);
    o1 = bond_sums(n1.x, n1.y, n1.z, nb1);
  }
  if (FLIP_BEFORE) {
    const bool a0 = v0 && metropolis(flip_dE(o0.c, n0.w, cp), u.flip[0], cp.inv_kT);
    const bool a1 = v1 && metropolis(flip_dE(o1.c, n1.w, cp), u.flip[1], cp.inv_kT);
    if (a0) n0.w = -n0.w;
    if (a1) n1.w = -n1.w;
    nflip += (unsigned int)a0 + (unsigned int)a1;
  }
  if (DIR) {
    const bool a0 = v0 && metropolis(director_dE(o0, m0, n0.w, cp), u.acc[0], cp.inv_kT);
    const bool a1 = v1 && metropolis(director_dE(o1, m1, n1.w, cp), u.acc[1], cp.inv_kT);
    if (a0) {
      n0.x = mx0;
      n0.y = my0;
      n0.z = mz0;
      if (FLIP_AFTER) o0 = m0;
    }
    if (a1) {
      n1.x = mx1;
      n1.y = my1;
      n1.z = mz1;
      if (FLIP_AFTER) o1 = m1;
    }
    nacc += (unsigned int)a0 + (unsigned int)a1;
  }
  if (FLIP_AFTER) {
    const bool a0 = v0 && metropolis(flip_dE(o0.c, n0.w, cp), u.flip[0], cp.inv_kT);
    const bool a1 = v1 && metropolis(flip_dE(o1.c, n1.w, cp), u.flip[1], cp.inv_kT);
    if (a0) n0.w = -n0.w;
    if (a1) n1.w = -n1.w;
    nflip += (unsigned int)a0 + (unsigned int)a1;
  }
}

}  // namespace chll
