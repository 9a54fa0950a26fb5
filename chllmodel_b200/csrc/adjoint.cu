// Adjoint of the lattice energy: dE/dn_i for every director and dE/d(eps,K,h).
//
// Total energy (each bond once, the sweep's boundary):
//   E = sum_<ij>, j=i+e_a [ eps*(1 - c^2) - K*c*X*sbar ] - h*sum_i s_i,
//   c = n_i.n_j,  X = (n_i x n_j).e_a = n_i.(n_j x e_a),  sbar = (s_i+s_j)/2.
// This is the bond sum behind the reference's local energy (chll_mod.f90:
// 363-412): the local energy of a site is the sum of the bonds touching it.
// Per bond, seen from site i with neighbour b in direction sigma*e_a
// (sigma = -1 forward, +1 backward):
//   dE_b/dn_i = -2*eps*c*b + sigma*K*sbar*(X*b + c*(b x e_a)),
// with c = n_i.b and X = (n_i x b).e_a.  The director gradient is optionally
// projected on the tangent plane, g - (g.n) n/|n|^2 (the torque direction).
// Coupling derivatives (FP64): dE/deps = sum(1-c^2), dE/dK = -sum(c*X*sbar),
// dE/dh = -sum(s), together with E itself.
#include <algorithm>
#include <atomic>

#include "chll_common.cuh"
#include "moments.cuh"
#include "sweep.cuh"
#include "sweep_unit.cuh"

namespace chll {

namespace {

constexpr int kGradThreads = 256;

// Slot t of colour `col` -> lattice site (i, j, k), with 32-bit divisions by
// multiplication (a colour holds < 2^31 slots); false for a padding slot.
__device__ __forceinline__ bool slot_site(const LatticeView& L, const MomentGeom& M, int col,
                                          uint32_t t, int& i, int& j, int& k) {
  const uint32_t r = M.by_hx.div(t);
  const int h = (int)(t - r * (uint32_t)L.hx);
  k = (int)M.by_nj.div(r);
  j = (int)(r - (uint32_t)k * (uint32_t)L.nj);
  i = 2 * h + ((col + j + k) & 1);
  return i < L.ni;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Adds one bond's dE/dn_i to (gx,gy,gz).  AXIS: 0,1,2; sigma = -1 forward.
template <int AXIS>
__device__ __forceinline__ void bond_grad(const float4& n, const float4& b, float sigma,
                                          const Coupling& cp, float& gx, float& gy, float& gz) {
  const float c = n.x * b.x + n.y * b.y + n.z * b.z;
  float X, ex, ey, ez;  // X = (n x b).e_a; (ex,ey,ez) = b x e_a
  if (AXIS == 0) {
    X = n.y * b.z - n.z * b.y;
    ex = 0.f; ey = b.z; ez = -b.y;
  } else if (AXIS == 1) {
    X = n.z * b.x - n.x * b.z;
    ex = -b.z; ey = 0.f; ez = b.x;
  } else {
    X = n.x * b.y - n.y * b.x;
    ex = b.y; ey = -b.x; ez = 0.f;
  }
  const float sbar = 0.5f * (n.w + b.w);
  const float a = -2.f * cp.eps * c;
  const float w = sigma * cp.K * sbar;
  gx += a * b.x + w * (X * b.x + c * ex);
  gy += a * b.y + w * (X * b.y + c * ey);
  gz += a * b.z + w * (X * b.z + c * ez);
}

// dE/dn of one site from its six neighbours (+x, -x, +y, -y, +z, -z; zero
// past an open boundary), optionally projected on the tangent plane.
__device__ __forceinline__ float4 site_grad(const float4& n, const float4& bxp, const float4& bxm,
                                            const float4& byp, const float4& bym,
                                            const float4& bzp, const float4& bzm,
                                            const Coupling& cp, int project) {
  float gx = 0.f, gy = 0.f, gz = 0.f;
  bond_grad<0>(n, bxp, -1.f, cp, gx, gy, gz);
  bond_grad<0>(n, bxm, +1.f, cp, gx, gy, gz);
  bond_grad<1>(n, byp, -1.f, cp, gx, gy, gz);
  bond_grad<1>(n, bym, +1.f, cp, gx, gy, gz);
  bond_grad<2>(n, bzp, -1.f, cp, gx, gy, gz);
  bond_grad<2>(n, bzm, +1.f, cp, gx, gy, gz);
  if (project) {
    const float nn = n.x * n.x + n.y * n.y + n.z * n.z;
    const float gn = (gx * n.x + gy * n.y + gz * n.z) / nn;
    gx -= gn * n.x;
    gy -= gn * n.y;
    gz -= gn * n.z;
  }
  return make_float4(gx, gy, gz, 0.f);
}

// FP64 sums of one site: its forward bonds (+x, +y, +z, each bond of the
// lattice once; hx, hy, hz = present) and its field term.
__device__ __forceinline__ void site_sums(const float4& n, const float4& bx, const float4& by,
                                          const float4& bz, bool hx, bool hy, bool hz,
                                          const CouplingD& cd, double acc[4]) {
  const double nx = n.x, ny = n.y, nz = n.z, s = n.w;
  const float4 fw[3] = {bx, by, bz};
  const bool hf[3] = {hx, hy, hz};
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    if (!hf[a]) continue;
    const float4 b = fw[a];
    const double c = nx * b.x + ny * b.y + nz * b.z;
    const double X = (a == 0) ? ny * b.z - nz * b.y
                   : (a == 1) ? nz * b.x - nx * b.z
                              : nx * b.y - ny * b.x;
    const double sbar = 0.5 * (s + (double)b.w);
    const double nem = 1.0 - c * c;
    const double chi = -c * X * sbar;
    acc[0] += cd.eps * nem + cd.K * chi;
    acc[1] += nem;
    acc[2] += chi;
  }
  acc[0] -= cd.g * s;
  acc[3] -= s;
}

// Block sums of the four FP64 accumulators into partials; the last block to
// finish (ticket) adds the partials into out4 with all its threads (blocks
// strided over the threads, then warp shuffles and the warps in order: a
// fixed order for a given grid, so the sums are reproducible).
__device__ __forceinline__ void finish_sums(const double acc[4], double* __restrict__ partials,
                                            unsigned int* __restrict__ ticket,
                                            double* __restrict__ out4) {
  __shared__ double s_part[kGradThreads / 32][4];
  __shared__ bool s_last;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int m = 0; m < 4; ++m) {
    const double v = warp_sum(acc[m]);
    if (lane == 0) s_part[warp][m] = v;
  }
  __syncthreads();
  if (threadIdx.x < 4) {
    double v = 0.0;
    for (int w = 0; w < kGradThreads / 32; ++w) v += s_part[w][threadIdx.x];
    partials[(size_t)blockIdx.x * 4 + threadIdx.x] = v;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_last = (atomicAdd(ticket, 1u) == gridDim.x - 1);
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  double v[4] = {0.0, 0.0, 0.0, 0.0};
  for (unsigned int b = threadIdx.x; b < gridDim.x; b += blockDim.x) {
#pragma unroll
    for (int m = 0; m < 4; ++m) v[m] += __ldcg(&partials[(size_t)b * 4 + m]);  // L2
  }
#pragma unroll
  for (int m = 0; m < 4; ++m) {
    const double w = warp_sum(v[m]);
    if (lane == 0) s_part[warp][m] = w;
  }
  __syncthreads();
  if (threadIdx.x < 4) {
    double t = 0.0;
    for (int w = 0; w < kGradThreads / 32; ++w) t += s_part[w][threadIdx.x];
    out4[threadIdx.x] = t;
  }
  if (threadIdx.x == 0) *ticket = 0;
}

// One slot per thread: colour arrays that are 16-byte aligned but not 32
// (caller-provided arrays of chll_energy_grad_noalloc; every slot is read as
// one float4).
__global__ void __launch_bounds__(kGradThreads)
    energy_grad_site_kernel(LatticeView L, MomentGeom M, CouplingD cd, float4* __restrict__ grad_rb,
                       int project,
                       double* __restrict__ partials, unsigned int* __restrict__ ticket,
                       double* __restrict__ out4) {
  Coupling cp;  // FP32 couplings of the per-site gradient
  cp.eps = (float)cd.eps;
  cp.K = (float)cd.K;
  cp.g = (float)cd.g;
  cp.inv_kT = 0.f;
  double acc[4] = {0.0, 0.0, 0.0, 0.0};  // E, dE/deps, dE/dK, dE/dh
  const uint64_t total = 2 * (uint64_t)M.per_colour;
  const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < total;
       e += (uint64_t)gridDim.x * blockDim.x) {
    const int col = e >= M.per_colour;
    const uint32_t t = (uint32_t)e - (col ? M.per_colour : 0u);
    int i, j, k;
    if (!slot_site(L, M, col, t, i, j, k)) {
      if (grad_rb) grad_rb[e] = zero;
      continue;
    }
    const float4 n = colour_array(L, col)[t];
    int ip = i + 1, im = i - 1, jp = j + 1, jm = j - 1, kp = k + 1, km = k - 1;
    bool hip = ip < L.ni, him = im >= 0, hjp = jp < L.nj, hjm = jm >= 0, hkp = kp < L.nk,
         hkm = km >= 0;
    if (L.periodic) {
      if (!hip) ip = 0;
      if (!him) im = L.ni - 1;
      if (!hjp) jp = 0;
      if (!hjm) jm = L.nj - 1;
      if (!hkp) kp = 0;
      if (!hkm) km = L.nk - 1;
      hip = him = hjp = hjm = hkp = hkm = true;
    }
    const float4 bxp = hip ? site_at(L, ip, j, k) : zero;
    const float4 bxm = him ? site_at(L, im, j, k) : zero;
    const float4 byp = hjp ? site_at(L, i, jp, k) : zero;
    const float4 bym = hjm ? site_at(L, i, jm, k) : zero;
    const float4 bzp = hkp ? site_at(L, i, j, kp) : zero;
    const float4 bzm = hkm ? site_at(L, i, j, km) : zero;

    if (grad_rb) grad_rb[e] = site_grad(n, bxp, bxm, byp, bym, bzp, bzm, cp, project);
    site_sums(n, bxp, byp, bzp, hip, hjp, hkp, cd, acc);
  }

  finish_sums(acc, partials, ticket, out4);
}

// Two sites per thread on the sweep's unit gather (256-bit accesses): colour
// 0's units, then colour 1's.  Needs 32-byte aligned colour and gradient
// arrays (unit_view_aligned).
template <int C, bool PERIODIC>
__device__ __forceinline__ void grad_units(const LatticeView& L, const SweepGeom& G,
                                           const Coupling& cp, const CouplingD& cd,
                                           float4* __restrict__ grad_c, int project,
                                           double acc[4]) {
  const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
  for (uint32_t g = blockIdx.x * kGradThreads + threadIdx.x; g < G.units;
       g += gridDim.x * kGradThreads) {
    UnitNbhd U;
    gather_unit<C, PERIODIC, PERIODIC>(L, G, g, U);
    float4 g0 = zero, g1 = zero;
    if (U.v0) {
      if (grad_c)
        g0 = site_grad(U.n0, U.nb0.b[0], U.nb0.b[1], U.nb0.b[2], U.nb0.b[3], U.nb0.b[4],
                       U.nb0.b[5], cp, project);
      site_sums(U.n0, U.nb0.b[0], U.nb0.b[2], U.nb0.b[4], U.fx0, U.fy, U.fz, cd, acc);
    }
    if (U.v1) {
      if (grad_c)
        g1 = site_grad(U.n1, U.nb1.b[0], U.nb1.b[1], U.nb1.b[2], U.nb1.b[3], U.nb1.b[4],
                       U.nb1.b[5], cp, project);
      site_sums(U.n1, U.nb1.b[0], U.nb1.b[2], U.nb1.b[4], U.fx1, U.fy, U.fz, cd, acc);
    }
    if (grad_c) st_unit(grad_c + (U.cen - L.col[C]), g0, g1);
  }
}

template <bool PERIODIC>
__global__ void __launch_bounds__(kGradThreads)
    energy_grad_unit_kernel(LatticeView L, SweepGeom G, CouplingD cd,
                            float4* __restrict__ grad_rb, uint32_t per_colour, int project,
                            double* __restrict__ partials, unsigned int* __restrict__ ticket,
                            double* __restrict__ out4) {
  Coupling cp;  // FP32 couplings of the per-site gradient
  cp.eps = (float)cd.eps;
  cp.K = (float)cd.K;
  cp.g = (float)cd.g;
  cp.inv_kT = 0.f;
  double acc[4] = {0.0, 0.0, 0.0, 0.0};  // E, dE/deps, dE/dK, dE/dh
  grad_units<0, PERIODIC>(L, G, cp, cd, grad_rb, project, acc);
  grad_units<1, PERIODIC>(L, G, cp, cd, grad_rb ? grad_rb + per_colour : nullptr, project, acc);
  finish_sums(acc, partials, ticket, out4);
}

// One site of a zero-temperature gradient quench: n moves against its
// tangent-projected energy gradient, n <- normalise(n - eta (I - n n^T) dE/dn),
// with the neighbours nb (+x, -x, +y, -y, +z, -z) held fixed.
__device__ __forceinline__ float4 quench_site(float4 n, const Nbrs& nb, const Coupling& cp,
                                              float eta) {
  float gx = 0.f, gy = 0.f, gz = 0.f;
  bond_grad<0>(n, nb.b[0], -1.f, cp, gx, gy, gz);
  bond_grad<0>(n, nb.b[1], +1.f, cp, gx, gy, gz);
  bond_grad<1>(n, nb.b[2], -1.f, cp, gx, gy, gz);
  bond_grad<1>(n, nb.b[3], +1.f, cp, gx, gy, gz);
  bond_grad<2>(n, nb.b[4], -1.f, cp, gx, gy, gz);
  bond_grad<2>(n, nb.b[5], +1.f, cp, gx, gy, gz);
  const float nn = n.x * n.x + n.y * n.y + n.z * n.z;
  const float gn = (gx * n.x + gy * n.y + gz * n.z) / nn;
  const float x = n.x - eta * (gx - gn * n.x);
  const float y = n.y - eta * (gy - gn * n.y);
  const float z = n.z - eta * (gz - gn * n.z);
  const float rn = rsqrtf(x * x + y * y + z * z);
  n.x = x * rn;
  n.y = y * rn;
  n.z = z * rn;
  return n;
}

// One colour of the quench: every site of colour C moves with the other
// colour fixed, so the two colours alternate like the Metropolis half-sweeps.
// A thread takes the sweep's unit of two same-colour sites (gather_unit,
// 256-bit accesses).  Chiralities are not changed.
template <int C, bool PERIODIC>
__global__ void __launch_bounds__(kGradThreads) quench_pass_kernel(LatticeView L, SweepGeom G,
                                                                   Coupling cp, float eta) {
  for (uint32_t g = blockIdx.x * kGradThreads + threadIdx.x; g < G.units;
       g += gridDim.x * kGradThreads) {
    UnitNbhd U;
    gather_unit<C, PERIODIC, PERIODIC>(L, G, g, U);
    if (U.v0) U.n0 = quench_site(U.n0, U.nb0, cp, eta);
    if (U.v1) U.n1 = quench_site(U.n1, U.nb1, cp, eta);
    st_unit(U.cen, U.n0, U.n1);
  }
}

// CTAs of `kernel` (kGradThreads threads) resident on the current device, one
// wave of a grid-stride launch; cached per device ordinal (threads that race
// on the first query store the same value).
template <class Kernel>
int resident_ctas(Kernel kernel, std::atomic<int> cache[16]) {
  int dev = 0;
  cudaGetDevice(&dev);
  std::atomic<int>& slot = cache[dev & 15];
  int res = slot.load(std::memory_order_relaxed);
  if (res == 0) {
    int sms = 0, per_sm = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kGradThreads, 0);
    res = std::max(1, sms) * std::max(1, per_sm);
    slot.store(res, std::memory_order_relaxed);
  }
  return res;
}

}  // namespace

int energy_grad_max_blocks() { return kGradMaxBlocks; }

void launch_quench_pass(const LatticeView& L, const CouplingD& cd, float eta, int colour,
                        cudaStream_t stream) {
  Coupling cp;
  cp.eps = (float)cd.eps;
  cp.K = (float)cd.K;
  cp.g = (float)cd.g;
  cp.inv_kT = 0.f;
  static std::atomic<int> resident[16];
  const int res = resident_ctas(quench_pass_kernel<0, true>, resident);
  const SweepGeom G = make_geom(L);
  size_t blocks = ((size_t)G.units + kGradThreads - 1) / kGradThreads;
  if (blocks > (size_t)res) blocks = (size_t)res;
  if (blocks == 0) blocks = 1;
  const unsigned int nb = (unsigned int)blocks;
  if (L.periodic) {
    if (colour == 0) quench_pass_kernel<0, true><<<nb, kGradThreads, 0, stream>>>(L, G, cp, eta);
    else quench_pass_kernel<1, true><<<nb, kGradThreads, 0, stream>>>(L, G, cp, eta);
  } else {
    if (colour == 0) quench_pass_kernel<0, false><<<nb, kGradThreads, 0, stream>>>(L, G, cp, eta);
    else quench_pass_kernel<1, false><<<nb, kGradThreads, 0, stream>>>(L, G, cp, eta);
  }
}

void launch_energy_grad(const LatticeView& L, const CouplingD& cp, float4* grad_rb, int project,
                        double* partials, unsigned int* ticket, double* out4,
                        cudaStream_t stream) {
  const size_t total = 2 * (size_t)L.nk * L.nj * L.hx;
  const bool units = unit_view_aligned(L) && ((uintptr_t)grad_rb % 32) == 0;
  static std::atomic<int> resident[16];
  const int res = units ? resident_ctas(energy_grad_unit_kernel<true>, resident) : kGradMaxBlocks;
  size_t blocks = ((units ? total / 4 : total) + kGradThreads - 1) / kGradThreads;
  if (blocks > (size_t)std::min(res, kGradMaxBlocks)) blocks = std::min(res, kGradMaxBlocks);
  if (blocks == 0) blocks = 1;
  const unsigned int nb = (unsigned int)blocks;
  if (units) {
    const SweepGeom G = make_geom(L);
    const uint32_t pc = (uint32_t)(total / 2);
    if (L.periodic)
      energy_grad_unit_kernel<true><<<nb, kGradThreads, 0, stream>>>(L, G, cp, grad_rb, pc, project,
                                                                     partials, ticket, out4);
    else
      energy_grad_unit_kernel<false><<<nb, kGradThreads, 0, stream>>>(
          L, G, cp, grad_rb, pc, project, partials, ticket, out4);
  } else {
    energy_grad_site_kernel<<<nb, kGradThreads, 0, stream>>>(L, make_moment_geom(L), cp, grad_rb,
                                                             project, partials, ticket, out4);
  }
}

}  // namespace chll
