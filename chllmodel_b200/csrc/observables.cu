// FP64 observables of one red/black lattice and the reference measurement row.
//
// Per site (FP64 arithmetic on the FP32 state):
//   - total energy with the sweep's boundary (each bond once, +x,+y,+z);
//   - the reference etot() sum (chll_mod.f90:414-456): periodic in x and y,
//     open in z, and the +y dot product's x component read from the
//     diagonal neighbour (ip1,jp1,k) exactly as chll_mod.f90:438 does;
//   - sum of s and the six raw moments of n (x) n (Q-tensor).
// Reduction: warp shuffle -> CTA partial in scratch -> the last CTA to finish
// sums the partials in a fixed order, so results are bit-reproducible.
#include "chll_common.cuh"
#include "sweep.cuh"

namespace chll {

namespace {

constexpr int kObsThreads = 256;
constexpr int kObsMaxBlocks = 148 * 4;

__device__ __forceinline__ float4 site(const LatticeView& L, int i, int j, int k) {
  return L.col[(i + j + k) & 1][((size_t)k * L.nj + j) * L.hx + (i >> 1)];
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// eps*(1 - dot^2) - K*dot*cross*sfac for a forward bond.
__device__ __forceinline__ double fwd_bond(double eps, double K, double dot, double cross,
                                           double si, double sj) {
  return eps * (1.0 - dot * dot) - K * dot * cross * (0.5 * (si + sj));
}

__global__ void __launch_bounds__(kObsThreads)
    observables_kernel(LatticeView L, CouplingD cp, const Control* __restrict__ ctl,
                       double* __restrict__ partials, unsigned int* __restrict__ ticket,
                       double* __restrict__ row, long long step) {
  const double eps = cp.eps, K = cp.K, g = cp.g;
  double acc[kObsMoments];
#pragma unroll
  for (int m = 0; m < kObsMoments; ++m) acc[m] = 0.0;

  const size_t per_colour = (size_t)L.nk * L.nj * L.hx;
  const size_t total = 2 * per_colour;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total;
       e += (size_t)gridDim.x * blockDim.x) {
    const int c = e >= per_colour;
    const size_t t = e - (c ? per_colour : 0);
    const size_t r = t / (size_t)L.hx;
    const int h = (int)(t - r * L.hx);
    const int k = (int)(r / (size_t)L.nj);
    const int j = (int)(r - (size_t)k * L.nj);
    const int i = 2 * h + ((c + j + k) & 1);
    if (i >= L.ni) continue;
    const float4 nf = L.col[c][t];
    const double nx = nf.x, ny = nf.y, nz = nf.z, s = nf.w;
    const int ip = (i + 1 == L.ni) ? 0 : i + 1;
    const int jp = (j + 1 == L.nj) ? 0 : j + 1;
    const int kp = (k + 1 == L.nk) ? 0 : k + 1;
    const float4 X = site(L, ip, j, k);
    const float4 Y = site(L, i, jp, k);
    const float4 Z = site(L, i, j, kp);
    const float4 T = site(L, ip, jp, k);  // diagonal read of chll_mod.f90:438

    // +x bond
    const double dx = nx * X.x + ny * X.y + nz * X.z;
    const double cx = ny * X.z - nz * X.y;
    const double bx = fwd_bond(eps, K, dx, cx, s, X.w);
    // +y bond
    const double dy = nx * Y.x + ny * Y.y + nz * Y.z;
    const double cy = nz * Y.x - nx * Y.z;
    const double by = fwd_bond(eps, K, dy, cy, s, Y.w);
    // +z bond
    const double dz = nx * Z.x + ny * Z.y + nz * Z.z;
    const double cz = nx * Z.y - ny * Z.x;
    const double bz = fwd_bond(eps, K, dz, cz, s, Z.w);

    const bool has_xp = L.periodic || (i + 1 < L.ni);
    const bool has_yp = L.periodic || (j + 1 < L.nj);
    const bool has_zp = L.periodic || (k + 1 < L.nk);
    acc[0] += (has_xp ? bx : 0.0) + (has_yp ? by : 0.0) + (has_zp ? bz : 0.0) - g * s;

    // reference etot(): x and y periodic, z open, +y dot with the typo
    const double dyt = nx * (double)T.x + ny * Y.y + nz * Y.z;
    const double byt = fwd_bond(eps, K, dyt, cy, s, Y.w);
    acc[1] += bx + byt + ((k + 1 < L.nk) ? bz : 0.0) - g * s;

    acc[2] += s;
    acc[3] += nx * nx;
    acc[4] += ny * ny;
    acc[5] += nz * nz;
    acc[6] += nx * ny;
    acc[7] += nx * nz;
    acc[8] += ny * nz;
  }

  __shared__ double s_part[kObsThreads / 32][kObsMoments];
  __shared__ bool s_last;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int m = 0; m < kObsMoments; ++m) {
    const double v = warp_sum(acc[m]);
    if (lane == 0) s_part[warp][m] = v;
  }
  __syncthreads();
  if (threadIdx.x < kObsMoments) {
    double v = 0.0;
    for (int w = 0; w < kObsThreads / 32; ++w) v += s_part[w][threadIdx.x];
    partials[(size_t)blockIdx.x * kObsMoments + threadIdx.x] = v;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_last = (atomicAdd(ticket, 1u) == gridDim.x - 1);
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  __shared__ double s_tot[kObsMoments];
  if (threadIdx.x < kObsMoments) {
    double v = 0.0;
    for (unsigned int b = 0; b < gridDim.x; ++b) {
      v += *((volatile double*)&partials[(size_t)b * kObsMoments + threadIdx.x]);
    }
    s_tot[threadIdx.x] = v;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    *ticket = 0;
    const long long n = (long long)L.ni * L.nj * L.nk;
    const float n3 = (float)n;  // float(ni*nj*nk)
    // etot = e/float(N), a default REAL function result (chll_mod.f90:453)
    row[kRowEtotRef] = (double)(float)(s_tot[1] / (double)n3);
    // e_excess = sum(float(s))/float(N) in FP32 (chll_mod.f90:97)
    row[kRowEta] = (double)((float)s_tot[2] / n3);
    row[kRowPaccept] = ctl ? (double)ctl->paccept : 0.0;
    row[kRowFaccept] = ctl ? (double)ctl->faccept : 0.0;
    row[kRowD] = ctl ? ctl->d : 0.0;
    row[kRowEnergy] = s_tot[0];
    row[kRowSumS] = s_tot[2];
    row[kRowQxx] = s_tot[3];
    row[kRowQyy] = s_tot[4];
    row[kRowQzz] = s_tot[5];
    row[kRowQxy] = s_tot[6];
    row[kRowQxz] = s_tot[7];
    row[kRowQyz] = s_tot[8];
    row[kRowEtotRefSum] = s_tot[1];
    row[kRowStep] = (double)step;
    row[kRowNsites] = (double)n;
  }
}

}  // namespace

int observables_max_blocks() { return kObsMaxBlocks; }

void launch_observables(const LatticeView& L, const CouplingD& cp, const Control* ctl,
                        double* partials, unsigned int* ticket, double* row, long long step,
                        cudaStream_t stream) {
  const size_t total = 2 * (size_t)L.nk * L.nj * L.hx;
  size_t blocks = (total + kObsThreads - 1) / kObsThreads;
  if (blocks > (size_t)kObsMaxBlocks) blocks = kObsMaxBlocks;
  if (blocks == 0) blocks = 1;
  observables_kernel<<<(unsigned int)blocks, kObsThreads, 0, stream>>>(L, cp, ctl, partials,
                                                                         ticket, row, step);
}

}  // namespace chll
