// FP64 observables of one red/black lattice and the reference measurement
// row.  The per-site moments are in moments.cuh.  Reduction: warp shuffle ->
// CTA partial in scratch -> the last CTA to finish sums the partials in a
// fixed order, so results are bit-reproducible.
#include "chll_common.cuh"
#include "moments.cuh"
#include "sweep.cuh"

namespace chll {

namespace {

constexpr int kObsThreads = 256;
constexpr int kObsMaxBlocks = 148 * 4;

__global__ void __launch_bounds__(kObsThreads)
    observables_kernel(LatticeView L, MomentGeom M, CouplingD cp,
                       const Control* __restrict__ ctl,
                       double* __restrict__ partials, unsigned int* __restrict__ ticket,
                       double* __restrict__ row, long long step) {
  double acc[kObsMoments];
#pragma unroll
  for (int m = 0; m < kObsMoments; ++m) acc[m] = 0.0;

  const uint64_t total = 2ull * M.per_colour;  // < 2^32
  for (uint64_t e = blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += gridDim.x * blockDim.x)
    site_moments<true>(L, M, cp, (uint32_t)e, acc);

  __shared__ double s_part[kObsThreads / 32][kObsMoments];
  __shared__ bool s_last;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int m = 0; m < kObsMoments; ++m) {
    const double v = warp_sum_d(acc[m]);
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
  // The partials summed by the whole CTA: thread t takes blocks t, t + 256,
  // ... (L2 reads, all in flight at once), then warp shuffles and the warps in
  // order -- a fixed order for a given grid, so the result is reproducible.
  double v[kObsMoments];
#pragma unroll
  for (int m = 0; m < kObsMoments; ++m) v[m] = 0.0;
  for (unsigned int b = threadIdx.x; b < gridDim.x; b += blockDim.x) {
#pragma unroll
    for (int m = 0; m < kObsMoments; ++m) v[m] += __ldcg(&partials[(size_t)b * kObsMoments + m]);
  }
#pragma unroll
  for (int m = 0; m < kObsMoments; ++m) {
    const double w = warp_sum_d(v[m]);
    if (lane == 0) s_part[warp][m] = w;
  }
  __syncthreads();
  __shared__ double s_tot[kObsMoments];
  if (threadIdx.x < kObsMoments) {
    double t = 0.0;
    for (int w = 0; w < kObsThreads / 32; ++w) t += s_part[w][threadIdx.x];
    s_tot[threadIdx.x] = t;
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

void launch_observables(const LatticeView& L, const MomentGeom& M, const CouplingD& cp,
                        const Control* ctl, double* partials, unsigned int* ticket, double* row,
                        long long step, cudaStream_t stream) {
  const size_t total = 2 * (size_t)L.nk * L.nj * L.hx;
  size_t blocks = (total + kObsThreads - 1) / kObsThreads;
  if (blocks > (size_t)kObsMaxBlocks) blocks = kObsMaxBlocks;
  if (blocks == 0) blocks = 1;
  observables_kernel<<<(unsigned int)blocks, kObsThreads, 0, stream>>>(L, M, cp, ctl, partials,
                                                                        ticket, row, step);
}

void launch_observables(const LatticeView& L, const CouplingD& cp, const Control* ctl,
                        double* partials, unsigned int* ticket, double* row, long long step,
                        cudaStream_t stream) {
  launch_observables(L, make_moment_geom(L), cp, ctl, partials, ticket, row, step, stream);
}

}  // namespace chll
