// Pooled passes over many lattices (pooled.cuh).
//
// The batched persistent kernel (batched.cu) keeps every replica's CTA group
// in one launch and meets at software barriers in global memory; CTAs are
// whole units of work, so groups carry uneven loads.  Here one launch per
// fused pass covers the units of every replica: the pooled units are cut
// into equal contiguous blocks, one per CTA (a block meets one or two
// replicas), so every thread walks the same number of units within one, and
// the kernel boundary -- the next pass launched as a programmatic dependent
// -- replaces the barriers.  Each replica's counts close in the last CTA that
// touches it (a ticket in its control block), with the plain kernels' control
// update, and every unit is the plain kernels' unit_step: a replica follows
// the chain it follows alone, bit for bit.
#include <algorithm>

#include "pooled.cuh"
#include "sweep.cuh"

namespace chll {

namespace {

// The first lattice whose range [begin, begin + count) holds pooled index x
// (ranges ascending and contiguous).
template <class F>
__device__ __forceinline__ int find_entry(int nent, uint32_t x, F begin_of) {
  int lo = 0, hi = nent - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (begin_of(mid) <= x) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Units [lo, hi) of one lattice by this CTA's threads; accepted director
// trials and flips added to nacc, nflip.  Out of line, with the lattice's
// fields and Philox round keys copied into registers here, so that the
// pool's bookkeeping in the caller does not crowd the unit code.
template <int PHASE, bool PERIODIC, bool FULL>
__device__ __noinline__ void pool_units(const PoolEntry& E, uint32_t lo, uint32_t hi,
                                        uint32_t step, float d, unsigned int& nacc,
                                        unsigned int& nflip) {
  constexpr int C = PHASE == kFusedB ? 1 : 0;
  constexpr bool FLIP_BEFORE = PHASE == kFusedA || PHASE == kFusedF;
  constexpr bool DIR = PHASE != kFusedF;
  constexpr bool FLIP_AFTER = PHASE == kFusedB;
  const LatticeView L = E.L;
  const SweepGeom G = E.G;
  const Coupling cp = E.cp;
  const PhiloxKeys key = philox_keys(E.key0, E.key1);
  const uint32_t replica = E.replica;
  const uint32_t plane = (uint32_t)L.hx * (uint32_t)L.nj;
  const uint32_t per_colour = plane * (uint32_t)L.nk;
  unsigned int na = 0, nf = 0;
  for (uint32_t g = lo + threadIdx.x; g < hi; g += kPoolThreads) {
    if (g + kPoolThreads < hi) prefetch_unit<C>(L, g + kPoolThreads, plane, per_colour);
    unit_step<C, PERIODIC, PERIODIC, FLIP_BEFORE, DIR, FLIP_AFTER, FULL>(L, G, g, step, d, cp,
                                                                         key, replica, na, nf);
  }
  nacc = na;
  nflip = nf;
}

// One lattice's units [lo, hi) (pool_units), then the CTA's counts into its
// control block; the last of the lattice's CTAs runs the control update.
template <int PHASE, bool PERIODIC, bool FULL>
__device__ __forceinline__ void pool_segment(const PoolEntry& E, uint32_t lo, uint32_t hi,
                                             long long step, float d) {
  constexpr bool DIR = PHASE != kFusedF;
  unsigned int nacc = 0, nflip = 0;
  pool_units<PHASE, PERIODIC, FULL>(E, lo, hi, (uint32_t)step, d, nacc, nflip);
  __shared__ unsigned int s_cnt[2];
  __shared__ bool s_last;
  if (threadIdx.x < 2) s_cnt[threadIdx.x] = 0;
  __syncthreads();
  if (DIR) {
    const unsigned int w = __reduce_add_sync(0xffffffffu, nacc);
    if ((threadIdx.x & 31) == 0 && w) atomicAdd(&s_cnt[0], w);
  }
  if (PHASE != kFusedA0) {
    const unsigned int w = __reduce_add_sync(0xffffffffu, nflip);
    if ((threadIdx.x & 31) == 0 && w) atomicAdd(&s_cnt[1], w);
  }
  __syncthreads();
  Control* ctl = E.ctl;
  if (threadIdx.x == 0) {
    if (s_cnt[0]) atomicAdd(&ctl->nacc, (unsigned long long)s_cnt[0]);
    if (s_cnt[1]) atomicAdd(&ctl->nflip, (unsigned long long)s_cnt[1]);
    __threadfence();
    s_last = atomicAdd(&ctl->done, 1u) == (unsigned int)E.pass_ctas - 1;
  }
  __syncthreads();
  if (s_last && threadIdx.x == 0) {
    __threadfence();
    ctl->done = 0;
    fused_control_update<PHASE>(ctl, step);
  }
}

template <int PHASE>
__global__ void __launch_bounds__(kPoolThreads, 2)
    pool_pass_kernel(const PoolEntry* __restrict__ ents, int nent, uint32_t total,
                     uint32_t per_cta) {
  wait_prerequisite_grids();
  const uint32_t begin = blockIdx.x * per_cta;
  const uint32_t end = min(begin + per_cta, total);
  if (begin < end) {
    int e = find_entry(nent, begin, [&](int i) { return ents[i].unit_begin; });
    for (uint32_t u0 = begin; u0 < end; ++e) {
      const PoolEntry& E = ents[e];
      const uint32_t u1 = min(end, E.unit_begin + E.G.units);
      const long long step = E.ctl->step;
      const float d = (float)E.ctl->d;
      const uint32_t lo = u0 - E.unit_begin, hi = u1 - E.unit_begin;
      if (E.L.periodic) {
        if (E.full) pool_segment<PHASE, true, true>(E, lo, hi, step, d);
        else pool_segment<PHASE, true, false>(E, lo, hi, step, d);
      } else {
        if (E.full) pool_segment<PHASE, false, true>(E, lo, hi, step, d);
        else pool_segment<PHASE, false, false>(E, lo, hi, step, d);
      }
      u0 = u1;
    }
  }
  allow_dependent_grids();
}

// Slots [lo, hi) of one lattice's concatenated colour arrays: FP64 moments
// (moments.cuh, without the reference etot column), CTA-reduced into the
// lattice's partial slot for this CTA.
__device__ __forceinline__ void pool_moment_segment(const PoolEntry& E, uint32_t lo, uint32_t hi,
                                                    double* __restrict__ partials) {
  double m[kObsMoments];
#pragma unroll
  for (int t = 0; t < kObsMoments; ++t) m[t] = 0.0;
  for (uint32_t e = lo + threadIdx.x; e < hi; e += kPoolThreads)
    site_moments<false>(E.L, E.M, E.cd, e, m);
  __shared__ double s_m[kPoolThreads / 32][kObsMoments];
#pragma unroll
  for (int t = 0; t < kObsMoments; ++t) {
    const double v = warp_sum_d(m[t]);
    if ((threadIdx.x & 31) == 0) s_m[threadIdx.x >> 5][t] = v;
  }
  __syncthreads();
  if (threadIdx.x < kObsMoments) {
    double v = 0.0;
    for (int w = 0; w < kPoolThreads / 32; ++w) v += s_m[w][threadIdx.x];
    const int slot = E.partial_first + ((int)blockIdx.x - E.mom_cta_first);
    partials[(size_t)slot * kObsMoments + threadIdx.x] = v;
  }
  __syncthreads();
}

__global__ void __launch_bounds__(kPoolThreads)
    pool_moments_kernel(const PoolEntry* __restrict__ ents, int nent, uint32_t total,
                        uint32_t per_cta, double* __restrict__ partials) {
  const uint32_t begin = blockIdx.x * per_cta;
  const uint32_t end = min(begin + per_cta, total);
  if (begin >= end) return;
  int e = find_entry(nent, begin, [&](int i) { return ents[i].slot_begin; });
  for (uint32_t s0 = begin; s0 < end; ++e) {
    const PoolEntry& E = ents[e];
    const uint32_t s1 = min(end, E.slot_begin + 2 * E.M.per_colour);
    pool_moment_segment(E, s0 - E.slot_begin, s1 - E.slot_begin, partials);
    s0 = s1;
  }
}

// One CTA per lattice: its partials summed in CTA order (the same bits for
// the same launch shape), then e = E/N, eta = sum(s)/N and the nematic order
// S (largest eigenvalue of Q = (3/2)<n n^T> - I/2) accumulated.
__global__ void __launch_bounds__(32)
    pool_moments_finish_kernel(const PoolEntry* __restrict__ ents,
                               const double* __restrict__ partials) {
  const PoolEntry& E = ents[blockIdx.x];
  __shared__ double s_tot[kObsMoments];
  if (threadIdx.x < kObsMoments) {
    double v = 0.0;
    for (int c = 0; c < E.mom_ctas; ++c)
      v += partials[(size_t)(E.partial_first + c) * kObsMoments + threadIdx.x];
    s_tot[threadIdx.x] = v;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const double* tot = s_tot;
    const double n = (double)E.nsites;
    const double e = tot[0] / n, eta = tot[2] / n;
    const double qxx = 1.5 * tot[3] / n - 0.5, qyy = 1.5 * tot[4] / n - 0.5,
                 qzz = 1.5 * tot[5] / n - 0.5;
    const double qxy = 1.5 * tot[6] / n, qxz = 1.5 * tot[7] / n, qyz = 1.5 * tot[8] / n;
    const double S = sym3_max_eig(qxx, qyy, qzz, qxy, qxz, qyz);
    double* mom = E.mom;
    mom[0] += 1.0;
    mom[1] += e;
    mom[2] += e * e;
    mom[3] += eta;
    mom[4] += eta * eta;
    mom[5] += fabs(eta);
    mom[6] += S;
    mom[7] += S * S;
    E.last[0] = e;
    E.last[1] = eta;
    E.last[2] = S;
  }
}

using PoolPassKernel = void (*)(const PoolEntry*, int, uint32_t, uint32_t);
const PoolPassKernel kPoolPass[4] = {pool_pass_kernel<kFusedA0>, pool_pass_kernel<kFusedA>,
                                     pool_pass_kernel<kFusedB>, pool_pass_kernel<kFusedF>};

}  // namespace

int pool_pass_ctas() {
  int dev = 0, sms = 0, occ = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kPoolPass[2], kPoolThreads, 0);
  return std::max(1, sms) * std::max(1, occ);
}

void launch_pool_pass(const PoolEntry* d_entries, int nent, uint32_t total_units,
                      uint32_t units_per_cta, int grid, int phase, cudaStream_t stream) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3(kPoolThreads);
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, kPoolPass[phase & 3], d_entries, nent, total_units, units_per_cta);
}

void launch_pool_moments(const PoolEntry* d_entries, int nent, uint32_t total_slots,
                         uint32_t slots_per_cta, int grid, double* partials,
                         cudaStream_t stream) {
  pool_moments_kernel<<<grid, kPoolThreads, 0, stream>>>(d_entries, nent, total_slots,
                                                         slots_per_cta, partials);
  pool_moments_finish_kernel<<<nent, 32, 0, stream>>>(d_entries, partials);
}

}  // namespace chll
