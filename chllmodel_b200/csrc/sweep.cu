// Plain checkerboard half-sweep kernels on one red/black float4 lattice.
//
// One launch is one of the reference's four half-sweeps per step
// (chll_mod.f90:70,74,78,81): director trials on colour 0, on colour 1, then
// chirality flips on colour 0, on colour 1.
//
// Work unit: the two same-colour sites of one 4-site x-block (storage slots
// 2q, 2q+1 of a row).  A thread draws both sites' randoms from a single
// Philox call keyed on the block and stores the pair back with two coalesced
// 128-bit stores.  Units are numbered row-major (g = q + Q*row) and CTAs walk
// them grid-stride, so a launch is a few CTAs per SM that stay resident for
// the whole pass: accept counts stay in registers and the CTA-wide reduction,
// the one atomic and the completion ticket happen once per CTA.  All index
// arithmetic is 32-bit (per-colour arrays < 2^31 slots); the row and plane
// of a unit come from multiply-shift divisions.
//
// The last CTA to finish a pass (ticket counter) runs the step epilogue of
// chll_mod.f90:83-93 on the device: paccept and the d adaptation after the
// second director pass, faccept and the step increment after the second flip
// pass.
#include <mutex>

#include "chll_common.cuh"
#include "sweep.cuh"
#include "sweep_unit.cuh"

namespace chll {

namespace {

constexpr int kThreads = 256;

template <bool DIRECTOR, int C, bool PERIODIC>
__global__ void __launch_bounds__(kThreads, 3)
    sweep_pass_kernel(LatticeView L, SweepGeom G, Coupling cp, uint32_t key0, uint32_t key1,
                      uint32_t replica, Control* __restrict__ ctl) {
  const long long step = ctl->step;
  const float d = (float)ctl->d;
  unsigned int accepted = 0;
  for (uint32_t g = blockIdx.x * kThreads + threadIdx.x; g < G.units;
       g += gridDim.x * kThreads) {
    accepted += sweep_unit<DIRECTOR, C, PERIODIC>(L, G, g, (uint32_t)step, d, cp, key0, key1,
                                                  replica);
  }

  // CTA-aggregated accept count, then the last-CTA epilogue.
  __shared__ unsigned int s_cnt;
  __shared__ bool s_last;
  const int tid = threadIdx.x;
  if (tid == 0) s_cnt = 0;
  __syncthreads();
  const unsigned int wsum = __reduce_add_sync(0xffffffffu, accepted);
  if ((tid & 31) == 0 && wsum) atomicAdd(&s_cnt, wsum);
  __syncthreads();
  if (tid == 0) {
    unsigned long long* counter = DIRECTOR ? &ctl->nacc : &ctl->nflip;
    if (s_cnt) atomicAdd(counter, (unsigned long long)s_cnt);
    __threadfence();
    const unsigned int ticket = atomicAdd(&ctl->done, 1u);
    s_last = (ticket == gridDim.x - 1);
  }
  __syncthreads();
  if (s_last && tid == 0) {
    __threadfence();
    ctl->done = 0;
    if (C == 1) {
      const float n3 = (float)ctl->nsites;
      if (DIRECTOR) {
        const unsigned long long na = atomicAdd(&ctl->nacc, 0ull);
        // paccept = float(naccept)/float(n3), FP32 (chll_mod.f90:83)
        const float pa = (float)na / n3;
        ctl->paccept = pa;
        ctl->nacc_last = (long long)na;
        ctl->nacc = 0;
        if (step < ctl->adapt_until) ctl->d = adapt_d(ctl->d, pa);
      } else {
        const unsigned long long nf = atomicAdd(&ctl->nflip, 0ull);
        ctl->faccept = (float)nf / n3;  // chll_mod.f90:93
        ctl->nflip_last = (long long)nf;
        ctl->nflip = 0;
        ctl->step = step + 1;
      }
    }
  }
}

// Resident CTAs per SM of each pass kernel and the SM count, queried once
// per device (outside any stream capture; see sweep_prepare).
using PassKernel = void (*)(LatticeView, SweepGeom, Coupling, uint32_t, uint32_t, uint32_t,
                           Control*);

// [periodic][pass]
const PassKernel kKernels[2][4] = {
    {sweep_pass_kernel<true, 0, false>, sweep_pass_kernel<true, 1, false>,
     sweep_pass_kernel<false, 0, false>, sweep_pass_kernel<false, 1, false>},
    {sweep_pass_kernel<true, 0, true>, sweep_pass_kernel<true, 1, true>,
     sweep_pass_kernel<false, 0, true>, sweep_pass_kernel<false, 1, true>}};

struct DeviceShape {
  int sms = 0;
  int per_sm[2][4] = {{0, 0, 0, 0}, {0, 0, 0, 0}};
};
std::mutex g_shape_mutex;
DeviceShape g_shape[64];

int occupancy(PassKernel k) {
  int n = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k, kThreads, 0);
  return n > 0 ? n : 1;
}

const DeviceShape& device_shape() {
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) dev = 0;
  std::lock_guard<std::mutex> lk(g_shape_mutex);
  DeviceShape& s = g_shape[dev];
  if (s.sms == 0) {
    cudaDeviceGetAttribute(&s.sms, cudaDevAttrMultiProcessorCount, dev);
    if (s.sms <= 0) s.sms = 148;
    for (int per = 0; per < 2; ++per)
      for (int p = 0; p < 4; ++p) s.per_sm[per][p] = occupancy(kKernels[per][p]);
  }
  return s;
}

}  // namespace

void sweep_prepare() { (void)device_shape(); }

void launch_sweep_pass(const LatticeView& L, const Coupling& cp, uint32_t key0, uint32_t key1,
                       uint32_t replica, Control* ctl, int pass, cudaStream_t stream) {
  const DeviceShape& ds = device_shape();
  const SweepGeom G = make_geom(L);
  const uint32_t need = (G.units + kThreads - 1) / kThreads;
  const int per = L.periodic ? 1 : 0;
  const uint32_t resident = (uint32_t)ds.sms * (uint32_t)ds.per_sm[per][pass & 3];
  const dim3 grid(need < resident ? (need ? need : 1) : resident);
  kKernels[per][pass & 3]<<<grid, kThreads, 0, stream>>>(L, G, cp, key0, key1, replica, ctl);
}

}  // namespace chll
