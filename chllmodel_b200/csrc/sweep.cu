// Plain checkerboard half-sweep kernels on one red/black float4 lattice.
//
// One launch is one of the reference's four half-sweeps per step
// (chll_mod.f90:70,74,78,81): director trials on colour 0, on colour 1, then
// chirality flips on colour 0, on colour 1.
//
// Work unit: the two same-colour sites of one 4-site x-block (storage slots
// 2q, 2q+1 of a row).  A thread draws both sites' randoms from a single
// Philox call keyed on the block and stores the pair back with one 256-bit
// store (sweep_unit.cuh).  Units are numbered row-major (g = q + Q*row) and
// CTAs walk them grid-stride, so a launch is a few CTAs per SM that stay
// resident for the whole pass: accept counts stay in registers and the
// CTA-wide reduction, the one atomic and the completion ticket happen once
// per CTA.  All index arithmetic is 32-bit (per-colour arrays < 2^31
// slots); the row and plane of a unit come from multiply-shift divisions.
//
// The last CTA to finish a pass (ticket counter) runs the step epilogue of
// chll_mod.f90:83-93 on the device: paccept and the d adaptation after the
// second director pass, faccept and the step increment after the second flip
// pass.
#include <cstdlib>
#include <mutex>

#include "chll_common.cuh"
#include "staged.cuh"
#include "sweep.cuh"
#include "sweep_unit.cuh"

namespace chll {

namespace {

constexpr int kThreads = 256;
constexpr uint32_t kWaitLimit = 1u << 22;  // mbarrier polls before a stage counts as lost

// CTA-aggregated accept count, then the step epilogue in the last CTA to
// finish (paccept and d after the second director pass, faccept and the step
// increment after the second flip pass; chll_mod.f90:83-93).
template <bool DIRECTOR, int C>
__device__ __forceinline__ void pass_epilogue(Control* __restrict__ ctl, unsigned int accepted,
                                              long long step) {
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

// Direct kernel: every unit loads its neighbours from global memory (L1/L2).
template <bool DIRECTOR, int C, bool PERIODIC>
__global__ void __launch_bounds__(kThreads, 3)
    sweep_pass_kernel(LatticeView L, SweepGeom G, Coupling cp, uint32_t key0, uint32_t key1,
                      uint32_t replica, Control* __restrict__ ctl) {
  const long long step = ctl->step;
  const float d = (float)ctl->d;
  unsigned int accepted = 0;
  const uint32_t stride = gridDim.x * kThreads;
  const uint32_t plane = (uint32_t)L.hx * (uint32_t)L.nj;
  const uint32_t per_colour = plane * (uint32_t)L.nk;
  for (uint32_t g = blockIdx.x * kThreads + threadIdx.x; g < G.units; g += stride) {
    if (g + stride < G.units) prefetch_unit<C>(L, g + stride, plane, per_colour);
    accepted += sweep_unit<DIRECTOR, C, PERIODIC>(L, G, g, (uint32_t)step, d, cp, key0, key1,
                                                  replica);
  }
  pass_epilogue<DIRECTOR, C>(ctl, accepted, step);
}

// Fused sweep: a sweep in two passes instead of four.  A flip's energy
// difference depends on the site's director and its neighbours' directors
// but not on their chiralities, and the directors do not change during the
// flip passes, so
//   pass A (colour 0): the previous sweep's colour-0 flips, then this
//                      sweep's colour-0 director trials,
//   pass B (colour 1): this sweep's colour-1 director trials, then its
//                      colour-1 flips,
// with a colour-0 flip pass (F) after the last sweep, give the chain of the
// four half-sweeps D0 D1 F0 F1 per sweep exactly: every trial sees the same
// state and draws the same counter.  Each site is read and written once per
// pass, so a sweep moves half the bytes of the four-pass form.
//
// Control epilogue: B closes the director count (paccept, d) and advances the
// step; A and F close the previous sweep's flip count (faccept), which B
// started with the colour-1 flips.  Each CTA's thread 0 adds the CTA's
// counts; the count the pass closes goes in together with one CTA ticket in
// bits 40 and up of the same 64-bit word (counts stay below 2^40: at most
// 2^32 sites), so the CTA that completes the grid's tickets has the pass total
// in its own atomic's return value and runs the update at once: no fence, no
// second read, no separate ticket word (the chain of fences and round trips
// that cost ~2.7 us per pass at 32^3-96^3).  The other count is a plain add
// for a later pass.  That CTA then clears the word -- or, on a slab whose
// counts are summed over the slabs before the update (deferred), leaves the
// bare total there.  A0 closes nothing and only adds.
constexpr int kTicketShift = 40;
constexpr unsigned long long kCountMask = (1ull << kTicketShift) - 1;

template <int PHASE>
__device__ __forceinline__ void fused_epilogue(Control* __restrict__ ctl, unsigned int nacc,
                                               unsigned int nflip, long long step) {
  constexpr bool DIR = PHASE != kFusedF;
  constexpr bool FLIPS = PHASE != kFusedA0;
  __shared__ unsigned int s_cnt[2];
  const int tid = threadIdx.x;
  if (tid < 2) s_cnt[tid] = 0;
  __syncthreads();
  if (DIR) {
    const unsigned int w = __reduce_add_sync(0xffffffffu, nacc);
    if ((tid & 31) == 0 && w) atomicAdd(&s_cnt[0], w);
  }
  if (FLIPS) {
    const unsigned int w = __reduce_add_sync(0xffffffffu, nflip);
    if ((tid & 31) == 0 && w) atomicAdd(&s_cnt[1], w);
  }
  __syncthreads();
  if (tid != 0) return;
  const unsigned long long na = s_cnt[0], nf = s_cnt[1];
  if (PHASE == kFusedA0) {
    if (na) atomicAdd(&ctl->nacc, na);
    return;
  }
  unsigned long long* closing = PHASE == kFusedB ? &ctl->nacc : &ctl->nflip;
  const unsigned long long mine = PHASE == kFusedB ? na : nf;
  if (PHASE == kFusedB) {
    if (nf) atomicAdd(&ctl->nflip, nf);
  } else if (DIR && na) {
    atomicAdd(&ctl->nacc, na);
  }
  // what the completing CTA needs, read before the ticket so that the loads
  // overlap its round trip (no pass writes them)
  const int deferred = ctl->deferred;
  const long long nsites = ctl->nsites, adapt_until = ctl->adapt_until;
  const double d = ctl->d;
  const unsigned long long old = atomicAdd(closing, mine + (1ull << kTicketShift));
  if ((old >> kTicketShift) != gridDim.x - 1) return;
  const unsigned long long total = (old & kCountMask) + mine;
  if (deferred)
    *closing = total;
  else
    fused_close<PHASE>(ctl, total, step, nsites, adapt_until, d);
}

// Two CTAs per SM: the two sites' interleaved trials want up to 128
// registers, and measured, 2 x 256 threads run these passes faster than 3 x 256
// at 80 registers.
// peer: the halo planes of neighbouring z-slabs that this slab's boundary
// planes are written to (null pointers for a whole lattice).  The periodic
// whole-lattice mode has no peers.
// FORM: 0 = grid-stride over units with padding checks, 1 = grid-stride, ni a
// multiple of 4 (no padding), 2 = column walk (sweep_unit.cuh walk_task), ni a
// multiple of 4.
template <int PHASE, int BMODE, int FORM>
__global__ void __launch_bounds__(kThreads, 2)
    fused_pass_kernel(LatticeView L, SweepGeom G, WalkGeom W, Coupling cp, PhiloxKeys keys,
                      uint32_t replica, Control* __restrict__ ctl, PeerPlanes peer) {
  constexpr int C = PHASE == kFusedB ? 1 : 0;
  constexpr bool FLIP_BEFORE = PHASE == kFusedA || PHASE == kFusedF;
  constexpr bool DIR = PHASE != kFusedF;
  constexpr bool FLIP_AFTER = PHASE == kFusedB;
  constexpr bool PXY = BMODE != kBoundOpen;
  constexpr bool PZ = BMODE == kBoundPeriodic;
  // the walk of a slab never leaves its storage in z (halo planes)
  constexpr int WZ = BMODE == kBoundPeriodic ? kWalkZPeriodic
                                             : (BMODE == kBoundSlabXY ? kWalkZHalo : kWalkZOpen);
  constexpr bool FULL = FORM != 0;
  wait_prerequisite_grids();
  const long long step = ctl->step;
  const float d = (float)ctl->d;
  unsigned int nacc = 0, nflip = 0;
  const uint32_t stride = gridDim.x * kThreads;
  const uint32_t plane = (uint32_t)L.hx * (uint32_t)L.nj;
  const uint32_t per_colour = plane * (uint32_t)L.nk;
  if (FORM == 2) {
    if (BMODE == kBoundPeriodic || (!peer.lo && !peer.hi)) {
      for (uint32_t t = blockIdx.x * kThreads + threadIdx.x; t < W.ntasks; t += stride)
        walk_task<C, PXY, WZ, FLIP_BEFORE, DIR, FLIP_AFTER>(L, W, t, (uint32_t)step, d, cp, keys,
                                                            replica, nacc, nflip);
    } else {
      for (uint32_t t = blockIdx.x * kThreads + threadIdx.x; t < W.ntasks; t += stride)
        walk_task<C, PXY, WZ, FLIP_BEFORE, DIR, FLIP_AFTER>(L, W, t, (uint32_t)step, d, cp, keys,
                                                            replica, nacc, nflip, peer);
      // the halo stores reach the other GPU before this kernel counts as done
      __threadfence_system();
    }
  } else if (BMODE == kBoundPeriodic || (!peer.lo && !peer.hi)) {
    for (uint32_t g = G.first + blockIdx.x * kThreads + threadIdx.x; g < G.units; g += stride) {
      if (g + stride < G.units) prefetch_unit<C>(L, g + stride, plane, per_colour);
      unit_step<C, PXY, PZ, FLIP_BEFORE, DIR, FLIP_AFTER, FULL>(L, G, g, (uint32_t)step, d, cp,
                                                                keys, replica, nacc, nflip);
    }
  } else {
    for (uint32_t g = G.first + blockIdx.x * kThreads + threadIdx.x; g < G.units; g += stride) {
      if (g + stride < G.units) prefetch_unit<C>(L, g + stride, plane, per_colour);
      unit_step<C, PXY, PZ, FLIP_BEFORE, DIR, FLIP_AFTER, FULL>(L, G, g, (uint32_t)step, d, cp,
                                                                keys, replica, nacc, nflip, peer);
    }
    // the halo stores reach the other GPU before this kernel counts as done
    __threadfence_system();
  }
  allow_dependent_grids();
  fused_epilogue<PHASE>(ctl, nacc, nflip, step);
}

// The deferred control update of a fused pass (one thread), after the caller
// has replaced the pass's count with its sum over all slabs.
template <int PHASE>
__global__ void control_update_kernel(Control* __restrict__ ctl) {
  fused_control_update<PHASE>(ctl, ctl->step);
}

// Staged kernel: row tiles come into shared memory by bulk copies one tile
// ahead of the compute (staged.cuh).  Same chain as the direct kernel.
template <bool DIRECTOR, int C, bool PERIODIC>
__global__ void __launch_bounds__(kThreads, 2)
    staged_pass_kernel(LatticeView L, TileGeom T, Coupling cp, uint32_t key0, uint32_t key1,
                       uint32_t replica, Control* __restrict__ ctl) {
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ __align__(8) unsigned long long bars[2];
  if (threadIdx.x == 0) {
    mbar_init(smem_addr(&bars[0]), 1);
    mbar_init(smem_addr(&bars[1]), 1);
    fence_mbar_init();
  }
  __syncthreads();
  const long long step = ctl->step;
  const float d = (float)ctl->d;
  uint32_t uses0 = 0, uses1 = 0;
  bool timed_out = false;
  const unsigned int accepted = staged_pass<DIRECTOR, C, PERIODIC>(
      T, L, reinterpret_cast<float4*>(smem), smem_addr(&bars[0]), smem_addr(&bars[1]), uses0,
      uses1, blockIdx.x, gridDim.x, (uint32_t)step, d, cp, key0, key1, replica, kWaitLimit,
      &timed_out);
  if (timed_out && threadIdx.x == 0) atomicOr(&ctl->status, 2u);
  pass_epilogue<DIRECTOR, C>(ctl, accepted, step);
}

using PassKernel = void (*)(LatticeView, SweepGeom, Coupling, uint32_t, uint32_t, uint32_t,
                           Control*);
using StagedKernel = void (*)(LatticeView, TileGeom, Coupling, uint32_t, uint32_t, uint32_t,
                             Control*);

// [periodic][pass]
const PassKernel kKernels[2][4] = {
    {sweep_pass_kernel<true, 0, false>, sweep_pass_kernel<true, 1, false>,
     sweep_pass_kernel<false, 0, false>, sweep_pass_kernel<false, 1, false>},
    {sweep_pass_kernel<true, 0, true>, sweep_pass_kernel<true, 1, true>,
     sweep_pass_kernel<false, 0, true>, sweep_pass_kernel<false, 1, true>}};
const StagedKernel kStaged[2][4] = {
    {staged_pass_kernel<true, 0, false>, staged_pass_kernel<true, 1, false>,
     staged_pass_kernel<false, 0, false>, staged_pass_kernel<false, 1, false>},
    {staged_pass_kernel<true, 0, true>, staged_pass_kernel<true, 1, true>,
     staged_pass_kernel<false, 0, true>, staged_pass_kernel<false, 1, true>}};

using FusedKernel = void (*)(LatticeView, SweepGeom, WalkGeom, Coupling, PhiloxKeys, uint32_t,
                            Control*, PeerPlanes);

// [boundary mode][phase][form]
#define CHLL_FUSED_PHASE(P, M) \
  {fused_pass_kernel<P, M, 0>, fused_pass_kernel<P, M, 1>, fused_pass_kernel<P, M, 2>}
#define CHLL_FUSED_ROW(M)                                                            \
  {CHLL_FUSED_PHASE(kFusedA0, M), CHLL_FUSED_PHASE(kFusedA, M), CHLL_FUSED_PHASE(kFusedB, M), \
   CHLL_FUSED_PHASE(kFusedF, M)}
const FusedKernel kFused[3][4][3] = {CHLL_FUSED_ROW(kBoundOpen), CHLL_FUSED_ROW(kBoundPeriodic),
                                     CHLL_FUSED_ROW(kBoundSlabXY)};
#undef CHLL_FUSED_ROW
#undef CHLL_FUSED_PHASE

// Largest dynamic shared memory a staged CTA may ask for (2 stages).
constexpr size_t kStagedSmemMax = 200 * 1024;

// Resident CTAs per SM of each pass kernel and the SM count, queried once
// per device (outside any stream capture; see sweep_prepare).  Staged
// kernels are queried per shared-memory size on first use of that size.
struct DeviceShape {
  int sms = 0;
  int per_sm[2][4] = {{0, 0, 0, 0}, {0, 0, 0, 0}};
  int fused_per_sm[3][4][3] = {};
  size_t staged_smem[8] = {0, 0, 0, 0, 0, 0, 0, 0};  // last size asked per kernel
  int staged_per_sm[8] = {0, 0, 0, 0, 0, 0, 0, 0};
};
std::mutex g_shape_mutex;
DeviceShape g_shape[64];

template <class KERNEL>
int occupancy(KERNEL k) {
  int n = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k, kThreads, 0);
  return n > 0 ? n : 1;
}

DeviceShape& device_shape() {
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) dev = 0;
  std::lock_guard<std::mutex> lk(g_shape_mutex);
  DeviceShape& s = g_shape[dev];
  if (s.sms == 0) {
    cudaDeviceGetAttribute(&s.sms, cudaDevAttrMultiProcessorCount, dev);
    if (s.sms <= 0) s.sms = 148;
    for (int per = 0; per < 2; ++per)
      for (int p = 0; p < 4; ++p) {
        s.per_sm[per][p] = occupancy(kKernels[per][p]);
        for (int f = 0; f < 3; ++f) {
          s.fused_per_sm[per][p][f] = occupancy(kFused[per][p][f]);
          if (per == 1) s.fused_per_sm[2][p][f] = occupancy(kFused[2][p][f]);
        }
        cudaFuncSetAttribute(kStaged[per][p], cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)kStagedSmemMax);
      }
  }
  return s;
}

int staged_occupancy(DeviceShape& ds, int per, int pass, size_t smem) {
  std::lock_guard<std::mutex> lk(g_shape_mutex);
  const int idx = per * 4 + pass;
  if (ds.staged_smem[idx] != smem) {
    int n = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kStaged[per][pass], kThreads, smem);
    ds.staged_smem[idx] = smem;
    ds.staged_per_sm[idx] = n > 0 ? n : 1;
  }
  return ds.staged_per_sm[idx];
}

// Planes per column-walk task for a launch of `threads` resident threads, or
// 0 for the grid-stride unit loop (walk_pass_cost).  CHLL_WALK_SEG fixes the
// segment (0: the unit loop) for measurements.
uint32_t walk_segment(const SweepGeom& G, const LatticeView& L, uint32_t threads) {
  static const int env = [] {
    const char* e = std::getenv("CHLL_WALK_SEG");
    return e ? std::atoi(e) : -1;
  }();
  const uint32_t ncols = G.Q * (uint32_t)L.nj;
  uint32_t seg = 0;
  walk_pass_cost(G.units - G.first, ncols, ncols ? (G.units - G.first) / ncols : 0,
                 L.ni % 4 == 0, threads, env, &seg);
  return seg;
}

}  // namespace

void sweep_prepare() { (void)device_shape(); }

// Rows per tile of the staged kernel: about one unit per thread.
uint32_t staged_rows(const LatticeView& L) {
  const uint32_t Q = (uint32_t)(L.hx >> 1);
  uint32_t R = Q ? kThreads / Q : 1;
  if (R < 1) R = 1;
  if (R > (uint32_t)L.nj) R = (uint32_t)L.nj;
  return R;
}

size_t staged_smem_bytes(const LatticeView& L) {
  const uint32_t R = staged_rows(L);
  return 2 * (size_t)(4 * R + 2) * (size_t)L.hx * sizeof(float4);
}

bool staged_fits(const LatticeView& L) {
  return staged_smem_bytes(L) <= kStagedSmemMax && (uint32_t)(L.hx >> 1) <= 4 * kThreads;
}

void launch_sweep_pass(const LatticeView& L, const Coupling& cp, uint32_t key0, uint32_t key1,
                       uint32_t replica, Control* ctl, int pass, cudaStream_t stream,
                       int kernel) {
  DeviceShape& ds = device_shape();
  const int per = L.periodic ? 1 : 0;
  if (kernel == kSweepStaged && staged_fits(L)) {
    const TileGeom T = make_tile_geom(L, staged_rows(L));
    const size_t smem = staged_smem_bytes(L);
    const uint32_t resident = (uint32_t)ds.sms * (uint32_t)staged_occupancy(ds, per, pass & 3, smem);
    const dim3 grid(T.ntiles < resident ? (T.ntiles ? T.ntiles : 1) : resident);
    kStaged[per][pass & 3]<<<grid, kThreads, smem, stream>>>(L, T, cp, key0, key1, replica, ctl);
    return;
  }
  const SweepGeom G = make_geom(L);
  const uint32_t need = (G.units + kThreads - 1) / kThreads;
  const uint32_t resident = (uint32_t)ds.sms * (uint32_t)ds.per_sm[per][pass & 3];
  const dim3 grid(need < resident ? (need ? need : 1) : resident);
  kKernels[per][pass & 3]<<<grid, kThreads, 0, stream>>>(L, G, cp, key0, key1, replica, ctl);
}

void launch_fused_pass(const LatticeView& L, const SweepGeom& G, int bmode, const Coupling& cp,
                       uint32_t key0, uint32_t key1, uint32_t replica, Control* ctl, int phase,
                       cudaStream_t stream, float4* peer_lo, float4* peer_hi) {
  DeviceShape& ds = device_shape();
  const int m = bmode < 0 ? 0 : (bmode > 2 ? 2 : bmode);
  const int full = L.ni % 4 == 0;
  const uint32_t res_walk = (uint32_t)ds.sms * (uint32_t)ds.fused_per_sm[m][phase & 3][2];
  const uint32_t seg = full ? walk_segment(G, L, res_walk * kThreads) : 0;
  const int form = seg ? 2 : full;
  const WalkGeom W = make_walk(G, L, seg ? seg : 1);
  const uint32_t n = form == 2 ? W.ntasks : G.units - G.first;
  const uint32_t need = (n + kThreads - 1) / kThreads;
  const uint32_t resident = (uint32_t)ds.sms * (uint32_t)ds.fused_per_sm[m][phase & 3][form];
  const dim3 grid(need < resident ? (need ? need : 1) : resident);
  // The first and last planes of the unit range: slots 2*first .. and the
  // plane before slot 2*units.
  PeerPlanes peer;
  peer.plane = (uint32_t)L.hx * (uint32_t)L.nj;
  peer.lo = m == kBoundPeriodic ? nullptr : peer_lo;
  peer.hi = m == kBoundPeriodic ? nullptr : peer_hi;
  peer.lo_first = 2 * G.first;
  peer.hi_first = 2 * G.units - peer.plane;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = dim3(kThreads);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, kFused[m][phase & 3][form], L, G, W, cp, philox_keys(key0, key1),
                     replica, ctl, peer);
}

void launch_fused_pass(const LatticeView& L, const Coupling& cp, uint32_t key0, uint32_t key1,
                       uint32_t replica, Control* ctl, int phase, cudaStream_t stream) {
  launch_fused_pass(L, make_geom(L), L.periodic ? kBoundPeriodic : kBoundOpen, cp, key0, key1,
                    replica, ctl, phase, stream);
}

void launch_control_update(Control* ctl, int phase, cudaStream_t stream) {
  switch (phase & 3) {
    case kFusedA: control_update_kernel<kFusedA><<<1, 1, 0, stream>>>(ctl); break;
    case kFusedB: control_update_kernel<kFusedB><<<1, 1, 0, stream>>>(ctl); break;
    case kFusedF: control_update_kernel<kFusedF><<<1, 1, 0, stream>>>(ctl); break;
    default: break;  // A0 closes no count
  }
}

}  // namespace chll
