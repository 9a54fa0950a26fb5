// Resident sweeps: a whole chunk of fused sweeps of one small lattice in ONE
// launch of ONE thread-block cluster.
//
// A small lattice's fused pass is latency-bound: at 32^3 a pass holds 8,192
// units, one per thread, and takes ~3.3 us from one launch to the next, most
// of it the grid's start, drain, count epilogue and completion rather than
// its work.  Here
// the cluster's CTAs (up to 16, one per SM) stay resident for the whole
// chunk and meet at the hardware cluster barrier between passes
// (barrier.cluster.arrive.release / wait.acquire): no launch, no grid drain,
// no software barrier in global memory.  Each CTA adds its pass counts into
// every CTA's shared memory through distributed shared memory
// (red.shared::cluster), and every CTA derives the next d and step from the
// same totals with the plain kernels' control arithmetic
// (fused_control_update), so the chain -- units, counters, arithmetic,
// control block -- is the fused form's bit for bit.
//
// The other colour is read through the coherent path (sweep_unit.cuh
// kLoadCoherentOrdered): it was written by other CTAs of the cluster earlier
// in the launch, and the barrier's release/acquire orders those stores
// before the loads; the loads carry a memory clobber, so the compiler cannot
// move them across a barrier either.
//
// Launched without a programmatic-dependent attribute: a chunk is one launch.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <mutex>

#include "sweep.cuh"
#include "sweep_unit.cuh"

namespace chll {
namespace {

constexpr int kResThreads = 512;

struct ResidentArgs {
  LatticeView L;
  SweepGeom G;
  WalkGeom W;
  Coupling cp;
  PhiloxKeys keys;
  uint32_t replica;
  uint32_t nct;  // CTAs in the cluster (= the grid)
  Control* ctl;
  int nsweeps;
};

__device__ __forceinline__ uint32_t cluster_rank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}

// Every thread of every CTA of the cluster: this thread's earlier writes
// (global and shared) are released, the others' acquired.
__device__ __forceinline__ void cluster_barrier() {
  asm volatile(
      "barrier.cluster.arrive.release.aligned;\n\t"
      "barrier.cluster.wait.acquire.aligned;" ::
          : "memory");
}

// Address of this CTA's shared variable `p` in CTA `rank` of the cluster.
__device__ __forceinline__ uint32_t dsmem_addr(const void* p, uint32_t rank) {
  const uint32_t a = (uint32_t)__cvta_generic_to_shared(p);
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(rank));
  return r;
}

__device__ __forceinline__ void dsmem_add(uint32_t addr, unsigned long long v) {
  asm volatile("red.shared::cluster.add.u64 [%0], %1;" ::"r"(addr), "l"(v) : "memory");
}

// The control block's running state, kept by thread 0 of every CTA (all the
// same) and written back by the first CTA at the end.
struct ResControl {
  double d;
  long long step;
  unsigned long long nacc, nflip;
  float paccept, faccept;
  long long nacc_last, nflip_last;
  float n3;                // site count as FP32 (chll_mod.f90:83,93)
  long long adapt_until;
};

// One fused pass (sweep.cuh FusedPhase) over the lattice by the cluster's
// threads: the plain kernels' column walk or unit loop, with coherent loads
// that the compiler keeps between the barriers around the pass.
template <int PHASE, int BMODE, int FORM>
__device__ __forceinline__ void resident_pass(const ResidentArgs& A, uint32_t rank, uint32_t step,
                                           float d, unsigned int& nacc, unsigned int& nflip) {
  constexpr int C = PHASE == kFusedB ? 1 : 0;
  constexpr bool FLIP_BEFORE = PHASE == kFusedA || PHASE == kFusedF;
  constexpr bool DIR = PHASE != kFusedF;
  constexpr bool FLIP_AFTER = PHASE == kFusedB;
  constexpr bool P = BMODE == kBoundPeriodic;
  constexpr bool FULL = FORM != 0;
  const LatticeView L = A.L;
  const Coupling cp = A.cp;
  const PhiloxKeys key = A.keys;
  const uint32_t replica = A.replica;
  const uint32_t stride = A.nct * kResThreads;
  unsigned int na = 0, nf = 0;
  if (FORM == 2) {
    const WalkGeom W = A.W;
    for (uint32_t t = rank * kResThreads + threadIdx.x; t < W.ntasks; t += stride)
      walk_task<C, P, P, FLIP_BEFORE, DIR, FLIP_AFTER, kLoadCoherentOrdered>(
          L, W, t, step, d, cp, key, replica, na, nf);
  } else {
    const SweepGeom G = A.G;
    const uint32_t plane = (uint32_t)L.hx * (uint32_t)L.nj;
    const uint32_t per_colour = plane * (uint32_t)L.nk;
    for (uint32_t g = rank * kResThreads + threadIdx.x; g < G.units; g += stride) {
      if (g + stride < G.units) prefetch_unit<C>(L, g + stride, plane, per_colour);
      unit_step<C, P, P, FLIP_BEFORE, DIR, FLIP_AFTER, FULL, kLoadCoherentOrdered>(
          L, G, g, step, d, cp, key, replica, na, nf);
    }
  }
  nacc = na;
  nflip = nf;
}

// Pass q and its counts: summed over the CTA, then added by CTA-many threads
// into slot q % 3 of EVERY CTA's counters (director accepts in the low, flips
// in the high 32 bits of one word), so that after the barrier each CTA reads
// the cluster's totals from its own shared memory.  Each CTA clears its own
// slot (q + 1) % 3 before it arrives at barrier q: it read that slot last,
// for pass q - 2, before arriving at barrier q (program order), and the next
// additions to it come from pass q + 1, after barrier q.
template <int PHASE, int BMODE, int FORM>
__device__ __forceinline__ void resident_pass_counted(const ResidentArgs& A, uint32_t rank,
                                                      uint32_t q, uint32_t step, float d,
                                                      unsigned long long* s_tot,
                                                      unsigned int* s_part) {
  unsigned int na = 0, nf = 0;
  resident_pass<PHASE, BMODE, FORM>(A, rank, step, d, na, nf);
  na = __reduce_add_sync(0xffffffffu, na);
  nf = __reduce_add_sync(0xffffffffu, nf);
  if ((threadIdx.x & 31) == 0) {
    if (na) atomicAdd(&s_part[0], na);
    if (nf) atomicAdd(&s_part[1], nf);
  }
  __syncthreads();
  const unsigned long long v = (unsigned long long)s_part[0] |
                               ((unsigned long long)s_part[1] << 32);
  if (threadIdx.x < A.nct && v) dsmem_add(dsmem_addr(&s_tot[q % 3], threadIdx.x), v);
  __syncthreads();  // s_part read by every sender before it is cleared
  if (threadIdx.x == 0) {
    s_part[0] = s_part[1] = 0;
    s_tot[(q + 1) % 3] = 0;
  }
  cluster_barrier();
}

// The control updates of fused_control_update for the counts of pass q
// (thread 0; the totals in this CTA's slot q % 3).
template <int PHASE>
__device__ __forceinline__ void resident_update(ResControl& S, const unsigned long long* s_tot,
                                                uint32_t q) {
  const unsigned long long t = s_tot[q % 3];
  S.nacc += t & 0xffffffffull;
  S.nflip += t >> 32;
  if (PHASE == kFusedB) {
    const float pa = (float)S.nacc / S.n3;
    S.paccept = pa;
    S.nacc_last = (long long)S.nacc;
    S.nacc = 0;
    if (S.step < S.adapt_until) S.d = adapt_d(S.d, pa);
    S.step = S.step + 1;
  } else if (PHASE == kFusedA || PHASE == kFusedF) {
    S.faccept = (float)S.nflip / S.n3;
    S.nflip_last = (long long)S.nflip;
    S.nflip = 0;
  }
}

// A sweep is pass A (A0 first) and pass B with a cluster barrier after each;
// the counts of both close after B's barrier (A's update first, as the fused
// passes apply them), and only B changes d and step, which thread 0 then
// hands to the CTA.  Passes A and F only need the lattice ordered by their
// barrier.
template <int BMODE, int FORM>
__global__ void __launch_bounds__(kResThreads, 1)
    resident_sweeps_kernel(const __grid_constant__ ResidentArgs A) {
  __shared__ unsigned long long s_tot[3];
  __shared__ unsigned int s_part[2];
  __shared__ double s_d;
  __shared__ long long s_step;
  const uint32_t rank = cluster_rank();
  Control* ctl = A.ctl;
  if (threadIdx.x < 3) s_tot[threadIdx.x] = 0;
  if (threadIdx.x < 2) s_part[threadIdx.x] = 0;
  double d = ctl->d;
  long long step = ctl->step;
  ResControl S;
  if (threadIdx.x == 0) {
    S.d = d;
    S.step = step;
    S.nacc = ctl->nacc;
    S.nflip = ctl->nflip;
    S.paccept = ctl->paccept;
    S.faccept = ctl->faccept;
    S.nacc_last = ctl->nacc_last;
    S.nflip_last = ctl->nflip_last;
    S.n3 = (float)ctl->nsites;
    S.adapt_until = ctl->adapt_until;
  }
  cluster_barrier();  // counters cleared in every CTA, the control block read
  uint32_t q = 0;
  for (int s = 0; s < A.nsweeps; ++s) {
    if (s)
      resident_pass_counted<kFusedA, BMODE, FORM>(A, rank, q, (uint32_t)step, (float)d, s_tot,
                                                  s_part);
    else
      resident_pass_counted<kFusedA0, BMODE, FORM>(A, rank, q, (uint32_t)step, (float)d, s_tot,
                                                   s_part);
    resident_pass_counted<kFusedB, BMODE, FORM>(A, rank, q + 1, (uint32_t)step, (float)d, s_tot,
                                                s_part);
    if (threadIdx.x == 0) {
      if (s)
        resident_update<kFusedA>(S, s_tot, q);
      else
        resident_update<kFusedA0>(S, s_tot, q);
      resident_update<kFusedB>(S, s_tot, q + 1);
      s_d = S.d;
      s_step = S.step;
    }
    __syncthreads();
    d = s_d;
    step = s_step;
    q += 2;
  }
  if (A.nsweeps > 0) {
    resident_pass_counted<kFusedF, BMODE, FORM>(A, rank, q, (uint32_t)step, (float)d, s_tot,
                                                s_part);
    if (threadIdx.x == 0) resident_update<kFusedF>(S, s_tot, q);
  }
  if (rank == 0 && threadIdx.x == 0) {
    ctl->d = S.d;
    ctl->step = S.step;
    ctl->nacc = S.nacc;
    ctl->nflip = S.nflip;
    ctl->paccept = S.paccept;
    ctl->faccept = S.faccept;
    ctl->nacc_last = S.nacc_last;
    ctl->nflip_last = S.nflip_last;
  }
}

using ResidentKernel = void (*)(const ResidentArgs);
// [periodic][form]
const ResidentKernel kResident[2][3] = {
    {resident_sweeps_kernel<kBoundOpen, 0>, resident_sweeps_kernel<kBoundOpen, 1>,
     resident_sweeps_kernel<kBoundOpen, 2>},
    {resident_sweeps_kernel<kBoundPeriodic, 0>, resident_sweeps_kernel<kBoundPeriodic, 1>,
     resident_sweeps_kernel<kBoundPeriodic, 2>}};

// The largest cluster (16, 8, 4, 2 or 1 CTAs) of which one can be resident
// on this device, per device; 0 if none.
std::mutex g_res_mutex;
int g_res_cluster[64];
bool g_res_known[64];

// CHLL_RESIDENT_CLUSTER caps the cluster size (for measurements).
int query_cluster() {
  int best = 0;
  const char* env = std::getenv("CHLL_RESIDENT_CLUSTER");
  const int cap = env ? std::atoi(env) : 16;
  for (int p = 0; p < 2; ++p)
    for (int f = 0; f < 3; ++f)
      cudaFuncSetAttribute(kResident[p][f], cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  for (int c : {16, 8, 4, 2, 1}) {
    if (c > cap) continue;
    bool all = true;
    for (int p = 0; p < 2 && all; ++p)
      for (int f = 0; f < 3 && all; ++f) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)c);
        cfg.blockDim = dim3(kResThreads);
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = (unsigned)c;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        int n = 0;
        if (cudaOccupancyMaxActiveClusters(&n, (const void*)kResident[p][f], &cfg) !=
                cudaSuccess ||
            n < 1)
          all = false;
      }
    if (all) {
      best = c;
      break;
    }
  }
  cudaGetLastError();
  return best;
}

}  // namespace

int resident_cluster() {
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) dev = 0;
  std::lock_guard<std::mutex> lk(g_res_mutex);
  if (!g_res_known[dev]) {
    g_res_cluster[dev] = query_cluster();
    g_res_known[dev] = true;
  }
  return g_res_cluster[dev];
}

uint32_t resident_units_per_thread(const LatticeView& L) {
  const int c = resident_cluster();
  if (c <= 0) return 0xffffffffu;
  const SweepGeom G = make_geom(L);
  const uint32_t threads = (uint32_t)c * kResThreads;
  return (G.units + threads - 1) / threads;
}

int launch_resident_sweeps(const LatticeView& L, const Coupling& cp, uint32_t key0,
                           uint32_t key1, uint32_t replica, Control* ctl, int nsweeps,
                           cudaStream_t stream) {
  const int c = resident_cluster();
  if (c <= 0) return -1;
  ResidentArgs A;
  A.L = L;
  A.G = make_geom(L);
  const uint32_t threads = (uint32_t)c * kResThreads;
  const bool full = L.ni % 4 == 0;
  const uint32_t ncols = A.G.Q * (uint32_t)L.nj;
  uint32_t seg = 0;
  if (full) walk_pass_cost(A.G.units, ncols, (uint32_t)L.nk, true, threads, -1, &seg);
  A.W = make_walk(A.G, L, seg ? seg : 1);
  const int form = seg ? 2 : (full ? 1 : 0);
  A.cp = cp;
  A.keys = philox_keys(key0, key1);
  A.replica = replica;
  A.nct = (uint32_t)c;
  A.ctl = ctl;
  A.nsweeps = nsweeps;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)c);
  cfg.blockDim = dim3(kResThreads);
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = (unsigned)c;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kResident[L.periodic ? 1 : 0][form], A) == cudaSuccess ? 0 : -1;
}

}  // namespace chll
