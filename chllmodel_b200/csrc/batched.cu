// Batched replicas: many independent lattices of uneven size, each with its
// own (kT, h, K, eps, seed, d), swept for a fixed number of steps and
// measured in FP64 inside ONE persistent cooperative launch.
//
// This replaces the reference's phase-diagram workflow of one process and
// one ChLLSim per (kT, K, g) point (e.g. scripts/phase_diagram.py:24-31,
// scripts/g_field0.5.py:24-31).
//
// Layout: each replica keeps the plain lattice layout (two red/black float4
// colour arrays) in one shared allocation, and a ReplicaState block holds its
// d, step, accept counters, barrier words and FP64 measurement accumulators.
//
// Schedule: the launch is sized to the co-resident CTA count (cooperative
// launch), and every group of one replica (or, with pairing, two of
// neighbouring sizes) owns a contiguous run of CTAs proportional to its
// units (at least one).  A group walks its replica's units with the plain
// kernels' code (the column walk or the grid-stride unit loop, as the cost
// model picks for the group's thread count), so a replica's chain is
// bit-identical to the same replica run alone.  Between passes the group
// meets at a software barrier in global memory (arrive counter + generation
// word), split into arrive and wait so that a paired group runs the other
// replica's pass in between.  Every wait is bounded: on timeout the CTA sets
// the replica's status word and returns, and so do the others at their next
// barrier, so a fault ends the launch instead of hanging it.  The pooled
// passes of pooled.cu are the alternative schedule (chll_batch_set_pooled).
//
// Measurements every `measure_every` sweeps (from sweep `measure_from`):
// per-CTA FP64 moments (moments.cuh) -> partial slots (two per CTA, one per
// replica of its group) -> the group's first CTA sums them in a fixed order
// and accumulates e = E/N, eta = sum(s)/N and the nematic order S = largest
// eigenvalue of Q = (3/2)<n n^T> - I/2.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../../include/chll_mod.h"
#include "chll_common.cuh"
#include "moments.cuh"
#include "pooled.cuh"
#include "sweep.cuh"
#include "sweep_unit.cuh"

namespace chll {
int record_error(int code, const char* msg);
int record_ok();
}  // namespace chll

namespace chll {
namespace {

struct ReplicaDesc {
  LatticeView L;
  SweepGeom G;
  WalkGeom W;  // column-walk tasks of the replica (W.seg = 0: grid-stride over units)
  MomentGeom M;
  Coupling cp;
  CouplingD cd;
  uint32_t key0, key1, replica;
  int cta_first, cta_count;
  long long nsites;
  long long adapt_until;
};

struct ReplicaState {
  double d;
  long long step;
  unsigned long long cnt[4];  // director counts by step parity [0,1], flips [2,3]
  unsigned int bar_count;
  unsigned int bar_gen;
  unsigned int status;
  unsigned int pad;
  float paccept, faccept;
  double mom[8];   // n, sum e, sum e^2, sum eta, sum eta^2, sum |eta|, sum S, sum S^2
  double last[3];  // last e, eta, S
};

constexpr int kMomLen = 16;  // chll_batch_moments row


// Group barrier of one replica's CTAs, split in two so that a CTA can do
// other work between arriving and waiting (a second replica's pass).
// group_arrive: every thread of the CTA has finished the phase; thread 0
// publishes the CTA's writes (fence) and counts itself in, the last CTA of
// the group advancing the generation word.  Returns, in thread 0, the
// generation to wait past.
__device__ unsigned int group_arrive(ReplicaState* st, int nct) {
  __syncthreads();
  unsigned int gen = 0;
  if (threadIdx.x == 0 && nct > 1) {
    gen = *(volatile unsigned int*)&st->bar_gen;
    __threadfence();
    const unsigned int arrived = atomicAdd(&st->bar_count, 1u);
    if (arrived == (unsigned int)nct - 1) {
      st->bar_count = 0;
      __threadfence();
      atomicAdd(&st->bar_gen, 1u);
    }
  }
  return gen;
}

// Waits until the generation moved past `gen` (every CTA of the group
// arrived).  Every wait is bounded: after `limit` polls it sets the replica's
// status word.  Returns false, in every thread, if the status word is set (a
// wait gave up here or in another CTA of the group).
__device__ bool group_wait(ReplicaState* st, int nct, unsigned int gen,
                           unsigned long long limit) {
  __shared__ int s_ok;
  if (threadIdx.x == 0) {
    volatile unsigned int* genp = &st->bar_gen;
    volatile unsigned int* statp = &st->status;
    if (nct > 1) {
      unsigned long long it = 0;
      while (*genp == gen) {
        if (*statp) break;
        if (++it > limit) {
          atomicOr(&st->status, 1u);
          break;
        }
        if (it > 64) __nanosleep(32);
      }
      __threadfence();
    }
    s_ok = *statp == 0;
  }
  __syncthreads();
  return s_ok != 0;
}

// CTA sums of three counts, valid in thread 0.
template <int THREADS>
__device__ __forceinline__ void cta_sum3(unsigned int& a, unsigned int& b, unsigned int& c) {
  __shared__ unsigned int s_w[3][THREADS / 32];
  a = __reduce_add_sync(0xffffffffu, a);
  b = __reduce_add_sync(0xffffffffu, b);
  c = __reduce_add_sync(0xffffffffu, c);
  if ((threadIdx.x & 31) == 0) {
    s_w[0][threadIdx.x >> 5] = a;
    s_w[1][threadIdx.x >> 5] = b;
    s_w[2][threadIdx.x >> 5] = c;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    a = b = c = 0;
    for (int w = 0; w < THREADS / 32; ++w) {
      a += s_w[0][w];
      b += s_w[1][w];
      c += s_w[2][w];
    }
  }
  __syncthreads();
}

// The other colour is read through the coherent path (sweep_unit.cuh
// ld_other): it was written by other CTAs of the group earlier in this launch.
constexpr int kCoherent = kLoadCoherent;

// One fused pass (sweep.cuh FusedPhase) of a replica by its CTA group: the
// group's CTAs walk the replica's units grid-stride with the plain kernels'
// unit_step, so the chain is the one the replica follows alone.
template <int PHASE, bool PERIODIC, bool FULL, int THREADS>
__device__ __noinline__ void group_loop(const ReplicaDesc& D, int rank, int nct,
                                           uint32_t step, float d, unsigned int& nacc,
                                           unsigned int& nflip) {
  constexpr int C = PHASE == kFusedB ? 1 : 0;
  constexpr bool FLIP_BEFORE = PHASE == kFusedA || PHASE == kFusedF;
  constexpr bool DIR = PHASE != kFusedF;
  constexpr bool FLIP_AFTER = PHASE == kFusedB;
  // The descriptor lives in global memory, which the lattice stores could
  // alias as far as the compiler knows: copied into locals, its fields stay
  // in registers instead of being reloaded for every unit.  The Philox round
  // keys are computed once per pass, not bumped per unit.
  const LatticeView L = D.L;
  const SweepGeom G = D.G;
  const Coupling cp = D.cp;
  const PhiloxKeys key = philox_keys(D.key0, D.key1);
  const uint32_t replica = D.replica;
  const uint32_t stride = (uint32_t)nct * THREADS;
  if (FULL && D.W.seg > 0) {
    const WalkGeom W = D.W;
    for (uint32_t t = (uint32_t)rank * THREADS + threadIdx.x; t < W.ntasks; t += stride)
      walk_task<C, PERIODIC, PERIODIC, FLIP_BEFORE, DIR, FLIP_AFTER, kCoherent>(
          L, W, t, step, d, cp, key, replica, nacc, nflip);
    return;
  }
  const uint32_t plane = (uint32_t)L.hx * (uint32_t)L.nj;
  const uint32_t per_colour = plane * (uint32_t)L.nk;
  for (uint32_t g = (uint32_t)rank * THREADS + threadIdx.x; g < G.units; g += stride) {
    if (g + stride < G.units) prefetch_unit<C>(L, g + stride, plane, per_colour);
    unit_step<C, PERIODIC, PERIODIC, FLIP_BEFORE, DIR, FLIP_AFTER, FULL, kCoherent>(
        L, G, g, step, d, cp, key, replica, nacc, nflip);
  }
}

template <int PHASE, int THREADS>
__device__ __forceinline__ void group_pass(const ReplicaDesc& D, int rank, int nct,
                                           uint32_t step, float d, unsigned int& nacc,
                                           unsigned int& nflip) {
  // a replica whose ni is a multiple of 4 has no padding slots
  const bool full = D.L.ni % 4 == 0;
  if (D.L.periodic) {
    if (full) group_loop<PHASE, true, true, THREADS>(D, rank, nct, step, d, nacc, nflip);
    else group_loop<PHASE, true, false, THREADS>(D, rank, nct, step, d, nacc, nflip);
  } else {
    if (full) group_loop<PHASE, false, true, THREADS>(D, rank, nct, step, d, nacc, nflip);
    else group_loop<PHASE, false, false, THREADS>(D, rank, nct, step, d, nacc, nflip);
  }
}

// FP64 moments of one replica's current state (moments.cuh): each CTA's
// partial sums into its slot (slot = 2 * CTA + which replica of its group).
// Kept out of line: it runs once per measurement and its FP64 registers would
// otherwise crowd the sweep loop.
template <int THREADS>
__device__ __noinline__ void measure_partials(const ReplicaDesc& D, int rank, int nct,
                                              double* __restrict__ slot) {
  double m[kObsMoments];
#pragma unroll
  for (int t = 0; t < kObsMoments; ++t) m[t] = 0.0;
  const uint64_t total = 2ull * D.M.per_colour;  // < 2^32
  for (uint64_t e = (uint64_t)rank * THREADS + threadIdx.x; e < total;
       e += (uint64_t)nct * THREADS)
    site_moments<false>(D.L, D.M, D.cd, (uint32_t)e, m);
  __shared__ double s_m[THREADS / 32][kObsMoments];
#pragma unroll
  for (int t = 0; t < kObsMoments; ++t) {
    const double v = warp_sum_d(m[t]);
    if ((threadIdx.x & 31) == 0) s_m[threadIdx.x >> 5][t] = v;
  }
  __syncthreads();
  if (threadIdx.x < kObsMoments) {
    double v = 0.0;
    for (int w = 0; w < THREADS / 32; ++w) v += s_m[w][threadIdx.x];
    slot[threadIdx.x] = v;
  }
}

// After the group's barrier: the group's first CTA sums the partials, one
// moment per thread in CTA order, and accumulates e = E/N, eta = sum(s)/N and
// S into the replica's state block.  L2 loads (the partials come from other
// SMs; the barrier's fences made them visible there).
__device__ __noinline__ void measure_sum(const ReplicaDesc& D, ReplicaState* st, int nct,
                                         const double* __restrict__ first_slot) {
  __shared__ double s_tot[kObsMoments];
  if (threadIdx.x < kObsMoments) {
    double v = 0.0;
    for (int c = 0; c < nct; ++c) v += __ldcg(first_slot + (size_t)c * 2 * kObsMoments +
                                               threadIdx.x);
    s_tot[threadIdx.x] = v;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const double* tot = s_tot;
    const double n = (double)D.nsites;
    const double e = tot[0] / n, eta = tot[2] / n;
    const double qxx = 1.5 * tot[3] / n - 0.5, qyy = 1.5 * tot[4] / n - 0.5,
                 qzz = 1.5 * tot[5] / n - 0.5;
    const double qxy = 1.5 * tot[6] / n, qxz = 1.5 * tot[7] / n, qyz = 1.5 * tot[8] / n;
    const double S = sym3_max_eig(qxx, qyy, qzz, qxy, qxz, qyz);
    st->mom[0] += 1.0;
    st->mom[1] += e;
    st->mom[2] += e * e;
    st->mom[3] += eta;
    st->mom[4] += eta * eta;
    st->mom[5] += fabs(eta);
    st->mom[6] += S;
    st->mom[7] += S * S;
    st->last[0] = e;
    st->last[1] = eta;
    st->last[2] = S;
  }
  __syncthreads();
}

// One replica as seen by one CTA of its group: where it is in its sweeps.
struct RepCtx {
  const ReplicaDesc* D;
  ReplicaState* st;
  int rank, nct, which;  // which: 0 or 1, the replica's place in its group
  double d;
  long long step;
  bool pending;          // colour-0 flips of the previous sweep still to run
  unsigned int gen;      // generation of the last arrival at the group barrier
  unsigned int na, nf_prev, nf;
};

__device__ __forceinline__ void ctx_init(RepCtx& c, const ReplicaDesc* descs,
                                         ReplicaState* states, int rep, int which) {
  c.D = descs + rep;
  c.st = states + rep;
  c.rank = (int)blockIdx.x - c.D->cta_first;
  c.nct = c.D->cta_count;
  c.which = which;
  c.d = c.st->d;
  c.step = c.st->step;
  c.pending = false;
  c.gen = 0;
}

// The fused two-pass sweep of the plain kernels (sweep.cu): pass A = the
// previous sweep's colour-0 flips (when pending) + colour-0 director trials,
// pass B = colour-1 director trials + colour-1 flips, and a colour-0 flip
// pass F closes the sweep before a measurement and after the last sweep.
// Counts: director accepts of step t in cnt[t&1], flips of step t in
// cnt[2 + (t&1)].  Each phase below ends where the group must meet; the
// caller arrives at the group barrier after it and waits before the next.

template <int THREADS>
__device__ __forceinline__ void phase_a(RepCtx& c) {
  c.na = c.nf_prev = c.nf = 0;
  if (c.pending)
    group_pass<kFusedA, THREADS>(*c.D, c.rank, c.nct, (uint32_t)c.step, (float)c.d, c.na,
                                 c.nf_prev);
  else
    group_pass<kFusedA0, THREADS>(*c.D, c.rank, c.nct, (uint32_t)c.step, (float)c.d, c.na,
                                  c.nf_prev);
}

template <int THREADS>
__device__ __forceinline__ void phase_b(RepCtx& c) {
  group_pass<kFusedB, THREADS>(*c.D, c.rank, c.nct, (uint32_t)c.step, (float)c.d, c.na, c.nf);
}

template <int THREADS>
__device__ __forceinline__ void phase_f(RepCtx& c) {
  group_pass<kFusedF, THREADS>(*c.D, c.rank, c.nct, (uint32_t)c.step + 1u, (float)c.d, c.na,
                               c.nf);
}

// The CTA's counts of the sweep into the replica's counters.
template <int THREADS>
__device__ __forceinline__ void phase_counts(RepCtx& c) {
  unsigned int na = c.na, nfp = c.nf_prev, nf = c.nf;
  cta_sum3<THREADS>(na, nfp, nf);
  if (threadIdx.x == 0) {
    const int par = (int)(c.step & 1);
    if (na) atomicAdd(&c.st->cnt[par], (unsigned long long)na);
    if (nfp) atomicAdd(&c.st->cnt[2 + (par ^ 1)], (unsigned long long)nfp);
    if (nf) atomicAdd(&c.st->cnt[2 + par], (unsigned long long)nf);
  }
}

// After the count barrier: every CTA of the group derives the same new d
// from the group's count (chll_mod.f90:83-90).  The counters read here are
// reset by the group's first CTA for their next use, which no CTA reaches
// before it passes the next barrier.
__device__ __forceinline__ void phase_d(RepCtx& c, bool flush) {
  __shared__ double s_d[2];
  if (threadIdx.x == 0) {
    ReplicaState* st = c.st;
    const int par = (int)(c.step & 1);
    const float n3 = (float)c.D->nsites;
    const unsigned long long na_all = *((volatile unsigned long long*)&st->cnt[par]);
    const float pa = (float)na_all / n3;
    s_d[c.which] = (c.step < c.D->adapt_until) ? adapt_d(c.d, pa) : c.d;
    if (c.rank == 0) {
      st->cnt[par ^ 1] = 0;
      st->paccept = pa;
      if (c.pending) {  // flips of step-1 are complete (chll_mod.f90:93)
        st->faccept = (float)*((volatile unsigned long long*)&st->cnt[2 + (par ^ 1)]) / n3;
        st->cnt[2 + (par ^ 1)] = 0;
      }
      if (flush) {
        st->faccept = (float)*((volatile unsigned long long*)&st->cnt[2 + par]) / n3;
        st->cnt[2 + par] = 0;
      }
    }
  }
  __syncthreads();
  c.d = s_d[c.which];
  c.pending = !flush;
  ++c.step;
}

// All sweeps of the one or two replicas of this CTA's group.  With two, the
// CTA alternates them phase by phase: after arriving at one replica's group
// barrier it runs the other replica's phase, and only then waits, so a wait
// for the group's slowest CTA overlaps useful work.  Each replica follows
// exactly the chain it follows alone.  Returns false if a group's status
// word was set (a barrier wait gave up).
template <int THREADS>
__device__ bool run_group(const ReplicaDesc* __restrict__ descs,
                          ReplicaState* __restrict__ states, int2 reps,
                          double* __restrict__ partials, int nsweeps, int measure_every,
                          int measure_from, unsigned long long limit) {
  RepCtx c[2];
  const int nrep = reps.y >= 0 ? 2 : 1;
  ctx_init(c[0], descs, states, reps.x, 0);
  if (nrep == 2) ctx_init(c[1], descs, states, reps.y, 1);
#define CHLL_EACH(body)                 \
  for (int r = 0; r < nrep; ++r) {      \
    RepCtx& x = c[r];                   \
    body;                               \
  }
#define CHLL_WAIT() \
  if (!group_wait(x.st, x.nct, x.gen, limit)) return false
#define CHLL_ARRIVE() x.gen = group_arrive(x.st, x.nct)
  for (int s = 0; s < nsweeps; ++s) {
    const int done = s + 1;
    const bool measure =
        measure_every > 0 && done >= measure_from && done % measure_every == 0;
    const bool flush = measure || done == nsweeps;
    CHLL_EACH({
      phase_a<THREADS>(x);
      CHLL_ARRIVE();
    });
    CHLL_EACH({
      CHLL_WAIT();
      phase_b<THREADS>(x);
      if (!flush) phase_counts<THREADS>(x);
      CHLL_ARRIVE();
    });
    if (flush) {
      CHLL_EACH({
        CHLL_WAIT();
        phase_f<THREADS>(x);
        phase_counts<THREADS>(x);
        CHLL_ARRIVE();
      });
    }
    CHLL_EACH({
      CHLL_WAIT();
      phase_d(x, flush);
      if (measure) {  // FP64 measurement of the completed sweep
        measure_partials<THREADS>(*x.D, x.rank, x.nct,
                                  partials + ((size_t)blockIdx.x * 2 + x.which) * kObsMoments);
        CHLL_ARRIVE();
      }
    });
    if (measure) {
      CHLL_EACH({
        CHLL_WAIT();
        if (x.rank == 0)
          measure_sum(*x.D, x.st, x.nct,
                      partials + ((size_t)x.D->cta_first * 2 + x.which) * kObsMoments);
      });
    }
  }
#undef CHLL_EACH
#undef CHLL_WAIT
#undef CHLL_ARRIVE
  if (threadIdx.x == 0)
    for (int r = 0; r < nrep; ++r)
      if (c[r].rank == 0) {
        c[r].st->d = c[r].d;
        c[r].st->step = c[r].step;
      }
  return true;
}

// The persistent launch walks the waves in order: in wave w, CTA b works on
// the group cta_map[w * gridDim.x + b] = {replica, second replica or -1}
// ({-1, -1}: idle in this wave).  Waves hold replicas whose state together
// fits the wave size, so each wave's sweeps can run from L2; CTAs move to
// their next wave as soon as their group is done.
template <int THREADS>
__global__ void __launch_bounds__(THREADS, 512 / THREADS)
    batch_kernel(const ReplicaDesc* __restrict__ descs, ReplicaState* __restrict__ states,
                 const int2* __restrict__ cta_map, int nwaves, double* __restrict__ partials,
                 int nsweeps, int measure_every, int measure_from, unsigned long long limit) {
  for (int w = 0; w < nwaves; ++w) {
    const int2 reps = cta_map[(size_t)w * gridDim.x + blockIdx.x];
    if (reps.x < 0) continue;
    if (!run_group<THREADS>(descs, states, reps, partials, nsweeps, measure_every,
                            measure_from, limit))
      return;
  }
}

// Pooled mode (pooled.cu): each replica's d and step move into a plain
// control block for the pooled passes, and back.
__global__ void states_to_controls(const ReplicaDesc* __restrict__ descs,
                                   const ReplicaState* __restrict__ states,
                                   Control* __restrict__ ctl, int n) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  Control c = {};
  c.d = states[r].d;
  c.step = states[r].step;
  c.adapt_until = descs[r].adapt_until;
  c.nsites = descs[r].nsites;
  ctl[r] = c;
}

__global__ void controls_to_states(const Control* __restrict__ ctl,
                                   ReplicaState* __restrict__ states, int n) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  states[r].d = ctl[r].d;
  states[r].step = ctl[r].step;
  states[r].paccept = ctl[r].paccept;
  states[r].faccept = ctl[r].faccept;
}

}  // namespace
}  // namespace chll

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
namespace chll {
namespace {

using BatchKernel = void (*)(const ReplicaDesc*, ReplicaState*, const int2*, int, double*, int,
                             int, int, unsigned long long);

BatchKernel kernel_for(int threads) {
  switch (threads) {
    case 128: return batch_kernel<128>;
    case 512: return batch_kernel<512>;
    default: return batch_kernel<256>;
  }
}

int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  return record_error(code, buf);
}

#define BATCH_CUDA(expr)                                                                      \
  do {                                                                                        \
    cudaError_t _e = (expr);                                                                  \
    if (_e != cudaSuccess)                                                                    \
      return fail(_e == cudaErrorMemoryAllocation ? CHLL_ENOMEM : CHLL_ECUDA, "%s: %s", #expr, \
                  cudaGetErrorString(_e));                                                    \
  } while (0)

constexpr int kMaxCtasPerSm = 16;

}  // namespace
}  // namespace chll

struct chll_batch {
  int n = 0;
  std::vector<chll_replica_spec> specs;
  std::vector<chll::ReplicaDesc> desc;  // host copy, cta ranges filled per launch shape
  std::vector<size_t> offset;           // first float4 slot of each replica
  std::vector<size_t> per_colour;
  float4* lat = nullptr;
  size_t slots = 0;
  chll::ReplicaDesc* d_desc = nullptr;
  chll::ReplicaState* d_state = nullptr;
  int2* d_cta_replica = nullptr;  // per wave and CTA: its group's replicas
  double* d_partials = nullptr;
  void* staging = nullptr;
  size_t staging_bytes = 0;
  float4* snap_lat = nullptr;
  chll::ReplicaState* snap_state = nullptr;
  cudaStream_t own_stream = nullptr, capture_stream = nullptr, stream = nullptr;
  int sms = 148;
  int threads = 256;
  int ctas_per_sm = 0;  // 0: as many as fit
  int grid = 0;         // CTAs of the current launch shape
  int shape_threads = -1, shape_ctas = -1;
  long long wave_bytes = 0;  // state per wave (0: all replicas in one wave)
  long long shape_wave_bytes = -1;
  int pair = 0;  // 1: groups of two replicas that alternate their passes (0: one replica each)
  int shape_pair = -1;
  int nwaves = 1;
  cudaGraphExec_t graph = nullptr;
  // pooled mode (pooled.cu): one launch per pass over all replicas' units
  int pooled = 0;
  chll::Control* d_ctl = nullptr;
  chll::PoolEntry* d_pool = nullptr;
  double* d_pool_partials = nullptr;
  uint32_t pool_units = 0, pool_units_per_cta = 0, pool_slots = 0, pool_slots_per_cta = 0;
  int pool_grid = 0, pool_mom_grid = 0;
  cudaGraphExec_t pool_graph[2] = {nullptr, nullptr};  // a chunk without / with a measurement
  int pool_graph_sweeps[2] = {-1, -1};
  int g_sweeps = -1, g_every = -1, g_from = -1, g_grid = -1, g_threads = -1;
  long long g_waves = -1;
  unsigned long long limit = 1ull << 24;  // polls of a group-barrier wait before it gives up
  unsigned long long g_limit = 0;
  int g_pair = -1;
  long long total_sites = 0;

  chll::LatticeView view(int r) const { return desc[r].L; }
};

namespace {

using chll::fail;

int occupancy_of(int threads) {
  int n = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, chll::kernel_for(threads), threads, 0);
  return n;
}

// Cost of one pass of replica D on `threads` threads and its loop form
// (sweep_unit.cuh walk_pass_cost).  CHLL_WALK_SEG fixes the segment (0: the
// unit loop) for measurements.
double pass_cost(const chll::ReplicaDesc& D, uint32_t threads, uint32_t* seg) {
  static const int env = [] {
    const char* e = std::getenv("CHLL_WALK_SEG");
    return e ? std::atoi(e) : -1;
  }();
  const uint32_t ncols = D.G.Q * (uint32_t)D.L.nj;
  return chll::walk_pass_cost(D.G.units, ncols, (uint32_t)D.L.nk, D.L.ni % 4 == 0, threads, env,
                              seg);
}

// Splits the replicas into waves whose float4 state together stays within
// wave_bytes (0: one wave), largest replicas first, and gives every replica of
// a wave CTAs in proportion to its units (at least one, at most one per
// `threads` units) out of the whole co-resident grid, then its loop form for
// that many threads (pass_cost).  Every CTA of the grid gets work: the CTAs
// of lightly loaded groups leave their SMs' issue slots to the heavier groups
// sharing those SMs, which measured faster than a split that minimises the
// heaviest group's work per thread with fewer CTAs (0.219 vs 0.233 s for the
// 64-replica benchmark grid).  Fills desc[].cta_first/cta_count/W and the
// per-wave CTA map (-1: idle).
int shape_launch(chll_batch* B) {
  if (B->shape_threads == B->threads && B->shape_ctas == B->ctas_per_sm &&
      B->shape_wave_bytes == B->wave_bytes && B->shape_pair == B->pair && B->grid > 0)
    return CHLL_OK;
  const int occ = occupancy_of(B->threads);
  if (occ <= 0) return fail(CHLL_ECUDA, "batch: kernel with %d threads cannot run", B->threads);
  const int per_sm = std::min(B->ctas_per_sm > 0 ? std::min(B->ctas_per_sm, occ) : occ,
                              chll::kMaxCtasPerSm);
  const int budget = B->sms * per_sm;
  // waves, largest first
  std::vector<int> order(B->n);
  for (int r = 0; r < B->n; ++r) order[r] = r;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
    return B->desc[a].G.units > B->desc[b].G.units;
  });
  std::vector<std::vector<int>> waves;
  std::vector<long long> wave_load;
  for (int r : order) {
    const long long bytes = (long long)(2 * B->per_colour[r] * sizeof(float4));
    bool placed = false;
    if (B->wave_bytes > 0) {
      for (size_t w = 0; w < waves.size() && !placed; ++w) {
        if (wave_load[w] + bytes <= B->wave_bytes && (int)waves[w].size() < budget) {
          waves[w].push_back(r);
          wave_load[w] += bytes;
          placed = true;
        }
      }
    } else if (!waves.empty() && (int)waves[0].size() < budget) {
      waves[0].push_back(r);
      wave_load[0] += bytes;
      placed = true;
    }
    if (!placed) {
      waves.push_back({r});
      wave_load.push_back(bytes);
    }
  }
  std::vector<int2> map((size_t)waves.size() * budget, make_int2(-1, -1));
  for (size_t w = 0; w < waves.size(); ++w) {
    // groups of one or, paired, two replicas of neighbouring sizes (the wave
    // is ordered largest first)
    const std::vector<int>& reps = waves[w];
    std::vector<int2> groups;
    const int step = B->pair ? 2 : 1;
    for (size_t t = 0; t < reps.size(); t += step)
      groups.push_back(make_int2(reps[t], t + 1 < reps.size() && B->pair ? reps[t + 1] : -1));
    const int n = (int)groups.size();
    auto units = [&](int2 g) {
      return (double)B->desc[g.x].G.units + (g.y >= 0 ? (double)B->desc[g.y].G.units : 0.0);
    };
    double tot = 0.0;
    for (const int2& g : groups) tot += units(g);
    std::vector<int> cnt(n, 1), cap(n);
    for (int t = 0; t < n; ++t) {
      const uint32_t u = B->desc[groups[t].x].G.units;  // the larger replica of the group
      cap[t] = std::max(1, (int)((u + B->threads - 1) / B->threads));
    }
    int used = n;
    const int extra = budget - n;
    std::vector<std::pair<double, int>> rem;
    for (int t = 0; t < n; ++t) {
      const double want = extra * units(groups[t]) / tot;
      const int add = std::min((int)want, cap[t] - 1);
      cnt[t] += add;
      used += add;
      rem.push_back({want - (int)want, t});
    }
    std::sort(rem.begin(), rem.end(), [](auto& a, auto& b) { return a.first > b.first; });
    for (auto& pr : rem) {
      if (used >= budget) break;
      if (cnt[pr.second] < cap[pr.second]) {
        ++cnt[pr.second];
        ++used;
      }
    }
    int next = 0;
    for (int t = 0; t < n; ++t) {
      for (int r : {groups[t].x, groups[t].y}) {
        if (r < 0) continue;
        chll::ReplicaDesc& D = B->desc[r];
        uint32_t seg = 0;
        pass_cost(D, (uint32_t)(cnt[t] * B->threads), &seg);
        D.W = chll::make_walk(D.G, D.L, seg ? seg : 1);
        if (!seg) D.W.seg = 0;
        D.cta_first = next;
        D.cta_count = cnt[t];
      }
      for (int c = 0; c < cnt[t]; ++c) map[w * (size_t)budget + next++] = groups[t];
    }
  }
  B->grid = budget;
  B->nwaves = (int)waves.size();
  if (B->d_cta_replica) cudaFree(B->d_cta_replica);
  B->d_cta_replica = nullptr;
  BATCH_CUDA(cudaMalloc(&B->d_cta_replica, sizeof(int2) * map.size()));
  BATCH_CUDA(cudaMemcpyAsync(B->d_cta_replica, map.data(), sizeof(int2) * map.size(),
                             cudaMemcpyHostToDevice, B->stream));
  BATCH_CUDA(cudaMemcpyAsync(B->d_desc, B->desc.data(), sizeof(chll::ReplicaDesc) * B->n,
                             cudaMemcpyHostToDevice, B->stream));
  BATCH_CUDA(cudaStreamSynchronize(B->stream));
  B->shape_threads = B->threads;
  B->shape_ctas = B->ctas_per_sm;
  B->shape_wave_bytes = B->wave_bytes;
  B->shape_pair = B->pair;
  return CHLL_OK;
}

int launch_batch(chll_batch* B, cudaStream_t s, int nsweeps, int every, int from) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)B->grid);
  cfg.blockDim = dim3((unsigned)B->threads);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  BATCH_CUDA(cudaLaunchKernelEx(&cfg, chll::kernel_for(B->threads),
                                (const chll::ReplicaDesc*)B->d_desc, B->d_state,
                                (const int2*)B->d_cta_replica, B->nwaves, B->d_partials, nsweeps,
                                every, from,
                                B->limit));
  return CHLL_OK;
}

// The pool's layout: replicas in order, each replica's units and storage
// slots contiguous; equal blocks of units (pass launches) and of slots
// (moments launches) per CTA, and for each replica the CTAs that meet it.
int pool_prepare(chll_batch* B) {
  if (B->d_pool) return CHLL_OK;
  const int grid = chll::pool_pass_ctas();
  std::vector<chll::PoolEntry> ent(B->n);
  uint64_t units = 0, slots = 0;
  for (int r = 0; r < B->n; ++r) {
    ent[r].unit_begin = (uint32_t)units;
    ent[r].slot_begin = (uint32_t)slots;
    units += B->desc[r].G.units;
    slots += 2ull * B->desc[r].M.per_colour;
  }
  if (units >= (1ull << 31) || slots >= (1ull << 32))
    return fail(CHLL_EINVAL, "batch: pooled mode takes fewer than 2^31 units in all");
  const uint32_t upc = (uint32_t)((units + grid - 1) / grid);
  const uint32_t spc = (uint32_t)((slots + grid - 1) / grid);
  B->pool_units = (uint32_t)units;
  B->pool_slots = (uint32_t)slots;
  B->pool_units_per_cta = std::max(upc, 1u);
  B->pool_slots_per_cta = std::max(spc, 1u);
  B->pool_grid = (int)((units + B->pool_units_per_cta - 1) / B->pool_units_per_cta);
  B->pool_mom_grid = (int)((slots + B->pool_slots_per_cta - 1) / B->pool_slots_per_cta);
  BATCH_CUDA(cudaMalloc(&B->d_ctl, sizeof(chll::Control) * B->n));
  int partials = 0;
  for (int r = 0; r < B->n; ++r) {
    const chll::ReplicaDesc& D = B->desc[r];
    chll::PoolEntry& E = ent[r];
    E.L = D.L;
    E.G = D.G;
    E.M = D.M;
    E.cp = D.cp;
    E.cd = D.cd;
    E.key0 = D.key0;
    E.key1 = D.key1;
    E.replica = D.replica;
    E.full = D.L.ni % 4 == 0;
    E.nsites = D.nsites;
    const uint32_t u0 = E.unit_begin, u1 = u0 + D.G.units - 1;
    E.pass_cta_first = (int)(u0 / B->pool_units_per_cta);
    E.pass_ctas = (int)(u1 / B->pool_units_per_cta) - E.pass_cta_first + 1;
    const uint32_t s0 = E.slot_begin, s1 = s0 + 2 * D.M.per_colour - 1;
    E.mom_cta_first = (int)(s0 / B->pool_slots_per_cta);
    E.mom_ctas = (int)(s1 / B->pool_slots_per_cta) - E.mom_cta_first + 1;
    E.partial_first = partials;
    partials += E.mom_ctas;
    E.ctl = B->d_ctl + r;
    // device addresses of the replica's accumulators (no host access)
    char* st = reinterpret_cast<char*>(B->d_state + r);
    E.mom = reinterpret_cast<double*>(st + offsetof(chll::ReplicaState, mom));
    E.last = reinterpret_cast<double*>(st + offsetof(chll::ReplicaState, last));
  }
  BATCH_CUDA(cudaMalloc(&B->d_pool_partials, sizeof(double) * chll::kObsMoments * partials));
  BATCH_CUDA(cudaMalloc(&B->d_pool, sizeof(chll::PoolEntry) * B->n));
  BATCH_CUDA(cudaMemcpyAsync(B->d_pool, ent.data(), sizeof(chll::PoolEntry) * B->n,
                             cudaMemcpyHostToDevice, B->stream));
  BATCH_CUDA(cudaStreamSynchronize(B->stream));
  return CHLL_OK;
}

// The launches of `sweeps` fused sweeps of every replica (A0 B (A B)... F),
// then, with `measure`, the FP64 moments.
void pool_chunk(chll_batch* B, cudaStream_t s, int sweeps, bool measure) {
  auto pass = [&](int phase) {
    chll::launch_pool_pass(B->d_pool, B->n, B->pool_units, B->pool_units_per_cta, B->pool_grid,
                           phase, s);
  };
  for (int t = 0; t < sweeps; ++t) {
    pass(t ? chll::kFusedA : chll::kFusedA0);
    pass(chll::kFusedB);
  }
  pass(chll::kFusedF);
  if (measure)
    chll::launch_pool_moments(B->d_pool, B->n, B->pool_slots, B->pool_slots_per_cta,
                              B->pool_mom_grid, B->d_pool_partials, s);
}

int pool_run(chll_batch* B, int nsweeps, int every, int from) {
  int rc = pool_prepare(B);
  if (rc != CHLL_OK) return rc;
  chll::states_to_controls<<<(B->n + 127) / 128, 128, 0, B->stream>>>(B->d_desc, B->d_state,
                                                                      B->d_ctl, B->n);
  BATCH_CUDA(cudaGetLastError());
  const int chunk = every > 0 ? every : nsweeps;
  for (int done = 0; done < nsweeps;) {
    const int c = std::min(chunk, nsweeps - done);
    done += c;
    const bool measure = every > 0 && done >= from && done % every == 0;
    cudaGraphExec_t& ge = B->pool_graph[measure];
    if (!ge || B->pool_graph_sweeps[measure] != c) {
      if (ge) cudaGraphExecDestroy(ge);
      ge = nullptr;
      cudaGraph_t g = nullptr;
      BATCH_CUDA(cudaStreamBeginCapture(B->capture_stream, cudaStreamCaptureModeThreadLocal));
      pool_chunk(B, B->capture_stream, c, measure);
      cudaError_t e = cudaStreamEndCapture(B->capture_stream, &g);
      if (e != cudaSuccess) return fail(CHLL_ECUDA, "batch: pooled capture: %s", cudaGetErrorString(e));
      e = cudaGraphInstantiate(&ge, g, 0);
      cudaGraphDestroy(g);
      if (e != cudaSuccess)
        return fail(CHLL_ECUDA, "batch: pooled instantiate: %s", cudaGetErrorString(e));
      B->pool_graph_sweeps[measure] = c;
    }
    BATCH_CUDA(cudaGraphLaunch(ge, B->stream));
  }
  chll::controls_to_states<<<(B->n + 127) / 128, 128, 0, B->stream>>>(B->d_ctl, B->d_state,
                                                                      B->n);
  BATCH_CUDA(cudaGetLastError());
  return CHLL_OK;
}

int run_impl(chll_batch* B, int nsweeps, int every, int from) {
  if (B->pooled) return pool_run(B, nsweeps, every, from);
  int rc = shape_launch(B);
  if (rc != CHLL_OK) return rc;
  if (!(B->graph && B->g_sweeps == nsweeps && B->g_every == every && B->g_from == from &&
        B->g_grid == B->grid && B->g_threads == B->threads && B->g_waves == B->wave_bytes &&
        B->g_limit == B->limit && B->g_pair == B->pair)) {
    if (B->graph) cudaGraphExecDestroy(B->graph);
    B->graph = nullptr;
    cudaGraph_t g = nullptr;
    BATCH_CUDA(cudaStreamBeginCapture(B->capture_stream, cudaStreamCaptureModeThreadLocal));
    rc = launch_batch(B, B->capture_stream, nsweeps, every, from);
    cudaError_t e = cudaStreamEndCapture(B->capture_stream, &g);
    if (rc != CHLL_OK) return rc;
    if (e != cudaSuccess) return fail(CHLL_ECUDA, "batch: capture: %s", cudaGetErrorString(e));
    e = cudaGraphInstantiate(&B->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return fail(CHLL_ECUDA, "batch: instantiate: %s", cudaGetErrorString(e));
    B->g_sweeps = nsweeps;
    B->g_every = every;
    B->g_from = from;
    B->g_grid = B->grid;
    B->g_threads = B->threads;
    B->g_waves = B->wave_bytes;
    B->g_limit = B->limit;
    B->g_pair = B->pair;
  }
  BATCH_CUDA(cudaGraphLaunch(B->graph, B->stream));
  return CHLL_OK;
}

int ensure_staging(chll_batch* B, size_t bytes) {
  if (B->staging_bytes >= bytes) return CHLL_OK;
  if (B->staging) cudaFree(B->staging);
  B->staging = nullptr;
  B->staging_bytes = 0;
  BATCH_CUDA(cudaMalloc(&B->staging, bytes));
  B->staging_bytes = bytes;
  return CHLL_OK;
}

bool device_ptr(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

}  // namespace

extern "C" {

int chll_batch_create(const chll_replica_spec* specs, int n, chll_batch** out) {
  if (!out) return fail(CHLL_EINVAL, "batch_create: null output pointer");
  *out = nullptr;
  if (!specs || n <= 0) return fail(CHLL_EINVAL, "batch_create: need at least one replica");
  for (int r = 0; r < n; ++r) {
    const chll_replica_spec& s = specs[r];
    if (s.ni < 1 || s.nj < 1 || s.nk < 1)
      return fail(CHLL_EINVAL, "batch_create: replica %d has dims %d %d %d", r, s.ni, s.nj, s.nk);
    if (s.boundary != CHLL_OPEN && s.boundary != CHLL_PERIODIC)
      return fail(CHLL_EINVAL, "batch_create: replica %d has boundary %d", r, s.boundary);
    if (s.boundary == CHLL_PERIODIC && ((s.ni | s.nj | s.nk) & 1))
      return fail(CHLL_EINVAL, "batch_create: replica %d is periodic with odd dims", r);
    if (!(s.kT >= 0.0)) return fail(CHLL_EINVAL, "batch_create: replica %d has kT < 0", r);
    const long long units = (long long)(chll::padded_ni(s.ni) / 4) * s.nj * s.nk;
    if (units >= (1LL << 30))  // 2 slots per unit: < 2^31 slots per colour
      return fail(CHLL_EINVAL, "batch_create: replica %d is too large (%lld units, limit 2^30)",
                  r, units);
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(CHLL_ECUDA, "no CUDA device available; libchll_mod has no CPU path");
  }
  chll::sweep_prepare();
  chll_batch* B = new chll_batch();
  B->n = n;
  B->specs.assign(specs, specs + n);
  cudaGetDevice(&B->sms);
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&B->sms, cudaDevAttrMultiProcessorCount, dev);
  size_t slots = 0;
  for (int r = 0; r < n; ++r) {
    const chll_replica_spec& s = specs[r];
    const size_t pc = (size_t)(chll::padded_ni(s.ni) / 2) * s.nj * s.nk;
    B->offset.push_back(slots);
    B->per_colour.push_back(pc);
    slots += 2 * pc;
    slots = (slots + 15) & ~(size_t)15;  // 256-byte aligned replica starts
    B->total_sites += (long long)s.ni * s.nj * s.nk;
  }
  B->slots = slots;
  auto bail = [&](cudaError_t e, const char* what) {
    chll_batch_destroy(B);
    return fail(e == cudaErrorMemoryAllocation ? CHLL_ENOMEM : CHLL_ECUDA, "batch_create: %s: %s",
                what, cudaGetErrorString(e));
  };
  cudaError_t e;
  if ((e = cudaStreamCreateWithFlags(&B->own_stream, cudaStreamNonBlocking))) return bail(e, "stream");
  if ((e = cudaStreamCreateWithFlags(&B->capture_stream, cudaStreamNonBlocking)))
    return bail(e, "stream");
  B->stream = B->own_stream;
  if ((e = cudaMalloc(&B->lat, slots * sizeof(float4)))) return bail(e, "lattices");
  if ((e = cudaMemsetAsync(B->lat, 0, slots * sizeof(float4), B->stream))) return bail(e, "memset");
  if ((e = cudaMalloc(&B->d_desc, sizeof(chll::ReplicaDesc) * n))) return bail(e, "descriptors");
  if ((e = cudaMalloc(&B->d_state, sizeof(chll::ReplicaState) * n))) return bail(e, "states");
  if ((e = cudaMalloc(&B->d_partials,
                      sizeof(double) * chll::kObsMoments * B->sms * chll::kMaxCtasPerSm * 2)))
    return bail(e, "partials");
  B->desc.resize(n);
  std::vector<chll::ReplicaState> st(n);
  for (int r = 0; r < n; ++r) {
    const chll_replica_spec& s = specs[r];
    chll::ReplicaDesc& D = B->desc[r];
    std::memset(&D, 0, sizeof(D));
    D.L.col[0] = B->lat + B->offset[r];
    D.L.col[1] = B->lat + B->offset[r] + B->per_colour[r];
    D.L.ni = s.ni;
    D.L.nj = s.nj;
    D.L.nk = s.nk;
    D.L.hx = chll::padded_ni(s.ni) / 2;
    D.L.periodic = s.boundary;
    if (!chll::unit_view_aligned(D.L)) {
      chll_batch_destroy(B);
      return fail(CHLL_ECUDA, "batch_create: replica %d storage is not 32-byte aligned", r);
    }
    D.G = chll::make_geom(D.L);
    D.M = chll::make_moment_geom(D.L);
    D.cp.eps = (float)s.eps;
    D.cp.K = (float)s.K;
    D.cp.g = (float)s.g;
    D.cp.inv_kT = (float)(1.0 / s.kT);
    D.cd.eps = s.eps;
    D.cd.K = s.K;
    D.cd.g = s.g;
    D.key0 = (uint32_t)s.seed;
    D.key1 = (uint32_t)(s.seed >> 32);
    D.replica = s.replica;
    D.nsites = (long long)s.ni * s.nj * s.nk;
    D.adapt_until = 10000;
    std::memset(&st[r], 0, sizeof(chll::ReplicaState));
    st[r].d = s.d;
    st[r].step = 1;
  }
  if ((e = cudaMemcpyAsync(B->d_state, st.data(), sizeof(chll::ReplicaState) * n,
                           cudaMemcpyHostToDevice, B->stream)))
    return bail(e, "state upload");
  if ((e = cudaStreamSynchronize(B->stream))) return bail(e, "sync");
  *out = B;
  return chll::record_ok();
}

void chll_batch_destroy(chll_batch* B) {
  if (!B) return;
  if (B->own_stream) cudaStreamSynchronize(B->own_stream);
  if (B->stream && B->stream != B->own_stream) cudaStreamSynchronize(B->stream);
  if (B->graph) cudaGraphExecDestroy(B->graph);
  for (cudaGraphExec_t g : B->pool_graph)
    if (g) cudaGraphExecDestroy(g);
  cudaFree(B->d_ctl);
  cudaFree(B->d_pool);
  cudaFree(B->d_pool_partials);
  cudaFree(B->lat);
  cudaFree(B->d_desc);
  cudaFree(B->d_state);
  cudaFree(B->d_cta_replica);
  cudaFree(B->d_partials);
  cudaFree(B->staging);
  cudaFree(B->snap_lat);
  cudaFree(B->snap_state);
  if (B->own_stream) cudaStreamDestroy(B->own_stream);
  if (B->capture_stream) cudaStreamDestroy(B->capture_stream);
  delete B;
}

int chll_batch_set_stream(chll_batch* B, void* stream) {
  if (!B) return fail(CHLL_EINVAL, "null batch");
  B->stream = stream ? (cudaStream_t)stream : B->own_stream;
  return chll::record_ok();
}

int chll_batch_sync(chll_batch* B) {
  if (!B) return fail(CHLL_EINVAL, "null batch");
  BATCH_CUDA(cudaStreamSynchronize(B->stream));
  return chll::record_ok();
}

int chll_batch_init_random(chll_batch* B) {
  if (!B) return fail(CHLL_EINVAL, "null batch");
  for (int r = 0; r < B->n; ++r)
    chll::launch_init_random(B->view(r), B->desc[r].key0, B->desc[r].key1, B->desc[r].replica,
                             B->stream);
  BATCH_CUDA(cudaGetLastError());
  return chll::record_ok();
}

int chll_batch_upload_f4(chll_batch* B, int r, const float* xyzs) {
  if (!B || !xyzs) return fail(CHLL_EINVAL, "batch_upload_f4: null argument");
  if (r < 0 || r >= B->n) return fail(CHLL_EINVAL, "batch_upload_f4: replica %d out of range", r);
  const size_t n = (size_t)B->desc[r].nsites;
  const float4* src = (const float4*)xyzs;
  if (!device_ptr(xyzs)) {
    int rc = ensure_staging(B, n * sizeof(float4));
    if (rc != CHLL_OK) return rc;
    BATCH_CUDA(cudaMemcpyAsync(B->staging, xyzs, n * sizeof(float4), cudaMemcpyDefault,
                               B->stream));
    src = (const float4*)B->staging;
  }
  chll::launch_pack_f4(B->view(r), src, B->stream);
  BATCH_CUDA(cudaGetLastError());
  BATCH_CUDA(cudaStreamSynchronize(B->stream));
  return chll::record_ok();
}

int chll_batch_download_f4(chll_batch* B, int r, float* xyzs) {
  if (!B || !xyzs) return fail(CHLL_EINVAL, "batch_download_f4: null argument");
  if (r < 0 || r >= B->n)
    return fail(CHLL_EINVAL, "batch_download_f4: replica %d out of range", r);
  const size_t n = (size_t)B->desc[r].nsites;
  if (device_ptr(xyzs)) {
    chll::launch_unpack_f4(B->view(r), (float4*)xyzs, B->stream);
  } else {
    int rc = ensure_staging(B, n * sizeof(float4));
    if (rc != CHLL_OK) return rc;
    chll::launch_unpack_f4(B->view(r), (float4*)B->staging, B->stream);
    BATCH_CUDA(cudaMemcpyAsync(xyzs, B->staging, n * sizeof(float4), cudaMemcpyDefault,
                               B->stream));
  }
  BATCH_CUDA(cudaGetLastError());
  BATCH_CUDA(cudaStreamSynchronize(B->stream));
  return chll::record_ok();
}

int chll_batch_run(chll_batch* B, int nsweeps, int measure_every, int measure_from) {
  if (!B) return fail(CHLL_EINVAL, "null batch");
  if (nsweeps < 0 || measure_every < 0)
    return fail(CHLL_EINVAL, "batch_run: nsweeps and measure_every must be >= 0");
  if (nsweeps == 0) return chll::record_ok();
  const int rc = run_impl(B, nsweeps, measure_every, measure_from);
  if (rc != CHLL_OK) return rc;
  return chll::record_ok();
}

int chll_batch_moments(chll_batch* B, double* out) {
  if (!B || !out) return fail(CHLL_EINVAL, "batch_moments: null argument");
  std::vector<chll::ReplicaState> st(B->n);
  BATCH_CUDA(cudaMemcpyAsync(st.data(), B->d_state, sizeof(chll::ReplicaState) * B->n,
                             cudaMemcpyDeviceToHost, B->stream));
  BATCH_CUDA(cudaStreamSynchronize(B->stream));
  bool bad = false;
  for (int r = 0; r < B->n; ++r) {
    double* o = out + (size_t)r * chll::kMomLen;
    for (int t = 0; t < 8; ++t) o[t] = st[r].mom[t];
    o[8] = st[r].last[0];
    o[9] = st[r].last[1];
    o[10] = st[r].last[2];
    o[11] = st[r].d;
    o[12] = (double)st[r].step;
    o[13] = st[r].paccept;
    o[14] = st[r].faccept;
    o[15] = (double)st[r].status;
    bad = bad || st[r].status;
  }
  if (bad) return fail(CHLL_EDEVICE, "batch: a replica group barrier timed out");
  return chll::record_ok();
}

int chll_batch_info(chll_batch* B, int64_t* total_sites, int32_t* nreplicas, int32_t* threads,
                    int32_t* grid) {
  if (!B) return fail(CHLL_EINVAL, "null batch");
  const int rc = shape_launch(B);
  if (rc != CHLL_OK) return rc;
  if (total_sites) *total_sites = B->total_sites;
  if (nreplicas) *nreplicas = B->n;
  if (threads) *threads = B->threads;
  if (grid) *grid = B->grid;
  return chll::record_ok();
}

int chll_batch_set_wait_limit(chll_batch* B, uint64_t polls) {
  if (!B || polls == 0) return fail(CHLL_EINVAL, "batch_set_wait_limit: need a batch and polls >= 1");
  B->limit = polls;
  return chll::record_ok();
}

int chll_batch_set_pooled(chll_batch* B, int pooled) {
  if (!B || (pooled != 0 && pooled != 1))
    return fail(CHLL_EINVAL, "batch_set_pooled: pooled must be 0 or 1");
  B->pooled = pooled;
  return chll::record_ok();
}

int chll_batch_get_pooled(chll_batch* B, int* pooled) {
  if (!B || !pooled) return fail(CHLL_EINVAL, "batch_get_pooled: null argument");
  *pooled = B->pooled;
  return chll::record_ok();
}

int chll_batch_set_pairing(chll_batch* B, int pair) {
  if (!B || (pair != 0 && pair != 1))
    return fail(CHLL_EINVAL, "batch_set_pairing: pair must be 0 or 1");
  B->pair = pair;
  return chll::record_ok();
}

int chll_batch_get_pairing(chll_batch* B, int* pair) {
  if (!B || !pair) return fail(CHLL_EINVAL, "batch_get_pairing: null argument");
  *pair = B->pair;
  return chll::record_ok();
}

int chll_batch_set_wave_bytes(chll_batch* B, int64_t wave_bytes) {
  if (!B || wave_bytes < 0) return fail(CHLL_EINVAL, "batch_set_wave_bytes: bad argument");
  B->wave_bytes = wave_bytes;
  return chll::record_ok();
}

int chll_batch_get_tuning(chll_batch* B, int32_t* threads, int32_t* ctas_per_sm,
                          int64_t* wave_bytes, int32_t* nwaves) {
  if (!B) return fail(CHLL_EINVAL, "null batch");
  const int rc = shape_launch(B);
  if (rc != CHLL_OK) return rc;
  if (threads) *threads = B->threads;
  if (ctas_per_sm) *ctas_per_sm = B->ctas_per_sm;
  if (wave_bytes) *wave_bytes = B->wave_bytes;
  if (nwaves) *nwaves = B->nwaves;
  return chll::record_ok();
}

int chll_batch_set_tuning(chll_batch* B, int threads, int ctas_per_sm) {
  if (!B) return fail(CHLL_EINVAL, "null batch");
  if (threads != 128 && threads != 256 && threads != 512)
    return fail(CHLL_EINVAL, "batch_set_tuning: threads must be 128, 256 or 512 (got %d)",
                threads);
  if (ctas_per_sm < 0 || ctas_per_sm > chll::kMaxCtasPerSm)
    return fail(CHLL_EINVAL, "batch_set_tuning: ctas_per_sm must be 0..%d", chll::kMaxCtasPerSm);
  if (threads * std::max(ctas_per_sm, 1) > 2048)
    return fail(CHLL_EINVAL, "batch_set_tuning: more than 2048 threads per SM");
  B->threads = threads;
  B->ctas_per_sm = ctas_per_sm;
  return chll::record_ok();
}

// Tries every (threads, CTAs per SM) shape that fits for `trial_sweeps`
// sweeps from a snapshot of the current state, keeps the fastest, and
// restores the snapshot.
int chll_batch_autotune(chll_batch* B, int trial_sweeps, int* best_threads, int* best_ctas,
                        double* best_ms) {
  if (!B) return fail(CHLL_EINVAL, "null batch");
  if (trial_sweeps <= 0) return fail(CHLL_EINVAL, "batch_autotune: trial_sweeps must be > 0");
  if (!B->snap_lat) BATCH_CUDA(cudaMalloc(&B->snap_lat, B->slots * sizeof(float4)));
  if (!B->snap_state)
    BATCH_CUDA(cudaMalloc(&B->snap_state, sizeof(chll::ReplicaState) * B->n));
  BATCH_CUDA(cudaMemcpyAsync(B->snap_lat, B->lat, B->slots * sizeof(float4),
                             cudaMemcpyDeviceToDevice, B->stream));
  BATCH_CUDA(cudaMemcpyAsync(B->snap_state, B->d_state, sizeof(chll::ReplicaState) * B->n,
                             cudaMemcpyDeviceToDevice, B->stream));
  const int keep_threads = B->threads, keep_ctas = B->ctas_per_sm, keep_pair = B->pair,
            keep_pooled = B->pooled;
  B->pooled = 0;
  const long long keep_waves = B->wave_bytes;
  cudaEvent_t e0, e1;
  BATCH_CUDA(cudaEventCreate(&e0));
  BATCH_CUDA(cudaEventCreate(&e1));
  double best = 1e300;
  int bt = keep_threads, bc = keep_ctas, bp = keep_pair;
  int rc = CHLL_OK;
  long long bw = B->wave_bytes;
  // Candidates: one wave, or waves of 40, 64 or 96 MiB of state (a wave that
  // fits in the 126 MB L2 runs its sweeps from L2, at the price of fewer
  // replicas sharing the grid); each block size at its two highest
  // occupancies (lower occupancies were never faster on this kernel).  Trials
  // measure every 10 sweeps like a production run.
  const long long kWaveOptions[] = {0ll, 40ll << 20, 64ll << 20, 96ll << 20};
  for (int pair : {1, 0})
  for (long long wb : kWaveOptions)
  for (int threads : {128, 256, 512}) {
    const int occ = occupancy_of(threads);
    for (int c = std::max(1, occ - 1); c <= occ && rc == CHLL_OK; ++c) {
      if (c * threads > 2048) break;
      B->threads = threads;
      B->ctas_per_sm = c;
      B->wave_bytes = wb;
      B->pair = pair;
      rc = shape_launch(B);
      if (rc != CHLL_OK) break;
      cudaMemcpyAsync(B->lat, B->snap_lat, B->slots * sizeof(float4), cudaMemcpyDeviceToDevice,
                      B->stream);
      cudaMemcpyAsync(B->d_state, B->snap_state, sizeof(chll::ReplicaState) * B->n,
                      cudaMemcpyDeviceToDevice, B->stream);
      rc = launch_batch(B, B->stream, 1, 0, 0);  // warm-up
      if (rc != CHLL_OK) break;
      cudaEventRecord(e0, B->stream);
      rc = launch_batch(B, B->stream, trial_sweeps, 10, 0);
      if (rc != CHLL_OK) break;
      cudaEventRecord(e1, B->stream);
      cudaError_t e = cudaEventSynchronize(e1);
      if (e != cudaSuccess) {
        rc = fail(CHLL_ECUDA, "batch_autotune: %s", cudaGetErrorString(e));
        break;
      }
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      if (std::getenv("CHLL_TUNE_VERBOSE"))
        std::fprintf(stderr,
                     "chll batch tune: pairs %d threads %d ctas/SM %d wave %lld MiB waves %d: "
                     "%.3f ms\n",
                     pair, threads, c, wb >> 20, B->nwaves, ms);
      if (ms < best) {
        best = ms;
        bt = threads;
        bc = c;
        bw = wb;
        bp = pair;
      }
    }
  }
  // the pooled passes (pooled.cu): no launch shape to choose; timed on the
  // second of two trials (the first captures the chunk graph)
  int bpool = 0;
  if (rc == CHLL_OK) {
    B->pooled = 1;
    for (int trial = 0; trial < 2 && rc == CHLL_OK; ++trial) {
      cudaMemcpyAsync(B->lat, B->snap_lat, B->slots * sizeof(float4), cudaMemcpyDeviceToDevice,
                      B->stream);
      cudaMemcpyAsync(B->d_state, B->snap_state, sizeof(chll::ReplicaState) * B->n,
                      cudaMemcpyDeviceToDevice, B->stream);
      cudaEventRecord(e0, B->stream);
      rc = pool_run(B, trial_sweeps, 10, 0);
      cudaEventRecord(e1, B->stream);
      if (rc != CHLL_OK) break;
      cudaError_t e = cudaEventSynchronize(e1);
      if (e != cudaSuccess) {
        rc = fail(CHLL_ECUDA, "batch_autotune: %s", cudaGetErrorString(e));
        break;
      }
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      if (trial == 1) {
        if (std::getenv("CHLL_TUNE_VERBOSE"))
          std::fprintf(stderr, "chll batch tune: pooled passes: %.3f ms\n", ms);
        if (ms < best) {
          best = ms;
          bpool = 1;
        }
      }
    }
    B->pooled = 0;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaMemcpyAsync(B->lat, B->snap_lat, B->slots * sizeof(float4), cudaMemcpyDeviceToDevice,
                  B->stream);
  cudaMemcpyAsync(B->d_state, B->snap_state, sizeof(chll::ReplicaState) * B->n,
                  cudaMemcpyDeviceToDevice, B->stream);
  BATCH_CUDA(cudaStreamSynchronize(B->stream));
  if (rc != CHLL_OK) {
    B->threads = keep_threads;
    B->ctas_per_sm = keep_ctas;
    B->wave_bytes = keep_waves;
    B->pair = keep_pair;
    B->pooled = keep_pooled;
    return rc;
  }
  B->threads = bt;
  B->ctas_per_sm = bc;
  B->wave_bytes = bw;
  B->pair = bp;
  B->pooled = bpool;
  if (best_threads) *best_threads = bt;
  if (best_ctas) *best_ctas = bc;
  if (best_ms) *best_ms = best;
  return chll::record_ok();
}

}  // extern "C"
