// Pooled passes: many lattices (the replicas of a batch) swept by ONE launch
// per pass over the concatenation of all their units, with the kernel
// boundary as the synchronisation between passes.  Declarations shared by
// the kernels (pooled.cu) and the batch host code (batched.cu).
#pragma once
#include <cuda_runtime.h>

#include "chll_common.cuh"
#include "moments.cuh"
#include "sweep_unit.cuh"

namespace chll {

// One lattice of the pool.  Pass launches split the pooled units [0, total)
// into equal contiguous blocks, one per CTA; a lattice's units are
// [unit_begin, unit_begin + G.units) and the CTAs whose blocks meet them are
// [pass_cta_first, pass_cta_first + pass_ctas).  Moments launches split the
// pooled storage slots (2 * M.per_colour per lattice, from slot_begin) the
// same way, and a lattice's CTAs there write partial sums to
// partials[partial_first + (cta - mom_cta_first)].
struct PoolEntry {
  LatticeView L;
  SweepGeom G;
  MomentGeom M;
  Coupling cp;
  CouplingD cd;
  uint32_t key0, key1, replica;
  int full;                 // ni a multiple of 4 (no padding slots)
  uint32_t unit_begin;
  uint32_t slot_begin;
  int pass_cta_first, pass_ctas;
  int mom_cta_first, mom_ctas, partial_first;
  long long nsites;
  Control* ctl;
  double* mom;   // 8 FP64 accumulators: n, sum e, sum e^2, sum eta, sum eta^2, sum |eta|, sum S, sum S^2
  double* last;  // last e, eta, S
};

constexpr int kPoolThreads = 256;

// Resident CTAs of the pass kernels on this device (2 per SM).
int pool_pass_ctas();
// One fused pass (FusedPhase) of every lattice of the pool, launched as a
// programmatic dependent of the work before it on `stream`.
void launch_pool_pass(const PoolEntry* d_entries, int nent, uint32_t total_units,
                      uint32_t units_per_cta, int grid, int phase, cudaStream_t stream);
// FP64 moments of every lattice into its partial slots, then the per-lattice
// sums in CTA order accumulated into mom / last.
void launch_pool_moments(const PoolEntry* d_entries, int nent, uint32_t total_slots,
                         uint32_t slots_per_cta, int grid, double* partials,
                         cudaStream_t stream);

}  // namespace chll
