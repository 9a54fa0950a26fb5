// Host-side launchers of the device kernels (one translation unit each).
#pragma once
#include <cuda_runtime.h>

#include "chll_common.cuh"

namespace chll {

// sweep.cu: per-device launch shapes (call once per device, outside any
// stream capture) and one half-sweep (pass = kPassDir0..kPassSpin1).
void sweep_prepare();
// Sweep form: the two-pass fused sweep, the fused passes of a chunk in one
// cluster launch (resident.cu; auto picks it where each of its threads walks
// at most one unit per pass, else the fused sweep), or the reference's four
// half-sweeps with the direct kernel or the staged kernel (shared-memory
// tiles by bulk copies).  All give the same chain.  Single half-sweeps
// (chll_lattice_pass) use the direct kernel unless staged is chosen.
enum SweepKernel : int {
  kSweepAuto = 0,
  kSweepDirect = 1,
  kSweepStaged = 2,
  kSweepFused = 3,
  kSweepResident = 4
};
void launch_sweep_pass(const LatticeView& L, const Coupling& cp, uint32_t key0, uint32_t key1,
                       uint32_t replica, Control* ctl, int pass, cudaStream_t stream,
                       int kernel = kSweepAuto);
bool staged_fits(const LatticeView& L);
// Fused sweep passes (sweep.cu): A0 = director trials of colour 0 (first
// sweep), A = previous sweep's colour-0 flips + colour-0 director trials,
// B = colour-1 director trials + colour-1 flips (ends the sweep),
// F = previous sweep's colour-0 flips (after the last sweep).
enum FusedPhase : int { kFusedA0 = 0, kFusedA = 1, kFusedB = 2, kFusedF = 3 };
void launch_fused_pass(const LatticeView& L, const Coupling& cp, uint32_t key0, uint32_t key1,
                       uint32_t replica, Control* ctl, int phase, cudaStream_t stream);
// The same on an explicit unit range and boundary mode (sweep_unit.cuh:
// make_slab_geom, BoundaryMode), for a z-slab with halo planes.  peer_lo /
// peer_hi: where the range's first / last plane is also written (the halo
// planes of the neighbouring slabs, 32-byte aligned), or null.
struct SweepGeom;
void launch_fused_pass(const LatticeView& L, const SweepGeom& G, int bmode, const Coupling& cp,
                       uint32_t key0, uint32_t key1, uint32_t replica, Control* ctl, int phase,
                       cudaStream_t stream, float4* peer_lo = nullptr,
                       float4* peer_hi = nullptr);
// The control update of a fused pass when the control block defers it.
void launch_control_update(Control* ctl, int phase, cudaStream_t stream);

// resident.cu: nsweeps fused sweeps of a whole lattice (A0 B (A B)... F, the
// same chain and control block as the fused passes) in one launch of one
// thread-block cluster whose CTAs meet at the cluster barrier between passes.
// resident_cluster: CTAs of that cluster on this device (0: none fits);
// resident_units_per_thread: units each of its threads walks per pass.
// The launcher returns 0, or -1 if the launch failed.
int resident_cluster();
uint32_t resident_units_per_thread(const LatticeView& L);
int launch_resident_sweeps(const LatticeView& L, const Coupling& cp, uint32_t key0,
                           uint32_t key1, uint32_t replica, Control* ctl, int nsweeps,
                           cudaStream_t stream);

// layout.cu: natural-order (F-order, i fastest) <-> red/black float4.
void launch_pack_f64(const LatticeView& L, const double* nx, const double* ny, const double* nz,
                     const int* s, cudaStream_t stream);
void launch_unpack_f64(const LatticeView& L, double* nx, double* ny, double* nz, int* s,
                       cudaStream_t stream);
void launch_pack_f4(const LatticeView& L, const float4* xyzs, cudaStream_t stream);
void launch_unpack_f4(const LatticeView& L, float4* xyzs, cudaStream_t stream);
void launch_init_random(const LatticeView& L, uint32_t key0, uint32_t key1, uint32_t replica,
                        cudaStream_t stream, uint64_t site0 = 0);

// observables.cu: FP64 moments and the measurement row.
int observables_max_blocks();
void launch_observables(const LatticeView& L, const CouplingD& cp, const Control* ctl,
                        double* partials, unsigned int* ticket, double* row, long long step,
                        cudaStream_t stream);
struct MomentGeom;
void launch_observables(const LatticeView& L, const MomentGeom& M, const CouplingD& cp,
                        const Control* ctl, double* partials, unsigned int* ticket, double* row,
                        long long step, cudaStream_t stream);

// adjoint.cu: energy gradient.
void launch_energy_grad(const LatticeView& L, const CouplingD& cp, float4* grad_rb, int project,
                        double* partials, unsigned int* ticket, double* out4,
                        cudaStream_t stream);
// The adjoint kernels run at most kGradMaxBlocks CTAs (grid-stride beyond
// that), each leaving four FP64 partial sums: the partial-sum buffers of the
// adjoint hold kGradMaxBlocks * 4 doubles on any GPU.
constexpr int kGradMaxBlocks = 148 * 4;
int energy_grad_max_blocks();
// adjoint.cu: one colour of the zero-temperature gradient quench.
void launch_quench_pass(const LatticeView& L, const CouplingD& cd, float eta, int colour,
                        cudaStream_t stream);

// analysis.cu: shell correlations over natural-order float4 sites (offsets
// {di, dj, dk, shell} sorted by shell; out = [sum (n.n')^2 per shell,
// sum s s' per shell, sum s]) and the chirality histogram along an integer
// direction p of m = p . (i+1, j+1, k+1) - m0.
constexpr int kMaxCorrShells = 64;
constexpr int kMaxProjectionBins = 12288;  // 48 KB of shared int bins
int shell_corr_blocks(uint64_t nsites);
void launch_shell_corr(const float4* site, int ni, int nj, int nk, const int4* offs, int noffs,
                       int nshells, bool wrap, double* partials, int blocks, double* out,
                       cudaStream_t stream);
void launch_projection(const LatticeView& L, int px, int py, int pz, long long m0, int nbins,
                       unsigned long long* hist, cudaStream_t stream);

}  // namespace chll
