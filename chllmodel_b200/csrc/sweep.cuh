// Host-side launchers of the device kernels (one translation unit each).
#pragma once
#include <cuda_runtime.h>

#include "chll_common.cuh"

namespace chll {

// sweep.cu: per-device launch shapes (call once per device, outside any
// stream capture) and one half-sweep (pass = kPassDir0..kPassSpin1).
void sweep_prepare();
void launch_sweep_pass(const LatticeView& L, const Coupling& cp, uint32_t key0, uint32_t key1,
                       uint32_t replica, Control* ctl, int pass, cudaStream_t stream);

// layout.cu: natural-order (F-order, i fastest) <-> red/black float4.
void launch_pack_f64(const LatticeView& L, const double* nx, const double* ny, const double* nz,
                     const int* s, cudaStream_t stream);
void launch_unpack_f64(const LatticeView& L, double* nx, double* ny, double* nz, int* s,
                       cudaStream_t stream);
void launch_pack_f4(const LatticeView& L, const float4* xyzs, cudaStream_t stream);
void launch_unpack_f4(const LatticeView& L, float4* xyzs, cudaStream_t stream);
void launch_init_random(const LatticeView& L, uint32_t key0, uint32_t key1, uint32_t replica,
                        cudaStream_t stream);

// observables.cu: FP64 moments and the measurement row.
int observables_max_blocks();
void launch_observables(const LatticeView& L, const CouplingD& cp, const Control* ctl,
                        double* partials, unsigned int* ticket, double* row, long long step,
                        cudaStream_t stream);

// adjoint.cu: energy gradient.
void launch_energy_grad(const LatticeView& L, const CouplingD& cp, float4* grad_rb, int project,
                        double* partials, unsigned int* ticket, double* out4,
                        cudaStream_t stream);
int energy_grad_max_blocks();
// adjoint.cu: one colour of the zero-temperature gradient quench.
void launch_quench_pass(const LatticeView& L, const CouplingD& cd, float eta, int colour,
                        cudaStream_t stream);

}  // namespace chll
