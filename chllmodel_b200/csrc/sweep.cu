// Plain checkerboard half-sweep kernels on one red/black float4 lattice.
//
// One launch is one of the reference's four half-sweeps per step
// (chll_mod.f90:70,74,78,81): director trials on colour 0, on colour 1, then
// chirality flips on colour 0, on colour 1.  Each thread owns the two
// same-colour sites of one 4-site x-block (storage slots 2q, 2q+1 of a row),
// draws both sites' randoms from a single Philox call keyed on the block, and
// stores the pair back with two coalesced 128-bit stores.
//
// Accept counts are warp-aggregated and added once per CTA; the last CTA to
// finish a pass (ticket counter) runs the step epilogue of chll_mod.f90:83-93
// on the device: paccept and the d adaptation after the second director pass,
// faccept and the step increment after the second flip pass.
#include "chll_common.cuh"
#include "chll_physics.cuh"
#include "sweep.cuh"

namespace chll {

namespace {

__device__ __forceinline__ float4 ld4(const float4* p) { return __ldg(p); }

// Loads the six neighbours of site i (row j,k) from the other colour array.
// hb: storage slot of this site's y/z neighbours (same h in the adjacent rows).
__device__ __forceinline__ void load_yz(const float4* __restrict__ oth, const LatticeView& L,
                                        int j, int k, int h, Nbrs& nb, bool have_jm,
                                        bool have_jp, bool have_km, bool have_kp, int jm, int jp,
                                        int km, int kp) {
  const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
  nb.b[2] = have_jp ? ld4(oth + ((size_t)k * L.nj + jp) * L.hx + h) : z;
  nb.b[3] = have_jm ? ld4(oth + ((size_t)k * L.nj + jm) * L.hx + h) : z;
  nb.b[4] = have_kp ? ld4(oth + ((size_t)kp * L.nj + j) * L.hx + h) : z;
  nb.b[5] = have_km ? ld4(oth + ((size_t)km * L.nj + j) * L.hx + h) : z;
}

}  // namespace

template <bool DIRECTOR, int C>
__global__ void __launch_bounds__(256) sweep_pass_kernel(LatticeView L, Coupling cp, uint32_t key0,
                                                         uint32_t key1, uint32_t replica,
                                                         Control* __restrict__ ctl) {
  constexpr uint32_t kPass = (DIRECTOR ? 0u : 2u) + (uint32_t)C;
  const int Q = L.hx >> 1;
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  const long long step = ctl->step;
  const float d = (float)ctl->d;

  unsigned int accepted = 0;
  if (q < Q && j < L.nj) {
    const int o = (C + j + k) & 1;
    const int i0 = 4 * q + o;
    const int i1 = i0 + 2;
    const bool v0 = i0 < L.ni;
    const bool v1 = i1 < L.ni;
    const size_t row = (size_t)k * L.nj + j;
    float4* __restrict__ cen = L.col[C] + row * L.hx + 2 * q;
    const float4* __restrict__ oth = L.col[C ^ 1];
    const float4* __restrict__ orow = oth + row * L.hx;
    float4 n0 = cen[0];
    float4 n1 = cen[1];

    int jm = j - 1, jp = j + 1, km = k - 1, kp = k + 1;
    bool hjm = true, hjp = true, hkm = true, hkp = true;
    // x neighbours: xa = i0-1, xb = i0+1 = i1-1, xc = i1+1.
    int xa = i0 - 1, xb = i0 + 1, xc = i1 + 1;
    bool hxa = true, hxb = true, hxc = true;
    if (L.periodic) {
      if (jm < 0) jm = L.nj - 1;
      if (jp >= L.nj) jp = 0;
      if (km < 0) km = L.nk - 1;
      if (kp >= L.nk) kp = 0;
      if (xa < 0) xa = L.ni - 1;
      if (xb >= L.ni) xb = 0;
      if (xc >= L.ni) xc = 0;
    } else {
      hjm = jm >= 0;
      hjp = jp < L.nj;
      hkm = km >= 0;
      hkp = kp < L.nk;
      hxa = xa >= 0;
      hxb = xb < L.ni;
      hxc = xc < L.ni;
    }
    const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
    const float4 fa = hxa ? ld4(orow + (xa >> 1)) : zero;
    const float4 fb = hxb ? ld4(orow + (xb >> 1)) : zero;
    const float4 fc = hxc ? ld4(orow + (xc >> 1)) : zero;

    Nbrs nb0, nb1;
    nb0.b[0] = fb;  // +x of i0
    nb0.b[1] = fa;  // -x of i0
    nb1.b[0] = fc;  // +x of i1
    nb1.b[1] = fb;  // -x of i1
    load_yz(oth, L, j, k, 2 * q, nb0, hjm, hjp, hkm, hkp, jm, jp, km, kp);
    load_yz(oth, L, j, k, 2 * q + 1, nb1, hjm, hjp, hkm, hkp, jm, jp, km, kp);

    const uint32_t group = (uint32_t)(q + (size_t)Q * row);
    Ctr4 ctr = {{group, (uint32_t)step, replica, kPass}};
    const Ctr4 r = philox4x32_10(ctr, key0, key1);

    if (DIRECTOR) {
      if (v0) {
        float mx, my, mz;
        propose_director(n0.x, n0.y, n0.z, d, u01(r.v[0]), mx, my, mz);
        const float dE = director_dE(n0, mx, my, mz, nb0, cp);
        if (metropolis(dE, u01(r.v[1]), cp.inv_kT)) {
          n0.x = mx;
          n0.y = my;
          n0.z = mz;
          ++accepted;
        }
      }
      if (v1) {
        float mx, my, mz;
        propose_director(n1.x, n1.y, n1.z, d, u01(r.v[2]), mx, my, mz);
        const float dE = director_dE(n1, mx, my, mz, nb1, cp);
        if (metropolis(dE, u01(r.v[3]), cp.inv_kT)) {
          n1.x = mx;
          n1.y = my;
          n1.z = mz;
          ++accepted;
        }
      }
    } else {
      if (v0) {
        const float dE = spin_dE(n0, nb0, cp);
        if (metropolis(dE, u01(r.v[0]), cp.inv_kT)) {
          n0.w = -n0.w;
          ++accepted;
        }
      }
      if (v1) {
        const float dE = spin_dE(n1, nb1, cp);
        if (metropolis(dE, u01(r.v[2]), cp.inv_kT)) {
          n1.w = -n1.w;
          ++accepted;
        }
      }
    }
    cen[0] = n0;
    cen[1] = n1;
  }

  // Block-aggregated accept count, then the last-CTA epilogue.
  __shared__ unsigned int s_cnt;
  __shared__ bool s_last;
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  if (tid == 0) s_cnt = 0;
  __syncthreads();
  const unsigned int wsum = __reduce_add_sync(0xffffffffu, accepted);
  if ((tid & 31) == 0 && wsum) atomicAdd(&s_cnt, wsum);
  __syncthreads();
  if (tid == 0) {
    unsigned long long* counter = DIRECTOR ? &ctl->nacc : &ctl->nflip;
    if (s_cnt) atomicAdd(counter, (unsigned long long)s_cnt);
    __threadfence();
    const unsigned int nblocks = gridDim.x * gridDim.y * gridDim.z;
    const unsigned int ticket = atomicAdd(&ctl->done, 1u);
    s_last = (ticket == nblocks - 1);
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
        if (step < ctl->adapt_until) {
          // The literal 0.995 is default REAL (chll_mod.f90:86,88).
          const double f = (double)0.995f;
          double dd = ctl->d;
          if ((double)pa < 0.4)
            dd = dd * f;
          else if ((double)pa > 0.6)
            dd = dd / f;
          ctl->d = dd;
        }
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

void launch_sweep_pass(const LatticeView& L, const Coupling& cp, uint32_t key0, uint32_t key1,
                       uint32_t replica, Control* ctl, int pass, cudaStream_t stream) {
  const int Q = L.hx >> 1;
  const dim3 block(32, 8, 1);
  const dim3 grid((Q + 31) / 32, (L.nj + 7) / 8, L.nk);
  switch (pass) {
    case kPassDir0:
      sweep_pass_kernel<true, 0><<<grid, block, 0, stream>>>(L, cp, key0, key1, replica, ctl);
      break;
    case kPassDir1:
      sweep_pass_kernel<true, 1><<<grid, block, 0, stream>>>(L, cp, key0, key1, replica, ctl);
      break;
    case kPassSpin0:
      sweep_pass_kernel<false, 0><<<grid, block, 0, stream>>>(L, cp, key0, key1, replica, ctl);
      break;
    default:
      sweep_pass_kernel<false, 1><<<grid, block, 0, stream>>>(L, cp, key0, key1, replica, ctl);
      break;
  }
}

}  // namespace chll
