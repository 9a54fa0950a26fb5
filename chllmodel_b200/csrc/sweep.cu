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
#include "chll_physics.cuh"
#include "sweep.cuh"

namespace chll {

namespace {

constexpr int kThreads = 256;

struct SweepGeom {
  uint32_t Q;        // units (4-site blocks) per row = hx/2
  uint32_t units;    // Q * nj * nk
  FastDiv by_Q;      // unit -> row
  FastDiv by_nj;     // row -> plane
};

__device__ __forceinline__ float4 ld4(const float4* p) { return __ldg(p); }

template <bool DIRECTOR, int C>
__global__ void __launch_bounds__(kThreads, 3)
    sweep_pass_kernel(LatticeView L, SweepGeom G, Coupling cp, uint32_t key0, uint32_t key1,
                      uint32_t replica, Control* __restrict__ ctl) {
  constexpr uint32_t kPass = (DIRECTOR ? 0u : 2u) + (uint32_t)C;
  const long long step = ctl->step;
  const float d = (float)ctl->d;
  const uint32_t hx = (uint32_t)L.hx;
  const uint32_t nj = (uint32_t)L.nj, nk = (uint32_t)L.nk, ni = (uint32_t)L.ni;
  const uint32_t plane = hx * nj;  // slots per plane
  float4* __restrict__ cen_base = L.col[C];
  const float4* __restrict__ oth = L.col[C ^ 1];
  const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);

  unsigned int accepted = 0;
  for (uint32_t g = blockIdx.x * kThreads + threadIdx.x; g < G.units;
       g += gridDim.x * kThreads) {
    const uint32_t row = G.by_Q.div(g);
    const uint32_t q = g - row * G.Q;
    const uint32_t k = G.by_nj.div(row);
    const uint32_t j = row - k * nj;
    const uint32_t o = (C + j + k) & 1u;
    const uint32_t i0 = 4 * q + o;
    const uint32_t i1 = i0 + 2;
    const bool v0 = i0 < ni;
    const bool v1 = i1 < ni;
    const uint32_t rs = row * hx;  // slot of the row start
    float4* cen = cen_base + rs + 2 * q;
    float4 n0 = cen[0];
    float4 n1 = cen[1];

    // neighbour rows (slot offsets) and their presence
    uint32_t sjm = rs - hx, sjp = rs + hx, skm = rs - plane, skp = rs + plane;
    bool hjm = j > 0, hjp = j + 1 < nj, hkm = k > 0, hkp = k + 1 < nk;
    // x neighbours of i0 and i1: xa = i0-1, xb = i0+1 = i1-1, xc = i1+1
    uint32_t xa = i0 - 1, xb = i0 + 1, xc = i1 + 1;
    bool hxa = i0 > 0, hxb = xb < ni, hxc = xc < ni;
    if (L.periodic) {
      if (!hjm) sjm = rs + (nj - 1) * hx;
      if (!hjp) sjp = rs - (nj - 1) * hx;
      if (!hkm) skm = rs + (nk - 1) * plane;
      if (!hkp) skp = rs - (nk - 1) * plane;
      if (!hxa) xa = ni - 1;
      if (!hxb) xb = 0;
      if (!hxc) xc = 0;
      hjm = hjp = hkm = hkp = hxa = hxb = hxc = true;
    }
    const float4* orow = oth + rs;
    const float4 fa = hxa ? ld4(orow + (xa >> 1)) : zero;
    const float4 fb = hxb ? ld4(orow + (xb >> 1)) : zero;
    const float4 fc = hxc ? ld4(orow + (xc >> 1)) : zero;
    const uint32_t h0 = 2 * q;
    Nbrs nb0, nb1;
    nb0.b[0] = fb;  // +x of i0
    nb0.b[1] = fa;  // -x of i0
    nb1.b[0] = fc;  // +x of i1
    nb1.b[1] = fb;  // -x of i1
    nb0.b[2] = hjp ? ld4(oth + sjp + h0) : zero;
    nb1.b[2] = hjp ? ld4(oth + sjp + h0 + 1) : zero;
    nb0.b[3] = hjm ? ld4(oth + sjm + h0) : zero;
    nb1.b[3] = hjm ? ld4(oth + sjm + h0 + 1) : zero;
    nb0.b[4] = hkp ? ld4(oth + skp + h0) : zero;
    nb1.b[4] = hkp ? ld4(oth + skp + h0 + 1) : zero;
    nb0.b[5] = hkm ? ld4(oth + skm + h0) : zero;
    nb1.b[5] = hkm ? ld4(oth + skm + h0 + 1) : zero;

    Ctr4 ctr = {{g, (uint32_t)step, replica, kPass}};
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

// Resident CTAs per SM of each pass kernel and the SM count, queried once
// per device (outside any stream capture; see sweep_prepare).
struct DeviceShape {
  int sms = 0;
  int per_sm[4] = {0, 0, 0, 0};
};
std::mutex g_shape_mutex;
DeviceShape g_shape[64];

template <bool D, int C>
int occupancy() {
  int n = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, sweep_pass_kernel<D, C>, kThreads, 0);
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
    s.per_sm[0] = occupancy<true, 0>();
    s.per_sm[1] = occupancy<true, 1>();
    s.per_sm[2] = occupancy<false, 0>();
    s.per_sm[3] = occupancy<false, 1>();
  }
  return s;
}

}  // namespace

void sweep_prepare() { (void)device_shape(); }

void launch_sweep_pass(const LatticeView& L, const Coupling& cp, uint32_t key0, uint32_t key1,
                       uint32_t replica, Control* ctl, int pass, cudaStream_t stream) {
  const DeviceShape& ds = device_shape();
  SweepGeom G;
  G.Q = (uint32_t)(L.hx >> 1);
  G.units = G.Q * (uint32_t)L.nj * (uint32_t)L.nk;
  G.by_Q = FastDiv(G.Q);
  G.by_nj = FastDiv((uint32_t)L.nj);
  const uint32_t need = (G.units + kThreads - 1) / kThreads;
  const uint32_t resident = (uint32_t)ds.sms * (uint32_t)ds.per_sm[pass & 3];
  const dim3 grid(need < resident ? (need ? need : 1) : resident);
  switch (pass) {
    case kPassDir0:
      sweep_pass_kernel<true, 0><<<grid, kThreads, 0, stream>>>(L, G, cp, key0, key1, replica, ctl);
      break;
    case kPassDir1:
      sweep_pass_kernel<true, 1><<<grid, kThreads, 0, stream>>>(L, G, cp, key0, key1, replica, ctl);
      break;
    case kPassSpin0:
      sweep_pass_kernel<false, 0><<<grid, kThreads, 0, stream>>>(L, G, cp, key0, key1, replica,
                                                                 ctl);
      break;
    default:
      sweep_pass_kernel<false, 1><<<grid, kThreads, 0, stream>>>(L, G, cp, key0, key1, replica,
                                                                 ctl);
      break;
  }
}

}  // namespace chll
