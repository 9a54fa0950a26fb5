// Shared-memory staged half-sweep: the rows a tile of units needs are brought
// into shared memory by bulk asynchronous copies (TMA, cp.async.bulk, each CTA
// loading its own tile) one tile ahead of the compute, so DRAM latency overlaps the
// Metropolis arithmetic instead of stalling it.
//
// Tile = R consecutive rows j0..j0+R-1 of one plane k (the last tile of a
// plane may have fewer rows).  Per stage, shared memory holds, hx float4 slots
// per row:
//   CEN  R rows     colour C,     plane k,   rows j0..j0+R-1   (the centres)
//   OTK  R+2 rows   other colour, plane k,   rows j0-1..j0+R   (x and y nbrs)
//   OTM  R rows     other colour, plane k-1, rows j0..j0+R-1   (z- nbrs)
//   OTP  R rows     other colour, plane k+1, rows j0..j0+R-1   (z+ nbrs)
// Rows beyond an open boundary are not copied; the unit code masks them out.
// Periodic halos come from the wrapped rows.  Results go straight to global
// memory; the next pass reads them after the kernel boundary.
//
// Unit numbering, Philox counters and per-site arithmetic are those of
// sweep_unit(), so the staged kernel's chain is bit-identical to it.
#pragma once
#include "chll_common.cuh"
#include "chll_physics.cuh"
#include "sweep_unit.cuh"

namespace chll {

struct TileGeom {
  uint32_t Q;        // units per row
  uint32_t R;        // rows per tile
  uint32_t tpp;      // tiles per plane = ceil(nj / R)
  uint32_t ntiles;   // tpp * nk
  uint32_t hx;       // slots per row
  FastDiv by_Q;      // unit-in-tile -> row-in-tile
  FastDiv by_tpp;    // tile -> plane
};

__host__ inline TileGeom make_tile_geom(const LatticeView& L, uint32_t R) {
  TileGeom T;
  T.hx = (uint32_t)L.hx;
  T.Q = T.hx / 2;
  T.R = R;
  T.tpp = ((uint32_t)L.nj + R - 1) / R;
  T.ntiles = T.tpp * (uint32_t)L.nk;
  T.by_Q = FastDiv(T.Q);
  T.by_tpp = FastDiv(T.tpp);
  return T;
}

// float4 slots of one stage: (4R + 2) rows.
__host__ __device__ inline uint32_t stage_slots(const TileGeom& T) { return (4 * T.R + 2) * T.hx; }

// ---- mbarrier / bulk copy primitives (PTX ISA 8.x, sm_90+) -----------------
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait: false if the phase did not complete within `limit` polls.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, uint32_t limit) {
  for (uint32_t it = 0; it < limit; ++it)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes,
                                         uint32_t bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
      ::"r"(dst), "l"(src), "r"(bytes), "r"(bar)
      : "memory");
}

__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Plane k and first row j0 of tile t, and its row count.
__device__ __forceinline__ void tile_rows(const TileGeom& T, const LatticeView& L, uint32_t t,
                                          uint32_t& k, uint32_t& j0, uint32_t& rows) {
  k = T.by_tpp.div(t);
  j0 = (t - k * T.tpp) * T.R;
  rows = min(T.R, (uint32_t)L.nj - j0);
}

// Issues the copies of tile t into stage buffer `buf` (one thread).  Returns
// nothing; the byte count is announced to the barrier first.
template <int C, bool PERIODIC>
__device__ __forceinline__ void issue_tile(const TileGeom& T, const LatticeView& L, uint32_t t,
                                           float4* buf, uint32_t bar) {
  uint32_t k, j0, rows;
  tile_rows(T, L, t, k, j0, rows);
  const uint32_t nj = (uint32_t)L.nj, nk = (uint32_t)L.nk, hx = T.hx;
  const uint32_t rowb = hx * (uint32_t)sizeof(float4);
  const float4* cen = L.col[C];
  const float4* oth = L.col[C ^ 1];
  float4* CEN = buf;
  float4* OTK = buf + T.R * hx;
  float4* OTM = OTK + (T.R + 2) * hx;
  float4* OTP = OTM + T.R * hx;
  // which rows exist
  const bool has_jm = PERIODIC || j0 > 0;
  const bool has_jp = PERIODIC || j0 + rows < nj;
  const bool has_km = PERIODIC || k > 0;
  const bool has_kp = PERIODIC || k + 1 < nk;
  const uint32_t jm = j0 > 0 ? j0 - 1 : nj - 1;
  const uint32_t jp = j0 + rows < nj ? j0 + rows : 0;
  const uint32_t km = k > 0 ? k - 1 : nk - 1;
  const uint32_t kp = k + 1 < nk ? k + 1 : 0;
  const uint32_t bytes = rows * rowb * 4 + (has_jm ? rowb : 0) + (has_jp ? rowb : 0) -
                         (has_km ? 0 : rows * rowb) - (has_kp ? 0 : rows * rowb);
  mbar_expect_tx(bar, bytes);
  const size_t plane_k = (size_t)k * nj;
  bulk_g2s(smem_addr(CEN), cen + (plane_k + j0) * hx, rows * rowb, bar);
  if (has_jm && has_jp && j0 > 0 && j0 + rows < nj) {
    bulk_g2s(smem_addr(OTK), oth + (plane_k + j0 - 1) * hx, (rows + 2) * rowb, bar);
  } else {
    bulk_g2s(smem_addr(OTK + hx), oth + (plane_k + j0) * hx, rows * rowb, bar);
    if (has_jm) bulk_g2s(smem_addr(OTK), oth + (plane_k + jm) * hx, rowb, bar);
    if (has_jp) bulk_g2s(smem_addr(OTK + (rows + 1) * hx), oth + (plane_k + jp) * hx, rowb, bar);
  }
  if (has_km) bulk_g2s(smem_addr(OTM), oth + ((size_t)km * nj + j0) * hx, rows * rowb, bar);
  if (has_kp) bulk_g2s(smem_addr(OTP), oth + ((size_t)kp * nj + j0) * hx, rows * rowb, bar);
}

// One unit of a staged tile: the arithmetic of sweep_unit(), with the
// neighbour rows read from the stage buffer.
template <bool DIRECTOR, int C, bool PERIODIC>
__device__ __forceinline__ unsigned int staged_unit(const TileGeom& T, const LatticeView& L,
                                                    const float4* buf, uint32_t k, uint32_t j0,
                                                    uint32_t u, uint32_t step, float d,
                                                    const Coupling& cp, uint32_t key0,
                                                    uint32_t key1, uint32_t replica) {
  const uint32_t hx = T.hx, ni = (uint32_t)L.ni, nj = (uint32_t)L.nj, nk = (uint32_t)L.nk;
  const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
  const uint32_t jr = T.by_Q.div(u);
  const uint32_t q = u - jr * T.Q;
  const uint32_t j = j0 + jr;
  const uint32_t o = (C + j + k) & 1u;
  const uint32_t i0 = 4 * q + o;
  const uint32_t i1 = i0 + 2;
  const bool v0 = i0 < ni;
  const bool v1 = i1 < ni;
  const uint32_t h0 = 2 * q;
  const float4* CEN = buf;
  const float4* OTK = buf + T.R * hx;
  const float4* OTM = OTK + (T.R + 2) * hx;
  const float4* OTP = OTM + T.R * hx;
  float4 n0 = CEN[jr * hx + h0];
  float4 n1 = CEN[jr * hx + h0 + 1];

  const bool hjm = PERIODIC || j > 0, hjp = PERIODIC || j + 1 < nj;
  const bool hkm = PERIODIC || k > 0, hkp = PERIODIC || k + 1 < nk;
  uint32_t xa = i0 - 1, xb = i0 + 1, xc = i1 + 1;
  bool hxa = i0 > 0, hxb = xb < ni, hxc = xc < ni;
  if (PERIODIC) {
    if (!hxa) xa = ni - 1;
    if (!hxb) xb = 0;
    if (!hxc) xc = 0;
    hxa = hxb = hxc = true;
  }
  const float4* xrow = OTK + (jr + 1) * hx;
  const float4 fa = hxa ? xrow[xa >> 1] : zero;
  const float4 fb = hxb ? xrow[xb >> 1] : zero;
  const float4 fc = hxc ? xrow[xc >> 1] : zero;
  Nbrs nb0, nb1;
  nb0.b[0] = fb;
  nb0.b[1] = fa;
  nb1.b[0] = fc;
  nb1.b[1] = fb;
  const float4* yp = OTK + (jr + 2) * hx + h0;
  const float4* ym = OTK + jr * hx + h0;
  const float4* zm = OTM + jr * hx + h0;
  const float4* zp = OTP + jr * hx + h0;
  nb0.b[2] = hjp ? yp[0] : zero;
  nb1.b[2] = hjp ? yp[1] : zero;
  nb0.b[3] = hjm ? ym[0] : zero;
  nb1.b[3] = hjm ? ym[1] : zero;
  nb0.b[4] = hkp ? zp[0] : zero;
  nb1.b[4] = hkp ? zp[1] : zero;
  nb0.b[5] = hkm ? zm[0] : zero;
  nb1.b[5] = hkm ? zm[1] : zero;

  const uint32_t g = q + T.Q * (k * nj + j);
  unsigned int nacc = 0, nflip = 0;
  unit_trials<C, false, DIRECTOR, !DIRECTOR>(n0, n1, nb0, nb1, v0, v1, g, step, d, cp,
                                             KeyPair{key0, key1}, replica, nacc, nflip);
  float4* out = L.col[C] + ((size_t)k * nj + j) * hx + h0;
  out[0] = n0;
  out[1] = n1;
  return DIRECTOR ? nacc : nflip;
}

// Walks tiles first, first + stride, ... of one pass with two stage buffers
// (the copies of the next tile fly while the current one is computed).
// Returns the number of accepted trials of this thread; sets *timed_out if a
// stage barrier did not complete in time (the caller records the error).
template <bool DIRECTOR, int C, bool PERIODIC>
__device__ __forceinline__ unsigned int staged_pass(const TileGeom& T, const LatticeView& L,
                                                    float4* stage0, uint32_t bar0, uint32_t bar1,
                                                    uint32_t& uses0, uint32_t& uses1,
                                                    uint32_t first, uint32_t stride,
                                                    uint32_t step, float d, const Coupling& cp,
                                                    uint32_t key0, uint32_t key1,
                                                    uint32_t replica, uint32_t wait_limit,
                                                    bool* timed_out) {
  const uint32_t slots = stage_slots(T);
  unsigned int accepted = 0;
  if (first >= T.ntiles) return 0;
  if (threadIdx.x == 0) {
    fence_proxy_async();
    issue_tile<C, PERIODIC>(T, L, first, stage0, bar0);
  }
  uint32_t pending = 1u;  // bit s: stage s has copies issued and not yet waited for
  uint32_t it = 0;
  for (uint32_t t = first; t < T.ntiles; t += stride, ++it) {
    const uint32_t s = it & 1u;
    const uint32_t next = t + stride;
    if (next < T.ntiles) {
      if (threadIdx.x == 0) {
        fence_proxy_async();
        issue_tile<C, PERIODIC>(T, L, next, stage0 + (s ^ 1u) * slots, s ? bar0 : bar1);
      }
      pending |= 1u << (s ^ 1u);
    }
    uint32_t& uses = s ? uses1 : uses0;
    const bool ok = __syncthreads_and(mbar_wait(s ? bar1 : bar0, uses & 1u, wait_limit));
    ++uses;
    pending &= ~(1u << s);
    if (!ok) {
      // A stage never completed: record it, let copies still in flight land
      // (bounded) before the CTA's shared memory is released, and stop.
      *timed_out = true;
      if (pending & (1u << (s ^ 1u)))
        mbar_wait(s ? bar0 : bar1, (s ? uses0 : uses1) & 1u, wait_limit);
      __syncthreads();
      return accepted;
    }
    uint32_t k, j0, rows;
    tile_rows(T, L, t, k, j0, rows);
    const uint32_t units = rows * T.Q;
    const float4* buf = stage0 + s * slots;
    for (uint32_t u = threadIdx.x; u < units; u += blockDim.x)
      accepted += staged_unit<DIRECTOR, C, PERIODIC>(T, L, buf, k, j0, u, step, d, cp, key0,
                                                     key1, replica);
    __syncthreads();  // the stage is free for the copies of tile t + 2*stride
  }
  return accepted;
}

}  // namespace chll
