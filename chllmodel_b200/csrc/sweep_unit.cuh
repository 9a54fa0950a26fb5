// One work unit of a checkerboard half-sweep, shared by the plain pass
// kernels (sweep.cu) and the batched persistent kernel (batched.cu), so that
// a replica in a batch follows exactly the same chain as the same replica run
// on its own.
//
// Unit g (row-major: g = q + Q*row, row = j + nj*k) is the two same-colour
// sites of the 4-site x-block q of row (j,k): storage slots 2q and 2q+1 of
// the colour-C array, lattice sites i0 = 4q + o and i1 = i0 + 2 with
// o = (C+j+k)&1.  Both sites draw all the uniforms of a pass from one
// Philox call on the counter {g, step, replica, C} (chll_common.cuh,
// UnitRandoms).
#pragma once
#include "chll_common.cuh"
#include "chll_physics.cuh"

namespace chll {

struct SweepGeom {
  uint32_t Q;      // units (4-site blocks) per row = hx/2
  uint32_t first;  // first unit updated (0, or a slab's first interior plane)
  uint32_t units;  // end of the units updated: Q * nj * nk for a whole lattice
  uint32_t goff;   // added to a unit's index for its random counter (mod 2^32)
  FastDiv by_Q;    // unit -> row
  FastDiv by_nj;   // row -> plane
};

__host__ inline SweepGeom make_geom(const LatticeView& L) {
  SweepGeom G;
  G.Q = (uint32_t)(L.hx >> 1);
  G.first = 0;
  G.units = G.Q * (uint32_t)L.nj * (uint32_t)L.nk;
  G.goff = 0;
  G.by_Q = FastDiv(G.Q);
  G.by_nj = FastDiv((uint32_t)L.nj);
  return G;
}

// A z-slab's storage: planes p = 0..nk-1 of L hold global planes kbase + p
// (kbase even, so storage and global checkerboards agree); the units of
// planes [p0, p0 + np) are updated and draw the counters of their global
// units.
__host__ inline SweepGeom make_slab_geom(const LatticeView& L, int p0, int np, int kbase) {
  SweepGeom G = make_geom(L);
  const uint32_t per_plane = G.Q * (uint32_t)L.nj;
  G.first = per_plane * (uint32_t)p0;
  G.units = per_plane * (uint32_t)(p0 + np);
  G.goff = per_plane * (uint32_t)kbase;  // two's complement for kbase < 0
  return G;
}

// Boundary modes of the fused passes: open, periodic, and periodic in x and y
// with z taken from the storage's own planes (a slab with halo planes).
enum BoundaryMode : int { kBoundOpen = 0, kBoundPeriodic = 1, kBoundSlabXY = 2 };

__device__ __forceinline__ float4 ld4(const float4* p) { return __ldg(p); }

// One unit's two float4 slots as one 256-bit access (sm_100 ld/st .v8): a
// warp's 32 units are then 1 KB of whole sectors per instruction instead of
// two half-used 512-byte requests.  Unit starts are 32-byte aligned: every
// colour array starts 32-byte aligned (unit_view_aligned) and a row holds an
// even number of slots.
struct UnitSlots {
  float4 a, b;
};

// Read-only path: the other colour's units, which no thread of the pass writes.
// Not a compiler barrier: every pass is one kernel launch or one call of a
// non-inlined group loop (batched.cu), so these loads cannot move into a
// pass that writes what they read.
__device__ __forceinline__ UnitSlots ld_unit_nc(const float4* p) {
  UnitSlots u;
  asm("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
      : "=f"(u.a.x), "=f"(u.a.y), "=f"(u.a.z), "=f"(u.a.w), "=f"(u.b.x), "=f"(u.b.y),
        "=f"(u.b.z), "=f"(u.b.w)
      : "l"(p));
  return u;
}

// Coherent path: the unit being updated (read, then written by this thread).
__device__ __forceinline__ UnitSlots ld_unit(const float4* p) {
  UnitSlots u;
  asm volatile("ld.global.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=f"(u.a.x), "=f"(u.a.y), "=f"(u.a.z), "=f"(u.a.w), "=f"(u.b.x), "=f"(u.b.y),
                 "=f"(u.b.z), "=f"(u.b.w)
               : "l"(p)
               : "memory");
  return u;
}

__device__ __forceinline__ void st_unit(float4* p, const float4& a, const float4& b) {
  asm volatile("st.global.v8.f32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"l"(p), "f"(a.x), "f"(a.y),
               "f"(a.z), "f"(a.w), "f"(b.x), "f"(b.y), "f"(b.z), "f"(b.w)
               : "memory");
}

// Neighbour unit pair, or zeros past an open boundary.
__device__ __forceinline__ void nbr_units(bool present, const float4* p, float4& s0, float4& s1) {
  if (present) {
    const UnitSlots u = ld_unit_nc(p);
    s0 = u.a;
    s1 = u.b;
  } else {
    s0 = s1 = make_float4(0.f, 0.f, 0.f, 0.f);
  }
}

// Starts the loads of a later unit g of colour C that miss in L2: its own
// slots (slot 2g, since a row of Q units holds hx = 2Q slots) and its +z
// neighbour pair, first read by this unit in the pass; the other neighbours
// were read by units walked just before.  A plain prefetch into L1, one
// grid-stride step ahead: +6.5% on the 480^3 fused passes.  Addresses stay
// inside the view.
template <int C>
__device__ __forceinline__ void prefetch_unit(const LatticeView& L, uint32_t g, uint32_t plane,
                                              uint32_t per_colour) {
  asm volatile("prefetch.global.L1 [%0];" ::"l"(L.col[C] + 2 * g));
  const uint32_t zs = 2 * g + plane;
  if (zs < per_colour) asm volatile("prefetch.global.L1 [%0];" ::"l"(L.col[C ^ 1] + zs));
}

// Unit g of colour C read from memory: its two sites (n0, n1; v0, v1 false
// for padding slots), their six neighbours each (+x, -x, +y, -y, +z, -z;
// zero past an open boundary) and the address of its slots.
struct UnitNbhd {
  float4* cen;
  float4 n0, n1;
  Nbrs nb0, nb1;
  bool v0, v1;
  // presence of the forward neighbours: +x of each site, +y, +z
  bool fx0, fx1, fy, fz;
};

// FULL: ni is a multiple of 4, so no unit holds a padding slot.
template <int C, bool PXY, bool PZ, bool FULL = false>
__device__ __forceinline__ void gather_unit(const LatticeView& L, const SweepGeom& G, uint32_t g,
                                            UnitNbhd& U) {
  const uint32_t hx = (uint32_t)L.hx;
  const uint32_t nj = (uint32_t)L.nj, nk = (uint32_t)L.nk, ni = (uint32_t)L.ni;
  const uint32_t plane = hx * nj;
  const float4* __restrict__ oth = L.col[C ^ 1];
  const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);

  const uint32_t row = G.by_Q.div(g);
  const uint32_t q = g - row * G.Q;
  const uint32_t k = G.by_nj.div(row);
  const uint32_t j = row - k * nj;
  const uint32_t o = (C + j + k) & 1u;
  const uint32_t i0 = 4 * q + o;
  const uint32_t i1 = i0 + 2;
  U.v0 = FULL || i0 < ni;
  U.v1 = FULL || i1 < ni;
  const uint32_t rs = row * hx;  // slot of the row start
  U.cen = L.col[C] + rs + 2 * q;
  const UnitSlots own = ld_unit(U.cen);
  U.n0 = own.a;
  U.n1 = own.b;

  // neighbour rows (slot offsets) and their presence
  uint32_t sjm = rs - hx, sjp = rs + hx, skm = rs - plane, skp = rs + plane;
  bool hjm = j > 0, hjp = j + 1 < nj, hkm = k > 0, hkp = k + 1 < nk;
  // x neighbours of i0 and i1: xa = i0-1, xb = i0+1 = i1-1, xc = i1+1
  uint32_t xa = i0 - 1, xb = i0 + 1, xc = i1 + 1;
  bool hxa = i0 > 0, hxb = xb < ni, hxc = xc < ni;
  if (PXY) {
    if (!hjm) sjm = rs + (nj - 1) * hx;
    if (!hjp) sjp = rs - (nj - 1) * hx;
    if (!hxa) xa = ni - 1;
    if (!hxb) xb = 0;
    if (!hxc) xc = 0;
    hjm = hjp = hxa = hxb = hxc = true;
  }
  if (PZ) {
    if (!hkm) skm = rs + (nk - 1) * plane;
    if (!hkp) skp = rs - (nk - 1) * plane;
    hkm = hkp = true;
  }
  U.fx0 = hxb;
  U.fx1 = hxc;
  U.fy = hjp;
  U.fz = hkp;
  const float4* orow = oth + rs;
  const float4 fa = hxa ? ld4(orow + (xa >> 1)) : zero;
  const float4 fb = hxb ? ld4(orow + (xb >> 1)) : zero;
  const float4 fc = hxc ? ld4(orow + (xc >> 1)) : zero;
  const uint32_t h0 = 2 * q;
  U.nb0.b[0] = fb;  // +x of i0
  U.nb0.b[1] = fa;  // -x of i0
  U.nb1.b[0] = fc;  // +x of i1
  U.nb1.b[1] = fb;  // -x of i1
  nbr_units(hjp, oth + sjp + h0, U.nb0.b[2], U.nb1.b[2]);
  nbr_units(hjm, oth + sjm + h0, U.nb0.b[3], U.nb1.b[3]);
  nbr_units(hkp, oth + skp + h0, U.nb0.b[4], U.nb1.b[4]);
  nbr_units(hkm, oth + skm + h0, U.nb0.b[5], U.nb1.b[5]);
}

// Where else an updated unit is written: nowhere (whole lattices), or, for a
// z-slab, into the neighbouring slabs' halo planes.
struct NoPeer {
  __device__ __forceinline__ void store(uint32_t, const float4&, const float4&) const {}
};

// A slab's first and last own planes of the pass's colour also go straight
// into the halo planes of the slabs below (lo) and above (hi): slots
// [lo_first, lo_first + plane) to lo + (slot - lo_first), likewise for hi.
// lo / hi are 32-byte aligned device addresses (another GPU's memory through
// an IPC mapping, or another slab's on this GPU), or null.
struct PeerPlanes {
  float4* lo;
  float4* hi;
  uint32_t lo_first, hi_first, plane;
  __device__ __forceinline__ void store(uint32_t slot, const float4& n0, const float4& n1) const {
    if (lo && slot - lo_first < plane) st_unit(lo + (slot - lo_first), n0, n1);
    if (hi && slot - hi_first < plane) st_unit(hi + (slot - hi_first), n0, n1);
  }
};

// Updates unit g in place with the trials FLIP_BEFORE / DIR / FLIP_AFTER of
// unit_trials (chll_physics.cuh), adding accepted director trials to nacc
// and accepted flips to nflip.  A unit's slots are 2g (rows of hx = 2Q).
template <int C, bool PXY, bool PZ, bool FLIP_BEFORE, bool DIR, bool FLIP_AFTER,
          bool FULL = false, class KEY, class PEER = NoPeer>
__device__ __forceinline__ void unit_step(const LatticeView& L, const SweepGeom& G, uint32_t g,
                                          uint32_t step, float d, const Coupling& cp,
                                          const KEY& key, uint32_t replica,
                                          unsigned int& nacc, unsigned int& nflip,
                                          const PEER& peer = PEER()) {
  UnitNbhd U;
  gather_unit<C, PXY, PZ, FULL>(L, G, g, U);
  unit_trials<C, FLIP_BEFORE, DIR, FLIP_AFTER>(U.n0, U.n1, U.nb0, U.nb1, U.v0, U.v1, g + G.goff,
                                               step, d, cp, key, replica, nacc, nflip);
  st_unit(U.cen, U.n0, U.n1);
  peer.store(2 * g, U.n0, U.n1);
}

// One of the reference's four half-sweeps on unit g; returns the number of
// accepted trials (0..2).
template <bool DIRECTOR, int C, bool PERIODIC>
__device__ __forceinline__ unsigned int sweep_unit(const LatticeView& L, const SweepGeom& G,
                                                   uint32_t g, uint32_t step, float d,
                                                   const Coupling& cp, uint32_t key0,
                                                   uint32_t key1, uint32_t replica) {
  unsigned int nacc = 0, nflip = 0;
  unit_step<C, PERIODIC, PERIODIC, false, DIRECTOR, !DIRECTOR>(L, G, g, step, d, cp,
                                                               KeyPair{key0, key1}, replica, nacc,
                                                               nflip);
  return DIRECTOR ? nacc : nflip;
}

// The reference's step-size rule (chll_mod.f90:83-90): paccept is an FP32
// fraction of N, the window is 0.4-0.6 in FP64 and the factor is the default
// REAL literal 0.995.
__host__ __device__ __forceinline__ double adapt_d(double d, float paccept) {
  const double f = (double)0.995f;
  if ((double)paccept < 0.4) return d * f;
  if ((double)paccept > 0.6) return d / f;
  return d;
}

}  // namespace chll
