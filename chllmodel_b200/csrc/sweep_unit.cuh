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
#include "sweep.cuh"

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
// Not a compiler barrier: every pass that uses it is one kernel launch, so
// these loads cannot move into a pass that writes what they read.
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

// The other colour's reads come in three flavours, chosen by the template
// argument COH of the unit code below.
//   kLoadNc (0): the read-only path (ld.global.nc), valid where every pass is
//     its own kernel launch (the plain, slab and pooled passes: a launch
//     boundary, or a programmatic dependent's grid-dependency wait, orders
//     one pass's stores before the next pass's loads).
//   kLoadCoherent (1): weak ld.global, still cached in L1, for the batched
//     persistent launch, whose passes are separated by software barriers
//     inside one launch; there the release/acquire of the barrier orders the
//     stores of the pass before against these loads, which the memory model
//     guarantees for ld.global and not for the non-coherent path.  Not a
//     compiler barrier: each batched pass is one call of a non-inlined group
//     loop, so the loads cannot move across the barrier between passes.
//   kLoadCoherentOrdered (2): the same loads with a memory clobber, for passes
//     inlined between barriers (resident.cu): the compiler keeps them between
//     the barriers around their pass.
enum LoadMode : int { kLoadNc = 0, kLoadCoherent = 1, kLoadCoherentOrdered = 2 };

__device__ __forceinline__ UnitSlots ld_unit_ca(const float4* p) {
  UnitSlots u;
  asm("ld.global.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
      : "=f"(u.a.x), "=f"(u.a.y), "=f"(u.a.z), "=f"(u.a.w), "=f"(u.b.x), "=f"(u.b.y),
        "=f"(u.b.z), "=f"(u.b.w)
      : "l"(p));
  return u;
}

__device__ __forceinline__ UnitSlots ld_unit_ca_ordered(const float4* p) {
  UnitSlots u;
  asm("ld.global.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
      : "=f"(u.a.x), "=f"(u.a.y), "=f"(u.a.z), "=f"(u.a.w), "=f"(u.b.x), "=f"(u.b.y),
        "=f"(u.b.z), "=f"(u.b.w)
      : "l"(p)
      : "memory");
  return u;
}

template <int COH>
__device__ __forceinline__ UnitSlots ld_other(const float4* p) {
  if (COH == kLoadCoherentOrdered) return ld_unit_ca_ordered(p);
  return COH == kLoadCoherent ? ld_unit_ca(p) : ld_unit_nc(p);
}

template <int COH>
__device__ __forceinline__ float4 ld4_other(const float4* p) {
  float4 v;
  if (COH == kLoadCoherentOrdered) {
    asm("ld.global.v4.f32 {%0,%1,%2,%3}, [%4];"
        : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
        : "l"(p)
        : "memory");
    return v;
  }
  if (COH == kLoadCoherent) {
    asm("ld.global.v4.f32 {%0,%1,%2,%3}, [%4];"
        : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
        : "l"(p));
    return v;
  }
  return ld4(p);
}

__device__ __forceinline__ void st_unit(float4* p, const float4& a, const float4& b) {
  asm volatile("st.global.v8.f32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"l"(p), "f"(a.x), "f"(a.y),
               "f"(a.z), "f"(a.w), "f"(b.x), "f"(b.y), "f"(b.z), "f"(b.w)
               : "memory");
}

// Neighbour unit pair, or zeros past an open boundary.
template <int COH = kLoadNc>
__device__ __forceinline__ void nbr_units(bool present, const float4* p, float4& s0, float4& s1) {
  if (present) {
    const UnitSlots u = ld_other<COH>(p);
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
template <int C, bool PXY, bool PZ, bool FULL = false, int COH = kLoadNc>
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
  const float4 fa = hxa ? ld4_other<COH>(orow + (xa >> 1)) : zero;
  const float4 fb = hxb ? ld4_other<COH>(orow + (xb >> 1)) : zero;
  const float4 fc = hxc ? ld4_other<COH>(orow + (xc >> 1)) : zero;
  const uint32_t h0 = 2 * q;
  U.nb0.b[0] = fb;  // +x of i0
  U.nb0.b[1] = fa;  // -x of i0
  U.nb1.b[0] = fc;  // +x of i1
  U.nb1.b[1] = fb;  // -x of i1
  nbr_units<COH>(hjp, oth + sjp + h0, U.nb0.b[2], U.nb1.b[2]);
  nbr_units<COH>(hjm, oth + sjm + h0, U.nb0.b[3], U.nb1.b[3]);
  nbr_units<COH>(hkp, oth + skp + h0, U.nb0.b[4], U.nb1.b[4]);
  nbr_units<COH>(hkm, oth + skm + h0, U.nb0.b[5], U.nb1.b[5]);
}

// Where else an updated unit is written: nowhere (whole lattices), or, for a
// z-slab, into the neighbouring slabs' halo planes.
struct NoPeer {
  __device__ __forceinline__ void store(uint32_t, const float4&, const float4&) const {}
  __device__ __forceinline__ void store_task_ends(const float4*, uint32_t, uint32_t) const {}
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
  // After a column-walk task over planes: only its first unit can lie in the
  // first own plane and only its last in the last own plane.  The units are
  // read back (this thread wrote them) and stored to the halos, so that the
  // walk's loop keeps no peer state in registers.
  __device__ __forceinline__ void store_task_ends(const float4* own, uint32_t first_slot,
                                                  uint32_t last_slot) const {
    if (lo && first_slot - lo_first < plane) {
      const UnitSlots v = ld_unit(own + first_slot);
      st_unit(lo + (first_slot - lo_first), v.a, v.b);
    }
    if (hi && last_slot - hi_first < plane) {
      const UnitSlots v = ld_unit(own + last_slot);
      st_unit(hi + (last_slot - hi_first), v.a, v.b);
    }
  }
};

// Updates unit g in place with the trials FLIP_BEFORE / DIR / FLIP_AFTER of
// unit_trials (chll_physics.cuh), adding accepted director trials to nacc
// and accepted flips to nflip.  A unit's slots are 2g (rows of hx = 2Q).
template <int C, bool PXY, bool PZ, bool FLIP_BEFORE, bool DIR, bool FLIP_AFTER,
          bool FULL = false, int COH = kLoadNc, class KEY, class PEER = NoPeer>
__device__ __forceinline__ void unit_step(const LatticeView& L, const SweepGeom& G, uint32_t g,
                                          uint32_t step, float d, const Coupling& cp,
                                          const KEY& key, uint32_t replica,
                                          unsigned int& nacc, unsigned int& nflip,
                                          const PEER& peer = PEER()) {
  UnitNbhd U;
  gather_unit<C, PXY, PZ, FULL, COH>(L, G, g, U);
  unit_trials<C, FLIP_BEFORE, DIR, FLIP_AFTER>(U.n0, U.n1, U.nb0, U.nb1, U.v0, U.v1, g + G.goff,
                                               step, d, cp, key, replica, nacc, nflip);
  st_unit(U.cen, U.n0, U.n1);
  peer.store(2 * g, U.n0, U.n1);
}

// ---------------------------------------------------------------------------
// Column walk (lattices whose ni is a multiple of 4, so no unit holds a
// padding slot).  A task is one column of units -- unit q of row j -- over a
// run of consecutive planes [k0, k1); a thread walks it plane by plane.  The
// other colour's unit pair q of row (j, k) serves three consecutive steps:
// as the +z pair of plane k-1, the x-row pair of plane k (carried in
// registers from the step before) and the -z pair of plane k+1 (read again,
// from L1: carrying it too cost registers that pass B then paid for in
// recomputed addresses, 5% on its time).  Per step the thread loads its own
// pair, the +y, -y, +z and -z pairs and one x neighbour that lies outside
// pair q, with offsets fixed for the whole column: no per-unit index decode
// and no boundary tests other than the z ends.  Units, counters and
// arithmetic are those of unit_step, so the chain is the same bit for bit.
//
// Which x neighbours pair q supplies: in row (j, k) the pass's colour has
// parity o = (C+j+k)&1 and its unit q holds sites i0 = 4q+o, i1 = i0+2; the
// other colour's pair q holds 4q+1-o, 4q+3-o.  For o = 0 that is i0+1 and
// i1+1 (+x of i0 and i1, and -x of i1), the extra one being i0-1 (slot 2q-1,
// or the row's last slot across a periodic x edge); for o = 1 it is i0-1
// and i0+1 (-x of i0 and i1, and +x of i0), the extra one being i1+1 (slot
// 2q+2, or slot 0 across the edge).  The y and z neighbour pairs are pair q
// of rows (j+-1, k) and (j, k+-1), which have parity o as well.
// ---------------------------------------------------------------------------
struct WalkGeom {
  uint32_t Q;        // units per row
  uint32_t ncols;    // columns (units per plane): Q * nj
  uint32_t seg;      // planes per task (the last task of a column may have fewer)
  uint32_t nseg;     // tasks per column
  uint32_t ntasks;   // ncols * nseg
  uint32_t k_first;  // planes walked: [k_first, k_end)
  uint32_t k_end;
  uint32_t goff;     // added to a unit's index for its random counter (mod 2^32)
  FastDiv by_cols;   // task -> segment
  FastDiv by_Q;      // column -> row
};

// The walk of the unit range of G (whole planes) in tasks of `seg` planes.
__host__ inline WalkGeom make_walk(const SweepGeom& G, const LatticeView& L, uint32_t seg) {
  WalkGeom W;
  W.Q = G.Q;
  W.ncols = G.Q * (uint32_t)L.nj;
  W.k_first = G.first / W.ncols;
  W.k_end = G.units / W.ncols;
  const uint32_t planes = W.k_end - W.k_first;
  W.seg = seg < 1 ? 1 : (seg > planes ? planes : seg);
  W.nseg = planes ? (planes + W.seg - 1) / W.seg : 0;
  W.ntasks = W.ncols * W.nseg;
  W.goff = G.goff;
  W.by_cols = FastDiv(W.ncols);
  W.by_Q = FastDiv(W.Q);
  return W;
}

// Cost of one pass of `units` units (ncols columns of `planes` planes) on
// `threads` threads: about the most work any thread does, counted in
// grid-stride units.  A walk step costs kWalkStep of a grid-stride unit (no
// index decode, two loads fewer; the 480^3 passes ran at 0.94 of the unit
// loop's time in 16-plane tasks) and a task kWalkPrime more (its first x-row
// and -z loads, the column decode); whole tasks per thread quantise more
// coarsely than units.
// *seg: planes per task of the cheapest walk, or 0 when the grid-stride unit
// loop is cheaper or ni is not a multiple of 4 (full = false).
// force_seg >= 0 fixes the segment instead (0: the unit loop).
constexpr double kWalkStep = 0.93, kWalkPrime = 0.5;

__host__ inline double walk_pass_cost(uint32_t units, uint32_t ncols, uint32_t planes, bool full,
                                      uint32_t threads, int force_seg, uint32_t* seg) {
  double best = (double)((units + threads - 1) / (threads ? threads : 1));
  *seg = 0;
  if (!full || force_seg == 0 || ncols == 0) return best;
  for (uint32_t s = 2; s <= planes; ++s) {
    if (force_seg > 0 && s != (uint32_t)force_seg) continue;
    const uint64_t tasks = (uint64_t)ncols * ((planes + s - 1) / s);
    const double cost =
        (double)((tasks + threads - 1) / threads) * ((double)s * kWalkStep + kWalkPrime);
    if (cost < best || force_seg > 0) {
      best = cost;
      *seg = s;
    }
  }
  return best;
}

// z handling of the column walk: open (no neighbour past the first and last
// plane), periodic (wrapped), or halo planes (a slab: the planes walked
// always have both z neighbours in storage).
enum WalkZ : int { kWalkZOpen = 0, kWalkZPeriodic = 1, kWalkZHalo = 2 };

// One task of the column walk: trials FLIP_BEFORE / DIR / FLIP_AFTER of
// unit_trials on every unit of column t % ncols over its planes.  PZ is a
// WalkZ (false / true for open / periodic).
template <int C, bool PXY, int PZ, bool FLIP_BEFORE, bool DIR, bool FLIP_AFTER,
          int COH = kLoadNc, class KEY, class PEER = NoPeer>
__device__ __forceinline__ void walk_task(const LatticeView& L, const WalkGeom& W, uint32_t t,
                                          uint32_t step, float d, const Coupling& cp,
                                          const KEY& key, uint32_t replica, unsigned int& nacc,
                                          unsigned int& nflip, const PEER& peer = PEER()) {
  const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
  const uint32_t sg = W.by_cols.div(t);
  const uint32_t col = t - sg * W.ncols;
  const uint32_t j = W.by_Q.div(col);
  const uint32_t q = col - j * W.Q;
  const uint32_t k0 = W.k_first + sg * W.seg;
  const uint32_t k1 = min(k0 + W.seg, W.k_end);
  const uint32_t hx = (uint32_t)L.hx, nj = (uint32_t)L.nj, nk = (uint32_t)L.nk;
  const uint32_t plane = hx * nj;
  const float4* __restrict__ oth = L.col[C ^ 1];
  float4* __restrict__ own = L.col[C];

  // Slot offsets from the unit's own slot, fixed per column: two's
  // complement for negative offsets, so every address is formed as
  // base + (u + offset) with the sum wrapping in 32 bits to the slot index.
  const bool hyp = PXY || j + 1 < nj, hym = PXY || j > 0;
  const uint32_t oyp = j + 1 < nj ? hx : (uint32_t)(-(int32_t)((nj - 1) * hx));
  const uint32_t oym = j > 0 ? (uint32_t)(-(int32_t)hx) : (nj - 1) * hx;
  // the extra x neighbour: parity 0 -> slot 2q-1 (q = 0: the row's last
  // slot), parity 1 -> slot 2q+2 (q = Q-1: slot 0)
  const bool hx0 = PXY || q > 0, hx1 = PXY || q + 1 < W.Q;
  const uint32_t ox0 = q > 0 ? (uint32_t)-1 : 2 * W.Q - 1;
  const uint32_t ox1 = q + 1 < W.Q ? 2u : (uint32_t)(-(int32_t)(2 * q));

  uint32_t u = (k0 * nj + j) * hx + 2 * q;  // own slot of the current step
  uint32_t g = col + W.ncols * k0;          // unit index
  uint32_t o = (C + j + k0) & 1u;

  // pair q of the x-row (j, k0)
  float4 xa, xb;
  {
    const UnitSlots x = ld_other<COH>(oth + u);
    xa = x.a;
    xb = x.b;
  }
  for (uint32_t k = k0; k < k1; ++k) {
    const bool hzp = PZ != kWalkZOpen || k + 1 < nk;
    const uint32_t ozp = (PZ == kWalkZHalo || k + 1 < nk)
                             ? plane
                             : (uint32_t)(-(int32_t)((nk - 1) * plane));
    if (k + 1 < k1) {
      // the next step's own pair and +z pair, the lines no thread has read yet
      asm volatile("prefetch.global.L1 [%0];" ::"l"(own + (u + plane)));
      if (k + 2 < nk) asm volatile("prefetch.global.L1 [%0];" ::"l"(oth + (u + 2 * plane)));
    }
    UnitNbhd U;
    U.cen = own + u;
    const UnitSlots ow = ld_unit(U.cen);
    U.n0 = ow.a;
    U.n1 = ow.b;
    nbr_units<COH>(hyp, oth + (u + oyp), U.nb0.b[2], U.nb1.b[2]);
    nbr_units<COH>(hym, oth + (u + oym), U.nb0.b[3], U.nb1.b[3]);
    float4 pa, pb;  // +z pair: the next step's x-row pair
    nbr_units<COH>(hzp, oth + (u + ozp), pa, pb);
    U.nb0.b[4] = pa;
    U.nb1.b[4] = pb;
    if (PZ != kWalkZOpen || k > 0) {  // -z pair: this thread's x-row pair of the step before
      const UnitSlots zr = ld_other<COH>(
          oth + ((PZ == kWalkZHalo || k > 0) ? u - plane : u + (nk - 1) * plane));
      U.nb0.b[5] = zr.a;
      U.nb1.b[5] = zr.b;
    } else {
      U.nb0.b[5] = U.nb1.b[5] = zero;
    }
    if (o == 0) {
      const float4 e = hx0 ? ld4_other<COH>(oth + (u + ox0)) : zero;
      U.nb0.b[0] = xa;  // +x of i0
      U.nb0.b[1] = e;   // -x of i0
      U.nb1.b[0] = xb;  // +x of i1
      U.nb1.b[1] = xa;  // -x of i1
    } else {
      const float4 e = hx1 ? ld4_other<COH>(oth + (u + ox1)) : zero;
      U.nb0.b[0] = xb;  // +x of i0
      U.nb0.b[1] = xa;  // -x of i0
      U.nb1.b[0] = e;   // +x of i1
      U.nb1.b[1] = xb;  // -x of i1
    }
    unit_trials<C, FLIP_BEFORE, DIR, FLIP_AFTER>(U.n0, U.n1, U.nb0, U.nb1, true, true,
                                                 g + W.goff, step, d, cp, key, replica, nacc,
                                                 nflip);
    st_unit(U.cen, U.n0, U.n1);
    xa = pa;
    xb = pb;
    u += plane;
    g += W.ncols;
    o ^= 1u;
  }
  if (k1 > k0) peer.store_task_ends(own, u - (k1 - k0) * plane, u - plane);
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

// The control update after a fused pass (sweep.cuh FusedPhase), from the
// counts in the control block: B closes the director count (paccept, d) and
// advances the step, A and F close the previous step's flip count (faccept).
// The same update from a pass's closing total (B: director accepts of the
// step, A and F: flips of the previous step) and the control block's fields
// read beforehand (site count, adaptation limit, d).
template <int PHASE>
__device__ __forceinline__ void fused_close(Control* __restrict__ ctl, unsigned long long total,
                                            long long step, long long nsites,
                                            long long adapt_until, double d) {
  const float n3 = (float)nsites;
  if (PHASE == kFusedB) {
    const float pa = (float)total / n3;  // chll_mod.f90:83
    ctl->paccept = pa;
    ctl->nacc_last = (long long)total;
    ctl->nacc = 0;
    if (step < adapt_until) ctl->d = adapt_d(d, pa);
    ctl->step = step + 1;
  } else if (PHASE == kFusedA || PHASE == kFusedF) {
    ctl->faccept = (float)total / n3;  // chll_mod.f90:93
    ctl->nflip_last = (long long)total;
    ctl->nflip = 0;
  }
}

template <int PHASE>
__device__ __forceinline__ void fused_control_update(Control* __restrict__ ctl, long long step) {
  if (PHASE == kFusedB)
    fused_close<PHASE>(ctl, atomicAdd(&ctl->nacc, 0ull), step, ctl->nsites, ctl->adapt_until,
                       ctl->d);
  else if (PHASE == kFusedA || PHASE == kFusedF)
    fused_close<PHASE>(ctl, atomicAdd(&ctl->nflip, 0ull), step, ctl->nsites, ctl->adapt_until,
                       ctl->d);
}

// Programmatic dependent launch (sm_90+): pass kernels are launched so that
// the next pass's grid may be scheduled while this one drains.  Each pass
// first waits for the grids it depends on to complete and their memory to be
// visible (griddepcontrol.wait, before any read of a lattice or a control
// block), and lets its dependents launch once its own units are done
// (griddepcontrol.launch_dependents, before the count epilogue).  Launches
// without the attribute ignore both.
__device__ __forceinline__ void wait_prerequisite_grids() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
}
__device__ __forceinline__ void allow_dependent_grids() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

}  // namespace chll
