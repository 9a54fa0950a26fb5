// Shared device/host definitions of the B200 chiral Lebwohl-Lasher library:
// the counter-based random stream, the red/black float4 lattice view, the
// coupling constants and the per-replica control block that the sweep
// kernels update on the device.
//
// Physics (restated from the reference module chll/chll_mod.f90):
//   local energy of site i with director n and chirality s
//     E_i = sum_b [ eps*(1 - (n.n_b)^2) + sigma_b*K*(n.n_b)*((n x n_b).e_b)*(s+s_b)/2 ] - g*s
//   over the six neighbours b, sigma_b = -1 for the +axis neighbour and +1
//   for the -axis neighbour (chll_mod.f90:363-412; eps = 1 in the reference).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace chll {

// ---------------------------------------------------------------------------
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel Random Numbers: As Easy
// as 1, 2, 3", SC'11): ten rounds of two 32x32->64 multiplies with the
// published multipliers, the key bumped by the published Weyl increments
// between rounds.  Counters used by this library:
//   sweeps      : {group, step', replica, colour}
//   random init : {site,  0xffffffff, replica, kStreamInit}
// where group = (i>>2) + (ceil(ni/4)) * (j + nj*k) is the index of the
// 4-site x-block holding the site (two sites of each colour), and
// site = i + ni*(j + nj*k) (0-based, F-order).  One sweep call (words
// v0..v3) gives the block's two sites w = 0, 1 of its colour all their
// uniforms (UnitRandoms): director acceptance = top 24 bits of v[w],
// director angle = the high (w = 0) or low (w = 1) 16 bits of v2, flip
// acceptance = top 24 bits of v3 (w = 0) or the 24 bits
// (v3 & 0xff)<<16 | (v0 & 0xff)<<8 | (v1 & 0xff) (w = 1).  step' is the step
// for the director trials and the colour-1 flips of a step, and the next step
// for the colour-0 flips (which the fused sweep runs at the start of the next
// step's colour-0 pass): every pass then needs exactly one call per block.
// ---------------------------------------------------------------------------
struct Ctr4 {
  uint32_t v[4];
};

constexpr uint32_t kPhiloxM0 = 0xD2511F53u, kPhiloxM1 = 0xCD9E8D57u;
constexpr uint32_t kPhiloxW0 = 0x9E3779B9u, kPhiloxW1 = 0xBB67AE85u;

// One Philox round with round key (ka, kb).
__host__ __device__ __forceinline__ Ctr4 philox_round(Ctr4 c, uint32_t ka, uint32_t kb) {
  const uint64_t p0 = (uint64_t)kPhiloxM0 * c.v[0];
  const uint64_t p1 = (uint64_t)kPhiloxM1 * c.v[2];
  Ctr4 n;
  n.v[0] = (uint32_t)(p1 >> 32) ^ c.v[1] ^ ka;
  n.v[1] = (uint32_t)p1;
  n.v[2] = (uint32_t)(p0 >> 32) ^ c.v[3] ^ kb;
  n.v[3] = (uint32_t)p0;
  return n;
}

__host__ __device__ __forceinline__ Ctr4 philox4x32_10(Ctr4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    c = philox_round(c, k0, k1);
    k0 += kPhiloxW0;
    k1 += kPhiloxW1;
  }
  return c;
}

// The ten round keys of one key, computed once on the host and passed to a
// kernel by value: the rounds then read them as launch constants instead of
// bumping the key in registers.
struct PhiloxKeys {
  uint32_t a[10], b[10];
};

__host__ __device__ inline PhiloxKeys philox_keys(uint32_t k0, uint32_t k1) {
  PhiloxKeys K;
  for (int r = 0; r < 10; ++r) {
    K.a[r] = k0 + (uint32_t)r * kPhiloxW0;
    K.b[r] = k1 + (uint32_t)r * kPhiloxW1;
  }
  return K;
}

// A key as its two words; the rounds bump it in registers.
struct KeyPair {
  uint32_t k0, k1;
};

__host__ __device__ __forceinline__ Ctr4 philox4x32_10(Ctr4 c, const KeyPair& K) {
  return philox4x32_10(c, K.k0, K.k1);
}

__host__ __device__ __forceinline__ Ctr4 philox4x32_10(Ctr4 c, const PhiloxKeys& K) {
#pragma unroll
  for (int r = 0; r < 10; ++r) c = philox_round(c, K.a[r], K.b[r]);
  return c;
}

// Top 24 bits of a word as a uniform in [0,1): exact in FP32 and FP64, so the
// host oracle and the device read identical numbers.
__host__ __device__ __forceinline__ float u01(uint32_t x) {
  return (float)(x >> 8) * 5.9604644775390625e-8f;  // 2^-24
}

// A float from its bits.
__host__ __device__ __forceinline__ float float_of_bits(uint32_t b) {
#ifdef __CUDA_ARCH__
  return __uint_as_float(b);
#else
  float f;
  __builtin_memcpy(&f, &b, sizeof f);
  return f;
#endif
}

// b * 2^-16 - 1/2 for a 16-bit b given as b << 7: the float 1 + b * 2^-16 is
// assembled from its bits (the exponent of 1, b at the top of the mantissa)
// and 1.5 subtracted, both exact, with no integer-to-float conversion.
__host__ __device__ __forceinline__ float centred_u16(uint32_t b16_shl7) {
  return float_of_bits(0x3f800000u | b16_shl7) - 1.5f;
}

// The uniforms of one block and colour from its sweep call (see above).
struct UnitRandoms {
  float acc[2];   // director acceptance
  float ang[2];   // director angle uniform u minus 1/2 (16-bit u), in [-1/2, 1/2)
  float flip[2];  // chirality-flip acceptance
};

__host__ __device__ __forceinline__ UnitRandoms unit_randoms(const Ctr4& r) {
  UnitRandoms u;
  u.acc[0] = u01(r.v[0]);
  u.acc[1] = u01(r.v[1]);
  u.ang[0] = centred_u16((r.v[2] >> 9) & 0x007fff80u);  // high 16 bits of v2
  u.ang[1] = centred_u16((r.v[2] << 7) & 0x007fff80u);  // low 16 bits
  u.flip[0] = u01(r.v[3]);
  u.flip[1] = (float)(((r.v[3] & 0xffu) << 16) | ((r.v[0] & 0xffu) << 8) | (r.v[1] & 0xffu)) *
              5.9604644775390625e-8f;
  return u;
}

enum Pass : uint32_t {
  kPassDir0 = 0,   // director trials on colour 0 (reference sublattice sl1)
  kPassDir1 = 1,   // director trials on colour 1 (sl2)
  kPassSpin0 = 2,  // chirality flips on colour 0
  kPassSpin1 = 3,  // chirality flips on colour 1
  kStreamInit = 4  // random initial state
};

// ---------------------------------------------------------------------------
// Red/black float4 lattice.  Site (i,j,k), 0-based, has colour
// c = (i+j+k)&1; colour 0 is the reference's "odd" sublattice sl1 (1-based
// i+j+k odd, chll_mod.f90:27).  Each colour is a dense array
//   col[c][(k*nj + j)*hx + h],   i = 2h + ((c+j+k)&1),
// of float4 (nx, ny, nz, s) with hx = ni_p/2 and ni_p = ni rounded up to a
// multiple of 4.  Storage slots with i >= ni are padding, held at zero.
// ---------------------------------------------------------------------------
struct LatticeView {
  float4* col[2];
  int ni, nj, nk;
  int hx;        // storage half-row length (even)
  int periodic;  // 0: open boundaries (reference sweep), 1: periodic
};

__host__ __device__ __forceinline__ int padded_ni(int ni) { return (ni + 3) & ~3; }

// The sweep kernels move a unit (two float4 slots) with one 256-bit access,
// which needs both colour arrays 32-byte aligned and rows of an even number
// of slots.
__host__ inline bool unit_view_aligned(const LatticeView& L) {
  return (L.hx % 2) == 0 && ((uintptr_t)L.col[0] % 32) == 0 && ((uintptr_t)L.col[1] % 32) == 0;
}

// Colour array by a runtime colour, as a select rather than an indexed load
// (an indexed access would move the whole view to local memory).
__host__ __device__ __forceinline__ float4* colour_array(const LatticeView& L, int c) {
  return c ? L.col[1] : L.col[0];
}

// Division of x < 2^31 by a fixed divisor d >= 1 as one 32x32->64 multiply
// and a shift: with s = ceil(log2 d), m = ceil(2^(31+s)/d) < 2^32 and
// x*m = x*2^(31+s)/d + x*e/d (0 <= e < d), the error term is below
// 2^31*d/(d*2^(31+s)) = 2^-s <= 1/d, so floor(x*m / 2^(31+s)) = floor(x/d)
// (Granlund and Montgomery, "Division by invariant integers using
// multiplication", PLDI 1994).
struct FastDiv {
  uint32_t d, m, shift;  // shift = 31 + s

  __host__ __device__ FastDiv() : d(1), m(0x80000000u), shift(31) {}
  __host__ explicit FastDiv(uint32_t divisor) : d(divisor) {
    uint32_t s = 0;
    while ((1ull << s) < divisor) ++s;
    shift = 31 + s;
    const unsigned __int128 num = (unsigned __int128)1 << shift;
    m = (uint32_t)((num + divisor - 1) / divisor);
  }
  __host__ __device__ __forceinline__ uint32_t div(uint32_t x) const {
    return (uint32_t)(((uint64_t)x * m) >> shift);
  }
};

struct Coupling {
  float eps;     // nematic coupling (reference: 1)
  float K;       // chiral coupling KK
  float g;       // field on the chirality
  float inv_kT;  // 1/kT (+inf at kT = 0, as the reference's division gives)
};

// Couplings in FP64 for the FP64 observables and adjoint sums, so that a
// coupling such as eps = 1.2 enters those sums unrounded.
struct CouplingD {
  double eps, K, g;
};

// Per-replica control block, resident in device memory so that graph-captured
// sweep loops need no host round trip (chll_mod.f90:62-90).
struct Control {
  double d;                  // proposal amplitude (reference: d, FP64)
  long long step;            // step number of the sweep in progress
  long long adapt_until;     // d is adapted after sweeps with step < adapt_until
  long long nsites;          // real site count ni*nj*nk
  unsigned long long nacc;   // director accepts in the current sweep
  unsigned long long nflip;  // chirality flips in the current sweep
  unsigned int done;         // blocks finished in the current pass
  unsigned int status;       // nonzero: device-detected error
  float paccept;             // accepted director fraction of the last sweep
  float faccept;             // accepted flip fraction of the last sweep
  long long nacc_last;       // raw counts of the last sweep
  long long nflip_last;
  int deferred;              // nonzero: passes only count; the epilogue runs apart
                             // (a slab, whose counts are summed over ranks first)
  int pad;
};

// Row written by the observables kernel (FP64).  Columns 0-4 are the
// reference's measurement row m(r,1:5) (chll_mod.f90:99-104).
enum RowCol : int {
  kRowEtotRef = 0,  // etot() per site, reference boundary quirks, FP32-rounded
  kRowEta = 1,      // sum(s)/N in FP32
  kRowPaccept = 2,
  kRowFaccept = 3,
  kRowD = 4,
  kRowEnergy = 5,   // total energy (sweep boundary), FP64
  kRowSumS = 6,     // sum of s
  kRowQxx = 7,      // sum nx*nx ... (Q-tensor raw moments)
  kRowQyy = 8,
  kRowQzz = 9,
  kRowQxy = 10,
  kRowQxz = 11,
  kRowQyz = 12,
  kRowEtotRefSum = 13,  // FP64 sum behind column 0
  kRowStep = 14,
  kRowNsites = 15,
  kRowLen = 16
};

constexpr int kObsMoments = 9;  // E, E_ref, sum s, 6 Q sums

}  // namespace chll
