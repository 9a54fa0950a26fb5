/*
 * chll_oracle.c -- TEST INFRASTRUCTURE ONLY.  A CPU restatement of the
 * reference's checkerboard Metropolis path (mdeutsc2/ChLLModel,
 * chll/chll_mod.f90) used as the checker for the CUDA library.  Only the
 * tests, __graft_entry__.smoke() and bench.py's CPU-baseline / reference arm
 * may load it; the product path never calls it.
 *
 * It follows the reference's arithmetic: FP64 state and FP64 bond terms, the
 * local energy accumulated in a default-REAL (FP32) variable and rounded
 * after every term (chll_mod.f90:363-412), FP64 proposal arithmetic
 * (chll_mod.f90:149-182), the Metropolis rule of chll_mod.f90:188-200 and
 * 235-243, the step loop with d adaptation of chll_mod.f90:62-110 and etot
 * of chll_mod.f90:414-456 including its boundary mix and the +y typo.
 *
 * Differences from the reference, all deliberate and shared with the GPU:
 *   - randoms come from Philox4x32-10 (Salmon et al., SC'11) keyed on
 *     (seed) and counted on (4-site x-block, step, replica, colour) instead
 *     of the unseeded Fortran random_number stream (chll_mod.f90:58,66-80);
 *     one call (words v0..v3) serves the block's two sites w = 0, 1 of that
 *     colour: director acceptance = top 24 bits of v[w], director angle = the
 *     high (w = 0) or low (w = 1) 16 bits of v2, flip acceptance = top 24
 *     bits of v3 (w = 0) or the 24 bits (v3 & 0xff)<<16 | (v0 & 0xff)<<8 |
 *     (v1 & 0xff) (w = 1).  The call of step t serves the director trials of
 *     step t and the colour-1 flips of step t; the colour-0 flips of step t
 *     use the colour-0 call of step t+1 (they run at the start of the next
 *     step's colour-0 pass on the device);
 *   - a periodic boundary mode and a nematic coupling eps (eps = 1 and open
 *     boundaries reproduce the reference).
 *
 * Arrays are F-order: site (i,j,k), 0-based, at i + ni*(j + nj*k).
 * Colour of a site: (i+j+k)&1; colour 0 is the reference's sl1 (1-based
 * i+j+k odd).  Pass p: 0/1 director trials on colour 0/1, 2/3 flips.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct oracle_cfg {
  int ni, nj, nk, periodic;
  double kT, K, g, eps;
  uint64_t seed;
  uint32_t replica;
  int32_t pad;
} oracle_cfg;

/* ---- Philox4x32-10 ------------------------------------------------------ */
void oracle_philox(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
  uint32_t k0 = key[0], k1 = key[1];
  for (int r = 0; r < 10; ++r) {
    const uint64_t p0 = (uint64_t)0xD2511F53u * c0;
    const uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
    const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
    const uint32_t n1 = (uint32_t)p1;
    const uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
    const uint32_t n3 = (uint32_t)p0;
    c0 = n0; c1 = n1; c2 = n2; c3 = n3;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

static double u01(uint32_t x) { return (double)(x >> 8) * (1.0 / 16777216.0); }
static double u24(uint32_t b24) { return (double)b24 * (1.0 / 16777216.0); }
static double u16(uint32_t b16) { return (double)b16 * (1.0 / 65536.0); }

static size_t at(const oracle_cfg* c, int i, int j, int k) {
  return (size_t)i + (size_t)c->ni * ((size_t)j + (size_t)c->nj * (size_t)k);
}

/* Neighbour coordinate along one axis; returns 0 if absent (open boundary). */
static int nbr(int x, int n, int dir, int periodic, int* out) {
  int y = x + dir;
  if (y < 0 || y >= n) {
    if (!periodic) return 0;
    y = (y + n) % n;
  }
  *out = y;
  return 1;
}

/* energy() of chll_mod.f90:363-412 for trial director (mx,my,mz) and trial
 * chirality snew at site (i,j,k): FP64 terms, FP32 accumulator. */
float oracle_site_energy(const oracle_cfg* c, const double* nx, const double* ny,
                         const double* nz, const int* s, int i, int j, int k, double mx,
                         double my, double mz, int snew) {
  float e = 0.0f;
  const double K = c->K, eps = c->eps;
  int q;
  size_t b;
  double dott, cr, sfac;
  /* +x, -x */
  if (nbr(i, c->ni, +1, c->periodic, &q)) {
    b = at(c, q, j, k);
    dott = mx * nx[b] + my * ny[b] + mz * nz[b];
    cr = my * nz[b] - mz * ny[b];
    sfac = 0.5 * (snew + s[b]);
    e = (float)((double)e + eps * (1.0 - dott * dott) - K * dott * cr * sfac);
  }
  if (nbr(i, c->ni, -1, c->periodic, &q)) {
    b = at(c, q, j, k);
    dott = mx * nx[b] + my * ny[b] + mz * nz[b];
    cr = my * nz[b] - mz * ny[b];
    sfac = 0.5 * (snew + s[b]);
    e = (float)((double)e + eps * (1.0 - dott * dott) + K * dott * cr * sfac);
  }
  /* +y, -y */
  if (nbr(j, c->nj, +1, c->periodic, &q)) {
    b = at(c, i, q, k);
    dott = mx * nx[b] + my * ny[b] + mz * nz[b];
    cr = mz * nx[b] - mx * nz[b];
    sfac = 0.5 * (snew + s[b]);
    e = (float)((double)e + eps * (1.0 - dott * dott) - K * dott * cr * sfac);
  }
  if (nbr(j, c->nj, -1, c->periodic, &q)) {
    b = at(c, i, q, k);
    dott = mx * nx[b] + my * ny[b] + mz * nz[b];
    cr = mz * nx[b] - mx * nz[b];
    sfac = 0.5 * (snew + s[b]);
    e = (float)((double)e + eps * (1.0 - dott * dott) + K * dott * cr * sfac);
  }
  /* +z, -z */
  if (nbr(k, c->nk, +1, c->periodic, &q)) {
    b = at(c, i, j, q);
    dott = mx * nx[b] + my * ny[b] + mz * nz[b];
    cr = mx * ny[b] - my * nx[b];
    sfac = 0.5 * (snew + s[b]);
    e = (float)((double)e + eps * (1.0 - dott * dott) - K * dott * cr * sfac);
  }
  if (nbr(k, c->nk, -1, c->periodic, &q)) {
    b = at(c, i, j, q);
    dott = mx * nx[b] + my * ny[b] + mz * nz[b];
    cr = mx * ny[b] - my * nx[b];
    sfac = 0.5 * (snew + s[b]);
    e = (float)((double)e + eps * (1.0 - dott * dott) + K * dott * cr * sfac);
  }
  e = (float)((double)e - c->g * snew);
  return e;
}

/* Tangent-plane trial director of chll_mod.f90:149-182 (FP64). */
void oracle_propose(double nnx, double nny, double nnz, double d, double u, double* mx,
                    double* my, double* mz) {
  const double twopi = 2.0 * (4.0 * atan(1.0));
  const double phi = u * twopi;
  if (fabs(nnz) > 0.999) {
    const double x = nnx + d * cos(phi), y = nny + d * sin(phi), z = nnz;
    const double r = sqrt(x * x + y * y + z * z);
    *mx = x / r; *my = y / r; *mz = z / r;
  } else {
    double ux = -nny, uy = nnx, uz = 0.0;
    double r = sqrt(ux * ux + uy * uy);
    ux /= r; uy /= r; uz /= r;
    double vx = -nnz * nnx, vy = -nnz * nny, vz = nnx * nnx + nny * nny;
    r = sqrt(vx * vx + vy * vy + vz * vz);
    vx /= r; vy /= r; vz /= r;
    const double dc = d * cos(phi), ds = d * sin(phi);
    double x = nnx + dc * ux + ds * vx;
    double y = nny + dc * uy + ds * vy;
    double z = nnz + dc * uz + ds * vz;
    r = sqrt(x * x + y * y + z * z);
    *mx = x / r; *my = y / r; *mz = z / r;
  }
}

/* One half-sweep.  Returns the number of accepted trials.  Optional per-site
 * outputs (natural order, written only for sites of the pass's colour):
 *   acc: 1 if accepted; de: (double)enew - (double)eold; u: acceptance
 *   uniform.  Sites of one colour have no same-colour neighbour, so the loop
 *   order (and the OpenMP split) does not change the result. */
long long oracle_pass(const oracle_cfg* c, int pass, uint32_t step, double d, double* nx,
                      double* ny, double* nz, int* s, int8_t* acc, double* de, double* u) {
  const int colour = pass & 1;
  const int director = pass < 2;
  const int ng = (c->ni + 3) / 4;
  const uint32_t key[2] = {(uint32_t)c->seed, (uint32_t)(c->seed >> 32)};
  long long count = 0;
#pragma omp parallel for collapse(2) reduction(+ : count) schedule(static)
  for (int k = 0; k < c->nk; ++k) {
    for (int j = 0; j < c->nj; ++j) {
      for (int i = (colour + j + k) & 1; i < c->ni; i += 2) {
        const size_t x = at(c, i, j, k);
        const uint32_t group = (uint32_t)((i >> 2) + (size_t)ng * ((size_t)j + (size_t)c->nj * k));
        const uint32_t cstep = (!director && colour == 0) ? step + 1u : step;
        const uint32_t ctr[4] = {group, cstep, c->replica, (uint32_t)colour};
        uint32_t r[4];
        oracle_philox(ctr, key, r);
        const int w = (i & 3) >> 1;
        const double nnx = nx[x], nny = ny[x], nnz = nz[x];
        const double eold = oracle_site_energy(c, nx, ny, nz, s, i, j, k, nnx, nny, nnz, s[x]);
        double enew, ua;
        double mx = nnx, my = nny, mz = nnz;
        int snew = s[x];
        if (director) {
          oracle_propose(nnx, nny, nnz, d, u16(w ? (r[2] & 0xffffu) : (r[2] >> 16)), &mx, &my,
                         &mz);
          enew = oracle_site_energy(c, nx, ny, nz, s, i, j, k, mx, my, mz, s[x]);
          ua = u01(r[w]);
        } else {
          snew = -s[x];
          enew = oracle_site_energy(c, nx, ny, nz, s, i, j, k, nnx, nny, nnz, snew);
          ua = w ? u24(((r[3] & 0xffu) << 16) | ((r[0] & 0xffu) << 8) | (r[1] & 0xffu))
                 : u01(r[3]);
        }
        int a = 0;
        if (enew < eold)
          a = 1;
        else if (ua <= exp(-(enew - eold) / c->kT))
          a = 1;
        if (a) {
          ++count;
          if (director) {
            nx[x] = mx; ny[x] = my; nz[x] = mz;
          } else {
            s[x] = snew;
          }
        }
        if (acc) acc[x] = (int8_t)a;
        if (de) de[x] = enew - eold;
        if (u) u[x] = ua;
      }
    }
  }
  return count;
}

/* etot() of chll_mod.f90:414-456.  mode 0: the reference's boundaries (x,y
 * periodic, z open) and the +y dot product reading nx(ip1,jp1,k) as at :438;
 * the FP64 sum is stored in *sum and the FP32 per-site value returned.
 * mode 1: every bond once with the lattice's own boundary mode. */
float oracle_etot(const oracle_cfg* c, const double* nx, const double* ny, const double* nz,
                  const int* s, int mode, double* sum) {
  double e = 0.0;
  const double K = c->K, eps = c->eps, g = c->g;
#pragma omp parallel for collapse(2) reduction(+ : e) schedule(static)
  for (int k = 0; k < c->nk; ++k) {
    for (int j = 0; j < c->nj; ++j) {
      for (int i = 0; i < c->ni; ++i) {
        const size_t x = at(c, i, j, k);
        const int per = (mode == 0) ? 1 : c->periodic;
        const int zper = (mode == 0) ? 0 : c->periodic;
        int ip, jp, kp;
        double ddot, cr, sfac;
        if (nbr(i, c->ni, +1, per, &ip)) {
          const size_t b = at(c, ip, j, k);
          ddot = nx[x] * nx[b] + ny[x] * ny[b] + nz[x] * nz[b];
          cr = ny[x] * nz[b] - nz[x] * ny[b];
          sfac = 0.5 * (s[x] + s[b]);
          e += eps * (1.0 - ddot * ddot) - K * ddot * cr * sfac;
        }
        if (nbr(j, c->nj, +1, per, &jp)) {
          const size_t b = at(c, i, jp, k);
          if (mode == 0) {
            const int ipw = (i + 1) % c->ni;
            const size_t t = at(c, ipw, jp, k);
            ddot = nx[x] * nx[t] + ny[x] * ny[b] + nz[x] * nz[b];
          } else {
            ddot = nx[x] * nx[b] + ny[x] * ny[b] + nz[x] * nz[b];
          }
          cr = nz[x] * nx[b] - nx[x] * nz[b];
          sfac = 0.5 * (s[x] + s[b]);
          e += eps * (1.0 - ddot * ddot) - K * ddot * cr * sfac;
        }
        if (nbr(k, c->nk, +1, zper, &kp)) {
          const size_t b = at(c, i, j, kp);
          ddot = nx[x] * nx[b] + ny[x] * ny[b] + nz[x] * nz[b];
          cr = nx[x] * ny[b] - ny[x] * nx[b];
          sfac = 0.5 * (s[x] + s[b]);
          e += eps * (1.0 - ddot * ddot) - K * ddot * cr * sfac;
        }
        e -= g * s[x];
      }
    }
  }
  if (sum) *sum = e;
  const float n3 = (float)((long long)c->ni * c->nj * c->nk);
  return (float)(e / (double)n3);
}

/* FP64 moments: {E (lattice boundary), E_ref (etot mode 0 sum), sum s,
 * sum nx^2, ny^2, nz^2, nx*ny, nx*nz, ny*nz}. */
void oracle_moments(const oracle_cfg* c, const double* nx, const double* ny, const double* nz,
                    const int* s, double out[9]) {
  oracle_etot(c, nx, ny, nz, s, 1, &out[0]);
  oracle_etot(c, nx, ny, nz, s, 0, &out[1]);
  double a2 = 0, a3 = 0, a4 = 0, a5 = 0, a6 = 0, a7 = 0, a8 = 0;
  const size_t n = (size_t)c->ni * c->nj * c->nk;
#pragma omp parallel for reduction(+ : a2, a3, a4, a5, a6, a7, a8) schedule(static)
  for (size_t x = 0; x < n; ++x) {
    a2 += s[x];
    a3 += nx[x] * nx[x];
    a4 += ny[x] * ny[x];
    a5 += nz[x] * nz[x];
    a6 += nx[x] * ny[x];
    a7 += nx[x] * nz[x];
    a8 += ny[x] * nz[x];
  }
  out[2] = a2; out[3] = a3; out[4] = a4; out[5] = a5; out[6] = a6; out[7] = a7; out[8] = a8;
}

/* The reference step loop (chll_mod.f90:62-110) on the Philox stream.
 * Fills msteps[r] and m[col*rows + r] (F-order rows x 5) for measured steps,
 * at most `rows` of them; returns the number of measured steps. */
int oracle_run(const oracle_cfg* c, int nstart, int nstop, int nout, long long adapt_until,
               double* d, double* nx, double* ny, double* nz, int* s, int* msteps, double* m,
               int rows) {
  const long long n3 = (long long)c->ni * c->nj * c->nk;
  int mc = 0;
  for (int istep = nstart; istep <= nstop; ++istep) {
    long long naccept = 0, nflip = 0;
    naccept += oracle_pass(c, 0, (uint32_t)istep, *d, nx, ny, nz, s, NULL, NULL, NULL);
    naccept += oracle_pass(c, 1, (uint32_t)istep, *d, nx, ny, nz, s, NULL, NULL, NULL);
    nflip += oracle_pass(c, 2, (uint32_t)istep, *d, nx, ny, nz, s, NULL, NULL, NULL);
    nflip += oracle_pass(c, 3, (uint32_t)istep, *d, nx, ny, nz, s, NULL, NULL, NULL);
    const double paccept = (double)((float)naccept / (float)n3);
    if (istep < adapt_until) {
      if (paccept < 0.4)
        *d = *d * (double)0.995f;
      else if (paccept > 0.6)
        *d = *d / (double)0.995f;
    }
    if (istep % nout == 0) {
      const double faccept = (double)((float)nflip / (float)n3);
      const double total_energy = oracle_etot(c, nx, ny, nz, s, 0, NULL);
      float ssum = 0.0f;
      for (long long x = 0; x < n3; ++x) ssum += (float)s[x];
      const double e_excess = (double)(ssum / (float)n3);
      if (mc < rows) {
        if (msteps) msteps[mc] = istep;
        if (m) {
          m[0 * rows + mc] = total_energy;
          m[1 * rows + mc] = e_excess;
          m[2 * rows + mc] = paccept;
          m[3 * rows + mc] = faccept;
          m[4 * rows + mc] = *d;
        }
      }
      ++mc;
    }
  }
  return mc;
}

/* An equilibrium chain of the same step loop, for the statistical parity
 * tests: sweeps istep = 1 .. burn + nmeas*every with the d rule while
 * istep < adapt_until, and after sweep burn, every `every` sweeps, the nine
 * FP64 moments of oracle_moments appended to out (nmeas x 9).  *d is the
 * proposal amplitude in and out. */
int oracle_chain(const oracle_cfg* c, int burn, int nmeas, int every, long long adapt_until,
                 double* d, double* nx, double* ny, double* nz, int* s, double* out) {
  const long long n3 = (long long)c->ni * c->nj * c->nk;
  const int total = burn + nmeas * every;
  int mc = 0;
  for (int istep = 1; istep <= total; ++istep) {
    long long naccept = 0;
    naccept += oracle_pass(c, 0, (uint32_t)istep, *d, nx, ny, nz, s, NULL, NULL, NULL);
    naccept += oracle_pass(c, 1, (uint32_t)istep, *d, nx, ny, nz, s, NULL, NULL, NULL);
    oracle_pass(c, 2, (uint32_t)istep, *d, nx, ny, nz, s, NULL, NULL, NULL);
    oracle_pass(c, 3, (uint32_t)istep, *d, nx, ny, nz, s, NULL, NULL, NULL);
    const double paccept = (double)((float)naccept / (float)n3);
    if (istep < adapt_until) {
      if (paccept < 0.4)
        *d = *d * (double)0.995f;
      else if (paccept > 0.6)
        *d = *d / (double)0.995f;
    }
    if (istep > burn && (istep - burn) % every == 0 && mc < nmeas) {
      oracle_moments(c, nx, ny, nz, s, out + 9 * (size_t)mc);
      ++mc;
    }
  }
  return mc;
}

/* Random initial state on the device's stream: counter {site, 0xffffffff,
 * replica, 4}; cos(theta) = 2u0-1, phi = 2*pi*u1, s = -1 if u2 < 1/2. */
void oracle_init_random(const oracle_cfg* c, double* nx, double* ny, double* nz, int* s) {
  const uint32_t key[2] = {(uint32_t)c->seed, (uint32_t)(c->seed >> 32)};
  const size_t n = (size_t)c->ni * c->nj * c->nk;
  const double twopi = 2.0 * (4.0 * atan(1.0));
  for (size_t x = 0; x < n; ++x) {
    const uint32_t ctr[4] = {(uint32_t)x, 0xffffffffu, c->replica, 4u};
    uint32_t r[4];
    oracle_philox(ctr, key, r);
    const double ct = 2.0 * u01(r[0]) - 1.0;
    const double st = sqrt(fmax(0.0, 1.0 - ct * ct));
    const double phi = u01(r[1]) * twopi;
    nx[x] = st * cos(phi);
    ny[x] = st * sin(phi);
    nz[x] = ct;
    s[x] = (u01(r[2]) < 0.5) ? -1 : 1;
  }
}

/* FP64 energy gradient: g = dE/dn for every site (optionally projected on
 * the tangent plane) and out4 = {E, dE/deps, dE/dK, dE/dh}, E with the
 * lattice's boundary mode, each bond once. */
void oracle_energy_grad(const oracle_cfg* c, const double* nx, const double* ny,
                        const double* nz, const int* s, double* gx, double* gy, double* gz,
                        int project, double out4[4]) {
  const double K = c->K, eps = c->eps;
  double E = 0, dEe = 0, dEK = 0, dEh = 0;
#pragma omp parallel for collapse(2) reduction(+ : E, dEe, dEK, dEh) schedule(static)
  for (int k = 0; k < c->nk; ++k) {
    for (int j = 0; j < c->nj; ++j) {
      for (int i = 0; i < c->ni; ++i) {
        const size_t x = at(c, i, j, k);
        const double n[3] = {nx[x], ny[x], nz[x]};
        double g[3] = {0, 0, 0};
        for (int a = 0; a < 3; ++a) {
          for (int dir = -1; dir <= 1; dir += 2) {
            int q;
            const int coord = a == 0 ? i : (a == 1 ? j : k);
            const int len = a == 0 ? c->ni : (a == 1 ? c->nj : c->nk);
            if (!nbr(coord, len, dir, c->periodic, &q)) continue;
            const size_t y = a == 0 ? at(c, q, j, k) : (a == 1 ? at(c, i, q, k) : at(c, i, j, q));
            const double b[3] = {nx[y], ny[y], nz[y]};
            const double cc = n[0] * b[0] + n[1] * b[1] + n[2] * b[2];
            double X, bxe[3];
            if (a == 0) {
              X = n[1] * b[2] - n[2] * b[1];
              bxe[0] = 0; bxe[1] = b[2]; bxe[2] = -b[1];
            } else if (a == 1) {
              X = n[2] * b[0] - n[0] * b[2];
              bxe[0] = -b[2]; bxe[1] = 0; bxe[2] = b[0];
            } else {
              X = n[0] * b[1] - n[1] * b[0];
              bxe[0] = b[1]; bxe[1] = -b[0]; bxe[2] = 0;
            }
            const double sbar = 0.5 * (s[x] + s[y]);
            const double sigma = (dir > 0) ? -1.0 : 1.0;
            for (int t = 0; t < 3; ++t)
              g[t] += -2.0 * eps * cc * b[t] + sigma * K * sbar * (X * b[t] + cc * bxe[t]);
            if (dir > 0) {
              E += eps * (1.0 - cc * cc) - K * cc * X * sbar;
              dEe += 1.0 - cc * cc;
              dEK += -cc * X * sbar;
            }
          }
        }
        E -= c->g * s[x];
        dEh -= s[x];
        if (project) {
          const double nn = n[0] * n[0] + n[1] * n[1] + n[2] * n[2];
          const double gn = (g[0] * n[0] + g[1] * n[1] + g[2] * n[2]) / nn;
          for (int t = 0; t < 3; ++t) g[t] -= gn * n[t];
        }
        if (gx) { gx[x] = g[0]; gy[x] = g[1]; gz[x] = g[2]; }
      }
    }
  }
  out4[0] = E; out4[1] = dEe; out4[2] = dEK; out4[3] = dEh;
}

int oracle_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

void oracle_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}
