// C ABI of libchll_mod.so: the reference's init/run entry points
// (chll/chll_mod.f90:9-115, bound by chll/chll.py:9-36) and the chll_*
// extensions declared in include/chll_mod.h.
//
// Host flow of run(): upload the caller's FP64 F-order arrays, pack them into
// the red/black float4 lattice, run the steps as CUDA-graph chunks that end at
// measurement steps, measure on the device, and unpack/download at the end.
// Step size adaptation and accept fractions live in the device control block,
// so no chunk needs a host round trip; measurement rows are copied back
// asynchronously and printed as they complete.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/chll_mod.h"
#include "chll_common.cuh"
#include "moments.cuh"
#include "sweep.cuh"
#include "sweep_unit.cuh"

using chll::Control;
using chll::Coupling;
using chll::LatticeView;

// ---------------------------------------------------------------------------
// Errors
// ---------------------------------------------------------------------------
namespace {

thread_local int t_status = CHLL_OK;
thread_local std::string t_error;

int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  t_status = code;
  t_error = buf;
  return code;
}

int ok() {
  t_status = CHLL_OK;
  t_error.clear();
  return CHLL_OK;
}

#define CHLL_CUDA_TRY(expr)                                                              \
  do {                                                                                   \
    cudaError_t _e = (expr);                                                             \
    if (_e != cudaSuccess) {                                                             \
      return fail(_e == cudaErrorMemoryAllocation ? CHLL_ENOMEM : CHLL_ECUDA, "%s: %s (%s:%d)", \
                  #expr, cudaGetErrorString(_e), __FILE__, __LINE__);                    \
    }                                                                                    \
  } while (0)

#define CHLL_TRY(expr)               \
  do {                               \
    int _r = (expr);                 \
    if (_r != CHLL_OK) return _r;    \
  } while (0)

std::mutex g_run_mutex;
uint64_t g_seed = 1;
uint32_t g_run_ordinal = 0;

uint32_t seed_lo(uint64_t s) { return (uint32_t)s; }
uint32_t seed_hi(uint64_t s) { return (uint32_t)(s >> 32); }

Coupling make_coupling(const chll_coupling& c) {
  Coupling cp;
  cp.eps = (float)c.eps;
  cp.K = (float)c.K;
  cp.g = (float)c.g;
  cp.inv_kT = (float)(1.0 / c.kT);  // +inf at kT = 0
  return cp;
}

chll::CouplingD make_coupling_d(const chll_coupling& c) {
  chll::CouplingD cd;
  cd.eps = c.eps;
  cd.K = c.K;
  cd.g = c.g;
  return cd;
}

bool same_coupling(const Coupling& a, const Coupling& b) {
  return std::memcmp(&a, &b, sizeof(Coupling)) == 0;
}

bool is_device_ptr(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

int check_device() {
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) {
    cudaGetLastError();
    return fail(CHLL_ECUDA, "no CUDA device available (%s); libchll_mod has no CPU path",
                e == cudaSuccess ? "0 devices" : cudaGetErrorString(e));
  }
  return CHLL_OK;
}

}  // namespace

namespace chll {
// Error recording for entry points defined in other translation units.
int record_error(int code, const char* msg) { return fail(code, "%s", msg); }
int record_ok() { return ok(); }
}  // namespace chll

// ---------------------------------------------------------------------------
// Lattice object
// ---------------------------------------------------------------------------
struct GraphEntry {
  int nsweeps = 0;
  Coupling cp{};
  uint32_t key0 = 0, key1 = 0, replica = 0;
  cudaGraphExec_t exec = nullptr;
  uint64_t last_use = 0;
};

struct chll_lattice {
  int ni = 0, nj = 0, nk = 0, hx = 0, periodic = 0;
  long long nsites = 0;
  size_t per_colour = 0;
  int device = 0;
  float4* lat = nullptr;
  Control* ctl = nullptr;
  double* partials = nullptr;
  unsigned int* tickets = nullptr;  // [0] observables, [1] gradient
  double* rows = nullptr;
  int rows_cap = 0;
  double* out4 = nullptr;
  void* staging = nullptr;
  size_t staging_bytes = 0;
  float4* grad = nullptr;
  cudaStream_t own_stream = nullptr;
  cudaStream_t capture_stream = nullptr;
  cudaStream_t stream = nullptr;
  std::vector<GraphEntry> graphs;
  uint64_t use_clock = 0;
  int kernel = chll::kSweepAuto;
  // z-slab of a larger lattice: global planes z0 .. z0+nk-1 of nk_global,
  // stored as planes 2 .. nk+1 of nk+3 (plane 1 and nk+2 are the halos,
  // plane 0 keeps the storage checkerboard equal to the global one).
  int slab = 0, z0 = 0, nk_global = 0;
  long long ctl_sites = 0;  // sites of the whole lattice (acceptance fractions)
  // where a slab's first / last own plane of each colour is also written by
  // its passes (the neighbouring slabs' halo planes), or null
  float4* peer_lo[2] = {nullptr, nullptr};
  float4* peer_hi[2] = {nullptr, nullptr};

  int store_planes() const { return slab ? nk + 3 : nk; }
  // The lattice's own sites (a slab's interior planes).
  LatticeView view() const {
    const size_t off = slab ? (size_t)2 * hx * nj : 0;
    LatticeView v;
    v.col[0] = lat + off;
    v.col[1] = lat + per_colour + off;
    v.ni = ni;
    v.nj = nj;
    v.nk = nk;
    v.hx = hx;
    v.periodic = periodic;
    return v;
  }
  // All stored planes (a slab with its halos).
  LatticeView store_view() const {
    LatticeView v = view();
    v.col[0] = lat;
    v.col[1] = lat + per_colour;
    v.nk = store_planes();
    return v;
  }
};

namespace {

int ensure_staging(chll_lattice* L, size_t bytes) {
  if (L->staging_bytes >= bytes) return CHLL_OK;
  if (L->staging) cudaFree(L->staging);
  L->staging = nullptr;
  L->staging_bytes = 0;
  CHLL_CUDA_TRY(cudaMalloc(&L->staging, bytes));
  L->staging_bytes = bytes;
  return CHLL_OK;
}

int ensure_rows(chll_lattice* L, int rows) {
  if (L->rows_cap >= rows) return CHLL_OK;
  if (L->rows) cudaFree(L->rows);
  L->rows = nullptr;
  L->rows_cap = 0;
  CHLL_CUDA_TRY(cudaMalloc(&L->rows, sizeof(double) * chll::kRowLen * (size_t)rows));
  L->rows_cap = rows;
  return CHLL_OK;
}

void drop_graphs(chll_lattice* L) {
  for (auto& g : L->graphs)
    if (g.exec) cudaGraphExecDestroy(g.exec);
  L->graphs.clear();
}

// Returns an executable graph of `nsweeps` steps for this coupling and key,
// capturing it on first use: 2 fused passes per step plus a closing flip
// pass, or the reference's 4 half-sweeps per step.
int get_graph(chll_lattice* L, const Coupling& cp, uint32_t k0, uint32_t k1, uint32_t rep,
              int nsweeps, cudaGraphExec_t* out) {
  for (auto& g : L->graphs) {
    if (g.nsweeps == nsweeps && g.key0 == k0 && g.key1 == k1 && g.replica == rep &&
        same_coupling(g.cp, cp)) {
      g.last_use = ++L->use_clock;
      *out = g.exec;
      return CHLL_OK;
    }
  }
  const LatticeView v = L->view();
  // auto: the resident cluster launch where its threads hold at most one
  // unit per pass (a pass is then mostly latency: up to 32^3), else the fused
  // passes (decided before the capture, which the cluster query must not
  // meet)
  const bool resident =
      L->kernel == chll::kSweepResident ||
      (L->kernel == chll::kSweepAuto && chll::resident_cluster() > 0 &&
       chll::resident_units_per_thread(v) <= 1);
  cudaGraph_t graph = nullptr;
  CHLL_CUDA_TRY(cudaStreamBeginCapture(L->capture_stream, cudaStreamCaptureModeThreadLocal));
  if (resident) {
    // the whole chunk in one cluster launch
    if (chll::launch_resident_sweeps(v, cp, k0, k1, rep, L->ctl, nsweeps, L->capture_stream)) {
      cudaGraph_t g = nullptr;
      cudaStreamEndCapture(L->capture_stream, &g);
      if (g) cudaGraphDestroy(g);
      cudaGetLastError();
      return fail(CHLL_ECUDA, "resident sweep launch failed");
    }
  } else if (L->kernel == chll::kSweepAuto || L->kernel == chll::kSweepFused) {
    // A0 B (A B)... F: the fused two-pass sweep, flips completed at the end
    for (int s = 0; s < nsweeps; ++s) {
      chll::launch_fused_pass(v, cp, k0, k1, rep, L->ctl, s ? chll::kFusedA : chll::kFusedA0,
                              L->capture_stream);
      chll::launch_fused_pass(v, cp, k0, k1, rep, L->ctl, chll::kFusedB, L->capture_stream);
    }
    chll::launch_fused_pass(v, cp, k0, k1, rep, L->ctl, chll::kFusedF, L->capture_stream);
  } else {
    for (int s = 0; s < nsweeps; ++s)
      for (int p = 0; p < 4; ++p)
        chll::launch_sweep_pass(v, cp, k0, k1, rep, L->ctl, p, L->capture_stream, L->kernel);
  }
  cudaError_t e = cudaStreamEndCapture(L->capture_stream, &graph);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(CHLL_ECUDA, "graph capture failed: %s", cudaGetErrorString(e));
  }
  cudaGraphExec_t exec = nullptr;
  e = cudaGraphInstantiate(&exec, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) return fail(CHLL_ECUDA, "graph instantiate: %s", cudaGetErrorString(e));
  if (L->graphs.size() >= 6) {
    auto victim = std::min_element(L->graphs.begin(), L->graphs.end(),
                                   [](const GraphEntry& a, const GraphEntry& b) {
                                     return a.last_use < b.last_use;
                                   });
    cudaGraphExecDestroy(victim->exec);
    L->graphs.erase(victim);
  }
  GraphEntry g;
  g.nsweeps = nsweeps;
  g.cp = cp;
  g.key0 = k0;
  g.key1 = k1;
  g.replica = rep;
  g.exec = exec;
  g.last_use = ++L->use_clock;
  L->graphs.push_back(g);
  *out = exec;
  return CHLL_OK;
}

constexpr int kGraphChunk = 100;

int sweep_impl(chll_lattice* L, const Coupling& cp, uint64_t seed, uint32_t rep, int nsweeps) {
  if (nsweeps <= 0) return CHLL_OK;
  const uint32_t k0 = seed_lo(seed), k1 = seed_hi(seed);
  const int chunk = std::min(nsweeps, kGraphChunk);
  const int full = nsweeps / chunk, rest = nsweeps % chunk;
  cudaGraphExec_t exec = nullptr;
  CHLL_TRY(get_graph(L, cp, k0, k1, rep, chunk, &exec));
  for (int c = 0; c < full; ++c) CHLL_CUDA_TRY(cudaGraphLaunch(exec, L->stream));
  if (rest) {
    CHLL_TRY(get_graph(L, cp, k0, k1, rep, rest, &exec));
    CHLL_CUDA_TRY(cudaGraphLaunch(exec, L->stream));
  }
  CHLL_CUDA_TRY(cudaGetLastError());
  return CHLL_OK;
}

int upload_f64_impl(chll_lattice* L, const double* nx, const double* ny, const double* nz,
                    const int* s) {
  if (!nx || !ny || !nz || !s) return fail(CHLL_EINVAL, "upload: null array");
  const size_t n = (size_t)L->nsites;
  const LatticeView v = L->view();
  CHLL_CUDA_TRY(cudaMemsetAsync(L->lat, 0, 2 * L->per_colour * sizeof(float4), L->stream));
  if (is_device_ptr(nx) && is_device_ptr(ny) && is_device_ptr(nz) && is_device_ptr(s)) {
    chll::launch_pack_f64(v, nx, ny, nz, s, L->stream);
  } else {
    CHLL_TRY(ensure_staging(L, n * (3 * sizeof(double) + sizeof(int))));
    double* dx = (double*)L->staging;
    double* dy = dx + n;
    double* dz = dy + n;
    int* ds = (int*)(dz + n);
    CHLL_CUDA_TRY(cudaMemcpyAsync(dx, nx, n * sizeof(double), cudaMemcpyDefault, L->stream));
    CHLL_CUDA_TRY(cudaMemcpyAsync(dy, ny, n * sizeof(double), cudaMemcpyDefault, L->stream));
    CHLL_CUDA_TRY(cudaMemcpyAsync(dz, nz, n * sizeof(double), cudaMemcpyDefault, L->stream));
    CHLL_CUDA_TRY(cudaMemcpyAsync(ds, s, n * sizeof(int), cudaMemcpyDefault, L->stream));
    chll::launch_pack_f64(v, dx, dy, dz, ds, L->stream);
  }
  CHLL_CUDA_TRY(cudaGetLastError());
  return CHLL_OK;
}

int download_f64_impl(chll_lattice* L, double* nx, double* ny, double* nz, int* s) {
  if (!nx || !ny || !nz || !s) return fail(CHLL_EINVAL, "download: null array");
  const size_t n = (size_t)L->nsites;
  const LatticeView v = L->view();
  if (is_device_ptr(nx) && is_device_ptr(ny) && is_device_ptr(nz) && is_device_ptr(s)) {
    chll::launch_unpack_f64(v, nx, ny, nz, s, L->stream);
    CHLL_CUDA_TRY(cudaGetLastError());
    CHLL_CUDA_TRY(cudaStreamSynchronize(L->stream));
    return CHLL_OK;
  }
  CHLL_TRY(ensure_staging(L, n * (3 * sizeof(double) + sizeof(int))));
  double* dx = (double*)L->staging;
  double* dy = dx + n;
  double* dz = dy + n;
  int* ds = (int*)(dz + n);
  chll::launch_unpack_f64(v, dx, dy, dz, ds, L->stream);
  CHLL_CUDA_TRY(cudaGetLastError());
  CHLL_CUDA_TRY(cudaMemcpyAsync(nx, dx, n * sizeof(double), cudaMemcpyDefault, L->stream));
  CHLL_CUDA_TRY(cudaMemcpyAsync(ny, dy, n * sizeof(double), cudaMemcpyDefault, L->stream));
  CHLL_CUDA_TRY(cudaMemcpyAsync(nz, dz, n * sizeof(double), cudaMemcpyDefault, L->stream));
  CHLL_CUDA_TRY(cudaMemcpyAsync(s, ds, n * sizeof(int), cudaMemcpyDefault, L->stream));
  CHLL_CUDA_TRY(cudaStreamSynchronize(L->stream));
  return CHLL_OK;
}

int set_control_impl(chll_lattice* L, double d, long long step, long long adapt_until) {
  Control c;
  std::memset(&c, 0, sizeof(c));
  c.d = d;
  c.step = step;
  c.adapt_until = adapt_until;
  c.nsites = L->ctl_sites;
  c.deferred = L->slab;
  CHLL_CUDA_TRY(cudaMemcpyAsync(L->ctl, &c, sizeof(c), cudaMemcpyHostToDevice, L->stream));
  CHLL_CUDA_TRY(cudaStreamSynchronize(L->stream));
  return CHLL_OK;
}

int observe_impl(chll_lattice* L, const chll::CouplingD& cp, double* dev_row, long long step) {
  const LatticeView v = L->view();
  const chll::MomentGeom M = L->slab ? chll::make_slab_moment_geom(v, L->z0, L->nk_global)
                                     : chll::make_moment_geom(v);
  chll::launch_observables(v, M, cp, L->ctl, L->partials, &L->tickets[0], dev_row, step,
                           L->stream);
  CHLL_CUDA_TRY(cudaGetLastError());
  return CHLL_OK;
}

int create_impl(int ni, int nj, int nk, int boundary, chll_lattice** out, int slab_z0 = -1,
                int slab_nk = 0) {
  if (!out) return fail(CHLL_EINVAL, "lattice_create: null output pointer");
  *out = nullptr;
  if (ni < 1 || nj < 1 || nk < 1)
    return fail(CHLL_EINVAL, "lattice dims must be >= 1 (got %d %d %d)", ni, nj, nk);
  if (boundary != CHLL_OPEN && boundary != CHLL_PERIODIC)
    return fail(CHLL_EINVAL, "boundary must be CHLL_OPEN or CHLL_PERIODIC (got %d)", boundary);
  if (boundary == CHLL_PERIODIC && ((ni | nj | nk) & 1))
    return fail(CHLL_EINVAL,
                "periodic boundaries need even ni, nj, nk for a consistent checkerboard "
                "(got %d %d %d)",
                ni, nj, nk);
  if (nk > 65535) return fail(CHLL_EINVAL, "nk must be <= 65535 (got %d)", nk);
  const long long n = (long long)ni * nj * nk;
  const long long groups = (long long)(chll::padded_ni(ni) / 4) * nj * nk;
  if (n >= (1LL << 32) || groups >= (1LL << 32))
    return fail(CHLL_EINVAL, "lattice too large for 32-bit random counters (%lld sites)", n);
  // The kernels index the slots of one colour (padded rows, a slab's halo
  // planes included) in 32 bits: fewer than 2^31 of them.
  const long long planes = slab_z0 >= 0 ? (long long)slab_nk + 3 : (long long)nk;
  const long long slots = (long long)(chll::padded_ni(ni) / 2) * nj * planes;
  if (slots >= (1LL << 31))
    return fail(CHLL_EINVAL,
                "lattice too large: %lld slots per colour (rows padded to a multiple of 4 "
                "sites%s); the limit is 2^31",
                slots, slab_z0 >= 0 ? ", halo planes included" : "");
  CHLL_TRY(check_device());
  chll::sweep_prepare();

  chll_lattice* L = new chll_lattice();
  L->ni = ni;
  L->nj = nj;
  L->nk = nk;
  L->hx = chll::padded_ni(ni) / 2;
  L->periodic = boundary;
  L->nsites = n;
  L->ctl_sites = n;
  if (slab_z0 >= 0) {
    L->slab = 1;
    L->z0 = slab_z0;
    L->nk_global = nk;
    L->nk = slab_nk;
    L->nsites = (long long)ni * nj * slab_nk;
  }
  L->per_colour = (size_t)L->hx * nj * L->store_planes();
  cudaGetDevice(&L->device);
  auto bail = [&](cudaError_t e, const char* what) {
    chll_lattice_destroy(L);
    return fail(e == cudaErrorMemoryAllocation ? CHLL_ENOMEM : CHLL_ECUDA, "%s: %s", what,
                cudaGetErrorString(e));
  };
  cudaError_t e;
  if ((e = cudaStreamCreateWithFlags(&L->own_stream, cudaStreamNonBlocking)) != cudaSuccess)
    return bail(e, "stream");
  if ((e = cudaStreamCreateWithFlags(&L->capture_stream, cudaStreamNonBlocking)) != cudaSuccess)
    return bail(e, "stream");
  L->stream = L->own_stream;
  if ((e = cudaMalloc(&L->lat, 2 * L->per_colour * sizeof(float4))) != cudaSuccess)
    return bail(e, "lattice allocation");
  if (!chll::unit_view_aligned(L->store_view()) || !chll::unit_view_aligned(L->view())) {
    chll_lattice_destroy(L);
    return fail(CHLL_ECUDA, "lattice allocation is not 32-byte aligned");
  }
  if ((e = cudaMalloc(&L->ctl, sizeof(Control))) != cudaSuccess) return bail(e, "control");
  const int pb = std::max(chll::observables_max_blocks() * chll::kObsMoments,
                          chll::energy_grad_max_blocks() * 4);
  if ((e = cudaMalloc(&L->partials, sizeof(double) * pb)) != cudaSuccess)
    return bail(e, "partials");
  if ((e = cudaMalloc(&L->tickets, 2 * sizeof(unsigned int))) != cudaSuccess)
    return bail(e, "tickets");
  if ((e = cudaMalloc(&L->out4, 4 * sizeof(double) + chll::kRowLen * sizeof(double))) !=
      cudaSuccess)
    return bail(e, "result buffer");
  if ((e = cudaMemsetAsync(L->tickets, 0, 2 * sizeof(unsigned int), L->stream)) != cudaSuccess)
    return bail(e, "memset");
  if ((e = cudaMemsetAsync(L->lat, 0, 2 * L->per_colour * sizeof(float4), L->stream)) !=
      cudaSuccess)
    return bail(e, "memset");
  *out = L;
  if (set_control_impl(L, 0.1, 1, 10000) != CHLL_OK) {
    chll_lattice_destroy(L);
    *out = nullptr;
    return t_status;
  }
  return CHLL_OK;
}

// ---- stdout table of chll_mod.f90:60,98 ----------------------------------
void fortran_f12_6(char* out, double v) {
  char buf[64];
  snprintf(buf, sizeof(buf), "%12.6f", v);
  if (std::strlen(buf) > 12 || !std::isfinite(v)) {
    std::memset(out, '*', 12);
    out[12] = 0;
  } else {
    std::memcpy(out, buf, 13);
  }
}

void print_header() {
  std::printf("Steps       Energy      E. excess      Paccept      Faccept      D\n");
  std::fflush(stdout);
}

void print_row(long long step, const double* row) {
  char f[5][16];
  for (int c = 0; c < 5; ++c) fortran_f12_6(f[c], row[c]);
  if (step > 99999999 || step < -9999999)
    std::printf("********");
  else
    std::printf("%8lld", step);
  for (int c = 0; c < 5; ++c) std::printf(" %s", f[c]);
  std::printf("\n");
  std::fflush(stdout);
}

// Shared body of run() and chll_run_ex().
int run_impl(const chll_run_config& cfg, int nstart, int nstop, int nout, double* nx, double* ny,
             double* nz, int* s, int ni, int nj, int nk, int* msteps, double* m, double* rows16,
             double* d_out) {
  if (!nx || !ny || !nz || !s) return fail(CHLL_EINVAL, "run: null state array");
  if (nout <= 0) return fail(CHLL_EINVAL, "run: nout must be positive (got %d)", nout);
  if (nstop < nstart) return fail(CHLL_EINVAL, "run: nstop < nstart (%d < %d)", nstop, nstart);
  if (!(cfg.kT >= 0.0)) return fail(CHLL_EINVAL, "run: kbt must be >= 0 (got %g)", cfg.kT);

  static chll_lattice* cache = nullptr;  // guarded by g_run_mutex
  if (cache && (cache->ni != ni || cache->nj != nj || cache->nk != nk ||
                cache->periodic != cfg.boundary)) {
    chll_lattice_destroy(cache);
    cache = nullptr;
  }
  if (!cache) CHLL_TRY(create_impl(ni, nj, nk, cfg.boundary, &cache));
  chll_lattice* L = cache;
  L->stream = L->own_stream;

  const long long rows = (1LL + nstop - nstart) / nout;
  CHLL_TRY(ensure_rows(L, (int)std::max(1LL, rows)));
  chll_coupling cc = {cfg.kT, cfg.K, cfg.g, cfg.eps};
  const Coupling cp = make_coupling(cc);

  CHLL_TRY(upload_f64_impl(L, nx, ny, nz, s));
  CHLL_TRY(set_control_impl(L, cfg.d, nstart, cfg.adapt_until));
  if (cfg.verbose && nstart == 1) print_header();

  double* host_rows = nullptr;
  if (rows > 0) {
    CHLL_CUDA_TRY(cudaMallocHost(&host_rows, sizeof(double) * chll::kRowLen * rows));
  }
  std::vector<cudaEvent_t> events;
  std::vector<long long> row_step;
  long long printed = 0, r = 0, dropped = 0;
  int rc = CHLL_OK;
  long long istep = nstart;
  auto flush_rows = [&](bool wait) {
    while (printed < r) {
      if (wait)
        cudaEventSynchronize(events[printed]);
      else if (cudaEventQuery(events[printed]) != cudaSuccess)
        break;
      if (cfg.verbose) print_row(row_step[printed], host_rows + printed * chll::kRowLen);
      ++printed;
    }
  };
  while (istep <= nstop && rc == CHLL_OK) {
    // next multiple of nout at or after istep
    long long meas = ((istep + nout - 1) / nout) * nout;
    if (istep <= 0) meas = istep - (istep % nout);  // Fortran MOD for non-positive steps
    const long long end = std::min<long long>(meas, nstop);
    rc = sweep_impl(L, cp, cfg.seed, cfg.replica, (int)(end - istep + 1));
    if (rc != CHLL_OK) break;
    if (end == meas) {
      if (r < rows) {
        double* drow = L->rows + r * chll::kRowLen;
        rc = observe_impl(L, make_coupling_d(cc), drow, end);
        if (rc != CHLL_OK) break;
        cudaEvent_t ev;
        cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
        cudaMemcpyAsync(host_rows + r * chll::kRowLen, drow, sizeof(double) * chll::kRowLen,
                        cudaMemcpyDeviceToHost, L->stream);
        cudaEventRecord(ev, L->stream);
        events.push_back(ev);
        row_step.push_back(end);
        ++r;
      } else {
        ++dropped;
      }
    }
    istep = end + 1;
    flush_rows(false);
  }
  cudaError_t e = cudaStreamSynchronize(L->stream);
  if (rc == CHLL_OK && e != cudaSuccess)
    rc = fail(CHLL_ECUDA, "run: %s", cudaGetErrorString(e));
  if (rc == CHLL_OK) flush_rows(true);
  for (auto ev : events) cudaEventDestroy(ev);

  if (rc == CHLL_OK) rc = download_f64_impl(L, nx, ny, nz, s);
  if (rc == CHLL_OK) {
    Control c;
    e = cudaMemcpy(&c, L->ctl, sizeof(c), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) rc = fail(CHLL_ECUDA, "run: %s", cudaGetErrorString(e));
    else if (d_out) *d_out = c.d;
  }
  if (rc == CHLL_OK) {
    for (long long q = 0; q < r; ++q) {
      const double* hr = host_rows + q * chll::kRowLen;
      if (msteps) msteps[q] = (int)row_step[q];
      if (m)
        for (int c = 0; c < 5; ++c) m[c * rows + q] = hr[c];
      if (rows16) std::memcpy(rows16 + q * chll::kRowLen, hr, sizeof(double) * chll::kRowLen);
    }
  }
  if (host_rows) cudaFreeHost(host_rows);
  if (rc == CHLL_OK && dropped)
    rc = fail(CHLL_ERANGE,
              "run: %lld measurement steps did not fit in the %lld rows of msteps/m "
              "(rows = (1+nstop-nstart)/nout); they were not stored",
              dropped, rows);
  if (rc == CHLL_OK) ok();
  return rc;
}

}  // namespace

// ---------------------------------------------------------------------------
// Exported entry points
// ---------------------------------------------------------------------------
extern "C" {

int chll_last_status(void) { return t_status; }
const char* chll_last_error(void) { return t_error.c_str(); }
const char* chll_version(void) { return "chll-b200 0.1 (sm_100a)"; }

void chll_set_seed(uint64_t seed) {
  std::lock_guard<std::mutex> lk(g_run_mutex);
  g_seed = seed;
  g_run_ordinal = 0;
}

void init(double* nx, double* ny, double* nz, int* s, int* dope, int* sl1, int* sl2,
          const int* ni, const int* nj, const int* nk, const int* nsub) {
  (void)nx; (void)ny; (void)nz; (void)s; (void)dope;
  if (!sl1 || !sl2 || !ni || !nj || !nk || !nsub) {
    fail(CHLL_EINVAL, "init: null argument");
    std::fprintf(stderr, "libchll_mod init: %s\n", t_error.c_str());
    return;
  }
  const long long cap = *nsub;
  long long n1 = 0, n2 = 0;
  for (int k = 1; k <= *nk; ++k)
    for (int j = 1; j <= *nj; ++j)
      for (int i = 1; i <= *ni; ++i) {
        const int idx = i + (j - 1) * *ni + (k - 1) * (*ni * *nj);
        if ((i + j + k) % 2 != 0) {
          if (n1 < cap) sl1[n1] = idx;
          ++n1;
        } else {
          if (n2 < cap) sl2[n2] = idx;
          ++n2;
        }
      }
  if (n1 > cap || n2 > cap) {
    fail(CHLL_ERANGE, "init: sublattice of %lld/%lld sites exceeds nsub=%lld; lists truncated",
         n1, n2, cap);
    std::fprintf(stderr, "libchll_mod init: %s\n", t_error.c_str());
    return;
  }
  ok();
}

void run(const int* nstart, const int* nstop, const int* nout, double* nx, double* ny,
         double* nz, int* s, int* dope, int* sl1, int* sl2, double* g, double* KK, double* d,
         double* kbt, const int* ni, const int* nj, const int* nk, int* nsub, int* msteps,
         double* m) {
  (void)dope; (void)sl1; (void)sl2;
  if (!nstart || !nstop || !nout || !g || !KK || !d || !kbt || !ni || !nj || !nk || !nsub) {
    fail(CHLL_EINVAL, "run: null scalar argument");
    std::fprintf(stderr, "libchll_mod run: %s\n", t_error.c_str());
    return;
  }
  std::lock_guard<std::mutex> lk(g_run_mutex);
  chll_run_config cfg;
  std::memset(&cfg, 0, sizeof(cfg));
  cfg.kT = *kbt;
  cfg.K = *KK;
  cfg.g = *g;
  cfg.eps = 1.0;
  cfg.d = *d;
  cfg.seed = g_seed;
  cfg.replica = g_run_ordinal++;
  cfg.boundary = CHLL_OPEN;
  cfg.adapt_until = 10000;
  cfg.verbose = 1;
  *nsub = (int)(((long long)*ni * *nj * *nk) / 2);
  double dout = *d;
  const int rc = run_impl(cfg, *nstart, *nstop, *nout, nx, ny, nz, s, *ni, *nj, *nk, msteps, m,
                          nullptr, &dout);
  if (rc != CHLL_OK && rc != CHLL_ERANGE) {
    std::fprintf(stderr, "libchll_mod run: %s\n", t_error.c_str());
    return;
  }
  if (rc == CHLL_ERANGE) std::fprintf(stderr, "libchll_mod run: %s\n", t_error.c_str());
  *d = dout;
}

int chll_run_ex(const chll_run_config* cfg, int nstart, int nstop, int nout, double* nx,
                double* ny, double* nz, int* s, int ni, int nj, int nk, int* msteps, double* m,
                double* rows16, double* d_out) {
  if (!cfg) return fail(CHLL_EINVAL, "chll_run_ex: null config");
  std::lock_guard<std::mutex> lk(g_run_mutex);
  return run_impl(*cfg, nstart, nstop, nout, nx, ny, nz, s, ni, nj, nk, msteps, m, rows16, d_out);
}

int chll_lattice_create(int ni, int nj, int nk, int boundary, chll_lattice** out) {
  const int rc = create_impl(ni, nj, nk, boundary, out);
  if (rc == CHLL_OK) ok();
  return rc;
}

void chll_lattice_destroy(chll_lattice* L) {
  if (!L) return;
  drop_graphs(L);
  if (L->own_stream) cudaStreamSynchronize(L->own_stream);
  if (L->stream && L->stream != L->own_stream) cudaStreamSynchronize(L->stream);
  cudaFree(L->lat);
  cudaFree(L->ctl);
  cudaFree(L->partials);
  cudaFree(L->tickets);
  cudaFree(L->rows);
  cudaFree(L->out4);
  cudaFree(L->staging);
  cudaFree(L->grad);
  if (L->own_stream) cudaStreamDestroy(L->own_stream);
  if (L->capture_stream) cudaStreamDestroy(L->capture_stream);
  delete L;
}

int chll_lattice_set_kernel(chll_lattice* L, int kernel) {
  if (!L) return fail(CHLL_EINVAL, "null lattice");
  if (kernel < 0 || kernel > 4)
    return fail(CHLL_EINVAL, "set_kernel: kernel must be 0, 1, 2, 3 or 4");
  if (kernel == chll::kSweepResident && L->slab)
    return fail(CHLL_EINVAL, "set_kernel: a slab cannot run the resident form");
  if (kernel == chll::kSweepResident && chll::resident_cluster() <= 0)
    return fail(CHLL_ECUDA, "set_kernel: no thread-block cluster fits on this device");
  if (kernel == chll::kSweepStaged && !chll::staged_fits(L->view()))
    return fail(CHLL_EINVAL, "set_kernel: rows of %d sites are too long for the staged kernel",
                L->ni);
  if (kernel != L->kernel) drop_graphs(L);
  L->kernel = kernel;
  return ok();
}

int chll_lattice_set_stream(chll_lattice* L, void* stream) {
  if (!L) return fail(CHLL_EINVAL, "null lattice");
  L->stream = stream ? (cudaStream_t)stream : L->own_stream;
  return ok();
}

int chll_lattice_sync(chll_lattice* L) {
  if (!L) return fail(CHLL_EINVAL, "null lattice");
  CHLL_CUDA_TRY(cudaStreamSynchronize(L->stream));
  return ok();
}

int chll_lattice_init_random(chll_lattice* L, uint64_t seed, uint32_t replica) {
  if (!L) return fail(CHLL_EINVAL, "null lattice");
  CHLL_CUDA_TRY(cudaMemsetAsync(L->lat, 0, 2 * L->per_colour * sizeof(float4), L->stream));
  // a slab draws the values of its global sites
  chll::launch_init_random(L->view(), seed_lo(seed), seed_hi(seed), replica, L->stream,
                           (uint64_t)L->ni * L->nj * L->z0);
  CHLL_CUDA_TRY(cudaGetLastError());
  return ok();
}

int chll_lattice_upload_f64(chll_lattice* L, const double* nx, const double* ny,
                            const double* nz, const int* s) {
  if (!L) return fail(CHLL_EINVAL, "null lattice");
  CHLL_TRY(upload_f64_impl(L, nx, ny, nz, s));
  CHLL_CUDA_TRY(cudaStreamSynchronize(L->stream));
  return ok();
}

int chll_lattice_download_f64(chll_lattice* L, double* nx, double* ny, double* nz, int* s) {
  if (!L) return fail(CHLL_EINVAL, "null lattice");
  CHLL_TRY(download_f64_impl(L, nx, ny, nz, s));
  return ok();
}

int chll_lattice_upload_f4(chll_lattice* L, const float* xyzs) {
  if (!L || !xyzs) return fail(CHLL_EINVAL, "upload_f4: null argument");
  const size_t n = (size_t)L->nsites;
  CHLL_CUDA_TRY(cudaMemsetAsync(L->lat, 0, 2 * L->per_colour * sizeof(float4), L->stream));
  const float4* src = (const float4*)xyzs;
  if (!is_device_ptr(xyzs)) {
    CHLL_TRY(ensure_staging(L, n * sizeof(float4)));
    CHLL_CUDA_TRY(cudaMemcpyAsync(L->staging, xyzs, n * sizeof(float4), cudaMemcpyDefault,
                                  L->stream));
    src = (const float4*)L->staging;
  }
  chll::launch_pack_f4(L->view(), src, L->stream);
  CHLL_CUDA_TRY(cudaGetLastError());
  CHLL_CUDA_TRY(cudaStreamSynchronize(L->stream));
  return ok();
}

int chll_lattice_download_f4(chll_lattice* L, float* xyzs) {
  if (!L || !xyzs) return fail(CHLL_EINVAL, "download_f4: null argument");
  const size_t n = (size_t)L->nsites;
  if (is_device_ptr(xyzs)) {
    chll::launch_unpack_f4(L->view(), (float4*)xyzs, L->stream);
  } else {
    CHLL_TRY(ensure_staging(L, n * sizeof(float4)));
    chll::launch_unpack_f4(L->view(), (float4*)L->staging, L->stream);
    CHLL_CUDA_TRY(cudaMemcpyAsync(xyzs, L->staging, n * sizeof(float4), cudaMemcpyDefault,
                                  L->stream));
  }
  CHLL_CUDA_TRY(cudaGetLastError());
  CHLL_CUDA_TRY(cudaStreamSynchronize(L->stream));
  return ok();
}

int chll_lattice_storage(chll_lattice* L, void** c0, void** c1, int64_t* per_colour,
                         int32_t* hx) {
  if (!L) return fail(CHLL_EINVAL, "null lattice");
  if (c0) *c0 = L->lat;
  if (c1) *c1 = L->lat + L->per_colour;
  if (per_colour) *per_colour = (int64_t)L->per_colour;
  if (hx) *hx = L->hx;
  return ok();
}

int chll_lattice_set_control(chll_lattice* L, double d, int64_t step, int64_t adapt_until) {
  if (!L) return fail(CHLL_EINVAL, "null lattice");
  CHLL_TRY(set_control_impl(L, d, step, adapt_until));
  return ok();
}

int chll_lattice_get_control(chll_lattice* L, double* d, int64_t* step, double* paccept,
                             double* faccept) {
  if (!L) return fail(CHLL_EINVAL, "null lattice");
  Control c;
  CHLL_CUDA_TRY(cudaStreamSynchronize(L->stream));
  CHLL_CUDA_TRY(cudaMemcpy(&c, L->ctl, sizeof(c), cudaMemcpyDeviceToHost));
  if (c.status) return fail(CHLL_EDEVICE, "device status word 0x%x", c.status);
  if (d) *d = c.d;
  if (step) *step = c.step;
  if (paccept) *paccept = c.paccept;
  if (faccept) *faccept = c.faccept;
  return ok();
}

int chll_lattice_sweep(chll_lattice* L, const chll_coupling* c, uint64_t seed, uint32_t replica,
                       int nsweeps) {
  if (!L || !c) return fail(CHLL_EINVAL, "sweep: null argument");
  if (nsweeps < 0) return fail(CHLL_EINVAL, "sweep: nsweeps < 0");
  if (!(c->kT >= 0.0)) return fail(CHLL_EINVAL, "sweep: kT must be >= 0");
  if (L->slab)
    return fail(CHLL_EINVAL, "sweep: a slab is swept pass by pass with halo exchanges between");
  CHLL_TRY(sweep_impl(L, make_coupling(*c), seed, replica, nsweeps));
  return ok();
}

int chll_lattice_pass(chll_lattice* L, const chll_coupling* c, uint64_t seed, uint32_t replica,
                      int pass) {
  if (!L || !c) return fail(CHLL_EINVAL, "pass: null argument");
  if (pass < 0 || pass > 7) return fail(CHLL_EINVAL, "pass must be 0..7 (got %d)", pass);
  if (!(c->kT >= 0.0)) return fail(CHLL_EINVAL, "pass: kT must be >= 0");
  if (L->slab) {
    if (pass < 4) return fail(CHLL_EINVAL, "pass: a slab runs the fused passes 4..7 only");
    const LatticeView sv = L->store_view();
    const chll::SweepGeom G = chll::make_slab_geom(sv, 2, L->nk, L->z0 - 2);
    const int colour = pass == 4 + chll::kFusedB ? 1 : 0;
    chll::launch_fused_pass(sv, G, L->periodic ? chll::kBoundSlabXY : chll::kBoundOpen,
                            make_coupling(*c), seed_lo(seed), seed_hi(seed), replica, L->ctl,
                            pass - 4, L->stream, L->peer_lo[colour], L->peer_hi[colour]);
    CHLL_CUDA_TRY(cudaGetLastError());
    return ok();
  }
  if (pass >= 4)
    chll::launch_fused_pass(L->view(), make_coupling(*c), seed_lo(seed), seed_hi(seed), replica,
                            L->ctl, pass - 4, L->stream);
  else
    chll::launch_sweep_pass(L->view(), make_coupling(*c), seed_lo(seed), seed_hi(seed),
                            replica, L->ctl, pass, L->stream, L->kernel);
  CHLL_CUDA_TRY(cudaGetLastError());
  return ok();
}

int chll_lattice_reserve_rows(chll_lattice* L, int n) {
  if (!L || n < 0) return fail(CHLL_EINVAL, "reserve_rows: bad argument");
  CHLL_CUDA_TRY(cudaStreamSynchronize(L->stream));
  CHLL_TRY(ensure_rows(L, std::max(1, n)));
  return ok();
}

int chll_lattice_measure(chll_lattice* L, const chll_coupling* c, int slot) {
  if (!L || !c) return fail(CHLL_EINVAL, "measure: null argument");
  if (slot < 0 || slot >= L->rows_cap)
    return fail(CHLL_ERANGE, "measure: row %d outside the %d reserved rows", slot, L->rows_cap);
  CHLL_TRY(observe_impl(L, make_coupling_d(*c), L->rows + (size_t)slot * chll::kRowLen, -1));
  return ok();
}

int chll_lattice_read_rows(chll_lattice* L, double* rows16, int first, int count) {
  if (!L || !rows16) return fail(CHLL_EINVAL, "read_rows: null argument");
  if (first < 0 || count < 0 || first + count > L->rows_cap)
    return fail(CHLL_ERANGE, "read_rows: rows [%d, %d) outside the %d reserved rows", first,
                first + count, L->rows_cap);
  CHLL_CUDA_TRY(cudaMemcpyAsync(rows16, L->rows + (size_t)first * chll::kRowLen,
                                sizeof(double) * chll::kRowLen * count, cudaMemcpyDeviceToHost,
                                L->stream));
  CHLL_CUDA_TRY(cudaStreamSynchronize(L->stream));
  return ok();
}

int chll_lattice_observe(chll_lattice* L, const chll_coupling* c, double* row16) {
  if (!L || !c || !row16) return fail(CHLL_EINVAL, "observe: null argument");
  double* drow = L->out4 + 4;
  Control ctl;
  CHLL_CUDA_TRY(cudaMemcpyAsync(&ctl, L->ctl, sizeof(ctl), cudaMemcpyDeviceToHost, L->stream));
  CHLL_CUDA_TRY(cudaStreamSynchronize(L->stream));
  CHLL_TRY(observe_impl(L, make_coupling_d(*c), drow, ctl.step - 1));
  CHLL_CUDA_TRY(cudaMemcpyAsync(row16, drow, sizeof(double) * chll::kRowLen,
                                cudaMemcpyDeviceToHost, L->stream));
  CHLL_CUDA_TRY(cudaStreamSynchronize(L->stream));
  return ok();
}

int chll_lattice_quench(chll_lattice* L, const chll_coupling* c, double eta, int nsteps) {
  if (!L || !c) return fail(CHLL_EINVAL, "quench: null argument");
  if (L->slab) return fail(CHLL_EINVAL, "quench: not available on a slab (whole lattices only)");
  if (nsteps < 0 || !(eta >= 0.0)) return fail(CHLL_EINVAL, "quench: need nsteps >= 0, eta >= 0");
  const LatticeView v = L->view();
  const chll::CouplingD cd = make_coupling_d(*c);
  for (int s = 0; s < nsteps; ++s) {
    chll::launch_quench_pass(v, cd, (float)eta, 0, L->stream);
    chll::launch_quench_pass(v, cd, (float)eta, 1, L->stream);
  }
  CHLL_CUDA_TRY(cudaGetLastError());
  return ok();
}

int chll_lattice_energy_grad(chll_lattice* L, const chll_coupling* c, float* grad, int project,
                             double* out4) {
  if (!L || !c) return fail(CHLL_EINVAL, "energy_grad: null argument");
  if (L->slab) return fail(CHLL_EINVAL, "energy_grad: not available on a slab (whole lattices only)");
  const size_t total = 2 * L->per_colour;
  if (grad && !L->grad) CHLL_CUDA_TRY(cudaMalloc(&L->grad, total * sizeof(float4)));
  chll::launch_energy_grad(L->view(), make_coupling_d(*c), grad ? L->grad : nullptr, project,
                           L->partials, &L->tickets[1], L->out4, L->stream);
  CHLL_CUDA_TRY(cudaGetLastError());
  if (grad) {
    LatticeView gv = L->view();
    gv.col[0] = L->grad;
    gv.col[1] = L->grad + L->per_colour;
    const size_t n = (size_t)L->nsites;
    if (is_device_ptr(grad)) {
      chll::launch_unpack_f4(gv, (float4*)grad, L->stream);
    } else {
      CHLL_TRY(ensure_staging(L, n * sizeof(float4)));
      chll::launch_unpack_f4(gv, (float4*)L->staging, L->stream);
      CHLL_CUDA_TRY(cudaMemcpyAsync(grad, L->staging, n * sizeof(float4), cudaMemcpyDefault,
                                    L->stream));
    }
    CHLL_CUDA_TRY(cudaGetLastError());
  }
  if (out4)
    CHLL_CUDA_TRY(cudaMemcpyAsync(out4, L->out4, 4 * sizeof(double), cudaMemcpyDeviceToHost,
                                  L->stream));
  CHLL_CUDA_TRY(cudaStreamSynchronize(L->stream));
  return ok();
}

int chll_lattice_shell_corr(chll_lattice* L, int nshells, int wrap, double* gn, double* gs,
                            double* counts) {
  if (!L || !gn || !gs || !counts) return fail(CHLL_EINVAL, "shell_corr: null argument");
  if (L->slab) return fail(CHLL_EINVAL, "shell_corr: not available on a slab (whole lattices only)");
  if (nshells < 1 || nshells > chll::kMaxCorrShells)
    return fail(CHLL_EINVAL, "shell_corr: nshells must be 1..%d (got %d)", chll::kMaxCorrShells,
                nshells);
  const int ni = L->ni, nj = L->nj, nk = L->nk, R = nshells;
  const double N = (double)L->nsites;
  // d = 0 and one half-space of offsets with |d|^2 < R^2, sorted by shell;
  // pair counts over all offsets in closed form.
  std::vector<int4> offs;
  std::vector<double> cnt(R, 0.0);
  auto wrapped = [](int d, int n) { return ((d % n) + n) % n; };
  for (int dk = -R + 1; dk < R; ++dk)
    for (int dj = -R + 1; dj < R; ++dj)
      for (int di = -R + 1; di < R; ++di) {
        const int r2 = di * di + dj * dj + dk * dk;
        if (r2 >= R * R) continue;
        const int shell = (int)std::floor(std::sqrt((double)r2));
        const double c = wrap ? N
                              : (double)std::max(0, ni - std::abs(di)) *
                                    (double)std::max(0, nj - std::abs(dj)) *
                                    (double)std::max(0, nk - std::abs(dk));
        cnt[shell] += c;
        const bool origin = di == 0 && dj == 0 && dk == 0;
        const bool half = dk > 0 || (dk == 0 && (dj > 0 || (dj == 0 && di > 0)));
        if (!(origin || half) || c == 0.0) continue;
        offs.push_back(wrap ? make_int4(wrapped(di, ni), wrapped(dj, nj), wrapped(dk, nk), shell)
                            : make_int4(di, dj, dk, shell));
      }
  std::stable_sort(offs.begin(), offs.end(),
                   [](const int4& a, const int4& b) { return a.w < b.w; });
  const int blocks = chll::shell_corr_blocks((uint64_t)L->nsites);
  const int width = 2 * R + 1;
  CHLL_TRY(ensure_staging(L, (size_t)L->nsites * sizeof(float4)));
  int4* d_offs = nullptr;
  double* d_part = nullptr;
  CHLL_CUDA_TRY(cudaMalloc(&d_offs, std::max<size_t>(1, offs.size()) * sizeof(int4)));
  cudaError_t e = cudaMalloc(&d_part, ((size_t)blocks + 1) * width * sizeof(double));
  if (e != cudaSuccess) {
    cudaFree(d_offs);
    return fail(CHLL_ENOMEM, "shell_corr: %s", cudaGetErrorString(e));
  }
  std::vector<double> out(width, 0.0);
  e = cudaMemcpyAsync(d_offs, offs.data(), offs.size() * sizeof(int4), cudaMemcpyHostToDevice,
                      L->stream);
  if (e == cudaSuccess) {
    chll::launch_unpack_f4(L->view(), (float4*)L->staging, L->stream);
    chll::launch_shell_corr((const float4*)L->staging, ni, nj, nk, d_offs, (int)offs.size(), R,
                            wrap != 0, d_part, blocks, d_part + (size_t)blocks * width,
                            L->stream);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(out.data(), d_part + (size_t)blocks * width, width * sizeof(double),
                        cudaMemcpyDeviceToHost, L->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(L->stream);
  cudaFree(d_offs);
  cudaFree(d_part);
  if (e != cudaSuccess) return fail(CHLL_ECUDA, "shell_corr: %s", cudaGetErrorString(e));
  const double s_mean = out[2 * R] / N;
  for (int r = 0; r < R; ++r) {
    const double w = r == 0 ? 1.0 : 2.0;  // shells >= 1 hold d and -d
    gn[r] = w * out[r] / cnt[r];
    gs[r] = w * out[R + r] / cnt[r] - s_mean * s_mean;
    counts[r] = cnt[r];
  }
  return ok();
}

int chll_lattice_projection(chll_lattice* L, const int* plane, long long* hist,
                            long long* m_min, int* nbins) {
  if (!L || !plane || !m_min || !nbins) return fail(CHLL_EINVAL, "projection: null argument");
  if (L->slab) return fail(CHLL_EINVAL, "projection: not available on a slab (whole lattices only)");
  const int n[3] = {L->ni, L->nj, L->nk};
  long long lo = 0, hi = 0;
  for (int d = 0; d < 3; ++d) {
    const long long p = plane[d];
    lo += p > 0 ? p : p * n[d];
    hi += p > 0 ? p * n[d] : p;
  }
  const long long nb = hi - lo + 1;
  if (nb > chll::kMaxProjectionBins)
    return fail(CHLL_ERANGE, "projection: %lld bins exceed %d (direction too long)", nb,
                chll::kMaxProjectionBins);
  *m_min = lo;
  *nbins = (int)nb;
  if (!hist) return ok();
  unsigned long long* d_hist = nullptr;
  CHLL_CUDA_TRY(cudaMalloc(&d_hist, (size_t)nb * sizeof(unsigned long long)));
  cudaError_t e = cudaMemsetAsync(d_hist, 0, (size_t)nb * sizeof(unsigned long long), L->stream);
  if (e == cudaSuccess) {
    chll::launch_projection(L->view(), plane[0], plane[1], plane[2], lo, (int)nb, d_hist,
                            L->stream);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(hist, d_hist, (size_t)nb * sizeof(long long), cudaMemcpyDeviceToHost,
                        L->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(L->stream);
  cudaFree(d_hist);
  if (e != cudaSuccess) return fail(CHLL_ECUDA, "projection: %s", cudaGetErrorString(e));
  return ok();
}

int chll_lattice_create_slab(int ni, int nj, int nk, int z0, int nkl, int boundary,
                             chll_lattice** out) {
  if (!out) return fail(CHLL_EINVAL, "create_slab: null output pointer");
  *out = nullptr;
  if (z0 < 0 || nkl < 2 || (z0 & 1) || (nkl & 1) || z0 + nkl > nk)
    return fail(CHLL_EINVAL,
                "create_slab: need even z0 >= 0 and even nkl >= 2 with z0 + nkl <= nk "
                "(got z0 %d, nkl %d, nk %d)",
                z0, nkl, nk);
  CHLL_TRY(create_impl(ni, nj, nk, boundary, out, z0, nkl));
  return ok();
}

int chll_lattice_slab_plane(chll_lattice* L, int colour, int which, void** ptr, int64_t* bytes) {
  if (!L || !ptr) return fail(CHLL_EINVAL, "slab_plane: null argument");
  if (!L->slab) return fail(CHLL_EINVAL, "slab_plane: not a slab");
  if (colour < 0 || colour > 1 || which < 0 || which > 3)
    return fail(CHLL_EINVAL, "slab_plane: colour 0/1 and which 0..3 (got %d, %d)", colour, which);
  // storage planes: 1 lower halo, 2 first own plane, nk+1 last own plane, nk+2 upper halo
  const int plane = which == 0 ? 1 : (which == 1 ? 2 : (which == 2 ? L->nk + 1 : L->nk + 2));
  const size_t per_plane = (size_t)L->hx * L->nj;
  *ptr = L->lat + (size_t)colour * L->per_colour + (size_t)plane * per_plane;
  if (bytes) *bytes = (int64_t)(per_plane * sizeof(float4));
  return ok();
}

static_assert(offsetof(Control, nflip) == offsetof(Control, nacc) + sizeof(unsigned long long),
              "the two pass counters are read as one array");

int chll_lattice_counters(chll_lattice* L, void** ptr) {
  if (!L || !ptr) return fail(CHLL_EINVAL, "counters: null argument");
  *ptr = &L->ctl->nacc;  // {nacc, nflip}: two consecutive uint64
  return ok();
}

int chll_lattice_slab_set_peers(chll_lattice* L, void* lower0, void* lower1, void* upper0,
                                void* upper1) {
  if (!L) return fail(CHLL_EINVAL, "null lattice");
  if (!L->slab) return fail(CHLL_EINVAL, "slab_set_peers: not a slab");
  void* const p[4] = {lower0, lower1, upper0, upper1};
  for (void* q : p) {
    if (!q) continue;
    if ((uintptr_t)q % 32)
      return fail(CHLL_EINVAL, "slab_set_peers: %p is not 32-byte aligned (a halo plane of a "
                  "slab from chll_lattice_slab_plane is)", q);
    if (!is_device_ptr(q))
      return fail(CHLL_EINVAL, "slab_set_peers: %p is not device memory", q);
  }
  CHLL_CUDA_TRY(cudaStreamSynchronize(L->stream));
  L->peer_lo[0] = (float4*)lower0;
  L->peer_lo[1] = (float4*)lower1;
  L->peer_hi[0] = (float4*)upper0;
  L->peer_hi[1] = (float4*)upper1;
  return ok();
}

int chll_lattice_slab_push(chll_lattice* L, int colour) {
  if (!L) return fail(CHLL_EINVAL, "null lattice");
  if (!L->slab) return fail(CHLL_EINVAL, "slab_push: not a slab");
  if (colour < 0 || colour > 1) return fail(CHLL_EINVAL, "slab_push: colour 0 or 1");
  const size_t per_plane = (size_t)L->hx * L->nj;
  const float4* base = L->lat + (size_t)colour * L->per_colour;
  if (L->peer_lo[colour])
    CHLL_CUDA_TRY(cudaMemcpyAsync(L->peer_lo[colour], base + 2 * per_plane,
                                  per_plane * sizeof(float4), cudaMemcpyDefault, L->stream));
  if (L->peer_hi[colour])
    CHLL_CUDA_TRY(cudaMemcpyAsync(L->peer_hi[colour], base + (size_t)(L->nk + 1) * per_plane,
                                  per_plane * sizeof(float4), cudaMemcpyDefault, L->stream));
  return ok();
}

int chll_lattice_ipc_handle(chll_lattice* L, void* handle64, uint64_t* base) {
  if (!L || !handle64 || !base) return fail(CHLL_EINVAL, "ipc_handle: null argument");
  static_assert(sizeof(cudaIpcMemHandle_t) == 64, "the ABI passes 64-byte IPC handles");
  cudaIpcMemHandle_t h;
  CHLL_CUDA_TRY(cudaIpcGetMemHandle(&h, L->lat));
  std::memcpy(handle64, &h, sizeof(h));
  *base = (uint64_t)(uintptr_t)L->lat;
  return ok();
}

int chll_ipc_open(const void* handle64, void** ptr) {
  if (!handle64 || !ptr) return fail(CHLL_EINVAL, "ipc_open: null argument");
  cudaIpcMemHandle_t h;
  std::memcpy(&h, handle64, sizeof(h));
  CHLL_CUDA_TRY(cudaIpcOpenMemHandle(ptr, h, cudaIpcMemLazyEnablePeerAccess));
  return ok();
}

int chll_ipc_close(void* ptr) {
  if (!ptr) return fail(CHLL_EINVAL, "ipc_close: null pointer");
  CHLL_CUDA_TRY(cudaIpcCloseMemHandle(ptr));
  return ok();
}

int chll_lattice_control_update(chll_lattice* L, int pass) {
  if (!L) return fail(CHLL_EINVAL, "null lattice");
  if (pass < 4 || pass > 7) return fail(CHLL_EINVAL, "control_update: pass 4..7 (got %d)", pass);
  chll::launch_control_update(L->ctl, pass - 4, L->stream);
  CHLL_CUDA_TRY(cudaGetLastError());
  return ok();
}

}  // extern "C"
