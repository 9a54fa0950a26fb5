// Energy adjoint with no device allocation: chll_energy_grad_noalloc.
//
// chll_lattice_energy_grad allocates (cudaMalloc) a red/black gradient buffer
// as large as the lattice the first time it runs, and keeps its reduction
// partials in the lattice object.  Some callers cannot let a library allocate
// device memory: a Fortran/OpenACC host (the reference's own kind of program)
// whose arrays live in its runtime's device pool, or an application that has
// handed nearly all of HBM to its own allocator, where a cudaMalloc either
// fails or competes with the owner's pool.  This entry point takes the
// caller's device buffers for the lattice and the results, and runs the same
// adjoint and unpack kernels with every intermediate buffer placed in one
// fixed array of this file:
//
//   g_noalloc_scratch = [ red/black gradient, at most kMaxSlots float4 ]
//                       [ per-CTA partial sums, kPartials doubles       ]
//                       [ completion ticket                              ]
//
// kMaxSlots = 262,144 float4 slots (4 MiB), enough for a 64^3 lattice.
// kPartials = kGradMaxBlocks (148 x 4 CTAs, the adjoint's grid cap on any
// GPU; larger grids are not launched, the kernels walk grid-stride) x 4
// sums.  The whole array is about 4.02 MiB and every GPU that loads the
// library holds it until the process exits.
//
// The host cannot use the array's name as a device address.  The first call
// on each device asks the runtime for the address (cudaGetSymbolAddress, with
// that device current), caches it, and passes it to the kernels; make that
// first call before any stream capture.  Later calls on a stream that is not
// being captured look the address up again (a cheap query), so a device
// reset, which reloads the module, does not leave a stale address behind;
// calls inside a capture use the cached one.  All calls share the array and
// it keeps the last call's contents: the completion ticket is cleared at the
// start of every call, everything else is fully rewritten before it is read.
// Two calls whose work overlaps on the GPU (different streams, or different
// host threads on the same device) race on the array and give wrong results;
// serialise them.
//
// Caller arrays are checked before anything is enqueued: device memory of
// the current device (or managed memory), the lattice and grad arrays 16-byte
// aligned (read and written as float4), out4 8-byte aligned (doubles).  A
// misaligned array would otherwise fault the kernel and lose the context.
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <mutex>

#include "../../include/chll_mod.h"
#include "chll_common.cuh"
#include "sweep.cuh"

namespace chll {
int record_error(int code, const char* msg);
int record_ok();
}  // namespace chll

namespace {

constexpr size_t kMaxSlots = 2ull * 32 * 64 * 64;  // red/black slots of a 64^3 lattice
constexpr size_t kPartials = (size_t)chll::kGradMaxBlocks * 4;  // 4 sums per adjoint CTA
constexpr size_t kGradBytes = kMaxSlots * sizeof(float4);
constexpr size_t kPartialBytes = kPartials * sizeof(double);
constexpr size_t kScratchBytes = kGradBytes + kPartialBytes + 256;
constexpr int kMaxDevices = 64;

static_assert(kPartials >= (size_t)chll::kGradMaxBlocks * 4,
              "the partial-sum scratch must hold four sums per adjoint CTA");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_setup_mutex;
unsigned char* g_scratch_addr[kMaxDevices] = {};

int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  return chll::record_error(code, buf);
}

// Device memory that kernels on device `dev` can address: memory of that
// device, or managed memory.
bool on_device(const void* p, int dev) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return (a.type == cudaMemoryTypeDevice && a.device == dev) ||
         a.type == cudaMemoryTypeManaged;
}

bool aligned(const void* p, uintptr_t a) { return ((uintptr_t)p % a) == 0; }

// Device address of g_noalloc_scratch on device `dev` (the current device):
// looked up on the first call, and again whenever the stream is not being
// captured.
int scratch_address(int dev, cudaStream_t stream, unsigned char** out) {
  if (dev < 0 || dev >= kMaxDevices)
    return fail(CHLL_EINVAL, "energy_grad_noalloc: device ordinal %d >= %d", dev, kMaxDevices);
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(stream, &cap) != cudaSuccess) {
    cudaGetLastError();
    cap = cudaStreamCaptureStatusNone;
  }
  std::lock_guard<std::mutex> lk(g_setup_mutex);
  if (!g_scratch_addr[dev] || cap == cudaStreamCaptureStatusNone) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      return fail(CHLL_ECUDA, "energy_grad_noalloc: cudaGetSymbolAddress failed on device %d: %s",
                  dev, cudaGetErrorString(e));
    }
    g_scratch_addr[dev] = (unsigned char*)p;
  }
  *out = g_scratch_addr[dev];
  return CHLL_OK;
}

}  // namespace

extern "C" int chll_energy_grad_noalloc(const void* colour0, const void* colour1, int ni, int nj,
                                        int nk, int boundary, const chll_coupling* c,
                                        int project, float* grad, double* out4, void* stream) {
  if (!colour0 || !colour1 || !c || !out4)
    return fail(CHLL_EINVAL, "energy_grad_noalloc: null lattice, coupling or out4");
  if (ni < 1 || nj < 1 || nk < 1)
    return fail(CHLL_EINVAL, "energy_grad_noalloc: dims must be >= 1 (got %d %d %d)", ni, nj, nk);
  if (boundary != CHLL_OPEN && boundary != CHLL_PERIODIC)
    return fail(CHLL_EINVAL, "energy_grad_noalloc: boundary must be CHLL_OPEN or CHLL_PERIODIC");
  if (boundary == CHLL_PERIODIC && ((ni | nj | nk) & 1))
    return fail(CHLL_EINVAL, "energy_grad_noalloc: periodic boundaries need even dims");
  const int hx = chll::padded_ni(ni) / 2;
  const size_t per_colour = (size_t)hx * nj * nk;
  if (2 * per_colour > kMaxSlots)
    return fail(CHLL_ERANGE,
                "energy_grad_noalloc: a %dx%dx%d lattice needs %zu red/black slots; the fixed "
                "scratch holds at most %zu (a 64^3 lattice). Use chll_lattice_energy_grad, "
                "which allocates.",
                ni, nj, nk, 2 * per_colour, kMaxSlots);
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(CHLL_ECUDA, "energy_grad_noalloc: no CUDA device available (%s)",
                cudaGetErrorString(e));
  }
  if (!on_device(colour0, dev) || !on_device(colour1, dev) || !on_device(out4, dev) ||
      (grad && !on_device(grad, dev)))
    return fail(CHLL_EINVAL,
                "energy_grad_noalloc: lattice, grad and out4 must be device memory of the "
                "current device %d (or managed memory)",
                dev);
  if (!aligned(colour0, 16) || !aligned(colour1, 16) || (grad && !aligned(grad, 16)))
    return fail(CHLL_EINVAL,
                "energy_grad_noalloc: colour0, colour1 and grad must be 16-byte aligned "
                "(float4 arrays)");
  if (!aligned(out4, 8))
    return fail(CHLL_EINVAL, "energy_grad_noalloc: out4 must be 8-byte aligned (doubles)");

  cudaStream_t s = (cudaStream_t)stream;
  unsigned char* base = nullptr;
  const int rc = scratch_address(dev, s, &base);
  if (rc != CHLL_OK) return rc;
  float4* grad_rb = (float4*)base;
  double* partials = (double*)(base + kGradBytes);
  unsigned int* ticket = (unsigned int*)(base + kGradBytes + kPartialBytes);

  e = cudaMemsetAsync(ticket, 0, sizeof(unsigned int), s);
  if (e != cudaSuccess)
    return fail(CHLL_ECUDA, "energy_grad_noalloc: %s", cudaGetErrorString(e));

  chll::LatticeView v;
  v.col[0] = (float4*)colour0;
  v.col[1] = (float4*)colour1;
  v.ni = ni;
  v.nj = nj;
  v.nk = nk;
  v.hx = hx;
  v.periodic = boundary;
  chll::CouplingD cp;
  cp.eps = c->eps;
  cp.K = c->K;
  cp.g = c->g;
  chll::launch_energy_grad(v, cp, grad ? grad_rb : nullptr, project, partials, ticket, out4, s);
  if (grad) {
    chll::LatticeView gv = v;
    gv.col[0] = grad_rb;
    gv.col[1] = grad_rb + per_colour;
    chll::launch_unpack_f4(gv, (float4*)grad, s);
  }
  e = cudaGetLastError();
  if (e != cudaSuccess)
    return fail(CHLL_ECUDA, "energy_grad_noalloc: launch failed: %s", cudaGetErrorString(e));
  return chll::record_ok();
}
