// Conversions between the caller's natural-order arrays and the red/black
// float4 lattice, and the on-device random initial state.
//
// The reference keeps nx, ny, nz (FP64) and s (int32) as four F-order
// (i fastest) arrays (chll/chll.py:57-61, chll_mod.f90:43-45).  The lattice
// here is one float4 (nx, ny, nz, s) per site split by colour, so a half-sweep
// reads each colour as one coalesced 128-bit stream.  One thread per natural
// site: reads are coalesced, and the writes of a warp land in two contiguous
// runs (one per colour).
#include "chll_common.cuh"
#include "sweep.cuh"

namespace chll {

namespace {

__device__ __forceinline__ size_t slot(const LatticeView& L, int i, int j, int k) {
  return ((size_t)k * L.nj + j) * L.hx + (i >> 1);
}

__device__ __forceinline__ void site_of(const LatticeView& L, size_t e, int& i, int& j, int& k) {
  const size_t r = e / (size_t)L.ni;
  i = (int)(e - r * (size_t)L.ni);
  k = (int)(r / (size_t)L.nj);
  j = (int)(r - (size_t)k * L.nj);
}

__global__ void pack_f64_kernel(LatticeView L, const double* __restrict__ nx,
                                const double* __restrict__ ny, const double* __restrict__ nz,
                                const int* __restrict__ s) {
  const size_t n = (size_t)L.ni * L.nj * L.nk;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n;
       e += (size_t)gridDim.x * blockDim.x) {
    int i, j, k;
    site_of(L, e, i, j, k);
    colour_array(L, (i + j + k) & 1)[slot(L, i, j, k)] =
        make_float4((float)nx[e], (float)ny[e], (float)nz[e], (float)s[e]);
  }
}

__global__ void unpack_f64_kernel(LatticeView L, double* __restrict__ nx, double* __restrict__ ny,
                                  double* __restrict__ nz, int* __restrict__ s) {
  const size_t n = (size_t)L.ni * L.nj * L.nk;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n;
       e += (size_t)gridDim.x * blockDim.x) {
    int i, j, k;
    site_of(L, e, i, j, k);
    const float4 v = colour_array(L, (i + j + k) & 1)[slot(L, i, j, k)];
    nx[e] = v.x;
    ny[e] = v.y;
    nz[e] = v.z;
    s[e] = (int)v.w;
  }
}

__global__ void pack_f4_kernel(LatticeView L, const float4* __restrict__ src) {
  const size_t n = (size_t)L.ni * L.nj * L.nk;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n;
       e += (size_t)gridDim.x * blockDim.x) {
    int i, j, k;
    site_of(L, e, i, j, k);
    colour_array(L, (i + j + k) & 1)[slot(L, i, j, k)] = src[e];
  }
}

__global__ void unpack_f4_kernel(LatticeView L, float4* __restrict__ dst) {
  const size_t n = (size_t)L.ni * L.nj * L.nk;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n;
       e += (size_t)gridDim.x * blockDim.x) {
    int i, j, k;
    site_of(L, e, i, j, k);
    dst[e] = colour_array(L, (i + j + k) & 1)[slot(L, i, j, k)];
  }
}

// Directors uniform on the sphere (cos(theta) = 2u-1, phi = 2*pi*u', as the
// reference drivers' init_random, scripts/pdanneal.py:5-16) and s = -1 with
// probability 1/2 (chll/chll.py:84-90).  site0: index of the view's first
// site in the whole lattice (a z-slab draws its global sites' values).
__global__ void init_random_kernel(LatticeView L, uint32_t key0, uint32_t key1, uint32_t replica,
                                   uint64_t site0) {
  const size_t n = (size_t)L.ni * L.nj * L.nk;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n;
       e += (size_t)gridDim.x * blockDim.x) {
    int i, j, k;
    site_of(L, e, i, j, k);
    Ctr4 c = {{(uint32_t)(e + site0), 0xffffffffu, replica, kStreamInit}};
    const Ctr4 r = philox4x32_10(c, key0, key1);
    const float ct = 2.0f * u01(r.v[0]) - 1.0f;
    const float st = sqrtf(fmaxf(0.f, 1.0f - ct * ct));
    float sp, cp;
    sincospif(2.0f * u01(r.v[1]), &sp, &cp);
    const float s = (u01(r.v[2]) < 0.5f) ? -1.0f : 1.0f;
    colour_array(L, (i + j + k) & 1)[slot(L, i, j, k)] = make_float4(st * cp, st * sp, ct, s);
  }
}

unsigned int grid_for(size_t n) {
  const size_t b = (n + 255) / 256;
  return (unsigned int)(b < 148 * 16 ? (b ? b : 1) : 148 * 16);
}

}  // namespace

void launch_pack_f64(const LatticeView& L, const double* nx, const double* ny, const double* nz,
                     const int* s, cudaStream_t stream) {
  const size_t n = (size_t)L.ni * L.nj * L.nk;
  pack_f64_kernel<<<grid_for(n), 256, 0, stream>>>(L, nx, ny, nz, s);
}

void launch_unpack_f64(const LatticeView& L, double* nx, double* ny, double* nz, int* s,
                       cudaStream_t stream) {
  const size_t n = (size_t)L.ni * L.nj * L.nk;
  unpack_f64_kernel<<<grid_for(n), 256, 0, stream>>>(L, nx, ny, nz, s);
}

void launch_pack_f4(const LatticeView& L, const float4* xyzs, cudaStream_t stream) {
  const size_t n = (size_t)L.ni * L.nj * L.nk;
  pack_f4_kernel<<<grid_for(n), 256, 0, stream>>>(L, xyzs);
}

void launch_unpack_f4(const LatticeView& L, float4* xyzs, cudaStream_t stream) {
  const size_t n = (size_t)L.ni * L.nj * L.nk;
  unpack_f4_kernel<<<grid_for(n), 256, 0, stream>>>(L, xyzs);
}

void launch_init_random(const LatticeView& L, uint32_t key0, uint32_t key1, uint32_t replica,
                        cudaStream_t stream, uint64_t site0) {
  const size_t n = (size_t)L.ni * L.nj * L.nk;
  init_random_kernel<<<grid_for(n), 256, 0, stream>>>(L, key0, key1, replica, site0);
}

}  // namespace chll
