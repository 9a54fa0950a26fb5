// Analysis kernels on one lattice's state: shell correlations of the director
// and the chirality, and integer projections of the chirality along a lattice
// direction (the input of the structure factor).
//
// Shell correlations restate calc_n_corr / calc_s_corr of the reference's
// analysis notebook (notebooks/paper_plots2.ipynb, cell 0, lines 61-112): over
// every ordered pair of sites (x, x + d) with |d|^2 < R^2 and both sites
// inside the lattice (open boundaries; optionally periodic images), shell
// floor(|d|) collects (n_x . n_{x+d})^2 and s_x s_{x+d}.  The sum over all
// sites of a pair term is the same for d and -d, so the kernel walks d = 0
// and one half-space of offsets (the host doubles shells >= 1; shell 0 holds
// d = 0 only) and the pair counts come from the host in closed form.
//
// Work layout: natural-order float4 sites (unpacked once into scratch), one
// thread per site, grid-stride in whole warps so every lane walks the same
// offset list (sorted by shell) and the warp reduces a shell's sums together.
// Per pair: FP32 dot product and FP32 running sums over at most kChunk
// offsets (the chirality term is exact: +-1 products), then an FP64 warp sum
// into per-warp shared slots; CTA partials are summed in a fixed order by a
// second kernel, so results are reproducible bit for bit.
//
// The projection kernel bins s by m = p . (i+1, j+1, k+1) for an integer
// direction p into an integer histogram (exact, order-free), from which the
// structure factor of hero_stripe.py's get_sc (a sum of s exp(-i k.(x+1)) for
// k along p) is a short one-dimensional transform on the host.
#include "chll_common.cuh"
#include "moments.cuh"
#include "sweep.cuh"

namespace chll {

namespace {

constexpr int kCorrThreads = 256;
constexpr int kCorrWarps = kCorrThreads / 32;
constexpr int kChunk = 128;  // FP32 terms per running sum before the FP64 flush

__device__ __forceinline__ void flush_shell(double (*s_n)[kMaxCorrShells],
                                            double (*s_s)[kMaxCorrShells], int warp, int lane,
                                            int shell, float an, float as) {
  const double vn = warp_sum_d((double)an);
  const double vs = warp_sum_d((double)as);
  if (lane == 0) {
    s_n[warp][shell] += vn;
    s_s[warp][shell] += vs;
  }
}

// offs[o] = {di, dj, dk, shell}, sorted by shell.  With WRAP the host has
// reduced di, dj, dk into [0, n) so one conditional subtraction wraps.
template <bool WRAP>
__global__ void __launch_bounds__(kCorrThreads)
    shell_corr_kernel(const float4* __restrict__ site, int ni, int nj, int nk,
                      const int4* __restrict__ offs, int noffs, int nshells,
                      double* __restrict__ partials) {
  __shared__ double s_n[kCorrWarps][kMaxCorrShells];
  __shared__ double s_s[kCorrWarps][kMaxCorrShells];
  __shared__ double s_sum[kCorrWarps];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int r = lane; r < nshells; r += 32) {
    s_n[warp][r] = 0.0;
    s_s[warp][r] = 0.0;
  }
  __syncwarp();
  const uint32_t uni = (uint32_t)ni, unj = (uint32_t)nj, unk = (uint32_t)nk;
  const uint64_t N = (uint64_t)uni * unj * unk;
  const uint64_t stride = (uint64_t)gridDim.x * kCorrThreads;
  const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
  double ssum = 0.0;
  for (uint64_t x0 = (uint64_t)blockIdx.x * kCorrThreads + (uint64_t)warp * 32; x0 < N;
       x0 += stride) {
    const uint64_t x = x0 + (uint64_t)lane;
    const bool valid = x < N;
    const uint32_t xi = valid ? (uint32_t)x : 0u;
    const uint32_t row = xi / uni;
    const int i = (int)(xi - row * uni);
    const int k = (int)(row / unj);
    const int j = (int)(row - (uint32_t)k * unj);
    const float4 a = valid ? site[xi] : zero;
    ssum += (double)a.w;
    int cur = -1, run = 0;
    float an = 0.f, as = 0.f;
    for (int o = 0; o < noffs; ++o) {
      const int4 d = __ldg(offs + o);
      if (d.w != cur || run == kChunk) {
        if (cur >= 0) flush_shell(s_n, s_s, warp, lane, cur, an, as);
        cur = d.w;
        run = 0;
        an = 0.f;
        as = 0.f;
      }
      ++run;
      uint32_t ii = (uint32_t)(i + d.x), jj = (uint32_t)(j + d.y), kk = (uint32_t)(k + d.z);
      bool in = valid;
      if (WRAP) {
        if (ii >= uni) ii -= uni;
        if (jj >= unj) jj -= unj;
        if (kk >= unk) kk -= unk;
      } else {
        in = in && ii < uni && jj < unj && kk < unk;
      }
      if (in) {
        const float4 b = site[ii + uni * (jj + unj * kk)];
        const float dt = fmaf(a.z, b.z, fmaf(a.y, b.y, __fmul_rn(a.x, b.x)));
        an = fmaf(dt, dt, an);
        as = fmaf(a.w, b.w, as);
      }
    }
    if (cur >= 0) flush_shell(s_n, s_s, warp, lane, cur, an, as);
  }
  ssum = warp_sum_d(ssum);
  if (lane == 0) s_sum[warp] = ssum;
  __syncthreads();
  const int width = 2 * nshells + 1;
  double* out = partials + (size_t)blockIdx.x * width;
  for (int t = threadIdx.x; t < width; t += kCorrThreads) {
    double v = 0.0;
    for (int w = 0; w < kCorrWarps; ++w)
      v += t < nshells ? s_n[w][t] : (t < 2 * nshells ? s_s[w][t - nshells] : s_sum[w]);
    out[t] = v;
  }
}

// Column t of the CTA partials summed over CTAs in index order.
__global__ void sum_partials_kernel(const double* __restrict__ partials, int rows, int width,
                                    double* __restrict__ out) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= width) return;
  double v = 0.0;
  for (int r = 0; r < rows; ++r) v += partials[(size_t)r * width + t];
  out[t] = v;
}

// hist[m - m0] += s over the real sites, m = p . (i+1, j+1, k+1).
__global__ void __launch_bounds__(256)
    projection_kernel(LatticeView L, MomentGeom M, int px, int py, int pz, long long m0,
                      int nbins, unsigned long long* __restrict__ hist) {
  extern __shared__ int s_hist[];
  for (int b = threadIdx.x; b < nbins; b += blockDim.x) s_hist[b] = 0;
  __syncthreads();
  const uint64_t total = 2ull * M.per_colour;
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t ee = (uint32_t)e;
    const int c = ee >= M.per_colour;
    const uint32_t t = ee - (c ? M.per_colour : 0u);
    const uint32_t r = M.by_hx.div(t);
    const int h = (int)(t - r * (uint32_t)L.hx);
    const int k = (int)M.by_nj.div(r);
    const int j = (int)(r - (uint32_t)k * (uint32_t)L.nj);
    const int i = 2 * h + ((c + j + k) & 1);
    if (i >= L.ni) continue;
    const float s = colour_array(L, c)[t].w;
    const long long m = (long long)px * (i + 1) + (long long)py * (j + 1) +
                        (long long)pz * (k + 1) - m0;
    atomicAdd(&s_hist[m], (int)s);
  }
  __syncthreads();
  for (int b = threadIdx.x; b < nbins; b += blockDim.x)
    if (s_hist[b]) atomicAdd(&hist[b], (unsigned long long)(long long)s_hist[b]);
}

int device_sms() {
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return sms > 0 ? sms : 148;
}

}  // namespace

int shell_corr_blocks(uint64_t nsites) {
  const uint64_t need = (nsites + kCorrThreads - 1) / kCorrThreads;
  const uint64_t cap = (uint64_t)device_sms() * 8;
  return (int)(need < cap ? (need ? need : 1) : cap);
}

void launch_shell_corr(const float4* site, int ni, int nj, int nk, const int4* offs, int noffs,
                       int nshells, bool wrap, double* partials, int blocks, double* out,
                       cudaStream_t stream) {
  if (wrap)
    shell_corr_kernel<true><<<blocks, kCorrThreads, 0, stream>>>(site, ni, nj, nk, offs, noffs,
                                                                  nshells, partials);
  else
    shell_corr_kernel<false><<<blocks, kCorrThreads, 0, stream>>>(site, ni, nj, nk, offs,
                                                                   noffs, nshells, partials);
  const int width = 2 * nshells + 1;
  sum_partials_kernel<<<(width + 127) / 128, 128, 0, stream>>>(partials, blocks, width, out);
}

void launch_projection(const LatticeView& L, int px, int py, int pz, long long m0, int nbins,
                       unsigned long long* hist, cudaStream_t stream) {
  const MomentGeom M = make_moment_geom(L);
  const uint64_t total = 2ull * M.per_colour;
  const uint64_t need = (total + 255) / 256;
  const uint64_t cap = (uint64_t)device_sms() * 4;
  const int blocks = (int)(need < cap ? (need ? need : 1) : cap);
  projection_kernel<<<blocks, 256, (size_t)nbins * sizeof(int), stream>>>(L, M, px, py, pz, m0,
                                                                          nbins, hist);
}

}  // namespace chll
