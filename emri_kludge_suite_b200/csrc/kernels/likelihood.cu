// likelihood.cu -- see likelihood.cuh.
//
// After cuFFT has turned each template channel into its half spectrum H_j,
// the reference multiplies by the weights (likelihood_prep) and calls
// cublasZdotc four times per template with a device sync after each.  Here one
// kernel reads every template bin once and produces both products for both
// channels: per thread a strided FP64 accumulation over bins, warp-shuffle
// and shared-memory reduction to one partial per CTA, then a second tiny
// kernel adds the partials of each template in a fixed order (deterministic,
// no atomics).  Data and weights (77 MB for N = 3.2e6) stay L2-resident
// across templates; the template spectra stream from HBM once.  An FP32
// variant reads FP32 spectra, data and weights and accumulates with Kahan
// compensation.
#include "likelihood.cuh"

#include <algorithm>

namespace aak {
namespace {

__global__ void __launch_bounds__(kIpThreads) k_inner_partial(InnerProductArgs a) {
  const int k = blockIdx.y;
  const int tid = threadIdx.x;
  double dh = 0.0, hh = 0.0;
  const int64_t stride = (int64_t)gridDim.x * kIpThreads;
  for (int ch = 0; ch < 2; ++ch) {
    const double2 *H = reinterpret_cast<const double2 *>(a.H[ch] + (int64_t)k * a.row_doubles);
    const double2 *D = reinterpret_cast<const double2 *>(a.D[ch]);
    const double *w = a.w[ch];
    for (int64_t j = (int64_t)blockIdx.x * kIpThreads + tid; j < a.nbins; j += stride) {
      const double2 h = H[j];
      const double2 d = __ldg(&D[j]);
      const double wj = __ldg(&w[j]);
      const double hr = wj * h.x, hi = wj * h.y;
      dh = fma(hr, d.x, fma(hi, d.y, dh));
      hh = fma(hr, hr, fma(hi, hi, hh));
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    dh += __shfl_xor_sync(0xffffffffu, dh, o);
    hh += __shfl_xor_sync(0xffffffffu, hh, o);
  }
  __shared__ double s[2][kIpThreads / 32];
  const int w = tid >> 5, l = tid & 31;
  if (l == 0) {
    s[0][w] = dh;
    s[1][w] = hh;
  }
  __syncthreads();
  if (tid == 0) {
    double a0 = 0.0, a1 = 0.0;
    for (int i = 0; i < kIpThreads / 32; ++i) {
      a0 += s[0][i];
      a1 += s[1][i];
    }
    a.partial[((int64_t)k * gridDim.x + blockIdx.x) * 2 + 0] = a0;
    a.partial[((int64_t)k * gridDim.x + blockIdx.x) * 2 + 1] = a1;
  }
}

// FP32 spectra: per-thread Kahan sums (the compensation c carries the low
// part each addition loses), then the warp's pairwise shuffle tree in FP32
// and the warps of the CTA in FP64.
__device__ __forceinline__ void kahan_add(float &sum, float &c, float x) {
  const float y = x - c;
  const float t = sum + y;
  c = (t - sum) - y;
  sum = t;
}

__global__ void __launch_bounds__(kIpThreads) k_inner_partial_f32(InnerProductArgs32 a) {
  const int k = blockIdx.y;
  const int tid = threadIdx.x;
  float dh = 0.f, hh = 0.f, cdh = 0.f, chh = 0.f;
  const int64_t stride = (int64_t)gridDim.x * kIpThreads;
  for (int ch = 0; ch < 2; ++ch) {
    const float2 *H = reinterpret_cast<const float2 *>(a.H[ch] + (int64_t)k * a.row_floats);
    const float2 *D = reinterpret_cast<const float2 *>(a.D[ch]);
    const float *w = a.w[ch];
    for (int64_t j = (int64_t)blockIdx.x * kIpThreads + tid; j < a.nbins; j += stride) {
      const float2 h = H[j];
      const float2 d = __ldg(&D[j]);
      const float wj = __ldg(&w[j]);
      const float hr = wj * h.x, hi = wj * h.y;
      kahan_add(dh, cdh, fmaf(hr, d.x, hi * d.y));
      kahan_add(hh, chh, fmaf(hr, hr, hi * hi));
    }
  }
  dh -= cdh;
  hh -= chh;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    dh += __shfl_xor_sync(0xffffffffu, dh, o);
    hh += __shfl_xor_sync(0xffffffffu, hh, o);
  }
  __shared__ double s[2][kIpThreads / 32];
  const int w = tid >> 5, l = tid & 31;
  if (l == 0) {
    s[0][w] = (double)dh;
    s[1][w] = (double)hh;
  }
  __syncthreads();
  if (tid == 0) {
    double a0 = 0.0, a1 = 0.0;
    for (int i = 0; i < kIpThreads / 32; ++i) {
      a0 += s[0][i];
      a1 += s[1][i];
    }
    a.partial[((int64_t)k * gridDim.x + blockIdx.x) * 2 + 0] = a0;
    a.partial[((int64_t)k * gridDim.x + blockIdx.x) * 2 + 1] = a1;
  }
}

__global__ void k_inner_final(const double *partial, int nblocks, int ntemplates, double *out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= ntemplates) return;
  double a0 = 0.0, a1 = 0.0;
  for (int b = 0; b < nblocks; ++b) {
    a0 += partial[((int64_t)k * nblocks + b) * 2 + 0];
    a1 += partial[((int64_t)k * nblocks + b) * 2 + 1];
  }
  out[2 * k + 0] = 4.0 * a0;
  out[2 * k + 1] = 4.0 * a1;
}

// Each CTA stages the weighted differences of kFisherBins bins of every
// derivative and both channels in shared memory (bins major, the derivative
// index padded to kFisherMaxDim + 1 so that the staging stores spread over
// the banks), then each thread adds the products of its one or two (channel,
// i <= j) pairs over the staged bins.  Each template row streams from HBM once.
__global__ void __launch_bounds__(kFisherThreads) k_fisher_partial(FisherArgs a) {
  __shared__ double2 sD[2][kFisherBins][kFisherMaxDim + 1];
  const int nd = a.nd, tid = threadIdx.x;
  const int npair = nd * (nd + 1) / 2, ncombo = 2 * npair;
  int cc[2] = {0, 0}, ii[2] = {0, 0}, jj[2] = {0, 0};
  double acc[2] = {0.0, 0.0};
  bool has[2];
#pragma unroll
  for (int m = 0; m < 2; ++m) {  // this thread's pairs q = tid, tid + kFisherThreads
    const int q = tid + m * kFisherThreads;
    has[m] = q < ncombo;
    if (!has[m]) continue;
    const int c = q / npair;
    int r = q - c * npair, i = 0;
    while (r >= nd - i) {  // row-major upper triangle: row i holds nd - i pairs
      r -= nd - i;
      ++i;
    }
    cc[m] = c;
    ii[m] = i;
    jj[m] = i + r;
  }
  const int64_t nchunks = (a.nbins + kFisherBins - 1) / kFisherBins;
  for (int64_t ck = blockIdx.x; ck < nchunks; ck += gridDim.x) {
    const int64_t b0 = ck * kFisherBins;
    __syncthreads();  // the previous chunk's products are done
#pragma unroll 4
    for (int idx = tid; idx < 2 * nd * kFisherBins; idx += kFisherThreads) {
      const int b = idx % kFisherBins, rest = idx / kFisherBins;
      const int i = rest % nd, c = rest / nd;
      const int64_t bin = b0 + b;
      double2 d = make_double2(0.0, 0.0);
      if (bin < a.nbins) {
        const double *Hc = c ? a.H[1] : a.H[0];  // selected, not indexed: the arguments stay in registers
        const double2 *Hu = reinterpret_cast<const double2 *>(Hc + (int64_t)(2 * i + 1) * a.row_doubles);
        const double2 *Hd = reinterpret_cast<const double2 *>(Hc + (int64_t)(2 * i) * a.row_doubles);
        const double2 u = Hu[bin], v = Hd[bin];
        const double wv = __ldg((c ? a.w[1] : a.w[0]) + bin) * a.scale;
        d = make_double2(wv * (u.x - v.x), wv * (u.y - v.y));
      }
      sD[c][b][i] = d;
    }
    __syncthreads();
#pragma unroll
    for (int m = 0; m < 2; ++m) {
      if (!has[m]) continue;
      const int c = cc[m], i = ii[m], j = jj[m];
      double s = acc[m];
#pragma unroll 8
      for (int b = 0; b < kFisherBins; ++b) {
        const double2 x = sD[c][b][i], y = sD[c][b][j];
        s = fma(x.x, y.x, fma(x.y, y.y, s));
      }
      acc[m] = s;
    }
  }
#pragma unroll
  for (int m = 0; m < 2; ++m)
    if (has[m]) a.partial[(int64_t)blockIdx.x * ncombo + tid + m * kFisherThreads] = acc[m];
}

// One warp per (channel, i <= j) pair: lane l adds the partials of CTAs
// l, l + 32, ... in order, then a fixed shuffle tree (deterministic).
__global__ void __launch_bounds__(kFisherThreads) k_fisher_final(FisherArgs a, int nblocks) {
  const int nd = a.nd, npair = nd * (nd + 1) / 2, ncombo = 2 * npair;
  const int q = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (q >= ncombo) return;
  double s = 0.0;
  for (int b = lane; b < nblocks; b += 32) s += a.partial[(int64_t)b * ncombo + q];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane != 0) return;
  const int c = q / npair;
  int r = q - c * npair, i = 0;
  while (r >= nd - i) {
    r -= nd - i;
    ++i;
  }
  const int j = i + r;
  a.out[(c * nd + i) * nd + j] = 4.0 * s;
  a.out[(c * nd + j) * nd + i] = 4.0 * s;
}

}  // namespace

int fisher_grid(int num_sms, int64_t nbins) {
  const int64_t nchunks = (nbins + kFisherBins - 1) / kFisherBins;
  return (int)std::max<int64_t>(1, std::min<int64_t>(nchunks, (int64_t)num_sms * 4));
}

void launch_fisher_gram(const FisherArgs &a, int num_sms, cudaStream_t stream) {
  if (a.nd <= 0 || a.nd > kFisherMaxDim) return;
  const int grid = fisher_grid(num_sms, a.nbins);
  k_fisher_partial<<<grid, kFisherThreads, 0, stream>>>(a);
  const int ncombo = a.nd * (a.nd + 1), warps = kFisherThreads / 32;
  k_fisher_final<<<(ncombo + warps - 1) / warps, kFisherThreads, 0, stream>>>(a, grid);
}

void launch_inner_products_f32(const InnerProductArgs32 &a, cudaStream_t stream) {
  if (a.ntemplates <= 0) return;
  dim3 grid(kIpBlocksPerTemplate, a.ntemplates);
  k_inner_partial_f32<<<grid, kIpThreads, 0, stream>>>(a);
  k_inner_final<<<(a.ntemplates + 127) / 128, 128, 0, stream>>>(a.partial, kIpBlocksPerTemplate, a.ntemplates, a.out);
}

void launch_inner_products(const InnerProductArgs &a, cudaStream_t stream) {
  if (a.ntemplates <= 0) return;
  dim3 grid(kIpBlocksPerTemplate, a.ntemplates);
  k_inner_partial<<<grid, kIpThreads, 0, stream>>>(a);
  k_inner_final<<<(a.ntemplates + 127) / 128, 128, 0, stream>>>(a.partial, kIpBlocksPerTemplate, a.ntemplates, a.out);
}

}  // namespace aak
