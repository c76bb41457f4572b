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
// across templates; the template spectra stream from HBM once.
#include "likelihood.cuh"

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

}  // namespace

void launch_inner_products(const InnerProductArgs &a, cudaStream_t stream) {
  if (a.ntemplates <= 0) return;
  dim3 grid(kIpBlocksPerTemplate, a.ntemplates);
  k_inner_partial<<<grid, kIpThreads, 0, stream>>>(a);
  k_inner_final<<<(a.ntemplates + 127) / 128, 128, 0, stream>>>(a.partial, kIpBlocksPerTemplate, a.ntemplates, a.out);
}

}  // namespace aak
