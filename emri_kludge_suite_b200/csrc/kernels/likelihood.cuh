// likelihood.cuh -- PSD-weighted inner products of batched template spectra
// with pre-weighted data (reference semantics: src/cuda/AAK_manager.cu:352-446,
// pygpuAAK/pygpuAAK.py:86-145).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace aak {

// Template spectra H (complex, interleaved re/im, row stride `row_doubles`
// doubles per template and channel), data D (pre-weighted, complex) and
// weights w (real) for both channels.  out[2k] = 4 Re sum conj(w H) D,
// out[2k+1] = 4 sum |w H|^2, summed over channels and the nbins bins.
struct InnerProductArgs {
  const double *H[2];  // channel I, II template spectra (ntemplates rows)
  int64_t row_doubles; // distance between template rows, in doubles
  const double *D[2];  // data spectra (nbins complex)
  const double *w[2];  // weights (nbins)
  int64_t nbins;
  int32_t ntemplates;
  double *partial;     // scratch: ntemplates x blocks_per_template x 2
  double *out;         // ntemplates x 2
};

constexpr int kIpThreads = 256;
constexpr int kIpBlocksPerTemplate = 64;

void launch_inner_products(const InnerProductArgs &a, cudaStream_t stream);

// The same products from FP32 spectra (an FP32 R2C transform of FP32
// template rows, row stride `row_floats` floats) and FP32 copies of the data
// and weights.  Each thread accumulates its bins in FP32 with Kahan
// compensation, a warp combines its lanes by a pairwise shuffle tree, and the
// warps' and CTAs' partial sums are added in FP64 in a fixed order.
struct InnerProductArgs32 {
  const float *H[2];   // channel I, II template spectra (ntemplates rows)
  int64_t row_floats;  // distance between template rows, in floats
  const float *D[2];   // data spectra (nbins complex, interleaved)
  const float *w[2];   // weights (nbins)
  int64_t nbins;
  int32_t ntemplates;
  double *partial;     // scratch: ntemplates x blocks_per_template x 2
  double *out;         // ntemplates x 2
};
void launch_inner_products_f32(const InnerProductArgs32 &a, cudaStream_t stream);

// Fisher-matrix Gram sums of finite-difference template spectra
// (pygpuAAK/pygpuAAK.py:269-300): rows 2i and 2i+1 of each channel hold the
// two evaluations of derivative i, D_i = scale w (H[2i+1] - H[2i]), and
// out[c][i][j] = 4 Re sum_f conj(D_i) D_j over the nbins bins, for both
// channels c (2 x nd x nd, symmetric).  Partial sums per CTA, then a fixed-
// order reduction (deterministic, no atomics).
constexpr int kFisherMaxDim = 16;
constexpr int kFisherBins = 64;     // bins staged per chunk
constexpr int kFisherThreads = 256;
struct FisherArgs {
  const double *H[2];
  int64_t row_doubles;
  const double *w[2];
  int64_t nbins;
  int32_t nd;
  double scale;        // applied to each difference
  double *partial;     // fisher_partial_doubles(nd, num_sms) scratch
  double *out;         // 2 x nd x nd
};
int fisher_grid(int num_sms, int64_t nbins);
inline int64_t fisher_partial_doubles(int nd, int grid) { return (int64_t)grid * nd * (nd + 1); }
void launch_fisher_gram(const FisherArgs &a, int num_sms, cudaStream_t stream);

}  // namespace aak
