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

}  // namespace aak
