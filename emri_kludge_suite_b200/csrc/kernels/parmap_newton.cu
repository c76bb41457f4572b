// parmap_newton.cu -- see parmap_newton.cuh.  Built with -fmad=false: the
// solve then performs the host's IEEE operations one for one, and each point's
// root equals the host's bit for bit.
#include "parmap_newton.cuh"

#include "../host/parmap_newton.hpp"

namespace aak {
namespace {

// One thread per coarse point; the solve is a few dozen residual evaluations
// of 3PN polynomials, so the batch is latency-bound and small.
__global__ void __launch_bounds__(128) k_parmap_newton(const ParmapJob *__restrict__ jobs, int64_t n,
                                                       const double *__restrict__ warm, double *__restrict__ map,
                                                       int32_t *__restrict__ iters, int32_t *__restrict__ fallback) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const ParmapJob j = jobs[i];
  double m[3];
  int fb = 0, it;
  if (warm) it = pm_newton_warm(j.Om, j.p, j.M, j.s, j.e, j.Y, warm + 3 * i, m, &fb, nullptr);
  else it = pm_newton(j.Om, j.p, j.M, j.s, j.e, j.Y, nullptr, m, nullptr);
  map[3 * i] = m[0];
  map[3 * i + 1] = m[1];
  map[3 * i + 2] = m[2];
  iters[i] = it;
  fallback[i] = fb;
}

}  // namespace

void launch_parmap_newton(const ParmapJob *jobs, int64_t n, const double *warm, double *map, int32_t *iters,
                          int32_t *fallback, cudaStream_t stream) {
  if (n <= 0) return;
  k_parmap_newton<<<(unsigned)((n + 127) / 128), 128, 0, stream>>>(jobs, n, warm, map, iters, fallback);
}

}  // namespace aak
