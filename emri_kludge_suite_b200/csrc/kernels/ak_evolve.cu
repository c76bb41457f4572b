// ak_evolve.cu -- the coarse AK evolution beyond the fit window on the GPU,
// one thread per source: the Adams-Bashforth-2 recurrence of the AK (e, v)
// equations with the reference's freezing once the trajectory turns
// unphysical (src/suite/AAK.cc:62-144; host version: pipeline.cpp evolve()).
//
// A source's recurrence is serial, so a GPU thread runs it at the latency of
// its dependent FP64 chain (a log, a square root, two 3PN polynomials and two
// divisions per step); the device gains where many sources of similar length
// run at once (likelihood template batches) and loses where one long source
// sets the critical path (batches with a few sources of millions of steps).
// Compiled without FMA contraction, as the host computes it: only log() may
// round differently from the host's.
#include <cuda_runtime.h>

#include "../ak_rates.hpp"
#include "../host/pipeline.hpp"
#include "ak_evolve.cuh"

namespace aak {
namespace {

__global__ void __launch_bounds__(128) k_ak_evolve(EvolveJob *jobs, int n, double *e, double *v) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  EvolveJob J = jobs[s];
  double *E = e + J.off, *V = v + J.off;
  int jm = J.j_max;
  const int jmt = J.j_max_temp;
  double ed = J.edot, vd = J.vdot;
  double ec = E[J.j_first], vc = V[J.j_first];
  for (int j = J.j_first; j < J.j_end; ++j) {
    const double edm = ed, vdm = vd;
    ak_rates(vc, ec, J.coslam, J.mu, J.M0, J.S0, &ed, &vd);
    double en = ec + (1.5 * ed - .5 * edm) * J.dt_large;
    double vn = vc + (1.5 * vd - .5 * vdm) * J.dt_large;
    if (en < 0. || vn < vc || isnan(en) || isnan(vn)) {
      if (jm == jmt) jm = j;
      en = E[jm];
      vn = V[jm];
    }
    E[j + 1] = en;
    V[j + 1] = vn;
    ec = en;
    vc = vn;
  }
  J.j_max = jm;
  J.j_max_temp = jm;
  J.edot = ed;
  J.vdot = vd;
  jobs[s] = J;
}

}  // namespace

void launch_ak_evolve(EvolveJob *d_jobs, int n, double *d_e, double *d_v, cudaStream_t stream) {
  if (n <= 0) return;
  k_ak_evolve<<<(n + 127) / 128, 128, 0, stream>>>(d_jobs, n, d_e, d_v);
}

}  // namespace aak
