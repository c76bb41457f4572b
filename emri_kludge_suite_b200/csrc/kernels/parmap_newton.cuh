// parmap_newton.cuh -- batched device solve of the Kerr -> AK map (ParMap,
// src/suite/KSParMap.cc:397-440) for every coarse point of a batch.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace aak {

// One coarse point: Kerr frequencies, p, the black-hole mass M and spin s, e,
// and Y = cos(iota) (taken on the host, so the device solve matches the host's).
struct ParmapJob {
  double Om[3];
  double p, M, s, e, Y;
};

// map (3 per point) = the solve of parmap_newton.hpp from the reference's
// guess, or from warm (3 per point, optional) with the fallback rule;
// iters / fallback (per point) as pm_newton / pm_newton_warm return them.
void launch_parmap_newton(const ParmapJob *jobs, int64_t n, const double *warm, double *map, int32_t *iters,
                          int32_t *fallback, cudaStream_t stream);

}  // namespace aak
