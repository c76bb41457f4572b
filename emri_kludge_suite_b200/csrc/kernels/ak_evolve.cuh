// ak_evolve.cuh -- device evolution of the coarse AK trajectories of a batch.
#pragma once

#include <cuda_runtime.h>

namespace aak {

struct EvolveJob;

// One thread per job: AK (e, v) entries j_first + 1 .. j_end of each job's
// segment of d_e, d_v (entries 0 .. j_first filled), as the host's evolve();
// each job's freeze indices and last rates are written back.
void launch_ak_evolve(EvolveJob *d_jobs, int n, double *d_e, double *d_v, cudaStream_t stream);

}  // namespace aak
