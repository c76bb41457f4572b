// mlp_model.hpp -- the learned ParMap warm-start model behind the aak_mlp
// handle of include/aak.h (shared by the C-ABI translation units).
#pragma once

#include <mutex>

#include "aak.h"
#include "../kernels/parmap_mlp.cuh"

struct aak_mlp {
  int device = 0;
  int num_sms = 148;
  aak::mlp::DeviceModel md{};
  void *block = nullptr;  // one allocation holding every device array of the model
  float *d_grad = nullptr;
  float *d_io = nullptr;  // staging for host-side predictions
  int64_t io_cap = 0;
  int64_t step = 0;
  float beta1 = 0.9f, beta2 = 0.999f, eps = 1e-8f;
  std::mutex mu;
};

namespace aak {
// Predictions y[n][3] (map coordinates) for host points x[n][4] = (p, e, iota, a).
int mlp_predict_host(aak_mlp *m, const double *x, double *y, int64_t n);
}  // namespace aak
