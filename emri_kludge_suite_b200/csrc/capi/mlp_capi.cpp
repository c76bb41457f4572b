// mlp_capi.cpp -- extern "C" surface of the learned ParMap warm start: the
// model handle (weights, Adam state, tensor-core kernels), the seeded
// point/label generator and the batched warm-vs-plain map solves.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "../host/parallel.hpp"
#include "../host/parmap_data.hpp"
#include "../host/pipeline.hpp"
#include "errors.hpp"
#include "mlp_model.hpp"

using namespace aak;

namespace {

int cuda_status(cudaError_t e) { return cuda_status_of(e); }

int use_device(int dev) {
  int n = 0;
  if (dev < 0) return AAK_ERR_INVALID_PARAM;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) {
    cudaGetLastError();
    return AAK_ERR_CUDA;
  }
  if (dev >= n) return AAK_ERR_INVALID_PARAM;
  return cuda_status(cudaSetDevice(dev));
}

size_t al256(size_t x) { return (x + 255) / 256 * 256; }

int check_error_flag(aak_mlp *m, cudaStream_t st) {
  int h = 0;
  int r = cuda_status(cudaMemcpyAsync(&h, m->md.error, sizeof(int), cudaMemcpyDeviceToHost, st));
  if (r == AAK_OK) r = cuda_status(cudaStreamSynchronize(st));
  if (r != AAK_OK) return r;
  return h ? AAK_ERR_DEVICE_TIMEOUT : AAK_OK;
}

int train_like(aak_mlp *m, const float *x, const float *y, const int32_t *perm, int64_t n, float lr, float *grad,
               float *loss, cudaStream_t st) {
  if (n <= 0 || n > mlp::kMaxTrainRows || !x || !y) return AAK_ERR_INVALID_PARAM;
  int r = use_device(m->device);
  if (r != AAK_OK) return r;
  const int ntiles = (int)((n + mlp::kTileRows - 1) / mlp::kTileRows);
  mlp::launch_gradients(m->md, x, y, perm, n, st);
  float bc1 = 1.f, bc2 = 1.f;
  if (lr > 0.f) {
    ++m->step;
    bc1 = 1.f - std::pow(m->beta1, (float)m->step);
    bc2 = 1.f - std::pow(m->beta2, (float)m->step);
  }
  mlp::launch_reduce_adam(m->md, ntiles, lr, m->beta1, m->beta2, m->eps, bc1, bc2, grad, st);
  if ((r = cuda_status(cudaGetLastError())) != AAK_OK) return r;
  if (loss) {
    std::vector<float> lp(ntiles);
    if ((r = cuda_status(cudaMemcpyAsync(lp.data(), m->md.loss_part, ntiles * sizeof(float), cudaMemcpyDeviceToHost,
                                         st))) != AAK_OK)
      return r;
    if ((r = check_error_flag(m, st)) != AAK_OK) return r;
    double s = 0.0;
    for (float v : lp) s += v;
    *loss = (float)(s / (3.0 * (double)n));
  }
  return AAK_OK;
}

}  // namespace

namespace aak {

int mlp_predict_host(aak_mlp *m, const double *x, double *y, int64_t n) {
  if (!m || n < 0 || (n > 0 && (!x || !y))) return AAK_ERR_INVALID_PARAM;
  if (n == 0) return AAK_OK;
  std::lock_guard<std::mutex> lk(m->mu);
  int r = use_device(m->device);
  if (r != AAK_OK) return r;
  if (m->io_cap < n) {
    if (m->d_io) cudaFree(m->d_io);
    m->d_io = nullptr;
    m->io_cap = 0;
    if ((r = cuda_status(cudaMalloc(&m->d_io, (size_t)n * 7 * sizeof(float)))) != AAK_OK) return r;
    m->io_cap = n;
  }
  std::vector<float> xf((size_t)n * 4), yf((size_t)n * 3);
  for (int64_t i = 0; i < 4 * n; ++i) xf[i] = (float)x[i];
  float *dx = m->d_io, *dy = m->d_io + 4 * n;
  if ((r = cuda_status(cudaMemcpy(dx, xf.data(), xf.size() * sizeof(float), cudaMemcpyHostToDevice))) != AAK_OK)
    return r;
  mlp::launch_forward(m->md, dx, dy, n, m->num_sms, 0);
  if ((r = cuda_status(cudaGetLastError())) != AAK_OK) return r;
  if ((r = cuda_status(cudaMemcpy(yf.data(), dy, yf.size() * sizeof(float), cudaMemcpyDeviceToHost))) != AAK_OK)
    return r;
  if ((r = check_error_flag(m, 0)) != AAK_OK) return r;
  for (int64_t i = 0; i < 3 * n; ++i) y[i] = (double)yf[i];
  return AAK_OK;
}

}  // namespace aak

extern "C" {

int aak_mlp_num_params(void) { return mlp::kParams; }
int aak_mlp_max_train_rows(void) { return mlp::kMaxTrainRows; }

int aak_mlp_create(int32_t device, aak_mlp **out) {
  if (!out) return AAK_ERR_INVALID_PARAM;
  *out = nullptr;
  int r = use_device(device);
  if (r != AAK_OK) return r;
  aak_mlp *m = new (std::nothrow) aak_mlp();
  if (!m) return AAK_ERR_NO_MEMORY;
  m->device = device;
  int sms = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) == cudaSuccess && sms > 0) m->num_sms = sms;
  const size_t P = mlp::kParams;
  const size_t o_w = 0, o_m = o_w + al256(P * 4), o_v = o_m + al256(P * 4), o_wq = o_v + al256(P * 4),
               o_img = o_wq + al256(P * 4), o_part = o_img + al256(4 * (size_t)mlp::kImgElems * 2),
               o_loss = o_part + al256((size_t)mlp::kMaxTrainTiles * mlp::kPartStride * 4),
               o_err = o_loss + al256(mlp::kMaxTrainTiles * 4), o_grad = o_err + 256, total = o_grad + al256(P * 4);
  unsigned char *b = nullptr;
  if ((r = cuda_status(cudaMalloc(&b, total))) != AAK_OK) {
    delete m;
    return r;
  }
  cudaMemset(b, 0, total);
  m->block = b;
  m->md.w = reinterpret_cast<float *>(b + o_w);
  m->md.m = reinterpret_cast<float *>(b + o_m);
  m->md.v = reinterpret_cast<float *>(b + o_v);
  m->md.wq = reinterpret_cast<float *>(b + o_wq);
  m->md.img = reinterpret_cast<uint16_t *>(b + o_img);
  m->md.partial = reinterpret_cast<float *>(b + o_part);
  m->md.loss_part = reinterpret_cast<float *>(b + o_loss);
  m->md.error = reinterpret_cast<int *>(b + o_err);
  m->d_grad = reinterpret_cast<float *>(b + o_grad);
  for (int k = 0; k < 4; ++k) {
    m->md.norm.in_shift[k] = 0.f;
    m->md.norm.in_scale[k] = 1.f;
  }
  for (int k = 0; k < 3; ++k) {
    m->md.norm.out_shift[k] = 0.f;
    m->md.norm.out_scale[k] = 1.f;
  }
  mlp::launch_publish(m->md, 0);
  if ((r = cuda_status(cudaDeviceSynchronize())) != AAK_OK) {
    cudaFree(b);
    delete m;
    return r;
  }
  *out = m;
  return AAK_OK;
}

void aak_mlp_destroy(aak_mlp *m) {
  if (!m) return;
  if (use_device(m->device) == AAK_OK) {
    if (m->block) cudaFree(m->block);
    if (m->d_io) cudaFree(m->d_io);
  }
  delete m;
}

int aak_mlp_set_params(aak_mlp *m, const float *params) {
  if (!m || !params) return AAK_ERR_INVALID_PARAM;
  std::lock_guard<std::mutex> lk(m->mu);
  int r = use_device(m->device);
  if (r != AAK_OK) return r;
  const size_t bytes = (size_t)mlp::kParams * sizeof(float);
  if ((r = cuda_status(cudaMemcpy(m->md.w, params, bytes, cudaMemcpyHostToDevice))) != AAK_OK) return r;
  cudaMemset(m->md.m, 0, bytes);
  cudaMemset(m->md.v, 0, bytes);
  cudaMemset(m->md.error, 0, sizeof(int));
  m->step = 0;
  mlp::launch_publish(m->md, 0);
  return cuda_status(cudaDeviceSynchronize());
}

int aak_mlp_get_params(aak_mlp *m, float *params) {
  if (!m || !params) return AAK_ERR_INVALID_PARAM;
  std::lock_guard<std::mutex> lk(m->mu);
  int r = use_device(m->device);
  if (r != AAK_OK) return r;
  return cuda_status(cudaMemcpy(params, m->md.w, (size_t)mlp::kParams * sizeof(float), cudaMemcpyDeviceToHost));
}

int aak_mlp_set_norm(aak_mlp *m, const float in_shift[4], const float in_scale[4], const float out_shift[3],
                     const float out_scale[3]) {
  if (!m || !in_shift || !in_scale || !out_shift || !out_scale) return AAK_ERR_INVALID_PARAM;
  std::lock_guard<std::mutex> lk(m->mu);
  for (int k = 0; k < 4; ++k) {
    m->md.norm.in_shift[k] = in_shift[k];
    m->md.norm.in_scale[k] = in_scale[k];
  }
  for (int k = 0; k < 3; ++k) {
    if (!(out_scale[k] != 0.f)) return AAK_ERR_INVALID_PARAM;
    m->md.norm.out_shift[k] = out_shift[k];
    m->md.norm.out_scale[k] = out_scale[k];
  }
  return AAK_OK;
}

int aak_mlp_set_adam(aak_mlp *m, float beta1, float beta2, float eps) {
  if (!m || !(beta1 >= 0.f && beta1 < 1.f) || !(beta2 >= 0.f && beta2 < 1.f) || !(eps > 0.f))
    return AAK_ERR_INVALID_PARAM;
  std::lock_guard<std::mutex> lk(m->mu);
  m->beta1 = beta1;
  m->beta2 = beta2;
  m->eps = eps;
  return AAK_OK;
}

int aak_mlp_forward(aak_mlp *m, const float *d_x, float *d_y, int64_t n, void *stream) {
  if (!m || n < 0 || (n > 0 && (!d_x || !d_y))) return AAK_ERR_INVALID_PARAM;
  std::lock_guard<std::mutex> lk(m->mu);
  int r = use_device(m->device);
  if (r != AAK_OK) return r;
  mlp::launch_forward(m->md, d_x, d_y, n, m->num_sms, (cudaStream_t)stream);
  return cuda_status(cudaGetLastError());
}

int aak_mlp_gradients(aak_mlp *m, const float *d_x, const float *d_y, const int32_t *d_perm, int64_t n, float *d_grad,
                      float *loss, void *stream) {
  if (!m || !d_grad) return AAK_ERR_INVALID_PARAM;
  std::lock_guard<std::mutex> lk(m->mu);
  return train_like(m, d_x, d_y, d_perm, n, 0.f, d_grad, loss, (cudaStream_t)stream);
}

int aak_mlp_train_step(aak_mlp *m, const float *d_x, const float *d_y, const int32_t *d_perm, int64_t n, float lr,
                       float *loss, void *stream) {
  if (!m || !(lr > 0.f)) return AAK_ERR_INVALID_PARAM;
  std::lock_guard<std::mutex> lk(m->mu);
  return train_like(m, d_x, d_y, d_perm, n, lr, nullptr, loss, (cudaStream_t)stream);
}

int aak_mlp_status(aak_mlp *m) {
  if (!m) return AAK_ERR_INVALID_PARAM;
  std::lock_guard<std::mutex> lk(m->mu);
  int r = use_device(m->device);
  if (r != AAK_OK) return r;
  return check_error_flag(m, 0);
}

int aak_mlp_predict_host(aak_mlp *m, const double *x, double *y, int64_t n) { return mlp_predict_host(m, x, y, n); }

// ------------------------------------------------------------------ points, labels, solves
int aak_parmap_separatrix(double e, double iota, double a, double *p_sep) {
  if (!p_sep || !(e > 0.0 && e < 1.0) || !(std::fabs(a) < 1.0) || !std::isfinite(iota)) return AAK_ERR_INVALID_PARAM;
  *p_sep = separatrix_p(e, std::cos(iota), a, 1e-12);
  return AAK_OK;
}

int aak_parmap_dataset(int64_t n, uint64_t seed, uint64_t first_index, int32_t nthreads, double *x, double *y,
                       double *omega, int32_t *iters) {
  if (n < 0 || (n > 0 && (!x || !y || !omega || !iters))) return AAK_ERR_INVALID_PARAM;
  parallel_for(n, nthreads, [&](int64_t i) {
    double *xi = x + 4 * i, *om = omega + 3 * i, map[3];
    parmap_draw(seed, first_index + (uint64_t)i, xi);
    kerr_frequencies(xi, om);
    const int it = parmap(om, xi[0], kParmapLabelMass, xi[3], xi[1], xi[2], nullptr, map);
    iters[i] = it;
    if (it >= 0) parmap_to_coords(xi, kParmapLabelMass, map, y + 3 * i);
    else y[3 * i] = y[3 * i + 1] = y[3 * i + 2] = NAN;
  });
  return AAK_OK;
}

int aak_parmap_solve_batch(int64_t n, const double *x, const double *omega, const double *guess, int32_t nthreads,
                           double *y, int32_t *iters, int32_t *iters_to_tol, double *residual, double *guess_residual,
                           int32_t *fallback) {
  if (n < 0 || (n > 0 && (!x || !omega || !y || !iters))) return AAK_ERR_INVALID_PARAM;
  parallel_for(n, nthreads, [&](int64_t i) {
    const double *xi = x + 4 * i, *om = omega + 3 * i;
    const double M = kParmapLabelMass;
    double x0[3], map[3];
    int it, fb = 0, tol = -1;
    if (guess) {
      parmap_from_coords(xi, M, guess + 3 * i, x0);
      if (guess_residual) guess_residual[i] = parmap_residual_norm(om, M, xi[1], xi[2], x0);
      it = parmap_warm(om, xi[0], M, xi[3], xi[1], xi[2], x0, map, &fb, &tol);
    } else {
      it = parmap(om, xi[0], M, xi[3], xi[1], xi[2], nullptr, map, &tol);
    }
    iters[i] = it;
    if (iters_to_tol) iters_to_tol[i] = tol;
    if (fallback) fallback[i] = fb;
    if (residual) residual[i] = parmap_residual_norm(om, M, xi[1], xi[2], map);
    parmap_to_coords(xi, M, map, y + 3 * i);
  });
  return AAK_OK;
}

}  // extern "C"
