// parmap_mlp.cuh -- the learned warm start of the Kerr -> AK map: a
// 4 -> 128 -> 128 -> 128 -> 3 SiLU network with BF16 weights and activations
// and FP32 accumulation.  The two 128 x 128 layers (forward and backward) run
// on the 5th-generation tensor cores (tcgen05.mma, accumulators in TMEM); the
// 4-wide input and 3-wide output layers run on the FP32 pipe.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace aak {
namespace mlp {

constexpr int kIn = 4, kHid = 128, kOut = 3;
// Flat FP32 parameter vector: W1[128][4] b1[128] W2[128][128] b2[128]
// W3[128][128] b3[128] W4[3][128] b4[3]; W[o][i] maps input i to output o.
constexpr int kOffW1 = 0;
constexpr int kOffB1 = kOffW1 + kHid * kIn;
constexpr int kOffW2 = kOffB1 + kHid;
constexpr int kOffB2 = kOffW2 + kHid * kHid;
constexpr int kOffW3 = kOffB2 + kHid;
constexpr int kOffB3 = kOffW3 + kHid * kHid;
constexpr int kOffW4 = kOffB3 + kHid;
constexpr int kOffB4 = kOffW4 + kOut * kHid;
constexpr int kParams = kOffB4 + kOut;  // 34051
// Row stride of the per-tile gradient partials: a multiple of 64 floats, so
// every row (and the W2 / W3 blocks in it) stays 16-byte aligned for float4 stores.
constexpr int kPartStride = (kParams + 63) / 64 * 64;

constexpr int kTileRows = 128;              // batch rows per CTA tile (= MMA M)
constexpr int kImgElems = kHid * kHid;      // one 128 x 128 BF16 operand image
constexpr int kMaxTrainRows = 16384;        // rows per training step
constexpr int kMaxTrainTiles = kMaxTrainRows / kTileRows;

// Input features f = (g(x) - in_shift) * in_scale with g(x) = (1/sqrt(p), e,
// cos iota, a); outputs y = net(f) * out_scale + out_shift (map coordinates).
struct Norm {
  float in_shift[4], in_scale[4];
  float out_shift[3], out_scale[3];
};

struct DeviceModel {
  float *w;          // kParams FP32 master weights
  float *m, *v;      // Adam moments
  float *wq;         // kParams: weights rounded to BF16 (biases unrounded), as FP32
  uint16_t *img;     // 4 x kImgElems BF16 operand images (tcgen05 K-major layout): W2, W3, W2^T, W3^T
  float *partial;    // kMaxTrainTiles x kPartStride per-tile gradients
  float *loss_part;  // kMaxTrainTiles per-tile loss sums
  int *error;        // nonzero after a bounded wait gave up
  Norm norm;
};

// wq and the operand images from the master weights.
void launch_publish(const DeviceModel &md, cudaStream_t st);
// y[n][3] (map coordinates) for x[n][4] = (p, e, iota, a).
void launch_forward(const DeviceModel &md, const float *x, float *y, int64_t n, int num_sms, cudaStream_t st);
// Per-tile gradients of the mean squared error in normalised output units for
// rows perm[0..n) (perm may be null: rows 0..n) of (x, y_true); n <= kMaxTrainRows.
void launch_gradients(const DeviceModel &md, const float *x, const float *y_true, const int32_t *perm, int64_t n,
                      cudaStream_t st);
// Sum the per-tile gradients (fixed order) into grad (optional) and, when
// lr > 0, apply one Adam step and republish.
void launch_reduce_adam(const DeviceModel &md, int ntiles, float lr, float beta1, float beta2, float eps, float bc1,
                        float bc2, float *grad, cudaStream_t st);

}  // namespace mlp
}  // namespace aak
