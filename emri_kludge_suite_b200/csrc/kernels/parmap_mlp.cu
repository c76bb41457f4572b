// parmap_mlp.cu -- see parmap_mlp.cuh.
//
// One CTA of 128 threads owns a tile of 128 batch rows, one thread per row.
// The 128 x 128 layers are tcgen05.mma (kind::f16, BF16 x BF16 -> FP32,
// M = N = 128, K = 16 per instruction) issued by one thread on operands staged
// in shared memory in the K-major, no-swizzle canonical layout, with the FP32
// accumulators in tensor memory; each thread reads its row back with
// tcgen05.ld (32x32b: warp w owns TMEM lanes 32w .. 32w + 31 = rows).
// Activations are rounded to BF16 where they enter a tensor-core product.
#include "parmap_mlp.cuh"

#include <cuda_bf16.h>

namespace aak {
namespace mlp {

namespace {

// ------------------------------------------------------------------ BF16
__device__ __forceinline__ uint32_t bf16_bits(float x) { return (uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(x)); }
__device__ __forceinline__ float bf16_round(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }
__device__ __forceinline__ float bf16_val(uint16_t b) { return __uint_as_float((uint32_t)b << 16); }

// ------------------------------------------------------------------ operand layout
// K-major, no swizzle: core matrices of 8 rows x 16 bytes (8 BF16) stored as
// 128 contiguous bytes; core (r/8, k/8) starts at byte (r/8) * 2048 + (k/8) * 128.
// In descriptor terms LBO = 128 B (K-adjacent cores), SBO = 2048 B (8-row groups).
__host__ __device__ __forceinline__ int canon(int r, int k) {
  return (((r >> 3) * 16 + (k >> 3)) << 6) + ((r & 7) << 3) + (k & 7);
}
constexpr uint32_t kLBO = 128, kSBO = 2048;
// Instruction descriptor (kind::f16): D F32 (bits 4-5 = 1), A BF16 (7-9 = 1),
// B BF16 (10-12 = 1), both K-major (15, 16 = 0), N >> 3 at 17-22, M >> 4 at 24-28.
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((128u >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ uint32_t saddr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor: start >> 4 (bits 0-13), LBO >> 4 (16-29),
// SBO >> 4 (32-45), descriptor version 1 (46-47), no swizzle (61-63 = 0).
__device__ __forceinline__ uint64_t smem_desc(uint32_t a) {
  return (uint64_t)((a & 0x3FFFFu) >> 4) | ((uint64_t)(kLBO >> 4) << 16) | ((uint64_t)(kSBO >> 4) << 32) |
         (1ull << 46);
}

// D[128 x 128] (+)= A[128 x K] B[128 x K]^T with K = 128 (8 instructions).
__device__ __forceinline__ void mma_128(uint32_t tmem_d, uint32_t a, uint32_t b, bool accumulate) {
#pragma unroll
  for (int s = 0; s < 8; ++s) {
    const uint64_t da = smem_desc(a + s * 256), db = smem_desc(b + s * 256);
    const uint32_t acc = (s > 0 || accumulate) ? 1u : 0u;
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(kIdesc), "r"(acc)
        : "memory");
  }
}
__device__ __forceinline__ void mma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// generic-proxy shared-memory writes -> visible to the tensor core (async proxy)
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint32_t mbar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// Bounded wait on the phase with the given parity (about two seconds of SM clock).
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
  const long long t0 = clock64();
  for (;;) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred P;\n\tmbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P;\n\t}\n"
        : "=r"(done)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (done) return true;
    if (clock64() - t0 > 4000000000ll) return false;
  }
}

__device__ __forceinline__ void tmem_alloc(uint32_t slot, uint32_t ncols) {  // whole warp
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot), "r"(ncols) : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_free(uint32_t taddr, uint32_t ncols) {  // whole warp
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
// 16 consecutive FP32 columns of this thread's TMEM lane (load + wait in one statement).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float v[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, "
      "[%16];\n\ttcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// ------------------------------------------------------------------ activation
__device__ __forceinline__ float sigm(float z) { return 1.0f / (1.0f + expf(-z)); }
__device__ __forceinline__ float silu(float z) { return z * sigm(z); }
__device__ __forceinline__ float dsilu(float z) {
  const float s = sigm(z);
  return s * (1.0f + z * (1.0f - s));
}

__device__ __forceinline__ void features(const Norm &nm, const float *xr, float f[4]) {
  const float g[4] = {rsqrtf(xr[0]), xr[1], cosf(xr[2]), xr[3]};
#pragma unroll
  for (int k = 0; k < 4; ++k) f[k] = (g[k] - nm.in_shift[k]) * nm.in_scale[k];
}

__device__ __forceinline__ float layer1(const float *W1, const float *b1, const float f[4], int o) {
  return b1[o] + W1[4 * o] * f[0] + W1[4 * o + 1] * f[1] + W1[4 * o + 2] * f[2] + W1[4 * o + 3] * f[3];
}

// store 8 BF16 (packed in q[4]) at row r, columns k0 .. k0 + 7 of a K-major image
__device__ __forceinline__ void put_row8(uint16_t *img, int r, int k0, const uint32_t q[4]) {
  *reinterpret_cast<uint4 *>(img + canon(r, k0)) = make_uint4(q[0], q[1], q[2], q[3]);
}
// store 8 BF16 at rows k0 .. k0 + 7, column c (transposed write)
__device__ __forceinline__ void put_col8(uint16_t *img, int k0, int c, const uint32_t q[4]) {
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    img[canon(k0 + 2 * j, c)] = (uint16_t)(q[j] & 0xFFFFu);
    img[canon(k0 + 2 * j + 1, c)] = (uint16_t)(q[j] >> 16);
  }
}

__device__ __forceinline__ void copy_img(uint16_t *dst, const uint16_t *src) {
  const uint4 *s = reinterpret_cast<const uint4 *>(src);
  uint4 *d = reinterpret_cast<uint4 *>(dst);
  for (int i = threadIdx.x; i < kImgElems / 8; i += blockDim.x) d[i] = s[i];
}

// One thread waits for the MMA phase; everyone learns the outcome.
__device__ __forceinline__ bool wait_mma(uint32_t mbar, uint32_t parity, volatile int *flag, int *err) {
  if (threadIdx.x == 0 && !mbar_wait(mbar, parity)) {
    *flag = 1;
    atomicExch(err, 1);
  }
  __syncthreads();
  return *flag == 0;
}

// ------------------------------------------------------------------ publish
__device__ __forceinline__ bool is_weight(int p) {
  return p < kOffB1 || (p >= kOffW2 && p < kOffB2) || (p >= kOffW3 && p < kOffB3) || (p >= kOffW4 && p < kOffB4);
}
__device__ __forceinline__ void publish_one(const DeviceModel &md, int p, float w) {
  md.wq[p] = is_weight(p) ? bf16_round(w) : w;
  if (p >= kOffW2 && p < kOffB2) {
    const int q = p - kOffW2, o = q >> 7, i = q & 127;
    const uint16_t b = (uint16_t)bf16_bits(w);
    md.img[canon(o, i)] = b;
    md.img[2 * kImgElems + canon(i, o)] = b;
  } else if (p >= kOffW3 && p < kOffB3) {
    const int q = p - kOffW3, o = q >> 7, i = q & 127;
    const uint16_t b = (uint16_t)bf16_bits(w);
    md.img[kImgElems + canon(o, i)] = b;
    md.img[3 * kImgElems + canon(i, o)] = b;
  }
}

__global__ void k_publish(DeviceModel md) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < kParams) publish_one(md, p, md.w[p]);
}

__global__ void k_reduce_adam(DeviceModel md, int ntiles, float lr, float beta1, float beta2, float eps, float bc1,
                              float bc2, float *grad) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= kParams) return;
  float g = 0.0f;
  for (int t = 0; t < ntiles; ++t) g += md.partial[(int64_t)t * kPartStride + p];
  if (grad) grad[p] = g;
  if (lr > 0.0f) {
    const float m = beta1 * md.m[p] + (1.0f - beta1) * g;
    const float v = beta2 * md.v[p] + (1.0f - beta2) * g * g;
    md.m[p] = m;
    md.v[p] = v;
    const float w = md.w[p] - lr * (m / bc1) / (sqrtf(v / bc2) + eps);
    md.w[p] = w;
    publish_one(md, p, w);
  }
}

// ------------------------------------------------------------------ inference
struct FwdSmem {
  uint16_t A[kImgElems];   // activations of the tile, K-major
  uint16_t W2[kImgElems];  // W2 image (B operand: N = out, K = in)
  uint16_t W3[kImgElems];
  float W1[kHid * kIn];
  float W4[kOut * kHid];
  float b1[kHid], b2[kHid], b3[kHid], b4[4];
  unsigned long long mbar;
  uint32_t tmem_slot;
  int flag;
};

__global__ void __launch_bounds__(kTileRows) k_forward(DeviceModel md, const float *__restrict__ x,
                                                       float *__restrict__ y, int64_t n) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  FwdSmem &S = *reinterpret_cast<FwdSmem *>(smem_raw);
  const int t = threadIdx.x, warp = t >> 5;
  copy_img(S.W2, md.img);
  copy_img(S.W3, md.img + kImgElems);
  for (int i = t; i < kHid * kIn; i += kTileRows) S.W1[i] = md.wq[kOffW1 + i];
  for (int i = t; i < kOut * kHid; i += kTileRows) S.W4[i] = md.wq[kOffW4 + i];
  S.b1[t] = md.w[kOffB1 + t];
  S.b2[t] = md.w[kOffB2 + t];
  S.b3[t] = md.w[kOffB3 + t];
  if (t < kOut) S.b4[t] = md.w[kOffB4 + t];
  const uint32_t mbar = saddr(&S.mbar);
  if (t == 0) {
    mbar_init(mbar);
    S.flag = 0;
  }
  if (warp == 0) tmem_alloc(saddr(&S.tmem_slot), 128);
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = S.tmem_slot;
  const uint32_t lane = tmem + ((uint32_t)(warp * 32) << 16);
  const Norm nm = md.norm;
  uint32_t phase = 0;
  bool ok = true;
  const int64_t ntiles = (n + kTileRows - 1) / kTileRows;
  for (int64_t g = blockIdx.x; g < ntiles && ok; g += gridDim.x) {
    const int64_t row = g * kTileRows + t;
    const bool valid = row < n;
    float f[4] = {0.f, 0.f, 0.f, 0.f};
    if (valid) features(nm, x + 4 * row, f);
    // layer 1 (FP32 pipe) -> A
    for (int c = 0; c < 16; ++c) {
      uint32_t q[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int o = 8 * c + 2 * j;
        const float a0 = valid ? silu(layer1(S.W1, S.b1, f, o)) : 0.f;
        const float a1 = valid ? silu(layer1(S.W1, S.b1, f, o + 1)) : 0.f;
        q[j] = bf16_bits(a0) | (bf16_bits(a1) << 16);
      }
      put_row8(S.A, t, 8 * c, q);
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    if (t == 0) {
      tc_fence_after();
      mma_128(tmem, saddr(S.A), saddr(S.W2), false);
      mma_commit(mbar);
    }
    if (!(ok = wait_mma(mbar, phase, &S.flag, md.error))) break;
    phase ^= 1;
    tc_fence_after();
    // layer 2 epilogue -> A
    for (int c = 0; c < 8; ++c) {
      float v[16];
      tmem_ld16(lane + 16 * c, v);
      uint32_t q[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const int o = 16 * c + 2 * j;
        const float a0 = valid ? silu(v[2 * j] + S.b2[o]) : 0.f;
        const float a1 = valid ? silu(v[2 * j + 1] + S.b2[o + 1]) : 0.f;
        q[j] = bf16_bits(a0) | (bf16_bits(a1) << 16);
      }
      put_row8(S.A, t, 16 * c, q);
      put_row8(S.A, t, 16 * c + 8, q + 4);
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    if (t == 0) {
      tc_fence_after();
      mma_128(tmem, saddr(S.A), saddr(S.W3), false);
      mma_commit(mbar);
    }
    if (!(ok = wait_mma(mbar, phase, &S.flag, md.error))) break;
    phase ^= 1;
    tc_fence_after();
    // layer 3 epilogue + output layer (FP32 pipe)
    float acc[3] = {S.b4[0], S.b4[1], S.b4[2]};
    for (int c = 0; c < 8; ++c) {
      float v[16];
      tmem_ld16(lane + 16 * c, v);
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const int o = 16 * c + j;
        const float a = bf16_round(silu(v[j] + S.b3[o]));
        acc[0] += S.W4[o] * a;
        acc[1] += S.W4[kHid + o] * a;
        acc[2] += S.W4[2 * kHid + o] * a;
      }
    }
    if (valid)
      for (int j = 0; j < 3; ++j) y[3 * row + j] = acc[j] * nm.out_scale[j] + nm.out_shift[j];
  }
  if (!ok && t == 0) mbar_wait(mbar, phase);  // let an MMA still in flight drain (bounded)
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) tmem_free(tmem, 128);
}

// ------------------------------------------------------------------ training
struct TrainSmem {
  uint16_t W[kImgElems];    // weight operand slot
  uint16_t X0[kImgElems];   // a1, then a2 ([row][in], K-major); then a3 (plain row-major)
  uint16_t D0[kImgElems];   // dz3, then dz2 ([row][out], K-major); X0|D0: 64 KB FP32 scratch for dz1
  uint16_t XT1[kImgElems];  // a1^T ([in][row], K-major)
  uint16_t XT2[kImgElems];  // a2^T
  uint16_t DT[kImgElems];   // dz^T ([out][row], K-major)
  float f[kTileRows][4];
  float dy[kTileRows][3];
  float W1[kHid * kIn];
  float W4[kOut * kHid];
  float b1[kHid], b2[kHid], b3[kHid], b4[4];
  float red[4];
  unsigned long long mbar;
  uint32_t tmem_slot;
  int flag;
};

__device__ __forceinline__ float sum_row_T(const uint16_t *img, int r) {  // sum over k of image row r
  float s = 0.f;
  for (int c = 0; c < 16; ++c) {
    const uint4 u = *reinterpret_cast<const uint4 *>(img + canon(r, 8 * c));
    const uint32_t w[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
    for (int j = 0; j < 4; ++j) s += bf16_val((uint16_t)(w[j] & 0xFFFFu)) + bf16_val((uint16_t)(w[j] >> 16));
  }
  return s;
}

__global__ void __launch_bounds__(kTileRows, 1) k_gradients(DeviceModel md, const float *__restrict__ x,
                                                            const float *__restrict__ yt,
                                                            const int32_t *__restrict__ perm, int64_t n,
                                                            float inv_count) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  TrainSmem &S = *reinterpret_cast<TrainSmem *>(smem_raw);
  const int t = threadIdx.x, warp = t >> 5;
  const int64_t g = blockIdx.x;
  const int64_t row = g * kTileRows + t;
  const bool valid = row < n;
  const int64_t idx = valid ? (perm ? (int64_t)perm[row] : row) : 0;
  float *part = md.partial + g * kPartStride;
  const Norm nm = md.norm;

  copy_img(S.W, md.img);  // W2
  for (int i = t; i < kHid * kIn; i += kTileRows) S.W1[i] = md.wq[kOffW1 + i];
  for (int i = t; i < kOut * kHid; i += kTileRows) S.W4[i] = md.wq[kOffW4 + i];
  S.b1[t] = md.w[kOffB1 + t];
  S.b2[t] = md.w[kOffB2 + t];
  S.b3[t] = md.w[kOffB3 + t];
  if (t < kOut) S.b4[t] = md.w[kOffB4 + t];
  const uint32_t mbar = saddr(&S.mbar);
  if (t == 0) {
    mbar_init(mbar);
    S.flag = 0;
  }
  if (warp == 0) tmem_alloc(saddr(&S.tmem_slot), 512);
  float f[4] = {0.f, 0.f, 0.f, 0.f};
  if (valid) features(nm, x + 4 * idx, f);
  for (int k = 0; k < 4; ++k) S.f[t][k] = f[k];
  __syncthreads();  // W1, b1 staged
  // layer 1 -> X0 (row t) and XT1 (column t)
  for (int c = 0; c < 16; ++c) {
    uint32_t q[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int o = 8 * c + 2 * j;
      const float a0 = valid ? silu(layer1(S.W1, S.b1, f, o)) : 0.f;
      const float a1 = valid ? silu(layer1(S.W1, S.b1, f, o + 1)) : 0.f;
      q[j] = bf16_bits(a0) | (bf16_bits(a1) << 16);
    }
    put_row8(S.X0, t, 8 * c, q);
    put_col8(S.XT1, 8 * c, t, q);
  }
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = S.tmem_slot;
  const uint32_t T0 = tmem, T1 = tmem + 128, T2 = tmem + 256, T3 = tmem + 384;
  const uint32_t lane = (uint32_t)(warp * 32) << 16;
  uint32_t phase = 0;
  bool ok = true;
  do {
    // ---- forward: z2 = a1 W2^T -> T0
    if (t == 0) {
      mma_128(T0, saddr(S.X0), saddr(S.W), false);
      mma_commit(mbar);
    }
    if (!(ok = wait_mma(mbar, phase, &S.flag, md.error))) break;
    phase ^= 1;
    tc_fence_after();
    copy_img(S.W, md.img + kImgElems);  // W3
    for (int c = 0; c < 8; ++c) {
      float v[16];
      tmem_ld16(T0 + lane + 16 * c, v);
      uint32_t q[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const int o = 16 * c + 2 * j;
        const float a0 = valid ? silu(v[2 * j] + S.b2[o]) : 0.f;
        const float a1 = valid ? silu(v[2 * j + 1] + S.b2[o + 1]) : 0.f;
        q[j] = bf16_bits(a0) | (bf16_bits(a1) << 16);
      }
      put_row8(S.X0, t, 16 * c, q);
      put_row8(S.X0, t, 16 * c + 8, q + 4);
      put_col8(S.XT2, 16 * c, t, q);
      put_col8(S.XT2, 16 * c + 8, t, q + 4);
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    // ---- forward: z3 = a2 W3^T -> T1
    if (t == 0) {
      tc_fence_after();
      mma_128(T1, saddr(S.X0), saddr(S.W), false);
      mma_commit(mbar);
    }
    if (!(ok = wait_mma(mbar, phase, &S.flag, md.error))) break;
    phase ^= 1;
    tc_fence_after();
    // ---- output layer, loss, dy; a3 kept (plain row-major) in X0
    float acc[3] = {S.b4[0], S.b4[1], S.b4[2]};
    for (int c = 0; c < 8; ++c) {
      float v[16];
      tmem_ld16(T1 + lane + 16 * c, v);
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const int o = 16 * c + j;
        const float a = bf16_round(silu(v[j] + S.b3[o]));
        S.X0[t * kHid + o] = (uint16_t)bf16_bits(a);
        acc[0] += S.W4[o] * a;
        acc[1] += S.W4[kHid + o] * a;
        acc[2] += S.W4[2 * kHid + o] * a;
      }
    }
    float dy[3], l = 0.f;
    for (int j = 0; j < 3; ++j) {
      const float d = valid ? acc[j] - (yt[3 * idx + j] - nm.out_shift[j]) / nm.out_scale[j] : 0.f;
      l += d * d;
      dy[j] = 2.0f * d * inv_count;
      S.dy[t][j] = dy[j];
    }
    for (int off = 16; off > 0; off >>= 1) l += __shfl_xor_sync(0xffffffffu, l, off);
    if ((t & 31) == 0) S.red[warp] = l;
    // dz3 = bf16(dy W4 * silu'(z3)) -> D0 (row t), DT (column t)
    for (int c = 0; c < 8; ++c) {
      float v[16];
      tmem_ld16(T1 + lane + 16 * c, v);
      uint32_t q[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        float dz[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int o = 16 * c + 2 * j + h;
          const float da = dy[0] * S.W4[o] + dy[1] * S.W4[kHid + o] + dy[2] * S.W4[2 * kHid + o];
          dz[h] = valid ? da * dsilu(v[2 * j + h] + S.b3[o]) : 0.f;
        }
        q[j] = bf16_bits(dz[0]) | (bf16_bits(dz[1]) << 16);
      }
      put_row8(S.D0, t, 16 * c, q);
      put_row8(S.D0, t, 16 * c + 8, q + 4);
      put_col8(S.DT, 16 * c, t, q);
      put_col8(S.DT, 16 * c + 8, t, q + 4);
    }
    copy_img(S.W, md.img + 3 * kImgElems);  // W3^T
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    // ---- dW3 = dz3^T a2 -> T2 ; da2 = dz3 W3 -> T3
    if (t == 0) {
      tc_fence_after();
      mma_128(T2, saddr(S.DT), saddr(S.XT2), false);
      mma_128(T3, saddr(S.D0), saddr(S.W), false);
      mma_commit(mbar);
      md.loss_part[g] = (S.red[0] + S.red[1]) + (S.red[2] + S.red[3]);
    }
    // meanwhile: output-layer gradients and db3 from shared memory
    {
      float s0 = 0.f, s1 = 0.f, s2 = 0.f;
      for (int b = 0; b < kTileRows; ++b) {
        const float a = bf16_val(S.X0[b * kHid + t]);
        s0 += S.dy[b][0] * a;
        s1 += S.dy[b][1] * a;
        s2 += S.dy[b][2] * a;
      }
      part[kOffW4 + t] = s0;
      part[kOffW4 + kHid + t] = s1;
      part[kOffW4 + 2 * kHid + t] = s2;
      if (t < kOut) {
        float s = 0.f;
        for (int b = 0; b < kTileRows; ++b) s += S.dy[b][t];
        part[kOffB4 + t] = s;
      }
      part[kOffB3 + t] = sum_row_T(S.DT, t);
    }
    if (!(ok = wait_mma(mbar, phase, &S.flag, md.error))) break;
    phase ^= 1;
    tc_fence_after();
    for (int c = 0; c < 8; ++c) {  // dW3 row t
      float v[16];
      tmem_ld16(T2 + lane + 16 * c, v);
      float4 *dst = reinterpret_cast<float4 *>(part + kOffW3 + t * kHid + 16 * c);
      for (int j = 0; j < 4; ++j) dst[j] = make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]);
    }
    // dz2 = bf16(da2 * silu'(z2)) -> D0, DT
    for (int c = 0; c < 8; ++c) {
      float da[16], z[16];
      tmem_ld16(T3 + lane + 16 * c, da);
      tmem_ld16(T0 + lane + 16 * c, z);
      uint32_t q[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const int o = 16 * c + 2 * j;
        const float d0 = valid ? da[2 * j] * dsilu(z[2 * j] + S.b2[o]) : 0.f;
        const float d1 = valid ? da[2 * j + 1] * dsilu(z[2 * j + 1] + S.b2[o + 1]) : 0.f;
        q[j] = bf16_bits(d0) | (bf16_bits(d1) << 16);
      }
      put_row8(S.D0, t, 16 * c, q);
      put_row8(S.D0, t, 16 * c + 8, q + 4);
      put_col8(S.DT, 16 * c, t, q);
      put_col8(S.DT, 16 * c + 8, t, q + 4);
    }
    copy_img(S.W, md.img + 2 * kImgElems);  // W2^T
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    // ---- dW2 = dz2^T a1 -> T2 ; da1 = dz2 W2 -> T3
    if (t == 0) {
      tc_fence_after();
      mma_128(T2, saddr(S.DT), saddr(S.XT1), false);
      mma_128(T3, saddr(S.D0), saddr(S.W), false);
      mma_commit(mbar);
    }
    part[kOffB2 + t] = sum_row_T(S.DT, t);
    if (!(ok = wait_mma(mbar, phase, &S.flag, md.error))) break;
    phase ^= 1;
    tc_fence_after();
    for (int c = 0; c < 8; ++c) {  // dW2 row t
      float v[16];
      tmem_ld16(T2 + lane + 16 * c, v);
      float4 *dst = reinterpret_cast<float4 *>(part + kOffW2 + t * kHid + 16 * c);
      for (int j = 0; j < 4; ++j) dst[j] = make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]);
    }
    // dz1 = da1 * silu'(z1) in FP32 -> scratch [row][out]
    float *scr = reinterpret_cast<float *>(S.X0);
    for (int c = 0; c < 8; ++c) {
      float v[16];
      tmem_ld16(T3 + lane + 16 * c, v);
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const int o = 16 * c + j;
        scr[t * kHid + o] = valid ? v[j] * dsilu(layer1(S.W1, S.b1, f, o)) : 0.f;
      }
    }
    __syncthreads();
    {
      float s[4] = {0.f, 0.f, 0.f, 0.f}, sb = 0.f;
      for (int b = 0; b < kTileRows; ++b) {
        const float d = scr[b * kHid + t];
        sb += d;
        for (int k = 0; k < 4; ++k) s[k] += d * S.f[b][k];
      }
      for (int k = 0; k < 4; ++k) part[kOffW1 + 4 * t + k] = s[k];
      part[kOffB1 + t] = sb;
    }
  } while (false);
  if (!ok && t == 0) mbar_wait(mbar, phase);  // let an MMA still in flight drain (bounded)
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) tmem_free(tmem, 512);
}

}  // namespace

void launch_publish(const DeviceModel &md, cudaStream_t st) {
  k_publish<<<(kParams + 255) / 256, 256, 0, st>>>(md);
}

void launch_forward(const DeviceModel &md, const float *x, float *y, int64_t n, int num_sms, cudaStream_t st) {
  if (n <= 0) return;
  const int smem = (int)sizeof(FwdSmem);
  cudaFuncSetAttribute(k_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  const int64_t ntiles = (n + kTileRows - 1) / kTileRows;
  const int grid = (int)std::min<int64_t>(ntiles, 2 * (int64_t)num_sms);
  k_forward<<<grid, kTileRows, smem, st>>>(md, x, y, n);
}

void launch_gradients(const DeviceModel &md, const float *x, const float *y_true, const int32_t *perm, int64_t n,
                      cudaStream_t st) {
  if (n <= 0 || n > kMaxTrainRows) return;
  const int smem = (int)sizeof(TrainSmem);
  cudaFuncSetAttribute(k_gradients, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  const int ntiles = (int)((n + kTileRows - 1) / kTileRows);
  k_gradients<<<ntiles, kTileRows, smem, st>>>(md, x, y_true, perm, n, 1.0f / (3.0f * (float)n));
}

void launch_reduce_adam(const DeviceModel &md, int ntiles, float lr, float beta1, float beta2, float eps, float bc1,
                        float bc2, float *grad, cudaStream_t st) {
  k_reduce_adam<<<(kParams + 255) / 256, 256, 0, st>>>(md, ntiles, lr, beta1, beta2, eps, bc1, bc2, grad);
}

}  // namespace mlp
}  // namespace aak
