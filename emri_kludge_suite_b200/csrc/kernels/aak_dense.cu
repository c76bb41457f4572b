// aak_dense.cu -- sm_100a kernels for the dense part of the AAK waveform:
// spline interpolation of the coarse (e, v, M, S) trajectory, the
// Adams-Bashforth-2 phase accumulation (gamma~, Phi, alpha) as a single-pass
// tiled scan, and the Peters-Mathews harmonic sum with the LISA h_I/h_II
// response and the Planck taper.  Reference semantics: src/suite/AAK.cc:213-547.
//
// k_waveform<precision>: persistent CTAs pull 1024-sample tiles from a work
//   queue; per tile, phase 1 evaluates the spline and the rates and scans the
//   AB2 increments inside the tile, a decoupled look-back over the tile's
//   phase chain (per-tile records in double-double arithmetic) supplies the
//   carry from the earlier tiles of the source, and phase 2 evaluates the
//   harmonic sums (FP64, or split precision); h_I, h_II are written with
//   coalesced stores.
#include <cuda_runtime.h>
#include <math.h>

#include <atomic>
#include <type_traits>
#include <utility>

#include "aak_dense.cuh"

namespace aak {
namespace {

constexpr double kTwoPi = 2.0 * kPi;
constexpr double kHalfSqrt3 = 0.86602540378443864676;

// Resident CTAs per SM requested for the waveform kernel (register budget).
#ifndef AAK_WAVE_MIN_BLOCKS
#define AAK_WAVE_MIN_BLOCKS 2
#endif

// ------------------------------------------------------------------ small helpers
// x mod 2pi in [-pi, pi], two-term Cody-Waite reduction in FP64
__device__ __forceinline__ double reduce_2pi_d(double x) {
  const double k = rint(x * (1.0 / kTwoPi));
  return fma(-k, 2.4492935982947064e-16, fma(-k, 6.283185307179586, x));
}
// the same, returned as float
__device__ __forceinline__ float reduce_2pi_f(double x) { return (float)reduce_2pi_d(x); }

__device__ __forceinline__ int find_source(const int64_t *tile_start, int nsrc, int64_t g) {
  int lo = 0, hi = nsrc;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (tile_start[mid] <= g) lo = mid;
    else hi = mid;
  }
  return lo;
}

struct Traj4 {
  double e, v, M, S;
};

// Coefficients b, d of the natural-spline piece y0 + dx (b + dx (c0 + dx d))
// on [x0, x0 + h] (the GSL cspline form, KSParMap.cc:487-498), from the
// piece's reciprocal length rh = 1 / h and rh3 = rh / 3: one division per
// piece instead of three per component.  Against the divided form the
// coefficients differ by an ulp or two; the pre-pass and the waveform kernel
// both evaluate the spline through here, so their values stay equal.
__device__ __forceinline__ void piece_bd(double y0, double y1, double c0, double c1, double h, double rh, double rh3,
                                         double &b, double &d) {
  b = (y1 - y0) * rh - h * (c1 + 2.0 * c0) * (1.0 / 3.0);
  d = (c1 - c0) * rh3;
}
__device__ __forceinline__ double piece(double y0, double y1, double c0, double c1, double h, double rh, double rh3,
                                        double dx) {
  double b, d;
  piece_bd(y0, y1, c0, c1, h, rh, rh3, b, d);
  return y0 + dx * (b + dx * (c0 + dx * d));
}

// ------------------------------------------------------------------ knot windows
// The knots a tile needs are a short contiguous run; each CTA brackets it once
// and stages it in shared memory, so per-sample lookups search a handful of
// shared-memory entries instead of walking the whole knot array in global
// memory.  Runs longer than kWin (sources whose coarse grid is finer than the
// sample spacing) are searched in global memory within the bracket.
constexpr int kWin = 64;

struct KnotWin {
  double *t;   // kWin
  double4 *y;  // kWin: values at the knots
  double4 *c;  // kWin: half second derivatives
  double4 *b;  // kWin: first-order coefficients of the pieces (staged windows)
  double4 *d;  // kWin: third-order coefficients of the pieces (staged windows)
  int k0;        // first knot of the window (source-relative)
  int n;         // knots in the window
  int staged;    // 1: window is in shared memory
  double inv_h;  // (n - 1) / (t_{n-1} - t_0): pieces per unit time
};

__device__ __forceinline__ Traj4 eval_piece(const double4 &y0, const double4 &y1, const double4 &c0, const double4 &c1,
                                            double x0, double x1, double t) {
  const double h = x1 - x0, dx = t - x0, rh = 1.0 / h, rh3 = rh * (1.0 / 3.0);
  Traj4 q;
  q.e = piece(y0.x, y1.x, c0.x, c1.x, h, rh, rh3, dx);
  q.v = piece(y0.y, y1.y, c0.y, c1.y, h, rh, rh3, dx);
  q.M = piece(y0.z, y1.z, c0.z, c1.z, h, rh, rh3, dx);
  q.S = piece(y0.w, y1.w, c0.w, c1.w, h, rh, rh3, dx);
  return q;
}

__device__ __forceinline__ Traj4 spline4w(const BatchView &bv, const SourceDesc &d, double t, const KnotWin &w) {
  if (w.staged) {
    // the knots are (nearly) evenly spaced: guess the piece, then step to the
    // largest k <= n - 2 with t_k <= t (the binary search's answer)
    int k = __double2int_rd((t - w.t[0]) * w.inv_h);
    k = min(max(k, 0), w.n - 2);
    while (k < w.n - 2 && w.t[k + 1] <= t) ++k;
    while (k > 0 && w.t[k] > t) --k;
    const double dx = t - w.t[k];
    const double4 y = w.y[k], b = w.b[k], c = w.c[k], dd = w.d[k];
    Traj4 q;
    q.e = y.x + dx * (b.x + dx * (c.x + dx * dd.x));
    q.v = y.y + dx * (b.y + dx * (c.y + dx * dd.y));
    q.M = y.z + dx * (b.z + dx * (c.z + dx * dd.z));
    q.S = y.w + dx * (b.w + dx * (c.w + dx * dd.w));
    return q;
  }
  // long windows stay in global memory: the same guess-and-step search there
  const double *kt = bv.knot_t + d.knot_offset;
  const int last = w.k0 + w.n - 2;
  int k = w.k0 + __double2int_rd((t - kt[w.k0]) * w.inv_h);
  k = min(max(k, w.k0), last);
  while (k < last && kt[k + 1] <= t) ++k;
  while (k > w.k0 && kt[k] > t) --k;
  const int64_t o = d.knot_offset + k;
  return eval_piece(bv.knot_y[o], bv.knot_y[o + 1], bv.knot_c[o], bv.knot_c[o + 1], kt[k], kt[k + 1], t);
}

// Knots per unit time of the window and, for a staged window, the piece
// coefficients (the knots are in shared memory and visible to every thread).
__device__ __forceinline__ void finish_window(const BatchView &bv, const SourceDesc &d, KnotWin &w) {
  if (!w.staged) {
    const double *kt = bv.knot_t + d.knot_offset;
    const double span = kt[w.k0 + w.n - 1] - kt[w.k0];
    w.inv_h = (span > 0.0) ? (double)(w.n - 1) / span : 0.0;
  } else {
    const double span = w.t[w.n - 1] - w.t[0];
    w.inv_h = (span > 0.0) ? (double)(w.n - 1) / span : 0.0;
    // piece coefficients y + dx (b + dx (c + dx d)) of the natural spline, once per window
    for (int k = threadIdx.x; k < w.n - 1; k += blockDim.x) {
      const double h = w.t[k + 1] - w.t[k], rh = 1.0 / h, rh3 = rh * (1.0 / 3.0);
      const double4 y0 = w.y[k], y1 = w.y[k + 1], c0 = w.c[k], c1 = w.c[k + 1];
      double4 b, d;
      piece_bd(y0.x, y1.x, c0.x, c1.x, h, rh, rh3, b.x, d.x);
      piece_bd(y0.y, y1.y, c0.y, c1.y, h, rh, rh3, b.y, d.y);
      piece_bd(y0.z, y1.z, c0.z, c1.z, h, rh, rh3, b.z, d.z);
      piece_bd(y0.w, y1.w, c0.w, c1.w, h, rh, rh3, b.w, d.w);
      w.b[k] = b;
      w.d[k] = d;
    }
    __syncthreads();
  }
}

// Stage the knots of tile g (bracket precomputed on the host, tile_knot).
__device__ __forceinline__ void load_window(const BatchView &bv, const SourceDesc &d, int64_t g, KnotWin &w) {
  w.k0 = bv.tile_knot[2 * g];
  w.n = bv.tile_knot[2 * g + 1];
  w.staged = w.n <= kWin;
  if (w.staged)
    for (int k = threadIdx.x; k < w.n; k += blockDim.x) {
      const int64_t o = d.knot_offset + w.k0 + k;
      w.t[k] = bv.knot_t[o];
      w.y[k] = bv.knot_y[o];
      w.c[k] = bv.knot_c[o];
    }
  __syncthreads();
  finish_window(bv, d, w);
}

// gamma~dot, Phidot, alphadot (AAK.cc:251-253) with one division:
// d(x)/dm / dt/dm / M = 16 v^3 num_x / (num_t M) for the 3PN numerators of
// aak_common.hpp (KSParMap.cc:86-144).  Here they are regrouped, exactly, as
// polynomials in x = v^2, w = q v, wy = w Y and E = e^2 (Y = cos iota is the
// source's; every coefficient below is an integer, so the regrouping holds
// term for term), and the rates are formed from
//   T = num_t,  A = num_theta - num_r,  B = num_r,  C = num_phi - num_theta,
// so that the differences are evaluated without cancellation: gamma~dot = A,
// Phidot = B, alphadot = C (times 16 v^3 / (T M)).  om (optional) receives
// Omega_phi, the ratio for phi with (Y, q) on prograde orbits and (-Y, -q) on
// retrograde ones (AAK.cc:15-23): num_phi(Y, q) = A + B + C and num_phi(-Y,
// -q) = A + B - C (the t numerator is even in (Y, q)).  Against the
// reference's evaluation order the rates differ by rounding only.
__device__ __forceinline__ void phase_rates(const SourceDesc &d, const Traj4 &q, double r[3], double *om = nullptr) {
  const double Y = d.coslam;
  const double E = q.e * q.e, x = q.v * q.v, w = q.S * q.v, wy = w * Y, w2 = w * w, wy2 = wy * wy;
  // T: coefficients of x^k w^a wy^b as cubics in E
  const double c00 = fma(fma(fma(560., E, 480.), E, 384.), E, 256.);
  const double c20 = fma(fma(fma(-360., E, -240.), E, -64.), E, 384.);
  const double t31 = E * fma(fma(960., E, 768.), E, 512.);
  const double t42a = fma(fma(fma(400., E, 336.), E, 256.), E, 128.);
  const double t42b = fma(fma(fma(-880., E, -720.), E, -512.), E, -128.);
  const double c40 = fma(fma(fma(-2742., E, -2268.), E, -1584.), E, 864.);
  const double t51 = fma(fma(fma(8816., E, 7392.), E, 5504.), E, -768.);
  const double t62a = fma(fma(fma(4800., E, 3992.), E, 3008.), E, -64.);
  const double t62b = fma(fma(fma(-15096., E, -12616.), E, -9600.), E, 192.);
  const double c60 = fma(fma(fma(-15565., E, -13134.), E, -9864.), E, 2160.);
  const double T4 = fma(x, c60, fma(wy2, t62b, fma(w2, t62a, fma(wy, t51, c40))));
  const double T2 = fma(x, T4, fma(wy2, t42b, fma(w2, t42a, fma(wy, t31, c20))));
  const double T = fma(x, T2, c00);
  // A = num_theta - num_r
  const double A6 = fma(fma(24., E, 270.), E, 486.);
  const double A4 = fma(x, A6, fma(-fma(90., E, 186.), w2, fma(fma(258., E, 522.), wy2,
                                                               fma(-fma(144., E, 384.), wy, fma(36., E, 144.)))));
  const double A = x * fma(x, A4, fma(-12., w2, fma(60., wy2, fma(-96., wy, 48.))));
  // B = num_r
  const double B6 = fma(fma(fma(5., E, 21.), E, -135.), E, -351.);
  const double B4 = fma(x, B6, fma(fma(fma(2., E, 14.), E, 132.), w2,
                                   fma(fma(fma(26., E, -78.), E, -408.), wy2,
                                       fma(fma(fma(-24., E, 32.), E, 264.), wy, fma(6., E * E, -90.)))));
  const double B2 = fma(x, B4, fma(fma(4., E, 8.), w2, fma(fma(4., E, -32.), wy2, fma(fma(-16., E, 48.), wy, fma(8., E, -24.)))));
  const double B = fma(x, B2, 16.);
  // C = num_phi - num_theta
  const double C = (x * w) * fma(x, fma(-fma(140., E, 36.), wy, fma(64., E, 48.)), fma(-24., wy, 32.));
  const double inv = 16. * (x * q.v) / (T * q.M);
  r[0] = A * inv;
  r[1] = B * inv;
  r[2] = C * inv;
  if (om) *om = ((Y > 0) ? (A + B) + C : (A + B) - C) * inv;
}

// h_I, h_II of one sample: FP64 outputs, or FP32 ones (rows of an FP32 FFT)
__device__ __forceinline__ void store_h(const BatchView &bv, int64_t o, double hI, double hII) {
  if (bv.hI_f32) {
    bv.hI_f32[o] = (float)hI;
    bv.hII_f32[o] = (float)hII;
  } else {
    bv.hI[o] = hI;
    bv.hII[o] = hII;
  }
}

__device__ __forceinline__ double sample_time(const SourceDesc &d, int i) {
  return (i == 0) ? d.t_first : (double)(i - d.i0) * d.dt;
}

// samples whose phases feed the output (the rest are zero after the taper)
__device__ __forceinline__ int n_eff(const SourceDesc &d) {
  const long long e = (long long)d.i_plunge + (long long)d.i_buffer;
  return (int)min((long long)d.vlength, e);
}

// error-free transformation for double-double accumulation
__device__ __forceinline__ void two_sum(double a, double b, double &s, double &err) {
  s = a + b;
  const double bb = s - a;
  err = (a - (s - bb)) + (b - bb);
}
__device__ __forceinline__ void dd_add(double &hi, double &lo, double x) {
  double s, e;
  two_sum(hi, x, s, e);
  e += lo;
  hi = s + e;
  lo = e - (hi - s);
}

// Warp-wide scan of three values: in[] becomes the inclusive prefix, ex[] the exclusive one.
__device__ __forceinline__ void warp_scan3(double in[3], double ex[3]) {
  const int l = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      const double n = __shfl_up_sync(0xffffffffu, in[q], o);
      if (l >= o) in[q] += n;
    }
  }
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    const double e = __shfl_up_sync(0xffffffffu, in[q], 1);
    ex[q] = (l == 0) ? 0.0 : e;
  }
}

// Block-wide exclusive scans of three values, the forward ones and (both, a
// block-uniform flag) the backward ones, with one barrier for the two: each
// warp's totals go to red[direction], and every thread adds the totals of the
// warps before it; every thread also gets the block totals.  The barrier also
// orders every shared-memory read before the call before any write after it.
__device__ __forceinline__ void block_exscan3x2(const double vf[3], const double vb[3], bool both,
                                                double (*red)[3][kTileThreads / 32], double exf[3], double totf[3],
                                                double exb[3], double totb[3]) {
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  double inf[3] = {vf[0], vf[1], vf[2]}, inb[3] = {vb[0], vb[1], vb[2]};
  warp_scan3(inf, exf);
  if (both) warp_scan3(inb, exb);
  if (l == 31) {
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      red[0][q][w] = inf[q];
      if (both) red[1][q][w] = inb[q];
    }
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    double pre = 0.0, t = 0.0;
#pragma unroll
    for (int k = 0; k < kTileThreads / 32; ++k) {
      const double r = red[0][q][k];
      if (k < w) pre += r;
      t += r;
    }
    exf[q] += pre;
    totf[q] = t;
  }
  if (both) {
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      double pre = 0.0, t = 0.0;
#pragma unroll
      for (int k = 0; k < kTileThreads / 32; ++k) {
        const double r = red[1][q][k];
        if (k < w) pre += r;
        t += r;
      }
      exb[q] += pre;
      totb[q] = t;
    }
  }
}

// ------------------------------------------------------------------ tile geometry
struct TileCtx {
  int s;        // source
  int start;    // first sample of the tile
  int end;      // one past the last sample of the tile
  int neff;     // samples feeding the output
  int lt;       // tile index inside the source
  int head;     // tile holding sample i0 (t = 0): head of both phase chains
  int64_t g;    // global tile index (records, knot windows)
};

// Queue item j -> tile.  Without a queue array (one-source views, the
// allocation-free launch) the queue runs source by source, and inside a
// source from the head tile through the later tiles in increasing order,
// then through the earlier tiles in decreasing order, so that every tile
// comes after its predecessor in its phase chain (the tile next to it,
// towards the head).  A queue array (batches) lists the same per-source
// orders interleaved across sources.
__device__ __forceinline__ TileCtx tile_ctx(const BatchView &bv, int64_t j, const SourceDesc *&dp) {
  TileCtx c;
  int T;
  if (bv.queue) {
    const QueueItem &q = bv.queue[j];
    c.s = q.s;
    c.lt = q.lt;
    c.g = q.g;
    dp = bv.src + c.s;
    T = dp->n_tiles;
    const int i0 = dp->i0;
    c.head = (i0 <= 0) ? 0 : min(i0 / kTileSamples, T - 1);
  } else {
    c.s = find_source(bv.tile_start, bv.nsrc, j);
    dp = bv.src + c.s;
    const int64_t t0 = bv.tile_start[c.s];
    T = (int)(bv.tile_start[c.s + 1] - t0);
    const int i0 = dp->i0;
    c.head = (i0 <= 0) ? 0 : min(i0 / kTileSamples, T - 1);
    const int jj = (int)(j - t0);
    c.lt = (jj < T - c.head) ? c.head + jj : T - 1 - jj;
    c.g = t0 + c.lt;
  }
  c.start = c.lt * kTileSamples;
  c.end = min(c.start + kTileSamples, dp->vlength);
  c.neff = n_eff(*dp);
  return c;
}

// ------------------------------------------------------------------ look-back
// Bounded waits: a wait gives up after bv.lookback_cycles SM clocks (default
// kLookBackCycles, about 2 s), or at once when another wait of the launch
// already gave up, sets *device_status and returns a zero carry.
constexpr long long kLookBackCycles = 4000000000LL;

__device__ __forceinline__ int ld_acquire(const int32_t *p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(int32_t *p, int v) {
  asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// double-double sum (hi, lo) += (bh, bl)
__device__ __forceinline__ void dd_add_dd(double &hi, double &lo, double bh, double bl) {
  double s, e;
  two_sum(hi, bh, s, e);
  e += lo + bl;
  hi = s + e;
  lo = e - (hi - s);
}

// Publish tile g's aggregate or inclusive record (one thread): the fields go
// to L2 (st.cg), then the flag's st.release.gpu orders them before it (a reader
// loads the flag with ld.acquire.gpu before the fields), so no separate fence.
__device__ __forceinline__ void publish_aggregate(const BatchView &bv, int64_t g, const double x[3], double C, bool hasC) {
  TileLink *L = bv.link + g;
#pragma unroll
  for (int q = 0; q < 3; ++q) __stcg(&L->agg[q], x[q]);
  __stcg(&L->agg_C, C);
  __stcg(&L->agg_hasC, hasC ? 1 : 0);
  st_release(bv.link_flag + g, 1);
}
__device__ __forceinline__ void publish_inclusive(const BatchView &bv, int64_t g, const double fh[3], const double fl[3],
                                                  const double bh[3], const double bl[3], double C) {
  TileLink *L = bv.link + g;
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    __stcg(&L->inc_f_hi[q], fh[q]);
    __stcg(&L->inc_f_lo[q], fl[q]);
    __stcg(&L->inc_b_hi[q], bh[q]);
    __stcg(&L->inc_b_lo[q], bl[q]);
  }
  __stcg(&L->inc_C, C);
  st_release(bv.link_flag + g, 2);
}

// This tile's aggregate, published by the look-back only when it has to wait.
struct TileAgg {
  double x[3];  // the tile's own sums of the chain's direction
  double C;     // the clamped Phidot of its last forward output sample
  bool hasC;
  bool publish;  // false: nothing to publish (the tile looks back before its phases are known)
};

// Exclusive prefix of tile c.lt along its chain (dir +1: forward, -1:
// backward), computed by one whole warp.  Each round looks at the 32 nearest
// predecessors not yet summed (lane k: k + 1 tiles further towards the head),
// waits until every one of them nearer than the first inclusive record (or
// than the head tile) is written, and sums their aggregates and that
// inclusive record in double-double.  C (forward chains): the clamped Phidot
// of the nearest record that sets one, else 0.  Every lane returns the sums.
// agg: the tile's aggregate, published before the first wait or
// second round, and not at all when the first round finds the prefix ready
// (the tile's inclusive record follows at once): successors never wait on a
// tile that waits itself without its aggregate out.
__device__ void look_back_warp(const BatchView &bv, const TileCtx &c, int dir, double hi[3], double lo[3], double &C,
                               TileAgg agg = TileAgg{{0.0, 0.0, 0.0}, 0.0, false, false}) {
  const unsigned kAll = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const int64_t t0 = c.g - c.lt;
  const long long bound = (bv.lookback_cycles > 0) ? bv.lookback_cycles : kLookBackCycles;
  const long long start = clock64();
  bool haveC = false, published = !agg.publish;
  C = 0.0;
#pragma unroll
  for (int q = 0; q < 3; ++q) hi[q] = lo[q] = 0.0;
  for (int p = c.lt - dir;; p -= 32 * dir) {
    const int q = p - dir * lane;
    const bool valid = (dir > 0) ? (q >= c.head) : (q <= c.head);
    int f = 0;
    unsigned stop_mask, need;
    for (;;) {
      f = valid ? ld_acquire(bv.link_flag + t0 + q) : 0;
      stop_mask = __ballot_sync(kAll, valid && (f == 2 || (f == 1 && q == c.head)));
      const unsigned vmask = __ballot_sync(kAll, valid);
      const unsigned ready = __ballot_sync(kAll, valid && f != 0);
      need = stop_mask ? ((stop_mask & (0u - stop_mask)) << 1) - 1u : vmask;  // lanes up to the first stop
      const bool done = (ready & need) == need;
      if (!published && !(done && stop_mask)) {  // a wait or a further round follows
        if (lane == 0) publish_aggregate(bv, c.g, agg.x, agg.C, agg.hasC);
        published = true;
      }
      if (done) break;
      int give_up = 0;
      if (lane == 0)
        give_up = (*(volatile unsigned int *)bv.device_status != 0u || clock64() - start > bound) ? 1 : 0;
      if (__shfl_sync(kAll, give_up, 0)) {
        if (lane == 0) {
          atomicExch(bv.device_status, 1u);
          if (bv.status_report) atomicExch(bv.status_report, 1u);
        }
#pragma unroll
        for (int k = 0; k < 3; ++k) hi[k] = lo[k] = 0.0;
        C = 0.0;
        return;
      }
      __nanosleep(32);
    }
    const bool use = (need >> lane) & 1u;
    const bool is_stop = stop_mask != 0u && lane == __ffs(stop_mask) - 1;
    double xh[3] = {0.0, 0.0, 0.0}, xl[3] = {0.0, 0.0, 0.0}, cv = 0.0;
    bool hasc = false;
    if (use) {
      const TileLink *L = bv.link + t0 + q;
      if (is_stop && f == 2) {
        const double *ph = (dir > 0) ? L->inc_f_hi : L->inc_b_hi, *pl = (dir > 0) ? L->inc_f_lo : L->inc_b_lo;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          xh[k] = __ldcg(ph + k);
          xl[k] = __ldcg(pl + k);
        }
        cv = __ldcg(&L->inc_C);
        hasc = true;
      } else {  // an aggregate (the head's too, when it holds only one)
#pragma unroll
        for (int k = 0; k < 3; ++k) xh[k] = __ldcg(&L->agg[k]);
        cv = __ldcg(&L->agg_C);
        hasc = __ldcg(&L->agg_hasC) != 0;
      }
    }
    if (dir > 0 && !haveC) {
      const unsigned cm = __ballot_sync(kAll, use && hasc);
      if (cm) {
        C = __shfl_sync(kAll, cv, __ffs(cm) - 1);
        haveC = true;
      }
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const double bh = __shfl_xor_sync(kAll, xh[k], o), bl = __shfl_xor_sync(kAll, xl[k], o);
        dd_add_dd(xh[k], xl[k], bh, bl);
      }
      dd_add_dd(hi[k], lo[k], xh[k], xl[k]);
    }
    if (stop_mask) return;
  }
}

// ------------------------------------------------------------------ bulk copies into shared memory
// One-dimensional TMA bulk copies (cp.async.bulk, global -> this CTA's
// shared memory; no multicast: the source is this GPU's own memory) that
// complete on an mbarrier with a byte count.  Addresses 16-byte aligned,
// sizes multiples of 16.  Every wait is bounded.
__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// order this thread's earlier generic-proxy accesses of shared memory before
// later async-proxy (bulk copy) writes to it
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_copy_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
               ::"r"(smem_addr(dst)), "l"(src), "r"(bytes), "r"(smem_addr(bar))
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(done)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return done != 0;
}
// Wait for phase `parity` of the barrier: at most 2^25 polls (seconds), false if it did not complete.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity) {
  for (int it = 0; it < (1 << 25); ++it) {
    if (mbar_try_wait(bar, parity)) return true;
    if (it >= 32) __nanosleep(64);
  }
  return false;
}

// Taylor-table term counts (defined with the harmonic sums); sources with
// more modes than kTabModes evaluate Bessel functions per sample
__device__ __forceinline__ int taylor_terms_fp64(double q, int nmodes);
__device__ __forceinline__ int taylor_terms_fp32(double q, int nmodes);

// ------------------------------------------------------------------ Bessel functions
// J_{lo..lo+4}(x) for x > 0 (lo = n-2 for n >= 2; lo = 0 for n = 1).
// x < 1: power series.  x >= 1: Miller's backward recurrence from the
// host-chosen start order, renormalised at J_lo, normalised by
// J_0 + 2 sum_k J_2k = 1.
__device__ __forceinline__ void bessel5_fp64(int lo, double x, int start, double J[5]) {
  if (x < 1.0) {
    const double hx = 0.5 * x, q = -hx * hx;
    double pref = exp((double)lo * log(hx) - lgamma((double)lo + 1.0));
#pragma unroll
    for (int m = 0; m < 5; ++m) {
      const double nu = (double)(lo + m);
      double term = 1.0, sum = 1.0;
#pragma unroll 1
      for (int k = 1; k < 14; ++k) {
        term *= q / ((double)k * (nu + (double)k));
        sum += term;
      }
      J[m] = pref * sum;
      pref *= hx / (nu + 1.0);
    }
    return;
  }
  const double tx = 2.0 / x;
  const int hi = lo + 4;
  double jk = 1.0e-300, jk1 = 0.0;  // J_k, J_{k+1} (unnormalised), k = start (even)
  double sum = 2.0 * jk, w = 0.0;   // w: weight 2 for even orders produced next
  int k = start;
  // phase 1: down to order hi + 1
#pragma unroll 2
  for (; k > hi + 1; --k) {
    const double jm = (double)k * tx * jk - jk1;
    jk1 = jk;
    jk = jm;
    sum = fma(w, jm, sum);
    w = 2.0 - w;
  }
  // phase 2: orders hi .. lo
  double v[5];
#pragma unroll
  for (int m = 4; m >= 0; --m) {
    const double jm = (double)k * tx * jk - jk1;
    jk1 = jk;
    jk = jm;
    sum = fma(w, jm, sum);
    w = 2.0 - w;
    v[m] = jm;
    --k;
  }
  // renormalise at J_lo to keep phase 3 in range
  const double sc = 1.0 / v[0];
  jk *= sc;
  jk1 *= sc;
  sum *= sc;
#pragma unroll
  for (int m = 0; m < 5; ++m) v[m] *= sc;
  // phase 3: orders lo-1 .. 0 (k == lo here)
#pragma unroll 2
  for (; k > 0; --k) {
    const double jm = (double)k * tx * jk - jk1;
    jk1 = jk;
    jk = jm;
    sum = fma(w, jm, sum);
    w = 2.0 - w;
  }
  // the last produced order is J_0, counted once (its weight was 2 or 0)
  if (w == 0.0) sum -= jk;       // J_0 was added with weight 2
  else sum += jk;                // J_0 was added with weight 0
  const double inv = 1.0 / sum;
#pragma unroll
  for (int m = 0; m < 5; ++m) J[m] = v[m] * inv;
}

// ------------------------------------------------------------------ per-tile Taylor table
// Within a 1024-sample tile the eccentricity moves by ~1e-4 at most.  The
// Peters-Mathews combinations of one harmonic,
//   A_n(e) = n [J_{n-2} - 2e J_{n-1} + (2/n) J_n + 2e J_{n+1} - J_{n+2}](n e),
//   B_n(e) = n [J_{n-2} - 2 J_n + J_{n+2}](n e),      C_n(e) = J_n(n e),
// are therefore tabulated per tile as Taylor polynomials in delta = e - e_c
// about the tile's central eccentricity e_c, so that a sample evaluates each
// with K fused multiply-adds.  The coefficients follow from
//   J_nu(n (e_c + delta)) = sum_k (n delta)^k / k! J_nu^(k)(n e_c),
//   J_nu^(k)(x) = 2^-k sum_j (-1)^j C(k, j) J_{nu-k+2j}(x)     (DLMF 10.6.7),
// with the J values of one row from a Miller backward recurrence (or the
// power series below x = 1), and the 2e factors of A_n expanded exactly.
// FP64 tables: row n holds [A_0 .. A_K | B_0 .. B_K | C_0 .. C_K].  FP32
// tables hold the harmonics in pairs (2p+1, 2p+2): pair row p is
// [A_0 B_0 .. A_K B_K of 2p+1 | the same of 2p+2 | C_0 of both, C_1 of both,
// .. C_K of both], so that a sample evaluates the A and B polynomials of one
// harmonic, and the C polynomials of the two harmonics of a pair, as packed
// FP32x2 Horner chains (__ffma2_rn, sm_100: each component rounds as fmaf,
// so the results are those of scalar chains with one instruction per step
// for two).  A pair row past an odd harmonic count holds zeros for the
// missing harmonic.
// (kTaylorMax64, kTaylorMax32, kRowD, kRowF: aak_dense.cuh)
// Stride of a tile with K terms, padded to 16 bytes: FP64, 3 (K + 1) doubles
// per harmonic; FP32, 6 (K + 1) floats per pair of harmonics.
template <typename T>
__host__ __device__ __forceinline__ int row_stride(int K) {
  const int per = 16 / (int)sizeof(T);
  const int vals = (sizeof(T) == 4) ? 6 * (K + 1) : 3 * (K + 1);
  return (vals + per - 1) / per * per;
}
// Harmonic rows a launch provides for `rows` harmonics: FP32 tables hold whole pairs.
template <typename T>
__host__ __device__ __forceinline__ int table_rows(int rows) {
  return (sizeof(T) == 4) ? (rows + 1) & ~1 : rows;
}

// J_m(x) for m = mlo .. mhi (x >= 0) into J[m - mlo]: Miller's backward
// recurrence from order max(start, mhi + 8), normalised by
// J_0 + 2 sum_k J_2k = 1 and rescaled on the way down whenever a value grows
// past 1e250.  Below x = 1e-3 the power series is used instead: there
// |x^2 / 4| <= 2.5e-7, so three terms leave a remainder below 1e-26.
__device__ void bessel_window(double x, int mlo, int mhi, int start, double *J) {
  if (x < 1.0e-3) {
    if (x <= 0.0) {
      for (int m = mlo; m <= mhi; ++m) J[m - mlo] = (m == 0) ? 1.0 : 0.0;
      return;
    }
    const double hx = 0.5 * x, q = -hx * hx;
    double pref = exp((double)mlo * log(hx) - lgamma((double)mlo + 1.0));
    for (int nu = mlo; nu <= mhi; ++nu) {
      double term = 1.0, sum = 1.0;
#pragma unroll
      for (int k = 1; k <= 3; ++k) {
        term *= q / ((double)k * ((double)nu + (double)k));
        sum += term;
      }
      J[nu - mlo] = pref * sum;
      pref *= hx / ((double)nu + 1.0);
    }
    return;
  }
  const double tx = 2.0 / x;
  int k = max(start, mhi + 8);
  if (k & 1) ++k;
  double jk = 1.0e-280, jk1 = 0.0, sum = 2.0 * jk, w = 0.0;
  for (; k > 0; --k) {
    const double jm = (double)k * tx * jk - jk1;  // order k - 1
    jk1 = jk;
    jk = jm;
    sum = fma(w, jm, sum);
    w = 2.0 - w;
    const int ord = k - 1;
    if (ord >= mlo && ord <= mhi) J[ord - mlo] = jm;
    if (fabs(jm) > 1.0e250) {  // rescale everything produced so far
      jk *= 1.0e-250;
      jk1 *= 1.0e-250;
      sum *= 1.0e-250;
      for (int o = max(ord, mlo); o <= mhi; ++o) J[o - mlo] *= 1.0e-250;
    }
  }
  sum -= jk;  // J_0 was added with weight 2; count it once
  const double inv = 1.0 / sum;
  for (int o = mlo; o <= mhi; ++o) J[o - mlo] *= inv;
}

// One table row (harmonic n, K + 1 terms), built by one thread in FP64.  The
// window holds J_m(n e_c) for m = n-2-K .. n+2+K (negative orders by
// J_{-m} = (-1)^m J_m); each derivative order comes from the previous one by
// J'_nu = (J_{nu-1} - J_{nu+1}) / 2 (DLMF 10.6.1) applied in place, which
// narrows the valid window by one order on each side and leaves orders
// n-2 .. n+2 at positions K .. K+4.
template <int K, typename T>
__device__ __forceinline__ void build_taylor_row_k(T *tab, int stride, int n, double ec, int start) {
  constexpr int W = 2 * K + 5;
  const int lo = n - 2 - K, mlo = max(0, lo);
  double Jw[W];
  bessel_window(n * ec, mlo, n + 2 + K, start, Jw + (mlo - lo));
  for (int m = lo; m < 0; ++m) Jw[m - lo] = ((-m) & 1) ? -Jw[-m - lo] : Jw[-m - lo];
  double D[W];
#pragma unroll
  for (int i = 0; i < W; ++i) D[i] = Jw[i];
  const double dn = (double)n, te = 2.0 * ec, tn = 2.0 / dn;
  double fac = 1.0;            // n^k / k!
  double p1 = 0.0, p3 = 0.0;   // previous order's coefficients of J_{n-1}, J_{n+1}
#pragma unroll
  for (int k = 0; k <= K; ++k) {
    if (k > 0) {
      double left = D[k - 1];
#pragma unroll
      for (int i = k; i <= W - 1 - k; ++i) {
        const double old = D[i];
        D[i] = 0.5 * (left - D[i + 1]);
        left = old;
      }
      fac *= dn * (1.0 / (double)k);
    }
    // delta^k coefficients of J_{n-2} .. J_{n+2} at e_c + delta
    const double c0 = fac * D[K], c1 = fac * D[K + 1], c2 = fac * D[K + 2], c3 = fac * D[K + 3], c4 = fac * D[K + 4];
    const double A = dn * (c0 - te * c1 - 2.0 * p1 + tn * c2 + te * c3 + 2.0 * p3 - c4);
    const double B = dn * (c0 - 2.0 * c2 + c4);
    if constexpr (sizeof(T) == 4) {
      T *pr = tab + ((n - 1) >> 1) * stride;
      const int h = (n - 1) & 1;
      pr[2 * (K + 1) * h + 2 * k] = (T)A;
      pr[2 * (K + 1) * h + 2 * k + 1] = (T)B;
      pr[4 * (K + 1) + 2 * k + h] = (T)c2;
    } else {
      T *row = tab + (n - 1) * stride;
      row[k] = (T)A;
      row[K + 1 + k] = (T)B;
      row[2 * (K + 1) + k] = (T)c2;
    }
    p1 = c1;
    p3 = c3;
  }
}

// Zero coefficients for harmonic n of an FP32 pair row (the harmonic past an odd count).
template <int K>
__device__ __forceinline__ void zero_taylor_row_k(float *tab, int stride, int n) {
  float *pr = tab + ((n - 1) >> 1) * stride;
  const int h = (n - 1) & 1;
#pragma unroll
  for (int k = 0; k <= K; ++k) {
    pr[2 * (K + 1) * h + 2 * k] = 0.f;
    pr[2 * (K + 1) * h + 2 * k + 1] = 0.f;
    pr[4 * (K + 1) + 2 * k + h] = 0.f;
  }
}

// Table row of harmonic n (tab: the tile's table, stride: row_stride of the
// tile, or larger); n = nmodes + 1 of an FP32 table writes the zero half of
// the last pair.
template <typename T>
__device__ void build_taylor_row(T *tab, int stride, int n, int nmodes, double ec, int K, int start) {
  if constexpr (sizeof(T) == 4) {
    if (n > nmodes) {
      switch (K) {
        case 2: zero_taylor_row_k<2>(tab, stride, n); break;
        case 3: zero_taylor_row_k<3>(tab, stride, n); break;
        case 4: zero_taylor_row_k<4>(tab, stride, n); break;
        default: zero_taylor_row_k<6>(tab, stride, n); break;
      }
      return;
    }
    switch (K) {
      case 2: build_taylor_row_k<2, T>(tab, stride, n, ec, start); break;
      case 3: build_taylor_row_k<3, T>(tab, stride, n, ec, start); break;
      case 4: build_taylor_row_k<4, T>(tab, stride, n, ec, start); break;
      default: build_taylor_row_k<6, T>(tab, stride, n, ec, start); break;
    }
  } else {
    switch (K) {
      case 4: build_taylor_row_k<4, T>(tab, stride, n, ec, start); break;
      case 5: build_taylor_row_k<5, T>(tab, stride, n, ec, start); break;
      case 6: build_taylor_row_k<6, T>(tab, stride, n, ec, start); break;
      case 8: build_taylor_row_k<8, T>(tab, stride, n, ec, start); break;
      default: build_taylor_row_k<10, T>(tab, stride, n, ec, start); break;
    }
  }
}

// Terms for a tile where n |delta| <= q: the remainder of A_n, B_n, C_n is
// below 8 nmodes q^(K+1) / (K+1)! e^q (|J^(k)| <= 1); 0 = per-sample Miller.
__device__ __forceinline__ double taylor_tail(double q, int nmodes, int K) {
  double t = 8.0 * nmodes * exp(q);
  for (int k = 1; k <= K + 1; ++k) t *= q / (double)k;
  return t;
}
__device__ __forceinline__ int taylor_terms_fp64(double q, int nmodes) {
  if (!(q <= 1.0)) return 0;
  const int opts[5] = {4, 5, 6, 8, 10};
  for (int i = 0; i < 5; ++i)
    if (taylor_tail(q, nmodes, opts[i]) < 1e-17) return opts[i];
  return 0;
}
__device__ __forceinline__ int taylor_terms_fp32(double q, int nmodes) {
  if (!(q <= 1.0)) return 0;
  const int opts[4] = {2, 3, 4, 6};
  for (int i = 0; i < 4; ++i)
    if (taylor_tail(q, nmodes, opts[i]) < 1e-9) return opts[i];
  return 0;
}

// Mode sums Sa = sum A_n cos(n Phi'), Sb = sum B_n sin(n Phi'), Sc = sum C_n
// cos(n Phi') from the tile table at delta = e - e_c, with the harmonic
// phases from the rotation recurrence w_n = w_{n-1} z_1, w_0 = z_D (so
// w_n = z_1^n z_D: one complex product per harmonic), for M samples of one
// tile at once: each table row is loaded once for all of them and the M
// recurrences run side by side.  FP64 tables.
template <int K, int M>
__device__ __forceinline__ void mode_sums_fp64(const double *tab, int nmodes, int stride, const double *dl,
                                               const double *c1, const double *s1, const double *cD, const double *sD,
                                               double *Sa, double *Sb, double *Sc) {
  constexpr int NV = 3 * (K + 1);
  double zr[M], zi[M], sa[M], sb[M], sc[M];
#pragma unroll
  for (int m = 0; m < M; ++m) {
    zr[m] = cD[m];  // w_0 = z_D; w_n = w_{n-1} z_1 = z_1^n z_D
    zi[m] = sD[m];
    sa[m] = sb[m] = sc[m] = 0.0;
  }
#pragma unroll 2  // two harmonics' Horner chains side by side (unrolling by four was slower)
  for (int n = 1; n <= nmodes; ++n) {
    double v[(NV + 1) / 2 * 2];
    const double2 *r2 = reinterpret_cast<const double2 *>(tab + (n - 1) * stride);
#pragma unroll
    for (int i = 0; i < (NV + 1) / 2; ++i) {
      const double2 q = r2[i];
      v[2 * i] = q.x;
      v[2 * i + 1] = q.y;
    }
#pragma unroll
    for (int m = 0; m < M; ++m) {
      double A = v[K], B = v[2 * K + 1], C = v[3 * K + 2];
#pragma unroll
      for (int k = K - 1; k >= 0; --k) {
        A = fma(A, dl[m], v[k]);
        B = fma(B, dl[m], v[K + 1 + k]);
        C = fma(C, dl[m], v[2 * (K + 1) + k]);
      }
      const double tr = zr[m] * c1[m] - zi[m] * s1[m];
      zi[m] = fma(zr[m], s1[m], zi[m] * c1[m]);
      zr[m] = tr;
      sa[m] = fma(A, zr[m], sa[m]);
      sb[m] = fma(B, zi[m], sb[m]);
      sc[m] = fma(C, zr[m], sc[m]);
    }
  }
#pragma unroll
  for (int m = 0; m < M; ++m) {
    Sa[m] = sa[m];
    Sb[m] = sb[m];
    Sc[m] = sc[m];
  }
}

// The same sums from an FP32 pair table (split precision).  Per pair of
// harmonics (2p+1, 2p+2): the A, B polynomials of each harmonic and the C
// polynomials of both as packed FP32x2 Horner chains, two rotor steps, and
// (Sa, Sb) += (A, B) (Re w, Im w) and (Sc_odd, Sc_even) += (C_odd, C_even)
// (Re w_odd, Re w_even) as packed FMAs.  The rotor is re-anchored at every
// harmonic n = 8j: exp(i (n Phi' + D0)) with n Phi' + D0 reduced in FP64, so
// the FP32 recurrence carries at most 7 steps (w_1 .. w_7 from z_D, w_{8j+1}
// .. w_{8j+7} from an anchor) of rounding and of the error of z_1, whatever n:
// the n Phi argument reduction stays FP64.  Pairs run in blocks of four
// (harmonics 8b+1 .. 8b+8, the last one the anchor), then the remaining
// fewer than four pairs, which hold no anchor.
constexpr int kAnchorEvery = 8;
template <int K, int M, bool kAnchorLast>
__device__ __forceinline__ void pair_step(const float *pr, int nlast, const float *dl, const float *c1, const float *s1,
                                          const double *ph, const float *d0, float *zr, float *zi, float2 *sab,
                                          float2 *sc2) {
  constexpr int PV = 6 * (K + 1), PV4 = (PV + 3) / 4;
  float v[PV4 * 4];
  const float4 *r4 = reinterpret_cast<const float4 *>(pr);
#pragma unroll
  for (int i = 0; i < PV4; ++i) {
    const float4 q = r4[i];
    v[4 * i] = q.x;
    v[4 * i + 1] = q.y;
    v[4 * i + 2] = q.z;
    v[4 * i + 3] = q.w;
  }
#pragma unroll
  for (int m = 0; m < M; ++m) {
    const float2 dd = make_float2(dl[m], dl[m]);
    float2 ABo = make_float2(v[2 * K], v[2 * K + 1]);
    float2 ABe = make_float2(v[2 * (K + 1) + 2 * K], v[2 * (K + 1) + 2 * K + 1]);
    float2 Cp = make_float2(v[4 * (K + 1) + 2 * K], v[4 * (K + 1) + 2 * K + 1]);
#pragma unroll
    for (int k = K - 1; k >= 0; --k) {
      ABo = __ffma2_rn(ABo, dd, make_float2(v[2 * k], v[2 * k + 1]));
      ABe = __ffma2_rn(ABe, dd, make_float2(v[2 * (K + 1) + 2 * k], v[2 * (K + 1) + 2 * k + 1]));
      Cp = __ffma2_rn(Cp, dd, make_float2(v[4 * (K + 1) + 2 * k], v[4 * (K + 1) + 2 * k + 1]));
    }
    // w of the odd harmonic, then of the even one (the anchor at the end of a block)
    const float ro = zr[m] * c1[m] - zi[m] * s1[m];
    const float io = fmaf(zr[m], s1[m], zi[m] * c1[m]);
    float re, ie;
    if constexpr (kAnchorLast) {
      __sincosf(reduce_2pi_f(fma((double)nlast, ph[m], (double)d0[m])), &ie, &re);
    } else {
      re = ro * c1[m] - io * s1[m];
      ie = fmaf(ro, s1[m], io * c1[m]);
    }
    sab[m] = __ffma2_rn(ABo, make_float2(ro, io), sab[m]);
    sab[m] = __ffma2_rn(ABe, make_float2(re, ie), sab[m]);
    sc2[m] = __ffma2_rn(Cp, make_float2(ro, re), sc2[m]);
    zr[m] = re;
    zi[m] = ie;
  }
}

template <int K, int M>
__device__ __forceinline__ void mode_sums_split(const float *tab, int nmodes, int stride, const float *dl,
                                                const float *c1, const float *s1, const float *cD, const float *sD,
                                                const double *ph, const float *d0, float *Sa, float *Sb, float *Sc) {
  static_assert(kAnchorEvery == 8, "a block of four pairs ends at the anchor");
  float zr[M], zi[M];
  float2 sab[M], sc2[M];
#pragma unroll
  for (int m = 0; m < M; ++m) {
    zr[m] = cD[m];  // w_0 = z_D
    zi[m] = sD[m];
    sab[m] = sc2[m] = make_float2(0.f, 0.f);
  }
  const int npairs = (nmodes + 1) >> 1;
  int p = 0;
#pragma unroll 1
  for (; p + 4 <= npairs; p += 4) {
    const float *pr = tab + p * stride;
    pair_step<K, M, false>(pr, 0, dl, c1, s1, ph, d0, zr, zi, sab, sc2);
    pair_step<K, M, false>(pr + stride, 0, dl, c1, s1, ph, d0, zr, zi, sab, sc2);
    pair_step<K, M, false>(pr + 2 * stride, 0, dl, c1, s1, ph, d0, zr, zi, sab, sc2);
    pair_step<K, M, true>(pr + 3 * stride, 2 * p + 8, dl, c1, s1, ph, d0, zr, zi, sab, sc2);
  }
#pragma unroll 1
  for (; p < npairs; ++p) pair_step<K, M, false>(tab + p * stride, 0, dl, c1, s1, ph, d0, zr, zi, sab, sc2);
#pragma unroll
  for (int m = 0; m < M; ++m) {
    Sa[m] = sab[m].x;
    Sb[m] = sab[m].y;
    Sc[m] = sc2[m].x + sc2[m].y;
  }
}

// Mode sums with a per-sample Miller recurrence (fallback when the table does not apply).
__device__ void mode_sums_miller(const int32_t *bstart, int nmodes, double e, double c1, double s1, double cD,
                                 double sD, double &Sa, double &Sb, double &Sc) {
  double zr = 1.0, zi = 0.0;
  double sa = 0.0, sb = 0.0, sc = 0.0;
  for (int n = 1; n <= nmodes; ++n) {
    const double tr = zr * c1 - zi * s1;
    zi = zr * s1 + zi * c1;
    zr = tr;
    const double cn = zr * cD - zi * sD;
    const double sn = zi * cD + zr * sD;
    double J[5];
    const double x = n * e;
    if (x <= 0.0) {
      J[0] = J[1] = J[2] = J[3] = J[4] = 0.0;
      if (n == 1) J[1] = 1.0;
      if (n == 2) J[0] = 1.0;
    } else if (n == 1) {
      double Jt[5];
      bessel5_fp64(0, x, bstart[0], Jt);
      J[0] = -Jt[1];
      J[1] = Jt[0];
      J[2] = Jt[1];
      J[3] = Jt[2];
      J[4] = Jt[3];
    } else {
      bessel5_fp64(n - 2, x, bstart[n - 1], J);
    }
    const double dn = (double)n;
    sa += dn * (J[0] - 2. * e * J[1] + 2. / dn * J[2] + 2. * e * J[3] - J[4]) * cn;
    sb += dn * (J[0] - 2. * J[2] + J[4]) * sn;
    sc += J[2] * cn;
  }
  Sa = sa;
  Sb = sb;
  Sc = sc;
}

// ------------------------------------------------------------------ harmonic sum
// cos 2 atan2(y, x) and sin 2 atan2(y, x) without the angle (atan2(0, 0) = 0)
template <typename T>
__device__ __forceinline__ void double_angle(T y, T x, T &c2, T &s2) {
  const T r2 = x * x + y * y;
  if (r2 > T(0)) {
    T inv;  // FP32: the approximate reciprocal (2 ulp), below the FP32 response's own rounding
    if constexpr (sizeof(T) == 4) inv = __fdividef(T(1), r2);
    else inv = T(1) / r2;
    c2 = (x * x - y * y) * inv;
    s2 = T(2) * x * y * inv;
  } else {
    c2 = T(1);
    s2 = T(0);
  }
}

// Response and orientation factors of one sample (AAK.cc:425-478 with the
// NK-frame rotation of KSParMap.cc:532-574), from the per-source constants of
// SourceDesc and the sample's (cos alpha, sin alpha), (cos 2 gamma~, sin 2 gamma~)
// and orbital phase (cos, sin).  The angles the reference forms with atan2
// (phi_L, beta, the LISA phi and psi) enter only through cos/sin of them or
// of twice them, which follow from the atan2 arguments algebraically.
// Output: the coefficients of Sa, Sb, Sc in h_I and h_II.
template <typename T>
struct Resp {
  T caI, cbI, ccI, caII, cbII, ccII;
  T cosorb_S;  // cos(orbital phase - phi_S), for the Doppler term
};

// The per-source constants response() reads, in the arithmetic type of the
// harmonic sum; one copy per tile in shared memory.
template <typename T>
struct Geom {
  T Lc[3], Ls[3], Lq[3], nv[3], Sv[3], nxS[3];
  T nxS_norm, inv_nxS_norm, Sdotn, coslam, beta_c, beta_s, cphiS, sphiS, cosphiK, sinphiK;
  T cosqS, sinqS, cosqK, sinqK, psd0, psd1, psd2, F0[4], zeta;
  int mich;
};

template <typename T>
__device__ void make_geom(const SourceDesc &d, Geom<T> &g) {
  for (int i = 0; i < 3; ++i) {
    g.Lc[i] = (T)d.Lc[i];
    g.Ls[i] = (T)d.Ls[i];
    g.Lq[i] = (T)d.Lq[i];
    g.nv[i] = (T)d.nv[i];
    g.Sv[i] = (T)d.Sv[i];
    g.nxS[i] = (T)d.nxS[i];
  }
  g.nxS_norm = (T)d.nxS_norm;
  g.inv_nxS_norm = (T)(1.0 / d.nxS_norm);
  g.Sdotn = (T)d.Sdotn;
  g.coslam = (T)d.coslam;
  g.beta_c = (T)d.beta_c;
  g.beta_s = (T)d.beta_s;
  g.cphiS = (T)d.cphiS;
  g.sphiS = (T)d.sphiS;
  g.cosphiK = (T)d.cosphiK;
  g.sinphiK = (T)d.sinphiK;
  g.cosqS = (T)d.cosqS;
  g.sinqS = (T)d.sinqS;
  g.cosqK = (T)d.cosqK;
  g.sinqK = (T)d.sinqK;
  g.psd0 = (T)d.psd0;
  g.psd1 = (T)d.psd1;
  g.psd2 = (T)d.psd2;
  for (int i = 0; i < 4; ++i) g.F0[i] = (T)d.F0[i];
  g.zeta = (T)d.zeta;
  g.mich = d.mich;
}

template <typename T>
__device__ __forceinline__ Resp<T> response(const Geom<T> &d, T ca, T sa, T c2g, T s2g, T co, T so) {
  const T L0 = (T)d.Lc[0] + sa * (T)d.Ls[0] + ca * (T)d.Lq[0];
  const T L1 = (T)d.Lc[1] + sa * (T)d.Ls[1] + ca * (T)d.Lq[1];
  const T L2 = (T)d.Lc[2] + ca * (T)d.Lq[2];
  const T n0 = (T)d.nv[0], n1 = (T)d.nv[1], n2 = (T)d.nv[2];
  const T Ldotn = L0 * n0 + L1 * n1 + L2 * n2;
  const T Ldotn2 = Ldotn * Ldotn;
  const T Sdotn = (T)d.Sdotn;
  // gamma = 2 (gamma~ + beta), beta = atan2(-S.n + cos(lambda) L.n, beta_c cos(alpha) + beta_s sin(alpha))
  T c2b, s2b;
  double_angle<T>(-Sdotn + (T)d.coslam * Ldotn, (T)d.beta_c * ca + (T)d.beta_s * sa, c2b, s2b);
  const T cos2gam = c2g * c2b - s2g * s2b, sin2gam = s2g * c2b + c2g * s2b;

  T FplusI, FcrosI, FplusII, FcrosII, Kr;
  T cosorb_S = T(0);
  if (d.mich) {
    const T hs3 = (T)kHalfSqrt3;
    const T cS = (T)d.cosqS, sS = (T)d.sinqS, cK = (T)d.cosqK, sK = (T)d.sinqK;
    cosorb_S = co * (T)d.cphiS + so * (T)d.sphiS;
    const T sinorb_S = so * (T)d.cphiS - co * (T)d.sphiS;
    const T cosorb_K = co * (T)d.cosphiK + so * (T)d.sinphiK;
    const T cosq = T(.5) * cS - hs3 * sS * cosorb_S;
    // 2 phi_w = 2 orb + 2 atan2(hs3 cos qS + sin qS cos(orb - phiS) / 2, sin qS sin(orb - phiS))
    T c2w, s2w;
    double_angle<T>(hs3 * cS + T(.5) * sS * cosorb_S, sS * sinorb_S, c2w, s2w);
    const T c2o = co * co - so * so, s2o = T(2) * so * co;
    const T cos2phi = c2o * c2w - s2o * s2w, sin2phi = s2o * c2w + c2o * s2w;
    T cos2psi, sin2psi;
    double_angle<T>(T(.5) * cK - hs3 * sK * cosorb_K - cosq * Sdotn, (T)d.psd0 - (T)d.psd1 * co - (T)d.psd2 * so,
                    cos2psi, sin2psi);
    const T cosq1 = T(.5) * (T(1) + cosq * cosq);
    FplusI = cosq1 * cos2phi * cos2psi - cosq * sin2phi * sin2psi;
    FcrosI = cosq1 * cos2phi * sin2psi + cosq * sin2phi * cos2psi;
    FplusII = cosq1 * sin2phi * cos2psi + cosq * cos2phi * sin2psi;
    FcrosII = cosq1 * sin2phi * sin2psi - cosq * cos2phi * cos2psi;
    Kr = hs3;
  } else {
    FplusI = (T)d.F0[0];
    FcrosI = (T)d.F0[1];
    FplusII = (T)d.F0[2];
    FcrosII = (T)d.F0[3];
    Kr = T(1);
  }
  // rotation to the NK wave frame: rot = [r0, r1, -r1, r0]
  const T nL0 = n1 * L2 - n2 * L1, nL1 = n2 * L0 - n0 * L2, nL2 = n0 * L1 - n1 * L0;
  const T S0 = (T)d.Sv[0], S1 = (T)d.Sv[1], S2 = (T)d.Sv[2];
  const T nS0 = (T)d.nxS[0], nS1 = (T)d.nxS[1], nS2 = (T)d.nxS[2];
  T cosrot, sinrot;
  if constexpr (sizeof(T) == 4) {
    // 1 / (|n x L| |n x S|) from the approximate reciprocal square root (2 ulp)
    const T rn = rsqrtf(nL0 * nL0 + nL1 * nL1 + nL2 * nL2) * d.inv_nxS_norm;
    cosrot = (nL0 * nS0 + nL1 * nS1 + nL2 * nS2) * rn;
    sinrot = ((L0 * nS0 + L1 * nS1 + L2 * nS2) - (S0 * nL0 + S1 * nL1 + S2 * nL2)) * rn;
  } else {
    const T norm = sqrt(nL0 * nL0 + nL1 * nL1 + nL2 * nL2) * (T)d.nxS_norm;
    cosrot = (nL0 * nS0 + nL1 * nS1 + nL2 * nS2) / norm;
    sinrot = ((L0 * nS0 + L1 * nS1 + L2 * nS2) - (S0 * nL0 + S1 * nL1 + S2 * nL2)) / norm;
  }
  const T r0 = T(2) * cosrot * cosrot - T(1), r1 = cosrot * sinrot;
  const T uI = FplusI * r0 - FcrosI * r1, wI = FplusI * r1 + FcrosI * r0;
  const T uII = FplusII * r0 - FcrosII * r1, wII = FplusII * r1 + FcrosII * r0;
  const T opL2 = T(1) + Ldotn2, omL2 = T(1) - Ldotn2, twoL = T(2) * Ldotn;
  Resp<T> R;
  R.caI = Kr * (-uI * opL2 * cos2gam + wI * twoL * sin2gam);
  R.cbI = Kr * (uI * opL2 * sin2gam + wI * twoL * cos2gam);
  R.ccI = Kr * uI * omL2;
  R.caII = Kr * (-uII * opL2 * cos2gam + wII * twoL * sin2gam);
  R.cbII = Kr * (uII * opL2 * sin2gam + wII * twoL * cos2gam);
  R.ccII = Kr * uII * omL2;
  R.cosorb_S = cosorb_S;
  return R;
}


// Everything of one sample's harmonic sum except the mode sums: response
// coefficients, amplitude and the harmonic phase rotors.
template <typename T>
struct SamplePrep {
  Resp<T> R;
  T Amp, se;            // amplitude, sqrt(1 - e^2)
  T c1, s1, cD, sD;     // harmonic n: (c1 + i s1)^n (cD + i sD)
  double ph;            // split: Phi + Doppler term reduced to [-pi, pi] in FP64 (the rotor's anchors)
  T d0;                 // split: the harmonic-independent phase D0 (cD + i sD = exp(i D0))
  T dl;                 // e - e_c
};

__device__ __forceinline__ SamplePrep<double> prep_fp64(const SourceDesc &d, const Geom<double> &g, double ec, double t, double e,
                                                         double om_M, double gim, double Phi, double alp, double nu,
                                                         double gimdot) {
  SamplePrep<double> P;
  double sa, ca, s2g, c2g, so = 0.0, co = 1.0;
  sincos(alp, &sa, &ca);
  sincos(2. * gim, &s2g, &c2g);
  if (d.mich) sincos(kTwoPi * t / kYear, &so, &co);
  P.R = response<double>(g, ca, sa, c2g, s2g, co, so);
  P.Amp = pow(om_M, 2. / 3.) * d.zeta;
  double D1 = 0.0, D0 = 0.0;
  if (d.mich) {
    D1 = kTwoPi * nu * kAUsec * d.sinqS * P.R.cosorb_S;
    D0 = 2.0 * gimdot * kAUsec * d.sinqS * P.R.cosorb_S;
  }
  sincos(Phi + D1, &P.s1, &P.c1);
  sincos(D0, &P.sD, &P.cD);
  P.ph = 0.0;  // the FP64 rotor needs no anchors
  P.d0 = 0.0;
  P.se = sqrt(1. - e * e);
  P.dl = e - ec;
  return P;
}

__device__ __forceinline__ SamplePrep<float> prep_split(const SourceDesc &d, const Geom<float> &g, double ec, double t, double e_d,
                                                        double om_M, double gim, double Phi, double alp, double nu,
                                                        double gimdot) {
  SamplePrep<float> P;
  float sa, ca, s2g, c2g, so = 0.f, co = 1.f;
  __sincosf(reduce_2pi_f(alp), &sa, &ca);
  __sincosf(reduce_2pi_f(2.0 * gim), &s2g, &c2g);
  if (d.mich) __sincosf(reduce_2pi_f(t * (kTwoPi / kYear)), &so, &co);  // a product, not a division, in FP64
  P.R = response<float>(g, ca, sa, c2g, s2g, co, so);
  P.Amp = exp2f((2.f / 3.f) * __log2f((float)om_M)) * g.zeta;
  double D1 = 0.0;
  float D0 = 0.f;
  if (d.mich) {
    D1 = kTwoPi * nu * kAUsec * d.sinqS * (double)P.R.cosorb_S;
    D0 = (float)(2.0 * gimdot * kAUsec * d.sinqS) * P.R.cosorb_S;
  }
  // the rotor z_1 from the FP64 reduction, with the accurate sincosf: its
  // phase error is multiplied by the harmonic number between two anchors
  P.ph = reduce_2pi_d(Phi + D1);
  sincosf((float)P.ph, &P.s1, &P.c1);
  P.d0 = D0;
  __sincosf(D0, &P.sD, &P.cD);
  const float e = (float)e_d;
  P.se = sqrtf(1.f - e * e);
  P.dl = (float)(e_d - ec);
  return P;
}

template <typename T>
__device__ __forceinline__ void finish(const SamplePrep<T> &P, T Sa, T Sb, T Sc, double &hI, double &hII) {
  const T a = -P.Amp * Sa, b = -P.Amp * P.se * Sb, cc = T(2) * P.Amp * Sc;
  hI = (double)(P.R.caI * a + P.R.cbI * b + P.R.ccI * cc);
  hII = (double)(P.R.caII * a + P.R.cbII * b + P.R.ccII * cc);
}


// ------------------------------------------------------------------ split precision
// FP64: spline, rates, phase sums and every angle reduction; FP32: geometry,
// antenna response, Bessel evaluation and the harmonic recurrence.



// ------------------------------------------------------------------ tile pre-pass
// The per-tile work of the waveform kernel that does not depend on the phase
// scan, done for every tile of the batch before it: (1) k_tile_params, one
// thread per tile: e at the tile's first, middle and last output samples
// (the Taylor-table centre e_c and term count K), and the raw rates of the
// samples just before and after the tile; (2) k_tile_table, one thread per
// (tile, harmonic): the tile's Taylor row of that harmonic.  Both evaluate
// the spline with the same window, search and arithmetic as the waveform
// kernel, so the values equal the ones it would compute itself.
template <bool kSplit>
__global__ void __launch_bounds__(128) k_tile_params(BatchView bv) {
  const int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (g >= bv.total_tiles) return;
  const int s = find_source(bv.tile_start, bv.nsrc, g);
  const SourceDesc &d = bv.src[s];
  TilePrep P;
  P.ec = 0.0;
  P.K = -1;
  P.stride = 0;
  P.src = s;
  for (int q = 0; q < 3; ++q) P.rb[q] = P.ra[q] = 0.0;
  P.rb[1] = -1.0;
  const int lt = (int)(g - bv.tile_start[s]);
  const int start = lt * kTileSamples, end = min(start + kTileSamples, d.vlength);
  const int lim = min(end, n_eff(d));
  // the rates either side of every tile (the phase product uses the tiles
  // after the taper as well); the table parameters of tiles with output
  KnotWin w{nullptr, nullptr, nullptr, nullptr, nullptr, 0, 0, 0};
  if (d.status == 0 && end > start) {
    w.k0 = bv.tile_knot[2 * g];
    w.n = bv.tile_knot[2 * g + 1];
    const double *kt = bv.knot_t + d.knot_offset;
    const double span = kt[w.k0 + w.n - 1] - kt[w.k0];
    w.inv_h = (span > 0.0) ? (double)(w.n - 1) / span : 0.0;
    {
      double r[3] = {0, 0, 0};
      const int i = start - 1;
      const bool ok = i >= 0 && i < d.vlength;
      if (ok) phase_rates(d, spline4w(bv, d, sample_time(d, i), w), r);
      P.rb[0] = r[0];
      P.rb[1] = ok ? r[1] : -1.0;
      P.rb[2] = r[2];
    }
    if (end - 1 < d.i0 && end < d.vlength) {
      double r[3] = {0, 0, 0};
      phase_rates(d, spline4w(bv, d, sample_time(d, end), w), r);
      P.ra[0] = r[0];
      P.ra[1] = r[1];
      P.ra[2] = r[2];
    }
  }
  if (d.status == 0 && lim > start) {  // lim <= end: the window above is set
    const double e0 = spline4w(bv, d, sample_time(d, start), w).e;
    const double em = spline4w(bv, d, sample_time(d, (start + lim - 1) / 2), w).e;
    const double e1 = spline4w(bv, d, sample_time(d, lim - 1), w).e;
    int K = 0;
    double ec = 0.0;
    if (d.nmodes <= kTabModes) {
      ec = em;
      const double de = fmax(fabs(e0 - ec), fabs(e1 - ec));
      if (ec > 1e-6) {
        const double q = d.nmodes * (1.25 * de + 1e-15);  // bounds n |e - e_c| over the tile
        K = kSplit ? taylor_terms_fp32(q, d.nmodes) : taylor_terms_fp64(q, d.nmodes);
      }
    }
    P.ec = ec;
    P.K = (int16_t)K;
    P.stride = (int16_t)(K > 0 ? (kSplit ? row_stride<float>(K) : row_stride<double>(K)) : 0);
  }
  bv.tile_prep[g] = P;
}

template <bool kSplit>
__global__ void __launch_bounds__(128) k_tile_table(BatchView bv, int rows) {
  using T = typename std::conditional<kSplit, float, double>::type;
  const int64_t id = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t g = id / rows;
  if (g >= bv.total_tiles) return;
  const int n = (int)(id - g * rows) + 1;
  const TilePrep &P = bv.tile_prep[g];
  const int K = P.K;
  if (K <= 0) return;
  const SourceDesc &d = bv.src[P.src];
  if (n > table_rows<T>(d.nmodes)) return;
  T *tab = reinterpret_cast<T *>(static_cast<unsigned char *>(bv.tile_tab) + g * bv.tab_slot);
  build_taylor_row<T>(tab, P.stride, n, d.nmodes, P.ec, K, (n <= d.nmodes) ? bv.bessel_start[d.bessel_offset + n - 1] : 0);
}

// ------------------------------------------------------------------ waveform kernel
// Samples per thread whose harmonic sums run side by side (divides kTileChunks).
// 1: build the Taylor table after phase 1, on warps 1-7 while warp 0 looks
// back; 0: before phase 1, overlapping its first chunk.
#ifndef AAK_TABLE_AFTER_SCAN
#define AAK_TABLE_AFTER_SCAN 1
#endif
#ifndef AAK_JOINT_SPLIT
#define AAK_JOINT_SPLIT 2
#endif
#ifndef AAK_JOINT_FP64
#define AAK_JOINT_FP64 1
#endif
static_assert(kTileChunks % AAK_JOINT_SPLIT == 0 && kTileChunks % AAK_JOINT_FP64 == 0, "joint samples must divide the chunks");
// Per tile: phase 1 computes, for the tile's 1024 samples, the spline, rates,
// clamped Phidot and the block-scanned AB2 phases (uniform, cheap work with
// the tile's barriers) and parks each sample's harmonic-sum inputs in shared
// memory; after one barrier, phase 2 evaluates the harmonic sums of each
// thread's own samples with no further barriers.
constexpr int kDynVals = 7;  // e, Omega_phi M_phys, gamma~, Phi, alpha, nu, gamma~dot
constexpr size_t kWaveDynSmem = (size_t)kDynVals * kTileSamples * sizeof(double);

// kMode 1, the phase product instead of the waveform (FP64 only): every
// sample of each source runs through phase 1, the harmonic sums are skipped,
// and the tile's samples are written to bv.phase_out as t, phase_r,
// phase_theta, phase_phi, omega_r, omega_theta, omega_phi, e (the per-sample
// packing of GenPhase, AAKPhase.cc:346-355).  The phases of the samples
// after the plunge buffer are frozen afterwards by k_phase_freeze.
// kMode 2, the phase grid of the frequency-domain TDI (PNevolutionTDI,
// AAKTDI.cc:311-469): the same pass writes kTdiRows rows (TdiRow order).
// kPre (waveform mode with the tile pre-pass): each tile's source record,
// TilePrep, knot window and Taylor table arrive in shared memory by bulk
// copies that thread 0 issues at the start of the tile (the table's on a
// second mbarrier, waited for only before phase 2); no table is built here.
// kJointT: samples per thread whose harmonic sums run side by side (0: the
// default of the precision); kMinB: resident CTAs per SM the register budget
// is sized for.  Both are launch-shape choices of the autotuner.
static_assert(sizeof(SourceDesc) % 16 == 0, "SourceDesc lands in shared memory with one bulk copy");

// kPre: one thread issues the bulk copies of queue item q's source record,
// its TilePrep and, when its knot window has at most kWin knots, the window's
// knot times (from a 16-byte boundary: one element of slack is allocated past
// the last knot), values and spline coefficients, all completing on bar; win
// gets the window's first knot, knot count and offset of the first time in
// wt.  The caller orders every earlier read of the destinations before it.
__device__ __forceinline__ void issue_stage(const BatchView &bv, const QueueItem &q, SourceDesc *desc, TilePrep *prep,
                                            int *win, double *wt, double4 *wy, double4 *wc, uint64_t *bar) {
  fence_proxy_async_smem();
  const int nk = q.nk;
  const bool staged = nk > 0 && nk <= kWin;
  const int64_t off = q.knot;
  const int64_t a = off & ~(int64_t)1;  // knot times from a 16-byte boundary
  const int toff = (int)(off - a);
  const int cnt = (nk + toff + 1) & ~1;
  const uint32_t b0 = (uint32_t)(sizeof(SourceDesc) + sizeof(TilePrep)) +
                      (staged ? (uint32_t)(cnt * sizeof(double) + 2 * nk * sizeof(double4)) : 0u);
  mbar_arrive_expect_tx(bar, b0);
  bulk_copy_g2s(desc, bv.src + q.s, (uint32_t)sizeof(SourceDesc), bar);
  bulk_copy_g2s(prep, bv.tile_prep + q.g, (uint32_t)sizeof(TilePrep), bar);
  if (staged) {
    bulk_copy_g2s(wt, bv.knot_t + a, (uint32_t)(cnt * sizeof(double)), bar);
    bulk_copy_g2s(wy, bv.knot_y + off, (uint32_t)(nk * sizeof(double4)), bar);
    bulk_copy_g2s(wc, bv.knot_c + off, (uint32_t)(nk * sizeof(double4)), bar);
  }
  win[0] = q.k0;
  win[1] = nk;
  win[2] = toff;
}

template <bool kSplit, int kMode = 0, bool kPre = false, int kJointT = 0, int kMinB = AAK_WAVE_MIN_BLOCKS>
__global__ void __launch_bounds__(kTileThreads, kMinB) k_waveform(BatchView bv) {
  constexpr bool kPhase = kMode != 0, kTdi = kMode == 2;
  static_assert(!kPre || kMode != 2, "the pre-pass serves the waveform and phase modes");
  extern __shared__ double s_dyn[];  // [kDynVals][kTileSamples]
  __shared__ double red[2][3][kTileThreads / 32];  // warp totals of the forward and backward scans
  __shared__ long long s_tile;
  __shared__ double s_par[3], s_rb[3], s_ra[3], s_cy[7], s_lastP;  // tile parameters, chain carry
  __shared__ __align__(16) SourceDesc s_desc;           // this tile's source
  __shared__ __align__(16) TilePrep s_prep;             // kPre: this tile's parameters
  __shared__ __align__(8) uint64_t s_mbar[2];           // kPre: bulk-copy barriers (record + window, table)
  __shared__ int s_win[4];                              // kPre: window first knot, knots, offset in s_wt, table
  __shared__ Geom<typename std::conditional<kSplit, float, double>::type> s_geom;
  __shared__ __align__(16) double s_wt[kWin + 2];
  __shared__ __align__(16) double4 s_wy[kWin], s_wc[kWin], s_wb[kWin], s_wd[kWin];
  double *sv_e = s_dyn, *sv_om = s_dyn + kTileSamples, *sv_gim = s_dyn + 2 * kTileSamples;
  double *sv_Phi = s_dyn + 3 * kTileSamples, *sv_alp = s_dyn + 4 * kTileSamples, *sv_nu = s_dyn + 5 * kTileSamples;
  double *sv_gd = s_dyn + 6 * kTileSamples;
  double *tabD = s_dyn + kDynVals * kTileSamples;  // Taylor table after the per-sample values
  float *tabF = reinterpret_cast<float *>(tabD);
  const int tid = threadIdx.x;
  uint32_t ph0 = 0u, ph1 = 0u;  // kPre: phase parity of the two barriers
  if constexpr (kPre) {
    if (tid == 0) {
      mbar_init(&s_mbar[0], 1);
      mbar_init(&s_mbar[1], 1);
      mbar_init_fence();
    }
    __syncthreads();
  }
  // Work queue: the first tile is fetched here, every later one by a thread
  // of warp 1 while warp 0 looks back in the tile before it (an empty tile:
  // by thread 0 at its end), so that the atomic's round trip overlaps the
  // look-back.  Items leave the queue in chain order, and a CTA's next item
  // always comes after its current one, so the earliest unfinished item is
  // always being worked on and its predecessors are done: holding one item
  // ahead cannot stall the chains.  (Fetching at the start of the tile was
  // slower: the CTAs then hold twice as many items, and more of them start
  // while their chain predecessors are still running.)
  if (tid == 0) s_tile = (long long)atomicAdd(bv.work_counter, 1ull);
  __syncthreads();
  for (;;) {
    const long long j = s_tile;
    __syncthreads();
    if (j >= bv.total_tiles) break;
    // kPre (batches, which have queue items): the tile's record, parameters
    // and knot window are requested first thing, straight from its item
    bool empty = false;
    if constexpr (kPre) {
      const QueueItem &q = bv.queue[j];
      empty = (q.flags & (kPhase ? kQueueFailed : kQueueNoWave)) != 0;
      if (tid == 0 && !empty) issue_stage(bv, q, &s_desc, &s_prep, s_win, s_wt, s_wy, s_wc, &s_mbar[0]);
    }
    const SourceDesc *dp;
    const TileCtx c = tile_ctx(bv, j, dp);
    const int64_t g = c.g;
    // samples [start, lim) feed the output (the phase product: every sample);
    // kPre: the item's flags say the same (failed source, or lim <= start)
    const int lim = kPhase ? c.end : min(c.end, c.neff);
    if (!kPre) empty = dp->status != 0 || lim <= c.start;
    if (empty) {
      // failed source, or a tile entirely after the taper: zeros, and an
      // empty aggregate for the chain
      const SourceDesc &dz = *dp;
      for (int ch = 0; ch < kTileChunks; ++ch) {
        const int i = c.start + ch * kTileThreads + tid;
        if (i < c.end) {
          if constexpr (kPhase) {
            for (int r = 0; r < (kTdi ? kTdiRows : 8); ++r) bv.phase_out[r * bv.phase_stride + dz.out_offset + i] = 0.0;
          } else {
            store_h(bv, dz.out_offset + i, 0.0, 0.0);
            if (bv.t_out) bv.t_out[dz.out_offset + i] = (dz.status != 0) ? 0.0 : sample_time(dz, i);
          }
        }
      }
      if (tid == 0) {
        const double zero[3] = {0.0, 0.0, 0.0};
        publish_aggregate(bv, g, zero, 0.0, false);
        s_tile = (long long)atomicAdd(bv.work_counter, 1ull);
      }
      __syncthreads();
      continue;
    }
    KnotWin w{s_wt, s_wy, s_wc, s_wb, s_wd, 0, 0, 0};
    if constexpr (kPre) {
      using TT = typename std::conditional<kSplit, float, double>::type;
      if (tid == kTileThreads - 1) make_geom(*dp, s_geom);
      const bool ok = mbar_wait_bounded(&s_mbar[0], ph0);
      ph0 ^= 1u;
      if (tid == 0 && ok) {
        // the tile's Taylor table (its term count and row stride came with
        // the record; the previous tile's reads of it are ordered before this
        // by the loop's barriers)
        const int nm = s_desc.nmodes;
        const bool tab = !kPhase && s_prep.K > 0 && nm <= kTabModes;
        if (tab) {
          fence_proxy_async_smem();
          // FP64: one row per harmonic; FP32: one row per pair of harmonics
          const uint32_t b1 = (uint32_t)(kSplit ? (nm + 1) >> 1 : nm) * (uint32_t)s_prep.stride * (uint32_t)sizeof(TT);
          mbar_arrive_expect_tx(&s_mbar[1], b1);
          bulk_copy_g2s(tabD, static_cast<const unsigned char *>(bv.tile_tab) + g * bv.tab_slot, b1, &s_mbar[1]);
        }
        s_win[3] = tab ? 1 : 0;
      }
      if (__syncthreads_or(!ok)) {  // a copy did not land: report it and stop this CTA
        if (tid == 0) {
          atomicExch(bv.device_status, 1u);
          if (bv.status_report) atomicExch(bv.status_report, 1u);
        }
        return;
      }
      w.k0 = s_win[0];
      w.n = s_win[1];
      w.staged = w.n > 0 && w.n <= kWin;
      w.t = s_wt + s_win[2];
      finish_window(bv, *dp, w);
    } else {
      // stage the source record and its response constants (the window's barrier publishes them)
      {
        const uint4 *src4 = reinterpret_cast<const uint4 *>(dp);
        uint4 *dst4 = reinterpret_cast<uint4 *>(&s_desc);
        for (int k = tid; k < (int)(sizeof(SourceDesc) / 16); k += kTileThreads) dst4[k] = src4[k];
        if (tid == kTileThreads - 1) make_geom(*dp, s_geom);
      }
      load_window(bv, *dp, g, w);
    }
    const SourceDesc &d = s_desc;
    const int32_t *bstart = bv.bessel_start + d.bessel_offset;
    const double X0[3] = {d.gim0, d.Phi0, d.alp0};
    // tile parameters from the staged window: e at the first, middle and last
    // output samples (Bessel-table centre and term count), and the raw rates
    // of the sample just before the tile (Phi: -1 if there is none); kPre:
    // from the pre-pass
    if (kPre) {
      if (tid < 3) {
        s_rb[tid] = s_prep.rb[tid];
        s_ra[tid] = s_prep.ra[tid];
      }
    } else if (tid < 3) {
      const int i = (tid == 0) ? c.start : (tid == 1) ? (c.start + lim - 1) / 2 : lim - 1;
      s_par[tid] = spline4w(bv, d, sample_time(d, i), w).e;
    } else if (tid == 32) {
      double r[3] = {0, 0, 0};
      const int i = c.start - 1;
      const bool ok = i >= 0 && i < d.vlength;
      if (ok) phase_rates(d, spline4w(bv, d, sample_time(d, i), w), r);
      s_rb[0] = r[0];
      s_rb[1] = ok ? r[1] : -1.0;
      s_rb[2] = r[2];
    } else if (tid == 64) {
      // rates of the sample just after the tile, for the backward AB2 step
      // of its last sample (a backward sample before i0 only)
      double r[3] = {0, 0, 0};
      if (c.end - 1 < d.i0 && c.end < d.vlength) phase_rates(d, spline4w(bv, d, sample_time(d, c.end), w), r);
      s_ra[0] = r[0];
      s_ra[1] = r[1];
      s_ra[2] = r[2];
    }
    // chain direction: +1 after the head tile, -1 before it, 0 the head
    const int dir = (c.lt > c.head) ? 1 : (c.lt < c.head) ? -1 : 0;
    __syncthreads();
    double ec = 0.0;
    int K = 0;
    if (kPre) {
      ec = s_prep.ec;
      K = max((int)s_prep.K, 0);
    } else if (d.nmodes <= kTabModes) {
      ec = s_par[1];
      const double de = fmax(fabs(s_par[0] - ec), fabs(s_par[2] - ec));
      if (ec > 1e-6) {
        const double q = d.nmodes * (1.25 * de + 1e-15);  // bounds n |e - e_c| over the tile
        K = kSplit ? taylor_terms_fp32(q, d.nmodes) : taylor_terms_fp64(q, d.nmodes);
      }
    }
    // A forward tile whose Phidot clamp reaches back past its first sample
    // (raw rate before it not positive) needs the chain's clamped Phidot
    // first: it waits for its whole prefix before phase 1.
    const bool needC = dir > 0 && !(s_rb[1] > 0.0);
    if (needC) {
      if (tid < 32) {
        double hi[3], lo[3], C;
        look_back_warp(bv, c, 1, hi, lo, C);
        if (tid == 0) {
          for (int q = 0; q < 3; ++q) {
            s_cy[q] = hi[q];
            s_cy[3 + q] = lo[q];
          }
          s_cy[6] = C;
        }
      }
      __syncthreads();
    }
    const double Cin = needC ? s_cy[6] : 0.0;
#if !AAK_TABLE_AFTER_SCAN
    // Taylor table rows (one thread per harmonic); its barrier is the first one of phase 1
    if (!kPhase && !kPre && K > 0 && !bv.trajectory_only)
      for (int n = tid + 1; n <= (kSplit ? table_rows<float>(d.nmodes) : d.nmodes); n += kTileThreads) {
        const int st = (n <= d.nmodes) ? bstart[n - 1] : 0;
        if (kSplit) build_taylor_row<float>(tabF, 2 * kRowF, n, d.nmodes, ec, K, st);
        else build_taylor_row<double>(tabD, kRowD, n, d.nmodes, ec, K, st);
      }
#endif
    // ---------------- phase 1: phases of the tile's samples, relative to the tile
    // (A) spline and rates of every sample, kTileChunks per thread (slots
    //     tid + 256 ch, independent of one another); the rates sit in the
    //     phase slots until (C)
    const double Pin = (s_rb[1] > 0.0) ? s_rb[1] : Cin;  // clamped Phidot just before the tile
    int nonpos = 0;                                      // a forward sample whose raw Phidot is not positive
#pragma unroll 1
    for (int ch = 0; ch < kTileChunks; ++ch) {
      const int sl = ch * kTileThreads + tid;
      const int i = c.start + sl;
      Traj4 q = {0, 0, 0, 0};
      double r[3] = {0, 0, 0}, om = 0.0;
      if (i < lim) {
        q = spline4w(bv, d, sample_time(d, i), w);
        phase_rates(d, q, r, &om);
        if (i >= d.i0 && !(r[1] > 0.0)) nonpos = 1;
        if (bv.traj_out) {
          const int64_t o = d.out_offset + i;
          const int64_t st = bv.traj_stride;
          bv.traj_out[0 * st + o] = q.e;
          bv.traj_out[1 * st + o] = q.v;
          bv.traj_out[2 * st + o] = q.M;
          bv.traj_out[3 * st + o] = q.S;
          bv.traj_out[8 * st + o] = r[0];
        }
        if constexpr (kTdi) {
          const int64_t o = d.out_offset + i;
          const int64_t st = bv.phase_stride;
          bv.phase_out[kTdiE * st + o] = q.e;
          bv.phase_out[kTdiAmp * st + o] = pow(om * d.M_phys_sec, 2. / 3.) * d.zeta;
          bv.phase_out[kTdiGd * st + o] = r[0];
          bv.phase_out[kTdiAd * st + o] = r[2];
        }
      }
      sv_e[sl] = q.e;
      sv_om[sl] = kPhase ? r[2] : om * d.M_phys_sec;  // the phase product keeps alphadot here
      sv_gim[sl] = r[0];
      sv_Phi[sl] = r[1];
      sv_alp[sl] = r[2];
      sv_gd[sl] = r[0];
    }
    nonpos = __syncthreads_or(nonpos);
    // (B) the clamped Phidot (AAK.cc:254: the raw rate if positive, else the
    //     previous clamped value) where the clamp acts: one thread walks the
    //     tile and parks it in the nu slots
    if (nonpos) {
      if (tid == 0) {
        double P = Pin;
        for (int sl = 0; sl < lim - c.start; ++sl)
          if (c.start + sl >= d.i0) {
            const double raw = sv_Phi[sl];
            if (raw > 0.0) P = raw;
            sv_nu[sl] = P;
          }
      }
      __syncthreads();
    }
    // (C) AB2 increments of the thread's kSPT consecutive slots,
    //     their running sums, and one block scan of the thread totals
    constexpr int kSPT = kTileSamples / kTileThreads;
    const int j0 = kSPT * tid;
    double incF[kSPT][3], incB[kSPT][3], nuv[kSPT], Pl = 0.0;
    {
      double rm[3], Pm;  // rates and clamped Phidot of the slot before
      if (j0 == 0) {
        rm[0] = s_rb[0];
        rm[1] = s_rb[1];
        rm[2] = s_rb[2];
        Pm = Pin;
      } else {
        rm[0] = sv_gim[j0 - 1];
        rm[1] = sv_Phi[j0 - 1];
        rm[2] = sv_alp[j0 - 1];
        Pm = nonpos ? sv_nu[j0 - 1] : rm[1];
      }
      double rc[3] = {sv_gim[j0], sv_Phi[j0], sv_alp[j0]};
#pragma unroll
      for (int k = 0; k < kSPT; ++k) {
        const int i = c.start + j0 + k;
        const bool in = i < lim;
        const bool vf = in && i >= d.i0;
        const bool vb = in && i >= 1 && i <= d.i0;
        double rn[3];  // rates of the slot after (the tile's last slot: the sample after the tile)
        if (k + 1 < kSPT || j0 + kSPT < kTileSamples) {
          rn[0] = sv_gim[j0 + k + 1];
          rn[1] = sv_Phi[j0 + k + 1];
          rn[2] = sv_alp[j0 + k + 1];
        } else {
          rn[0] = s_ra[0];
          rn[1] = s_ra[1];
          rn[2] = s_ra[2];
        }
        const double P = (vf && nonpos) ? sv_nu[j0 + k] : rc[1];
        for (int qq = 0; qq < 3; ++qq) incF[k][qq] = incB[k][qq] = 0.0;
        if (vf) {
          if (i == d.i0) {
            incF[k][0] = rc[0] * d.dt;
            incF[k][1] = P * d.dt;
            incF[k][2] = rc[2] * d.dt;
          } else {
            incF[k][0] = (1.5 * rc[0] - .5 * rm[0]) * d.dt;
            incF[k][1] = (1.5 * P - .5 * Pm) * d.dt;
            incF[k][2] = (1.5 * rc[2] - .5 * rm[2]) * d.dt;
          }
          if (i == lim - 1) Pl = P;
        }
        if (vb) {
          if (i == d.i0) {
            incB[k][0] = rc[0] * d.dt;
            incB[k][1] = rc[1] * d.dt;
            incB[k][2] = rc[2] * d.dt;
          } else {
            incB[k][0] = (1.5 * rc[0] - .5 * rn[0]) * d.dt;
            incB[k][1] = (1.5 * rc[1] - .5 * rn[1]) * d.dt;
            incB[k][2] = (1.5 * rc[2] - .5 * rn[2]) * d.dt;
          }
        }
        // nu (the phase product: Phidot itself, clamped after i0 only,
        // as PNevolutionPhase records it, AAKPhase.cc:246-248, 266-270)
        nuv[k] = kPhase ? ((i > d.i0) ? P : rc[1]) : ((i > d.i0) ? P : rc[1]) / 2. / kPi;
        rm[0] = rc[0];
        rm[1] = rc[1];
        rm[2] = rc[2];
        Pm = P;
        rc[0] = rn[0];
        rc[1] = rn[1];
        rc[2] = rn[2];
      }
      // the owner of the tile's last output sample records its clamped Phidot (forward samples)
      if (lim - 1 >= d.i0 && lim - 1 >= c.start + j0 && lim - 1 < c.start + j0 + kSPT) s_lastP = Pl;
    }
    double tF[3] = {0, 0, 0}, tB[3] = {0, 0, 0};
#pragma unroll
    for (int k = 0; k < kSPT; ++k)
#pragma unroll
      for (int qq = 0; qq < 3; ++qq) {
        tF[qq] += incF[k][qq];
        tB[qq] += incB[k][qq];
      }
    double runF[3], runB[3] = {0.0, 0.0, 0.0}, eF[3], eB[3] = {0.0, 0.0, 0.0};
    // (the backward scan only where the tile has a backward region; its
    // barrier orders every read of (C) before the writes of (D))
    block_exscan3x2(tF, tB, d.i0 > 0 && c.start <= d.i0, red, eF, runF, eB, runB);
    // (D) tile-local phases: forward, the increments of the tile's samples
    //     before i; backward, those of its samples up to i; the chain's carry
    //     is added after the look-back
#pragma unroll
    for (int k = 0; k < kSPT; ++k) {
      const int sl = j0 + k;
      const int i = c.start + sl;
      if (i >= lim) break;
      double *const svq[3] = {sv_gim, sv_Phi, sv_alp};
#pragma unroll
      for (int qq = 0; qq < 3; ++qq) {
        double x;
        if (i > d.i0) x = eF[qq];
        else if (i == d.i0) x = X0[qq];
        else x = eB[qq] + incB[k][qq];
        svq[qq][sl] = x;
        eF[qq] += incF[k][qq];
        eB[qq] += incB[k][qq];
      }
      sv_nu[sl] = nuv[k];
      if (bv.traj_out) bv.traj_out[7 * bv.traj_stride + d.out_offset + i] = nuv[k];
    }
    __syncthreads();
    if (tid == 32) s_tile = (long long)atomicAdd(bv.work_counter, 1ull);  // the next tile, read after the loop's barrier
    // ---------------- chain carries: warp 0 publishes this tile's aggregate,
    // looks back for the exclusive prefix and publishes the inclusive record
    if (tid < 32) {
      const bool hasF = lim - 1 >= max(c.start, d.i0);  // forward output samples in the tile
      double hi[3] = {0, 0, 0}, lo[3] = {0, 0, 0}, C = 0.0;
      if (needC) {
        for (int q = 0; q < 3; ++q) {
          hi[q] = s_cy[q];
          lo[q] = s_cy[3 + q];
        }
        C = s_cy[6];
      } else if (dir != 0) {
        const TileAgg agg{{(dir > 0) ? runF[0] : runB[0], (dir > 0) ? runF[1] : runB[1], (dir > 0) ? runF[2] : runB[2]},
                          hasF ? s_lastP : 0.0, hasF, true};
        look_back_warp(bv, c, dir, hi, lo, C, agg);
      }
      if (tid == 0) {
        double fh[3] = {0, 0, 0}, fl[3] = {0, 0, 0}, bh[3] = {0, 0, 0}, bl[3] = {0, 0, 0};
        for (int q = 0; q < 3; ++q) {
          s_cy[q] = hi[q];
          s_cy[3 + q] = lo[q];
          if (dir >= 0) {
            fh[q] = hi[q];
            fl[q] = lo[q];
            dd_add(fh[q], fl[q], runF[q]);
          }
          if (dir <= 0) {
            bh[q] = hi[q];
            bl[q] = lo[q];
            dd_add(bh[q], bl[q], runB[q]);
          }
        }
        publish_inclusive(bv, g, fh, fl, bh, bl, hasF ? s_lastP : C);
      }
    }
#if AAK_TABLE_AFTER_SCAN
    // Taylor table rows (one thread of warps 1-7 per harmonic) while warp 0 looks back
    else if (!kPhase && !kPre && K > 0 && !bv.trajectory_only)
      for (int n = tid - 31; n <= (kSplit ? table_rows<float>(d.nmodes) : d.nmodes); n += kTileThreads - 32) {
        const int st = (n <= d.nmodes) ? bstart[n - 1] : 0;
        if (kSplit) build_taylor_row<float>(tabF, 2 * kRowF, n, d.nmodes, ec, K, st);
        else build_taylor_row<double>(tabD, kRowD, n, d.nmodes, ec, K, st);
      }
#endif
    __syncthreads();
    // the phases of this thread's own samples: X0 + carry + local part
    // (forward), X0 - (carry + increments after the sample) (backward)
    {
      const double cy_hi[3] = {s_cy[0], s_cy[1], s_cy[2]}, cy_lo[3] = {s_cy[3], s_cy[4], s_cy[5]};
      for (int ch = 0; ch < kTileChunks; ++ch) {
        const int i = c.start + ch * kTileThreads + tid;
        const int sl = ch * kTileThreads + tid;
        if (i >= lim) break;
        double X[3];
#pragma unroll
        for (int qq = 0; qq < 3; ++qq) {
          double *sv = s_dyn + (2 + qq) * kTileSamples;
          const double v = sv[sl];
          if (i > d.i0) X[qq] = X0[qq] + (cy_hi[qq] + (cy_lo[qq] + v));
          else if (i == d.i0) X[qq] = v;
          else X[qq] = X0[qq] - (cy_hi[qq] + (cy_lo[qq] + (runB[qq] - v)));
          sv[sl] = X[qq];
        }
        if (bv.traj_out) {
          const int64_t o = d.out_offset + i;
          const int64_t st = bv.traj_stride;
          bv.traj_out[4 * st + o] = X[0];
          bv.traj_out[5 * st + o] = X[1];
          bv.traj_out[6 * st + o] = X[2];
        }
        if constexpr (kTdi) {
          const int64_t o = d.out_offset + i;
          const int64_t st = bv.phase_stride;
          bv.phase_out[kTdiT * st + o] = sample_time(d, i);
          bv.phase_out[kTdiGim * st + o] = X[0];
          bv.phase_out[kTdiPhi * st + o] = X[1];
          bv.phase_out[kTdiAlp * st + o] = X[2];
          bv.phase_out[kTdiNu * st + o] = sv_nu[sl] / 2. / kPi;  // nuvec = Phidot / 2 / pi
          bv.phase_out[kTdiPd * st + o] = sv_nu[sl];
        } else if constexpr (kPhase) {
          // GenPhase's packing, sums in its order (AAKPhase.cc:347-354)
          const int64_t o = d.out_offset + i;
          const int64_t st = bv.phase_stride;
          const double Pd = sv_nu[sl], gd = sv_gd[sl], ad = sv_om[sl];
          bv.phase_out[o] = sample_time(d, i);
          bv.phase_out[st + o] = X[1];
          bv.phase_out[2 * st + o] = X[1] + X[0];
          bv.phase_out[3 * st + o] = X[1] + X[0] + X[2];
          bv.phase_out[4 * st + o] = Pd;
          bv.phase_out[5 * st + o] = Pd + gd;
          bv.phase_out[6 * st + o] = Pd + gd + ad;
          bv.phase_out[7 * st + o] = sv_e[sl];
        }
      }
    }
    // ---------------- phase 2: harmonic sums of this thread's own samples,
    // kJoint of them at a time (shared table loads, independent recurrences)
    if (kPhase || bv.trajectory_only) continue;
    if constexpr (kPre) {
      if (s_win[3]) {  // the tile's table (uniform)
        const bool ok = mbar_wait_bounded(&s_mbar[1], ph1);
        ph1 ^= 1u;
        if (__syncthreads_or(!ok)) {
          if (tid == 0) {
            atomicExch(bv.device_status, 1u);
            if (bv.status_report) atomicExch(bv.status_report, 1u);
          }
          return;
        }
      }
    }
    const double t_plunge = sample_time(d, d.i_plunge);
    const double t_zero = t_plunge + d.dt * d.i_buffer;
    using T = typename std::conditional<kSplit, float, double>::type;
    constexpr int kJoint = kJointT > 0 ? kJointT : (kSplit ? AAK_JOINT_SPLIT : AAK_JOINT_FP64);
    static_assert(kTileChunks % kJoint == 0, "joint samples must divide the chunks");
    const T *tab = kSplit ? reinterpret_cast<const T *>(tabF) : reinterpret_cast<const T *>(tabD);
    const int rs = kPre ? (int)s_prep.stride : (kSplit ? 2 * kRowF : kRowD);  // table row (FP32: pair row) stride
#pragma unroll 1
    for (int g0 = 0; g0 < kTileChunks; g0 += kJoint) {
      SamplePrep<T> P[kJoint];
      T dl[kJoint], c1[kJoint], s1[kJoint], cD[kJoint], sD[kJoint], Sa[kJoint], Sb[kJoint], Sc[kJoint], d0[kJoint];
      double ph[kJoint];
#pragma unroll
      for (int m = 0; m < kJoint; ++m) {
        const int i = c.start + (g0 + m) * kTileThreads + tid;
        const int sl = (g0 + m) * kTileThreads + tid;
        if (i < c.end && i < c.neff) {
          if constexpr (kSplit)
            P[m] = prep_split(d, s_geom, ec, sample_time(d, i), sv_e[sl], sv_om[sl], sv_gim[sl], sv_Phi[sl], sv_alp[sl],
                              sv_nu[sl], sv_gd[sl]);
          else
            P[m] = prep_fp64(d, s_geom, ec, sample_time(d, i), sv_e[sl], sv_om[sl], sv_gim[sl], sv_Phi[sl], sv_alp[sl],
                             sv_nu[sl], sv_gd[sl]);
        } else {
          P[m] = SamplePrep<T>{};
          P[m].c1 = P[m].cD = T(1);
        }
        dl[m] = P[m].dl;
        ph[m] = P[m].ph;
        d0[m] = P[m].d0;
        c1[m] = P[m].c1;
        s1[m] = P[m].s1;
        cD[m] = P[m].cD;
        sD[m] = P[m].sD;
      }
      if constexpr (kSplit) {
        switch (K) {
          case 2: mode_sums_split<2, kJoint>(tab, d.nmodes, rs, dl, c1, s1, cD, sD, ph, d0, Sa, Sb, Sc); break;
          case 3: mode_sums_split<3, kJoint>(tab, d.nmodes, rs, dl, c1, s1, cD, sD, ph, d0, Sa, Sb, Sc); break;
          case 4: mode_sums_split<4, kJoint>(tab, d.nmodes, rs, dl, c1, s1, cD, sD, ph, d0, Sa, Sb, Sc); break;
          case 6: mode_sums_split<6, kJoint>(tab, d.nmodes, rs, dl, c1, s1, cD, sD, ph, d0, Sa, Sb, Sc); break;
          default: break;
        }
      } else {
        switch (K) {
          case 4: mode_sums_fp64<4, kJoint>(tab, d.nmodes, rs, dl, c1, s1, cD, sD, Sa, Sb, Sc); break;
          case 5: mode_sums_fp64<5, kJoint>(tab, d.nmodes, rs, dl, c1, s1, cD, sD, Sa, Sb, Sc); break;
          case 6: mode_sums_fp64<6, kJoint>(tab, d.nmodes, rs, dl, c1, s1, cD, sD, Sa, Sb, Sc); break;
          case 8: mode_sums_fp64<8, kJoint>(tab, d.nmodes, rs, dl, c1, s1, cD, sD, Sa, Sb, Sc); break;
          case 10: mode_sums_fp64<10, kJoint>(tab, d.nmodes, rs, dl, c1, s1, cD, sD, Sa, Sb, Sc); break;
          default: break;
        }
      }
#pragma unroll
      for (int m = 0; m < kJoint; ++m) {
        const int i = c.start + (g0 + m) * kTileThreads + tid;
        const int sl = (g0 + m) * kTileThreads + tid;
        if (i >= c.end) continue;
        const double t = sample_time(d, i);
        double hI = 0.0, hII = 0.0;
        if (i < c.neff) {
          if (K == 0) {  // no table for this tile: per-sample Miller recurrence in FP64
            double a64, b64, c64;
            mode_sums_miller(bstart, d.nmodes, sv_e[sl], (double)c1[m], (double)s1[m], (double)cD[m], (double)sD[m],
                             a64, b64, c64);
            Sa[m] = (T)a64;
            Sb[m] = (T)b64;
            Sc[m] = (T)c64;
          }
          finish<T>(P[m], Sa[m], Sb[m], Sc[m], hI, hII);
          if (i > d.i_plunge) {
            const double wgt = exp((t_plunge - t_zero) / (t - t_plunge) + (t_plunge - t_zero) / (t - t_zero)) + 1.;
            hI = hI / wgt;
            hII = hII / wgt;
          }
        }
        store_h(bv, d.out_offset + i, hI, hII);
        if (bv.t_out) bv.t_out[d.out_offset + i] = t;
      }
    }
  }
}

// ------------------------------------------------------------------ plain FP64 per-source path
// One thread per sample, everything per harmonic, as the reference's CUDA
// port evaluates it (src/cuda/kernel.cu:374-555); the response, orientation
// and taper conventions are those of the FP64 path above, so the two agree.
__global__ void __launch_bounds__(256) k_plain_waveform(const SourceDesc *__restrict__ src, int s,
                                                        const double *__restrict__ traj, int64_t st,
                                                        double *__restrict__ hI_out, double *__restrict__ hII_out) {
  const SourceDesc &d = src[s];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.vlength) return;
  const int64_t o = d.out_offset + i;
  const double t = sample_time(d, i);
  if (i >= n_eff(d)) {
    hI_out[o] = 0.0;
    hII_out[o] = 0.0;
    return;
  }
  const double e = traj[o], gim = traj[4 * st + o], Phi = traj[5 * st + o], alp = traj[6 * st + o];
  const double nu = traj[7 * st + o], gimdot = traj[8 * st + o];
  const double om_M = omega_phi(traj[st + o], e, d.coslam, traj[3 * st + o], traj[2 * st + o]) * d.M_phys_sec;

  const double cosalp = cos(alp), sinalp = sin(alp);
  const double cosqL = d.cosqK * d.coslam + d.sinqK * d.sinlam * cosalp;
  const double sinqL = sqrt(1. - cosqL * cosqL);
  const double phiLup = d.sinqK * d.sinphiK * d.coslam - d.cosphiK * d.sinlam * sinalp - d.cosqK * d.sinphiK * d.sinlam * cosalp;
  const double phiLdown = d.sinqK * d.cosphiK * d.coslam + d.sinphiK * d.sinlam * sinalp - d.cosqK * d.cosphiK * d.sinlam * cosalp;
  const double Ldotn = cosqL * d.cosqS + sinqL * d.sinqS * cos(atan2(phiLup, phiLdown) - d.phiS);
  const double Ldotn2 = Ldotn * Ldotn;
  const double Sdotn = d.cosqK * d.cosqS + d.sinqK * d.sinqS * cos(d.phiK - d.phiS);
  const double beta = atan2(-Sdotn + d.coslam * Ldotn,
                            d.sinqS * sin(d.phiK - d.phiS) * d.sinlam * cosalp + (d.cosqK * Sdotn - d.cosqS) / d.sinqK * d.sinlam * sinalp);
  const double cos2gam = cos(2. * (gim + beta)), sin2gam = sin(2. * (gim + beta));

  double cosorbphs = 0.0, FplusI, FcrosI, FplusII, FcrosII, Kresp;
  if (d.mich) {
    const double orbphs = kTwoPi * t / kYear;
    cosorbphs = cos(orbphs - d.phiS);
    const double sinorbphs = sin(orbphs - d.phiS);
    const double cosq = .5 * d.cosqS - kHalfSqrt3 * d.sinqS * cosorbphs;
    const double phiw = orbphs + atan2(kHalfSqrt3 * d.cosqS + .5 * d.sinqS * cosorbphs, d.sinqS * sinorbphs);
    const double psiup = .5 * d.cosqK - kHalfSqrt3 * d.sinqK * cos(orbphs - d.phiK) - cosq * Sdotn;
    const double psidown = .5 * d.sinqK * d.sinqS * sin(d.phiK - d.phiS) -
                           kHalfSqrt3 * cos(orbphs) * (d.cosqK * d.sinqS * sin(d.phiS) - d.cosqS * d.sinqK * sin(d.phiK)) -
                           kHalfSqrt3 * sin(orbphs) * (d.cosqS * d.sinqK * cos(d.phiK) - d.cosqK * d.sinqS * cos(d.phiS));
    const double psi = atan2(psiup, psidown);
    const double cosq1 = .5 * (1. + cosq * cosq);
    const double cos2phi = cos(2. * phiw), sin2phi = sin(2. * phiw), cos2psi = cos(2. * psi), sin2psi = sin(2. * psi);
    FplusI = cosq1 * cos2phi * cos2psi - cosq * sin2phi * sin2psi;
    FcrosI = cosq1 * cos2phi * sin2psi + cosq * sin2phi * cos2psi;
    FplusII = cosq1 * sin2phi * cos2psi + cosq * cos2phi * sin2psi;
    FcrosII = cosq1 * sin2phi * sin2psi - cosq * cos2phi * cos2psi;
    Kresp = kHalfSqrt3;
  } else {
    const double up_ldc = d.cosqS * d.sinqK * cos(d.phiS - d.phiK) - d.cosqK * d.sinqS;
    const double dw_ldc = d.sinqK * sin(d.phiS - d.phiK);
    const double psi_ldc = (dw_ldc != 0.0) ? -atan2(up_ldc, dw_ldc) : 0.5 * kPi;
    FplusI = cos(2. * psi_ldc);
    FcrosI = -sin(2. * psi_ldc);
    FplusII = sin(2. * psi_ldc);
    FcrosII = cos(2. * psi_ldc);
    Kresp = 1.0;
  }
  const double Amp = pow(om_M, 2. / 3.) * d.zeta;
  const double se = sqrt(1. - e * e);
  double hI = 0.0, hII = 0.0;
  for (int n = 1; n <= d.nmodes; ++n) {
    double nPhi = n * Phi;
    if (d.mich) nPhi += kTwoPi * (n * nu + gimdot / kPi) * kAUsec * d.sinqS * cosorbphs;
    const double ne = n * e;
    double J[5];
    if (n == 1) {
      J[0] = -j1(ne);
      J[1] = j0(ne);
      J[2] = j1(ne);
      J[3] = jn(2, ne);
      J[4] = jn(3, ne);
    } else {
      for (int k = 0; k < 5; ++k) J[k] = jn(n - 2 + k, ne);
    }
    const double cn = cos(nPhi), sn = sin(nPhi);
    const double a = -n * Amp * (J[0] - 2. * e * J[1] + 2. / n * J[2] + 2. * e * J[3] - J[4]) * cn;
    const double b = -n * Amp * se * (J[0] - 2. * J[2] + J[4]) * sn;
    const double c = 2. * Amp * J[2] * cn;
    const double Aplus = -(1. + Ldotn2) * (a * cos2gam - b * sin2gam) + c * (1. - Ldotn2);
    const double Acros = 2. * Ldotn * (b * cos2gam + a * sin2gam);
    // rotation to the NK wave frame, per harmonic as in the port
    const double n0 = d.sinqS * cos(d.phiS), n1 = d.sinqS * sin(d.phiS), n2 = d.cosqS;
    const double S0 = d.sinqK * d.cosphiK, S1 = d.sinqK * d.sinphiK, S2 = d.cosqK;
    const double L0 = d.coslam * d.sinqK * d.cosphiK + d.sinlam * (sinalp * d.sinphiK - cosalp * d.cosqK * d.cosphiK);
    const double L1 = d.coslam * d.sinqK * d.sinphiK - d.sinlam * (sinalp * d.cosphiK + cosalp * d.cosqK * d.sinphiK);
    const double L2 = d.coslam * d.cosqK + d.sinlam * cosalp * d.sinqK;
    const double nL0 = n1 * L2 - n2 * L1, nL1 = n2 * L0 - n0 * L2, nL2 = n0 * L1 - n1 * L0;
    const double nS0 = n1 * S2 - n2 * S1, nS1 = n2 * S0 - n0 * S2, nS2 = n0 * S1 - n1 * S0;
    const double norm = sqrt(nL0 * nL0 + nL1 * nL1 + nL2 * nL2) * sqrt(nS0 * nS0 + nS1 * nS1 + nS2 * nS2);
    const double cosrot = (nL0 * nS0 + nL1 * nS1 + nL2 * nS2) / norm;
    const double sinrot = ((L0 * nS0 + L1 * nS1 + L2 * nS2) - (S0 * nL0 + S1 * nL1 + S2 * nL2)) / norm;
    const double r0 = 2. * cosrot * cosrot - 1., r1 = cosrot * sinrot;
    const double Ap = Aplus * r0 + Acros * r1, Ac = -Aplus * r1 + Acros * r0;
    hI += Kresp * (FplusI * Ap + FcrosI * Ac);
    hII += Kresp * (FplusII * Ap + FcrosII * Ac);
  }
  if (i > d.i_plunge) {
    const double t_plunge = sample_time(d, d.i_plunge);
    const double t_zero = t_plunge + d.dt * d.i_buffer;
    const double wgt = exp((t_plunge - t_zero) / (t - t_plunge) + (t_plunge - t_zero) / (t - t_zero)) + 1.;
    hI /= wgt;
    hII /= wgt;
  }
  hI_out[o] = hI;
  hII_out[o] = hII;
}

}  // namespace

namespace {
__global__ void __launch_bounds__(128) k_spline_coeffs(const SourceDesc *src, int nsrc, const int64_t *blk_start,
                                                       int64_t total_blocks, const double *knot_t,
                                                       const double4 *knot_y, double4 *knot_c) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= total_blocks) return;
  const int s = find_source(blk_start, nsrc, g);
  const SourceDesc &d = src[s];
  if (d.status != 0) return;  // a failed source has no knots
  const int n = d.n_knots;
  const double *x = knot_t + d.knot_offset;
  const double4 *y = knot_y + d.knot_offset;
  double4 *c = knot_c + d.knot_offset;
  const double4 zero = make_double4(0.0, 0.0, 0.0, 0.0);
  if (n < 3) {
    for (int i = 0; i < n; ++i) c[i] = zero;
    return;
  }
  // interior unknowns 1 .. n-2; this block owns [a, e), the widened window is [wa, wb)
  const int b = (int)(g - blk_start[s]);
  const int a = 1 + b * kSplineBlock, e = min(a + kSplineBlock, n - 1);
  if (a == 1) c[0] = zero;
  if (e == n - 1) c[n - 1] = zero;
  const int wa = max(1, a - kSplineHalo), wb = min(n - 1, e + kSplineHalo);
  double cp[kSplineBlock + kSplineHalo];
  double4 dp[kSplineBlock + kSplineHalo];
  double cprev = 0.0;
  double4 dprev = zero;
  double inv_h0 = 1.0 / (x[wa] - x[wa - 1]);
  for (int i = wa; i < wb; ++i) {
    const double h0 = x[i] - x[i - 1], h1 = x[i + 1] - x[i];
    const double inv_h1 = 1.0 / h1;
    const double inv = 1.0 / (2.0 * (h0 + h1) - h0 * cprev);
    const double cc = (i + 1 < wb) ? h1 * inv : 0.0;
    const double4 y0 = y[i - 1], y1 = y[i], y2 = y[i + 1];
    double4 dd;
    dd.x = (3.0 * ((y2.x - y1.x) * inv_h1 - (y1.x - y0.x) * inv_h0) - h0 * dprev.x) * inv;
    dd.y = (3.0 * ((y2.y - y1.y) * inv_h1 - (y1.y - y0.y) * inv_h0) - h0 * dprev.y) * inv;
    dd.z = (3.0 * ((y2.z - y1.z) * inv_h1 - (y1.z - y0.z) * inv_h0) - h0 * dprev.z) * inv;
    dd.w = (3.0 * ((y2.w - y1.w) * inv_h1 - (y1.w - y0.w) * inv_h0) - h0 * dprev.w) * inv;
    if (i >= a) {
      cp[i - a] = cc;
      dp[i - a] = dd;
    }
    cprev = cc;
    dprev = dd;
    inv_h0 = inv_h1;
  }
  double4 v = dp[wb - 1 - a];  // c at wb - 1 (its neighbour beyond the window taken as 0)
  if (wb - 1 < e) c[wb - 1] = v;
  for (int i = wb - 2; i >= a; --i) {
    const double k = cp[i - a];
    const double4 q = dp[i - a];
    v = make_double4(q.x - k * v.x, q.y - k * v.y, q.z - k * v.z, q.w - k * v.w);
    if (i < e) c[i] = v;
  }
}
}  // namespace

void launch_spline_coeffs(const SourceDesc *src, int nsrc, const int64_t *blk_start, int64_t total_blocks,
                          const double *knot_t, const double4 *knot_y, double4 *knot_c, cudaStream_t stream) {
  if (total_blocks <= 0) return;
  const int threads = 128;
  k_spline_coeffs<<<(unsigned)((total_blocks + threads - 1) / threads), threads, 0, stream>>>(
      src, nsrc, blk_start, total_blocks, knot_t, knot_y, knot_c);
}

void launch_plain_waveform(const SourceDesc *src, int s, int vlength, const double *traj, int64_t traj_stride,
                           double *hI, double *hII, cudaStream_t stream) {
  if (vlength <= 0) return;
  k_plain_waveform<<<(vlength + 255) / 256, 256, 0, stream>>>(src, s, traj, traj_stride, hI, hII);
}

void launch_dense_fp64(const BatchView &bv, int num_sms, cudaStream_t stream, cudaEvent_t *ev) {
  launch_dense(bv, num_sms, stream, ev, 0);
}

template <bool kSplit, size_t... I>
void set_variant_smem(int bytes, std::index_sequence<I...>) {
  (cudaFuncSetAttribute(k_waveform<kSplit, 0, wave_variant(kSplit, (int)I).pre, wave_variant(kSplit, (int)I).joint,
                                   wave_variant(kSplit, (int)I).min_blocks>,
                        cudaFuncAttributeMaxDynamicSharedMemorySize, bytes),
   ...);
}

void prepare_dense_launch() {
  static std::atomic<unsigned long long> attrs_set{0};  // opt in to > 48 KB of shared memory once per device
  int dev = 0;
  cudaGetDevice(&dev);
  const unsigned long long bit = 1ull << (dev & 63);
  if (!(attrs_set.load() & bit)) {
    const int most = (int)(kWaveDynSmem + (size_t)kTabModes * kRowD * sizeof(double));
    cudaFuncSetAttribute(k_waveform<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, most);
    cudaFuncSetAttribute(k_waveform<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, most);
    set_variant_smem<true>(most, std::make_index_sequence<kNumVariants>{});
    set_variant_smem<false>(most, std::make_index_sequence<kNumVariants>{});
    cudaFuncSetAttribute(k_waveform<false, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kWaveDynSmem);
    cudaFuncSetAttribute(k_waveform<false, 1, true, 0, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)kWaveDynSmem);
    cudaFuncSetAttribute(k_waveform<false, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kWaveDynSmem);
    attrs_set.fetch_or(bit);
  }
}

// Launch one waveform-kernel instantiation as a persistent grid: every CTA
// that fits on the device at once.
template <typename K>
void launch_persistent(K kernel, const BatchView &bv, int num_sms, size_t dyn, cudaStream_t stream) {
  int resident = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident, kernel, kTileThreads, dyn);
  resident = std::max(resident, 1);
  const int grid = (int)std::min<int64_t>(bv.total_tiles, (int64_t)num_sms * resident);
  kernel<<<grid, kTileThreads, dyn, stream>>>(bv);
}

template <bool kSplit, int v>
void launch_variant(const BatchView &bv, int num_sms, size_t dyn, cudaStream_t stream) {
  constexpr WaveVariant w = wave_variant(kSplit, v);
  launch_persistent(k_waveform<kSplit, 0, w.pre, w.joint, w.min_blocks>, bv, num_sms, dyn, stream);
}

template <bool kSplit, size_t... I>
void launch_variant_index(int v, const BatchView &bv, int num_sms, size_t dyn, cudaStream_t stream,
                          std::index_sequence<I...>) {
  ((v == (int)I ? launch_variant<kSplit, (int)I>(bv, num_sms, dyn, stream) : void()), ...);
}

template <bool kSplit>
void launch_dense_t(const BatchView &bv, int num_sms, cudaStream_t stream, cudaEvent_t *ev) {
  if (ev) cudaEventRecord(ev[0], stream);
  cudaMemsetAsync(bv.work_counter, 0, sizeof(unsigned long long), stream);
  cudaMemsetAsync(bv.link_flag, 0, (size_t)bv.total_tiles * sizeof(int32_t), stream);
  if (ev) cudaEventRecord(ev[1], stream);
  // per-sample values, then the Taylor table sized for the batch's harmonic count
  const int rows = table_rows<typename std::conditional<kSplit, float, double>::type>(
      (bv.max_nmodes > 0 && bv.max_nmodes < kTabModes) ? bv.max_nmodes : kTabModes);
  const size_t dyn = kWaveDynSmem + (size_t)rows * (kSplit ? kRowF * sizeof(float) : kRowD * sizeof(double));
  const int v = (bv.variant >= 0 && bv.variant < kNumVariants) ? bv.variant : 0;
  const bool pre = wave_variant(kSplit, v).pre && bv.tile_prep && bv.tile_tab && bv.queue && !bv.trajectory_only &&
                   bv.tab_slot >= tile_table_slot_bytes(rows, kSplit);
  prepare_dense_launch();
  if (pre) {
    const int64_t tiles = bv.total_tiles;
    k_tile_params<kSplit><<<(unsigned)((tiles + 127) / 128), 128, 0, stream>>>(bv);
    k_tile_table<kSplit><<<(unsigned)((tiles * rows + 127) / 128), 128, 0, stream>>>(bv, rows);
  }
  if (ev) cudaEventRecord(ev[2], stream);
  if (pre) launch_variant_index<kSplit>(v, bv, num_sms, dyn, stream, std::make_index_sequence<kNumVariants>{});
  else launch_persistent(k_waveform<kSplit>, bv, num_sms, dyn, stream);
  if (ev) cudaEventRecord(ev[3], stream);
}

void launch_dense(const BatchView &bv, int num_sms, cudaStream_t stream, cudaEvent_t *ev, int precision) {
  if (bv.total_tiles <= 0) return;
  if (precision == 1) launch_dense_t<true>(bv, num_sms, stream, ev);
  else launch_dense_t<false>(bv, num_sms, stream, ev);
}

// The phases of the samples after the plunge buffer hold their values at
// i_plunge: GenPhase's evolution sets gim/Phi/alp[i+1] to their values at
// i_plunge for every forward step i > i_plunge + i_buffer (AAKPhase.cc:253-257),
// i.e. the samples from max(i_plunge + i_buffer + 2, i0 + 1) on.  Rows 1-3 of
// phase_out are sums of those three phases, so they take their own values at
// i_plunge.  y strides over sources, x over each source's frozen samples.
__global__ void __launch_bounds__(256) k_phase_freeze(const SourceDesc *__restrict__ src, int nsrc,
                                                      double *__restrict__ out, int64_t st) {
  for (int s = blockIdx.y; s < nsrc; s += gridDim.y) {
    const SourceDesc &d = src[s];
    if (d.status != 0 || d.i_plunge < 0 || d.i_plunge >= d.vlength) continue;
    const long long first = max((long long)d.i_plunge + (long long)d.i_buffer + 2, (long long)d.i0 + 1);
    if (first >= d.vlength) continue;
    const int64_t o = d.out_offset;
    const double pr = out[st + o + d.i_plunge], pt = out[2 * st + o + d.i_plunge];
    const double pp = out[3 * st + o + d.i_plunge];
    for (long long i = first + (long long)blockIdx.x * blockDim.x + threadIdx.x; i < d.vlength;
         i += (long long)gridDim.x * blockDim.x) {
      out[st + o + i] = pr;
      out[2 * st + o + i] = pt;
      out[3 * st + o + i] = pp;
    }
  }
}

void launch_phase(const BatchView &bv, int num_sms, cudaStream_t stream, cudaEvent_t *ev) {
  if (bv.total_tiles <= 0 || !bv.phase_out) return;
  if (ev) cudaEventRecord(ev[0], stream);
  cudaMemsetAsync(bv.work_counter, 0, sizeof(unsigned long long), stream);
  cudaMemsetAsync(bv.link_flag, 0, (size_t)bv.total_tiles * sizeof(int32_t), stream);
  if (ev) {
    cudaEventRecord(ev[1], stream);
    cudaEventRecord(ev[2], stream);
  }
  prepare_dense_launch();
  if (bv.tile_prep) {
    // the tile parameters from the pre-pass, each tile's inputs staged by bulk copies
    k_tile_params<false><<<(unsigned)((bv.total_tiles + 127) / 128), 128, 0, stream>>>(bv);
    launch_persistent(k_waveform<false, 1, true, 0, 3>, bv, num_sms, kWaveDynSmem, stream);
  } else {
    launch_persistent(k_waveform<false, 1>, bv, num_sms, kWaveDynSmem, stream);
  }
  const dim3 fgrid(64, (unsigned)std::min(std::max(bv.nsrc, 1), 1024));
  k_phase_freeze<<<fgrid, 256, 0, stream>>>(bv.src, bv.nsrc, bv.phase_out, bv.phase_stride);
  if (ev) cudaEventRecord(ev[3], stream);
}

void launch_tdi_grid(const BatchView &bv, int num_sms, cudaStream_t stream, cudaEvent_t *ev) {
  if (bv.total_tiles <= 0 || !bv.phase_out) return;
  if (ev) cudaEventRecord(ev[0], stream);
  cudaMemsetAsync(bv.work_counter, 0, sizeof(unsigned long long), stream);
  cudaMemsetAsync(bv.link_flag, 0, (size_t)bv.total_tiles * sizeof(int32_t), stream);
  if (ev) {
    cudaEventRecord(ev[1], stream);
    cudaEventRecord(ev[2], stream);
  }
  prepare_dense_launch();
  int resident = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident, k_waveform<false, 2>, kTileThreads, kWaveDynSmem);
  resident = std::max(resident, 1);
  const int grid = (int)std::min<int64_t>(bv.total_tiles, (int64_t)num_sms * resident);
  k_waveform<false, 2><<<grid, kTileThreads, kWaveDynSmem, stream>>>(bv);
  if (ev) cudaEventRecord(ev[3], stream);
}

// ------------------------------------------------------------------ stationary-phase TDI
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 cscale(double r, double2 a) { return make_double2(r * a.x, r * a.y); }
// exp(-i x)
__device__ __forceinline__ double2 cexpm(double x) {
  double sx, cx;
  sincos(x, &sx, &cx);
  return make_double2(cx, -sx);
}
// normalised sinc, sin(pi x) / (pi x)
__device__ __forceinline__ double sinc_pi(double x) { return x == 0.0 ? 1.0 : sinpi(x) / (kPi * x); }

// TDI transfer functions of one harmonic of angular frequency om at time t
// (AAKTDI.cc:345-392, the LISA constellation of KSParMap.cc:576-596 with
// kappa0 = lambda0 = 0): F[0..5] = Xp, Xc, Yp, Yc, Zp, Zc.
__device__ void tdi_transfer(const TdiDesc &d, double t, double om, double2 F[6]) {
  const double alpha = 2. * kPi * 3.1709791983764586e-8 * t;
  double sa, ca;
  sincos(alpha, &sa, &ca);
  double q[3][3], n[3][3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const double xi = i * 2.0 * kPi / 3.0;
    double sx, cx;
    sincos(xi, &sx, &cx);
    q[i][0] = (sa * ca * sx - (1. + sa * sa) * cx) / (2.0 * sqrt(3.));
    q[i][1] = (sa * ca * cx - (1. + ca * ca) * sx) / (2.0 * sqrt(3.));
    q[i][2] = -0.5 * cos(alpha - xi);
  }
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    n[0][i] = q[1][i] - q[2][i];
    n[1][i] = q[2][i] - q[0][i];
    n[2][i] = q[0][i] - q[1][i];
  }
  double kn[3], kq[3], u[3], v[3];
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    double a = 0, b = 0, nU = 0, nV = 0;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      a += d.k[i] * n[j][i];
      b += d.k[i] * q[j][i];
      nU += d.uhat[i] * n[j][i];
      nV += d.vhat[i] * n[j][i];
    }
    kn[j] = a;
    kq[j] = b;
    u[j] = 0.5 * (nU * nU - nV * nV);
    v[j] = nU * nV;
  }
  const double x = om * d.arm, x2 = 0.5 * x, xs = x * sin(x);
  const double2 emx = cexpm(x);
  // link a: its two chi forms; the phase uses the kq of the other two spacecraft
  double2 chim[3], chip[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const int p0 = (a == 0) ? 2 : (a == 1) ? 0 : 1, p1 = (a == 0) ? 1 : (a == 1) ? 2 : 0;
    const double2 ph = cexpm(x2 * (3.0 + kq[p0] + kq[p1]));
    const double s1 = sinc_pi(x2 * (1. - kn[a])), s2 = sinc_pi(x2 * (1. + kn[a]));
    chim[a] = cmul(cscale(-xs, cadd(cscale(s1, emx), make_double2(s2, 0.0))), ph);
    chip[a] = cmul(cscale(xs, cadd(make_double2(s1, 0.0), cscale(s2, emx))), ph);
  }
  // X: link 1 (first form) and 2 (second); Y: 2 and 0; Z: 0 and 1
#pragma unroll
  for (int ch = 0; ch < 3; ++ch) {
    const int a = (ch == 0) ? 1 : (ch == 1) ? 2 : 0, b = (ch == 0) ? 2 : (ch == 1) ? 0 : 1;
    F[2 * ch] = cadd(cscale(u[a] * d.c2psi - v[a] * d.s2psi, chim[a]), cscale(u[b] * d.c2psi - v[b] * d.s2psi, chip[b]));
    F[2 * ch + 1] =
        cadd(cscale(v[a] * d.c2psi + u[a] * d.s2psi, chim[a]), cscale(v[b] * d.c2psi + u[b] * d.s2psi, chip[b]));
  }
}

// Second derivative at grid point idx as PNevolutionTDI leaves it: forward
// differences after i0 (the last point repeats the one before), backward ones
// at and before i0, point 0 repeating point 1 (AAKTDI.cc:334-343, 407-416).
__device__ __forceinline__ double tdi_ddot(const double *row, int64_t base, int idx, int i0, int ip, double scale,
                                           double dt) {
  if (idx == 0) idx = 1;
  if (idx <= i0) return scale * (row[base + idx] - row[base + idx - 1]) / dt;
  if (idx >= ip - 1) idx = ip - 2;
  return scale * (row[base + idx + 1] - row[base + idx]) / dt;
}

__global__ void __launch_bounds__(256) k_tdi_zero(double *out, int64_t n) {
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x)
    out[j] = 0.0;
}

// Per-item state of the stationary-phase sum, kept in shared memory while the
// warp spreads the item's bins over its lanes.
struct TdiItem {
  double t0, t1, om_in, delom, xi_in, dxi, dd0, dd1, fz0, fz1, A0, A1, e0, e1, omT0, omT1;
  double2 F0[6], F1[6];
  int s, j, lo, pad;
};
constexpr int kTdiWarps = 4;  // warps per CTA of k_tdi_spa

// Each warp takes 32 consecutive work items (source, interval, harmonic n,
// sideband m).  A lane finds its item's bins (most items cross none: a
// harmonic moves by far less than a bin over one grid interval) and, if it
// has some, stages the item's end-point quantities in shared memory.  The
// transfer functions of the items with bins (two per item, one per end) are
// then dealt out over the lanes, and a warp scan of the bin counts deals the
// warp's bins out one per lane, so that both heavy parts (constellation and
// transfer functions; Bessel recurrence, phase, interpolation, atomic adds)
// run with full warps.
__global__ void __launch_bounds__(kTdiWarps * 32) k_tdi_spa(TdiArgs a) {
  __shared__ TdiItem items[kTdiWarps][32];
  __shared__ int incl_s[kTdiWarps][32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  TdiItem *my = items[warp];
  int *incl_w = incl_s[warp];
  const double orbOm = 2. * kPi / kYear;
  const int64_t stride = (int64_t)gridDim.x * kTdiWarps * 32;
  for (int64_t base = ((int64_t)blockIdx.x * kTdiWarps + warp) * 32; base < a.total_work; base += stride) {
    const int64_t w = base + lane;
    int cnt = 0;
    if (w < a.total_work) {
      int lo = 0, hi = a.nsrc - 1;  // source holding work item w
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (a.work_start[mid] <= w) lo = mid;
        else hi = mid - 1;
      }
      const TdiDesc &d = a.src[lo];
      const int64_t local = w - a.work_start[lo];
      const int nh = 5 * d.nmodes;
      const int i = 1 + (int)(local / nh), ind = (int)(local % nh);
      const int j = ind / 5, jj = ind - 5 * j;
      const double nn = j + 1, mm = jj - 2.;
      const int64_t st = a.grid_stride, g = d.grid_offset;
      const double *G = a.grid;
      const double nu0 = G[kTdiNu * st + g + i - 1], nu1 = G[kTdiNu * st + g + i];
      const double gd0 = G[kTdiGd * st + g + i - 1], gd1 = G[kTdiGd * st + g + i];
      const double ad0 = G[kTdiAd * st + g + i - 1], ad1 = G[kTdiAd * st + g + i];
      const double om_in = nn * 2. * kPi * nu0 + 2. * gd0 + mm * ad0;
      const double om_fin = nn * 2. * kPi * nu1 + 2. * gd1 + mm * ad1;
      // bins ceil(om_in / dOm) .. floor(om_fin / dOm), the last one dropped when
      // om_fin falls on it (AAKTDI.cc:705-713); kept in doubles until clamped.
      // No bin lies in a falling, negative or NaN range.
      if (d.status == 0 && om_in > 0.0 && om_fin > om_in) {
        const double lo_b = ceil(om_in / d.dOm);
        double up_b = floor(om_fin / d.dOm);
        if (om_fin == up_b * d.dOm) up_b -= 1.0;
        const double mx_b = fmin(up_b + 1.0, (double)d.nbins);
        if (lo_b < mx_b) {
          cnt = (int)(mx_b - lo_b);
          TdiItem &it = my[lane];
          it.s = lo;
          it.j = ind;
          it.lo = (int)lo_b;
          it.om_in = om_in;
          it.delom = om_fin - om_in;
          it.t0 = G[kTdiT * st + g + i - 1];
          it.t1 = G[kTdiT * st + g + i];
          it.xi_in = it.t0 - d.DM * cos(orbOm * it.t0 - d.phiS);
          it.dxi = (it.t1 - d.DM * cos(orbOm * it.t1 - d.phiS)) - it.xi_in;
          it.dd0 = nn * tdi_ddot(G, kTdiNu * st + g, i - 1, d.i0, d.ip, 2. * kPi, d.dt_ph) +
                   2. * tdi_ddot(G, kTdiGd * st + g, i - 1, d.i0, d.ip, 1.0, d.dt_ph) +
                   mm * tdi_ddot(G, kTdiAd * st + g, i - 1, d.i0, d.ip, 1.0, d.dt_ph);
          it.dd1 = nn * tdi_ddot(G, kTdiNu * st + g, i, d.i0, d.ip, 2. * kPi, d.dt_ph) +
                   2. * tdi_ddot(G, kTdiGd * st + g, i, d.i0, d.ip, 1.0, d.dt_ph) +
                   mm * tdi_ddot(G, kTdiAd * st + g, i, d.i0, d.ip, 1.0, d.dt_ph);
          it.fz0 = nn * G[kTdiPhi * st + g + i - 1] + 2. * G[kTdiGim * st + g + i - 1] + mm * G[kTdiAlp * st + g + i - 1];
          it.fz1 = nn * G[kTdiPhi * st + g + i] + 2. * G[kTdiGim * st + g + i] + mm * G[kTdiAlp * st + g + i];
          it.A0 = G[kTdiAmp * st + g + i - 1];
          it.A1 = G[kTdiAmp * st + g + i];
          it.e0 = G[kTdiE * st + g + i - 1];
          it.e1 = G[kTdiE * st + g + i];
          it.omT0 = nn * G[kTdiPd * st + g + i - 1] + 2. * gd0 + mm * ad0;
          it.omT1 = nn * G[kTdiPd * st + g + i] + 2. * gd1 + mm * ad1;
        }
      }
    }
    // warp scan of the bin counts
    int incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int v = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += v;
    }
    const int total = __shfl_sync(0xffffffffu, incl, 31);
    if (total == 0) continue;  // warp-uniform
    incl_w[lane] = incl;
    // transfer functions: task t is end (t & 1) of the (t >> 1)-th item with bins
    const unsigned act = __ballot_sync(0xffffffffu, cnt > 0);
    const int nact = __popc(act);
    __syncwarp();
    for (int t = lane; t < 2 * nact; t += 32) {
      unsigned m = act;
      for (int r = t >> 1; r > 0; --r) m &= m - 1;  // drop the lower set bits
      TdiItem &it = my[__ffs(m) - 1];
      const bool hi_end = t & 1;
      tdi_transfer(a.src[it.s], hi_end ? it.t1 : it.t0, hi_end ? it.omT1 : it.omT0, hi_end ? it.F1 : it.F0);
    }
    __syncwarp();
    for (int b = lane; b < total; b += 32) {
      int l = 0, h = 31;  // owner: first lane whose inclusive count exceeds b
      while (l < h) {
        const int mid = (l + h) >> 1;
        if (incl_w[mid] > b) h = mid;
        else l = mid + 1;
      }
      const TdiItem &it = my[l];
      const TdiDesc &d = a.src[it.s];
      const int ii = it.lo + (b - (l > 0 ? incl_w[l - 1] : 0));
      const int j = it.j / 5, jj = it.j - 5 * j;
      const double nn = j + 1;
      const double Om = (double)ii * d.dOm;
      double delta = (Om - it.om_in) / it.delom, eps = 1. - delta;
      const double T = it.t1 * delta + it.t0 * eps;
      const double xi = T - d.DM * cos(orbOm * T - d.phiS);
      delta = (xi - it.xi_in) / it.dxi;
      eps = 1. - delta;
      const double dom = it.dd0 * eps + it.dd1 * delta;
      const double faza = it.fz0 * eps + it.fz1 * delta;
      const double amp = it.A0 * eps + it.A1 * delta;
      const double ec = it.e0 * eps + it.e1 * delta;
      const double ne = nn * ec;
      const int32_t bstart = a.bessel_start[d.bessel_offset + j];
      double J[5];
      if (!(ne > 0.0)) {
        for (int m = 0; m < 5; ++m) J[m] = 0.0;
        if (j == 0) J[1] = 1.0;        // J_0(0) at slot n - 1 for n = 1
        else if (j == 1) J[0] = 1.0;   // J_0(0) at slot n - 2 for n = 2
      } else if (j == 0) {
        double Jt[5];
        bessel5_fp64(0, ne, bstart, Jt);
        J[0] = -Jt[1];
        J[1] = Jt[0];
        J[2] = Jt[1];
        J[3] = Jt[2];
        J[4] = Jt[3];
      } else {
        bessel5_fp64(j - 1, ne, bstart, J);
      }
      const double hamp = -nn * ((J[0] - 2. * ec * J[1] + 2. / nn * J[2] + 2. * ec * J[3] - J[4]) +
                                 sqrt(1 - ec * ec) * (J[0] - 2. * J[2] + J[4]));
      delta = (T - it.t0) / d.dt_ph;
      eps = 1. - delta;
      const double Apc = hamp * d.AA[jj], Aps = hamp * d.AA[5 + jj];
      const double Acc = hamp * (2. * d.AA[10 + jj]), Acs = hamp * (2. * d.AA[15 + jj]);
      double sinph, cosph;
      sincos(faza - Om * xi + kPi * 0.25, &sinph, &cosph);
      const double fact = 0.5 * amp * sqrt(2. * kPi / dom);
      const double2 xp = make_double2(fact * (Apc * cosph + Aps * sinph), fact * (Apc * sinph - Aps * cosph));
      const double2 xc = make_double2(fact * (Acc * cosph + Acs * sinph), fact * (Acc * sinph - Acs * cosph));
      const int64_t o = d.bin_offset + ii;
#pragma unroll
      for (int ch = 0; ch < 3; ++ch) {
        const double2 cFp = cadd(cscale(eps, it.F0[2 * ch]), cscale(delta, it.F1[2 * ch]));
        const double2 cFc = cadd(cscale(eps, it.F0[2 * ch + 1]), cscale(delta, it.F1[2 * ch + 1]));
        const double2 r = cadd(cmul(cFp, xp), cmul(cFc, xc));
        atomicAdd(a.out + (2 * ch) * a.out_stride + o, r.x);
        atomicAdd(a.out + (2 * ch + 1) * a.out_stride + o, r.y);
      }
    }
    __syncwarp();  // the items and counts are reused by the next chunk
  }
}

void launch_tdi_spa(const TdiArgs &a, cudaStream_t stream) {
  if (a.out_stride > 0) k_tdi_zero<<<1184, 256, 0, stream>>>(a.out, 6 * a.out_stride);
  if (a.total_work <= 0) return;
  constexpr int per_block = kTdiWarps * 32;
  const int64_t blocks = std::min<int64_t>((a.total_work + per_block - 1) / per_block, 148 * 64);
  k_tdi_spa<<<(unsigned)blocks, per_block, 0, stream>>>(a);
}

namespace {
// 8 independent FMA chains per thread; the result is stored so nothing is elided.
__global__ void __launch_bounds__(256) k_fp64_fma_probe(double *out, int reps, double a, double b) {
  double x0 = threadIdx.x * 1e-9, x1 = x0 + 1e-9, x2 = x0 + 2e-9, x3 = x0 + 3e-9;
  double x4 = x0 + 4e-9, x5 = x0 + 5e-9, x6 = x0 + 6e-9, x7 = x0 + 7e-9;
  for (int r = 0; r < reps; ++r) {
#pragma unroll
    for (int u = 0; u < 16; ++u) {
      x0 = fma(x0, a, b);
      x1 = fma(x1, a, b);
      x2 = fma(x2, a, b);
      x3 = fma(x3, a, b);
      x4 = fma(x4, a, b);
      x5 = fma(x5, a, b);
      x6 = fma(x6, a, b);
      x7 = fma(x7, a, b);
    }
  }
  out[blockIdx.x * blockDim.x + threadIdx.x] = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
}
}  // namespace

double probe_fp64_fma_tflops(int num_sms, int iters, cudaStream_t stream) {
  const int blocks = num_sms * 8, threads = 256, reps = 2048;
  double *out = nullptr;
  if (cudaMalloc(&out, (size_t)blocks * threads * sizeof(double)) != cudaSuccess) return -1.0;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  k_fp64_fma_probe<<<blocks, threads, 0, stream>>>(out, reps, 0.999999, 1e-7);  // warm-up
  cudaEventRecord(e0, stream);
  for (int i = 0; i < iters; ++i) k_fp64_fma_probe<<<blocks, threads, 0, stream>>>(out, reps, 0.999999, 1e-7);
  cudaEventRecord(e1, stream);
  cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  const double flops = 2.0 * 8.0 * 16.0 * reps * (double)blocks * threads * iters;
  return cudaGetLastError() == cudaSuccess && ms > 0 ? flops / (ms * 1e-3) / 1e12 : -1.0;
}

namespace {
// 8 independent FP32 FMA chains per thread.
__global__ void __launch_bounds__(256) k_fp32_fma_probe(float *out, int reps, float a, float b) {
  float x[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) x[k] = threadIdx.x * 1e-6f + k * 1e-6f;
  for (int r = 0; r < reps; ++r) {
#pragma unroll
    for (int u = 0; u < 16; ++u) {
#pragma unroll
      for (int k = 0; k < 8; ++k) x[k] = fmaf(x[k], a, b);
    }
  }
  float acc = 0.f;
#pragma unroll
  for (int k = 0; k < 8; ++k) acc += x[k];
  out[blockIdx.x * blockDim.x + threadIdx.x] = acc;
}
}  // namespace

double probe_fp32_fma_tflops(int num_sms, int iters, cudaStream_t stream) {
  const int blocks = num_sms * 8, threads = 256, reps = 4096;
  float *out = nullptr;
  if (cudaMalloc(&out, (size_t)blocks * threads * sizeof(float)) != cudaSuccess) return -1.0;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  k_fp32_fma_probe<<<blocks, threads, 0, stream>>>(out, reps, 0.999999f, 1e-7f);  // warm-up
  cudaEventRecord(e0, stream);
  for (int i = 0; i < iters; ++i) k_fp32_fma_probe<<<blocks, threads, 0, stream>>>(out, reps, 0.999999f, 1e-7f);
  cudaEventRecord(e1, stream);
  cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  const double flops = 2.0 * 8.0 * 16.0 * reps * (double)blocks * threads * iters;
  return cudaGetLastError() == cudaSuccess && ms > 0 ? flops / (ms * 1e-3) / 1e12 : -1.0;
}

// ------------------------------------------------------------------ allocation-free launch
// Tile scratch (look-back records and flags, the work-queue head, the
// per-launch status word and the report word) for callers that must not
// allocate device memory.  The array is part of the module image: every GPU
// that loads this library holds kStaticScratchBytes (about 4.9 MB) until the
// process exits.  All calls share it and it keeps the last call's contents;
// launches that overlap on the GPU race on it.
namespace {
static __device__ __align__(256) unsigned char g_tile_scratch[kStaticScratchBytes];
// counters at kStaticCounterOffset: work-queue head (8 bytes), this launch's
// status word, the report word
constexpr size_t kStaticStatusOffset = kStaticCounterOffset + sizeof(unsigned long long);
constexpr size_t kStaticReportOffset = kStaticStatusOffset + sizeof(unsigned int);

// devices on which an allocation-free launch has run (their report word is live)
std::atomic<bool> g_scratch_used[kMaxStaticDevices];

// The array's device address in the current context (the caller has made the
// device current).  Looked up on every call: the lookup allocates nothing,
// and a cached address would be stale after a cudaDeviceReset or in another
// context of the same device.
void *static_scratch_base() {
  void *p = nullptr;
  if (cudaGetSymbolAddress(&p, g_tile_scratch) != cudaSuccess || !p) {
    cudaGetLastError();
    return nullptr;
  }
  return p;
}
}  // namespace

namespace {
// Tile 1 of a two-tile chain looks back at tile 0, whose flag stays 0 (one warp).
__global__ void k_lookback_selftest(BatchView bv) {
  if (blockIdx.x != 0) return;
  TileCtx c{};
  c.lt = 1;
  c.head = 0;
  c.g = 1;
  double hi[3], lo[3], C;
  look_back_warp(bv, c, 1, hi, lo, C);
}
}  // namespace

int lookback_timeout_selftest(long long cycles, cudaStream_t stream) {
  void *buf = nullptr;
  const size_t bytes = 2 * sizeof(TileLink) + 256;
  if (cudaMalloc(&buf, bytes) != cudaSuccess) return -1;
  unsigned char *b = static_cast<unsigned char *>(buf);
  BatchView bv{};
  bv.link = reinterpret_cast<TileLink *>(b);
  bv.link_flag = reinterpret_cast<int32_t *>(b + 2 * sizeof(TileLink));
  bv.device_status = reinterpret_cast<unsigned int *>(b + 2 * sizeof(TileLink) + 64);
  bv.lookback_cycles = cycles > 0 ? cycles : 1;
  unsigned int v = 0;
  int out = -1;
  if (cudaMemsetAsync(buf, 0, bytes, stream) == cudaSuccess) {
    k_lookback_selftest<<<1, 32, 0, stream>>>(bv);
    if (cudaGetLastError() == cudaSuccess && cudaStreamSynchronize(stream) == cudaSuccess &&
        cudaMemcpy(&v, bv.device_status, sizeof(v), cudaMemcpyDeviceToHost) == cudaSuccess)
      out = v ? 1 : 0;
  }
  cudaFree(buf);
  return out;
}

int static_scratch_status(int device, bool clear) {
  if (device < 0 || device >= kMaxStaticDevices) return 0;
  if (!g_scratch_used[device].load()) return 0;  // no allocation-free launch on this device yet
  void *base = static_scratch_base();
  if (!base) return -1;
  unsigned int *word = reinterpret_cast<unsigned int *>(static_cast<unsigned char *>(base) + kStaticReportOffset);
  unsigned int v = 0;
  if (cudaMemcpy(&v, word, sizeof(v), cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
  if (v && clear && cudaMemset(word, 0, sizeof(v)) != cudaSuccess) return -1;
  return v ? 1 : 0;
}

int launch_dense_static_scratch(BatchView bv, int device, int num_sms, cudaStream_t stream, int precision) {
  if (bv.total_tiles > kStaticScratchTiles) return 8;  // AAK_ERR_CAPACITY
  if (device < 0 || device >= kMaxStaticDevices || (precision != 0 && precision != 1)) return 1;
  void *base = static_scratch_base();
  if (!base) return 5;  // AAK_ERR_CUDA
  g_scratch_used[device].store(true);
  unsigned char *b = static_cast<unsigned char *>(base);
  bv.link = reinterpret_cast<TileLink *>(b);
  bv.link_flag = reinterpret_cast<int32_t *>(b + kStaticFlagOffset);
  bv.work_counter = reinterpret_cast<unsigned long long *>(b + kStaticCounterOffset);
  bv.device_status = reinterpret_cast<unsigned int *>(b + kStaticStatusOffset);
  bv.status_report = reinterpret_cast<unsigned int *>(b + kStaticReportOffset);
  // this launch's waits give up early only on a give-up of this launch
  if (cudaMemsetAsync(bv.device_status, 0, sizeof(unsigned int), stream) != cudaSuccess) return 5;
  // launch_dense clears the work-queue head and the look-back flags on
  // `stream`; every record is written before its flag is
  launch_dense(bv, num_sms, stream, nullptr, precision);
  return cudaGetLastError() == cudaSuccess ? 0 : 5;
}

}  // namespace aak
