// aak_dense.cuh -- device-side layout shared by the dense AAK kernels and
// their host launcher.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../aak_common.hpp"

namespace aak {

constexpr int kTileThreads = 256;                      // threads per CTA
#ifndef AAK_TILE_CHUNKS
#define AAK_TILE_CHUNKS 4
#endif
constexpr int kTileChunks = AAK_TILE_CHUNKS;           // 256-sample chunks per tile
constexpr int kTileSamples = kTileThreads * kTileChunks;  // 1024 samples per tile

// Per-tile partial sums of the Adams-Bashforth-2 phase increments written by
// pass 1.  For each phase q (0: gamma~, 1: Phi, 2: alpha) the forward sum over
// the tile is fA[q] + fB[q] * C[q], where C[q] is the (clamped) rate of the
// sample just before the tile; the backward sum is bA[q] + bB[q] * C'[q] with
// C'[q] the rate of the sample just after the tile.
struct TileSummary {
  double fA[3], fB[3];
  double bA[3], bB[3];
  double last_rate[3];   // gim/alp: rate of the last forward sample; Phi: last positive raw rate
  double first_rate[3];  // raw rates of the first sample in the tile
  int32_t has_last[3];   // last_rate valid
  int32_t pad;
  double rate_before[3]; // raw rates of the sample just before the tile (Phi: -1 if none)
  double ec;             // Bessel-table centre eccentricity of the tile (0: no output samples)
  int32_t k64, k32;      // multiplication-theorem terms for the FP64 / split harmonic sums (0: per-sample)
};

// Per-tile carries written by the carry kernel and read by pass 2.
struct TileCarry {
  double fwd_hi[3], fwd_lo[3];  // sum of forward increments before the tile (double-double)
  double bwd_hi[3], bwd_lo[3];  // sum of backward increments after the tile
  double Cf[3];                 // rate carried into the tile's first forward increment
  double Cb[3];                 // rate carried into the tile's last backward increment
};

// Everything the kernels read about a batch.
struct BatchView {
  const SourceDesc *src;
  int32_t nsrc;
  int64_t total_tiles;
  const int64_t *tile_start;    // nsrc + 1 prefix of tiles (device)
  const int32_t *tile_knot;     // 2 per tile: first knot of the tile's window, knots in it
  const double *knot_t;         // knots
  const double4 *knot_y;        // (e, v, M, S) at the knots
  const double4 *knot_c;        // natural-spline half second derivatives
  const int32_t *bessel_start;  // Miller start orders, per source x mode
  TileSummary *summ;
  TileCarry *carry;
  double *hI, *hII;             // outputs, indexed by src.out_offset + i
  double *t_out;                // optional
  double *traj_out;             // optional dense trajectory, 9 x total samples (e,v,M,S,gim,Phi,alp,nu,gimdot)
  int64_t traj_stride;
  unsigned long long *work_counter;  // persistent work queue head (pass 2)
  int32_t trajectory_only = 0;       // 1: pass 2 writes traj_out and skips the harmonic sums
  int32_t max_nmodes = 0;            // largest harmonic count of the batch (0: unknown) -- sizes the tile table
};

// Launch pass 1, the carry scan and pass 2 on `stream`.  ev (optional, 4
// events) brackets the three kernels for per-kernel timing.
void launch_dense_fp64(const BatchView &bv, int num_sms, cudaStream_t stream, cudaEvent_t *ev);
// precision 0: FP64 throughout; 1: split (FP64 phases and reductions, FP32
// geometry, response, Bessel evaluation and harmonic recurrence).
void launch_dense(const BatchView &bv, int num_sms, cudaStream_t stream, cudaEvent_t *ev, int precision);

// Plain FP64 per-source harmonic sum: the per-sample algorithm of the
// reference's CUDA port (src/cuda/kernel.cu:374-555) -- five Bessel functions
// jn(n-2 .. n+2, n e), one cos/sin of n Phi and the NK-frame rotation per
// harmonic -- on the dense trajectory (9 x traj_stride doubles, as pass 2
// writes with trajectory_only) of source s of the batch.
void launch_plain_waveform(const SourceDesc *src, int s, int vlength, const double *traj, int64_t traj_stride,
                           double *hI, double *hII, cudaStream_t stream);

// Diagnostic: sustained FP64 FMA issue rate of this device in TFLOP/s
// (2 flops per FMA), measured with CUDA events over `iters` launches.
double probe_fp64_fma_tflops(int num_sms, int iters, cudaStream_t stream);
// The same for FP32 FMA.
double probe_fp32_fma_tflops(int num_sms, int iters, cudaStream_t stream);

// Per-device launch set-up of the dense kernels (shared-memory opt-in); done
// by launch_dense itself, and needed before capturing it into a CUDA graph.
void prepare_dense_launch();

// Largest batch (in 1024-sample tiles) the allocation-free launch accepts,
// and the number of devices whose scratch address is cached.
constexpr int64_t kStaticScratchTiles = 32768;
constexpr int kMaxStaticDevices = 64;

// Same kernels as launch_dense_fp64, with the tile scratch (bv.summ,
// bv.carry, bv.work_counter are ignored) taken from a file-scope __device__
// array instead of caller or context allocations.  Returns an aak_status.
// The first call on a device looks the array's address up (once per device).
int launch_dense_fp64_static_scratch(BatchView bv, int device, int num_sms, cudaStream_t stream);

}  // namespace aak
