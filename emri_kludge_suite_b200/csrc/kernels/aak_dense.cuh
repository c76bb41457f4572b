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

// Look-back record of one tile in its source's phase chain (the single-pass
// scan of the waveform kernel).  The tile holding t = 0 (sample i0) heads two
// chains: the forward one runs through the later tiles in increasing order,
// the backward one through the earlier tiles in decreasing order, and the
// work queue hands tiles out in that order.  link_flag[g] (0: not written,
// 1: aggregate, 2: inclusive) is stored with release semantics after the
// record: an aggregate holds the tile's own increments, an inclusive record
// the increments from the chain head through the tile; the two sets of
// fields are separate, so that a reader never sees one half-overwritten.
struct TileLink {
  // aggregate (flag >= 1): the tile's own increments along its chain
  double agg[3];            // forward tiles: forward increments; backward tiles: backward increments
  double agg_C;             // clamped Phidot after the tile's last forward sample
  int32_t agg_hasC;         // agg_C was set inside the tile
  int32_t pad;
  // inclusive (flag == 2): increments from the chain head through the tile, double-double
  double inc_f_hi[3], inc_f_lo[3];
  double inc_b_hi[3], inc_b_lo[3];
  double inc_C;             // clamped Phidot after the tile (0 before the first forward sample)
};

// Per-tile values the waveform kernel needs before its phase pass, computed
// for every tile of a batch by the tile pre-pass (k_tile_params): the centre
// e_c and term count K of the tile's Bessel table, and the raw AB2 rates of
// the samples just before and just after the tile.  64 bytes, so that it
// lands in shared memory with one bulk copy.
struct alignas(16) TilePrep {
  double ec;
  int16_t K;        // Taylor terms (0: per-sample Miller recurrence; -1: no harmonic sums in the tile)
  int16_t stride;   // elements per table row of the tile
  int32_t src;      // source of the tile
  double rb[3];     // rates of sample start - 1 (rb[1] = -1: there is none)
  double ra[3];     // rates of sample end (for the backward AB2 step of the tile's last sample)
};
static_assert(sizeof(TilePrep) == 64, "TilePrep is one 64-byte bulk copy");

// Taylor-table rows: FP64 terms at most (K <= 10) and FP32 terms at most
// (K <= 6); a tile's FP64 rows hold 3 (K + 1) coefficients of one harmonic,
// its FP32 rows 6 (K + 1) of a pair of harmonics, padded to 16 bytes.
constexpr int kTaylorMax64 = 10;
constexpr int kTaylorMax32 = 6;
constexpr int kRowD = (3 * (kTaylorMax64 + 1) + 1) / 2 * 2;  // doubles per FP64 row at most (34)
constexpr int kRowF = (3 * (kTaylorMax32 + 1) + 3) / 4 * 4;  // floats per FP32 row at most (24)
// Harmonic counts up to kTabModes use the tables (more: per-sample Bessel recurrences).
constexpr int kTabModes = 128;
// Bytes of one tile's slot in the pre-built table array for `rows` harmonics
// (largest harmonic count of the batch) in FP64 (split = false) or FP32 rows.
inline int64_t tile_table_slot_bytes(int rows, bool split) {
  const int r = (rows > 0 && rows < kTabModes) ? rows : kTabModes;
  // FP32 tables hold pairs of harmonics (a pair row is at most 2 kRowF floats)
  return split ? (int64_t)((r + 1) & ~1) * kRowF * (int64_t)sizeof(float)
               : (int64_t)r * kRowD * (int64_t)sizeof(double);
}

// Launch shapes of the waveform stage, the autotuner's candidates: with the
// tile pre-pass or tables built inside the tiles, samples per thread whose
// harmonic sums run side by side, and resident CTAs per SM the register
// budget is sized for.  Variant 0 is the default of each precision: the
// autotuner's choice on both the 512-source configuration-1 batch and a
// 256-template configuration-4 chunk, in both precisions.
struct WaveVariant {
  bool pre;
  int joint;
  int min_blocks;
};
constexpr int kNumVariants = 6;
constexpr WaveVariant wave_variant(bool split, int v) {
  return split ? (v == 1 ? WaveVariant{false, 0, 2} : v == 2 ? WaveVariant{true, 1, 2} : v == 3 ? WaveVariant{true, 4, 2}
                  : v == 4 ? WaveVariant{true, 2, 3} : v == 5 ? WaveVariant{true, 2, 2} : WaveVariant{true, 1, 3})
               : (v == 1 ? WaveVariant{false, 0, 2} : v == 2 ? WaveVariant{true, 2, 2} : v == 3 ? WaveVariant{true, 4, 2}
                  : v == 4 ? WaveVariant{true, 1, 2} : v == 5 ? WaveVariant{true, 2, 3} : WaveVariant{true, 1, 3});
}

// One work-queue item: a tile, its place in its source, and what staging it
// needs, so that a CTA can issue the tile's bulk copies and find its source
// with one load (no search over the tile prefix, no dependent lookups).
struct alignas(16) QueueItem {
  int64_t knot;   // absolute index (in the knot arrays) of the first knot of the tile's window
  int32_t g;      // global tile index
  int32_t s;      // source
  int32_t lt;     // tile index inside the source
  int32_t k0;     // first knot of the window, source-relative
  int32_t nk;     // knots in the window
  int32_t flags;  // kQueueNoWave, kQueueFailed
};
static_assert(sizeof(QueueItem) == 32, "a queue item is two 16-byte loads");
constexpr int32_t kQueueNoWave = 1;  // no waveform output: failed source, or a tile entirely after the taper
constexpr int32_t kQueueFailed = 2;  // failed source (the phase passes have no output either)

// Everything the kernels read about a batch.
struct BatchView {
  const SourceDesc *src;
  int32_t nsrc;
  int64_t total_tiles;
  const int64_t *tile_start;    // nsrc + 1 prefix of tiles (device)
  const QueueItem *queue = nullptr;  // work-queue order; null: source by source, each in chain order
  const int32_t *tile_knot;     // 2 per tile: first knot of the tile's window, knots in it
  const double *knot_t;         // knots
  const double4 *knot_y;        // (e, v, M, S) at the knots
  const double4 *knot_c;        // natural-spline half second derivatives
  const int32_t *bessel_start;  // Miller start orders, per source x mode
  TileLink *link;               // one per tile
  int32_t *link_flag;           // one per tile, cleared before every launch
  double *hI, *hII;             // outputs, indexed by src.out_offset + i
  float *hI_f32 = nullptr, *hII_f32 = nullptr;  // FP32 outputs instead (same indexing), when set
  double *t_out;                // optional
  double *traj_out;             // optional dense trajectory, 9 x total samples (e,v,M,S,gim,Phi,alp,nu,gimdot)
  int64_t traj_stride;
  unsigned long long *work_counter;  // persistent work queue head, cleared before every launch
  unsigned int *device_status;       // set to 1 when a bounded look-back wait gave up (never cleared here)
  unsigned int *status_report = nullptr;  // optional second word set with it: a report kept across launches
  int32_t trajectory_only = 0;       // 1: write traj_out and skip the harmonic sums
  int32_t max_nmodes = 0;            // largest harmonic count of the batch (0: unknown) -- sizes the tile table
  long long lookback_cycles = 0;     // bound of one look-back wait in SM clocks (<= 0: about 2 s)
  double *phase_out = nullptr;       // launch_phase: 8 x phase_stride (t, phase_r, phase_theta, phase_phi,
  int64_t phase_stride = 0;          //   omega_r, omega_theta, omega_phi, e), indexed by src.out_offset + i
  // optional tile pre-pass buffers (launch_dense): one TilePrep per tile and
  // one table slot of tab_slot bytes per tile; without them the waveform
  // kernel computes both inside each tile
  TilePrep *tile_prep = nullptr;
  void *tile_tab = nullptr;
  int64_t tab_slot = 0;
  int32_t variant = 0;  // launch shape of the waveform stage (wave_variant), chosen by the autotuner
};

// Clear the work queue and the look-back flags, then launch the waveform
// kernel, on `stream`.  With bv.tile_prep and bv.tile_tab set (and no
// trajectory output), the tile pre-pass (tile parameters, then every tile's
// Taylor table, harmonics in parallel) runs first and the waveform kernel
// stages each tile's source record, parameters, knot window and table in
// shared memory with bulk copies.  ev (optional, 4 events): ev[0]..ev[1]
// bracket the clears, ev[1]..ev[2] the pre-pass (empty without it),
// ev[2]..ev[3] the waveform kernel.
void launch_dense_fp64(const BatchView &bv, int num_sms, cudaStream_t stream, cudaEvent_t *ev);
// precision 0: FP64 throughout; 1: split (FP64 phases and reductions, FP32
// geometry, response, Bessel evaluation and harmonic recurrence).
void launch_dense(const BatchView &bv, int num_sms, cudaStream_t stream, cudaEvent_t *ev, int precision);
// ------------------------------------------------------------------ frequency-domain TDI
// Rows of the TDI phase grid that launch_tdi_grid writes to bv.phase_out
// (kTdiRows x phase_stride, indexed by src.out_offset + i): the grid time,
// e, the amplitude (Omega_phi M)^(2/3) zeta, the three phases, nu = Phidot /
// 2 pi, gamma~dot, alphadot and Phidot (clamped after i0, raw elsewhere).
constexpr int kTdiT = 0, kTdiE = 1, kTdiAmp = 2, kTdiGim = 3, kTdiPhi = 4, kTdiAlp = 5, kTdiNu = 6, kTdiGd = 7,
              kTdiAd = 8, kTdiPd = 9, kTdiRows = 10;
// The phase grid of PNevolutionTDI (src/suite/AAKTDI.cc:27-469) for every
// source of a batch planned on that grid (length Nph, dt = dt_ph): the
// waveform kernel's phase pass over all grid points, writing the rows above.
void launch_tdi_grid(const BatchView &bv, int num_sms, cudaStream_t stream, cudaEvent_t *ev);

// One source of the stationary-phase sum (waveformTDI, AAKTDI.cc:520-797).
struct TdiDesc {
  int64_t grid_offset;   // first grid point of the source in the grid rows
  int64_t bin_offset;    // first output bin of the source
  int32_t i0, ip;        // grid index of t = 0; intervals i = 1 .. ip - 1 are summed
  int32_t nmodes, nbins; // harmonics; (length + 1) / 2 output bins
  int32_t bessel_offset, status;
  double dt_ph, dOm, DM, phiS, arm;
  double k[3], uhat[3], vhat[3], c2psi, s2psi;  // propagation direction, polarisation basis and angle
  double AA[20];         // sideband amplitudes: cos / sin of plus, cos / sin of cross, m = -2..2 each
};
struct TdiArgs {
  const TdiDesc *src;
  int32_t nsrc;
  const int64_t *work_start;  // nsrc + 1 prefix of (ip - 1) x 5 nmodes work items
  int64_t total_work;
  const double *grid;         // kTdiRows x grid_stride
  int64_t grid_stride;
  const int32_t *bessel_start;
  double *out;                // 6 x out_stride: Xr, Xi, Yr, Yi, Zr, Zi (zeroed by the launch)
  int64_t out_stride;
};
// Zero the outputs, then one thread per (source, interval, harmonic n, sideband m):
// the bins the harmonic crosses in the interval, each added to X, Y, Z with a
// double atomic add (the order of the adds into one bin is not fixed).
void launch_tdi_spa(const TdiArgs &a, cudaStream_t stream);

// The AAK phase product of GenPhase (src/suite/AAKPhase.cc:315-374) for
// every source of the batch into bv.phase_out: the waveform kernel's phase
// pass over all samples (no harmonic sums), then the freeze of the phases
// after the plunge buffer.  ev (optional, 4 events) as launch_dense, ev[3]
// after the freeze.
void launch_phase(const BatchView &bv, int num_sms, cudaStream_t stream, cudaEvent_t *ev);

// Plain FP64 per-source harmonic sum: the per-sample algorithm of the
// reference's CUDA port (src/cuda/kernel.cu:374-555) -- five Bessel functions
// jn(n-2 .. n+2, n e), one cos/sin of n Phi and the NK-frame rotation per
// harmonic -- on the dense trajectory (9 x traj_stride doubles, as the waveform kernel
// writes with trajectory_only) of source s of the batch.
// Natural-spline coefficients c (half second derivatives, c = 0 at both ends)
// of every source's knots, solved on the device: the interior knots of a
// source are cut into blocks of kSplineBlock, and one thread solves each block
// by Thomas elimination over the block widened by kSplineHalo knots on either
// side, taking c = 0 where the widened window is cut.  The system is
// diagonally dominant (|h0| + |h1| = half the diagonal 2 (h0 + h1)), so the
// influence of a cut decays at least as 0.27^k with the distance k in knots:
// 40 knots leave it below 1e-22.  blk_start: nsrc + 1 prefix of the blocks per
// source (spline_blocks).
constexpr int kSplineBlock = 256;
constexpr int kSplineHalo = 40;
inline int64_t spline_blocks(int n_knots) { return n_knots < 3 ? 1 : (n_knots - 2 + kSplineBlock - 1) / kSplineBlock; }
void launch_spline_coeffs(const SourceDesc *src, int nsrc, const int64_t *blk_start, int64_t total_blocks,
                          const double *knot_t, const double4 *knot_y, double4 *knot_c, cudaStream_t stream);

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
// Size of the file-scope scratch array: 32768 look-back records of 144 bytes,
// 32768 flags and 256 bytes of counters (4,849,920 bytes, about 4.9 MB).
constexpr size_t kStaticLinkBytes = (size_t)kStaticScratchTiles * sizeof(TileLink);
constexpr size_t kStaticFlagOffset = (kStaticLinkBytes + 255) / 256 * 256;
constexpr size_t kStaticCounterOffset =
    (kStaticFlagOffset + (size_t)kStaticScratchTiles * sizeof(int32_t) + 255) / 256 * 256;
constexpr size_t kStaticScratchBytes = kStaticCounterOffset + 256;

// Same kernels as launch_dense (precision 0 or 1), with the tile scratch
// (bv.link, bv.link_flag, bv.work_counter, bv.device_status and
// bv.status_report are ignored) taken from a file-scope __device__ array
// instead of caller or context allocations.  Every launch starts with its own
// status word cleared, so a wait that gave up in an earlier launch does not
// cut the waits of this one short; a give-up is also recorded in a report
// word that stays set until static_scratch_status clears it.  Returns an
// aak_status.  The first call on a device looks the array's address up (once
// per device).
int launch_dense_static_scratch(BatchView bv, int device, int num_sms, cudaStream_t stream, int precision);
// Report word of the allocation-free scratch on `device` (current): 1 if a
// bounded look-back wait of one of its launches gave up since the last clear,
// 0 if not (or no such launch yet), -1 on a CUDA error; `clear` resets it.
// Synchronous.
int static_scratch_status(int device, bool clear);

// Self-test of the bounded look-back wait: one CTA waits on a flag that
// nothing sets, for at most `cycles` SM clocks, on `stream`; returns the
// device status word it left (1: the wait gave up as it should) or -1 on a
// CUDA error.  Synchronous.
int lookback_timeout_selftest(long long cycles, cudaStream_t stream);

}  // namespace aak
