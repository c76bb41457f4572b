/*
 * aak.h -- C ABI of libaak_b200.so, the B200 (sm_100a) implementation of the
 * augmented analytic kludge (AAK) EMRI waveform and its LISA noise-weighted
 * inner product.
 *
 * Plain C types only.  Every entry point returns an aak_status (0 = OK) and
 * never terminates the process; the library keeps no global mutable state
 * besides one lazily created default context per device, so independent
 * contexts may be used from independent host threads.
 *
 * Each declaration names the reference interface it replaces
 * (alvincjk/EMRI_Kludge_Suite, path:line).
 */
#ifndef AAK_B200_H
#define AAK_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ status */
enum aak_status {
  AAK_OK = 0,
  AAK_ERR_INVALID_PARAM = 1,            /* reference: undefined behaviour / Die()      */
  AAK_ERR_UNSTABLE_START = 2,           /* p0 inside the LSO (GKTrajFast flag -1)      */
  AAK_ERR_FIT_TOO_CLOSE_TO_PLUNGE = 3,  /* reference: exit(EXIT_FAILURE), AAK.cc:88    */
  AAK_ERR_SOLVER_NO_CONVERGE = 4,       /* Kerr->AK map did not reach |f|_1 < 1e-6     */
  AAK_ERR_CUDA = 5,                     /* no usable GPU, or a CUDA/cuFFT call failed  */
  AAK_ERR_NO_MEMORY = 6,
  AAK_ERR_TOO_FEW_STEPS = 7,            /* coarse inspiral gave fewer than 3 points    */
  AAK_ERR_CAPACITY = 8,                 /* request exceeds a fixed-size buffer         */
  AAK_ERR_DEVICE_TIMEOUT = 9            /* a bounded device-side wait gave up          */
};

const char *aak_status_string(int status);
int aak_version(void);
/* Name and text of the last CUDA error this thread's calls turned into a
 * status (empty if none). */
const char *aak_last_error_detail(void);

/* ------------------------------------------------------------------ parameters */
/* Numeric fields of the reference's SetPar (include/KSTools.h:21-53) and the
 * keys of AAKwrapper.wave's pars dict (AAKwrapper/AAKwrapper.pyx:50-80). */
typedef struct aak_params {
  int64_t length; /* waveform samples                               */
  double dt;      /* sample spacing [s]                             */
  double p;       /* initial semi-latus rectum [M]                  */
  double T;       /* duration [yr] (informational, as in SetPar)    */
  double f;       /* reference GW frequency [Hz] (informational)    */
  double T_fit;   /* local-fit duration [M^2/mu]                    */
  double mu;      /* compact-object mass [Msun]                     */
  double M;       /* black-hole mass [Msun]                         */
  double s;       /* spin a/M                                       */
  double e;       /* initial eccentricity                           */
  double iota;    /* inclination of L from S [rad]                  */
  double gamma;   /* initial periapsis angle from L x S             */
  double psi;     /* initial true anomaly                           */
  double theta_S, phi_S, theta_K, phi_K; /* ecliptic source / spin angles */
  double alpha;   /* initial azimuthal orientation                  */
  double D;       /* distance [Gpc]                                 */
  int32_t backint; /* integrate backwards from plunge              */
  int32_t LISA;    /* LISA h_I/h_II response (else detector-frame) */
} aak_params;

/* Output of the front end: the arrays the reference hands to GenWave
 * (src/suite/AAKpy.cc:29-44).  Arrays hold up to 100 entries. */
typedef struct aak_mapped {
  int32_t steps;
  int32_t inspiral_flag;     /* GKTrajFast::Eccentric return value */
  int32_t newton_iterations; /* summed over the coarse points      */
  int32_t pad;
  double Phi0;               /* initial mean anomaly (ParAng)      */
  double e_traj[100], v_map[100], M_map[100], s_map[100], dt_map[100];
} aak_mapped;

/* ------------------------------------------------------------------ host-only stages */
/* Front end of AAKwave (src/suite/AAKpy.cc:20-44): coarse Kerr inspiral
 * (GKTrajFast::Eccentric), Kerr frequencies (IEKG::Frequencies), initial mean
 * anomaly (ParAng) and the Kerr->AK map (ParMap, KSParMap.cc:397-440).
 * warm_start: optional steps x 3 initial guesses (v_map, M_map, s_map), or NULL. */
int aak_front_end(const aak_params *p, const double *warm_start, aak_mapped *out);

/* Coarse Kerr inspiral + fundamental frequencies only (no map).
 * out_t/p/e/cosi/Omega hold up to 100 (Omega: 100 x 3) entries. */
int aak_coarse_kerr(const aak_params *p, int32_t *steps, double *t_rr, double *pp, double *e, double *cosi,
                    double *Omega);

/* One Kerr->AK map solve (ParMap, src/suite/KSParMap.cc:397-440); x0 may be NULL
 * for the reference's initial guess.  *iterations receives the Newton count. */
int aak_parmap(const double Omega[3], double p, double M, double s, double e, double iota, const double *x0,
               double map[3], int32_t *iterations);

/* ------------------------------------------------------------------ single-source waveform (GPU) */
/* Replaces AAKwave (include/AAKpy.h:19, src/suite/AAKpy.cc:16-51).  Host
 * buffers of p->length doubles.  *seconds (optional) receives the wall time.
 * Runs on the current CUDA device; fails with AAK_ERR_CUDA without one. */
int aak_wave(const aak_params *p, double *t, double *hI, double *hII, double *seconds);

/* ------------------------------------------------------------------ frequency-domain AAK TDI (GPU) */
/* Replaces AAKTDI (include/AAKpy.h, src/suite/AAKpy.cc:90-125; GenTDI and
 * waveformTDI, src/suite/AAKTDI.cc:27-829): stationary-phase Michelson TDI
 * channels X, Y, Z of the AAK source on the (p->length + 1) / 2 bins
 * f = i / ((length - 1) dt).  Host buffers of (length + 1) / 2 doubles; f
 * optional.  The phase grid (spacing 0.01 M^2 / mu) is generated on the
 * GPU; each (interval, harmonic, sideband) adds its bins with double atomic
 * adds, so the last bits of a bin may differ between calls.  FP64.  Errors as
 * aak_wave. */
int aak_tdi(const aak_params *p, double *f, double *Xf_r, double *Xf_im, double *Yf_r, double *Yf_im, double *Zf_r,
            double *Zf_im, double *seconds);

/* ------------------------------------------------------------------ AAK phases (GPU) */
/* Replaces AAKphase (include/AAKpy.h:21, src/suite/AAKpy.cc:53-88, GenPhase
 * src/suite/AAKPhase.cc:315-374).  Host buffers of p->length doubles: t, the
 * three phases Phi, Phi + gamma~, Phi + gamma~ + alpha, the three rates Phidot
 * (clamped after t = 0), Phidot + gamma~dot, Phidot + gamma~dot + alphadot, and
 * the eccentricity; the phases after i_plunge + i_buffer + 1 hold their values
 * at i_plunge.  FP64.  *seconds (optional) receives the wall time.  Errors as
 * aak_wave. */
int aak_phase(const aak_params *p, double *t, double *phase_r, double *phase_theta, double *phase_phi,
              double *omega_r, double *omega_theta, double *omega_phi, double *eccentricity, double *seconds);

/* Replaces GenWave -> waveform (src/suite/AAK.cc:321-591) on an already
 * mapped trajectory; nmodes_override <= 0 keeps the reference harmonic rule
 * int(30 e0) (4 below e0 = 0.135).  Host buffers of vlength doubles. */
int aak_genwave(double *t, double *hI, double *hII, double timestep, int32_t vlength, const double *e_traj,
                const double *v_map, double M_phys, const double *M_map, double mu, double S_phys, const double *S_map,
                double dist, double inc, double gim0, double Phi0, double qS, double phiS, double alp0, double qK,
                double phiK, const double *dt_map, int32_t steps, int32_t backint, int32_t mich,
                int32_t nmodes_override);

/* ------------------------------------------------------------------ batched waveforms */
/* A context owns the device buffers of one batch on one device.  device -1
 * makes a host-only context: planning and the plan queries work without a
 * GPU, the upload and run calls return AAK_ERR_INVALID_PARAM. */
typedef struct aak_ctx aak_ctx;

int aak_ctx_create(int32_t device, aak_ctx **out);
void aak_ctx_destroy(aak_ctx *ctx);

/* Host planning of a batch (front end + coarse AK evolution + spline knots),
 * spread over nthreads host threads (<= 0: all hardware threads).
 * nmodes_override: per-source harmonic counts (<= 0 entries keep the
 * reference rule) or NULL.  Per-source failures are reported in the source
 * status (aak_batch_info) and yield zero waveforms; the call itself fails
 * only for context-level errors.  Replaces the per-template host loop of
 * pygpuAAK.pyGPUAAK.NLL (pygpuAAK/pygpuAAK.py:204-232). */
int aak_batch_plan(aak_ctx *ctx, const aak_params *P, int32_t nsrc, const int32_t *nmodes_override, int32_t nthreads);

/* Plan from already mapped trajectories (one aak_mapped per source). */
int aak_batch_plan_mapped(aak_ctx *ctx, const aak_params *P, const aak_mapped *maps, int32_t nsrc,
                          const int32_t *nmodes_override, int32_t nthreads);

/* Batch geometry after planning: offsets (nsrc + 1 prefix of sample counts),
 * per-source status, plunge index and buffer length; any pointer may be NULL. */
int aak_batch_info(aak_ctx *ctx, int64_t *total_samples, int64_t *offsets, int32_t *status, int32_t *i_plunge,
                   int32_t *i_buffer);

/* Bytes aak_batch_upload copies to the device for the planned batch. */
int aak_batch_plan_bytes(aak_ctx *ctx, int64_t *bytes);

/* Copy the planned batch to the device (stream-ordered on `stream`, a
 * cudaStream_t or NULL for the legacy default stream). */
int aak_batch_upload(aak_ctx *ctx, void *stream);

/* Run the dense kernels into caller device buffers indexed by offsets:
 * hI, hII (required), t (optional), traj (optional 9 x traj_stride dense
 * trajectory e, v, M, S, gamma~, Phi, alpha, nu, gamma~dot; diagnostic).
 * precision: 0 = FP64 throughout; 1 = split precision (FP64 spline, phases
 * and angle reductions; FP32 geometry, LISA response, Bessel evaluation and
 * harmonic recurrence). */
int aak_batch_run(aak_ctx *ctx, double *d_hI, double *d_hII, double *d_t, double *d_traj, int64_t traj_stride,
                  int32_t precision, void *stream);

/* The AAK phase product (as aak_phase) of every source of the uploaded batch
 * into caller device memory: 8 rows of `stride` doubles (stride >= the
 * batch's total samples) -- t, phase_r, phase_theta, phase_phi, omega_r,
 * omega_theta, omega_phi, eccentricity -- each indexed by the batch offsets.
 * Batched counterpart of AAKphase (src/suite/AAKpy.cc:53-88); three kernels
 * (per-tile parameters, the phase pass, the post-plunge freeze). */
int aak_batch_run_phase(aak_ctx *ctx, double *d_out, int64_t stride, void *stream);

/* Plan + upload + phase product + copy back for nsrc sources: h_out holds
 * 8 rows of sum(P[s].length) doubles in the aak_batch_run_phase layout;
 * offsets (nsrc + 1) and status (nsrc) optional.  A source that fails has
 * status != 0 and zeros in its rows. */
int aak_phase_batch_host(aak_ctx *ctx, const aak_params *P, int32_t nsrc, int32_t nthreads, double *h_out,
                         int64_t *offsets, int32_t *status);

/* aak_tdi for nsrc sources in one batch: h_out holds 6 rows (Xr, Xi, Yr, Yi,
 * Zr, Zi) of sum((P[s].length + 1) / 2) doubles; source s starts at bin
 * bin_offsets[s] (nsrc + 1 entries, optional); status optional. */
int aak_tdi_batch_host(aak_ctx *ctx, const aak_params *P, int32_t nsrc, int32_t nthreads, double *h_out,
                       int64_t *bin_offsets, int32_t *status);

/* Allocation-free variant of aak_batch_run, for callers that cannot call
 * cudaMalloc: code whose device memory belongs to a host framework or a
 * pre-reserved pool (a sampler that owns the GPU's memory budget, a caching
 * allocator), where an allocation would synchronise the device or break the
 * budget.  No counterpart in the reference.
 * The caller passes the planned ctx (aak_batch_plan* only -- no upload),
 * one device buffer of its own for the plan (256-byte aligned, plan_bytes
 * long) and the outputs hI, hII (indexed by the batch offsets).  Call with
 * d_plan == NULL to receive the required size in *required_bytes.  The
 * precision is the context's (aak_ctx_set_precision: 0 FP64, the default, or
 * 1 split).  The tile scratch lives in a file-scope device array of
 * 4,849,920 bytes (about 4.9 MB) held by every GPU that loads the library
 * until exit; batches above 32768 tiles of 1024 samples (33,554,432 samples)
 * are rejected with AAK_ERR_CAPACITY.  Each call looks the array's address
 * up in the current context (no allocation), so the entry point stays usable
 * after a cudaDeviceReset.  Each call copies the plan from host memory into
 * d_plan on `stream`.  Every call shares the array: calls that overlap on the
 * GPU race.  Each call clears its
 * own look-back status word before its kernel, so a wait that gave up in an
 * earlier call does not affect it; a give-up is kept in a report word that
 * aak_batch_device_status of a context that made such a call reads and
 * clears (one word per device, shared by every context using this entry
 * point there).  Nothing here calls cudaMalloc, cudaFree or an allocating
 * library routine. */
int aak_batch_run_noalloc(aak_ctx *ctx, void *d_plan, int64_t plan_bytes, int64_t *required_bytes, double *d_hI,
                          double *d_hII, void *stream);

/* Number of CUDA kernels the last aak_batch_run (or aak_batch_run_phase)
 * launched. */
int aak_batch_last_launches(aak_ctx *ctx);

/* Waits for the device, then reports whether a bounded device-side wait of
 * the batch kernels gave up since the last upload or the last call (the
 * look-back of the phase scan; for a context that used
 * aak_batch_run_noalloc, that entry point's report word on the device
 * included): AAK_ERR_DEVICE_TIMEOUT, else AAK_OK.  Clears the condition. No
 * reference counterpart (the reference's kernels do not wait on one another). */
int aak_batch_device_status(aak_ctx *ctx);

/* Autotuner of the waveform stage's launch shape.  The candidates
 * (AAK_NUM_VARIANTS of them, per precision) are the tile pre-pass with bulk
 * copies or tables built inside the tiles, 1, 2 or 4 samples per thread in the
 * harmonic loop, and 2 or 3 resident CTAs per SM; tiles are 1024 samples in
 * every candidate (the host plan is laid out per tile).  On the context's
 * uploaded batch, with the caller's output buffers d_hI, d_hII, every
 * candidate runs once as a warm-up and twice timed (CUDA events); the fastest
 * becomes the context's choice for `precision`, used by aak_batch_run,
 * aak_batch_run_graph and the host-buffer entry points.  Key: device name and
 * SM count, precision, largest harmonic count, and the numbers of sources and
 * of samples of the median source in powers of two.  cache_path (optional): a
 * text file of "key variant ms_0 .. ms_5" lines; an entry for the key is used
 * without timing, a new choice is appended.  variant (optional) receives the
 * choice, ms_per_variant (optional, AAK_NUM_VARIANTS entries) the timings in
 * ms (-1 when read from the cache).  No reference counterpart: the
 * reference's launch shape is fixed (src/cuda/AAK_manager.cu:233, 245). */
#define AAK_NUM_VARIANTS 6
int aak_ctx_autotune(aak_ctx *ctx, double *d_hI, double *d_hII, int32_t precision, const char *cache_path,
                     int32_t *variant, float *ms_per_variant);
/* Set the launch shape of `precision` directly (0 .. AAK_NUM_VARIANTS - 1;
 * 0 is the default). */
int aak_ctx_set_variant(aak_ctx *ctx, int32_t precision, int32_t variant);

/* Bound of one look-back wait of this context's batch launches, in SM clocks
 * (<= 0: the default, about 2 s).  A wait that reaches it gives up, the tile
 * takes a zero carry and aak_batch_device_status reports
 * AAK_ERR_DEVICE_TIMEOUT: a watchdog for callers that want a shorter one.  No
 * reference counterpart. */
int aak_ctx_set_lookback_bound(aak_ctx *ctx, int64_t cycles);

/* Self-test of that bounded wait on the current device: one thread waits on a
 * look-back flag that nothing sets, for at most `cycles` SM clocks (a few
 * million: about a millisecond), and gives up.  Returns AAK_OK when the wait
 * gave up and reported it, AAK_ERR_CUDA otherwise.  Synchronous. */
int aak_selftest_lookback_timeout(int64_t cycles);

/* Per-kernel timing of aak_batch_run with CUDA events on its stream: after
 * aak_batch_set_profiling(ctx, 1), aak_batch_kernel_ms returns the durations
 * of (work-queue and look-back flag clears, the tile pre-pass -- 0 without
 * it --, the waveform kernel) of the last run in ms. */
int aak_batch_set_profiling(aak_ctx *ctx, int32_t on);
int aak_batch_kernel_ms(aak_ctx *ctx, float *ms3);

/* Plain FP64 per-source path (the baseline the batched paths are measured
 * against; no reference counterpart as an entry point): source by source,
 * the phase kernels write the dense FP64 trajectory (9 x traj_stride doubles
 * in d_traj: e, v, M, S, gamma~, Phi, alpha, nu, gamma~dot), then one thread
 * per sample evaluates the harmonic sum as the reference's CUDA port does
 * (src/cuda/kernel.cu:374-555): five jn() Bessel calls, cos/sin of n Phi and
 * the NK-frame rotation per harmonic.  Same outputs as aak_batch_run with
 * precision 0, to Bessel-evaluation rounding. */
int aak_batch_run_plain(aak_ctx *ctx, double *d_hI, double *d_hII, double *d_traj, int64_t traj_stride, void *stream);

/* The whole dense stage in one CUDA graph: the natural-spline solve of every
 * source's knots (as aak_batch_upload runs it; the same knots give the same
 * coefficients) and the three launches of aak_batch_run (no t / trajectory
 * outputs), captured on the first call for a given (d_hI, d_hII, precision,
 * upload) and replayed on later calls; a new upload or other outputs
 * recapture.  Capture runs on a stream of the context, so `stream`
 * may be the legacy default stream.  No reference counterpart: the
 * reference launches its kernels one by one with a device synchronisation
 * after each (src/cuda/AAK_manager.cu:154-260). */
int aak_batch_run_graph(aak_ctx *ctx, double *d_hI, double *d_hII, int32_t precision, void *stream);

/* Precision of the host-buffer entry points of this context
 * (aak_wave_batch_host): 0 = FP64 throughout (default), 1 = split. */
int aak_ctx_set_precision(aak_ctx *ctx, int32_t precision);

/* Diagnostic: sustained FP32 FMA rate of `device` in TFLOP/s (roofline denominator of the split path). */
int aak_probe_fp32_tflops(int32_t device, double *tflops);

/* Diagnostic: sustained FP64 FMA rate of `device` in TFLOP/s (roofline denominator). */
int aak_probe_fp64_tflops(int32_t device, double *tflops);

/* End to end with host buffers: plan + upload + run + copy back.
 * h_hI / h_hII hold total_samples doubles (offsets as from aak_batch_info).
 * From 32 sources on, the call streams: groups of sources that finished
 * planning are uploaded, generated and copied back on two internal contexts
 * while the others are still planned; page-locked output buffers let those
 * copies overlap.  Either way the context holds the whole batch's plan
 * afterwards (as after aak_batch_plan). */
int aak_wave_batch_host(aak_ctx *ctx, const aak_params *P, int32_t nsrc, const int32_t *nmodes_override,
                        int32_t nthreads, double *h_hI, double *h_hII, int64_t *offsets, int32_t *status);

/* ------------------------------------------------------------------ GPU likelihood */
/* Counterpart of the reference class GPUAAK (include/AAK_manager.hh:106-153,
 * src/cuda/AAK_manager.cu, pygpuAAK/GPUAAK.pyx:50-93), on the current CUDA
 * device.  init_length / init_dt are accepted for call compatibility; the
 * coarse grid follows the reference CPU AAK.  Templates are generated with
 * the reference CPU conventions (the AAKwave path, src/suite/AAK.cc), not the
 * GPU port's own coarse grid. */
typedef struct aak_gpu aak_gpu;

/* GPUAAK(T_fit, init_length, length, init_dt, dt, LISA, backint) */
int aak_gpu_create(double T_fit, int32_t init_length, int32_t length, double init_dt, double dt, int32_t LISA,
                   int32_t backint, aak_gpu **out);
void aak_gpu_destroy(aak_gpu *g);

/* input_data (AAK_manager.cu:135-152): pre-weighted data spectra of both
 * channels as interleaved complex (2 x len doubles) and the weights
 * S_n^{-1/2} sqrt(dt/N) (len doubles); len must be length/2 + 1. */
int aak_gpu_input_data(aak_gpu *g, const double *hI_f, const double *hII_f, const double *ASDinv1,
                       const double *ASDinv2, int32_t len);

/* gpu_gen_AAK (AAK_manager.cu:154-260): pars14 = iota, s, p, e, M, mu, gamma,
 * psi, alph, theta_S, phi_S, theta_K, phi_K, D. */
int aak_gpu_gen(aak_gpu *g, const double *pars14);

/* GetWaveform (AAK_manager.cu:454-458): t, hI, hII of length+2 doubles; after
 * aak_gpu_likelihood hI/hII hold the interleaved half spectra. */
int aak_gpu_get_waveform(aak_gpu *g, double *t, double *hI, double *hII);

/* Likelihood (AAK_manager.cu:352-446): out2 = [4 Re<h|d>, 4 <h|h>]. */
int aak_gpu_likelihood(aak_gpu *g, double *out2);

/* Batched likelihoods (no reference counterpart; replaces the serial loop of
 * pygpuAAK.py:204-232): params nsrc x 14 (gpu_gen_AAK order), out nsrc x 2,
 * per-template status (optional).  Templates run in batches of max_batch
 * (<= 0: 256); host planning uses nthreads threads (<= 0: all). */
int aak_gpu_likelihood_batch(aak_gpu *g, const double *params, int32_t nsrc, int32_t max_batch, int32_t nthreads,
                             double *out, int32_t *status);

/* Fisher-matrix Gram sums of one point (replaces the template loop and host
 * dot products of pyGPUAAK.get_Fisher, pygpuAAK/pygpuAAK.py:269-300):
 * params holds 2 nd rows x 14 (gpu_gen_AAK order, 1 <= nd <= 16), rows 2i
 * and 2i + 1 the two evaluations of derivative i.  The 2 nd templates are
 * generated as one batch, transformed, weighted by the input_data weights w,
 * and reduced on the device: D_i = scale w (FFT h_{2i+1} - FFT h_{2i}),
 * gram[c nd^2 + i nd + j] = 4 Re sum_f conj(D_i) D_j for channels c = I, II
 * (2 x nd x nd, symmetric).  status (optional, 2 nd) per template. */
int aak_gpu_fisher(aak_gpu *g, const double *params, int32_t nd, double scale, int32_t nthreads, double *gram,
                   int32_t *status);

/* Fisher-matrix Gram sums of npts points in one call (the reference computes
 * one point per get_Fisher call, pygpuAAK/pygpuAAK.py:269-300; this is its
 * loop over points): params holds npts blocks of 2 nd rows x 14, each laid
 * out as for aak_gpu_fisher, and gram npts blocks of 2 x nd x nd, block k
 * equal to aak_gpu_fisher of block k of params.  Point k + 1 is planned on
 * host threads into a second planning context while the device generates,
 * transforms and reduces point k.  status (optional, npts x 2 nd) per
 * template. */
int aak_gpu_fisher_batch(aak_gpu *g, const double *params, int32_t npts, int32_t nd, double scale, int32_t nthreads,
                         double *gram, int32_t *status);

/* Template precision: 0 = FP64 throughout (default), 1 = split (FP64 phases
 * and angle reductions, FP32 geometry, response, Bessel evaluation), 2 =
 * split templates written as FP32 rows, an FP32 R2C transform and FP32 inner
 * products with Kahan-compensated sums (aak_gpu_likelihood_batch only; the
 * other calls run as precision 1). */
int aak_gpu_set_precision(aak_gpu *g, int32_t precision);

/* Launch shape of the template waveform stage for `precision` (0 FP64, 1
 * split, also used by precision 2): one of the AAK_NUM_VARIANTS candidates of
 * aak_ctx_autotune, applied to both planning contexts of the batches.  No
 * reference counterpart (the reference's launch shape is fixed,
 * src/cuda/AAK_manager.cu:233,245). */
int aak_gpu_set_variant(aak_gpu *g, int32_t precision, int32_t variant);

/* Milliseconds of the last batch: host planning, waveform kernels, FFT, reduction. */
int aak_gpu_last_timing(aak_gpu *g, double *ms4);

/* ------------------------------------------------------------------ learned ParMap warm start */
/* No reference counterpart: a 4 -> 128 -> 128 -> 128 -> 3 SiLU network (BF16
 * weights and activations, FP32 accumulation, tcgen05 tensor cores for the
 * 128 x 128 layers) that predicts the solution of the Kerr -> AK map
 * (ParMap, src/suite/KSParMap.cc:397-440) from (p, e, iota, a), as the
 * initial guess of the plain Newton solve, which stays the fallback and the
 * judge (|f|_1 < 1e-6).  Outputs are map coordinates
 * y = (v_map sqrt(p), M_map / M, s_map - a).  Parameters are one FP32 vector
 * of aak_mlp_num_params() values: W1[128][4] b1 W2[128][128] b2 W3[128][128]
 * b3 W4[3][128] b4.  Inputs enter as ((1/sqrt(p), e, cos iota, a) - in_shift)
 * * in_scale; outputs leave as net * out_scale + out_shift. */
typedef struct aak_mlp aak_mlp;

int aak_mlp_num_params(void);
int aak_mlp_max_train_rows(void);
int aak_mlp_create(int32_t device, aak_mlp **out);
void aak_mlp_destroy(aak_mlp *m);
/* Host FP32 parameters in / out; set_params also resets the Adam state. */
int aak_mlp_set_params(aak_mlp *m, const float *params);
int aak_mlp_get_params(aak_mlp *m, float *params);
int aak_mlp_set_norm(aak_mlp *m, const float in_shift[4], const float in_scale[4], const float out_shift[3],
                     const float out_scale[3]);
int aak_mlp_set_adam(aak_mlp *m, float beta1, float beta2, float eps);
/* Device pointers: d_x n x 4 (p, e, iota, a), d_y n x 3 map coordinates. */
int aak_mlp_forward(aak_mlp *m, const float *d_x, float *d_y, int64_t n, void *stream);
/* Gradient of the mean squared error in normalised output units over rows
 * d_perm[0..n) (d_perm NULL: rows 0..n) of (d_x, d_y); n <= aak_mlp_max_train_rows().
 * d_grad: aak_mlp_num_params() floats (device).  *loss (optional, host)
 * synchronises the stream. */
int aak_mlp_gradients(aak_mlp *m, const float *d_x, const float *d_y, const int32_t *d_perm, int64_t n, float *d_grad,
                      float *loss, void *stream);
/* One Adam step (learning rate lr) on the same loss. */
int aak_mlp_train_step(aak_mlp *m, const float *d_x, const float *d_y, const int32_t *d_perm, int64_t n, float lr,
                       float *loss, void *stream);
/* AAK_ERR_DEVICE_TIMEOUT if a kernel of the model gave up a bounded wait. */
int aak_mlp_status(aak_mlp *m);
/* Host convenience: x n x 4 -> y n x 3 (synchronous). */
int aak_mlp_predict_host(aak_mlp *m, const double *x, double *y, int64_t n);

/* Separatrix p_sep(e, iota, a) by bisection on geodesic stability (the test
 * of the reference's LSO search, src/suite/GKTrajFast.cc constructor). */
int aak_parmap_separatrix(double e, double iota, double a, double *p_sep);
/* Points first_index .. first_index + n - 1 of the seeded distribution
 * p ~ U(p_sep + 0.1, 20), e ~ U(0, 0.7) (redrawn below 1e-3), iota ~ U(0, pi),
 * a ~ U(0, 0.95), labelled by the plain map solve at M = 1e6: x n x 4, y n x 3
 * (map coordinates, NaN where the solve failed), omega n x 3 Kerr frequencies,
 * iters n (Newton iterations; < 0: failed). */
int aak_parmap_dataset(int64_t n, uint64_t seed, uint64_t first_index, int32_t nthreads, double *x, double *y,
                       double *omega, int32_t *iters);
/* Map solves from the guesses (n x 3 map coordinates; NULL: the reference's
 * plain initial guess).  A guess whose solve fails the residual test, or
 * converges more than 0.05 (in map coordinates) away from the guess, is
 * re-solved from the plain guess (fallback[i] = 1; iters counts both).
 * iters: Newton iterations to the converged (rounding-level) solution;
 * iters_to_tol (optional): iterations until |f|_1 < 1e-6, the reference's
 * stopping test (-1: never reached). 
 * residual / guess_residual: |f|_1 at the solution / at the guess (optional). */
int aak_parmap_solve_batch(int64_t n, const double *x, const double *omega, const double *guess, int32_t nthreads,
                           double *y, int32_t *iters, int32_t *iters_to_tol, double *residual, double *guess_residual,
                           int32_t *fallback);

/* Batch planning with the warm start: every coarse point of every source is
 * predicted in one launch, then solved from its prediction.  m NULL restores
 * the plain initial guess.  The model must outlive its use by the context. */
int aak_ctx_set_parmap_model(aak_ctx *ctx, aak_mlp *m);
/* Map statistics of the last plan: coarse points solved, Newton iterations,
 * warm starts that fell back to the plain guess. */
int aak_batch_newton_stats(aak_ctx *ctx, int64_t *points, int64_t *iterations, int64_t *fallbacks);
/* The same for the likelihood object's template batches. */
int aak_gpu_set_parmap_model(aak_gpu *g, aak_mlp *m);

/* Solve the Kerr->AK map of every coarse point of a batch on the GPU (one
 * launch after the host's coarse inspirals) instead of on the planning
 * threads.  Part of the batched front end the reference has no counterpart
 * for; the device solve performs the host's operations in the same order
 * without fused multiply-adds, so the mapped trajectories, and every output,
 * are the same bit for bit.  on = 0 (default) solves on the host.  Not for
 * host-only contexts. */
int aak_ctx_set_parmap_device(aak_ctx *ctx, int32_t on);
int aak_gpu_set_parmap_device(aak_gpu *g, int32_t on);

/* Coarse AK evolution of a batch on the GPU: planning runs in three passes
 * (front end, map and fit window on host threads; every source's AK
 * recurrence beyond the fit window in one launch, one GPU thread per source;
 * fitted knots and plunge search on host threads) instead of the host's
 * grouped recurrences (AAK.cc:62-144 is the reference's serial loop).  The
 * device rounds as the host does except in log(), so knots agree to about
 * 1e-15 relative rather than bit for bit.  on = 0 (default): host.  Not for
 * host-only contexts.  No reference counterpart. */
int aak_ctx_set_evolve_device(aak_ctx *ctx, int32_t on);
/* Wall times of the last plan with the device evolution, in ms: the host
 * pass before it, the device pass (copies included), the host pass after it,
 * and the total.  Zero for plans without it. */
int aak_batch_plan_ms(aak_ctx *ctx, double *ms4);

/* ---------------------------------------------------------------- several devices
 * Split of one batch over `parts` devices (or ranks): the reference's
 * pyGPUAAK accepts an ndevices argument and evaluates every template on one
 * device in a serial loop (pygpuAAK/pygpuAAK.py:31, 204-232).  Here a batch of
 * n units with costs cost[i] (samples x harmonics for waveforms; equal for the
 * templates of one likelihood batch) is divided by greedy LPT: units in
 * decreasing cost, each to the part with the least cost so far, ties to the
 * lowest index (the split depends on the costs alone, so every rank computes
 * the same one).  assign[i] receives the part of unit i; load (optional,
 * `parts` entries) the summed cost per part.  Host only. */
int aak_lpt_partition(const double *cost, int64_t n, int32_t parts, int32_t *assign, double *load);

#ifdef __cplusplus
}
#endif

#endif /* AAK_B200_H */
