// pipeline.hpp -- host half of the AAK waveform: parameter record, the front
// end (coarse Kerr inspiral -> Kerr frequencies -> Kerr-to-AK parameter map)
// and the coarse AK evolution that yields the spline knots the dense kernels
// interpolate.  Everything here is re-entrant (no static state).
#pragma once

#include "parmap_newton.hpp"
#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdlib>
#include <cstring>
#include <new>
#include <memory>
#include <vector>

#include "../aak_common.hpp"

namespace aak {

// Status codes returned through the C-ABI (mirrored in include/aak.h).
enum Status : int32_t {
  kOk = 0,
  kErrInvalidParam = 1,
  kErrUnstableStart = 2,       // p0 inside the last stable orbit
  kErrFitTooCloseToPlunge = 3, // fewer than three usable fit points
  kErrSolverNoConverge = 4,    // Kerr->AK map did not converge
  kErrCuda = 5,
  kErrNoMemory = 6,
  kErrTooFewSteps = 7,         // coarse inspiral produced < 3 points
  kErrCapacity = 8,            // request larger than a fixed-size buffer
};

// Numeric fields of the reference SetPar record (include/KSTools.h:21-53).
struct Params {
  int64_t length;
  double dt, p, T, f, T_fit, mu, M, s, e, iota, gamma, psi, theta_S, phi_S, theta_K, phi_K, alpha, D;
  int32_t backint, LISA;
};

constexpr int kMaxCoarseSteps = 100;  // the reference's maxsteps (AAKpy.cc:23)

// What the reference front end hands to GenWave (AAKpy.cc:20-44).
struct MappedTrajectory {
  int steps = 0;
  double e_traj[kMaxCoarseSteps];
  double v_map[kMaxCoarseSteps];
  double M_map[kMaxCoarseSteps];
  double s_map[kMaxCoarseSteps];
  double dt_map[kMaxCoarseSteps];
  double Phi0 = 0;
  int inspiral_flag = 0;
  int newton_iterations = 0;  // total Kerr->AK Newton iterations over all points
};

// Kerr fundamental frequencies at each coarse inspiral point, for callers
// that want to solve the map themselves (e.g. with a learned warm start).
struct CoarseKerr {
  int steps = 0;
  double t_rr[kMaxCoarseSteps], p[kMaxCoarseSteps], e[kMaxCoarseSteps], cosi[kMaxCoarseSteps];
  double Omega[kMaxCoarseSteps][3];
  int inspiral_flag = 0;
};

int validate(const Params &P);
int coarse_kerr(const Params &P, CoarseKerr *out);

// Kerr -> AK map at one point (KSParMap.cc:397-440): solve for
// x = (v_map, M_map, s_map).  x0 == nullptr uses the reference's initial
// guess (1/sqrt(p), M, s).  The solve first reaches the reference's stopping
// test |f|_1 < 1e-6 (after *iters_to_tol iterations, optional; -1 never) and
// then polishes until the Newton step stalls at rounding level.  Returns the
// Newton iterations (< 0 on failure).
int parmap(const double Omega[3], double p, double M, double s, double e, double iota, const double *x0, double map[3],
           int *iters_to_tol = nullptr);

// The map from a warm guess.  The plain solve from the reference's guess
// redoes a point when the warm solve fails the residual test or converges
// farther than kWarmAcceptance (in v_map sqrt(p), M_map / M, s_map) from the
// guess; *fallback (optional) is set then.  Returns the Newton iterations of
// both solves (< 0 on failure).
int parmap_warm(const double Omega[3], double p, double M, double s, double e, double iota, const double guess[3],
                double map[3], int *fallback, int *iters_to_tol = nullptr);

// Initial mean anomaly from the initial true anomaly psi (KSParMap.cc:25).
double initial_mean_anomaly(double e, double psi);

// Full front end (AAKpy.cc:20-44).  warm (optional, steps x 3) seeds the map.
int front_end(const Params &P, MappedTrajectory *out, const double *warm = nullptr);
// Second half of the front end: the map at every coarse point of ck.  Points
// whose warm solve fails the residual test are re-solved from the plain
// initial guess and counted in *fallbacks (optional).
int map_coarse(const Params &P, const CoarseKerr &ck, MappedTrajectory *out, const double *warm, int *fallbacks);

// Inputs of the reference GenWave/waveform (AAK.cc:321, 565).
struct WaveInputs {
  double timestep;
  int vlength;
  int nmodes;
  double zeta;
  double par[12];
  const double *e_traj, *v_map, *M_map, *S_map, *dt_map;
  double M_phys, S_phys;
  int steps;
  int backint;
  int mich;
};

// Pack GenWave's par[12], zeta and harmonic count (AAK.cc:565-591).
void genwave_inputs(const Params &P, const MappedTrajectory &mt, int nmodes_override, WaveInputs *w);

// Growable array for a source's knots.  With want_pinned it lives in
// page-locked host memory (falling back to pageable memory when that fails,
// e.g. without a GPU), so that the batch upload copies straight from it to the
// device with no host-side repacking.  Capacity is kept across plans; growth
// keeps the contents, like std::vector::resize, but new elements are not
// initialised.
template <typename T>
struct KnotBuf {
  T *p = nullptr;
  size_t n = 0, cap = 0;
  bool pinned = false, want_pinned = false;
  KnotBuf() = default;
  KnotBuf(const KnotBuf &) = delete;
  KnotBuf &operator=(const KnotBuf &) = delete;
  KnotBuf(KnotBuf &&o) noexcept { take(o); }
  KnotBuf &operator=(KnotBuf &&o) noexcept {
    if (this != &o) {
      release();
      take(o);
    }
    return *this;
  }
  ~KnotBuf() { release(); }
  void resize(size_t m) {
    if (m > cap) {
      const size_t want = m + m / 8;
      void *q = nullptr;
      bool pin = false;
      if (want_pinned && cudaHostAlloc(&q, want * sizeof(T), cudaHostAllocPortable) == cudaSuccess) {
        pin = true;
      } else {
        if (want_pinned) cudaGetLastError();
        q = std::malloc(want * sizeof(T));
        if (!q) throw std::bad_alloc();
      }
      if (n) std::memcpy(q, p, n * sizeof(T));
      release_storage();
      p = static_cast<T *>(q);
      cap = want;
      pinned = pin;
    }
    n = m;
  }
  void clear() { n = 0; }
  T *data() { return p; }
  const T *data() const { return p; }
  size_t size() const { return n; }
  T &operator[](size_t i) { return p[i]; }
  const T &operator[](size_t i) const { return p[i]; }

 private:
  void take(KnotBuf &o) {
    p = o.p;
    n = o.n;
    cap = o.cap;
    pinned = o.pinned;
    want_pinned = o.want_pinned;
    o.p = nullptr;
    o.n = o.cap = 0;
  }
  void release_storage() {
    if (p) {
      if (pinned) cudaFreeHost(p);
      else std::free(p);
    }
    p = nullptr;
  }
  void release() {
    release_storage();
    n = cap = 0;
  }
};

// Coarse AK evolution and spline knots (AAK.cc:27-242): everything of
// PNevolution except the dense loops, which the kernels perform.
struct SourcePlan {
  int status = kOk;
  int vlength = 0;
  int i0 = 0, i_plunge = 0, i_buffer = 0;
  int nmodes = 0;
  double dt = 0, t_first = 0, t_last = 0;
  double e_max = 0;
  KnotBuf<double> knot_t;       // n_knots
  KnotBuf<double> knot_y;       // n_knots x 4 (e, v, M, S): the layout of double4[n_knots]
                                // (the spline coefficients are solved on the device)
  SourceDesc desc;              // offsets filled in by the batch builder
};

int plan_source(const WaveInputs &w, SourcePlan *plan);
// plan_source of two sources on one thread, their coarse AK evolutions
// interleaved (same results; each plan's status in its own plan->status).
void plan_source_pair(const WaveInputs &wa, SourcePlan *pa, const WaveInputs &wb, SourcePlan *pb);
// plan_source of up to kPlanGroup sources on one thread: their coarse AK
// evolutions run in the lanes of kPlanGroup / 4 AVX2 vectors (where the CPU
// has AVX2 and all kPlanGroup plan_heads succeed), else two interleaved;
// every plan equals plan_source's bit for bit.  Each plan's status is in
// plan->status.  Four measured faster than eight on the 512-source
// configuration-1 batch: a group waits for its longest member.
constexpr int kPlanGroup = 4;
static_assert(kPlanGroup % 4 == 0, "whole AVX2 vectors");
void plan_source_group(const WaveInputs *const w[], SourcePlan *const p[], int n);
// Per-source geometry constants of the waveform (orientation fields set).
void fill_geometry(SourceDesc *d);

// plan_source split at the coarse AK evolution beyond the fit window, so
// that the recurrence can run elsewhere (one GPU thread per source,
// ak_evolve.cu).  Indices are relative to j0, the first knot of the fit
// window: a source's AK (e, v) occupy entries 0 .. j_end of a segment at
// `off` in the batch's arrays; the fit window fills entries 0 .. j_first and
// the recurrence entries j_first + 1 .. j_end, with evolve()'s freezing.
struct EvolveJob {
  int64_t off;                // the source's first entry in the batch's e, v arrays
  int32_t j_first, j_end;     // the recurrence computes entries j_first + 1 .. j_end
  int32_t j_max, j_max_temp;  // freeze indices: in, after the fit window; out, after the recurrence
  double edot, vdot;          // AK rates of the step before j_first (out: of the last step)
  double coslam, mu, M0, S0, dt_large;
};
struct PlanCarry;  // a source's planning state between the two halves
struct PlanCarryDelete {
  void operator()(PlanCarry *c) const;
};
using PlanCarryPtr = std::unique_ptr<PlanCarry, PlanCarryDelete>;
// The first half (the fit window and its corrections).  Returns plan->status;
// on success *carry holds the state (w and plan must outlive it) and *job the
// recurrence (off left to the caller).
int plan_source_begin(const WaveInputs &w, SourcePlan *plan, PlanCarryPtr *carry, EvolveJob *job);
// e, v of the fit window: entries 0 .. job.j_first.
void plan_carry_prefix(const PlanCarry &c, const EvolveJob &job, double *e, double *v);
// The second half, with e, v holding entries 0 .. job.j_end and the job's
// outputs: the fitted knots, the plunge search and the descriptor, as
// plan_source.  Returns plan->status.
int plan_source_end(PlanCarry &c, const EvolveJob &job, const double *e, const double *v);

// (e, v, M, S) of the natural spline through the n knots (x, y[4 n]) at xv,
// with the coefficients of its piece from the windowed solve the device
// applies to every knot (no full solve).
void spline_eval4_local(const double *x, const double *y, int n, double xv, double out[4]);

// Miller start order for J_{n-2..n+2+extra}(n e) accurate to ~1e-17 for all e <= e_max.
int bessel_start_order(int n, double e_max, int extra = 0);

}  // namespace aak
