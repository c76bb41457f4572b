// aak_capi.cpp -- the extern "C" surface declared in include/aak.h: batch
// planning on host threads, device buffers of a context, kernel launches.
#include "aak.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <condition_variable>
#include <functional>
#include <thread>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <mutex>
#include <thread>
#include <vector>

#include <cufft.h>

#include "../host/parallel.hpp"
#include "../host/parmap_data.hpp"
#include "../host/pipeline.hpp"
#include "../kernels/aak_dense.cuh"
#include "../kernels/ak_evolve.cuh"
#include "../kernels/likelihood.cuh"
#include "../kernels/parmap_newton.cuh"
#include "errors.hpp"
#include "mlp_model.hpp"

using namespace aak;

namespace {

template <typename T>
struct DevBuf {
  T *ptr = nullptr;
  size_t cap = 0;
  int reserve(size_t n) {
    if (n <= cap && ptr) return AAK_OK;
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    cap = 0;
    size_t want = std::max<size_t>(n, 1);
    want += want / 4;  // growth headroom
    if (cudaMalloc(&ptr, want * sizeof(T)) != cudaSuccess) {
      cudaGetLastError();
      ptr = nullptr;
      return AAK_ERR_NO_MEMORY;
    }
    cap = want;
    return AAK_OK;
  }
  void release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    cap = 0;
  }
};

int cuda_ok(cudaError_t e) { return cuda_status_of(e); }


}  // namespace

struct aak_ctx {
  int device = 0;
  int num_sms = 148;
  // host plan
  int32_t nsrc = 0;
  std::vector<SourcePlan> plans;
  std::vector<int64_t> offsets;
  std::vector<int32_t> status;
  std::vector<SourceDesc> descs;
  std::vector<int64_t> tile_start;
  std::vector<int64_t> tile_pairs;  // per source {0, its tiles}: the tile prefix of a one-source view
  std::vector<QueueItem> queue;     // work-queue order of the tiles, with what staging each needs
  std::vector<int32_t> tile_knot;  // 2 per tile: first knot of the tile window, knots in it
  std::vector<int64_t> kofs;       // nsrc + 1 prefix of knots (the sources' knots stay in their plans)
  std::vector<int64_t> spl_blk;    // nsrc + 1 prefix of the device spline solve's blocks
  bool want_pinned = true;         // plans' knot arrays in page-locked memory
  std::vector<int32_t> bessel;
  int64_t total_samples = 0, total_tiles = 0, total_knots = 0;
  int32_t max_nmodes = 0;
  int64_t out_stride = 0;  // > 0: source s writes at s * out_stride (FFT-padded rows)
  bool uploaded = false;
  // device buffers
  DevBuf<SourceDesc> d_src;
  DevBuf<int64_t> d_tile_start, d_tile_pairs, d_spl_blk;
  DevBuf<QueueItem> d_queue;
  DevBuf<int32_t> d_tile_knot;
  DevBuf<double> d_knot_t;
  DevBuf<double4> d_knot_y, d_knot_c;
  DevBuf<int32_t> d_bessel;
  DevBuf<TileLink> d_link;                // look-back records, one per tile
  DevBuf<int32_t> d_flag;                 // look-back flags, one per tile
  DevBuf<unsigned long long> d_counter;   // [0] work-queue head, [1] device status word
  DevBuf<TilePrep> d_tile_prep;           // tile pre-pass: per-tile parameters
  DevBuf<unsigned char> d_tile_tab;       //   and per-tile Taylor tables
  DevBuf<double> d_out;  // outputs for the host-buffer entry points
  // batched device solve of the Kerr -> AK map (opt-in: parmap_device)
  bool parmap_device = false;
  bool evolve_device = false;      // coarse AK evolution of a batch on the GPU (one thread per source)
  double plan_ms[4] = {0, 0, 0, 0};  // last plan: before / on the device / after the evolution, total
  DevBuf<ParmapJob> d_pm_jobs;
  DevBuf<double> d_pm_warm, d_pm_map;
  DevBuf<int32_t> d_pm_it;
  cudaStream_t pm_stream = nullptr;
  DevBuf<TdiDesc> d_tdi;        // frequency-domain TDI: per-source stationary-phase records
  DevBuf<int64_t> d_tdi_work;   //   and the prefix of their work items
  int last_launches = 0;
  bool profile = false;
  aak_mlp *model = nullptr;  // learned warm start of the map (optional)
  int precision = 0;         // precision of the host-buffer entry points and of aak_batch_run_noalloc
  bool noalloc_used = false; // an allocation-free launch ran since the last status query
  long long lookback_cycles = 0;  // bound of one look-back wait in SM clocks (<= 0: the kernels' default, about 2 s)
  uint64_t upload_gen = 0;   // bumped by every upload (device buffers may move)
  // CUDA graph of the dense launch (clears + waveform kernel) for fixed outputs / precision / upload
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  cudaStream_t cap_stream = nullptr;
  // streamed host-buffer batches: two auxiliary contexts, each with its own stream
  aak_ctx *aux[2] = {nullptr, nullptr};
  cudaStream_t pipe_stream = nullptr;
  double *g_hI = nullptr, *g_hII = nullptr;
  int g_prec = -1;
  uint64_t g_gen = ~0ull;
  int g_variant = -1;
  int variant[2] = {0, 0};  // launch shape of the waveform stage per precision (autotuner; 0: default)
  int64_t newton_points = 0, newton_iters = 0, newton_fallbacks = 0;
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  std::mutex mu;
};

namespace {

int select_device(int dev) {
  if (dev < 0) return AAK_ERR_INVALID_PARAM;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) {
    cudaGetLastError();
    return AAK_ERR_CUDA;
  }
  if (dev < 0 || dev >= n) return AAK_ERR_INVALID_PARAM;
  return cuda_ok(cudaSetDevice(dev));
}

Params to_params(const aak_params &a) {
  Params P;
  P.length = a.length;
  P.dt = a.dt;
  P.p = a.p;
  P.T = a.T;
  P.f = a.f;
  P.T_fit = a.T_fit;
  P.mu = a.mu;
  P.M = a.M;
  P.s = a.s;
  P.e = a.e;
  P.iota = a.iota;
  P.gamma = a.gamma;
  P.psi = a.psi;
  P.theta_S = a.theta_S;
  P.phi_S = a.phi_S;
  P.theta_K = a.theta_K;
  P.phi_K = a.phi_K;
  P.alpha = a.alpha;
  P.D = a.D;
  P.backint = a.backint;
  P.LISA = a.LISA;
  return P;
}

void to_mapped(const MappedTrajectory &m, aak_mapped *o) {
  std::memset(o, 0, sizeof(*o));
  o->steps = m.steps;
  o->inspiral_flag = m.inspiral_flag;
  o->newton_iterations = m.newton_iterations;
  o->Phi0 = m.Phi0;
  for (int i = 0; i < m.steps; ++i) {
    o->e_traj[i] = m.e_traj[i];
    o->v_map[i] = m.v_map[i];
    o->M_map[i] = m.M_map[i];
    o->s_map[i] = m.s_map[i];
    o->dt_map[i] = m.dt_map[i];
  }
}

void from_mapped(const aak_mapped &o, MappedTrajectory *m) {
  m->steps = std::min<int>(o.steps, kMaxCoarseSteps);
  m->inspiral_flag = o.inspiral_flag;
  m->newton_iterations = o.newton_iterations;
  m->Phi0 = o.Phi0;
  for (int i = 0; i < m->steps; ++i) {
    m->e_traj[i] = o.e_traj[i];
    m->v_map[i] = o.v_map[i];
    m->M_map[i] = o.M_map[i];
    m->s_map[i] = o.s_map[i];
    m->dt_map[i] = o.dt_map[i];
  }
}


// Pack per-source plans into the flat arrays the kernels read.
int pack(aak_ctx *ctx, const std::vector<aak_params> &P, int nthreads) {
  const int n = ctx->nsrc;
  ctx->offsets.assign(n + 1, 0);
  ctx->tile_start.assign(n + 1, 0);
  ctx->descs.resize(n);
  int64_t knots = 0, bes = 0;
  for (int s = 0; s < n; ++s) {
    const SourcePlan &pl = ctx->plans[s];
    const int64_t len = P[s].length;
    ctx->offsets[s + 1] = ctx->offsets[s] + (ctx->out_stride > 0 ? ctx->out_stride : len);
    ctx->tile_start[s + 1] = ctx->tile_start[s] + (len + kTileSamples - 1) / kTileSamples;
    if (ctx->status[s] == AAK_OK) {
      knots += (int64_t)pl.knot_t.size();
      bes += pl.nmodes;
    }
  }
  ctx->max_nmodes = 0;
  for (int s = 0; s < n; ++s)
    if (ctx->status[s] == AAK_OK) ctx->max_nmodes = std::max(ctx->max_nmodes, (int32_t)ctx->plans[s].nmodes);
  ctx->total_samples = ctx->offsets[n];
  ctx->total_tiles = ctx->tile_start[n];
  ctx->total_knots = knots;
  ctx->bessel.resize(std::max<int64_t>(bes, 1));
  // per-source offsets into the device arrays; the knots themselves are
  // uploaded from each plan's page-locked arrays (no host-side repacking)
  std::vector<int64_t> &kofs = ctx->kofs;
  kofs.assign(n + 1, 0);
  std::vector<int64_t> bofs(n + 1, 0);
  for (int s = 0; s < n; ++s) {
    const bool ok = ctx->status[s] == AAK_OK;
    kofs[s + 1] = kofs[s] + (ok ? (int64_t)ctx->plans[s].knot_t.size() : 0);
    bofs[s + 1] = bofs[s] + (ok ? ctx->plans[s].nmodes : 0);
  }
  ctx->spl_blk.assign(n + 1, 0);
  for (int s = 0; s < n; ++s)
    ctx->spl_blk[s + 1] = ctx->spl_blk[s] + (ctx->status[s] == AAK_OK ? spline_blocks((int)ctx->plans[s].knot_t.size()) : 0);
  ctx->tile_pairs.assign(2 * (size_t)n, 0);
  for (int s = 0; s < n; ++s) ctx->tile_pairs[2 * s + 1] = ctx->tile_start[s + 1] - ctx->tile_start[s];
  ctx->tile_knot.assign(2 * std::max<int64_t>(ctx->total_tiles, 1), 0);
  parallel_for(n, nthreads, [&](int64_t s64) {
    const int s = (int)s64;
    SourceDesc d;
    const SourcePlan &pl = ctx->plans[s];
    if (ctx->status[s] == AAK_OK) {
      d = pl.desc;
      const int64_t ko = kofs[s], bo = bofs[s];
      d.knot_offset = ko;
      d.bessel_offset = (int32_t)bo;
      for (int m = 1; m <= pl.nmodes; ++m) ctx->bessel[bo + m - 1] = bessel_start_order(m, pl.e_max, 12);  // table rows reach order n + 2 + 12
    } else {
      std::memset(&d, 0, sizeof(d));
      d.status = ctx->status[s];
      d.vlength = (int32_t)P[s].length;
    }
    d.out_offset = ctx->offsets[s];
    d.tile_offset = ctx->tile_start[s];
    d.n_tiles = (int32_t)(ctx->tile_start[s + 1] - ctx->tile_start[s]);
    ctx->descs[s] = d;
    if (ctx->status[s] != AAK_OK) return;
    // knot window of every tile: knots bracketing samples start-1 .. start+1024.
    // k0 is the last knot in [k0, nk - 2] with kt[k0] <= ta (kept at least at
    // its previous value), k1 the same for tb; found by binary search, so the
    // cost follows the tiles, not the knots (sources may have thousands of
    // knots per tile)
    const double *kt = pl.knot_t.data();
    const int nk = d.n_knots;
    auto tsample = [&](int i) { return (i == 0) ? d.t_first : (double)(i - d.i0) * d.dt; };
    auto last_le = [&](int lo, double x) {  // largest k in [lo, nk - 2] with kt[k] <= x, else lo
      if (lo + 1 > nk - 2) return lo;
      return (int)(std::upper_bound(kt + lo + 1, kt + nk - 1, x) - kt) - 1;
    };
    int k0 = 0, k1 = 0;
    for (int64_t t = 0; t < d.n_tiles; ++t) {
      const int start = (int)(t * kTileSamples);
      const double ta = tsample(std::max(start - 1, 0));
      const double tb = tsample(std::min(start + kTileSamples, d.vlength - 1));
      k0 = last_le(k0, ta);
      k1 = last_le(std::max(k1, k0), tb);
      ctx->tile_knot[2 * (d.tile_offset + t)] = k0;
      ctx->tile_knot[2 * (d.tile_offset + t) + 1] = k1 + 2 - k0;
    }
  });
  // work-queue order: chain step major, source minor.  Step 0 of a source is
  // its head tile (the one holding t = 0), then come its later tiles in
  // increasing order, then its earlier ones in decreasing order; interleaving
  // the sources puts a tile's chain predecessor a whole batch row earlier in
  // the queue, so that on many-source batches it is finished when the tile
  // looks back at it.  The head rule is the waveform kernel's.
  std::vector<int> T(n), head(n);
  int maxT = 0;
  for (int s = 0; s < n; ++s) {
    T[s] = (int)(ctx->tile_start[s + 1] - ctx->tile_start[s]);
    const int i0 = ctx->descs[s].i0;
    head[s] = (i0 <= 0 || T[s] == 0) ? 0 : std::min(i0 / kTileSamples, T[s] - 1);
    maxT = std::max(maxT, T[s]);
  }
  // Each item also carries the tile's knot window and whether it has output
  // (the waveform kernel's test: a failed source, or a tile that starts at or
  // after the taper's end, min(vlength, i_plunge + i_buffer)).
  ctx->queue.assign(std::max<int64_t>(ctx->total_tiles, 1), QueueItem{});
  int64_t q = 0;
  for (int k = 0; k < maxT; ++k)
    for (int s = 0; s < n; ++s)
      if (k < T[s]) {
        const SourceDesc &d = ctx->descs[s];
        const int lt = (k < T[s] - head[s]) ? head[s] + k : T[s] - 1 - k;
        const int64_t g = ctx->tile_start[s] + lt;
        const long long neff = std::min<long long>(d.vlength, (long long)d.i_plunge + (long long)d.i_buffer);
        QueueItem &it = ctx->queue[q++];
        it.g = (int32_t)g;
        it.s = s;
        it.lt = lt;
        it.k0 = ctx->tile_knot[2 * g];
        it.nk = ctx->tile_knot[2 * g + 1];
        it.knot = d.knot_offset + it.k0;
        it.flags = (d.status != 0 ? kQueueFailed | kQueueNoWave : 0) |
                   ((long long)lt * kTileSamples >= neff ? kQueueNoWave : 0);
      }
  ctx->uploaded = false;
  return AAK_OK;
}

// Coarse AK evolution and knots of up to kPlanGroup sources idx[0..n) on one
// thread, their coarse AK evolutions run together (plan_source_group: the
// same results as one at a time).
void finish_group(aak_ctx *ctx, int n, const int *idx, const Params *P, const MappedTrajectory *const *mt, int *st,
                  const int32_t *nm) {
  WaveInputs w[kPlanGroup];
  const WaveInputs *wp[kPlanGroup];
  SourcePlan *pp[kPlanGroup];
  int go[kPlanGroup], ngo = 0;
  for (int i = 0; i < n; ++i) {
    if (st[i] != kOk) continue;
    genwave_inputs(P[i], *mt[i], nm ? nm[idx[i]] : 0, &w[i]);
    if (w[i].nmodes > 4096) {
      st[i] = kErrCapacity;
      continue;
    }
    wp[ngo] = &w[i];
    pp[ngo] = &ctx->plans[idx[i]];
    go[ngo++] = i;
  }
  if (ngo > 0) plan_source_group(wp, pp, ngo);
  for (int g = 0; g < ngo; ++g) st[go[g]] = ctx->plans[idx[go[g]]].status;
  for (int i = 0; i < n; ++i) {
    ctx->status[idx[i]] = st[i];
    if (st[i] != kOk) {
      ctx->plans[idx[i]].knot_t.clear();
      ctx->plans[idx[i]].knot_y.clear();
    }
  }
}

void finish_source(aak_ctx *ctx, int s, const Params &Pp, const MappedTrajectory &mt, const int32_t *nm, int st) {
  if (st == kOk) {
    WaveInputs w;
    genwave_inputs(Pp, mt, nm ? nm[s] : 0, &w);
    if (w.nmodes > 4096) st = kErrCapacity;
    else st = plan_source(w, &ctx->plans[s]);
  }
  ctx->status[s] = st;
  if (st != kOk) {
    ctx->plans[s].knot_t.clear();
    ctx->plans[s].knot_y.clear();
  }
}

// Planning stages (1)-(3) for every source of Pv (lengths already checked);
// on_done(s), if set, is called on the worker thread right after source s is
// planned (its plan and status final from then on).
int plan_sources(aak_ctx *ctx, const std::vector<aak_params> &Pv, const aak_mapped *maps, const int32_t *nm,
                 int32_t nthreads, const std::function<void(int)> &on_done, bool stream_order = false) {
  const int32_t nsrc = (int32_t)Pv.size();
  // worker threads page-lock knot arrays: make this context's device theirs
  // (a new thread starts on device 0, where it would otherwise open a context)
  const int dev = ctx->device;
  auto on_device = [dev]() {
    int cur = -1;
    if (dev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != dev) cudaSetDevice(dev);
  };
  int caller_dev = -1;  // the calling thread's device, put back at the end
  if (dev >= 0 && cudaGetDevice(&caller_dev) != cudaSuccess) caller_dev = -1;
  struct Restore {
    int d;
    ~Restore() {
      if (d >= 0) cudaSetDevice(d);
    }
  } restore{caller_dev};
  ctx->nsrc = nsrc;
  // the plan array only grows: plans past nsrc keep their page-locked knot
  // arrays for later, larger batches (pinning is slow; only nsrc bounds the live part)
  if ((int32_t)ctx->plans.size() < nsrc) ctx->plans.resize(nsrc);
  for (auto &pl : ctx->plans) pl.knot_t.want_pinned = pl.knot_y.want_pinned = ctx->want_pinned;
  ctx->status.assign(nsrc, AAK_OK);
  ctx->newton_points = ctx->newton_iters = ctx->newton_fallbacks = 0;
  if (maps) {
    parallel_for(nsrc, nthreads, [&](int64_t s) {
      on_device();
      const Params Pp = to_params(Pv[s]);
      MappedTrajectory mt;
      const int st = validate(Pp);
      if (st == kOk) from_mapped(maps[s], &mt);
      finish_source(ctx, (int)s, Pp, mt, nm, st);
      if (on_done) on_done((int)s);
    });
    return AAK_OK;
  }
  // (1) coarse Kerr inspiral and Kerr frequencies: a pass of its own when a
  // warm-start model needs every coarse point at once, else inside each
  // source's planning task (the long sources then start at once)
  std::vector<CoarseKerr> ck(nsrc);
  const bool dev_map = ctx->parmap_device && dev >= 0;
  const bool fused = !ctx->model && !dev_map;
  if (!fused)
    parallel_for(nsrc, nthreads, [&](int64_t s) {
      const Params Pp = to_params(Pv[s]);
      int st = validate(Pp);
      if (st == kOk) st = coarse_kerr(Pp, &ck[s]);
      ctx->status[s] = st;
    });
  // (2) optional learned warm start: every coarse point of the batch in one launch
  std::vector<int64_t> first(nsrc + 1, 0);
  std::vector<double> warm;
  if (!fused)
    for (int s = 0; s < nsrc; ++s) first[s + 1] = first[s] + (ctx->status[s] == kOk ? ck[s].steps : 0);
  if (ctx->model) {
    const int64_t np = first[nsrc];
    std::vector<double> xs(4 * np), ys(3 * np);
    for (int s = 0; s < nsrc; ++s)
      for (int64_t i = 0; i < first[s + 1] - first[s]; ++i) {
        double *x = &xs[4 * (first[s] + i)];
        x[0] = ck[s].p[i];
        x[1] = ck[s].e[i];
        x[2] = Pv[s].iota;
        x[3] = Pv[s].s;
      }
    const int r = mlp_predict_host(ctx->model, xs.data(), ys.data(), np);
    if (r != AAK_OK) return r;
    warm.resize(3 * np);
    for (int s = 0; s < nsrc; ++s)
      for (int64_t i = first[s]; i < first[s + 1]; ++i) parmap_from_coords(&xs[4 * i], Pv[s].M, &ys[3 * i], &warm[3 * i]);
  }
  // (2b) optional device solve of the map: every coarse point of the batch in
  // one launch (the same root as the host solve, bit for bit)
  std::vector<double> dmap;
  std::vector<int32_t> dit;
  if (dev_map) {
    on_device();
    const int64_t np = first[nsrc];
    std::vector<ParmapJob> jobs(np);
    for (int s = 0; s < nsrc; ++s) {
      const double Y = std::cos(Pv[s].iota);
      for (int64_t i = 0; i < first[s + 1] - first[s]; ++i) {
        ParmapJob &j = jobs[first[s] + i];
        for (int k = 0; k < 3; ++k) j.Om[k] = ck[s].Omega[i][k];
        j.p = ck[s].p[i];
        j.M = Pv[s].M;
        j.s = Pv[s].s;
        j.e = ck[s].e[i];
        j.Y = Y;
      }
    }
    dmap.assign(3 * np, 0.0);
    dit.assign(2 * np, 0);
    if (np > 0) {
      int r;
      if (!ctx->pm_stream &&
          (r = cuda_ok(cudaStreamCreateWithFlags(&ctx->pm_stream, cudaStreamNonBlocking))) != AAK_OK)
        return r;
      if ((r = ctx->d_pm_jobs.reserve(np)) || (r = ctx->d_pm_map.reserve(3 * np)) ||
          (r = ctx->d_pm_it.reserve(2 * np)) || (!warm.empty() && (r = ctx->d_pm_warm.reserve(3 * np))))
        return r;
      cudaStream_t st = ctx->pm_stream;
      if ((r = cuda_ok(cudaMemcpyAsync(ctx->d_pm_jobs.ptr, jobs.data(), np * sizeof(ParmapJob),
                                       cudaMemcpyHostToDevice, st))) ||
          (!warm.empty() && (r = cuda_ok(cudaMemcpyAsync(ctx->d_pm_warm.ptr, warm.data(), 3 * np * sizeof(double),
                                                         cudaMemcpyHostToDevice, st)))))
        return r;
      launch_parmap_newton(ctx->d_pm_jobs.ptr, np, warm.empty() ? nullptr : ctx->d_pm_warm.ptr, ctx->d_pm_map.ptr,
                           ctx->d_pm_it.ptr, ctx->d_pm_it.ptr + np, st);
      if ((r = cuda_ok(cudaGetLastError())) ||
          (r = cuda_ok(cudaMemcpyAsync(dmap.data(), ctx->d_pm_map.ptr, 3 * np * sizeof(double),
                                       cudaMemcpyDeviceToHost, st))) ||
          (r = cuda_ok(cudaMemcpyAsync(dit.data(), ctx->d_pm_it.ptr, 2 * np * sizeof(int32_t),
                                       cudaMemcpyDeviceToHost, st))) ||
          (r = cuda_ok(cudaStreamSynchronize(st))))
        return r;
    }
  }
  // (3) Kerr -> AK map, coarse AK evolution, knots; largest sources first.
  // A source's knot count is about (steps - 1) max(1, r / T_fit), r its
  // observation time in radiation-reaction units (the coarse grid spans
  // min(T_fit, r)), and the coarse evolution costs about the same per knot,
  // so handing sources out in that order keeps host threads from idling
  // behind one long source at the end.
  std::vector<int> order(nsrc);
  int nbig = 0;  // the leading sources of order that run alone (the rest in groups)
  int64_t ntasks = 0;
  std::vector<int64_t> task_order;  // the order in which threads take the tasks
  const int threads = nthreads > 0 ? nthreads : (int)std::max(1u, std::thread::hardware_concurrency());
  {
    std::vector<double> cost(nsrc, 0.0);
    for (int s = 0; s < nsrc; ++s) {
      const aak_params &q = Pv[s];
      const double r = q.length * q.dt * q.mu / (kMsunSec * q.M * q.M);
      cost[s] = (q.T_fit > 0 && std::isfinite(r)) ? std::max(1.0, r / q.T_fit) : 0.0;
    }
    for (int s = 0; s < nsrc; ++s) order[s] = s;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost[a] > cost[b]; });
    // The sources that bound the planning time (more than a quarter of a
    // thread's fair share each) go first and alone: a lone recurrence has
    // the shortest latency per step.  The others are planned kPlanGroup at a
    // time, neighbours in cost, their recurrences run together in vector
    // lanes (the same results, at a fraction of the cost per source).
    double total = 0.0;
    for (double c : cost) total += c;
    const double big = total / threads / 4.0;
    const auto split = std::find_if(order.begin(), order.end(), [&](int s) { return cost[s] <= big; });
    nbig = (int)(split - order.begin());
    ntasks = nbig + (nsrc - nbig + kPlanGroup - 1) / kPlanGroup;
    task_order.resize(ntasks);
    for (int64_t t = 0; t < ntasks; ++t) task_order[t] = t;
    if (stream_order && ntasks > threads) {
      // Streaming: cheap tasks, whose sources carry many samples per unit
      // of planning time, should finish early (their waveforms start the
      // device work and the copies back) without the long tasks ending
      // late.  The order comes from list scheduling simulated on estimated
      // task times: a free thread takes the costliest task left when it is
      // a big source or would otherwise end after kSlack of the makespan
      // bound (total / threads), else the cheapest task left.  Estimated
      // time of a task, in cost units: its sources' costs (x kLaneShare in
      // vector lanes) plus kSourceFixed per source for the front end; both
      // constants were fitted to measured task times on a 16-core host, and
      // kSlack = 0.75 was the most robust to 15 % estimate errors in
      // simulation of the 512-source benchmark batch.
      constexpr double kSlack = 0.75, kLaneShare = 0.54, kSourceFixed = 270.0;
      std::vector<double> est(ntasks);
      for (int64_t t = 0; t < ntasks; ++t) {
        const int64_t k = (t < nbig) ? t : nbig + kPlanGroup * (t - nbig);
        const int n = (t < nbig) ? 1 : (int)std::min<int64_t>(kPlanGroup, nsrc - k);
        double c = 0.0;
        for (int i = 0; i < n; ++i) c += cost[order[k + i]];
        est[t] = (t < nbig ? c : kLaneShare * c) + kSourceFixed * n;
      }
      std::vector<int64_t> desc(ntasks);
      for (int64_t t = 0; t < ntasks; ++t) desc[t] = t;
      std::stable_sort(desc.begin(), desc.end(), [&](int64_t a, int64_t b) { return est[a] > est[b]; });
      double sum = 0.0;
      for (double x : est) sum += x;
      const double bound = kSlack * sum / threads;
      std::vector<double> busy(threads, 0.0);
      int64_t hi = 0, lo = ntasks - 1, q = 0;
      while (hi <= lo) {
        const int p = (int)(std::min_element(busy.begin(), busy.end()) - busy.begin());
        const int64_t t = (desc[hi] < nbig || busy[p] + est[desc[hi]] >= bound) ? desc[hi++] : desc[lo--];
        task_order[q++] = t;
        busy[p] += est[t];
      }
    }
  }
  std::atomic<int64_t> points(0), iters(0), fallbacks(0);
  auto map_one = [&](int s, const Params &Pp, MappedTrajectory *mt) {
    if (fused) {
      int st0 = validate(Pp);
      if (st0 == kOk) st0 = coarse_kerr(Pp, &ck[s]);
      ctx->status[s] = st0;
    }
    int st = ctx->status[s];
    if (st == kOk && dev_map) {
      // the device-solved map of this source's coarse points (map_coarse's layout)
      const CoarseKerr &c = ck[s];
      const int64_t np = first[nsrc], f0 = first[s];
      mt->steps = c.steps;
      mt->inspiral_flag = c.inspiral_flag;
      mt->Phi0 = initial_mean_anomaly(Pp.e, Pp.psi);
      mt->newton_iterations = 0;
      int fb = 0;
      for (int i = 0; i < c.steps && st == kOk; ++i) {
        const int it = dit[f0 + i];
        if (it < 0) {
          st = kErrSolverNoConverge;
          break;
        }
        mt->newton_iterations += it;
        fb += dit[np + f0 + i];
        mt->e_traj[i] = c.e[i];
        mt->v_map[i] = dmap[3 * (f0 + i)];
        mt->M_map[i] = dmap[3 * (f0 + i) + 1];
        mt->s_map[i] = dmap[3 * (f0 + i) + 2];
        mt->dt_map[i] = c.t_rr[i] * kMsunSec * Pp.M * Pp.M / Pp.mu;
      }
      if (st == kOk) {
        points += c.steps;
        iters += mt->newton_iterations;
        fallbacks += fb;
      }
    } else if (st == kOk) {
      int fb = 0;
      st = map_coarse(Pp, ck[s], mt, warm.empty() ? nullptr : &warm[3 * first[s]], &fb);
      if (st == kOk) {
        points += ck[s].steps;
        iters += mt->newton_iterations;
        fallbacks += fb;
      }
    }
    return st;
  };
  if (ctx->evolve_device && dev >= 0) {
    // Planning in three passes around a device evolution: (a) front end, map
    // and the fit window of every source on host threads; (b) every source's
    // AK recurrence beyond the fit window in one launch, one GPU thread per
    // source; (c) fitted knots, plunge search and descriptors on host threads.
    using clk = std::chrono::steady_clock;
    const auto t_a = clk::now();
    std::vector<MappedTrajectory> mts(nsrc);
    std::vector<WaveInputs> ws(nsrc);
    std::vector<PlanCarryPtr> carry(nsrc);
    std::vector<EvolveJob> jobs(nsrc);
    parallel_for(nsrc, nthreads, [&](int64_t t) {
      on_device();
      const int s = order[t];
      const Params Pp = to_params(Pv[s]);
      int st = map_one(s, Pp, &mts[s]);
      if (st == kOk) {
        genwave_inputs(Pp, mts[s], nm ? nm[s] : 0, &ws[s]);
        if (ws[s].nmodes > 4096) st = kErrCapacity;
        else st = plan_source_begin(ws[s], &ctx->plans[s], &carry[s], &jobs[s]);
      }
      ctx->status[s] = st;
    });
    const auto t_b = clk::now();
    // the jobs of the sources still in play, their segments one after another
    std::vector<int> live;
    int64_t total = 0;
    for (int s = 0; s < nsrc; ++s)
      if (ctx->status[s] == kOk) {
        jobs[s].off = total;
        total += jobs[s].j_end + 1;
        live.push_back(s);
      }
    std::vector<EvolveJob> lj(live.size());
    for (size_t k = 0; k < live.size(); ++k) lj[k] = jobs[live[k]];
    std::vector<double> ev(2 * (size_t)std::max<int64_t>(total, 1));
    double *eh = ev.data(), *vh = eh + std::max<int64_t>(total, 1);
    parallel_for((int64_t)live.size(), nthreads, [&](int64_t k) {
      const int s = live[k];
      plan_carry_prefix(*carry[s], jobs[s], eh + jobs[s].off, vh + jobs[s].off);
    });
    if (!live.empty()) {
      on_device();
      int r;
      if (!ctx->pm_stream &&
          (r = cuda_ok(cudaStreamCreateWithFlags(&ctx->pm_stream, cudaStreamNonBlocking))) != AAK_OK)
        return r;
      DevBuf<double> d_ev;
      DevBuf<EvolveJob> d_jobs;
      if ((r = d_ev.reserve(2 * (size_t)total)) || (r = d_jobs.reserve(live.size()))) return r;
      cudaStream_t st = ctx->pm_stream;
      // every entry goes up (the recurrence's part is overwritten): one copy each way
      r = cuda_ok(cudaMemcpyAsync(d_ev.ptr, eh, (size_t)total * sizeof(double), cudaMemcpyHostToDevice, st));
      if (r == AAK_OK)
        r = cuda_ok(cudaMemcpyAsync(d_ev.ptr + total, vh, (size_t)total * sizeof(double), cudaMemcpyHostToDevice, st));
      if (r == AAK_OK)
        r = cuda_ok(cudaMemcpyAsync(d_jobs.ptr, lj.data(), lj.size() * sizeof(EvolveJob), cudaMemcpyHostToDevice, st));
      if (r == AAK_OK) {
        launch_ak_evolve(d_jobs.ptr, (int)lj.size(), d_ev.ptr, d_ev.ptr + total, st);
        r = cuda_ok(cudaGetLastError());
      }
      if (r == AAK_OK)
        r = cuda_ok(cudaMemcpyAsync(eh, d_ev.ptr, (size_t)total * sizeof(double), cudaMemcpyDeviceToHost, st));
      if (r == AAK_OK)
        r = cuda_ok(cudaMemcpyAsync(vh, d_ev.ptr + total, (size_t)total * sizeof(double), cudaMemcpyDeviceToHost, st));
      if (r == AAK_OK)
        r = cuda_ok(cudaMemcpyAsync(lj.data(), d_jobs.ptr, lj.size() * sizeof(EvolveJob), cudaMemcpyDeviceToHost, st));
      if (r == AAK_OK) r = cuda_ok(cudaStreamSynchronize(st));
      d_ev.release();
      d_jobs.release();
      if (r != AAK_OK) return r;
      for (size_t k = 0; k < live.size(); ++k) jobs[live[k]] = lj[k];
    }
    const auto t_c = clk::now();
    parallel_for((int64_t)live.size(), nthreads, [&](int64_t k) {
      on_device();
      const int s = live[k];
      const int st = plan_source_end(*carry[s], jobs[s], eh + jobs[s].off, vh + jobs[s].off);
      carry[s].reset();
      ctx->status[s] = st;
    });
    for (int s = 0; s < nsrc; ++s)
      if (ctx->status[s] != kOk) {
        ctx->plans[s].knot_t.clear();
        ctx->plans[s].knot_y.clear();
      }
    if (on_done)
      for (int s = 0; s < nsrc; ++s) on_done(s);
    const auto t_d = clk::now();
    auto ms = [](clk::time_point a, clk::time_point b) { return std::chrono::duration<double, std::milli>(b - a).count(); };
    ctx->plan_ms[0] = ms(t_a, t_b);
    ctx->plan_ms[1] = ms(t_b, t_c);
    ctx->plan_ms[2] = ms(t_c, t_d);
    ctx->plan_ms[3] = ms(t_a, t_d);
    ctx->newton_points = points;
    ctx->newton_iters = iters;
    ctx->newton_fallbacks = fallbacks;
    return AAK_OK;
  }
  parallel_for(ntasks, nthreads, [&](int64_t q) {
    on_device();
    const int64_t t = task_order[q];
    const int64_t k = (t < nbig) ? t : nbig + kPlanGroup * (t - nbig);
    const int n = (t < nbig) ? 1 : (int)std::min<int64_t>(kPlanGroup, nsrc - k);
    int idx[kPlanGroup], st[kPlanGroup];
    Params Pg[kPlanGroup];
    std::vector<MappedTrajectory> mg(n);
    const MappedTrajectory *mp[kPlanGroup];
    for (int i = 0; i < n; ++i) {
      idx[i] = order[k + i];
      Pg[i] = to_params(Pv[idx[i]]);
      st[i] = map_one(idx[i], Pg[i], &mg[i]);
      mp[i] = &mg[i];
    }
    finish_group(ctx, n, idx, Pg, mp, st, nm);
    if (on_done)
      for (int i = 0; i < n; ++i) on_done(idx[i]);
  });
  ctx->newton_points = points;
  ctx->newton_iters = iters;
  ctx->newton_fallbacks = fallbacks;
  return AAK_OK;
}

int plan_common(aak_ctx *ctx, const aak_params *P, const aak_mapped *maps, int32_t nsrc, const int32_t *nm,
                int32_t nthreads) {
  if (!ctx || !P || nsrc <= 0) return AAK_ERR_INVALID_PARAM;
  std::vector<aak_params> Pv(P, P + nsrc);
  for (auto &p : Pv)
    if (p.length < 2 || p.length > ((int64_t)1 << 31)) return AAK_ERR_INVALID_PARAM;
  const int r = plan_sources(ctx, Pv, maps, nm, nthreads, nullptr);
  if (r != AAK_OK) return r;
  return pack(ctx, Pv, nthreads);
}

// wait_pinned: finish the copies from page-locked plan arrays before
// returning (callers whose next plan may refill those arrays); a caller that
// keeps the plans untouched until it synchronises the stream passes false.
int upload(aak_ctx *ctx, cudaStream_t st, bool wait_pinned = true) {
  int r;
  if ((r = select_device(ctx->device)) != AAK_OK) return r;
  const int n = ctx->nsrc;
  if ((r = ctx->d_src.reserve(n)) || (r = ctx->d_tile_start.reserve(n + 1)) ||
      (r = ctx->d_tile_knot.reserve(ctx->tile_knot.size())) || (r = ctx->d_tile_pairs.reserve(ctx->tile_pairs.size())) ||
      (r = ctx->d_queue.reserve(ctx->queue.size())) || (r = ctx->d_spl_blk.reserve(ctx->spl_blk.size())) ||
      // knot times: two entries of slack past the last knot (a window's bulk
      // copy starts on a 16-byte boundary and may read one element beyond it)
      (r = ctx->d_knot_t.reserve(std::max<int64_t>(ctx->total_knots, 1) + 2)) ||
      (r = ctx->d_knot_y.reserve(std::max<int64_t>(ctx->total_knots, 1))) ||
      (r = ctx->d_knot_c.reserve(std::max<int64_t>(ctx->total_knots, 1))) || (r = ctx->d_bessel.reserve(ctx->bessel.size())) ||
      (r = ctx->d_link.reserve(std::max<int64_t>(ctx->total_tiles, 1))) ||
      (r = ctx->d_flag.reserve(std::max<int64_t>(ctx->total_tiles, 1))) || (r = ctx->d_counter.reserve(2)))
    return r;
  // the work-queue head is cleared by every launch; the status word here
  if ((r = cuda_ok(cudaMemsetAsync(ctx->d_counter.ptr, 0, 2 * sizeof(unsigned long long), st))) != AAK_OK) return r;
  auto cp = [&](void *dst, const void *src, size_t bytes) {
    return cuda_ok(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st));
  };
  if ((r = cp(ctx->d_src.ptr, ctx->descs.data(), n * sizeof(SourceDesc))) ||
      (r = cp(ctx->d_tile_start.ptr, ctx->tile_start.data(), (n + 1) * sizeof(int64_t))) ||
      (r = cp(ctx->d_tile_knot.ptr, ctx->tile_knot.data(), ctx->tile_knot.size() * sizeof(int32_t))) ||
      (r = cp(ctx->d_tile_pairs.ptr, ctx->tile_pairs.data(), ctx->tile_pairs.size() * sizeof(int64_t))) ||
      (r = cp(ctx->d_queue.ptr, ctx->queue.data(), ctx->queue.size() * sizeof(QueueItem))) ||
      (r = cp(ctx->d_spl_blk.ptr, ctx->spl_blk.data(), ctx->spl_blk.size() * sizeof(int64_t))) ||
      (r = cp(ctx->d_bessel.ptr, ctx->bessel.data(), ctx->bessel.size() * sizeof(int32_t))))
    return r;
  // knots straight from each source's plan arrays to its slice of the device arrays
  for (int s = 0; s < n; ++s) {
    const SourcePlan &pl = ctx->plans[s];
    const int64_t nk = ctx->kofs[s + 1] - ctx->kofs[s];
    if (nk <= 0) continue;
    const int64_t ko = ctx->kofs[s];
    if ((r = cp(ctx->d_knot_t.ptr + ko, pl.knot_t.data(), nk * sizeof(double))) ||
        (r = cp(ctx->d_knot_y.ptr + ko, pl.knot_y.data(), nk * sizeof(double4))))
      return r;
  }
  // spline coefficients of every source, solved on the device
  launch_spline_coeffs(ctx->d_src.ptr, n, ctx->d_spl_blk.ptr, ctx->spl_blk[n], ctx->d_knot_t.ptr, ctx->d_knot_y.ptr,
                       ctx->d_knot_c.ptr, st);
  if ((r = cuda_ok(cudaGetLastError())) != AAK_OK) return r;
  // copies from page-locked memory run asynchronously: finish them before the
  // host arrays can be refilled by the next plan
  if (wait_pinned && ctx->want_pinned && (r = cuda_ok(cudaStreamSynchronize(st))) != AAK_OK) return r;
  ctx->uploaded = true;
  ++ctx->upload_gen;
  return AAK_OK;
}

BatchView batch_view(aak_ctx *ctx, double *hI, double *hII, double *t, double *traj, int64_t traj_stride);

// The tile pre-pass buffers of a waveform launch in `precision` (one
// TilePrep and one Taylor-table slot per tile), grown as needed, set in bv.
void drop_graph(aak_ctx *ctx);

int tile_tables(aak_ctx *ctx, int precision, BatchView &bv) {
  const int64_t tiles = std::max<int64_t>(ctx->total_tiles, 1);
  const int64_t slot = tile_table_slot_bytes(ctx->max_nmodes, precision == 1);
  const void *p0 = ctx->d_tile_prep.ptr, *t0 = ctx->d_tile_tab.ptr;
  int r;
  if ((r = ctx->d_tile_prep.reserve(tiles)) != AAK_OK || (r = ctx->d_tile_tab.reserve(tiles * slot)) != AAK_OK)
    return r;
  // a captured dense graph holds the old buffers: recapture on its next use
  if (ctx->d_tile_prep.ptr != p0 || ctx->d_tile_tab.ptr != t0) drop_graph(ctx);
  bv.tile_prep = ctx->d_tile_prep.ptr;
  bv.tile_tab = ctx->d_tile_tab.ptr;
  bv.tab_slot = slot;
  return AAK_OK;
}

int run(aak_ctx *ctx, double *hI, double *hII, double *t, double *traj, int64_t traj_stride, int precision,
        cudaStream_t st) {
  if (!ctx->uploaded) return AAK_ERR_INVALID_PARAM;
  if (!hI || !hII) return AAK_ERR_INVALID_PARAM;
  if (traj && traj_stride < ctx->total_samples) return AAK_ERR_INVALID_PARAM;
  if (precision != 0 && precision != 1) return AAK_ERR_INVALID_PARAM;
  int r;
  if ((r = select_device(ctx->device)) != AAK_OK) return r;
  BatchView bv = batch_view(ctx, hI, hII, t, traj, traj_stride);
  bv.variant = ctx->variant[precision];
  if (!traj && (r = tile_tables(ctx, precision, bv)) != AAK_OK) return r;
  if (ctx->profile && !ctx->ev[0])
    for (auto &e : ctx->ev) cudaEventCreate(&e);
  launch_dense(bv, ctx->num_sms, st, ctx->profile ? ctx->ev : nullptr, precision);
  ctx->last_launches = (bv.tile_prep && wave_variant(precision == 1, bv.variant).pre) ? 3 : 1;
  return cuda_ok(cudaGetLastError());
}

// The waveform kernel into FP32 rows (hI32, hII32 indexed as the FP64 outputs).
int run_rows32(aak_ctx *ctx, float *hI32, float *hII32, int precision, cudaStream_t st) {
  if (!ctx->uploaded || !hI32 || !hII32 || (precision != 0 && precision != 1)) return AAK_ERR_INVALID_PARAM;
  int r;
  if ((r = select_device(ctx->device)) != AAK_OK) return r;
  BatchView bv = batch_view(ctx, nullptr, nullptr, nullptr, nullptr, 0);
  bv.hI_f32 = hI32;
  bv.hII_f32 = hII32;
  bv.variant = ctx->variant[precision];
  if ((r = tile_tables(ctx, precision, bv)) != AAK_OK) return r;
  launch_dense(bv, ctx->num_sms, st, nullptr, precision);
  ctx->last_launches = 3;
  return cuda_ok(cudaGetLastError());
}

void drop_graph(aak_ctx *ctx) {
  if (ctx->gexec) cudaGraphExecDestroy(ctx->gexec);
  if (ctx->graph) cudaGraphDestroy(ctx->graph);
  ctx->gexec = nullptr;
  ctx->graph = nullptr;
}

// The dense stage (spline solve, two clears and the waveform kernel) as one CUDA graph, captured on the
// first call for a given (outputs, precision, upload) and replayed afterwards.
int run_graph(aak_ctx *ctx, double *hI, double *hII, int precision, cudaStream_t st) {
  if (!ctx->uploaded || !hI || !hII || (precision != 0 && precision != 1)) return AAK_ERR_INVALID_PARAM;
  int r;
  if ((r = select_device(ctx->device)) != AAK_OK) return r;
  if (ctx->gexec && (ctx->g_hI != hI || ctx->g_hII != hII || ctx->g_prec != precision || ctx->g_gen != ctx->upload_gen ||
                     ctx->g_variant != ctx->variant[precision]))
    drop_graph(ctx);
  if (!ctx->gexec) {
    if (!ctx->cap_stream && (r = cuda_ok(cudaStreamCreateWithFlags(&ctx->cap_stream, cudaStreamNonBlocking))) != AAK_OK)
      return r;
    prepare_dense_launch();
    BatchView bv = batch_view(ctx, hI, hII, nullptr, nullptr, 0);
    bv.variant = ctx->variant[precision];
    if ((r = tile_tables(ctx, precision, bv)) != AAK_OK) return r;
    if ((r = cuda_ok(cudaStreamBeginCapture(ctx->cap_stream, cudaStreamCaptureModeThreadLocal))) != AAK_OK) return r;
    // the whole dense stage: natural-spline solve of every source's knots
    // (idempotent: the same knots give the same coefficients), then the clears
    // and the waveform kernel
    launch_spline_coeffs(ctx->d_src.ptr, ctx->nsrc, ctx->d_spl_blk.ptr, ctx->spl_blk[ctx->nsrc], ctx->d_knot_t.ptr,
                         ctx->d_knot_y.ptr, ctx->d_knot_c.ptr, ctx->cap_stream);
    launch_dense(bv, ctx->num_sms, ctx->cap_stream, nullptr, precision);
    const cudaError_t launch_err = cudaGetLastError();
    cudaGraph_t g = nullptr;
    const cudaError_t end_err = cudaStreamEndCapture(ctx->cap_stream, &g);
    if (launch_err != cudaSuccess || end_err != cudaSuccess || !g) {
      if (g) cudaGraphDestroy(g);
      return cuda_ok(launch_err != cudaSuccess ? launch_err : (end_err != cudaSuccess ? end_err : cudaErrorUnknown));
    }
    ctx->graph = g;
    if ((r = cuda_ok(cudaGraphInstantiate(&ctx->gexec, ctx->graph, 0))) != AAK_OK) {
      drop_graph(ctx);
      return r;
    }
    ctx->g_hI = hI;
    ctx->g_hII = hII;
    ctx->g_prec = precision;
    ctx->g_gen = ctx->upload_gen;
    ctx->g_variant = ctx->variant[precision];
  }
  // spline solve, tile parameters and tables (with the pre-pass), waveform kernel
  ctx->last_launches = wave_variant(precision == 1, ctx->variant[precision]).pre ? 4 : 2;
  return cuda_ok(cudaGraphLaunch(ctx->gexec, st));
}

BatchView batch_view(aak_ctx *ctx, double *hI, double *hII, double *t, double *traj, int64_t traj_stride) {
  BatchView bv;
  bv.src = ctx->d_src.ptr;
  bv.nsrc = ctx->nsrc;
  bv.total_tiles = ctx->total_tiles;
  bv.tile_start = ctx->d_tile_start.ptr;
  bv.queue = ctx->d_queue.ptr;
  bv.tile_knot = ctx->d_tile_knot.ptr;
  bv.knot_t = ctx->d_knot_t.ptr;
  bv.knot_y = ctx->d_knot_y.ptr;
  bv.knot_c = ctx->d_knot_c.ptr;
  bv.bessel_start = ctx->d_bessel.ptr;
  bv.link = ctx->d_link.ptr;
  bv.link_flag = ctx->d_flag.ptr;
  bv.hI = hI;
  bv.hII = hII;
  bv.t_out = t;
  bv.traj_out = traj;
  bv.traj_stride = traj_stride;
  bv.work_counter = ctx->d_counter.ptr;
  bv.device_status = reinterpret_cast<unsigned int *>(ctx->d_counter.ptr + 1);
  bv.max_nmodes = ctx->max_nmodes;
  bv.lookback_cycles = ctx->lookback_cycles;
  return bv;
}

// The phase product of every source of the uploaded batch into device memory:
// 8 rows of `stride` doubles (t, phase_r, phase_theta, phase_phi, omega_r,
// omega_theta, omega_phi, e) indexed by the batch offsets.
int run_phase(aak_ctx *ctx, double *out, int64_t stride, cudaStream_t st) {
  if (!ctx->uploaded || !out || stride < ctx->total_samples) return AAK_ERR_INVALID_PARAM;
  int r;
  if ((r = select_device(ctx->device)) != AAK_OK) return r;
  BatchView bv = batch_view(ctx, nullptr, nullptr, nullptr, nullptr, 0);
  bv.phase_out = out;
  bv.phase_stride = stride;
  bv.trajectory_only = 1;
  // the tile pre-pass's parameters (no tables in the phase product)
  const void *p0 = ctx->d_tile_prep.ptr;
  if ((r = ctx->d_tile_prep.reserve(std::max<int64_t>(ctx->total_tiles, 1))) != AAK_OK) return r;
  if (ctx->d_tile_prep.ptr != p0) drop_graph(ctx);
  bv.tile_prep = ctx->d_tile_prep.ptr;
  if (ctx->profile && !ctx->ev[0])
    for (auto &e : ctx->ev) cudaEventCreate(&e);
  launch_phase(bv, ctx->num_sms, st, ctx->profile ? ctx->ev : nullptr);
  ctx->last_launches = 3;
  return cuda_ok(cudaGetLastError());
}

// Plain FP64 per-source path: source by source, the phase kernels on a
// one-source view write the dense trajectory, then the per-harmonic kernel.
int run_plain(aak_ctx *ctx, double *hI, double *hII, double *traj, int64_t traj_stride, cudaStream_t st) {
  if (!ctx->uploaded || !hI || !hII || !traj || traj_stride < ctx->total_samples) return AAK_ERR_INVALID_PARAM;
  int r;
  if ((r = select_device(ctx->device)) != AAK_OK) return r;
  int launches = 0;
  for (int s = 0; s < ctx->nsrc; ++s) {
    const SourceDesc &d = ctx->descs[s];
    if (ctx->status[s] != AAK_OK) {
      cudaMemsetAsync(hI + d.out_offset, 0, sizeof(double) * d.vlength, st);
      cudaMemsetAsync(hII + d.out_offset, 0, sizeof(double) * d.vlength, st);
      continue;
    }
    BatchView v;
    v.src = ctx->d_src.ptr + s;
    v.nsrc = 1;
    v.total_tiles = d.n_tiles;
    v.tile_start = ctx->d_tile_pairs.ptr + 2 * s;
    v.tile_knot = ctx->d_tile_knot.ptr + 2 * d.tile_offset;
    v.knot_t = ctx->d_knot_t.ptr;
    v.knot_y = ctx->d_knot_y.ptr;
    v.knot_c = ctx->d_knot_c.ptr;
    v.bessel_start = ctx->d_bessel.ptr;
    v.link = ctx->d_link.ptr + d.tile_offset;
    v.link_flag = ctx->d_flag.ptr + d.tile_offset;
    v.hI = hI;
    v.hII = hII;
    v.t_out = nullptr;
    v.traj_out = traj;
    v.traj_stride = traj_stride;
    v.work_counter = ctx->d_counter.ptr;
    v.device_status = reinterpret_cast<unsigned int *>(ctx->d_counter.ptr + 1);
    v.trajectory_only = 1;
    v.max_nmodes = ctx->max_nmodes;
    launch_dense(v, ctx->num_sms, st, nullptr, 0);
    launch_plain_waveform(ctx->d_src.ptr, s, d.vlength, traj, traj_stride, hI, hII, st);
    launches += 2;
  }
  ctx->last_launches = launches;
  return cuda_ok(cudaGetLastError());
}

std::mutex g_default_mu;
aak_ctx *g_default[64] = {nullptr};

int default_ctx(aak_ctx **out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return AAK_ERR_CUDA;
  }
  if (dev < 0 || dev >= 64) return AAK_ERR_CUDA;
  std::lock_guard<std::mutex> lk(g_default_mu);
  if (!g_default[dev]) {
    int r = aak_ctx_create(dev, &g_default[dev]);
    if (r != AAK_OK) return r;
  }
  *out = g_default[dev];
  return AAK_OK;
}

// Synchronise the device and read (and clear) the status words of the
// context and of the allocation-free scratch.
int device_status(aak_ctx *ctx) {
  int r;
  if ((r = select_device(ctx->device)) != AAK_OK) return r;
  if ((r = cuda_ok(cudaDeviceSynchronize())) != AAK_OK) return r;
  bool gave_up = false;
  if (ctx->d_counter.ptr) {
    unsigned int v = 0;
    unsigned int *word = reinterpret_cast<unsigned int *>(ctx->d_counter.ptr + 1);
    if ((r = cuda_ok(cudaMemcpy(&v, word, sizeof(v), cudaMemcpyDeviceToHost))) != AAK_OK) return r;
    if (v && (r = cuda_ok(cudaMemset(word, 0, sizeof(v)))) != AAK_OK) return r;
    gave_up = v != 0;
  }
  // the allocation-free scratch's report word, only for a context that used it
  // (every context that launches through it on this device shares that word)
  int sv = 0;
  if (ctx->noalloc_used) {
    sv = static_scratch_status(ctx->device, true);
    if (sv < 0) return cuda_ok(cudaGetLastError());
    ctx->noalloc_used = false;
  }
  return (gave_up || sv > 0) ? AAK_ERR_DEVICE_TIMEOUT : AAK_OK;
}

// Plan, upload and run one batch into ctx-owned device outputs, then copy to host.
int host_roundtrip(aak_ctx *ctx, double *t, double *hI, double *hII) {
  int r;
  const int64_t N = ctx->total_samples;
  if ((r = upload(ctx, 0)) != AAK_OK) return r;
  if ((r = ctx->d_out.reserve((size_t)(t ? 3 : 2) * N)) != AAK_OK) return r;
  double *dI = ctx->d_out.ptr, *dII = dI + N, *dt = t ? dII + N : nullptr;
  if ((r = run(ctx, dI, dII, dt, nullptr, 0, ctx->precision, 0)) != AAK_OK) return r;
  if ((r = cuda_ok(cudaMemcpyAsync(hI, dI, N * sizeof(double), cudaMemcpyDeviceToHost, 0))) ||
      (r = cuda_ok(cudaMemcpyAsync(hII, dII, N * sizeof(double), cudaMemcpyDeviceToHost, 0))))
    return r;
  if (t && (r = cuda_ok(cudaMemcpyAsync(t, dt, N * sizeof(double), cudaMemcpyDeviceToHost, 0)))) return r;
  if ((r = cuda_ok(cudaStreamSynchronize(0))) != AAK_OK) return r;
  return device_status(ctx);
}

// Upload, run_phase into the context's device buffer, copy back: rows[k]
// receives row k (total_samples doubles), or at row k of `base` (stride
// ldh) when rows is null.
int phase_roundtrip(aak_ctx *ctx, double *const *rows, double *base, int64_t ldh) {
  int r;
  const int64_t N = ctx->total_samples;
  if ((r = upload(ctx, 0)) != AAK_OK) return r;
  if ((r = ctx->d_out.reserve((size_t)8 * std::max<int64_t>(N, 1))) != AAK_OK) return r;
  double *d = ctx->d_out.ptr;
  if ((r = run_phase(ctx, d, N, 0)) != AAK_OK) return r;
  for (int k = 0; k < 8; ++k) {
    double *h = rows ? rows[k] : base + k * ldh;
    if (h && (r = cuda_ok(cudaMemcpyAsync(h, d + k * N, N * sizeof(double), cudaMemcpyDeviceToHost, 0))) != AAK_OK)
      return r;
  }
  if ((r = cuda_ok(cudaStreamSynchronize(0))) != AAK_OK) return r;
  return device_status(ctx);
}

// ---------------------------------------------------------------- frequency-domain TDI
// Per-source geometry of the TDI response (AAKTDI.cc:51-84): propagation
// direction k = -n, polarisation basis u, v and angle psi.
void tdi_geometry(double qS, double phiS, double qK, double phiK, TdiDesc *d) {
  const double ctS = std::cos(qS), stS = std::sin(qS), cpS = std::cos(phiS), spS = std::sin(phiS);
  const double up = ctS * std::sin(qK) * std::cos(phiS - phiK) - std::cos(qK) * stS;
  const double dw = std::sin(qK) * std::sin(phiS - phiK);
  const double psi = (dw != 0.0) ? -std::atan2(up, dw) : 0.5 * kPi;
  d->c2psi = std::cos(2. * psi);
  d->s2psi = std::sin(2. * psi);
  d->k[0] = -stS * cpS;
  d->k[1] = -stS * spS;
  d->k[2] = -ctS;
  d->uhat[0] = ctS * cpS;
  d->uhat[1] = ctS * spS;
  d->uhat[2] = -stS;
  d->vhat[0] = spS;
  d->vhat[1] = -cpS;
  d->vhat[2] = 0.0;
}

// Plus / cross amplitudes of the sidebands m = -2..2 of a harmonic
// (AAKTDI.cc:586-667): the projection of the orbital-plane basis (L at
// inclination lambda from the spin) onto the sky frame, as trigonometric
// polynomials in alpha.  AA = [plus cos | plus sin | cross cos | cross sin].
void tdi_sidebands(double qS, double phiS, double qK, double phiK, double clam, double slam, double AA[20]) {
  const double cS = std::cos(qS), sS = std::sin(qS), cK = std::cos(qK), sK = std::sin(qK);
  const double cSp = std::cos(phiS), sSp = std::sin(phiS), cKp = std::cos(phiK), sKp = std::sin(phiK);
  const double cX = cS * cK + sS * sK * std::cos(phiS - phiK);
  const double sX = std::sqrt(sS * sS * cK * cK - 2. * sS * sSp * cK * cS * sK * sKp + cS * cS * sK * sK -
                              2. * cS * sK * cKp * sS * cSp * cK + sS * sS * cSp * cSp * sK * sK * sKp * sKp -
                              2. * sS * sS * cSp * sK * sK * sKp * sSp * cKp + sS * sS * sSp * sSp * sK * sK * cKp * cKp);
  // orbital-plane basis vectors p and q, cos / sin / constant parts in alpha, for the two polarisation axes
  const double pc1 = (-cK * cKp * sS * cSp - cK * sKp * sS * sSp + sK * cS) / sX;
  const double ps1 = (sKp * sS * cSp - cKp * sS * sSp) / sX;
  const double pn1 = (cK * cS + sK * cKp * sS * cSp + sK * sKp * sS * sSp - cX) * clam / (sX * slam);
  const double pc2 = (sS * cSp * sKp - sS * sSp * cKp) * clam / sX;
  const double ps2 = (cK * cKp * sS * cSp + cK * sKp * sS * sSp - cS * sK) * clam / sX;
  const double pn2 = 0.0;
  const double qc1 = (sS * cSp * sKp - sS * sSp * cKp) * cX / sX;
  const double qs1 = (cK * cKp * sS * cSp + cK * sKp * sS * sSp - cS * sK) * cX / sX;
  const double qn1 = 0.0;
  const double qc2 = cX * clam * (cK * cKp * sS * cSp + cK * sKp * sS * sSp - sK * cS) / sX;
  const double qs2 = -cX * clam * sS * (sKp * cSp - cKp * sSp) / sX;
  const double qn2 = -(cX * clam * clam * (cK * cS + sK * cKp * sS * cSp + sK * sKp * sS * sSp) + 1. - cX * cX -
                       clam * clam) / (sX * slam);
  // products of the two axes: plus (p p - q q) and cross (p q) parts at frequencies 0, alpha, 2 alpha
  const double P1c1 = 2.0 * (pc1 * pn1 - qc1 * qn1 + qc2 * qn2 - pc2 * pn2);
  const double P1c2 = 0.5 * (ps2 * ps2 - qc1 * qc1 + pc1 * pc1 - ps1 * ps1 + qc2 * qc2 + qs1 * qs1 - pc2 * pc2 - qs2 * qs2);
  const double P1s1 = 2.0 * (qs2 * qn2 - ps2 * pn2 - qs1 * qn1 + ps1 * pn1);
  const double P1s2 = (pc1 * ps1 + qc2 * qs2 - pc2 * ps2 - qc1 * qs1);
  const double P1cn = 0.5 * (pc1 * pc1 + ps1 * ps1 - qc1 * qc1 - qs1 * qs1 - pc2 * pc2 + qc2 * qc2 + qs2 * qs2 - ps2 * ps2) +
                      qn2 * qn2 - qn1 * qn1 + pn1 * pn1 - pn2 * pn2;
  const double P2c1 = (pn1 * pc2 + pc1 * pn2 - qn1 * qc2 - qc1 * qn2);
  const double P2c2 = 0.5 * (qs1 * qs2 - ps1 * ps2 + pc1 * pc2 - qc1 * qc2);
  const double P2s1 = (ps1 * pn2 + pn1 * ps2 - qn1 * qs2 - qs1 * qn2);
  const double P2s2 = 0.5 * (pc1 * ps2 - qc1 * qs2 + ps1 * pc2 - qs1 * qc2);
  const double P2cn = 0.5 * (ps1 * ps2 - qs1 * qs2 - qc1 * qc2 + pc1 * pc2) - qn1 * qn2 + pn1 * pn2;
  const double C1c1 = (-pc2 * qn2 - pn2 * qc2 + pc1 * qn1 + pn1 * qc1);
  const double C1c2 = 0.5 * (pc1 * qc1 - ps1 * qs1 - pc2 * qc2 + ps2 * qs2);
  const double C1s1 = (pn1 * qs1 - ps2 * qn2 + ps1 * qn1 - pn2 * qs2);
  const double C1s2 = 0.5 * (-pc2 * qs2 + pc1 * qs1 - ps2 * qc2 + ps1 * qc1);
  const double C1cn = -pn2 * qn2 + pn1 * qn1 + 0.5 * (pc1 * qc1 - ps2 * qs2 + ps1 * qs1 - pc2 * qc2);
  const double C2c1 = (qc1 * pn2 + qn1 * pc2 + pc1 * qn2 + pn1 * qc2);
  const double C2c2 = 0.5 * (pc1 * qc2 - ps1 * qs2 + qc1 * pc2 - qs1 * ps2);
  const double C2s1 = (pn1 * qs2 + qs1 * pn2 + ps1 * qn2 + qn1 * ps2);
  const double C2s2 = 0.5 * (qc1 * ps2 + pc1 * qs2 + qs1 * pc2 + ps1 * qc2);
  const double C2cn = qn1 * pn2 + pn1 * qn2 + 0.5 * (pc1 * qc2 + qs1 * ps2 + ps1 * qs2 + qc1 * pc2);
  // sideband m: e^{i m alpha} weights (m = -2, -1, 0, 1, 2)
  const double pcs[5] = {0.5 * (P1c2 + P2s2), 0.5 * (P1c1 + P2s1), P1cn, 0.5 * (P1c1 - P2s1), 0.5 * (P1c2 - P2s2)};
  const double pss[5] = {0.5 * (P2c2 - P1s2), 0.5 * (P2c1 - P1s1), P2cn, 0.5 * (P2c1 + P1s1), 0.5 * (P2c2 + P1s2)};
  const double ccs[5] = {0.5 * (C1c2 + C2s2), 0.5 * (C1c1 + C2s1), C1cn, 0.5 * (C1c1 - C2s1), 0.5 * (C1c2 - C2s2)};
  const double css[5] = {0.5 * (C2c2 - C1s2), 0.5 * (C2c1 - C1s1), C2cn, 0.5 * (C2c1 + C1s1), 0.5 * (C2c2 + C1s2)};
  for (int m = 0; m < 5; ++m) {
    AA[m] = pcs[m];
    AA[5 + m] = pss[m];
    AA[10 + m] = ccs[m];
    AA[15 + m] = css[m];
  }
}

// The frequency-domain TDI of nsrc sources (GenTDI, AAKTDI.cc:799-829) into
// host rows: Xr, Xi, Yr, Yi, Zr, Zi, each sum((length + 1) / 2) bins, source s
// from bin_ofs[s].  Front end on the sources' own (length, dt); then each
// source's phase grid (dt_ph = 0.01 M^2 / mu, Nph points over the span) is
// planned, generated by the phase pass and summed by stationary phase.
int tdi_batch(aak_ctx *ctx, const aak_params *P, int32_t nsrc, int32_t nthreads, double *const *rows,
              std::vector<int64_t> &bin_ofs, std::vector<int32_t> &st_out) {
  if (!P || nsrc < 1) return AAK_ERR_INVALID_PARAM;
  int r;
  if ((r = select_device(ctx->device)) != AAK_OK) return r;
  std::vector<aak_mapped> maps(nsrc);
  std::vector<aak_params> G(P, P + nsrc);
  std::vector<int32_t> fe(nsrc, AAK_OK), nm(nsrc, 4);
  std::vector<double> dt_ph(nsrc, 0.0), Tobs(nsrc, 0.0);
  parallel_for(nsrc, nthreads, [&](int64_t s) {
    fe[s] = aak_front_end(&P[s], nullptr, &maps[s]);
    if (fe[s] != AAK_OK) {
      G[s].e = -1.0;  // fails the grid plan's validation; the front end's status is reported
      return;
    }
    const double mu_s = P[s].mu * kMsunSec, M_s = maps[s].M_map[0] * kMsunSec;
    Tobs[s] = (double)(P[s].length - 1) * P[s].dt;
    double h = 0.01 * M_s * M_s / mu_s;
    const double nph = Tobs[s] / h;
    if (!(nph >= 3.0 && nph < 2.0e9)) {
      fe[s] = AAK_ERR_INVALID_PARAM;
      G[s].e = -1.0;
      return;
    }
    const int Nph = (int)nph;
    dt_ph[s] = Tobs[s] / (Nph - 1);
    G[s].length = Nph;
    G[s].dt = dt_ph[s];
    const double e0 = maps[s].e_traj[0];
    nm[s] = (e0 < 0.135) ? 4 : std::max(1, (int)(30 * e0));
  });
  ctx->out_stride = 0;
  if ((r = plan_common(ctx, G.data(), maps.data(), nsrc, nm.data(), nthreads)) != AAK_OK) return r;
  if ((r = upload(ctx, 0)) != AAK_OK) return r;
  // records of the stationary-phase sum
  std::vector<TdiDesc> td(nsrc);
  std::vector<int64_t> work(nsrc + 1, 0);
  bin_ofs.assign(nsrc + 1, 0);
  st_out.assign(nsrc, AAK_OK);
  for (int s = 0; s < nsrc; ++s) {
    const int32_t st = (fe[s] != AAK_OK) ? fe[s] : ctx->status[s];
    st_out[s] = st;
    bin_ofs[s + 1] = bin_ofs[s] + (P[s].length + 1) / 2;
    TdiDesc &d = td[s];
    std::memset(&d, 0, sizeof(d));
    d.status = st;
    d.bin_offset = bin_ofs[s];
    d.nbins = (int32_t)((P[s].length + 1) / 2);
    if (st == AAK_OK) {
      const SourceDesc &sd = ctx->descs[s];
      d.grid_offset = ctx->offsets[s];
      d.i0 = sd.i0;
      d.ip = std::min(sd.i_plunge, sd.vlength - 1);  // the sum reads grid points 0 .. ip - 1
      d.nmodes = nm[s];
      d.bessel_offset = sd.bessel_offset;
      d.dt_ph = dt_ph[s];
      d.dOm = 2. * kPi / Tobs[s];
      d.DM = kAUsec * std::sin(P[s].theta_S);
      d.phiS = P[s].phi_S;
      d.arm = 2.5e9 / kC;
      tdi_geometry(P[s].theta_S, P[s].phi_S, P[s].theta_K, P[s].phi_K, &d);
      tdi_sidebands(P[s].theta_S, P[s].phi_S, P[s].theta_K, P[s].phi_K, std::cos(P[s].iota), std::sin(P[s].iota), d.AA);
    }
    const int64_t items = (st == AAK_OK && d.ip >= 2) ? (int64_t)(d.ip - 1) * 5 * d.nmodes : 0;
    work[s + 1] = work[s] + items;
  }
  const int64_t N = ctx->total_samples, nb = bin_ofs[nsrc];
  if ((r = ctx->d_out.reserve((size_t)kTdiRows * std::max<int64_t>(N, 1) + 6 * (size_t)nb)) != AAK_OK ||
      (r = ctx->d_tdi.reserve(nsrc)) != AAK_OK || (r = ctx->d_tdi_work.reserve(nsrc + 1)) != AAK_OK)
    return r;
  double *grid = ctx->d_out.ptr, *out = grid + (size_t)kTdiRows * std::max<int64_t>(N, 1);
  BatchView bv = batch_view(ctx, nullptr, nullptr, nullptr, nullptr, 0);
  bv.phase_out = grid;
  bv.phase_stride = N;
  bv.trajectory_only = 1;
  launch_tdi_grid(bv, ctx->num_sms, 0, nullptr);
  if ((r = cuda_ok(cudaMemcpyAsync(ctx->d_tdi.ptr, td.data(), nsrc * sizeof(TdiDesc), cudaMemcpyHostToDevice, 0))) ||
      (r = cuda_ok(cudaMemcpyAsync(ctx->d_tdi_work.ptr, work.data(), (nsrc + 1) * sizeof(int64_t),
                                   cudaMemcpyHostToDevice, 0))))
    return r;
  TdiArgs a;
  a.src = ctx->d_tdi.ptr;
  a.nsrc = nsrc;
  a.work_start = ctx->d_tdi_work.ptr;
  a.total_work = work[nsrc];
  a.grid = grid;
  a.grid_stride = N;
  a.bessel_start = ctx->d_bessel.ptr;
  a.out = out;
  a.out_stride = nb;
  launch_tdi_spa(a, 0);
  ctx->last_launches = 3;
  if ((r = cuda_ok(cudaGetLastError())) != AAK_OK) return r;
  for (int k = 0; k < 6; ++k)
    if ((r = cuda_ok(cudaMemcpyAsync(rows[k], out + k * nb, nb * sizeof(double), cudaMemcpyDeviceToHost, 0))) != AAK_OK)
      return r;
  if ((r = cuda_ok(cudaStreamSynchronize(0))) != AAK_OK) return r;
  return device_status(ctx);
}

// aak_wave_batch_host for batches worth streaming.  Host threads plan the
// sources (the few that bound the planning time first, the cheap ones early
// wherever the long ones can wait: plan_sources' streaming order); as they finish, the calling thread gathers them in groups of about
// nsrc / kStreamGroups (or takes what has finished when 10 ms pass without a
// full group) and, on one of two auxiliary
// contexts in turn, packs, uploads, generates and copies back each group on
// that context's own stream while planning goes on.  Most sources are small
// and finish early, so nearly all of the transfers and kernels hide behind
// the planning of the few long sources.  A group's plans are lent to the
// auxiliary context for its pack and upload and then handed back; at the end
// this context holds the whole batch's plan, as after aak_batch_plan (not
// uploaded).  Copies into pageable host buffers are synchronous: correct,
// with less overlap.
constexpr int kStreamMinSources = 32;
constexpr int kStreamGroups = 8;

int wave_batch_streamed(aak_ctx *ctx, const aak_params *P, int32_t nsrc, const int32_t *nm, int32_t nthreads,
                        double *hI, double *hII) {
  int r;
  if ((r = select_device(ctx->device)) != AAK_OK) return r;
  const std::vector<aak_params> Pv(P, P + nsrc);
  for (int k = 0; k < 2; ++k) {
    if (!ctx->aux[k]) {
      if ((r = aak_ctx_create(ctx->device, &ctx->aux[k])) != AAK_OK) return r;
      if ((r = cuda_ok(cudaStreamCreateWithFlags(&ctx->aux[k]->pipe_stream, cudaStreamNonBlocking))) != AAK_OK)
        return r;
    }
    ctx->aux[k]->precision = ctx->precision;
    ctx->aux[k]->variant[0] = ctx->variant[0];
    ctx->aux[k]->variant[1] = ctx->variant[1];
  }
  std::vector<int64_t> pre(nsrc + 1, 0);  // sample offsets of the sources in the host outputs
  for (int s = 0; s < nsrc; ++s) pre[s + 1] = pre[s] + Pv[s].length;
  std::mutex mu;
  std::condition_variable cv;
  std::vector<int> done;  // planned sources, in completion order
  done.reserve(nsrc);
  bool finished = false;
  int plan_rc = AAK_OK;
  std::thread planner([&]() {
    cudaSetDevice(ctx->device);
    const int rr = plan_sources(
        ctx, Pv, nullptr, nm, nthreads,
        [&](int s) {
          std::lock_guard<std::mutex> lk(mu);
          done.push_back(s);
          cv.notify_one();
        },
        true);
    std::lock_guard<std::mutex> lk(mu);
    finished = true;
    plan_rc = rr;
    cv.notify_one();
  });
  const int G = std::max(8, (nsrc + kStreamGroups - 1) / kStreamGroups);
  int taken = 0, slot = 0, rc = AAK_OK;
  bool pending[2] = {false, false};
  std::vector<int> grp;
  std::vector<aak_params> Pg;
  for (;;) {
    {
      // a full group, or whatever has finished once completions slow down
      // (the long sources at the end): each then leaves as soon as it is done
      std::unique_lock<std::mutex> lk(mu);
      cv.wait_for(lk, std::chrono::milliseconds(10), [&]() { return finished || (int)done.size() - taken >= G; });
      if (finished && plan_rc != AAK_OK) {
        rc = plan_rc;
        break;
      }
      const int avail = (int)done.size() - taken;
      if (avail == 0) {
        if (finished) break;  // all dispatched
        continue;
      }
      const int k = std::min(avail, G);
      grp.assign(done.begin() + taken, done.begin() + taken + k);
      taken += k;
    }
    aak_ctx *A = ctx->aux[slot];
    if (pending[slot]) {  // this context's previous group must be done with its device buffers
      pending[slot] = false;
      if ((rc = cuda_ok(cudaStreamSynchronize(A->pipe_stream))) != AAK_OK) break;
    }
    const int k = (int)grp.size();
    if ((int)A->plans.size() < k) A->plans.resize(k);
    Pg.resize(k);
    A->nsrc = k;
    A->status.resize(k);
    for (int i = 0; i < k; ++i) {
      std::swap(A->plans[i], ctx->plans[grp[i]]);
      A->status[i] = ctx->status[grp[i]];
      Pg[i] = Pv[grp[i]];
    }
    rc = pack(A, Pg, 2);
    // the knot copies read the plans' page-locked arrays, which nothing
    // refills before this call's streams are drained: no wait here
    if (rc == AAK_OK) rc = upload(A, A->pipe_stream, false);
    for (int i = 0; i < k; ++i) std::swap(A->plans[i], ctx->plans[grp[i]]);
    if (rc != AAK_OK) break;
    const int64_t N = A->total_samples;
    if ((rc = A->d_out.reserve((size_t)(2 * N))) != AAK_OK) break;
    double *dI = A->d_out.ptr, *dII = dI + N;
    if ((rc = run(A, dI, dII, nullptr, nullptr, 0, A->precision, A->pipe_stream)) != AAK_OK) break;
    for (int i = 0; i < k && rc == AAK_OK; ++i) {
      const int s = grp[i];
      const size_t bytes = (size_t)Pv[s].length * sizeof(double);
      if ((rc = cuda_ok(cudaMemcpyAsync(hI + pre[s], dI + A->offsets[i], bytes, cudaMemcpyDeviceToHost, A->pipe_stream))) ==
          AAK_OK)
        rc = cuda_ok(cudaMemcpyAsync(hII + pre[s], dII + A->offsets[i], bytes, cudaMemcpyDeviceToHost, A->pipe_stream));
    }
    if (rc != AAK_OK) break;
    pending[slot] = true;
    slot ^= 1;
  }
  planner.join();
  // the whole batch's plan in this context (every plan is back), packed while
  // the last groups' kernels and copies run
  if (rc == AAK_OK) rc = pack(ctx, Pv, nthreads);
  for (int k = 0; k < 2; ++k)  // drain both streams whatever happened
    if (pending[k]) {
      const int e = cuda_ok(cudaStreamSynchronize(ctx->aux[k]->pipe_stream));
      if (rc == AAK_OK) rc = e;
    }
  if (rc != AAK_OK) return rc;
  for (int k = 0; k < 2; ++k)
    if ((r = device_status(ctx->aux[k])) != AAK_OK) return r;
  return AAK_OK;
}

}  // namespace

extern "C" {

const char *aak_status_string(int s) {
  switch (s) {
    case AAK_OK: return "ok";
    case AAK_ERR_INVALID_PARAM: return "invalid parameter";
    case AAK_ERR_UNSTABLE_START: return "initial orbit inside the last stable orbit";
    case AAK_ERR_FIT_TOO_CLOSE_TO_PLUNGE: return "fitting error: t_0 too close to plunge";
    case AAK_ERR_SOLVER_NO_CONVERGE: return "Kerr-to-AK parameter map did not converge";
    case AAK_ERR_CUDA: return "CUDA error or no CUDA device";
    case AAK_ERR_NO_MEMORY: return "out of device memory";
    case AAK_ERR_TOO_FEW_STEPS: return "coarse inspiral produced fewer than 3 points";
    case AAK_ERR_CAPACITY: return "request exceeds a fixed-size buffer";
    case AAK_ERR_DEVICE_TIMEOUT: return "a bounded device-side wait gave up";
    default: return "unknown status";
  }
}

int aak_version(void) { return 10000; }

const char *aak_last_error_detail(void) { return last_error_buffer(); }

int aak_front_end(const aak_params *p, const double *warm, aak_mapped *out) {
  if (!p || !out) return AAK_ERR_INVALID_PARAM;
  MappedTrajectory mt;
  const int st = front_end(to_params(*p), &mt, warm);
  if (st == kOk) to_mapped(mt, out);
  else std::memset(out, 0, sizeof(*out));
  return st;
}

int aak_coarse_kerr(const aak_params *p, int32_t *steps, double *t_rr, double *pp, double *e, double *cosi,
                    double *Omega) {
  if (!p || !steps) return AAK_ERR_INVALID_PARAM;
  CoarseKerr ck;
  const int st = coarse_kerr(to_params(*p), &ck);
  *steps = ck.steps;
  for (int i = 0; i < ck.steps; ++i) {
    if (t_rr) t_rr[i] = ck.t_rr[i];
    if (pp) pp[i] = ck.p[i];
    if (e) e[i] = ck.e[i];
    if (cosi) cosi[i] = ck.cosi[i];
    if (Omega)
      for (int k = 0; k < 3; ++k) Omega[3 * i + k] = ck.Omega[i][k];
  }
  return st;
}

int aak_parmap(const double Omega[3], double p, double M, double s, double e, double iota, const double *x0,
               double map[3], int32_t *iterations) {
  if (!Omega || !map) return AAK_ERR_INVALID_PARAM;
  const int it = parmap(Omega, p, M, s, e, iota, x0, map);
  if (iterations) *iterations = it < 0 ? -it - 1 : it;
  return it < 0 ? AAK_ERR_SOLVER_NO_CONVERGE : AAK_OK;
}

int aak_ctx_create(int32_t device, aak_ctx **out) {
  if (!out) return AAK_ERR_INVALID_PARAM;
  *out = nullptr;
  if (device != -1) {  // -1: host-only context (planning without a GPU)
    const int r = select_device(device);
    if (r != AAK_OK) return r;
  }
  aak_ctx *c = new (std::nothrow) aak_ctx();
  if (!c) return AAK_ERR_NO_MEMORY;
  c->device = device;
  c->want_pinned = device >= 0;
  int sms = 0;
  if (device >= 0 && cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) == cudaSuccess && sms > 0)
    c->num_sms = sms;
  *out = c;
  return AAK_OK;
}

void aak_ctx_destroy(aak_ctx *c) {
  if (!c) return;
  if (c->device >= 0 && select_device(c->device) == AAK_OK) {
    c->d_src.release();
    c->d_tile_start.release();
    c->d_tile_knot.release();
    c->d_tile_pairs.release();
    c->d_queue.release();
    c->d_spl_blk.release();
    c->d_knot_t.release();
    c->d_knot_y.release();
    c->d_knot_c.release();
    c->d_bessel.release();
    c->d_link.release();
    c->d_flag.release();
    c->d_counter.release();
    c->d_tile_prep.release();
    c->d_tile_tab.release();
    c->d_out.release();
    c->d_tdi.release();
    c->d_tdi_work.release();
    c->d_pm_jobs.release();
    c->d_pm_warm.release();
    c->d_pm_map.release();
    c->d_pm_it.release();
    if (c->pm_stream) cudaStreamDestroy(c->pm_stream);
    for (auto &e : c->ev)
      if (e) cudaEventDestroy(e);
    drop_graph(c);
    if (c->cap_stream) cudaStreamDestroy(c->cap_stream);
    if (c->pipe_stream) cudaStreamDestroy(c->pipe_stream);
  }
  aak_ctx_destroy(c->aux[0]);
  aak_ctx_destroy(c->aux[1]);
  delete c;
}

int aak_batch_plan(aak_ctx *ctx, const aak_params *P, int32_t nsrc, const int32_t *nm, int32_t nthreads) {
  if (!ctx) return AAK_ERR_INVALID_PARAM;
  std::lock_guard<std::mutex> lk(ctx->mu);
  return plan_common(ctx, P, nullptr, nsrc, nm, nthreads);
}

int aak_batch_plan_mapped(aak_ctx *ctx, const aak_params *P, const aak_mapped *maps, int32_t nsrc, const int32_t *nm,
                          int32_t nthreads) {
  if (!ctx || !maps) return AAK_ERR_INVALID_PARAM;
  std::lock_guard<std::mutex> lk(ctx->mu);
  return plan_common(ctx, P, maps, nsrc, nm, nthreads);
}

int aak_ctx_set_parmap_model(aak_ctx *ctx, aak_mlp *m) {
  if (!ctx) return AAK_ERR_INVALID_PARAM;
  std::lock_guard<std::mutex> lk(ctx->mu);
  ctx->model = m;
  return AAK_OK;
}

int aak_batch_newton_stats(aak_ctx *ctx, int64_t *points, int64_t *iterations, int64_t *fallbacks) {
  if (!ctx) return AAK_ERR_INVALID_PARAM;
  std::lock_guard<std::mutex> lk(ctx->mu);
  if (points) *points = ctx->newton_points;
  if (iterations) *iterations = ctx->newton_iters;
  if (fallbacks) *fallbacks = ctx->newton_fallbacks;
  return AAK_OK;
}

int aak_batch_info(aak_ctx *ctx, int64_t *total, int64_t *offsets, int32_t *status, int32_t *i_plunge, int32_t *i_buffer) {
  if (!ctx) return AAK_ERR_INVALID_PARAM;
  std::lock_guard<std::mutex> lk(ctx->mu);
  if (total) *total = ctx->total_samples;
  for (int s = 0; s < ctx->nsrc; ++s) {
    if (status) status[s] = ctx->status[s];
    if (i_plunge) i_plunge[s] = ctx->status[s] == AAK_OK ? ctx->plans[s].i_plunge : -1;
    if (i_buffer) i_buffer[s] = ctx->status[s] == AAK_OK ? ctx->plans[s].i_buffer : -1;
  }
  if (offsets)
    for (int s = 0; s <= ctx->nsrc; ++s) offsets[s] = ctx->offsets[s];
  return AAK_OK;
}

int aak_batch_plan_bytes(aak_ctx *ctx, int64_t *bytes) {
  if (!ctx || !bytes) return AAK_ERR_INVALID_PARAM;
  std::lock_guard<std::mutex> lk(ctx->mu);
  // everything upload() copies: descriptors, tile and queue arrays, knots (t and
  // (e, v, M, S); the spline coefficients are solved on the device), Miller
  // start orders and the spline-block prefix
  *bytes = (int64_t)(ctx->descs.size() * sizeof(SourceDesc) + ctx->tile_start.size() * sizeof(int64_t) +
                     ctx->tile_knot.size() * sizeof(int32_t) + ctx->tile_pairs.size() * sizeof(int64_t) +
                     ctx->queue.size() * sizeof(QueueItem) + ctx->total_knots * (sizeof(double) + sizeof(double4)) +
                     ctx->bessel.size() * sizeof(int32_t) + ctx->spl_blk.size() * sizeof(int64_t));
  return AAK_OK;
}

int aak_batch_upload(aak_ctx *ctx, void *stream) {
  if (!ctx) return AAK_ERR_INVALID_PARAM;
  std::lock_guard<std::mutex> lk(ctx->mu);
  return upload(ctx, (cudaStream_t)stream);
}

int aak_batch_run(aak_ctx *ctx, double *hI, double *hII, double *t, double *traj, int64_t traj_stride,
                  int32_t precision, void *stream) {
  if (!ctx) return AAK_ERR_INVALID_PARAM;
  std::lock_guard<std::mutex> lk(ctx->mu);
  return run(ctx, hI, hII, t, traj, traj_stride, precision, (cudaStream_t)stream);
}

int aak_batch_run_plain(aak_ctx *ctx, double *d_hI, double *d_hII, double *d_traj, int64_t traj_stride, void *stream) {
  if (!ctx) return AAK_ERR_INVALID_PARAM;
  std::lock_guard<std::mutex> lk(ctx->mu);
  return run_plain(ctx, d_hI, d_hII, d_traj, traj_stride, (cudaStream_t)stream);
}

int aak_batch_run_noalloc(aak_ctx *ctx, void *d_plan, int64_t plan_bytes, int64_t *required_bytes, double *d_hI,
                          double *d_hII, void *stream) {
  if (!ctx) return AAK_ERR_INVALID_PARAM;
  std::lock_guard<std::mutex> lk(ctx->mu);
  if (ctx->nsrc <= 0) return AAK_ERR_INVALID_PARAM;
  // caller buffer layout: descriptors | tile prefix | tile knot windows | knot times |
  // knot values | knot second derivatives | Bessel start orders, each segment 256-byte
  // aligned
  auto al = [](size_t x) { return (x + 255) / 256 * 256; };
  const size_t o_ts = al(ctx->descs.size() * sizeof(SourceDesc));
  const size_t o_tk = o_ts + al(ctx->tile_start.size() * sizeof(int64_t));
  const size_t o_kt = o_tk + al(ctx->tile_knot.size() * sizeof(int32_t));
  const size_t nknots = (size_t)std::max<int64_t>(ctx->total_knots, 1);
  const size_t o_ky = o_kt + al(nknots * sizeof(double));
  const size_t o_kc = o_ky + al(nknots * sizeof(double4));
  const size_t o_bs = o_kc + al(nknots * sizeof(double4));
  const size_t o_sb = o_bs + al(ctx->bessel.size() * sizeof(int32_t));
  const size_t need = o_sb + al(ctx->spl_blk.size() * sizeof(int64_t));
  if (required_bytes) *required_bytes = (int64_t)need;
  if (!d_plan) return AAK_OK;  // size query only
  if (plan_bytes < 0 || (size_t)plan_bytes < need) return AAK_ERR_CAPACITY;
  if (ctx->total_tiles > kStaticScratchTiles) return AAK_ERR_CAPACITY;
  if (!d_hI || !d_hII || ((uintptr_t)d_plan & 255u) != 0) return AAK_ERR_INVALID_PARAM;
  int r;
  if ((r = select_device(ctx->device)) != AAK_OK) return r;
  cudaStream_t st = (cudaStream_t)stream;
  unsigned char *base = static_cast<unsigned char *>(d_plan);
  auto cp = [&](size_t off, const void *src, size_t bytes) {
    return cuda_ok(cudaMemcpyAsync(base + off, src, bytes, cudaMemcpyHostToDevice, st));
  };
  if ((r = cp(0, ctx->descs.data(), ctx->descs.size() * sizeof(SourceDesc))) ||
      (r = cp(o_ts, ctx->tile_start.data(), ctx->tile_start.size() * sizeof(int64_t))) ||
      (r = cp(o_tk, ctx->tile_knot.data(), ctx->tile_knot.size() * sizeof(int32_t))) ||
      (r = cp(o_bs, ctx->bessel.data(), ctx->bessel.size() * sizeof(int32_t))) ||
      (r = cp(o_sb, ctx->spl_blk.data(), ctx->spl_blk.size() * sizeof(int64_t))))
    return r;
  for (int s = 0; s < ctx->nsrc; ++s) {
    const SourcePlan &pl = ctx->plans[s];
    const int64_t nk = ctx->kofs[s + 1] - ctx->kofs[s];
    if (nk <= 0) continue;
    const size_t ko = (size_t)ctx->kofs[s];
    if ((r = cp(o_kt + ko * sizeof(double), pl.knot_t.data(), nk * sizeof(double))) ||
        (r = cp(o_ky + ko * sizeof(double4), pl.knot_y.data(), nk * sizeof(double4))))
      return r;
  }
  launch_spline_coeffs(reinterpret_cast<const SourceDesc *>(base), ctx->nsrc, reinterpret_cast<const int64_t *>(base + o_sb),
                       ctx->spl_blk[ctx->nsrc], reinterpret_cast<const double *>(base + o_kt),
                       reinterpret_cast<const double4 *>(base + o_ky), reinterpret_cast<double4 *>(base + o_kc), st);
  if ((r = cuda_ok(cudaGetLastError())) != AAK_OK) return r;
  if (ctx->want_pinned && (r = cuda_ok(cudaStreamSynchronize(st))) != AAK_OK) return r;  // host arrays reusable on return
  BatchView bv;
  std::memset(&bv, 0, sizeof(bv));
  bv.src = reinterpret_cast<const SourceDesc *>(base);
  bv.nsrc = ctx->nsrc;
  bv.total_tiles = ctx->total_tiles;
  bv.tile_start = reinterpret_cast<const int64_t *>(base + o_ts);
  bv.tile_knot = reinterpret_cast<const int32_t *>(base + o_tk);
  bv.knot_t = reinterpret_cast<const double *>(base + o_kt);
  bv.knot_y = reinterpret_cast<const double4 *>(base + o_ky);
  bv.knot_c = reinterpret_cast<const double4 *>(base + o_kc);
  bv.bessel_start = reinterpret_cast<const int32_t *>(base + o_bs);
  bv.max_nmodes = ctx->max_nmodes;
  bv.lookback_cycles = ctx->lookback_cycles;
  bv.hI = d_hI;
  bv.hII = d_hII;
  ctx->noalloc_used = true;
  return launch_dense_static_scratch(bv, ctx->device, ctx->num_sms, st, ctx->precision);
}

int aak_batch_last_launches(aak_ctx *ctx) { return ctx ? ctx->last_launches : 0; }

int aak_selftest_lookback_timeout(int64_t cycles) {
  const int v = lookback_timeout_selftest((long long)cycles, nullptr);
  if (v < 0) return cuda_ok(cudaGetLastError());
  return v == 1 ? AAK_OK : AAK_ERR_CUDA;
}

int aak_batch_device_status(aak_ctx *ctx) {
  if (!ctx) return AAK_ERR_INVALID_PARAM;
  std::lock_guard<std::mutex> lk(ctx->mu);
  return device_status(ctx);
}

int aak_batch_set_profiling(aak_ctx *ctx, int32_t on) {
  if (!ctx) return AAK_ERR_INVALID_PARAM;
  std::lock_guard<std::mutex> lk(ctx->mu);
  ctx->profile = on != 0;
  return AAK_OK;
}

int aak_batch_kernel_ms(aak_ctx *ctx, float *ms3) {
  if (!ctx || !ms3 || !ctx->profile || !ctx->ev[0]) return AAK_ERR_INVALID_PARAM;
  std::lock_guard<std::mutex> lk(ctx->mu);
  if (cudaEventSynchronize(ctx->ev[3]) != cudaSuccess) return cuda_ok(cudaGetLastError());
  for (int k = 0; k < 3; ++k)
    if (cudaEventElapsedTime(&ms3[k], ctx->ev[k], ctx->ev[k + 1]) != cudaSuccess) return cuda_ok(cudaGetLastError());
  return AAK_OK;
}

int aak_probe_fp32_tflops(int32_t device, double *tflops) {
  if (!tflops) return AAK_ERR_INVALID_PARAM;
  int r = select_device(device);
  if (r != AAK_OK) return r;
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  *tflops = probe_fp32_fma_tflops(sms, 20, 0);
  return *tflops > 0 ? AAK_OK : AAK_ERR_CUDA;
}

int aak_ctx_set_precision(aak_ctx *ctx, int32_t precision) {
  if (!ctx || (precision != 0 && precision != 1)) return AAK_ERR_INVALID_PARAM;
  std::lock_guard<std::mutex> lk(ctx->mu);
  ctx->precision = precision;
  return AAK_OK;
}

// ---------------------------------------------------------------- autotuner
// The launch shape of the waveform stage (wave_variant: tile pre-pass or
// tables inside the tiles, samples per thread in the harmonic loop, resident
// CTAs per SM) is chosen per (device, precision, largest harmonic count,
// sources and median length in powers of two) by timing every candidate on
// the uploaded batch; the choice and the timings are appended to a tuning
// cache file, and a later call with the same key reads the choice from there.
static_assert(AAK_NUM_VARIANTS == kNumVariants, "the header states the number of launch shapes");

namespace {

std::string tune_key(aak_ctx *ctx, int precision) {
  cudaDeviceProp prop;
  std::memset(&prop, 0, sizeof(prop));
  cudaGetDeviceProperties(&prop, ctx->device);
  std::string name(prop.name);
  for (auto &c : name)
    if (c == ' ' || c == '|') c = '_';
  std::vector<int32_t> len;
  for (const auto &d : ctx->descs) len.push_back(d.vlength);
  std::sort(len.begin(), len.end());
  const int32_t med = len.empty() ? 0 : len[len.size() / 2];
  auto lg = [](double x) { return x > 0 ? (int)std::lround(std::log2(x)) : 0; };
  char buf[256];
  std::snprintf(buf, sizeof(buf), "%s|sm%d|p%d|nm%d|src2^%d|len2^%d", name.c_str(), prop.multiProcessorCount, precision,
                ctx->max_nmodes, lg((double)ctx->nsrc), lg((double)med));
  return buf;
}

int tune_lookup(const char *path, const std::string &key, int *variant) {
  if (!path) return 0;
  FILE *f = std::fopen(path, "r");
  if (!f) return 0;
  char line[1024];
  int found = 0;
  while (std::fgets(line, sizeof(line), f)) {
    char k[512];
    int v = -1;
    if (std::sscanf(line, "%511s %d", k, &v) == 2 && key == k && v >= 0 && v < kNumVariants) {
      *variant = v;  // the last entry for a key wins
      found = 1;
    }
  }
  std::fclose(f);
  return found;
}

}  // namespace

int aak_ctx_autotune(aak_ctx *ctx, double *d_hI, double *d_hII, int32_t precision, const char *cache_path,
                     int32_t *variant, float *ms_per_variant) {
  if (!ctx || !d_hI || !d_hII || (precision != 0 && precision != 1)) return AAK_ERR_INVALID_PARAM;
  std::lock_guard<std::mutex> lk(ctx->mu);
  if (!ctx->uploaded) return AAK_ERR_INVALID_PARAM;
  int r;
  if ((r = select_device(ctx->device)) != AAK_OK) return r;
  const std::string key = tune_key(ctx, precision);
  if (ms_per_variant)
    for (int v = 0; v < kNumVariants; ++v) ms_per_variant[v] = -1.0f;
  int best = 0;
  if (tune_lookup(cache_path, key, &best)) {
    ctx->variant[precision] = best;
    if (variant) *variant = best;
    return AAK_OK;
  }
  cudaStream_t st = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if ((r = cuda_ok(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking))) != AAK_OK) return r;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float ms[kNumVariants];
  float best_ms = 0.0f;
  for (int v = 0; v < kNumVariants && r == AAK_OK; ++v) {
    BatchView bv = batch_view(ctx, d_hI, d_hII, nullptr, nullptr, 0);
    bv.variant = v;
    if ((r = tile_tables(ctx, precision, bv)) != AAK_OK) break;
    ms[v] = 0.0f;
    for (int rep = 0; rep < 3 && r == AAK_OK; ++rep) {  // one warm-up, then the faster of two
      cudaEventRecord(e0, st);
      launch_dense(bv, ctx->num_sms, st, nullptr, precision);
      cudaEventRecord(e1, st);
      if ((r = cuda_ok(cudaEventSynchronize(e1))) != AAK_OK) break;
      float t = 0.0f;
      cudaEventElapsedTime(&t, e0, e1);
      if (rep == 1 || (rep == 2 && t < ms[v])) ms[v] = t;
    }
    if (r != AAK_OK) break;
    if (ms_per_variant) ms_per_variant[v] = ms[v];
    if (v == 0 || ms[v] < best_ms) {
      best = v;
      best_ms = ms[v];
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaStreamDestroy(st);
  if (r != AAK_OK) return r;
  if ((r = device_status(ctx)) != AAK_OK) return r;  // a timing run must not have given up a wait
  ctx->variant[precision] = best;
  if (variant) *variant = best;
  if (cache_path) {
    FILE *f = std::fopen(cache_path, "a");
    if (f) {
      std::fprintf(f, "%s %d", key.c_str(), best);
      for (int v = 0; v < kNumVariants; ++v) std::fprintf(f, " %.4f", ms[v]);
      std::fprintf(f, "\n");
      std::fclose(f);
    }
  }
  return AAK_OK;
}

int aak_ctx_set_variant(aak_ctx *ctx, int32_t precision, int32_t variant) {
  if (!ctx || (precision != 0 && precision != 1) || variant < 0 || variant >= kNumVariants) return AAK_ERR_INVALID_PARAM;
  std::lock_guard<std::mutex> lk(ctx->mu);
  ctx->variant[precision] = variant;
  return AAK_OK;
}

int aak_ctx_set_lookback_bound(aak_ctx *ctx, int64_t cycles) {
  if (!ctx) return AAK_ERR_INVALID_PARAM;
  std::lock_guard<std::mutex> lk(ctx->mu);
  ctx->lookback_cycles = cycles > 0 ? (long long)cycles : 0;
  drop_graph(ctx);  // a captured launch holds the old bound
  return AAK_OK;
}

int aak_batch_run_graph(aak_ctx *ctx, double *d_hI, double *d_hII, int32_t precision, void *stream) {
  if (!ctx) return AAK_ERR_INVALID_PARAM;
  std::lock_guard<std::mutex> lk(ctx->mu);
  return run_graph(ctx, d_hI, d_hII, precision, (cudaStream_t)stream);
}

int aak_probe_fp64_tflops(int32_t device, double *tflops) {
  if (!tflops) return AAK_ERR_INVALID_PARAM;
  int r = select_device(device);
  if (r != AAK_OK) return r;
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  *tflops = probe_fp64_fma_tflops(sms, 20, 0);
  return *tflops > 0 ? AAK_OK : AAK_ERR_CUDA;
}

int aak_wave_batch_host(aak_ctx *ctx, const aak_params *P, int32_t nsrc, const int32_t *nm, int32_t nthreads,
                        double *h_hI, double *h_hII, int64_t *offsets, int32_t *status) {
  if (!ctx || !h_hI || !h_hII) return AAK_ERR_INVALID_PARAM;
  std::lock_guard<std::mutex> lk(ctx->mu);
  int r;
  if (nsrc >= kStreamMinSources && ctx->device >= 0 && ctx->out_stride == 0) {
    if (!P) return AAK_ERR_INVALID_PARAM;
    for (int32_t s = 0; s < nsrc; ++s)
      if (P[s].length < 2 || P[s].length > ((int64_t)1 << 31)) return AAK_ERR_INVALID_PARAM;
    r = wave_batch_streamed(ctx, P, nsrc, nm, nthreads, h_hI, h_hII);
  } else {
    r = plan_common(ctx, P, nullptr, nsrc, nm, nthreads);
    if (r == AAK_OK) r = host_roundtrip(ctx, nullptr, h_hI, h_hII);
  }
  if (r != AAK_OK) return r;
  if (offsets)
    for (int s = 0; s <= nsrc; ++s) offsets[s] = ctx->offsets[s];
  if (status)
    for (int s = 0; s < nsrc; ++s) status[s] = ctx->status[s];
  return AAK_OK;
}

int aak_wave(const aak_params *p, double *t, double *hI, double *hII, double *seconds) {
  if (!p || !t || !hI || !hII) return AAK_ERR_INVALID_PARAM;
  const auto t0 = std::chrono::steady_clock::now();
  aak_ctx *ctx = nullptr;
  int r = default_ctx(&ctx);
  if (r != AAK_OK) return r;
  std::lock_guard<std::mutex> lk(ctx->mu);
  r = plan_common(ctx, p, nullptr, 1, nullptr, 1);
  if (r != AAK_OK) return r;
  if (ctx->status[0] != AAK_OK) return ctx->status[0];
  r = host_roundtrip(ctx, t, hI, hII);
  if (seconds) *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return r;
}

int aak_phase(const aak_params *p, double *t, double *phase_r, double *phase_theta, double *phase_phi,
              double *omega_r, double *omega_theta, double *omega_phi, double *eccentricity, double *seconds) {
  if (!p || !t || !phase_r || !phase_theta || !phase_phi || !omega_r || !omega_theta || !omega_phi || !eccentricity)
    return AAK_ERR_INVALID_PARAM;
  const auto t0 = std::chrono::steady_clock::now();
  aak_ctx *ctx = nullptr;
  int r = default_ctx(&ctx);
  if (r != AAK_OK) return r;
  std::lock_guard<std::mutex> lk(ctx->mu);
  r = plan_common(ctx, p, nullptr, 1, nullptr, 1);
  if (r != AAK_OK) return r;
  if (ctx->status[0] != AAK_OK) return ctx->status[0];
  double *const rows[8] = {t, phase_r, phase_theta, phase_phi, omega_r, omega_theta, omega_phi, eccentricity};
  r = phase_roundtrip(ctx, rows, nullptr, 0);
  if (seconds) *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return r;
}

int aak_tdi(const aak_params *p, double *f, double *Xf_r, double *Xf_im, double *Yf_r, double *Yf_im, double *Zf_r,
            double *Zf_im, double *seconds) {
  if (!p || !Xf_r || !Xf_im || !Yf_r || !Yf_im || !Zf_r || !Zf_im) return AAK_ERR_INVALID_PARAM;
  const auto t0 = std::chrono::steady_clock::now();
  aak_ctx *ctx = nullptr;
  int r = default_ctx(&ctx);
  if (r != AAK_OK) return r;
  std::lock_guard<std::mutex> lk(ctx->mu);
  double *const rows[6] = {Xf_r, Xf_im, Yf_r, Yf_im, Zf_r, Zf_im};
  std::vector<int64_t> ofs;
  std::vector<int32_t> st;
  r = tdi_batch(ctx, p, 1, 1, rows, ofs, st);
  if (r != AAK_OK) return r;
  if (st[0] != AAK_OK) return st[0];
  if (f) {
    const double df = 1. / ((double)(p->length - 1) * p->dt);
    for (int64_t i = 0; i < (p->length + 1) / 2; ++i) f[i] = (double)i * df;
  }
  if (seconds) *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return AAK_OK;
}

int aak_tdi_batch_host(aak_ctx *ctx, const aak_params *P, int32_t nsrc, int32_t nthreads, double *h_out,
                       int64_t *bin_offsets, int32_t *status) {
  if (!ctx || !P || !h_out || nsrc < 1) return AAK_ERR_INVALID_PARAM;
  std::lock_guard<std::mutex> lk(ctx->mu);
  int64_t nb = 0;
  for (int s = 0; s < nsrc; ++s) {
    if (P[s].length < 2) return AAK_ERR_INVALID_PARAM;
    nb += (P[s].length + 1) / 2;
  }
  double *const rows[6] = {h_out, h_out + nb, h_out + 2 * nb, h_out + 3 * nb, h_out + 4 * nb, h_out + 5 * nb};
  std::vector<int64_t> ofs;
  std::vector<int32_t> st;
  const int r = tdi_batch(ctx, P, nsrc, nthreads, rows, ofs, st);
  if (r != AAK_OK) return r;
  if (bin_offsets)
    for (int s = 0; s <= nsrc; ++s) bin_offsets[s] = ofs[s];
  if (status)
    for (int s = 0; s < nsrc; ++s) status[s] = st[s];
  return AAK_OK;
}

int aak_batch_run_phase(aak_ctx *ctx, double *d_out, int64_t stride, void *stream) {
  if (!ctx) return AAK_ERR_INVALID_PARAM;
  std::lock_guard<std::mutex> lk(ctx->mu);
  return run_phase(ctx, d_out, stride, (cudaStream_t)stream);
}

int aak_phase_batch_host(aak_ctx *ctx, const aak_params *P, int32_t nsrc, int32_t nthreads, double *h_out,
                         int64_t *offsets, int32_t *status) {
  if (!ctx || !P || !h_out || nsrc < 1) return AAK_ERR_INVALID_PARAM;
  std::lock_guard<std::mutex> lk(ctx->mu);
  int r = plan_common(ctx, P, nullptr, nsrc, nullptr, nthreads);
  if (r == AAK_OK) r = phase_roundtrip(ctx, nullptr, h_out, ctx->total_samples);
  if (r != AAK_OK) return r;
  if (offsets)
    for (int s = 0; s <= nsrc; ++s) offsets[s] = ctx->offsets[s];
  if (status)
    for (int s = 0; s < nsrc; ++s) status[s] = ctx->status[s];
  return AAK_OK;
}

int aak_genwave(double *t, double *hI, double *hII, double timestep, int32_t vlength, const double *e_traj,
                const double *v_map, double M_phys, const double *M_map, double mu, double S_phys, const double *S_map,
                double dist, double inc, double gim0, double Phi0, double qS, double phiS, double alp0, double qK,
                double phiK, const double *dt_map, int32_t steps, int32_t backint, int32_t mich, int32_t nmodes_override) {
  if (!t || !hI || !hII || !e_traj || !v_map || !M_map || !S_map || !dt_map) return AAK_ERR_INVALID_PARAM;
  if (steps < 3 || steps > kMaxCoarseSteps || vlength < 2) return AAK_ERR_INVALID_PARAM;
  aak_params p;
  std::memset(&p, 0, sizeof(p));
  p.length = vlength;
  p.dt = timestep;
  p.mu = mu;
  p.M = M_phys;
  p.s = S_phys;
  p.e = e_traj[0];
  p.iota = inc;
  p.gamma = gim0;
  p.theta_S = qS;
  p.phi_S = phiS;
  p.theta_K = qK;
  p.phi_K = phiK;
  p.alpha = alp0;
  p.D = dist;
  p.p = 1.0;
  p.T_fit = 1.0;
  p.backint = backint;
  p.LISA = mich;
  aak_mapped m;
  std::memset(&m, 0, sizeof(m));
  m.steps = steps;
  m.Phi0 = Phi0;
  for (int i = 0; i < steps; ++i) {
    m.e_traj[i] = e_traj[i];
    m.v_map[i] = v_map[i];
    m.M_map[i] = M_map[i];
    m.s_map[i] = S_map[i];
    m.dt_map[i] = dt_map[i];
  }
  aak_ctx *ctx = nullptr;
  int r = default_ctx(&ctx);
  if (r != AAK_OK) return r;
  std::lock_guard<std::mutex> lk(ctx->mu);
  const int32_t nm = nmodes_override;
  r = plan_common(ctx, &p, &m, 1, &nm, 1);
  if (r != AAK_OK) return r;
  if (ctx->status[0] != AAK_OK) return ctx->status[0];
  return host_roundtrip(ctx, t, hI, hII);
}


// ====================================================================== GPU likelihood
// GPUAAK counterpart (include/AAK_manager.hh:106-153, src/cuda/AAK_manager.cu):
// templates are generated into FFT-padded rows, transformed in place by a
// batched cuFFT D2Z plan and reduced against the pre-weighted data.
struct aak_gpu {
  aak_ctx *ctx = nullptr;
  double T_fit = 1.0, dt = 0.0, init_dt = 0.0;
  int32_t length = 0, init_length = 0, LISA = 1, backint = 0, precision = 0;
  int64_t nbins = 0;  // length / 2 + 1
  int64_t row = 0;    // doubles per padded template row = 2 * nbins
  DevBuf<double> d_H[2], d_D[2], d_w[2], d_partial, d_out, d_t;
  DevBuf<double> d_fisher;  // Fisher Gram partial sums and the 2 x nd x nd result
  cufftHandle plan = 0;
  int plan_batch = 0;
  // precision 2: FP32 template rows, an FP32 R2C transform and the FP32 copies
  // of the data and weights (the compensated FP32 inner products)
  DevBuf<float> d_H32[2], d_D32[2], d_w32[2];
  cufftHandle plan32 = 0;
  int plan32_batch = 0;
  bool rows32 = false;   // the rows of the last generation are the FP32 ones
  int32_t count = 0;     // templates currently in the rows
  bool spectral = false; // rows hold spectra (after a likelihood)
  std::vector<double> like;
  double ms[4] = {0, 0, 0, 0};  // host plan, generate, FFT, reduce of the last batch
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  // device work of the templates: its own non-blocking stream, so that host
  // planning (and the warm-start model's copies) can overlap it
  cudaStream_t stream = nullptr;
  // likelihood batches in chunks, double-buffered: chunk c is planned into
  // ctxs()[c & 1] and uploaded on up_stream while the chunk before it runs
  aak_ctx *ctx2 = nullptr;
  cudaStream_t up_stream = nullptr;
  // per parity: upload done, generation done, generation start, transform
  // done, reduction done, results copied
  cudaEvent_t pev[2][6] = {{nullptr}};
  double *h_stage = nullptr;  // page-locked results of the two chunks in flight (2 x 2 x stage_cap)
  int stage_cap = 0;
};

namespace {

int gpu_capacity(aak_gpu *g, int B) {
  int r;
  if ((r = g->d_H[0].reserve((size_t)B * g->row)) || (r = g->d_H[1].reserve((size_t)B * g->row)) ||
      (r = g->d_partial.reserve((size_t)B * kIpBlocksPerTemplate * 2)) || (r = g->d_out.reserve((size_t)B * 2)))
    return r;
  if (g->plan_batch < B) {
    if (g->plan) cufftDestroy(g->plan);
    g->plan = 0;
    g->plan_batch = 0;
    int n = g->length;
    int inembed = (int)g->row, onembed = (int)(g->row / 2);
    if (cufftPlanMany(&g->plan, 1, &n, &inembed, 1, (int)g->row, &onembed, 1, (int)(g->row / 2), CUFFT_D2Z, B) !=
        CUFFT_SUCCESS) {
      g->plan = 0;
      return AAK_ERR_CUDA;
    }
    g->plan_batch = B;
  }
  return AAK_OK;
}

int gpu_capacity32(aak_gpu *g, int B) {
  int r;
  if ((r = g->d_H32[0].reserve((size_t)B * g->row)) || (r = g->d_H32[1].reserve((size_t)B * g->row)) ||
      (r = g->d_partial.reserve((size_t)B * kIpBlocksPerTemplate * 2)) || (r = g->d_out.reserve((size_t)B * 2)))
    return r;
  if (g->plan32_batch != B) {  // an exact-size plan: a larger one would transform stale rows
    if (g->plan32) cufftDestroy(g->plan32);
    g->plan32 = 0;
    g->plan32_batch = 0;
    int n = g->length;
    int inembed = (int)g->row, onembed = (int)(g->row / 2);
    if (cufftPlanMany(&g->plan32, 1, &n, &inembed, 1, (int)g->row, &onembed, 1, (int)(g->row / 2), CUFFT_R2C, B) !=
        CUFFT_SUCCESS) {
      g->plan32 = 0;
      return AAK_ERR_CUDA;
    }
    g->plan32_batch = B;
  }
  return AAK_OK;
}

// Parameters in gpu_gen_AAK order: iota, s, p, e, M, mu, gamma, psi, alph, theta_S, phi_S, theta_K, phi_K, D.
aak_params gpu_params(const aak_gpu *g, const double *x) {
  aak_params p;
  std::memset(&p, 0, sizeof(p));
  p.length = g->length;
  p.dt = g->dt;
  p.T = g->length * g->dt / kYear;
  p.f = 0.0;
  p.T_fit = g->T_fit;
  p.iota = x[0];
  p.s = x[1];
  p.p = x[2];
  p.e = x[3];
  p.M = x[4];
  p.mu = x[5];
  p.gamma = x[6];
  p.psi = x[7];
  p.alpha = x[8];
  p.theta_S = x[9];
  p.phi_S = x[10];
  p.theta_K = x[11];
  p.phi_K = x[12];
  p.D = x[13];
  p.LISA = g->LISA;
  p.backint = g->backint;
  return p;
}

// Host half of a batch of templates: plan them into the context's rows.
// Plan B templates into context C (rows of g->row doubles); *ms: host time.
// The front end of a chunk of templates with the learned warm start, done
// ahead of the chunk's planning: coarse Kerr inspirals on host threads, one
// prediction launch for every coarse point of the chunk, then the map solves
// from the predictions (the planner's own warm-started front end, step for
// step).  fe[k]: the front end's status of template k, maps[k] its mapped
// trajectory where that is AAK_OK.
struct WarmFrontEnd {
  std::vector<aak_mapped> maps;
  std::vector<int32_t> fe;
};

int front_end_warm(aak_ctx *ctx, const aak_params *P, int B, int nthreads, WarmFrontEnd *out) {
  out->maps.resize(B);
  out->fe.assign(B, AAK_OK);
  std::vector<CoarseKerr> ck(B);
  parallel_for(B, nthreads, [&](int64_t s) {
    const Params Pp = to_params(P[s]);
    int st = validate(Pp);
    if (st == kOk) st = coarse_kerr(Pp, &ck[s]);
    out->fe[s] = st;
  });
  std::vector<int64_t> first(B + 1, 0);
  for (int s = 0; s < B; ++s) first[s + 1] = first[s] + (out->fe[s] == kOk ? ck[s].steps : 0);
  const int64_t np = first[B];
  std::vector<double> xs(4 * np), ys(3 * np), warm(3 * np);
  for (int s = 0; s < B; ++s)
    for (int64_t i = 0; i < first[s + 1] - first[s]; ++i) {
      double *x = &xs[4 * (first[s] + i)];
      x[0] = ck[s].p[i];
      x[1] = ck[s].e[i];
      x[2] = P[s].iota;
      x[3] = P[s].s;
    }
  if (np > 0) {
    const int r = mlp_predict_host(ctx->model, xs.data(), ys.data(), np);
    if (r != AAK_OK) return r;
  }
  for (int s = 0; s < B; ++s)
    for (int64_t i = first[s]; i < first[s + 1]; ++i) parmap_from_coords(&xs[4 * i], P[s].M, &ys[3 * i], &warm[3 * i]);
  parallel_for(B, nthreads, [&](int64_t s) {
    if (out->fe[s] != kOk) return;
    MappedTrajectory mt;
    int fb = 0;
    const int st = map_coarse(to_params(P[s]), ck[s], &mt, &warm[3 * first[s]], &fb);
    out->fe[s] = st;
    if (st == kOk) to_mapped(mt, &out->maps[s]);
  });
  return AAK_OK;
}

// Plan a chunk of templates into C.  With fe (a warm front end done ahead),
// the planner starts from its mapped trajectories; templates whose front end
// failed are planned as invalid and reported with the front end's status.
int gpu_plan_into(aak_gpu *g, aak_ctx *C, const double *x, int B, int nthreads, int32_t *status, double *ms,
                  const WarmFrontEnd *fe = nullptr) {
  std::vector<aak_params> P(B);
  for (int k = 0; k < B; ++k) P[k] = gpu_params(g, x + 14 * (size_t)k);
  if (fe)
    for (int k = 0; k < B; ++k)
      if (fe->fe[k] != AAK_OK) P[k].e = 0.0;  // rejected by the per-source validation, not planned
  const auto t0 = std::chrono::steady_clock::now();
  C->out_stride = g->row;
  const int r = plan_common(C, P.data(), fe ? fe->maps.data() : nullptr, B, nullptr, nthreads);
  C->out_stride = 0;
  *ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  if (r != AAK_OK) return r;
  if (fe)
    for (int k = 0; k < B; ++k)
      if (fe->fe[k] != AAK_OK) C->status[k] = fe->fe[k];
  for (int k = 0; k < B; ++k)
    if (status) status[k] = C->status[k];
  return AAK_OK;
}

int gpu_plan(aak_gpu *g, const double *x, int B, int nthreads, int32_t *status) {
  return gpu_plan_into(g, g->ctx, x, B, nthreads, status, &g->ms[0]);
}

// Device half: upload the planned batch and generate it into the rows
// (asynchronous after the upload, on the legacy default stream).
int gpu_launch(aak_gpu *g, int B, bool with_t, bool rows32 = false) {
  int r;
  if (rows32 && !with_t) {  // precision 2 (likelihood batches): split templates into FP32 rows
    if ((r = gpu_capacity32(g, B)) != AAK_OK) return r;
    if ((r = upload(g->ctx, g->stream)) != AAK_OK) return r;
    if (!g->ev[0])
      for (auto &e : g->ev) cudaEventCreate(&e);
    cudaEventRecord(g->ev[0], g->stream);
    if ((r = run_rows32(g->ctx, g->d_H32[0].ptr, g->d_H32[1].ptr, 1, g->stream)) != AAK_OK) return r;
    cudaEventRecord(g->ev[1], g->stream);
    g->count = B;
    g->spectral = false;
    g->rows32 = true;
    return AAK_OK;
  }
  g->rows32 = false;
  if ((r = gpu_capacity(g, B)) != AAK_OK) return r;
  if ((r = upload(g->ctx, g->stream)) != AAK_OK) return r;
  double *dt = nullptr;
  if (with_t) {
    if ((r = g->d_t.reserve((size_t)g->row)) != AAK_OK) return r;
    if ((r = cuda_ok(cudaMemsetAsync(g->d_t.ptr, 0, g->row * sizeof(double), g->stream))) != AAK_OK) return r;
    dt = g->d_t.ptr;
  }
  if (!g->ev[0])
    for (auto &e : g->ev) cudaEventCreate(&e);
  cudaEventRecord(g->ev[0], g->stream);
  if ((r = run(g->ctx, g->d_H[0].ptr, g->d_H[1].ptr, dt, nullptr, 0, g->precision == 0 ? 0 : 1, g->stream)) !=
      AAK_OK)
    return r;
  cudaEventRecord(g->ev[1], g->stream);
  g->count = B;
  g->spectral = false;
  return AAK_OK;
}

int gpu_generate(aak_gpu *g, const double *x, int B, int nthreads, int32_t *status, bool with_t) {
  const int r = gpu_plan(g, x, B, nthreads, status);
  return r != AAK_OK ? r : gpu_launch(g, B, with_t);
}

// In-place D2Z transforms of the rows of both channels (once per generation).
int gpu_fft_rows(aak_gpu *g) {
  if (!g->spectral && g->rows32) {
    int r = gpu_capacity32(g, g->count);
    if (r != AAK_OK) return r;
    if (cufftSetStream(g->plan32, g->stream) != CUFFT_SUCCESS) return AAK_ERR_CUDA;
    if (cufftExecR2C(g->plan32, g->d_H32[0].ptr, reinterpret_cast<cufftComplex *>(g->d_H32[0].ptr)) != CUFFT_SUCCESS ||
        cufftExecR2C(g->plan32, g->d_H32[1].ptr, reinterpret_cast<cufftComplex *>(g->d_H32[1].ptr)) != CUFFT_SUCCESS)
      return AAK_ERR_CUDA;
    g->spectral = true;
    return AAK_OK;
  }
  if (!g->spectral) {
    if (g->plan_batch != g->count) {
      // a plan of a larger batch would transform stale rows: make one of this size
      if (g->plan) cufftDestroy(g->plan);
      g->plan = 0;
      g->plan_batch = 0;
      int r = gpu_capacity(g, g->count);
      if (r != AAK_OK) return r;
    }
    if (cufftSetStream(g->plan, g->stream) != CUFFT_SUCCESS) return AAK_ERR_CUDA;
    if (cufftExecD2Z(g->plan, g->d_H[0].ptr, reinterpret_cast<cufftDoubleComplex *>(g->d_H[0].ptr)) != CUFFT_SUCCESS ||
        cufftExecD2Z(g->plan, g->d_H[1].ptr, reinterpret_cast<cufftDoubleComplex *>(g->d_H[1].ptr)) != CUFFT_SUCCESS)
      return AAK_ERR_CUDA;
    g->spectral = true;
  }
  return AAK_OK;
}

// The weighted inner products of the transformed rows into d_out, on the
// likelihood's stream.
int gpu_inner_products(aak_gpu *g) {
  if (g->rows32) {
    InnerProductArgs32 a;
    for (int ch = 0; ch < 2; ++ch) {
      a.H[ch] = g->d_H32[ch].ptr;
      a.D[ch] = g->d_D32[ch].ptr;
      a.w[ch] = g->d_w32[ch].ptr;
    }
    a.row_floats = g->row;
    a.nbins = g->nbins;
    a.ntemplates = g->count;
    a.partial = g->d_partial.ptr;
    a.out = g->d_out.ptr;
    launch_inner_products_f32(a, g->stream);
    return cuda_ok(cudaGetLastError());
  }
  InnerProductArgs a;
  a.H[0] = g->d_H[0].ptr;
  a.H[1] = g->d_H[1].ptr;
  a.row_doubles = g->row;
  a.D[0] = g->d_D[0].ptr;
  a.D[1] = g->d_D[1].ptr;
  a.w[0] = g->d_w[0].ptr;
  a.w[1] = g->d_w[1].ptr;
  a.nbins = g->nbins;
  a.ntemplates = g->count;
  a.partial = g->d_partial.ptr;
  a.out = g->d_out.ptr;
  launch_inner_products(a, g->stream);
  return cuda_ok(cudaGetLastError());
}

// FFT of the rows and the weighted inner products, queued on the
// likelihood's stream; gpu_likelihood_finish copies the results back.
int gpu_likelihood_launch(aak_gpu *g) {
  if (g->count <= 0) return AAK_ERR_INVALID_PARAM;
  if (!g->ev[0])
    for (auto &e : g->ev) cudaEventCreate(&e);
  int r0 = gpu_fft_rows(g);
  if (r0 != AAK_OK) return r0;
  cudaEventRecord(g->ev[2], g->stream);
  if ((r0 = gpu_inner_products(g)) != AAK_OK) return r0;
  cudaEventRecord(g->ev[3], g->stream);
  return AAK_OK;
}

// ------------------------------------------------------------ pipelined likelihood batches
// The second planning context, the upload stream, the events and the
// page-locked result slots of aak_gpu_likelihood_batch (created on first use,
// grown with max_batch); the second context takes the first one's settings.
int gpu_pipeline_ready(aak_gpu *g, int max_batch) {
  int r;
  if (!g->ctx2 && (r = aak_ctx_create(g->ctx->device, &g->ctx2)) != AAK_OK) return r;
  aak_ctx *a = g->ctx, *b = g->ctx2;
  b->want_pinned = a->want_pinned;
  b->parmap_device = a->parmap_device;
  b->evolve_device = a->evolve_device;
  b->model = a->model;
  b->precision = a->precision;
  b->lookback_cycles = a->lookback_cycles;
  b->variant[0] = a->variant[0];
  b->variant[1] = a->variant[1];
  if (!g->up_stream && (r = cuda_ok(cudaStreamCreateWithFlags(&g->up_stream, cudaStreamNonBlocking))) != AAK_OK)
    return r;
  for (auto &row : g->pev)
    for (auto &e : row)
      if (!e && (r = cuda_ok(cudaEventCreate(&e))) != AAK_OK) return r;
  if (g->stage_cap < max_batch) {
    if (g->h_stage) cudaFreeHost(g->h_stage);
    g->h_stage = nullptr;
    g->stage_cap = 0;
    if ((r = cuda_ok(cudaHostAlloc(reinterpret_cast<void **>(&g->h_stage), 4 * (size_t)max_batch * sizeof(double),
                                   cudaHostAllocDefault))) != AAK_OK)
      return r;
    g->stage_cap = max_batch;
  }
  return AAK_OK;
}

// Chunk of B templates planned in C, result slot p: C's plan is uploaded on
// up_stream (after the generation of the chunk two back, the last reader of
// C's device buffers), then on the likelihood's stream the rows are
// generated, transformed and reduced, and the results copied to slot p.
int gpu_chunk_launch(aak_gpu *g, aak_ctx *C, int p, int B) {
  cudaEvent_t *E = g->pev[p];
  const bool r32 = g->precision == 2 && g->d_D32[0].ptr;
  int r;
  if ((r = r32 ? gpu_capacity32(g, B) : gpu_capacity(g, B)) != AAK_OK) return r;
  if ((r = cuda_ok(cudaStreamWaitEvent(g->up_stream, E[1], 0))) != AAK_OK) return r;
  if ((r = upload(C, g->up_stream, false)) != AAK_OK) return r;
  if ((r = cuda_ok(cudaEventRecord(E[0], g->up_stream))) != AAK_OK ||
      (r = cuda_ok(cudaStreamWaitEvent(g->stream, E[0], 0))) != AAK_OK)
    return r;
  cudaEventRecord(E[2], g->stream);
  if (r32) r = run_rows32(C, g->d_H32[0].ptr, g->d_H32[1].ptr, 1, g->stream);
  else r = run(C, g->d_H[0].ptr, g->d_H[1].ptr, nullptr, nullptr, 0, g->precision == 0 ? 0 : 1, g->stream);
  if (r != AAK_OK) return r;
  cudaEventRecord(E[1], g->stream);
  g->count = B;
  g->spectral = false;
  g->rows32 = r32;
  if ((r = gpu_fft_rows(g)) != AAK_OK) return r;
  cudaEventRecord(E[3], g->stream);
  if ((r = gpu_inner_products(g)) != AAK_OK) return r;
  cudaEventRecord(E[4], g->stream);
  if ((r = cuda_ok(cudaMemcpyAsync(g->h_stage + 2 * (size_t)g->stage_cap * p, g->d_out.ptr,
                                   2 * (size_t)B * sizeof(double), cudaMemcpyDeviceToHost, g->stream))) != AAK_OK)
    return r;
  return cuda_ok(cudaEventRecord(E[5], g->stream));
}

// Wait for the chunk in slot p, copy its B results to out and add its device
// times (generate, FFT, reduce) to ms[1..3].
int gpu_chunk_collect(aak_gpu *g, int p, int B, double *out, double *ms) {
  cudaEvent_t *E = g->pev[p];
  const int r = cuda_ok(cudaEventSynchronize(E[5]));
  if (r != AAK_OK) return r;
  std::memcpy(out, g->h_stage + 2 * (size_t)g->stage_cap * p, 2 * (size_t)B * sizeof(double));
  float f;
  if (cudaEventElapsedTime(&f, E[2], E[1]) == cudaSuccess) ms[1] += f;
  if (cudaEventElapsedTime(&f, E[1], E[3]) == cudaSuccess) ms[2] += f;
  if (cudaEventElapsedTime(&f, E[3], E[4]) == cudaSuccess) ms[3] += f;
  cudaGetLastError();
  return AAK_OK;
}

int gpu_likelihood_finish(aak_gpu *g, double *out) {
  int r = cuda_ok(cudaMemcpyAsync(out, g->d_out.ptr, (size_t)g->count * 2 * sizeof(double), cudaMemcpyDeviceToHost,
                                  g->stream));
  if (r == AAK_OK) r = cuda_ok(cudaStreamSynchronize(g->stream));
  if (r != AAK_OK) return r;
  float f;
  if (cudaEventElapsedTime(&f, g->ev[0], g->ev[1]) == cudaSuccess) g->ms[1] = f;
  if (cudaEventElapsedTime(&f, g->ev[1], g->ev[2]) == cudaSuccess) g->ms[2] = f;
  if (cudaEventElapsedTime(&f, g->ev[2], g->ev[3]) == cudaSuccess) g->ms[3] = f;
  cudaGetLastError();
  return AAK_OK;
}

int gpu_likelihood(aak_gpu *g, double *out) {
  const int r = gpu_likelihood_launch(g);
  return r != AAK_OK ? r : gpu_likelihood_finish(g, out);
}

// Fisher matrix of one point (pygpuAAK/pygpuAAK.py:269-300): the 2 nd
// finite-difference templates are planned and generated as one batch into
// the rows, transformed, and reduced on the device to the per-channel Gram
// matrices of the weighted differences; only 2 nd^2 doubles come back.
int gpu_fisher(aak_gpu *g, const double *x, int nd, double scale, int nthreads, double *gram, int32_t *status) {
  if (nd < 1 || nd > kFisherMaxDim || !x || !gram || !std::isfinite(scale)) return AAK_ERR_INVALID_PARAM;
  if (!g->d_w[0].ptr || !g->d_w[1].ptr) return AAK_ERR_INVALID_PARAM;  // input_data first: the weights
  const int B = 2 * nd;
  int r = gpu_generate(g, x, B, nthreads, status, false);
  if (r != AAK_OK) return r;
  if ((r = gpu_fft_rows(g)) != AAK_OK) return r;
  const int grid = fisher_grid(g->ctx->num_sms, g->nbins);
  const int64_t need = fisher_partial_doubles(nd, grid) + 2 * (int64_t)nd * nd;
  if ((r = g->d_fisher.reserve((size_t)need)) != AAK_OK) return r;
  cudaEventRecord(g->ev[2], g->stream);
  FisherArgs a;
  a.H[0] = g->d_H[0].ptr;
  a.H[1] = g->d_H[1].ptr;
  a.row_doubles = g->row;
  a.w[0] = g->d_w[0].ptr;
  a.w[1] = g->d_w[1].ptr;
  a.nbins = g->nbins;
  a.nd = nd;
  a.scale = scale;
  a.partial = g->d_fisher.ptr;
  a.out = g->d_fisher.ptr + fisher_partial_doubles(nd, grid);
  launch_fisher_gram(a, g->ctx->num_sms, g->stream);
  cudaEventRecord(g->ev[3], g->stream);
  if ((r = cuda_ok(cudaGetLastError())) != AAK_OK) return r;
  if ((r = cuda_ok(cudaMemcpyAsync(gram, a.out, 2 * (size_t)nd * nd * sizeof(double), cudaMemcpyDeviceToHost,
                                   g->stream))) != AAK_OK)
    return r;
  if ((r = cuda_ok(cudaStreamSynchronize(g->stream))) != AAK_OK) return r;
  float f;
  if (cudaEventElapsedTime(&f, g->ev[0], g->ev[1]) == cudaSuccess) g->ms[1] = f;
  if (cudaEventElapsedTime(&f, g->ev[1], g->ev[2]) == cudaSuccess) g->ms[2] = f;
  if (cudaEventElapsedTime(&f, g->ev[2], g->ev[3]) == cudaSuccess) g->ms[3] = f;
  cudaGetLastError();
  return device_status(g->ctx);
}

// The device half of one Fisher point planned in C, slot p: C's plan is
// uploaded on up_stream (after the generation of the point two back, the
// last reader of C's device buffers), then on the likelihood's stream the 2 nd
// rows are generated, transformed and reduced to the Gram matrices, which are
// copied to page-locked slot p.  Events as gpu_chunk_launch's.
int gpu_fisher_point_launch(aak_gpu *g, aak_ctx *C, int p, int nd, double scale, int grid) {
  cudaEvent_t *E = g->pev[p];
  int r;
  if ((r = cuda_ok(cudaStreamWaitEvent(g->up_stream, E[1], 0))) != AAK_OK) return r;
  if ((r = upload(C, g->up_stream, false)) != AAK_OK) return r;
  if ((r = cuda_ok(cudaEventRecord(E[0], g->up_stream))) != AAK_OK ||
      (r = cuda_ok(cudaStreamWaitEvent(g->stream, E[0], 0))) != AAK_OK)
    return r;
  cudaEventRecord(E[2], g->stream);
  if ((r = run(C, g->d_H[0].ptr, g->d_H[1].ptr, nullptr, nullptr, 0, g->precision == 0 ? 0 : 1, g->stream)) != AAK_OK)
    return r;
  cudaEventRecord(E[1], g->stream);
  g->count = 2 * nd;
  g->spectral = false;
  g->rows32 = false;
  if ((r = gpu_fft_rows(g)) != AAK_OK) return r;
  cudaEventRecord(E[3], g->stream);
  FisherArgs a;
  a.H[0] = g->d_H[0].ptr;
  a.H[1] = g->d_H[1].ptr;
  a.row_doubles = g->row;
  a.w[0] = g->d_w[0].ptr;
  a.w[1] = g->d_w[1].ptr;
  a.nbins = g->nbins;
  a.nd = nd;
  a.scale = scale;
  a.partial = g->d_fisher.ptr;
  a.out = g->d_fisher.ptr + fisher_partial_doubles(nd, grid);
  launch_fisher_gram(a, g->ctx->num_sms, g->stream);
  if ((r = cuda_ok(cudaGetLastError())) != AAK_OK) return r;
  cudaEventRecord(E[4], g->stream);
  if ((r = cuda_ok(cudaMemcpyAsync(g->h_stage + 2 * (size_t)g->stage_cap * p, a.out, 2 * (size_t)nd * nd * sizeof(double),
                                   cudaMemcpyDeviceToHost, g->stream))) != AAK_OK)
    return r;
  return cuda_ok(cudaEventRecord(E[5], g->stream));
}

// Fisher matrices of npts points, pipelined as the likelihood batches are:
// point k + 1 is planned on host threads into the other planning context while
// the device generates, transforms and reduces point k.
int gpu_fisher_batch(aak_gpu *g, const double *x, int npts, int nd, double scale, int nthreads, double *gram,
                     int32_t *status) {
  if (npts < 1 || nd < 1 || nd > kFisherMaxDim || !x || !gram || !std::isfinite(scale)) return AAK_ERR_INVALID_PARAM;
  if (!g->d_w[0].ptr || !g->d_w[1].ptr) return AAK_ERR_INVALID_PARAM;  // input_data first: the weights
  const int B = 2 * nd;
  int r;
  // result slots of 2 nd^2 doubles (the page-locked stage holds two of 2 x stage_cap)
  if ((r = gpu_pipeline_ready(g, std::max(B, nd * nd))) != AAK_OK) return r;
  if (g->plan_batch != B) {  // an exact-size transform plan of the rows, made once before the loop
    if (g->plan) cufftDestroy(g->plan);
    g->plan = 0;
    g->plan_batch = 0;
  }
  if ((r = gpu_capacity(g, B)) != AAK_OK) return r;
  const int grid = fisher_grid(g->ctx->num_sms, g->nbins);
  if ((r = g->d_fisher.reserve((size_t)(fisher_partial_doubles(nd, grid) + 2 * (int64_t)nd * nd))) != AAK_OK) return r;
  aak_ctx *ctxs[2] = {g->ctx, g->ctx2};
  auto fail = [&](int e) {
    cudaStreamSynchronize(g->up_stream);
    cudaStreamSynchronize(g->stream);
    return e;
  };
  auto collect = [&](int p, int k, double *tot) -> int {
    cudaEvent_t *E = g->pev[p];
    const int e = cuda_ok(cudaEventSynchronize(E[5]));
    if (e != AAK_OK) return e;
    std::memcpy(gram + 2 * (int64_t)nd * nd * k, g->h_stage + 2 * (size_t)g->stage_cap * p, 2 * (size_t)nd * nd * sizeof(double));
    float f;
    if (cudaEventElapsedTime(&f, E[2], E[1]) == cudaSuccess) tot[1] += f;
    if (cudaEventElapsedTime(&f, E[1], E[3]) == cudaSuccess) tot[2] += f;
    if (cudaEventElapsedTime(&f, E[3], E[4]) == cudaSuccess) tot[3] += f;
    cudaGetLastError();
    return AAK_OK;
  };
  double tot[4] = {0, 0, 0, 0}, ms = 0.0;
  if ((r = gpu_plan_into(g, ctxs[0], x, B, nthreads, status, &ms)) != AAK_OK) return r;
  tot[0] += ms;
  for (int c = 0; c < npts; ++c) {
    const int p = c & 1;
    if ((r = gpu_fisher_point_launch(g, ctxs[p], p, nd, scale, grid)) != AAK_OK) return fail(r);
    if (c + 1 < npts) {
      const int64_t k1 = (int64_t)(c + 1) * B;
      if ((r = cuda_ok(cudaEventSynchronize(g->pev[1 - p][0]))) != AAK_OK) return fail(r);
      if ((r = gpu_plan_into(g, ctxs[1 - p], x + 14 * k1, B, nthreads, status ? status + k1 : nullptr, &ms)) != AAK_OK)
        return fail(r);
      tot[0] += ms;
    }
    if (c > 0 && (r = collect(1 - p, c - 1, tot)) != AAK_OK) return fail(r);
  }
  if ((r = collect((npts - 1) & 1, npts - 1, tot)) != AAK_OK) return fail(r);
  for (int q = 0; q < 4; ++q) g->ms[q] = tot[q];
  const int s1 = device_status(g->ctx), s2 = device_status(g->ctx2);
  return s1 != AAK_OK ? s1 : s2;
}

}  // namespace

extern "C" {

int aak_gpu_create(double T_fit, int32_t init_length, int32_t length, double init_dt, double dt, int32_t LISA,
                   int32_t backint, aak_gpu **out) {
  if (!out) return AAK_ERR_INVALID_PARAM;
  *out = nullptr;
  if (length < 2 || !(dt > 0) || !(T_fit > 0)) return AAK_ERR_INVALID_PARAM;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return AAK_ERR_CUDA;
  }
  aak_gpu *g = new (std::nothrow) aak_gpu();
  if (!g) return AAK_ERR_NO_MEMORY;
  int r = aak_ctx_create(dev, &g->ctx);
  if (r != AAK_OK) {
    delete g;
    return r;
  }
  g->T_fit = T_fit;
  g->init_length = init_length;
  g->length = length;
  g->init_dt = init_dt;
  g->dt = dt;
  g->LISA = LISA;
  g->backint = backint;
  g->nbins = length / 2 + 1;
  g->row = 2 * g->nbins;
  // until input_data: zero data, unit weights
  for (int ch = 0; ch < 2; ++ch) {
    if ((r = g->d_D[ch].reserve(2 * g->nbins)) || (r = g->d_w[ch].reserve(g->nbins))) {
      aak_gpu_destroy(g);
      return r;
    }
    cudaMemset(g->d_D[ch].ptr, 0, 2 * g->nbins * sizeof(double));
    std::vector<double> ones(g->nbins, 1.0);
    cudaMemcpy(g->d_w[ch].ptr, ones.data(), g->nbins * sizeof(double), cudaMemcpyHostToDevice);
  }
  if ((r = cuda_ok(cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking))) != AAK_OK) {
    aak_gpu_destroy(g);
    return r;
  }
  *out = g;
  return cuda_ok(cudaGetLastError());
}

void aak_gpu_destroy(aak_gpu *g) {
  if (!g) return;
  if (g->stream) {
    cudaStreamSynchronize(g->stream);
    cudaStreamDestroy(g->stream);
  }
  if (g->plan) cufftDestroy(g->plan);
  if (g->plan32) cufftDestroy(g->plan32);
  for (int ch = 0; ch < 2; ++ch) {
    g->d_H32[ch].release();
    g->d_D32[ch].release();
    g->d_w32[ch].release();
    g->d_H[ch].release();
    g->d_D[ch].release();
    g->d_w[ch].release();
  }
  g->d_partial.release();
  g->d_out.release();
  g->d_t.release();
  for (auto &e : g->ev)
    if (e) cudaEventDestroy(e);
  if (g->up_stream) {
    cudaStreamSynchronize(g->up_stream);
    cudaStreamDestroy(g->up_stream);
  }
  for (auto &row : g->pev)
    for (auto &e : row)
      if (e) cudaEventDestroy(e);
  if (g->h_stage) cudaFreeHost(g->h_stage);
  aak_ctx_destroy(g->ctx2);
  aak_ctx_destroy(g->ctx);
  delete g;
}

int aak_gpu_input_data(aak_gpu *g, const double *hI_f, const double *hII_f, const double *ASDinv1,
                       const double *ASDinv2, int32_t len) {
  if (!g || !hI_f || !hII_f || !ASDinv1 || !ASDinv2) return AAK_ERR_INVALID_PARAM;
  if (len != g->nbins) return AAK_ERR_INVALID_PARAM;  // the reference asserts len == fft_length
  int r;
  if ((r = select_device(g->ctx->device)) != AAK_OK) return r;  // callers may drive several devices from one thread
  if ((r = cuda_ok(cudaMemcpy(g->d_D[0].ptr, hI_f, 2 * (size_t)len * sizeof(double), cudaMemcpyHostToDevice))) ||
      (r = cuda_ok(cudaMemcpy(g->d_D[1].ptr, hII_f, 2 * (size_t)len * sizeof(double), cudaMemcpyHostToDevice))) ||
      (r = cuda_ok(cudaMemcpy(g->d_w[0].ptr, ASDinv1, (size_t)len * sizeof(double), cudaMemcpyHostToDevice))) ||
      (r = cuda_ok(cudaMemcpy(g->d_w[1].ptr, ASDinv2, (size_t)len * sizeof(double), cudaMemcpyHostToDevice))))
    return r;
  // FP32 copies for precision 2 (rounded once, on the host)
  const double *hd[2] = {hI_f, hII_f}, *hw[2] = {ASDinv1, ASDinv2};
  std::vector<float> f(2 * (size_t)len);
  for (int ch = 0; ch < 2; ++ch) {
    if ((r = g->d_D32[ch].reserve(2 * (size_t)len)) || (r = g->d_w32[ch].reserve((size_t)len))) return r;
    for (size_t j = 0; j < 2 * (size_t)len; ++j) f[j] = (float)hd[ch][j];
    if ((r = cuda_ok(cudaMemcpy(g->d_D32[ch].ptr, f.data(), 2 * (size_t)len * sizeof(float), cudaMemcpyHostToDevice))))
      return r;
    for (size_t j = 0; j < (size_t)len; ++j) f[j] = (float)hw[ch][j];
    if ((r = cuda_ok(cudaMemcpy(g->d_w32[ch].ptr, f.data(), (size_t)len * sizeof(float), cudaMemcpyHostToDevice))))
      return r;
  }
  return AAK_OK;
}

int aak_gpu_gen(aak_gpu *g, const double *pars14) {
  if (!g || !pars14) return AAK_ERR_INVALID_PARAM;
  std::lock_guard<std::mutex> lk(g->ctx->mu);
  int32_t st = 0;
  int r = select_device(g->ctx->device);
  if (r != AAK_OK) return r;
  r = gpu_generate(g, pars14, 1, 1, &st, true);
  if (r != AAK_OK) return r;
  return st;
}

int aak_gpu_get_waveform(aak_gpu *g, double *t, double *hI, double *hII) {
  if (!g || !t || !hI || !hII || g->count < 1) return AAK_ERR_INVALID_PARAM;
  const size_t n = (size_t)g->length + 2;
  std::vector<double> buf(n, 0.0);
  int r;
  const size_t m = std::min(n, (size_t)g->row);
  if ((r = select_device(g->ctx->device)) != AAK_OK) return r;
  if ((r = cuda_ok(cudaStreamSynchronize(g->stream))) != AAK_OK) return r;  // the template's generation
  double *dst[3] = {t, hI, hII};
  const double *src[3] = {g->d_t.ptr, g->d_H[0].ptr, g->d_H[1].ptr};
  for (int k = 0; k < 3; ++k) {
    std::fill(dst[k], dst[k] + n, 0.0);
    if (!src[k]) continue;
    if ((r = cuda_ok(cudaMemcpy(dst[k], src[k], m * sizeof(double), cudaMemcpyDeviceToHost))) != AAK_OK) return r;
  }
  return AAK_OK;
}

int aak_gpu_likelihood(aak_gpu *g, double *out2) {
  if (!g || !out2) return AAK_ERR_INVALID_PARAM;
  std::lock_guard<std::mutex> lk(g->ctx->mu);
  if (g->count != 1) return AAK_ERR_INVALID_PARAM;
  const int r = select_device(g->ctx->device);
  if (r != AAK_OK) return r;
  return gpu_likelihood(g, out2);
}

int aak_gpu_likelihood_batch(aak_gpu *g, const double *params, int32_t nsrc, int32_t max_batch, int32_t nthreads,
                             double *out, int32_t *status) {
  if (!g || !params || !out || nsrc <= 0) return AAK_ERR_INVALID_PARAM;
  std::lock_guard<std::mutex> lk(g->ctx->mu);
  if (max_batch <= 0) max_batch = 256;
  double tot[4] = {0, 0, 0, 0};
  if (select_device(g->ctx->device) != AAK_OK) return AAK_ERR_CUDA;
  int r;
  if ((r = gpu_pipeline_ready(g, max_batch)) != AAK_OK) return r;
  // Chunk c is planned into ctxs[c & 1]: while the device generates,
  // transforms and reduces chunk c, the host plans chunk c + 1 into the other
  // context (whose upload, of chunk c - 1, has finished reading its plan
  // arrays) and then queues it, so that the device goes from one chunk to the
  // next without waiting for the host; chunk c - 1's results are collected
  // after that.  With a learned warm start, its prediction needs the device,
  // which is busy with the persistent waveform kernel of the chunk in flight:
  // the front end of chunk c + 2 (coarse inspirals, prediction, maps) is then
  // done after chunk c + 1 is planned, so that its prediction runs between
  // chunk c's kernels and the planning of a chunk never waits for the device.
  aak_ctx *ctxs[2] = {g->ctx, g->ctx2};
  const bool ahead = g->ctx->model != nullptr;
  WarmFrontEnd fe[3];
  const int32_t nch = (nsrc + max_batch - 1) / max_batch;
  auto chunk_size = [&](int32_t c) { return std::min<int32_t>(max_batch, nsrc - c * max_batch); };
  auto fail = [&](int e) {
    cudaStreamSynchronize(g->up_stream);
    cudaStreamSynchronize(g->stream);
    return e;
  };
  double ms = 0.0;
  // the warm front end of chunk c (ahead only), timed with the planning
  auto front = [&](int32_t c) {
    const auto t0 = std::chrono::steady_clock::now();
    std::vector<aak_params> P(chunk_size(c));
    for (int k = 0; k < chunk_size(c); ++k) P[k] = gpu_params(g, params + 14 * ((int64_t)c * max_batch + k));
    const int e = front_end_warm(g->ctx, P.data(), chunk_size(c), nthreads, &fe[c % 3]);
    tot[0] += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return e;
  };
  if (ahead && ((r = front(0)) != AAK_OK || (nch > 1 && (r = front(1)) != AAK_OK))) return r;
  if ((r = gpu_plan_into(g, ctxs[0], params, chunk_size(0), nthreads, status, &ms, ahead ? &fe[0] : nullptr)) !=
      AAK_OK)
    return r;
  tot[0] += ms;
  for (int32_t c = 0; c < nch; ++c) {
    const int p = c & 1;
    if ((r = gpu_chunk_launch(g, ctxs[p], p, chunk_size(c))) != AAK_OK) return fail(r);
    if (c + 1 < nch) {
      const int64_t k1 = (int64_t)(c + 1) * max_batch;
      if ((r = cuda_ok(cudaEventSynchronize(g->pev[1 - p][0]))) != AAK_OK) return fail(r);
      if ((r = gpu_plan_into(g, ctxs[1 - p], params + 14 * k1, chunk_size(c + 1), nthreads,
                             status ? status + k1 : nullptr, &ms, ahead ? &fe[(c + 1) % 3] : nullptr)) != AAK_OK)
        return fail(r);
      tot[0] += ms;
    }
    if (ahead && c + 2 < nch && (r = front(c + 2)) != AAK_OK) return fail(r);
    if (c > 0 && (r = gpu_chunk_collect(g, 1 - p, chunk_size(c - 1), out + 2 * (int64_t)(c - 1) * max_batch, tot)) !=
                     AAK_OK)
      return fail(r);
  }
  if ((r = gpu_chunk_collect(g, (nch - 1) & 1, chunk_size(nch - 1), out + 2 * (int64_t)(nch - 1) * max_batch, tot)) !=
      AAK_OK)
    return fail(r);
  for (int q = 0; q < 4; ++q) g->ms[q] = tot[q];
  return AAK_OK;
}

int aak_gpu_fisher(aak_gpu *g, const double *params, int32_t nd, double scale, int32_t nthreads, double *gram,
                   int32_t *status) {
  if (!g) return AAK_ERR_INVALID_PARAM;
  std::lock_guard<std::mutex> lk(g->ctx->mu);
  const int r = select_device(g->ctx->device);
  if (r != AAK_OK) return r;
  return gpu_fisher(g, params, nd, scale, nthreads, gram, status);
}

int aak_gpu_fisher_batch(aak_gpu *g, const double *params, int32_t npts, int32_t nd, double scale, int32_t nthreads,
                         double *gram, int32_t *status) {
  if (!g) return AAK_ERR_INVALID_PARAM;
  std::lock_guard<std::mutex> lk(g->ctx->mu);
  const int r = select_device(g->ctx->device);
  if (r != AAK_OK) return r;
  return gpu_fisher_batch(g, params, npts, nd, scale, nthreads, gram, status);
}

int aak_ctx_set_evolve_device(aak_ctx *ctx, int32_t on) {
  if (!ctx || (on && ctx->device < 0)) return AAK_ERR_INVALID_PARAM;
  std::lock_guard<std::mutex> lk(ctx->mu);
  ctx->evolve_device = on != 0;
  return AAK_OK;
}

int aak_batch_plan_ms(aak_ctx *ctx, double *ms4) {
  if (!ctx || !ms4) return AAK_ERR_INVALID_PARAM;
  std::lock_guard<std::mutex> lk(ctx->mu);
  for (int k = 0; k < 4; ++k) ms4[k] = ctx->plan_ms[k];
  return AAK_OK;
}

int aak_ctx_set_parmap_device(aak_ctx *ctx, int32_t on) {
  if (!ctx || (on && ctx->device < 0)) return AAK_ERR_INVALID_PARAM;
  std::lock_guard<std::mutex> lk(ctx->mu);
  ctx->parmap_device = on != 0;
  return AAK_OK;
}

int aak_gpu_set_parmap_device(aak_gpu *g, int32_t on) {
  if (!g) return AAK_ERR_INVALID_PARAM;
  return aak_ctx_set_parmap_device(g->ctx, on);
}

int aak_gpu_set_parmap_model(aak_gpu *g, aak_mlp *m) {
  if (!g) return AAK_ERR_INVALID_PARAM;
  return aak_ctx_set_parmap_model(g->ctx, m);
}

int aak_gpu_set_variant(aak_gpu *g, int32_t precision, int32_t variant) {
  if (!g) return AAK_ERR_INVALID_PARAM;
  return aak_ctx_set_variant(g->ctx, precision, variant);  // the second planning context copies it per batch
}

int aak_gpu_set_precision(aak_gpu *g, int32_t precision) {
  if (!g || precision < 0 || precision > 2) return AAK_ERR_INVALID_PARAM;
  g->precision = precision;
  return AAK_OK;
}

int aak_gpu_last_timing(aak_gpu *g, double *ms4) {
  if (!g || !ms4) return AAK_ERR_INVALID_PARAM;
  for (int q = 0; q < 4; ++q) ms4[q] = g->ms[q];
  return AAK_OK;
}

}  // extern "C"
}  // extern "C" (GPU likelihood)
