// C ABI of the B200 chemistry engine (include/pelephysics_b200.h).
//
// A ppb_reactor plays the role of the reference's ReactorCvode / ReactorRK64
// object (Source/Reactions/ReactorCvode.{H,cpp}, ReactorRK64.{H,cpp}): it is
// created by name, initialised once, and then advances batches of cells.
// The reference's driver calls one reactor's react() from several OpenMP
// threads at once (Testing/Exec/ReactEval/main.cpp:478-520), and
// ReactorCvode survives that because it creates its CVODE memory per call
// (ReactorCvode.cpp:1307).  Here every host thread that calls a reactor gets
// its own call context -- device scratch grown on demand, the cost order of
// its previous call, its captured CUDA graph, its per-cell flags -- so calls
// from different threads never share mutable state.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <atomic>
#include <map>
#include <memory>
#include <numeric>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/pelephysics_b200.h"
#include "ppb_bdf.cuh"
#include "ppb_engine.h"

using namespace ppb;

// last error message of the calling thread (fixed storage, so that setting
// it never allocates)
static thread_local char g_err[512];

static int fail(int code, const std::string& msg)
{
  snprintf(g_err, sizeof(g_err), "%s", msg.c_str());
  return code;
}

namespace ppb {
void set_error(const char* msg) { snprintf(g_err, sizeof(g_err), "%s", msg); }
} // namespace ppb

static int cuda_fail(int e, const char* where)
{
  if (e == 0) return 0;
  return fail(PPB_E_CUDA, std::string(where) + ": " + cudaGetErrorString((cudaError_t)e));
}

#define PPB_CUDA(call, where)                                                                                      \
  do {                                                                                                             \
    int _e = (int)(call);                                                                                          \
    if (_e) return cuda_fail(_e, where);                                                                           \
  } while (0)

// One device copy of each mechanism per device, shared by all reactors.
static std::mutex g_mech_mu;
static std::vector<DeviceMechanism*> g_mechs;

static int device_mechanism(const PPBMechTables* t, DeviceMechanism** out)
{
  int dev = 0;
  PPB_CUDA(cudaGetDevice(&dev), "cudaGetDevice");
  std::lock_guard<std::mutex> lk(g_mech_mu);
  for (auto* m : g_mechs) {
    if (m->host == t && m->device == dev) {
      *out = m;
      return 0;
    }
  }
  auto* m = new DeviceMechanism();
  int e = upload_mechanism(t, m);
  if (e) {
    delete m;
    return cuda_fail(e, "upload_mechanism");
  }
  g_mechs.push_back(m);
  *out = m;
  return 0;
}

struct GraphKey {
  const void* p[6];
  int ncells, ld;
  double dt;
  cudaStream_t st;
  unsigned gen, tune_gen; // reactor and autotuner generations at capture
  bool operator==(const GraphKey& o) const
  {
    return memcmp(p, o.p, sizeof(p)) == 0 && ncells == o.ncells && ld == o.ld && dt == o.dt && st == o.st &&
           gen == o.gen && tune_gen == o.tune_gen;
  }
};

// Per-thread call context of a reactor: everything a react() call writes.
struct CallCtx {
  size_t cap = 0;
  double *aos = nullptr, *aos_src = nullptr, *soa = nullptr, *soa_src = nullptr, *rhoe = nullptr, *rhoesrc = nullptr;
  int *status = nullptr, *nfe = nullptr, *queue = nullptr, *mask = nullptr, *stats = nullptr;
  int last_ncells = 0;
  // work-queue order by the previous call's per-cell cost
  int *order = nullptr, *order_keys = nullptr, *iota = nullptr;
  void* sort_tmp = nullptr;
  size_t sort_tmp_bytes = 0;
  // ReactorArkode: cell-major state, stage-0 and FSAL derivatives, sources,
  // block partial sums, grid barrier, batch result
  size_t ark_cap = 0;
  double *ark_y0 = nullptr, *ark_y1 = nullptr, *ark_f0 = nullptr, *ark_f1 = nullptr, *ark_s = nullptr;
  double* ark_partial = nullptr;
  unsigned* ark_bar = nullptr;
  ArkInfo* ark_info = nullptr;
  ArkInfo ark_last{};
  // graph cache for the device paths; capture runs on a private stream (the
  // legacy default stream cannot be captured) and the graph is launched on
  // the caller's stream
  cudaGraphExec_t gexec = nullptr;
  GraphKey gkey{};
  cudaStream_t cap_stream = nullptr;
};

struct ppb_reactor {
  std::string mech;
  int method = METHOD_BDF;
  const PPBMechTables* t = nullptr;
  DeviceMechanism* dm = nullptr;
  int reactor_type = 0;
  bool inited = false;
  ppb_options opt{};
  std::vector<double> typ_vals;
  double* atolv = nullptr;
  // SRK / QSS kernels: a 16-warp block is compiled and fits one SM
  bool dq16 = false;
  // bumped whenever something a captured graph holds changes (typical
  // values, Arrhenius tables, options): graphs of older generations are
  // captured again
  std::atomic<unsigned> gen{0};
  // call contexts by host thread
  std::mutex ctx_mu;
  std::map<std::thread::id, std::unique_ptr<CallCtx>> ctxs;
  // the adjoint and tangent calls share the adjoint scratch: one at a time
  std::mutex adj_mu;
  // reactor-private mechanism tables (ppb_set_arrhenius)
  PPBMechTables own_t{};
  std::vector<double> own_A, own_beta, own_EaR;
  DeviceMechanism* own = nullptr;
  // adjoint scratch (grown on demand)
  void *adj_cp = nullptr, *adj_tape = nullptr, *adj_ys = nullptr, *adj_gw = nullptr;
  size_t adj_cp_bytes = 0, adj_tape_bytes = 0, adj_ys_bytes = 0, adj_gw_bytes = 0;
  // batched reverse sweep
  void *adj_yinfo = nullptr, *adj_cpidx = nullptr, *adj_ints = nullptr, *adj_dbl = nullptr, *adj_lam = nullptr,
       *adj_items = nullptr, *adj_ioff = nullptr, *adj_tpool = nullptr;
  size_t adj_yinfo_bytes = 0, adj_cpidx_bytes = 0, adj_ints_bytes = 0, adj_dbl_bytes = 0, adj_lam_bytes = 0,
         adj_items_bytes = 0, adj_ioff_bytes = 0, adj_tpool_bytes = 0;
};

// The calling thread's context of reactor r (created on first use).
static CallCtx* ctx_of(ppb_reactor* r)
{
  std::lock_guard<std::mutex> lk(r->ctx_mu);
  std::unique_ptr<CallCtx>& c = r->ctxs[std::this_thread::get_id()];
  if (!c) c.reset(new CallCtx());
  return c.get();
}

// Generation of the autotuner's picks: a pick that changes makes every
// reactor capture its graphs again.
static std::atomic<unsigned> g_tune_gen{0};

static void free_adjoint_scratch(ppb_reactor* r)
{
  cudaFree(r->adj_cp);
  cudaFree(r->adj_tape);
  cudaFree(r->adj_ys);
  cudaFree(r->adj_gw);
  r->adj_cp = r->adj_tape = r->adj_ys = r->adj_gw = nullptr;
  r->adj_cp_bytes = r->adj_tape_bytes = r->adj_ys_bytes = r->adj_gw_bytes = 0;
  for (void** q : {&r->adj_yinfo, &r->adj_cpidx, &r->adj_ints, &r->adj_dbl, &r->adj_lam, &r->adj_items, &r->adj_ioff,
                   &r->adj_tpool}) {
    cudaFree(*q);
    *q = nullptr;
  }
  r->adj_yinfo_bytes = r->adj_cpidx_bytes = r->adj_ints_bytes = r->adj_dbl_bytes = r->adj_lam_bytes = 0;
  r->adj_items_bytes = r->adj_ioff_bytes = r->adj_tpool_bytes = 0;
}

static int grow(void*& p, size_t& cap, size_t bytes)
{
  if (p && bytes <= cap) return 0;
  cudaFree(p);
  p = nullptr;
  cap = 0;
  if (bytes == 0) return 0;
  PPB_CUDA(cudaMalloc(&p, bytes), "cudaMalloc (adjoint scratch)");
  cap = bytes;
  return 0;
}

static void free_scratch(CallCtx* c)
{
  cudaFree(c->aos);
  cudaFree(c->aos_src);
  cudaFree(c->soa);
  cudaFree(c->soa_src);
  cudaFree(c->rhoe);
  cudaFree(c->rhoesrc);
  cudaFree(c->status);
  cudaFree(c->nfe);
  cudaFree(c->queue);
  cudaFree(c->mask);
  cudaFree(c->stats);
  c->stats = nullptr;
  cudaFree(c->order);
  cudaFree(c->order_keys);
  cudaFree(c->iota);
  cudaFree(c->sort_tmp);
  c->order = c->order_keys = c->iota = nullptr;
  c->sort_tmp = nullptr;
  c->sort_tmp_bytes = 0;
  c->aos = c->aos_src = c->soa = c->soa_src = c->rhoe = c->rhoesrc = nullptr;
  c->status = c->nfe = c->queue = c->mask = nullptr;
  c->cap = 0;
  if (c->gexec) cudaGraphExecDestroy(c->gexec);
  c->gexec = nullptr;
  for (double** q : {&c->ark_y0, &c->ark_y1, &c->ark_f0, &c->ark_f1, &c->ark_s, &c->ark_partial}) {
    cudaFree(*q);
    *q = nullptr;
  }
  cudaFree(c->ark_bar);
  cudaFree(c->ark_info);
  c->ark_bar = nullptr;
  c->ark_info = nullptr;
  c->ark_cap = 0;
}

// capacity of the ARKODE partial-sum buffer, in blocks (>= SMs x resident blocks)
static const int ARK_MAX_GRID = 4096;

static int ensure_scratch(ppb_reactor* r, CallCtx* c, int ncells, cudaStream_t st = nullptr)
{
  if ((size_t)ncells <= c->cap && c->queue) return 0;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (st && cudaStreamIsCapturing(st, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone)
    return fail(PPB_E_STATE, "react inside a stream capture needs device scratch for at least this many cells: "
                             "call ppb_init with ncells >= the batch (or react once) on this thread before capturing");
  free_scratch(c);
  const size_t n = r->t->nsp + 1, nc = (size_t)ncells;
  PPB_CUDA(cudaMalloc(&c->aos, n * nc * 8), "cudaMalloc");
  PPB_CUDA(cudaMalloc(&c->aos_src, n * nc * 8), "cudaMalloc");
  PPB_CUDA(cudaMalloc(&c->soa, n * nc * 8), "cudaMalloc");
  PPB_CUDA(cudaMalloc(&c->soa_src, n * nc * 8), "cudaMalloc");
  PPB_CUDA(cudaMalloc(&c->rhoe, nc * 8), "cudaMalloc");
  PPB_CUDA(cudaMalloc(&c->rhoesrc, nc * 8), "cudaMalloc");
  PPB_CUDA(cudaMalloc(&c->status, nc * 4), "cudaMalloc");
  PPB_CUDA(cudaMalloc(&c->nfe, nc * 4), "cudaMalloc");
  PPB_CUDA(cudaMalloc(&c->mask, nc * 4), "cudaMalloc");
  PPB_CUDA(cudaMalloc(&c->stats, nc * 7 * 4), "cudaMalloc");
  PPB_CUDA(cudaMalloc(&c->queue, 16), "cudaMalloc");
  // no costs yet: zeros keep the first call in index order (stable sort)
  PPB_CUDA(cudaMemset(c->nfe, 0, nc * 4), "cudaMemset");
  PPB_CUDA(cudaMalloc(&c->order, nc * 4), "cudaMalloc");
  PPB_CUDA(cudaMalloc(&c->order_keys, nc * 4), "cudaMalloc");
  PPB_CUDA(cudaMalloc(&c->iota, nc * 4), "cudaMalloc");
  PPB_CUDA(launch_iota(c->iota, (int)nc, nullptr), "iota");
  c->sort_tmp_bytes = cost_order_tmp_bytes((int)nc);
  PPB_CUDA(cudaMalloc(&c->sort_tmp, c->sort_tmp_bytes > 0 ? c->sort_tmp_bytes : 16), "cudaMalloc");
  PPB_CUDA(cudaDeviceSynchronize(), "cudaDeviceSynchronize");
  c->cap = nc;
  if (r->method == METHOD_ARK) {
    const size_t N = r->t->nsp;
    PPB_CUDA(cudaMalloc(&c->ark_y0, n * nc * 8), "cudaMalloc");
    PPB_CUDA(cudaMalloc(&c->ark_y1, n * nc * 8), "cudaMalloc");
    PPB_CUDA(cudaMalloc(&c->ark_f0, n * nc * 8), "cudaMalloc");
    PPB_CUDA(cudaMalloc(&c->ark_f1, n * nc * 8), "cudaMalloc");
    PPB_CUDA(cudaMalloc(&c->ark_s, N * nc * 8), "cudaMalloc");
    PPB_CUDA(cudaMalloc(&c->ark_partial, 2 * ARK_MAX_GRID * 8), "cudaMalloc");
    PPB_CUDA(cudaMalloc(&c->ark_bar, 16), "cudaMalloc");
    PPB_CUDA(cudaMalloc(&c->ark_info, sizeof(ArkInfo)), "cudaMalloc");
    c->ark_cap = nc;
  }
  return 0;
}

// The ERK table of a reference ode.rk_method number; unknown numbers select
// the default, as the reference's switch does (ReactorArkode.cpp:80-83).
static const ErkTable& erk_table(int id)
{
  for (int i = 0; i < ppb_erk_ntables; i++)
    if (ppb_erk_tables[i].id == id) return ppb_erk_tables[i];
  return erk_table(40);
}

static bool erk_fsal(const ErkTable& t)
{
  const int s = t.stages;
  if (t.c[s - 1] != 1.0 || t.b[s - 1] != 0.0) return false;
  for (int j = 0; j < s - 1; j++)
    if (t.A[s - 1][j] != t.b[j]) return false;
  return true;
}

// ReactorArkode over a species-major device batch: one cooperative launch.
// box: the box path (rk_method / rk_controller apply); rhoe_out: where the
// energies advanced by the time reached go (nullable).
static int run_ark(ppb_reactor* r, CallCtx* c, const Batch& b, double dt, cudaStream_t st, double* rhoe_out,
                   bool box)
{
  ArkParams P{};
  P.tab = erk_table(box ? r->opt.rk_method : 40);
  P.rtol = r->opt.rtol;
  P.atol = r->opt.atol;
  P.tout = dt;
  P.reactor_type = r->reactor_type;
  const int ctl = box ? r->opt.rk_controller : 0;
  P.controller = (ctl >= 0 && ctl <= 3) ? ctl : 0; // unknown: PID (ReactorArkode.cpp:110-114)
  P.max_steps = r->opt.arkode_max_steps;
  P.fsal = erk_fsal(P.tab) ? 1 : 0;
  P.barrier_ns = 1000ull * (unsigned long long)r->opt.arkode_barrier_us;
  ArkBuffers B{};
  B.ncells = b.ncells;
  B.ld = b.ld;
  B.ysoa = b.y;
  B.srcsoa = b.src;
  B.rhoe = b.rhoe;
  B.rhoesrc = b.rhoesrc;
  B.mask = b.mask;
  B.atolv = r->atolv;
  B.rhoe_out = rhoe_out;
  B.Y0 = c->ark_y0;
  B.Y1 = c->ark_y1;
  B.F0 = c->ark_f0;
  B.F1 = c->ark_f1;
  B.S = c->ark_s;
  B.partial = c->ark_partial;
  B.bar = c->ark_bar;
  B.info = c->ark_info;
  B.status = c->status;
  B.nfe = c->nfe;
  B.stats = c->stats;
  PPB_CUDA(cudaMemsetAsync(c->ark_info, 0, sizeof(ArkInfo), st), "cudaMemsetAsync");
  // a call that timed out can leave arrivals counted: every launch starts
  // from a clear barrier
  PPB_CUDA(cudaMemsetAsync(c->ark_bar, 0, 16, st), "cudaMemsetAsync");
  int grid = ARK_MAX_GRID;
  return cuda_fail(launch_ark(*r->dm, P, B, &grid, st), "launch_ark");
}

// Result of the last ReactorArkode launch (synchronises the stream).
static int ark_result(CallCtx* c, cudaStream_t st)
{
  PPB_CUDA(cudaMemcpyAsync(&c->ark_last, c->ark_info, sizeof(ArkInfo), cudaMemcpyDeviceToHost, st), "D2H info");
  PPB_CUDA(cudaStreamSynchronize(st), "cudaStreamSynchronize");
  if (c->ark_last.barrier_timeout) return fail(PPB_E_CUDA, "ReactorArkode: grid barrier timed out");
  return 0;
}

static Options engine_options(const ppb_reactor* r)
{
  Options o{};
  o.rtol = r->opt.rtol;
  o.atol = r->opt.atol;
  o.max_order = r->opt.max_order;
  o.max_steps = r->opt.max_steps;
  o.max_nls_iters = r->opt.max_nls_iters;
  o.max_err_fails = r->opt.max_err_fails;
  o.jac_eval_freq = r->opt.jac_eval_freq;
  o.reactor_type = r->reactor_type;
  o.lu_fp32 = r->opt.lu_fp32;
  o.refine_sweeps = r->opt.refine_sweeps;
  o.rk_guess = r->opt.rk64_nsubsteps_guess;
  o.rk_min = r->opt.rk64_nsubsteps_min;
  o.rk_max = r->opt.rk64_nsubsteps_max;
  o.use_typ_vals = r->typ_vals.empty() ? 0 : 1;
  o.rendezvous = r->opt.rendezvous_cycles;
  return o;
}

// ---- autotuner: per (mechanism tables, device, integrator, reactor type,
// LU precision, typical values) the fastest tuned-engine configuration on a
// sample of the first batch
struct TuneEntry {
  const PPBMechTables* t;
  int dev, method, rtype, lu_fp32, typ;
  LaunchConfig lc;
  double ms;
  int sample, target; // cells timed, and the sample size wanted (32 resident waves)
};
static std::mutex g_tune_mu;
static std::vector<TuneEntry> g_tune;

static TuneEntry* find_tune(const ppb_reactor* r)
{
  int dev = 0;
  cudaGetDevice(&dev);
  for (auto& e : g_tune) {
    if (e.t == r->dm->host && e.dev == dev && e.method == r->method && e.rtype == r->reactor_type &&
        e.lu_fp32 == r->opt.lu_fp32 && e.typ == (int)!r->typ_vals.empty())
      return &e;
  }
  return nullptr;
}

static bool tuned_config(const ppb_reactor* r, LaunchConfig* lc, double* ms, int* sample = nullptr,
                         int* target = nullptr)
{
  std::lock_guard<std::mutex> lk(g_tune_mu);
  const TuneEntry* e = find_tune(r);
  if (!e) return false;
  *lc = e->lc;
  if (ms) *ms = e->ms;
  if (sample) *sample = e->sample;
  if (target) *target = e->target;
  return true;
}

static LaunchConfig launch_config(const ppb_reactor* r)
{
  LaunchConfig lc;
  lc.engine = r->opt.engine;
  lc.lu_fp32 = r->opt.lu_fp32;
  lc.persistent = 1;
  if (r->opt.eos == PPB_EOS_SRK || r->t->nqss > 0) {
    // the SRK or QSS kernel: warp teams, <= 128 registers; the block size
    // the caller gives, else 16 warps (one block per SM, one rendezvous)
    // where that kernel is compiled and fits, else the largest <= 8 that fits
    lc.rhsv = r->opt.eos == PPB_EOS_SRK ? 1 : 2;
    lc.team = 32;
    lc.minb = 2;
    if (r->opt.warps_per_block > 0) {
      lc.warps_per_block = r->opt.warps_per_block;
    } else if (r->dq16) {
      lc.warps_per_block = 16;
    } else {
      const size_t cb = team_cell_bytes(r->t, 0);
      int w = 8;
      while (w > 1 && cb * w > 200 * 1024) w--;
      lc.warps_per_block = w;
    }
    return lc;
  }
  if (r->opt.warps_per_block > 0) {
    lc.warps_per_block = r->opt.warps_per_block;
    lc.team = (r->opt.team_lanes == 16 || r->opt.team_lanes == 64 || r->opt.team_lanes == 128) ? r->opt.team_lanes : 32;
    lc.minb = r->opt.register_budget == 1 ? 1 : 2;
    if (lc.team > 32) { // one cell per block of team / 32 warps, <= 255 registers
      lc.warps_per_block = lc.team / 32;
      lc.minb = 1;
    }
    return lc;
  }
  if (lc.engine == ENGINE_TUNED && tuned_config(r, &lc, nullptr)) {
    lc.engine = ENGINE_TUNED;
    lc.lu_fp32 = r->opt.lu_fp32;
    return lc;
  }
  // untuned default: the largest block (<= 8 warps) that fits, one warp per
  // cell, <= 128 registers
  const size_t cb = team_cell_bytes(r->t, r->opt.lu_fp32);
  int w = 8;
  while (w > 1 && cb * w > 200 * 1024) w--;
  lc.warps_per_block = w;
  return lc;
}

// Time the candidate configurations on copies of the batch's first cells
// (up to 4, then 32 resident waves) and cache the fastest; a batch that gives
// at least twice the cells of an earlier, smaller-than-wanted sample tunes
// again.  Not during a stream capture (the caller checks).
static int autotune(ppb_reactor* r, const Batch& b, double dt, cudaStream_t st)
{
  if (r->opt.engine != PPB_ENGINE_TUNED || r->opt.warps_per_block > 0) return 0;
  LaunchConfig have;
  int had = 0, want = 0;
  if (tuned_config(r, &have, nullptr, &had, &want) && (had >= want || b.ncells < 2 * had)) return 0;
  const int N = r->t->nsp, n = N + 1;
  std::vector<LaunchConfig> cand;
  int max_res = 0;
  const int big = N <= 21 ? 0 : N <= 64 ? 64 : 128;
  for (int team : {32, 16, big}) {
    if (team == 0 || (team == 16 && N > 21)) continue;
    for (int minb : {2, 1}) {
      if (minb == 1 && (r->method != METHOD_BDF || r->opt.lu_fp32) && team <= 32) continue;
      if (team > 32 && minb != 1) continue;
      for (int wpb : {16, 12, 8, 4, 2, 1}) {
        if (team > 32 && wpb != team / 32) continue;
        if (wpb > 8 && (team != 32 || minb != 2)) continue;
        LaunchConfig lc;
        lc.engine = ENGINE_TUNED;
        lc.lu_fp32 = r->opt.lu_fp32;
        lc.warps_per_block = wpb;
        lc.team = team;
        lc.minb = minb;
        const int res = react_occupancy(*r->dm, r->method, lc);
        if (res <= 0) continue;
        max_res = std::max(max_res, res);
        if (wpb > 8 && r->opt.rendezvous_cycles < 0) {
          // one block per SM: the rendezvous bound is tuned too (drm19, 16
          // warps: the 64^3 field runs faster at 3e5 SM clocks, long
          // integrations of h/cp reactors at 1e6)
          for (int rv : {300000, 1000000}) {
            lc.rv = rv;
            cand.push_back(lc);
          }
        } else {
          cand.push_back(lc);
        }
      }
    }
  }
  if (cand.empty()) return 0;
  int dev = 0, nsm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  // Two samples of the batch's first cells: a short one (4 resident waves of
  // the largest candidate) times every candidate, then a long one (32 waves,
  // or the whole batch) times those within 1.5x of the fastest.  On a short
  // sample the few longest cells decide the time, and with them the
  // configurations that finish one cell soonest; the long one weighs
  // throughput as a full call does (drm19, 65,536 h/cp reactors over 5e-4 s:
  // the short sample picked 8 warps per block, 188 ms a call, against 131 ms
  // for 16).
  const int m1 = (int)std::min<long>(b.ncells, 4L * max_res * nsm);
  const int m2 = (int)std::min<long>(b.ncells, 32L * max_res * nsm);
  const size_t nm = (size_t)m2;
  double *y0 = nullptr, *y = nullptr, *sr = nullptr, *re = nullptr, *rs = nullptr;
  int *stt = nullptr, *nfe = nullptr, *q = nullptr, *ord = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int err = 0;
  auto cleanup = [&]() {
    cudaFree(y0);
    cudaFree(y);
    cudaFree(sr);
    cudaFree(re);
    cudaFree(rs);
    cudaFree(stt);
    cudaFree(nfe);
    cudaFree(q);
    cudaFree(ord);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
  };
  if ((err = cudaMalloc(&y0, n * nm * 8)) || (err = cudaMalloc(&y, n * nm * 8)) || (err = cudaMalloc(&sr, n * nm * 8)) ||
      (err = cudaMalloc(&re, nm * 8)) || (err = cudaMalloc(&rs, nm * 8)) || (err = cudaMalloc(&stt, nm * 4)) ||
      (err = cudaMalloc(&nfe, nm * 4)) || (err = cudaMalloc(&q, 16)) || (err = cudaMalloc(&ord, nm * 4)) ||
      (err = cudaEventCreate(&e0)) ||
      (err = cudaEventCreate(&e1))) {
    cleanup();
    return cuda_fail(err, "autotune scratch");
  }
  err = cudaMemcpy2DAsync(y0, nm * 8, b.y, (size_t)b.ld * 8, nm * 8, n, cudaMemcpyDeviceToDevice, st);
  if (!err) err = cudaMemcpy2DAsync(sr, nm * 8, b.src, (size_t)b.ld * 8, nm * 8, N, cudaMemcpyDeviceToDevice, st);
  if (!err) err = cudaMemcpyAsync(re, b.rhoe, nm * 8, cudaMemcpyDeviceToDevice, st);
  if (!err) err = cudaMemcpyAsync(rs, b.rhoesrc, nm * 8, cudaMemcpyDeviceToDevice, st);
  const Options o = engine_options(r);
  bool use_ord = false;
  // one launch of candidate lc on the first m cells of the sample (device time)
  auto timed = [&](const LaunchConfig& lc, int m, float* ms) -> int {
    Batch tb{};
    tb.y = y;
    tb.src = sr;
    tb.rhoe = re;
    tb.rhoesrc = rs;
    tb.atolv = r->atolv;
    tb.status = stt;
    tb.nfe = nfe;
    tb.ncells = m;
    tb.ld = m2;
    tb.order = use_ord ? ord : nullptr;
    int e = cudaMemcpyAsync(y, y0, n * nm * 8, cudaMemcpyDeviceToDevice, st);
    if (!e) e = cudaEventRecord(e0, st);
    if (!e) e = launch_react(*r->dm, o, r->method, lc, tb, dt, q, st);
    if (!e) e = cudaEventRecord(e1, st);
    if (!e) e = cudaEventSynchronize(e1);
    if (!e) e = cudaEventElapsedTime(ms, e0, e1);
    return e;
  };
  // One warm-up launch, then two interleaved passes over the candidates
  // `which`; each keeps its faster time, so a clock ramp or a neighbour's
  // burst during one pass does not decide the pick.  With cost_order the
  // timed launches take the cells in the order the calls after the first one
  // use: by descending cost (right-hand sides) in the warm-up launch, ties in
  // index order.
  auto stage = [&](int m, const std::vector<size_t>& which, std::vector<double>& t) -> int {
    float ms = 0.f;
    use_ord = false;
    int e = timed(cand[which[0]], m, &ms);
    if (!e && r->opt.cost_order && m > 1) {
      std::vector<int> cost((size_t)m), idx((size_t)m);
      e = cudaMemcpyAsync(cost.data(), nfe, (size_t)m * 4, cudaMemcpyDeviceToHost, st);
      if (!e) e = cudaStreamSynchronize(st);
      if (e) return e;
      std::iota(idx.begin(), idx.end(), 0);
      std::stable_sort(idx.begin(), idx.end(), [&](int a, int c) { return cost[a] > cost[c]; });
      e = cudaMemcpyAsync(ord, idx.data(), (size_t)m * 4, cudaMemcpyHostToDevice, st);
      if (!e) e = cudaStreamSynchronize(st);
      use_ord = true;
    }
    for (size_t k = 0; k < 2 * which.size() && !e; k++) {
      const size_t ci = which[k % which.size()];
      e = timed(cand[ci], m, &ms);
      if (!e) t[ci] = std::min(t[ci], (double)ms);
    }
    return e;
  };
  const size_t nc = cand.size();
  std::vector<size_t> all(nc);
  std::iota(all.begin(), all.end(), 0);
  std::vector<double> t1(nc, 1e300), t2(nc, 1e300);
  err = stage(m1, all, t1);
  size_t bi = 0;
  for (size_t ci = 0; ci < nc; ci++)
    if (t1[ci] < t1[bi]) bi = ci;
  double best = t1[bi];
  int sample = m1;
  if (!err && m2 > m1) {
    std::vector<size_t> keep;
    for (size_t ci : all)
      if (t1[ci] <= 1.5 * t1[bi]) keep.push_back(ci);
    std::stable_sort(keep.begin(), keep.end(), [&](size_t a, size_t c) { return t1[a] < t1[c]; });
    err = stage(m2, keep, t2);
    if (!err) {
      bi = keep[0];
      for (size_t ci : keep)
        if (t2[ci] < t2[bi]) bi = ci;
      best = t2[bi];
      sample = m2;
    }
  }
  const LaunchConfig pick = cand[bi];
  cleanup();
  if (err) return cuda_fail(err, "autotune");
  const int target = (int)std::min<long>(1L << 30, 32L * max_res * nsm);
  TuneEntry te{r->dm->host, dev, r->method, r->reactor_type, r->opt.lu_fp32, (int)!r->typ_vals.empty(), pick, best,
               sample, target};
  std::lock_guard<std::mutex> lk(g_tune_mu);
  if (TuneEntry* e = find_tune(r)) {
    *e = te;
  } else {
    g_tune.push_back(te);
  }
  g_tune_gen++; // graphs captured with the earlier choice are captured again
  return 0;
}

// Run the autotuner on this batch unless the stream is being captured.
static int maybe_autotune(ppb_reactor* r, const Batch& b, double dt, cudaStream_t st)
{
  if (r->method == METHOD_ARK || r->opt.eos == PPB_EOS_SRK || r->t->nqss > 0 || r->opt.engine != PPB_ENGINE_TUNED ||
      r->opt.warps_per_block > 0)
    return 0;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(st, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) return 0;
  // one tuner at a time: a thread that waited finds the pick made
  static std::mutex tuner_mu;
  std::lock_guard<std::mutex> lk(tuner_mu);
  return autotune(r, b, dt, st);
}

// Capture body() on the reactor's private stream into r->gexec.
template <typename F>
static int capture(CallCtx* r, const GraphKey& key, F body)
{
  if (r->gexec && r->gkey == key) return 0;
  if (r->gexec) cudaGraphExecDestroy(r->gexec);
  r->gexec = nullptr;
  if (!r->cap_stream) PPB_CUDA(cudaStreamCreateWithFlags(&r->cap_stream, cudaStreamNonBlocking), "cudaStreamCreate");
  cudaGraph_t g;
  PPB_CUDA(cudaStreamBeginCapture(r->cap_stream, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
  int be = body(r->cap_stream);
  cudaError_t ce = cudaStreamEndCapture(r->cap_stream, &g);
  if (be) return be;
  PPB_CUDA(ce, "cudaStreamEndCapture");
  cudaError_t ie = cudaGraphInstantiate(&r->gexec, g, 0);
  cudaGraphDestroy(g);
  PPB_CUDA(ie, "cudaGraphInstantiate");
  r->gkey = key;
  return 0;
}

extern "C" {

void ppb_default_options(ppb_options* o)
{
  if (!o) return;
  memset(o, 0, sizeof(*o));
  o->rtol = 1e-6;
  o->atol = 1e-10;
  o->max_order = 2;
  o->max_steps = 10000;
  o->max_nls_iters = 3;
  o->max_err_fails = 100;
  o->jac_eval_freq = 100;
  o->clean_init_massfrac = 0;
  o->rk64_nsubsteps_guess = 10;
  o->rk64_nsubsteps_min = 5;
  o->rk64_nsubsteps_max = 500;
  o->verbose = 0;
  o->engine = PPB_ENGINE_TUNED;
  o->lu_fp32 = 0;
  o->refine_sweeps = 1;
  o->warps_per_block = 0;
  o->use_graph = 1;
  o->adjoint_checkpoint_interval = 16;
  o->adjoint_memory_mb = 16384;
  o->team_lanes = 32;
  o->register_budget = 2;
  o->rk_method = 40;
  o->rk_controller = 0;
  o->use_erkstep = 1;
  o->arkode_max_steps = 500;
  o->eos = PPB_EOS_IDEAL;
  o->cost_order = 1;
  o->rendezvous_cycles = -1;
  o->arkode_barrier_us = 20000000;
  o->adjoint_keep_segments = 1;
}

const char* ppb_last_error(void) { return g_err; }

int ppb_mechanism_info(const char* mechanism, int* nspecies, int* nreactions)
{
  const PPBMechTables* t = mechanism ? find_mechanism(mechanism) : nullptr;
  if (!t) return fail(PPB_E_MECH, std::string("unknown mechanism ") + (mechanism ? mechanism : "(null)"));
  if (nspecies) *nspecies = t->nsp;
  if (nreactions) *nreactions = t->nrxn;
  return 0;
}

const char* ppb_species_name(const char* mechanism, int k)
{
  const PPBMechTables* t = mechanism ? find_mechanism(mechanism) : nullptr;
  if (!t || k < 0 || k >= t->nsp) return nullptr;
  return t->species[k];
}

int ppb_molecular_weights(const char* mechanism, double* mw)
{
  const PPBMechTables* t = mechanism ? find_mechanism(mechanism) : nullptr;
  if (!t) return fail(PPB_E_MECH, std::string("unknown mechanism ") + (mechanism ? mechanism : "(null)"));
  if (!mw) return fail(PPB_E_ARG, "ppb_molecular_weights: null output");
  for (int k = 0; k < t->nsp; k++) mw[k] = t->mw[k];
  return 0;
}

int ppb_create(const char* mechanism, const char* integrator, ppb_reactor** out)
{
  if (!out) return fail(PPB_E_ARG, "ppb_create: null output");
  *out = nullptr;
  const PPBMechTables* t = mechanism ? find_mechanism(mechanism) : nullptr;
  if (!t) return fail(PPB_E_MECH, std::string("unknown mechanism ") + (mechanism ? mechanism : "(null)"));
  int method;
  if (!integrator || !strcmp(integrator, "ReactorCvode") || !strcmp(integrator, "ReactorB200")) {
    method = METHOD_BDF;
  } else if (!strcmp(integrator, "ReactorRK64") || !strcmp(integrator, "ReactorB200RK")) {
    method = METHOD_RK64;
  } else if (!strcmp(integrator, "ReactorArkode")) {
    method = METHOD_ARK;
  } else {
    return fail(PPB_E_ARG, std::string("unknown integrator ") + integrator);
  }
  auto* r = new ppb_reactor();
  r->mech = mechanism;
  r->method = method;
  r->t = t;
  ppb_default_options(&r->opt);
  *out = r;
  return 0;
}

int ppb_init(ppb_reactor* r, int reactor_type, int ncells, const ppb_options* opt)
{
  if (!r) return fail(PPB_E_ARG, "ppb_init: null reactor");
  // ReactorTypes::check_reactor_type (ReactorTypes.H:12-18)
  if (reactor_type != PPB_REACTOR_E && reactor_type != PPB_REACTOR_H)
    return fail(PPB_E_ARG, "Wrong reactor type. Choose between 1 (e) or 2 (h).");
  if (opt) r->opt = *opt;
  if (r->opt.max_order < 1 || r->opt.max_order > 5) return fail(PPB_E_ARG, "max_order must be in 1..5");
  if (r->opt.max_nls_iters < 1 || r->opt.max_steps < 1 || r->opt.rtol < 0 || r->opt.atol < 0)
    return fail(PPB_E_ARG, "invalid integrator options");
  if (r->opt.engine != PPB_ENGINE_PLAIN && r->opt.engine != PPB_ENGINE_TUNED)
    return fail(PPB_E_ARG, "engine must be PPB_ENGINE_PLAIN or PPB_ENGINE_TUNED");
  if (r->opt.engine == PPB_ENGINE_PLAIN && r->opt.lu_fp32)
    return fail(PPB_E_ARG, "the plain engine is FP64 only");
  if (r->opt.eos != PPB_EOS_IDEAL && r->opt.eos != PPB_EOS_SRK) return fail(PPB_E_ARG, "eos must be 0 or 1");
  if (r->opt.rendezvous_cycles < -1 || r->opt.rendezvous_cycles > 10000000)
    return fail(PPB_E_ARG, "rendezvous_cycles must be -1 or in 0..10000000");
  if (r->opt.warps_per_block > 16) return fail(PPB_E_ARG, "warps_per_block must be at most 16");
  if (r->opt.arkode_barrier_us < 0 || r->opt.arkode_barrier_us > 60000000)
    return fail(PPB_E_ARG, "arkode_barrier_us must be in 0..60000000");
  if (r->opt.adjoint_keep_segments != 0 && r->opt.adjoint_keep_segments != 1)
    return fail(PPB_E_ARG, "adjoint_keep_segments must be 0 or 1");
  if (r->opt.eos == PPB_EOS_SRK) {
    // SRK::RHY2T is not supported (Source/Eos/SRK.H:499-507), nor an
    // analytical Jacobian; this engine runs it on the tuned FP64 BDF
    if (r->method != METHOD_BDF || reactor_type != PPB_REACTOR_E || r->opt.engine != PPB_ENGINE_TUNED ||
        r->opt.lu_fp32)
      return fail(PPB_E_ARG, "the SRK EOS needs ReactorCvode, reactor type 1, the tuned engine and the FP64 LU");
    if (!find_srk(r->t->name)) return fail(PPB_E_MECH, "the mechanism has no SRK parameters");
    if (r->opt.warps_per_block > 8 && r->opt.warps_per_block != 16)
      return fail(PPB_E_ARG, "the SRK EOS runs 1 to 8 or 16 warps per block");
  }
  if (r->t->nqss > 0) {
    // a QSS mechanism: the QSS species solved in every right-hand side, the
    // Jacobian by differences (the reference's dense_direct solve; its
    // analytical QSS Jacobian needs CEPTR's symbolic build); one compiled
    // kernel, the tuned FP64 BDF
    if (r->method != METHOD_BDF || r->opt.engine != PPB_ENGINE_TUNED || r->opt.lu_fp32 ||
        r->opt.eos != PPB_EOS_IDEAL)
      return fail(PPB_E_ARG, "a QSS mechanism needs ReactorCvode, the tuned engine, the FP64 LU and the ideal-gas EOS");
    if (r->opt.warps_per_block > 8 && r->opt.warps_per_block != 16)
      return fail(PPB_E_ARG, "a QSS mechanism runs 1 to 8 or 16 warps per block");
  }
  r->reactor_type = reactor_type;
  int e = 0;
  if (r->own) {
    r->dm = r->own;
  } else {
    e = device_mechanism(r->t, &r->dm);
    if (e) return e;
  }
  if (ncells > 0) {
    e = ensure_scratch(r, ctx_of(r), ncells);
    if (e) return e;
  }
  r->dq16 = false;
  if (r->opt.eos == PPB_EOS_SRK || r->t->nqss > 0) {
    LaunchConfig l16 = launch_config(r);
    l16.warps_per_block = 16;
    r->dq16 = react_occupancy(*r->dm, r->method, l16) >= 16;
  }
  r->gen++;
  r->inited = true;
  return 0;
}

int ppb_set_typ_vals(ppb_reactor* r, const double* typ_vals, int n)
{
  if (!r || !typ_vals) return fail(PPB_E_ARG, "ppb_set_typ_vals: null argument");
  if (n != r->t->nsp + 1) return fail(PPB_E_ARG, "ppb_set_typ_vals: expected N+1 values");
  r->typ_vals.assign(typ_vals, typ_vals + n);
  if (!r->atolv) PPB_CUDA(cudaMalloc(&r->atolv, n * 8), "cudaMalloc");
  std::vector<double> at(n);
  for (int i = 0; i < n; i++) at[i] = typ_vals[i] * r->opt.atol;
  PPB_CUDA(cudaMemcpy(r->atolv, at.data(), n * 8, cudaMemcpyHostToDevice), "cudaMemcpy");
  r->gen++;
  return 0;
}

int ppb_close(ppb_reactor* r)
{
  if (!r) return fail(PPB_E_ARG, "ppb_close: null reactor");
  {
    std::lock_guard<std::mutex> lk(r->ctx_mu);
    for (auto& kv : r->ctxs) {
      free_scratch(kv.second.get());
      if (kv.second->cap_stream) cudaStreamDestroy(kv.second->cap_stream);
    }
    r->ctxs.clear();
  }
  cudaFree(r->atolv);
  r->atolv = nullptr;
  free_adjoint_scratch(r);
  r->inited = false;
  return 0;
}

void ppb_destroy(ppb_reactor* r)
{
  if (!r) return;
  ppb_close(r);
  if (r->own) {
    free_mechanism(r->own);
    delete r->own;
  }
  delete r;
}

// Integrate a species-major batch already on the device (the core call).
static int run_batch(ppb_reactor* r, CallCtx* c, Batch b, double dt, cudaStream_t st, double* rhoe_out = nullptr,
                     bool box = false)
{
  b.atolv = r->atolv;
  b.status = c->status;
  b.nfe = c->nfe;
  b.stats = c->stats;
  if (r->method == METHOD_ARK) return run_ark(r, c, b, dt, st, rhoe_out, box);
  int te = maybe_autotune(r, b, dt, st);
  if (te) return te;
  const Options o = engine_options(r);
  const LaunchConfig lc = launch_config(r);
  if (r->opt.cost_order && lc.engine == ENGINE_TUNED && lc.persistent && b.ncells > 1) {
    // longest first: the previous call's per-cell cost (c->nfe) sorted
    // descending; the kernel then overwrites c->nfe with this call's costs
    int e = launch_cost_order(c->nfe, c->order_keys, c->iota, c->order, c->sort_tmp, c->sort_tmp_bytes, b.ncells,
                              st);
    if (e) return cuda_fail(e, "cost order");
    b.order = c->order;
  }
  int e = launch_react(*r->dm, o, r->method, lc, b, dt, c->queue, st);
  return cuda_fail(e, "launch_react");
}

// True when the caller's stream is being captured into a CUDA graph.
static bool capturing(cudaStream_t st)
{
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  return cudaStreamIsCapturing(st, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone;
}

static int finish(ppb_reactor* r, CallCtx* c, int ncells, cudaStream_t st, long* cost)
{
  c->last_ncells = ncells;
  if (capturing(st)) { // stream-ordered only: flags and costs stay on the device
    if (cost) *cost = 0;
    return 0;
  }
  std::vector<int> stat(ncells), nfe(ncells);
  PPB_CUDA(cudaMemcpyAsync(stat.data(), c->status, ncells * 4, cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
  PPB_CUDA(cudaMemcpyAsync(nfe.data(), c->nfe, ncells * 4, cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync");
  PPB_CUDA(cudaStreamSynchronize(st), "cudaStreamSynchronize");
  long tot = 0;
  int bad = 0;
  for (int i = 0; i < ncells; i++) {
    tot += nfe[i];
    if (stat[i] < 0) bad++;
  }
  if (r->method == METHOD_ARK) {
    int ae = ark_result(c, st);
    if (ae) return ae;
    tot = c->ark_last.nfe; // one integrator for the batch: its RHS evaluations
  }
  if (cost) *cost = (r->method == METHOD_RK64) ? (ncells ? tot / ncells : 0) : tot;
  if (bad) return fail(PPB_E_INTEGRATE, std::to_string(bad) + " cell(s) failed to integrate");
  return 0;
}

int ppb_react_flat(ppb_reactor* r, double* rY, double* rYsrc, double* rX, double* rX_src, double* dt_react,
                   double* time, int ncells, void* stream, long* cost)
{
  if (!r || !r->inited) return fail(PPB_E_STATE, "react before init");
  if (ncells < 0 || !dt_react || !time || (ncells > 0 && (!rY || !rYsrc || !rX || !rX_src)))
    return fail(PPB_E_ARG, "ppb_react_flat: invalid arguments");
  if (ncells == 0) {
    if (cost) *cost = 0;
    *time += *dt_react;
    return 0;
  }
  cudaStream_t st = (cudaStream_t)stream;
  if (capturing(st)) return fail(PPB_E_STATE, "ppb_react_flat copies host arrays and waits: not inside a stream capture");
  CallCtx* c = ctx_of(r);
  int e = ensure_scratch(r, c, ncells, st);
  if (e) return e;
  const int N = r->t->nsp, n = N + 1;
  PPB_CUDA(cudaMemcpyAsync(c->aos, rY, (size_t)ncells * n * 8, cudaMemcpyHostToDevice, st), "H2D rY");
  PPB_CUDA(cudaMemcpyAsync(c->aos_src, rYsrc, (size_t)ncells * N * 8, cudaMemcpyHostToDevice, st), "H2D rYsrc");
  PPB_CUDA(cudaMemcpyAsync(c->rhoe, rX, (size_t)ncells * 8, cudaMemcpyHostToDevice, st), "H2D rX");
  PPB_CUDA(cudaMemcpyAsync(c->rhoesrc, rX_src, (size_t)ncells * 8, cudaMemcpyHostToDevice, st), "H2D rX_src");
  PPB_CUDA(launch_aos_to_soa(c->aos, n, c->soa, ncells, n, ncells, st), "aos_to_soa");
  PPB_CUDA(launch_aos_to_soa(c->aos_src, N, c->soa_src, ncells, N, ncells, st), "aos_to_soa");
  Batch b{};
  b.y = c->soa;
  b.src = c->soa_src;
  b.rhoe = c->rhoe;
  b.rhoesrc = c->rhoesrc;
  b.mask = nullptr;
  b.ncells = ncells;
  b.ld = ncells;
  e = run_batch(r, c, b, *dt_react, st);
  if (e) return e;
  PPB_CUDA(launch_soa_to_aos(c->soa, ncells, n, c->aos, n, ncells, st), "soa_to_aos");
  PPB_CUDA(cudaMemcpyAsync(rY, c->aos, (size_t)ncells * n * 8, cudaMemcpyDeviceToHost, st), "D2H rY");
  e = finish(r, c, ncells, st, cost);
  if (r->method == METHOD_ARK) *dt_react = c->ark_last.t; // the interval integrated
  // ReactorCvode.cpp:1652-1655: rX += dt * rX_src on the host arrays
  for (int i = 0; i < ncells; i++) rX[i] = rX[i] + *dt_react * rX_src[i];
  *time += *dt_react;
  return e;
}

// Device YCOrder path, optionally replayed as a CUDA graph.
int ppb_react_flat_device(ppb_reactor* r, double* rY, double* rYsrc, double* rX, double* rX_src,
                          double* dt_react, double* time, int ncells, void* stream, long* cost)
{
  if (!r || !r->inited) return fail(PPB_E_STATE, "react before init");
  if (ncells < 0 || !dt_react || !time || (ncells > 0 && (!rY || !rYsrc || !rX || !rX_src)))
    return fail(PPB_E_ARG, "ppb_react_flat_device: invalid arguments");
  if (ncells == 0) {
    if (cost) *cost = 0;
    *time += *dt_react;
    return 0;
  }
  cudaStream_t st = (cudaStream_t)stream;
  const bool cap = capturing(st);
  if (cap && r->method == METHOD_ARK)
    return fail(PPB_E_STATE, "ReactorArkode reads its batch result on the host: not inside a stream capture");
  CallCtx* c = ctx_of(r);
  int e = ensure_scratch(r, c, ncells, st);
  if (e) return e;
  const int N = r->t->nsp, n = N + 1;
  const double dt = *dt_react;
  GraphKey key{{rY, rYsrc, rX, rX_src, nullptr, nullptr}, ncells, ncells, dt, st, r->gen.load(), g_tune_gen.load()};
  auto body = [&](cudaStream_t s) -> int {
    int ee = launch_aos_to_soa(rY, n, c->soa, ncells, n, ncells, s);
    if (!ee) ee = launch_aos_to_soa(rYsrc, N, c->soa_src, ncells, N, ncells, s);
    if (ee) return cuda_fail(ee, "aos_to_soa");
    Batch b{};
    b.y = c->soa;
    b.src = c->soa_src;
    b.rhoe = rX;
    b.rhoesrc = rX_src;
    b.ncells = ncells;
    b.ld = ncells;
    ee = run_batch(r, c, b, dt, s, rX);
    if (ee) return ee;
    ee = launch_soa_to_aos(c->soa, ncells, n, rY, n, ncells, s);
    if (!ee && r->method != METHOD_ARK) ee = launch_energy_update(rX, rX_src, dt, ncells, s);
    if (ee) return cuda_fail(ee, "soa_to_aos");
    return 0;
  };
  if (r->opt.use_graph && r->method != METHOD_ARK && !cap) {
    if (!c->gexec || !(c->gkey == key)) {
      // tune outside the capture, on the batch converted to species-major
      PPB_CUDA(launch_aos_to_soa(rY, n, c->soa, ncells, n, ncells, st), "aos_to_soa");
      PPB_CUDA(launch_aos_to_soa(rYsrc, N, c->soa_src, ncells, N, ncells, st), "aos_to_soa");
      Batch tb{};
      tb.y = c->soa;
      tb.src = c->soa_src;
      tb.rhoe = rX;
      tb.rhoesrc = rX_src;
      tb.ncells = ncells;
      tb.ld = ncells;
      e = maybe_autotune(r, tb, dt, st);
      if (e) return e;
    }
    e = capture(c, key, body);
    if (e) return e;
    PPB_CUDA(cudaGraphLaunch(c->gexec, st), "cudaGraphLaunch");
  } else {
    e = body(st);
    if (e) return e;
  }
  e = finish(r, c, ncells, st, cost);
  if (r->method == METHOD_ARK) *dt_react = c->ark_last.t;
  *time += *dt_react;
  return e;
}

int ppb_react_soa_device(ppb_reactor* r, double* y, const double* src, double* rX, const double* rX_src, int ld,
                         double* dt_react, double* time, int ncells, void* stream, long* cost)
{
  if (!r || !r->inited) return fail(PPB_E_STATE, "react before init");
  if (ncells < 0 || ld < ncells || !dt_react || !time || (ncells > 0 && (!y || !src || !rX || !rX_src)))
    return fail(PPB_E_ARG, "ppb_react_soa_device: invalid arguments");
  if (ncells == 0) {
    if (cost) *cost = 0;
    *time += *dt_react;
    return 0;
  }
  cudaStream_t st = (cudaStream_t)stream;
  const bool cap = capturing(st);
  if (cap && r->method == METHOD_ARK)
    return fail(PPB_E_STATE, "ReactorArkode reads its batch result on the host: not inside a stream capture");
  CallCtx* c = ctx_of(r);
  int e = ensure_scratch(r, c, ncells, st);
  if (e) return e;
  const double dt = *dt_react;
  GraphKey key{{y, src, rX, rX_src, (void*)1, nullptr}, ncells, ld, dt, st, r->gen.load(), g_tune_gen.load()};
  Batch b{};
  b.y = y;
  b.src = const_cast<double*>(src);
  b.rhoe = rX;
  b.rhoesrc = rX_src;
  b.ncells = ncells;
  b.ld = ld;
  auto body = [&](cudaStream_t s) -> int {
    int ee = run_batch(r, c, b, dt, s, rX);
    if (!ee && r->method != METHOD_ARK)
      ee = cuda_fail(launch_energy_update(rX, rX_src, dt, ncells, s), "energy_update");
    return ee;
  };
  if (r->opt.use_graph && r->method != METHOD_ARK && !cap) {
    if (!c->gexec || !(c->gkey == key)) {
      e = maybe_autotune(r, b, dt, st); // outside the capture
      if (e) return e;
    }
    e = capture(c, key, body);
    if (e) return e;
    PPB_CUDA(cudaGraphLaunch(c->gexec, st), "cudaGraphLaunch");
  } else {
    e = body(st);
    if (e) return e;
  }
  e = finish(r, c, ncells, st, cost);
  if (r->method == METHOD_ARK) *dt_react = c->ark_last.t;
  *time += *dt_react;
  return e;
}

static BoxView view(const ppb_array4& a)
{
  BoxView v;
  v.p = a.p;
  v.jstride = a.jstride;
  v.kstride = a.kstride;
  v.nstride = a.nstride;
  for (int d = 0; d < 3; d++) v.lo[d] = a.lo[d];
  return v;
}

static bool covers(const ppb_array4& a, const int lo[3], const int hi[3], int ncomp)
{
  if (!a.p || a.ncomp < ncomp) return false;
  for (int d = 0; d < 3; d++)
    if (lo[d] < a.lo[d] || hi[d] > a.hi[d]) return false;
  return true;
}

int ppb_react_box(ppb_reactor* r, const int lo[3], const int hi[3], ppb_array4 rY, ppb_array4 rYsrc, ppb_array4 T,
                  ppb_array4 rEner, ppb_array4 rEner_src, ppb_array4 FC, ppb_array4i mask, double* dt_react,
                  double* time, void* stream)
{
  if (!r || !r->inited) return fail(PPB_E_STATE, "react before init");
  if (!lo || !hi || !dt_react || !time) return fail(PPB_E_ARG, "ppb_react_box: null argument");
  if (r->opt.eos == PPB_EOS_SRK) return fail(PPB_E_ARG, "ppb_react_box: the SRK EOS runs on the flat paths only");
  const int N = r->t->nsp;
  long ncl = 1;
  for (int d = 0; d < 3; d++) {
    if (hi[d] < lo[d]) return fail(PPB_E_ARG, "ppb_react_box: empty box");
    ncl *= (hi[d] - lo[d] + 1);
  }
  if (ncl > (1L << 30)) return fail(PPB_E_ARG, "ppb_react_box: box too large");
  if (!covers(rY, lo, hi, N) || !covers(rYsrc, lo, hi, N) || !covers(T, lo, hi, 1) || !covers(rEner, lo, hi, 1) ||
      !covers(rEner_src, lo, hi, 1) || !covers(FC, lo, hi, 1))
    return fail(PPB_E_ARG, "ppb_react_box: an Array4 does not cover the box");
  if (mask.p) {
    for (int d = 0; d < 3; d++)
      if (lo[d] < mask.lo[d] || hi[d] > mask.hi[d]) return fail(PPB_E_ARG, "ppb_react_box: mask does not cover the box");
  }
  const int ncells = (int)ncl;
  cudaStream_t st = (cudaStream_t)stream;
  const bool cap = capturing(st);
  if (cap && r->method == METHOD_ARK)
    return fail(PPB_E_STATE, "ReactorArkode reads its batch result on the host: not inside a stream capture");
  CallCtx* c = ctx_of(r);
  int e = ensure_scratch(r, c, ncells, st);
  if (e) return e;
  BoxArgs a{};
  for (int d = 0; d < 3; d++) {
    a.lo[d] = lo[d];
    a.hi[d] = hi[d];
  }
  a.rY = view(rY);
  a.rYsrc = view(rYsrc);
  a.T = view(T);
  a.rE = view(rEner);
  a.rEs = view(rEner_src);
  a.FC = view(FC);
  a.mask.p = mask.p;
  a.mask.jstride = mask.jstride;
  a.mask.kstride = mask.kstride;
  a.mask.nstride = mask.nstride;
  for (int d = 0; d < 3; d++) a.mask.lo[d] = mask.lo[d];
  Batch b{};
  b.y = c->soa;
  b.src = c->soa_src;
  b.rhoe = c->rhoe;
  b.rhoesrc = c->rhoesrc;
  b.mask = c->mask;
  b.ncells = ncells;
  b.ld = ncells;
  b.nfe = c->nfe;
  PPB_CUDA(launch_box_flatten(*r->dm, r->reactor_type, r->opt.clean_init_massfrac, a, b, st), "box_flatten");
  e = run_batch(r, c, b, *dt_react, st, nullptr, true);
  if (e) return e;
  if (r->method == METHOD_ARK) {
    e = ark_result(c, st);
    if (e) return e;
    *dt_react = c->ark_last.t; // the interval integrated (ReactorArkode.cpp:223-226)
  }
  PPB_CUDA(launch_box_unflatten(*r->dm, r->reactor_type, r->opt.clean_init_massfrac, a, b, *dt_react, st),
           "box_unflatten");
  e = finish(r, c, ncells, st, nullptr);
  *time += *dt_react;
  return e;
}

// Box bounds and cell count of a flatten/unflatten call.
static int box_cells(const int lo[3], const int hi[3], long* ncl)
{
  *ncl = 1;
  for (int d = 0; d < 3; d++) {
    if (hi[d] < lo[d]) return fail(PPB_E_ARG, "empty box");
    *ncl *= (hi[d] - lo[d] + 1);
  }
  if (*ncl > (1L << 30)) return fail(PPB_E_ARG, "box too large");
  return 0;
}

int ppb_flatten(ppb_reactor* r, const int lo[3], const int hi[3], ppb_array4 rhoY, ppb_array4 frcExt,
                ppb_array4 temperature, ppb_array4 rhoE, ppb_array4 frcEExt, double* y_vect, double* src_vect,
                double* vect_energy, double* src_vect_energy, void* stream)
{
  if (!r || !r->inited) return fail(PPB_E_STATE, "flatten before init");
  if (!lo || !hi || !y_vect || !src_vect || !vect_energy || !src_vect_energy)
    return fail(PPB_E_ARG, "ppb_flatten: null argument");
  long ncl = 0;
  if (box_cells(lo, hi, &ncl)) return PPB_E_ARG;
  const int N = r->t->nsp;
  if (!covers(rhoY, lo, hi, N) || !covers(frcExt, lo, hi, N) || !covers(temperature, lo, hi, 1) ||
      !covers(rhoE, lo, hi, 1) || !covers(frcEExt, lo, hi, 1))
    return fail(PPB_E_ARG, "ppb_flatten: an Array4 does not cover the box");
  BoxArgs a{};
  for (int d = 0; d < 3; d++) {
    a.lo[d] = lo[d];
    a.hi[d] = hi[d];
  }
  a.rY = view(rhoY);
  a.rYsrc = view(frcExt);
  a.T = view(temperature);
  a.rE = view(rhoE);
  a.rEs = view(frcEExt);
  Batch b{};
  b.y = y_vect;
  b.src = src_vect;
  b.rhoe = vect_energy;
  b.rhoesrc = src_vect_energy;
  b.ncells = (int)ncl;
  b.ld = (int)ncl;
  PPB_CUDA(launch_box_flatten(*r->dm, r->reactor_type, r->opt.clean_init_massfrac, a, b, (cudaStream_t)stream),
           "box_flatten");
  return 0;
}

int ppb_unflatten(ppb_reactor* r, const int lo[3], const int hi[3], ppb_array4 rhoY, ppb_array4 temperature,
                  ppb_array4 rhoE, ppb_array4 frcEExt, ppb_array4 FC, const double* y_vect,
                  const double* vect_energy, const long* FCunt, double dt, void* stream)
{
  if (!r || !r->inited) return fail(PPB_E_STATE, "unflatten before init");
  if (!lo || !hi || !y_vect || !vect_energy || !FCunt) return fail(PPB_E_ARG, "ppb_unflatten: null argument");
  long ncl = 0;
  if (box_cells(lo, hi, &ncl)) return PPB_E_ARG;
  const int N = r->t->nsp;
  if (!covers(rhoY, lo, hi, N) || !covers(temperature, lo, hi, 1) || !covers(rhoE, lo, hi, 1) ||
      !covers(frcEExt, lo, hi, 1) || !covers(FC, lo, hi, 1))
    return fail(PPB_E_ARG, "ppb_unflatten: an Array4 does not cover the box");
  BoxArgs a{};
  for (int d = 0; d < 3; d++) {
    a.lo[d] = lo[d];
    a.hi[d] = hi[d];
  }
  a.rY = view(rhoY);
  a.T = view(temperature);
  a.rE = view(rhoE);
  a.rEs = view(frcEExt);
  a.FC = view(FC);
  a.fcunt = FCunt;
  Batch b{};
  b.y = const_cast<double*>(y_vect);
  b.rhoe = vect_energy;
  b.ncells = (int)ncl;
  b.ld = (int)ncl;
  PPB_CUDA(launch_box_unflatten(*r->dm, r->reactor_type, r->opt.clean_init_massfrac, a, b, dt,
                                (cudaStream_t)stream),
           "box_unflatten");
  return 0;
}

// ---------------------------------------------------------------- transport
static int transport_tables(const char* mechanism, DeviceMechanism** dm, DeviceTransport** dt)
{
  const PPBMechTables* t = mechanism ? find_mechanism(mechanism) : nullptr;
  const PPBTransTables* tr = mechanism ? find_transport(mechanism) : nullptr;
  if (!t || !tr) return fail(PPB_E_MECH, std::string("unknown mechanism ") + (mechanism ? mechanism : "(null)"));
  int e = device_mechanism(t, dm);
  if (e) return e;
  e = device_transport(tr, dt);
  return e ? cuda_fail(e, "transport tables") : 0;
}

static BoxView flat_view(const double* p, long nstride)
{
  BoxView v{};
  v.p = const_cast<double*>(p);
  v.nstride = nstride;
  return v;
}

int ppb_transport(const char* mechanism, int flags, const double* T, const double* rho, const double* Y, int ld,
                  double* D, double* chi, double* mu, double* xi, double* lam, int ncells, void* stream)
{
  if (ncells < 0 || ld < ncells || (flags & ~31)) return fail(PPB_E_ARG, "ppb_transport: invalid arguments");
  if (ncells > 0 && (!T || !Y || ((flags & PPB_TR_DIAG) && !D) || ((flags & PPB_TR_CHI) && !chi) ||
                     ((flags & PPB_TR_MU) && !mu) || ((flags & PPB_TR_XI) && !xi) || ((flags & PPB_TR_LAM) && !lam)))
    return fail(PPB_E_ARG, "ppb_transport: null array for a selected output");
  DeviceMechanism* dm = nullptr;
  DeviceTransport* dt = nullptr;
  int e = transport_tables(mechanism, &dm, &dt);
  if (e || ncells == 0) return e;
  TrBox b{};
  b.hi[0] = ncells - 1;
  b.Y = flat_view(Y, ld);
  b.T = flat_view(T, 0);
  b.rho = flat_view(rho, 0);
  b.D = flat_view(D, ld);
  b.chi = flat_view(chi, ld);
  b.mu = flat_view((flags & PPB_TR_MU) ? mu : nullptr, 0);
  b.xi = flat_view((flags & PPB_TR_XI) ? xi : nullptr, 0);
  b.lam = flat_view((flags & PPB_TR_LAM) ? lam : nullptr, 0);
  return cuda_fail(launch_transport(*dm, *dt, flags, b, (cudaStream_t)stream), "launch_transport");
}

int ppb_transport_box(const char* mechanism, int use_soret, const int lo[3], const int hi[3], ppb_array4 Y,
                      ppb_array4 T, ppb_array4 rho, ppb_array4 D, ppb_array4 chi, ppb_array4 mu, ppb_array4 xi,
                      ppb_array4 lam, void* stream)
{
  if (!lo || !hi) return fail(PPB_E_ARG, "ppb_transport_box: null box");
  const PPBMechTables* t = mechanism ? find_mechanism(mechanism) : nullptr;
  if (!t) return fail(PPB_E_MECH, std::string("unknown mechanism ") + (mechanism ? mechanism : "(null)"));
  const int N = t->nsp;
  for (int d = 0; d < 3; d++)
    if (hi[d] < lo[d]) return fail(PPB_E_ARG, "ppb_transport_box: empty box");
  if (!covers(Y, lo, hi, N) || !covers(T, lo, hi, 1) || !covers(rho, lo, hi, 1) || !covers(D, lo, hi, N) ||
      !covers(mu, lo, hi, 1) || !covers(xi, lo, hi, 1) || !covers(lam, lo, hi, 1) ||
      (use_soret && !covers(chi, lo, hi, N)))
    return fail(PPB_E_ARG, "ppb_transport_box: an Array4 does not cover the box");
  DeviceMechanism* dm = nullptr;
  DeviceTransport* dt = nullptr;
  int e = transport_tables(mechanism, &dm, &dt);
  if (e) return e;
  TrBox b{};
  for (int d = 0; d < 3; d++) {
    b.lo[d] = lo[d];
    b.hi[d] = hi[d];
  }
  b.Y = view(Y);
  b.T = view(T);
  b.rho = view(rho);
  b.D = view(D);
  b.chi = use_soret ? view(chi) : BoxView{};
  b.mu = view(mu);
  b.xi = view(xi);
  b.lam = view(lam);
  const int flags = PPB_TR_XI | PPB_TR_MU | PPB_TR_LAM | PPB_TR_DIAG | (use_soret ? PPB_TR_CHI : 0);
  return cuda_fail(launch_transport(*dm, *dt, flags, b, (cudaStream_t)stream), "launch_transport");
}

int ppb_get_cell_status(ppb_reactor* r, int* status, int* cost, int ncells)
{
  if (!r) return fail(PPB_E_ARG, "ppb_get_cell_status: null reactor");
  CallCtx* c = ctx_of(r);
  if (ncells < 0 || ncells > c->last_ncells) return fail(PPB_E_ARG, "ppb_get_cell_status: bad arguments");
  if (status) PPB_CUDA(cudaMemcpy(status, c->status, (size_t)ncells * 4, cudaMemcpyDeviceToHost), "cudaMemcpy");
  if (cost) PPB_CUDA(cudaMemcpy(cost, c->nfe, (size_t)ncells * 4, cudaMemcpyDeviceToHost), "cudaMemcpy");
  return 0;
}

int ppb_last_ncells(ppb_reactor* r)
{
  if (!r) return fail(PPB_E_ARG, "ppb_last_ncells: null reactor");
  return ctx_of(r)->last_ncells;
}

int ppb_get_cell_stats(ppb_reactor* r, int* stats, int ncells)
{
  if (!r || !stats) return fail(PPB_E_ARG, "ppb_get_cell_stats: null argument");
  CallCtx* c = ctx_of(r);
  if (ncells < 0 || ncells > c->last_ncells) return fail(PPB_E_ARG, "ppb_get_cell_stats: bad arguments");
  PPB_CUDA(cudaMemcpy(stats, c->stats, (size_t)ncells * 7 * 4, cudaMemcpyDeviceToHost), "cudaMemcpy");
  return 0;
}

int ppb_probe_fp64_peak(double* gflops, void* stream)
{
  if (!gflops) return fail(PPB_E_ARG, "ppb_probe_fp64_peak: null output");
  return cuda_fail(probe_fp64_peak(gflops, (cudaStream_t)stream), "probe_fp64_peak");
}

int ppb_get_launch_config(ppb_reactor* r, int* warps_per_block, int* team_lanes, int* register_budget,
                          double* tuned_ms)
{
  if (!r || !r->inited) return fail(PPB_E_STATE, "ppb_get_launch_config before init");
  const LaunchConfig lc = launch_config(r);
  double ms = 0.0;
  LaunchConfig tl;
  if (r->opt.warps_per_block <= 0) tuned_config(r, &tl, &ms);
  if (warps_per_block) *warps_per_block = lc.warps_per_block;
  if (team_lanes) *team_lanes = lc.team;
  if (register_budget) *register_budget = lc.minb;
  if (tuned_ms) *tuned_ms = ms;
  return 0;
}

int ppb_get_rendezvous_cycles(ppb_reactor* r, int* cycles)
{
  if (!r || !r->inited) return fail(PPB_E_STATE, "ppb_get_rendezvous_cycles before init");
  if (!cycles) return fail(PPB_E_ARG, "ppb_get_rendezvous_cycles: null argument");
  const LaunchConfig lc = launch_config(r);
  // the rendezvous runs in the tuned BDF kernels of one warp per cell
  if (r->method != METHOD_BDF || lc.engine != ENGINE_TUNED || lc.team != 32) {
    *cycles = 0;
    return 0;
  }
  const int o = r->opt.rendezvous_cycles;
  *cycles = (o < 0 && lc.rv > 0) ? lc.rv : rendezvous_bound(o, lc.warps_per_block);
  return 0;
}

int ppb_get_arrhenius(ppb_reactor* r, double* A, double* beta, double* EaR)
{
  if (!r || !A || !beta || !EaR) return fail(PPB_E_ARG, "ppb_get_arrhenius: null argument");
  const PPBMechTables* t = r->own ? &r->own_t : r->t;
  for (int k = 0; k < t->nrxn; k++) {
    A[k] = t->rx_A[k];
    beta[k] = t->rx_beta[k];
    EaR[k] = t->rx_EaR[k];
  }
  return 0;
}

int ppb_set_arrhenius(ppb_reactor* r, const double* A, const double* beta, const double* EaR)
{
  if (!r || !A || !beta || !EaR) return fail(PPB_E_ARG, "ppb_set_arrhenius: null argument");
  const int R = r->t->nrxn;
  r->own_A.assign(A, A + R);
  r->own_beta.assign(beta, beta + R);
  r->own_EaR.assign(EaR, EaR + R);
  r->own_t = *r->t;
  r->own_t.rx_A = r->own_A.data();
  r->own_t.rx_beta = r->own_beta.data();
  r->own_t.rx_EaR = r->own_EaR.data();
  auto* m = new DeviceMechanism();
  const int e = upload_mechanism(&r->own_t, m);
  if (e) {
    delete m;
    return cuda_fail(e, "upload_mechanism");
  }
  if (r->own) {
    free_mechanism(r->own);
    delete r->own;
  }
  r->own = m;
  if (r->inited) r->dm = m;
  r->gen++;
  return 0;
}

static int grow_items(void* ctx, void** p, size_t bytes)
{
  ppb_reactor* r = static_cast<ppb_reactor*>(ctx);
  r->adj_items = *p;
  const int e = grow(r->adj_items, r->adj_items_bytes, bytes);
  *p = r->adj_items;
  return e;
}

// The adjoint integration, batched over cells segment by segment (chunks of
// cells within adjoint_memory_mb).
static int run_adjoint_batched(ppb_reactor* r, CallCtx* cx, AdjBatch b, double dt, double* grad, cudaStream_t st)
{
  const int N = r->t->nsp, n = N + 1, R = r->t->nrxn;
  const int seg = r->opt.adjoint_checkpoint_interval > 0 ? r->opt.adjoint_checkpoint_interval : 16;
  AdjCells C{};
  C.seg_steps = seg;
  C.close_rec = 128;
  C.cap_rec = C.close_rec + 2 * (r->opt.max_err_fails + 10) + 8;
  C.close_y = 32;
  C.cap_y = C.close_y + r->opt.max_err_fails + 2;
  C.max_seg = r->opt.max_steps / seg + 2;
  C.cp_stride = adj_cp_bytes(N, r->opt.lu_fp32);
  const size_t item_b = adj_item_bytes(N, R);
  const size_t budget = (size_t)(r->opt.adjoint_memory_mb > 0 ? r->opt.adjoint_memory_mb : 16384) << 20;
  const size_t per_cell = (size_t)C.max_seg * 4 + (size_t)C.cap_rec * ADJ_TAPE_BYTES + (size_t)C.cap_y * (8 * n + 16) +
                          3 * 4 + 3 * 8 + (size_t)7 * n * 8 + (size_t)3 * R * 8 + 4;
  // the budget: the per-cell arrays of the cells of one chunk (all cells when
  // they take at most two fifths), then the rest in equal parts for the
  // checkpoints, the segment copies (a segment whose copy fits is not
  // recomputed in the reverse sweep; without copies the checkpoints get
  // their part) and the evaluated points of one segment
  const long cells = std::max<long>(1, std::min<long>(b.ncells, (long)(budget * 2 / 5 / per_cell)));
  const size_t rest = budget - std::min(budget, (size_t)cells * per_cell);
  const bool keep = r->opt.adjoint_keep_segments != 0;
  const size_t pool_bytes = keep ? rest / 3 : rest / 3 * 2;
  C.pool_cap = (int)std::min<size_t>(pool_bytes / C.cp_stride, 1u << 30);
  C.tpool_bytes = keep ? (rest / 3) & ~size_t(15) : 0;
  C.items_cap = std::max<long>((long)(rest / 3 / item_b), C.cap_y + 1);
  if (C.pool_cap < 2) return fail(PPB_E_ARG, "adjoint: adjoint_memory_mb too small for the checkpoints");
  const size_t nc = (size_t)cells;
  int e;
  if ((e = grow(r->adj_cp, r->adj_cp_bytes, (size_t)C.pool_cap * C.cp_stride + 16)) ||
      (e = grow(r->adj_cpidx, r->adj_cpidx_bytes, nc * C.max_seg * 4)) ||
      (e = grow(r->adj_tape, r->adj_tape_bytes, nc * C.cap_rec * ADJ_TAPE_BYTES)) ||
      (e = grow(r->adj_ys, r->adj_ys_bytes, nc * C.cap_y * n * 8)) ||
      (e = grow(r->adj_yinfo, r->adj_yinfo_bytes, nc * C.cap_y * 16)) ||
      (e = grow(r->adj_ints, r->adj_ints_bytes, nc * 3 * 4 + 16)) ||
      (e = grow(r->adj_dbl, r->adj_dbl_bytes, nc * 3 * 8)) || (e = grow(r->adj_lam, r->adj_lam_bytes, nc * 7 * n * 8)) ||
      (e = grow(r->adj_tpool, r->adj_tpool_bytes, C.tpool_bytes ? C.tpool_bytes + 16 : 0)) ||
      (e = grow(r->adj_gw, r->adj_gw_bytes, nc * 3 * R * 8)) ||
      (e = grow(r->adj_items, r->adj_items_bytes, (size_t)C.items_cap * item_b)) ||
      (e = grow(r->adj_ioff, r->adj_ioff_bytes, (nc + 1) * 4)))
    return e;
  C.cp_pool = (char*)r->adj_cp;
  C.pool_next = (int*)((char*)r->adj_cp + (size_t)C.pool_cap * C.cp_stride);
  C.cp_idx = (int*)r->adj_cpidx;
  C.tape = r->adj_tape;
  C.ys = (double*)r->adj_ys;
  C.yinfo = (double*)r->adj_yinfo;
  C.nrec = (int*)r->adj_ints;
  C.ny = C.nrec + nc;
  C.nseg = C.ny + nc;
  C.h0 = (double*)r->adj_dbl;
  C.lamE = C.h0 + nc;
  C.toff = (long long*)(C.lamE + nc);
  C.tpool = C.tpool_bytes ? (char*)r->adj_tpool : nullptr;
  C.tpool_next = C.tpool ? (unsigned long long*)(C.tpool + C.tpool_bytes) : nullptr;
  C.lam = (double*)r->adj_lam;
  C.gw = (double*)r->adj_gw;
  C.items = (double*)r->adj_items;
  C.item_off = (int*)r->adj_ioff;
  b.atolv = r->atolv;
  b.status = cx->status;
  b.stats = cx->stats;
  const Options o = engine_options(r);
  for (long c0 = 0; c0 < b.ncells; c0 += cells) {
    AdjBatch bc = b;
    const size_t cn = (size_t)c0 * n, cN = (size_t)c0 * N;
    bc.ncells = (int)std::min<long>(cells, b.ncells - c0);
    bc.y0 = b.y0 + cn;
    bc.src = b.src ? b.src + cN : nullptr;
    bc.rhoe = b.rhoe + c0;
    bc.rhoesrc = b.rhoesrc ? b.rhoesrc + c0 : nullptr;
    bc.lam_y = b.lam_y + cn;
    bc.y_out = b.y_out ? b.y_out + cn : nullptr;
    bc.lam_y0 = b.lam_y0 ? b.lam_y0 + cn : nullptr;
    bc.lam_e = b.lam_e ? b.lam_e + c0 : nullptr;
    bc.status = b.status + c0;
    bc.stats = b.stats + (size_t)c0 * 7;
    e = launch_adjoint_batched(*r->dm, o, r->opt.lu_fp32, bc, C, dt, cx->queue, grad, c0 > 0 ? 1 : 0, grow_items, r,
                               st);
    if (e) return cuda_fail(e, "launch_adjoint_batched");
  }
  cx->last_ncells = b.ncells;
  std::vector<int> stat(b.ncells);
  PPB_CUDA(cudaMemcpyAsync(stat.data(), cx->status, (size_t)b.ncells * 4, cudaMemcpyDeviceToHost, st),
           "cudaMemcpyAsync");
  PPB_CUDA(cudaStreamSynchronize(st), "cudaStreamSynchronize");
  int bad = 0;
  for (int c = 0; c < b.ncells; c++) bad += stat[c] < 0;
  if (bad) return fail(PPB_E_INTEGRATE, std::to_string(bad) + " cell(s) failed in the adjoint integration");
  return 0;
}

// Shared set-up and launch of the adjoint (mode ADJ_REVERSE) and tangent
// (ADJ_TANGENT) integrations.
static int run_adjoint(ppb_reactor* r, int mode, AdjBatch b, double dt, double* grad, cudaStream_t st)
{
  if (!r || !r->inited) return fail(PPB_E_ARG, "adjoint: reactor not initialised");
  if (r->method != METHOD_BDF)
    return fail(PPB_E_ARG, "adjoint: only the BDF integrator (ReactorCvode) is differentiated");
  if (r->opt.eos != PPB_EOS_IDEAL) return fail(PPB_E_ARG, "adjoint: the ideal-gas EOS only");
  if (r->t->nqss > 0) return fail(PPB_E_ARG, "adjoint: not for QSS mechanisms");
  if (r->opt.engine != PPB_ENGINE_TUNED) return fail(PPB_E_ARG, "adjoint: runs on the tuned engine only");
  if (b.ncells < 0 || (b.ncells > 0 && (!b.y0 || !b.rhoe))) return fail(PPB_E_ARG, "adjoint: invalid arguments");
  if (mode == ADJ_REVERSE && b.ncells > 0 && !b.lam_y) return fail(PPB_E_ARG, "adjoint: lam_y is required");
  if (b.ncells == 0) {
    if (grad) PPB_CUDA(cudaMemsetAsync(grad, 0, sizeof(double) * 3 * r->t->nrxn, st), "cudaMemsetAsync");
    return 0;
  }
  if (capturing(st)) return fail(PPB_E_STATE, "adjoint: not inside a stream capture");
  std::lock_guard<std::mutex> lk(r->adj_mu);
  CallCtx* cx = ctx_of(r);
  int e = ensure_scratch(r, cx, b.ncells, st);
  if (e) return e;
  if (mode == ADJ_REVERSE) return run_adjoint_batched(r, cx, b, dt, grad, st);
  const int N = r->t->nsp, n = N + 1, R = r->t->nrxn;
  AdjPlan p;
  e = plan_adjoint(*r->dm, mode, r->opt.lu_fp32, &p);
  if (e) return cuda_fail(e, "plan_adjoint");
  const int seg = r->opt.adjoint_checkpoint_interval > 0 ? r->opt.adjoint_checkpoint_interval : 16;
  AdjLayout L{};
  L.seg_steps = seg;
  L.close_rec = 256;
  L.cap_rec = L.close_rec + 2 * (r->opt.max_err_fails + 10) + 8;
  L.close_y = 64;
  L.cap_y = L.close_y + r->opt.max_err_fails + 2;
  L.cp_stride = p.cp_stride;
  L.cap_cp = (mode == ADJ_REVERSE) ? r->opt.max_steps / seg + 2 : 0;
  L.warp_smem = p.warp_smem;
  const size_t tape_w = (size_t)L.cap_rec * ADJ_TAPE_BYTES;
  const size_t ys_w = (size_t)L.cap_y * n * 8;
  const size_t gw_cell = (size_t)3 * R * 8;
  // cells per launch: the per-cell gradients of one launch stay under 512 MiB
  const int chunk = (int)std::min<size_t>((size_t)b.ncells, std::max<size_t>(1, (size_t(512) << 20) / gw_cell));
  const size_t budget = (size_t)(r->opt.adjoint_memory_mb > 0 ? r->opt.adjoint_memory_mb : 8192) << 20;
  // no more warps than cells, and within the memory budget
  int blocks = std::min(p.blocks, (chunk + p.wpb - 1) / p.wpb);
  size_t per_warp = (size_t)L.cap_cp * L.cp_stride + tape_w + ys_w;
  if ((size_t)blocks * p.wpb * per_warp > budget) {
    blocks = (int)std::max<size_t>(1, budget / (per_warp * p.wpb));
    if ((size_t)blocks * p.wpb * per_warp > budget) {
      const size_t room = budget / p.wpb;
      if (room <= tape_w + ys_w + 2 * L.cp_stride)
        return fail(PPB_E_ARG, "adjoint: adjoint_memory_mb too small for one block of checkpoints");
      L.cap_cp = (int)((room - tape_w - ys_w) / L.cp_stride);
    }
  }
  p.blocks = blocks;
  const size_t W = (size_t)blocks * p.wpb;
  if ((e = grow(r->adj_cp, r->adj_cp_bytes, W * L.cap_cp * L.cp_stride)) ||
      (e = grow(r->adj_tape, r->adj_tape_bytes, W * tape_w)) || (e = grow(r->adj_ys, r->adj_ys_bytes, W * ys_w)) ||
      (e = grow(r->adj_gw, r->adj_gw_bytes, mode == ADJ_REVERSE ? (size_t)chunk * gw_cell : 0)))
    return e;
  L.cp = (char*)r->adj_cp;
  L.tape = r->adj_tape;
  L.ys = (double*)r->adj_ys;
  L.gw = mode == ADJ_REVERSE ? (double*)r->adj_gw : nullptr;
  b.atolv = r->atolv;
  b.status = cx->status;
  b.stats = cx->stats;
  const Options o = engine_options(r);
  for (int c0 = 0; c0 < b.ncells; c0 += chunk) {
    AdjBatch bc = b;
    const size_t cn = (size_t)c0 * n, cN = (size_t)c0 * N;
    bc.ncells = std::min(chunk, b.ncells - c0);
    bc.y0 = b.y0 + cn;
    bc.src = b.src ? b.src + cN : nullptr;
    bc.rhoe = b.rhoe + c0;
    bc.rhoesrc = b.rhoesrc ? b.rhoesrc + c0 : nullptr;
    bc.lam_y = b.lam_y ? b.lam_y + cn : nullptr;
    bc.dy0 = b.dy0 ? b.dy0 + cn : nullptr;
    bc.dE = b.dE ? b.dE + c0 : nullptr;
    bc.y_out = b.y_out ? b.y_out + cn : nullptr;
    bc.lam_y0 = b.lam_y0 ? b.lam_y0 + cn : nullptr;
    bc.lam_e = b.lam_e ? b.lam_e + c0 : nullptr;
    bc.status = b.status + c0;
    bc.stats = b.stats + (size_t)c0 * 7;
    e = launch_adjoint(*r->dm, o, mode, r->opt.lu_fp32, p, bc, L, dt, cx->queue, grad, c0 > 0 ? 1 : 0, st);
    if (e) return cuda_fail(e, "launch_adjoint");
  }
  cx->last_ncells = b.ncells;
  std::vector<int> stat(b.ncells);
  PPB_CUDA(cudaMemcpyAsync(stat.data(), cx->status, (size_t)b.ncells * 4, cudaMemcpyDeviceToHost, st),
           "cudaMemcpyAsync");
  PPB_CUDA(cudaStreamSynchronize(st), "cudaStreamSynchronize");
  int bad = 0;
  for (int c = 0; c < b.ncells; c++) bad += stat[c] < 0;
  if (bad) return fail(PPB_E_INTEGRATE, std::to_string(bad) + " cell(s) failed in the adjoint integration");
  return 0;
}

int ppb_adjoint_flat_device(ppb_reactor* r, const double* rY0, const double* rYsrc, const double* rX,
                            const double* rX_src, double dt_react, int ncells, const double* lam_y, double* y_out,
                            double* lam_y0, double* lam_e, double* grad_params, void* stream)
{
  AdjBatch b{};
  b.y0 = rY0;
  b.src = rYsrc;
  b.rhoe = rX;
  b.rhoesrc = rX_src;
  b.lam_y = lam_y;
  b.y_out = y_out;
  b.lam_y0 = lam_y0;
  b.lam_e = lam_e;
  b.ncells = ncells;
  return run_adjoint(r, ADJ_REVERSE, b, dt_react, grad_params, (cudaStream_t)stream);
}

int ppb_tangent_flat_device(ppb_reactor* r, const double* rY0, const double* rYsrc, const double* rX,
                            const double* rX_src, double dt_react, int ncells, const double* dy0, const double* drX,
                            const double* dparams, double* y_out, double* dy_out, void* stream)
{
  if (!dparams) return fail(PPB_E_ARG, "ppb_tangent_flat_device: dparams is required (zeros for none)");
  AdjBatch b{};
  b.y0 = rY0;
  b.src = rYsrc;
  b.rhoe = rX;
  b.rhoesrc = rX_src;
  b.dy0 = dy0;
  b.dE = drX;
  b.dp = dparams;
  b.y_out = y_out;
  b.lam_y0 = dy_out;
  b.ncells = ncells;
  return run_adjoint(r, ADJ_TANGENT, b, dt_react, nullptr, (cudaStream_t)stream);
}

int ppb_rhs_exact(const char* mechanism, int reactor_type, double t, const double* y, const double* rhoe,
                  const double* rhoesrc, const double* src, const double* v, double* f, double* dfdy, double* dfde,
                  double* vjp_y, double* vjp_e, double* vjp_p, int ncells, void* stream)
{
  DeviceMechanism* dm;
  const PPBMechTables* tab = mechanism ? find_mechanism(mechanism) : nullptr;
  if (!tab) return fail(PPB_E_MECH, std::string("unknown mechanism ") + (mechanism ? mechanism : "(null)"));
  int e = device_mechanism(tab, &dm);
  if (e) return e;
  if (ncells < 0 || !y || !rhoe || (reactor_type != 1 && reactor_type != 2))
    return fail(PPB_E_ARG, "ppb_rhs_exact: bad arguments");
  return cuda_fail(launch_rhs_exact(*dm, reactor_type, t, y, rhoe, rhoesrc, src, v, f, dfdy, dfde, vjp_y, vjp_e,
                                    vjp_p, ncells, (cudaStream_t)stream),
                   "rhs_exact");
}

static int point_mech(const char* mechanism, DeviceMechanism** dm)
{
  const PPBMechTables* t = mechanism ? find_mechanism(mechanism) : nullptr;
  if (!t) return fail(PPB_E_MECH, std::string("unknown mechanism ") + (mechanism ? mechanism : "(null)"));
  return device_mechanism(t, dm);
}

int ppb_production_rate(const char* mechanism, const double* sc, const double* T, double* wdot, int ncells, int team,
                        void* stream)
{
  DeviceMechanism* dm;
  int e = point_mech(mechanism, &dm);
  if (e) return e;
  if (ncells < 0 || (team != 1 && team != 32)) return fail(PPB_E_ARG, "ppb_production_rate: bad arguments");
  return cuda_fail(launch_production_rate(*dm, sc, T, wdot, ncells, team, (cudaStream_t)stream), "production_rate");
}

int ppb_ajacobian(const char* mechanism, const double* sc, const double* T, int consP, double* J, int ncells,
                  int team, void* stream)
{
  DeviceMechanism* dm;
  int e = point_mech(mechanism, &dm);
  if (e) return e;
  if (ncells < 0 || (team != 1 && team != 32)) return fail(PPB_E_ARG, "ppb_ajacobian: bad arguments");
  return cuda_fail(launch_ajacobian(*dm, sc, T, consP, J, ncells, team, (cudaStream_t)stream), "ajacobian");
}

int ppb_t_from_energy(const char* mechanism, int eh, const double* e_in, const double* Y, double* T, int ncells,
                      int team, void* stream)
{
  DeviceMechanism* dm;
  int e = point_mech(mechanism, &dm);
  if (e) return e;
  if (ncells < 0 || (team != 1 && team != 32)) return fail(PPB_E_ARG, "ppb_t_from_energy: bad arguments");
  return cuda_fail(launch_t_from_energy(*dm, eh, e_in, Y, T, ncells, team, (cudaStream_t)stream), "t_from_energy");
}

int ppb_reactor_rhs(const char* mechanism, int reactor_type, double t, const double* y, const double* rhoe,
                    const double* rhoesrc, const double* src, double* ydot, int ncells, int team, void* stream)
{
  DeviceMechanism* dm;
  int e = point_mech(mechanism, &dm);
  if (e) return e;
  if (ncells < 0 || (team != 1 && team != 32) || (reactor_type != 1 && reactor_type != 2))
    return fail(PPB_E_ARG, "ppb_reactor_rhs: bad arguments");
  return cuda_fail(launch_reactor_rhs(*dm, reactor_type, t, y, rhoe, rhoesrc, src, ydot, ncells, team,
                                      (cudaStream_t)stream),
                   "reactor_rhs");
}

int ppb_pyt2re(const char* mechanism, int eh, const double* P, const double* T, const double* Y, double* rho,
               double* e_out, int ncells, void* stream)
{
  DeviceMechanism* dm;
  int e = point_mech(mechanism, &dm);
  if (e) return e;
  if (ncells < 0 || (eh != 0 && eh != 1)) return fail(PPB_E_ARG, "ppb_pyt2re: bad arguments");
  return cuda_fail(launch_pyt2re(*dm, eh, P, T, Y, rho, e_out, ncells, (cudaStream_t)stream), "pyt2re");
}

#ifdef PPB_PHASE_TIMERS
// Profiling builds only: per-phase cycle totals of the BDF kernels.
int ppb_phase_cycles(unsigned long long* out, int reset) { return cuda_fail(phase_cycles(out, reset), "phase"); }
#endif

} // extern "C"
