// Allocation-free variant of the flat device react path
// (ppb_react_flat_device_noalloc in include/pelephysics_b200.h).
//
// Some callers cannot have a library allocate GPU memory: applications whose
// device memory is owned by their own arena allocator (AMReX-based codes such
// as PeleC and PeleLMeX hand every device buffer out of the AMReX Arena, whose
// size and out-of-memory handling assume nobody else calls cudaMalloc), and
// codes that run next to them in the same process with the memory budget
// already spent.  For them this entry point works entirely out of one
// file-scope device array, PPB_NOALLOC_BYTES (32 MiB) per GPU, which holds
// the mechanism tables and the per-call scratch (species-major copies of the
// state and sources, per-cell flags and costs, the work-queue counter and a
// failure counter).  The array is part of the library image: every GPU that
// loads the library holds it until the process exits.
//
// Set-up: the first call on each device (with that device current) resolves
// the array's device address with cudaGetSymbolAddress and copies the
// mechanism tables into it with a synchronous cudaMemcpy; the first use of a
// further mechanism on that device copies its tables the same way.  That
// first call should therefore come before any stream capture.
//
// All calls on a device share the array, and it keeps the previous call's
// contents: the kernels clear what must start at zero (queue and failure
// counters); calls that overlap on the GPU (different streams or host
// threads without ordering) race on the scratch and must not be issued.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <mutex>

#include "../../include/pelephysics_b200.h"
#include "ppb_bdf.cuh"
#include "ppb_engine.h"

namespace ppb {
enum : size_t {
  PPB_NOALLOC_BYTES = size_t(32) << 20,  // whole array
  PPB_NOALLOC_TABLES = size_t(2) << 20,  // mechanism tables region
  PPB_NOALLOC_MAX_DEVICES = 64,
  PPB_NOALLOC_MAX_MECHS = 8,
};
} // namespace ppb

static __device__ __align__(256) unsigned char g_ppb_noalloc[ppb::PPB_NOALLOC_BYTES];

namespace {
using namespace ppb;

struct DeviceSlot {
  bool ready = false;
  unsigned char* base = nullptr; // device address of g_ppb_noalloc
  size_t tables_used = 0;
  const PPBMechTables* mech[PPB_NOALLOC_MAX_MECHS] = {};
  DevMech dm[PPB_NOALLOC_MAX_MECHS];
};

std::mutex g_mu;
DeviceSlot g_slots[PPB_NOALLOC_MAX_DEVICES];
char g_stage[PPB_NOALLOC_TABLES]; // host staging image of one mechanism's tables
int nf(int code, const char* msg)
{
  set_error(msg);
  return code;
}

// per-device set-up and per-mechanism table upload (under g_mu)
int setup(const PPBMechTables* t, DeviceMechanism* out)
{
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return nf(PPB_E_CUDA, "cudaGetDevice failed");
  if (dev < 0 || dev >= (int)PPB_NOALLOC_MAX_DEVICES) return nf(PPB_E_ARG, "device index out of range");
  std::lock_guard<std::mutex> lk(g_mu);
  DeviceSlot& s = g_slots[dev];
  if (!s.ready) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_ppb_noalloc);
    if (e != cudaSuccess || !p) return nf(PPB_E_CUDA, "cudaGetSymbolAddress of the scratch array failed");
    s.base = (unsigned char*)p;
    s.ready = true;
  }
  for (int i = 0; i < (int)PPB_NOALLOC_MAX_MECHS; i++) {
    if (s.mech[i] == t) {
      out->host = t;
      out->device = dev;
      out->blob = s.base;
      out->dm = &s.dm[i];
      return 0;
    }
  }
  int slot = -1;
  for (int i = 0; i < (int)PPB_NOALLOC_MAX_MECHS; i++)
    if (!s.mech[i]) {
      slot = i;
      break;
    }
  const size_t bytes = packed_mechanism_bytes(t);
  const size_t off = (s.tables_used + 255) & ~size_t(255);
  if (slot < 0 || off + bytes > PPB_NOALLOC_TABLES)
    return nf(PPB_E_ARG, "no room left for this mechanism's tables in the scratch array");
  if (pack_mechanism(t, g_stage, sizeof(g_stage), s.base + off, &s.dm[slot]))
    return nf(PPB_E_ARG, "mechanism tables larger than the staging buffer");
  if (cudaMemcpy(s.base + off, g_stage, bytes, cudaMemcpyHostToDevice) != cudaSuccess)
    return nf(PPB_E_CUDA, "copying the mechanism tables to the device failed");
  s.tables_used = off + bytes;
  s.mech[slot] = t;
  out->host = t;
  out->device = dev;
  out->blob = s.base;
  out->dm = &s.dm[slot];
  return 0;
}

__global__ void k_count_failures(const int* status, int n, int* nfail)
{
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < n && status[c] < 0) atomicAdd(nfail, 1);
}
} // namespace

// Largest ncells one call accepts for a mechanism with N species: the scratch
// region holds 2N+1 doubles and 3 ints per cell.
static long noalloc_max_cells(int N)
{
  const size_t per_cell = 8 * (size_t)(2 * N + 1) + 3 * sizeof(int);
  return (long)((PPB_NOALLOC_BYTES - PPB_NOALLOC_TABLES - 1024) / per_cell);
}

extern "C" int ppb_react_flat_device_noalloc(const char* mechanism, const char* integrator, int reactor_type,
                                             const ppb_options* opt, double* rY, double* rYsrc, double* rX,
                                             double* rX_src, double dt_react, int ncells, void* stream, int* nfailed)
{
  const PPBMechTables* t = mechanism ? find_mechanism(mechanism) : nullptr;
  if (!t) return nf(PPB_E_MECH, "unknown mechanism");
  int method;
  if (!integrator || !strcmp(integrator, "ReactorCvode")) {
    method = METHOD_BDF;
  } else if (!strcmp(integrator, "ReactorRK64")) {
    method = METHOD_RK64;
  } else {
    return nf(PPB_E_ARG, "unknown integrator");
  }
  if (reactor_type != PPB_REACTOR_E && reactor_type != PPB_REACTOR_H)
    return nf(PPB_E_ARG, "Wrong reactor type. Choose between 1 (e) or 2 (h).");
  ppb_options o;
  if (opt) {
    o = *opt;
  } else {
    ppb_default_options(&o);
  }
  if (o.max_order < 1 || o.max_order > 5 || o.max_nls_iters < 1 || o.max_steps < 1)
    return nf(PPB_E_ARG, "invalid integrator options");
  if (o.engine != PPB_ENGINE_TUNED)
    return nf(PPB_E_ARG, "the allocation-free path runs the tuned engine only (engine = PPB_ENGINE_TUNED)");
  if (t->nqss > 0) return nf(PPB_E_ARG, "the allocation-free path does not take QSS mechanisms");
  // options this path cannot honour are rejected, never silently dropped
  if (o.eos != PPB_EOS_IDEAL && o.eos != PPB_EOS_SRK) return nf(PPB_E_ARG, "eos must be 0 or 1");
  if (o.eos == PPB_EOS_SRK &&
      (method != METHOD_BDF || reactor_type != PPB_REACTOR_E || o.lu_fp32 || !find_srk(t->name)))
    return nf(PPB_E_ARG, "the SRK EOS needs ReactorCvode, reactor type 1, the FP64 LU and a mechanism with SRK "
                         "parameters");
  if (o.warps_per_block < 0 || o.warps_per_block > 16)
    return nf(PPB_E_ARG, "warps_per_block must be in 0..16 (0: the largest block of <= 8 warps that fits)");
  if (o.team_lanes != 0 && o.team_lanes != 16 && o.team_lanes != 32 && o.team_lanes != 64 && o.team_lanes != 128)
    return nf(PPB_E_ARG, "team_lanes must be 0, 16, 32, 64 or 128");
  if (o.register_budget != 0 && o.register_budget != 1 && o.register_budget != 2)
    return nf(PPB_E_ARG, "register_budget must be 0, 1 or 2");
  if (o.warps_per_block == 0 && ((o.team_lanes != 0 && o.team_lanes != 32) || o.register_budget == 1))
    return nf(PPB_E_ARG, "the allocation-free path does not autotune: give warps_per_block with team_lanes or "
                         "register_budget");
  if (o.eos == PPB_EOS_SRK && ((o.team_lanes != 0 && o.team_lanes != 32) || o.register_budget == 1))
    return nf(PPB_E_ARG, "the SRK kernel runs one warp per cell with <= 128 registers");
  if (ncells < 0 || (ncells > 0 && (!rY || !rYsrc || !rX || !rX_src)))
    return nf(PPB_E_ARG, "invalid arguments");
  const int N = t->nsp, n = N + 1;
  if ((long)ncells > noalloc_max_cells(N)) {
    char msg[200];
    snprintf(msg, sizeof(msg),
             "ncells = %d exceeds the allocation-free path's maximum of %ld cells for %s; split the batch", ncells,
             noalloc_max_cells(N), t->name);
    return nf(PPB_E_ARG, msg);
  }
  if (nfailed) *nfailed = 0;
  if (ncells == 0) return 0;
  DeviceMechanism dm;
  int e = setup(t, &dm);
  if (e) return e;
  cudaStream_t st = (cudaStream_t)stream;
  // scratch layout after the tables region
  unsigned char* p = (unsigned char*)dm.blob + PPB_NOALLOC_TABLES;
  double* soa = (double*)p;
  double* soa_src = soa + (size_t)n * ncells;
  int* status = (int*)(soa_src + (size_t)N * ncells);
  int* cost = status + ncells;
  int* counters = cost + ncells; // [0] work queue, [1] failures
  Options eo{};
  eo.rtol = o.rtol;
  eo.atol = o.atol;
  eo.max_order = o.max_order;
  eo.max_steps = o.max_steps;
  eo.max_nls_iters = o.max_nls_iters;
  eo.max_err_fails = o.max_err_fails;
  eo.jac_eval_freq = o.jac_eval_freq;
  eo.reactor_type = reactor_type;
  eo.lu_fp32 = o.lu_fp32;
  eo.refine_sweeps = o.refine_sweeps;
  eo.rk_guess = o.rk64_nsubsteps_guess;
  eo.rk_min = o.rk64_nsubsteps_min;
  eo.rk_max = o.rk64_nsubsteps_max;
  eo.use_typ_vals = 0;
  if (o.rendezvous_cycles < -1 || o.rendezvous_cycles > 10000000)
    return nf(PPB_E_ARG, "rendezvous_cycles must be -1 or in 0..10000000");
  eo.rendezvous = o.rendezvous_cycles;
  // the launch the allocating path makes for the same options with a fixed
  // block size (no autotuner here: it would need scratch of its own)
  LaunchConfig lc;
  lc.engine = o.engine;
  lc.lu_fp32 = o.lu_fp32;
  lc.persistent = 1;
  lc.rhsv = o.eos == PPB_EOS_SRK ? 1 : 0;
  lc.warps_per_block = o.warps_per_block;
  lc.team = (o.team_lanes == 16 || o.team_lanes == 64 || o.team_lanes == 128) ? o.team_lanes : 32;
  lc.minb = o.register_budget == 1 ? 1 : 2;
  if (lc.team > 32) { // one cell per block of team / 32 warps, <= 255 registers
    lc.warps_per_block = lc.team / 32;
    lc.minb = 1;
  }
  if (lc.warps_per_block <= 0) {
    const size_t cb = team_cell_bytes(t, o.lu_fp32);
    int w = 8;
    while (w > 1 && cb * w > 200 * 1024) w--;
    lc.warps_per_block = w;
  }
  if (react_occupancy(dm, method, lc) < 1)
    return nf(PPB_E_ARG, "this launch configuration is not compiled or does not fit for the mechanism");
  Batch b{};
  b.y = soa;
  b.src = soa_src;
  b.rhoe = rX;
  b.rhoesrc = rX_src;
  b.status = status;
  b.nfe = cost;
  b.ncells = ncells;
  b.ld = ncells;
  if ((e = launch_aos_to_soa(rY, n, soa, ncells, n, ncells, st)) ||
      (e = launch_aos_to_soa(rYsrc, N, soa_src, ncells, N, ncells, st)) ||
      (e = launch_react(dm, eo, method, lc, b, dt_react, counters, st)) ||
      (e = launch_soa_to_aos(soa, ncells, n, rY, n, ncells, st)) ||
      (e = launch_energy_update(rX, rX_src, dt_react, ncells, st)))
    return nf(PPB_E_CUDA, cudaGetErrorString((cudaError_t)e));
  if (cudaMemsetAsync(counters + 1, 0, sizeof(int), st) != cudaSuccess)
    return nf(PPB_E_CUDA, "cudaMemsetAsync failed");
  k_count_failures<<<(ncells + 255) / 256, 256, 0, st>>>(status, ncells, counters + 1);
  if (cudaGetLastError() != cudaSuccess) return nf(PPB_E_CUDA, "launch failed");
  if (!nfailed) return 0;
  int h = 0;
  if (cudaMemcpyAsync(&h, counters + 1, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return nf(PPB_E_CUDA, "reading the failure count failed");
  *nfailed = h;
  return h ? PPB_E_INTEGRATE : 0;
}
