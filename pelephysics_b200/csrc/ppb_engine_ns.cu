// Kernels of the B200 chemistry engine instantiated for one species count
// (compiled once per mechanism size with -DPPB_NS=<N>).
#include "ppb_engine.h"
#include "ppb_work.cuh"

#ifndef PPB_NS
#error "compile with -DPPB_NS=<number of species>"
#endif
#ifndef PPB_PART
#error "compile with -DPPB_PART=<0..4> (the kernel group of this object)"
#endif

namespace ppb {

// ------------------------------------------------------------ react kernels
template <int NS, int TEAM, typename LT, int METHOD, int RHSV = RHS_IDEAL>
__device__ void react_one(const Team<TEAM>& tm, const DevMech& M, const Options& o, Work<LT>& w, const Batch& b,
                          int c, double dt)
{
  const int n = NS + 1;
  if (b.mask && b.mask[c] == -1) {
    if (tm.lane == 0) {
      if (b.status) b.status[c] = ST_SKIPPED;
      if (b.nfe) b.nfe[c] = 0;
    }
    return;
  }
  for (int i = tm.lane; i < n; i += TEAM) {
    const double v = b.y[(size_t)i * b.ld + c];
    w.zn[0][i] = v;
    w.y[i] = v;
    w.src[i] = (i < NS) ? b.src[(size_t)i * b.ld + c] : 0.0;
    if (o.use_typ_vals) w.atolv[i] = b.atolv[i];
  }
  tm.sync();
  const CellIn cin{b.rhoe[c], b.rhoesrc[c]};
  int flag, cost;
  if (METHOD == METHOD_BDF) {
    Bdf<NS, TEAM, LT, NoRec, RHSV> bdf(tm, M, o, w, cin);
    flag = bdf.run(dt);
    cost = bdf.s.nfe;
    if (b.stats && tm.lane == 0) {
      int* st = b.stats + (size_t)c * 7;
      st[0] = bdf.s.nst;
      st[1] = bdf.s.nfe;
      st[2] = bdf.ar.nje;
      st[3] = bdf.ar.nsetups;
      st[4] = bdf.ar.nni;
      st[5] = bdf.ar.netf;
      st[6] = bdf.ar.ncfn;
    }
  } else {
    cost = rk64_cell<TEAM, LT>(tm, M, o, w, cin, dt);
    flag = ST_OK;
    if (b.stats && tm.lane == 0) {
      int* st = b.stats + (size_t)c * 7;
      st[0] = cost;
      st[1] = 6 * cost;
      for (int q = 2; q < 7; q++) st[q] = 0;
    }
  }
  for (int i = tm.lane; i < n; i += TEAM) b.y[(size_t)i * b.ld + c] = w.y[i];
  if (tm.lane == 0) {
    if (b.status) b.status[c] = flag;
    if (b.nfe) b.nfe[c] = cost;
  }
  tm.sync();
}

// plain: one thread per cell, FP64, per-cell arrays in thread-local memory
template <int NS, int METHOD>
__global__ void __launch_bounds__(128) k_react_plain(const __grid_constant__ DevMech M,
                                                     const __grid_constant__ Options o,
                                                     const __grid_constant__ Batch b, double dt)
{
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= b.ncells) return;
  constexpr int n = NS + 1;
  double buf[n * n + 22 * n];
  double A[n * n];
  int piv[n], perm[n];
  BdfArrays ba;
  Work<double> w;
  {
    double* p = buf;
    for (int j = 0; j < 6; j++) {
      w.zn[j] = p;
      p += n;
    }
    w.ewt = p; p += n;
    w.acor = p; p += n;
    w.y = p; p += n;
    w.tempv = p; p += n;
    w.ftemp = p; p += n;
    w.delta = p; p += n;
    w.J = p;
    w.jtmp = p;
    w.jx = nullptr;
    p += n * n;
    w.src = p; p += n;
    w.atolv = p; p += n;
    w.Y = p; p += n;
    w.sc = p; p += n;
    w.g = p; p += n;
    w.wdot = p; p += n;
    w.ei = p; p += n;
    w.h1 = p; p += n;
    w.h2 = p; p += n;
    w.h3 = p; p += n;
    w.qd = nullptr;
    w.A = A;
    w.piv = piv;
    w.perm = perm;
    w.ba = &ba;
  }
  Team<1> tm;
  react_one<NS, 1, double, METHOD>(tm, M, o, w, b, c, dt);
}

// tuned: one team (a warp, or half a warp for small mechanisms) per cell,
// shared-memory workspace, persistent work queue.  MINB is the register
// budget: at least MINB blocks of 256 threads per SM (2: <= 128 registers a
// thread, 1: <= 255).
template <int NS, typename LT, int METHOD, int TEAM>
__device__ __forceinline__ void react_team_body(const Team<TEAM>& tm, const DevMech& M, const Options& o,
                                                const Batch& b, double dt, int* queue, size_t cell_bytes,
                                                int persistent, char* smem, BdfArrays* warp_arrays)
{
  const int team = threadIdx.x / TEAM;
  Work<LT> w;
  carve<LT>(w, smem + (size_t)team * cell_bytes, NS, M.nrxn);
  w.ba = warp_arrays; // one copy of the coefficient arrays per warp of the team
  const int tpb = blockDim.x / TEAM;
  if (persistent) {
    for (;;) {
      int c = 0;
      if (tm.lane == 0) c = atomicAdd(queue, 1);
      c = tm.bcast_int(c, 0);
      if (c >= b.ncells) break;
      react_one<NS, TEAM, LT, METHOD>(tm, M, o, w, b, b.order ? b.order[c] : c, dt);
    }
  } else {
    const int c = blockIdx.x * tpb + team;
    if (c < b.ncells) react_one<NS, TEAM, LT, METHOD>(tm, M, o, w, b, c, dt);
  }
}

// Warp teams carry no block-shared scratch; a multi-warp team gets 16
// doubles for its cross-warp reductions.  MAXT = 384 / 512 are the 12- and
// 16-warp blocks (one block per SM, <= 168 / <= 128 registers) whose warps
// share one rendezvous.
template <int NS, typename LT, int METHOD, int TEAM, int MINB, int RHSV = RHS_IDEAL, int MAXT = 256>
__global__ void __launch_bounds__(MAXT, MINB) k_react_team(const __grid_constant__ DevMech M,
                                                          const __grid_constant__ Options o,
                                                          const __grid_constant__ Batch b, double dt, int* queue,
                                                          size_t cell_bytes, int persistent)
{
  extern __shared__ __align__(16) char smem[];
  if constexpr (TEAM > 32) {
    __shared__ double red[16];
    __shared__ BdfArrays warp_arrays[TEAM / 32];
    const Team<TEAM> tm(red);
    react_team_body<NS, LT, METHOD, TEAM>(tm, M, o, b, dt, queue, cell_bytes, persistent, smem, warp_arrays);
  } else {
    Team<TEAM> tm;
    const int team = threadIdx.x / TEAM;
    Work<LT> w;
    if constexpr (RHSV == RHS_QSS) {
      carve<LT>(w, smem + (size_t)team * cell_bytes, NS, M.nrxn, M.nqss, M.nrq);
    } else {
      carve<LT>(w, smem + (size_t)team * cell_bytes, NS, M.nrxn);
    }
    const int tpb = blockDim.x / TEAM;
    if (persistent) {
      __shared__ int rv[3];
      if (TEAM == 32) w.rv = rendezvous_init(rv, tpb, o.rendezvous);
      for (;;) {
        int c = 0;
        if (tm.lane == 0) c = atomicAdd(queue, 1);
        c = __shfl_sync(tm.mask, c, 0, TEAM);
        if (c >= b.ncells) break;
        react_one<NS, TEAM, LT, METHOD, RHSV>(tm, M, o, w, b, b.order ? b.order[c] : c, dt);
      }
      rendezvous_leave(w.rv);
    } else {
      const int c = blockIdx.x * tpb + team;
      if (c < b.ncells) react_one<NS, TEAM, LT, METHOD, RHSV>(tm, M, o, w, b, c, dt);
    }
  }
}

typedef void (*TeamKernel)(DevMech, Options, Batch, double, int*, size_t, int);

// Lanes per cell of the multi-warp team compiled for a mechanism: one lane
// per species (64 for 33..64 species, 128 for 65..128), 0 for <= 21 species.
template <int NS>
constexpr int big_team()
{
  return NS <= 21 ? 0 : NS <= 64 ? 64 : 128;
}

// The compiled variants: 32 lanes per cell with both register budgets for
// the FP64 BDF kernel; 16 lanes per cell as well for mechanisms of at most
// 21 species, and a multi-warp team (one cell per block, one lane per
// species) for larger ones.  They are compiled in five parts (PPB_PART 0..4,
// one object each, built in parallel); each part returns the kernels it holds
// and nullptr for the others:
//   0: FP64 BDF, 32 lanes, 8 warps (<= 128 and <= 255 registers)
//   1: FP64 BDF, 32 lanes, 12 and 16 warps per block (one block per SM)
//   2: the multi-warp teams (FP64 and FP32 BDF, RK64); the SRK kernel at 16
//      warps per block (<= 21 species)
//   3: FP32 BDF and RK64 with 32 lanes, the 16-lane variants, the SRK kernel
//      (<= 8 warps per block)
//   4: FP32 BDF, 32 lanes, 12 and 16 warps per block
// Species counts compiled for a QSS mechanism only (transported species of
// CH4_lean_qss 13, LuEthylene_qss 22, C1-C2-NO_qss 39): the QSS kernel at
// <= 8 warps per block (part 3) and, for <= 21 species, at 16 (part 1); no
// other variant.
template <int NS>
constexpr bool qss_only()
{
  return NS == 13 || NS == 22 || NS == 39;
}

template <int NS>
static TeamKernel team_kernel_part(int method, bool fp32, int team, int minb, int srk, int wpb)
{
  constexpr bool small = NS <= 21;
  constexpr int P = PPB_PART;
  // the QSS reactor (srk == RHS_QSS): FP64 BDF, one warp per cell, <= 128
  // registers, difference-quotient Jacobian
  if constexpr (qss_only<NS>()) {
    if (srk != RHS_QSS || method != METHOD_BDF || fp32 || team != 32 || minb != 2) return nullptr;
    if constexpr (P == 3)
      return wpb <= 8 ? (TeamKernel)k_react_team<NS, double, METHOD_BDF, 32, 2, RHS_QSS> : nullptr;
    // 16 warps per block, one block per SM (<= 21 species: sixteen cell
    // workspaces fit one SM's shared memory), all under one rendezvous
    if constexpr (P == 1 && small)
      return wpb == 16 ? (TeamKernel)k_react_team<NS, double, METHOD_BDF, 32, 1, RHS_QSS, 512> : nullptr;
    return nullptr;
  } else {
    if (srk == RHS_QSS) return nullptr;
    // 12 or 16 warps per block (one block per SM: <= 168 or <= 128 registers):
    // the FP64 BDF warp-per-cell kernel; the SRK e-reactor at 16
    if (wpb > 8) {
      if (method != METHOD_BDF || team != 32 || minb != 2) return nullptr;
      if (srk) {
        if constexpr (P == 2 && small)
          return (!fp32 && wpb == 16) ? (TeamKernel)k_react_team<NS, double, METHOD_BDF, 32, 1, RHS_SRK, 512>
                                      : nullptr;
        return nullptr;
      }
      if constexpr (P == 1) {
        if (fp32) return nullptr;
        if (wpb == 16) return (TeamKernel)k_react_team<NS, double, METHOD_BDF, 32, 1, RHS_IDEAL, 512>;
        if (wpb == 12) return (TeamKernel)k_react_team<NS, double, METHOD_BDF, 32, 1, RHS_IDEAL, 384>;
      }
      if constexpr (P == 4) {
        if (!fp32) return nullptr;
        if (wpb == 16) return (TeamKernel)k_react_team<NS, float, METHOD_BDF, 32, 1, RHS_IDEAL, 512>;
        if (wpb == 12) return (TeamKernel)k_react_team<NS, float, METHOD_BDF, 32, 1, RHS_IDEAL, 384>;
      }
      return nullptr;
    }
    // the SRK e-reactor: FP64 BDF, one warp per cell, <= 128 registers
    if (srk) {
      if constexpr (P == 3)
        return (method == METHOD_BDF && !fp32 && team == 32 && minb == 2)
                 ? (TeamKernel)k_react_team<NS, double, METHOD_BDF, 32, 2, RHS_SRK>
                 : nullptr;
      return nullptr;
    }
    if (team > 32) {
      if constexpr (big_team<NS>() > 0 && P == 2) {
        constexpr int BT = big_team<NS>();
        if (team != BT) return nullptr;
        if (method == METHOD_RK64) return (TeamKernel)k_react_team<NS, double, METHOD_RK64, BT, 1>;
        if (fp32) return (TeamKernel)k_react_team<NS, float, METHOD_BDF, BT, 1>;
        return (TeamKernel)k_react_team<NS, double, METHOD_BDF, BT, 1>;
      }
      return nullptr;
    }
    if (team == 16 && !small) return nullptr;
    if constexpr (P == 3) {
      if (method == METHOD_RK64) {
        if (team == 16) return small ? (TeamKernel)k_react_team<NS, double, METHOD_RK64, (small ? 16 : 32), 2> : nullptr;
        return (TeamKernel)k_react_team<NS, double, METHOD_RK64, 32, 2>;
      }
      if (fp32) {
        if (team == 16) return small ? (TeamKernel)k_react_team<NS, float, METHOD_BDF, (small ? 16 : 32), 2> : nullptr;
        return (TeamKernel)k_react_team<NS, float, METHOD_BDF, 32, 2>;
      }
      if (team == 16) {
        if (!small) return nullptr;
        return minb == 1 ? (TeamKernel)k_react_team<NS, double, METHOD_BDF, (small ? 16 : 32), 1>
                         : (TeamKernel)k_react_team<NS, double, METHOD_BDF, (small ? 16 : 32), 2>;
      }
      return nullptr;
    }
    if constexpr (P == 0) {
      if (method == METHOD_RK64 || fp32 || team == 16) return nullptr;
      return minb == 1 ? (TeamKernel)k_react_team<NS, double, METHOD_BDF, 32, 1>
                       : (TeamKernel)k_react_team<NS, double, METHOD_BDF, 32, 2>;
    }
    return nullptr;
  }
}

#define PPB_CAT2(a, b) a##b
#define PPB_CAT(a, b) PPB_CAT2(a, b)
#define PPB_CAT4(a, b, c, d) PPB_CAT(PPB_CAT(a, b), PPB_CAT(c, d))
// this part's kernels, under a name of its own
TeamKernel PPB_CAT4(team_kernel_, PPB_NS, _p, PPB_PART)(int method, bool fp32, int team, int minb, int srk, int wpb)
{
  return team_kernel_part<PPB_NS>(method, fp32, team, minb, srk, wpb);
}

#if PPB_PART == 0
TeamKernel PPB_CAT4(team_kernel_, PPB_NS, _p, 1)(int, bool, int, int, int, int);
TeamKernel PPB_CAT4(team_kernel_, PPB_NS, _p, 2)(int, bool, int, int, int, int);
TeamKernel PPB_CAT4(team_kernel_, PPB_NS, _p, 3)(int, bool, int, int, int, int);
TeamKernel PPB_CAT4(team_kernel_, PPB_NS, _p, 4)(int, bool, int, int, int, int);

template <int NS>
static TeamKernel team_kernel(int method, bool fp32, int team, int minb, int srk, int wpb)
{
  TeamKernel (*parts[5])(int, bool, int, int, int, int) = {
    PPB_CAT4(team_kernel_, PPB_NS, _p, 0), PPB_CAT4(team_kernel_, PPB_NS, _p, 1),
    PPB_CAT4(team_kernel_, PPB_NS, _p, 2), PPB_CAT4(team_kernel_, PPB_NS, _p, 3),
    PPB_CAT4(team_kernel_, PPB_NS, _p, 4)};
  for (auto f : parts)
    if (TeamKernel k = f(method, fp32, team, minb, srk, wpb)) return k;
  return nullptr;
}

// the plain engine's kernels (part 3)
void PPB_CAT4(launch_plain_, PPB_NS, _p, 3)(const DevMech& M, const Options& o, int method, Batch b, double dt,
                                            cudaStream_t st);

template <int NS>
static int launch_react_ns(const DeviceMechanism& m, const Options& o, int method, const LaunchConfig& lc,
                           Batch b, double dt, int* queue, cudaStream_t st)
{
  const DevMech& M = *m.dm;
  if (b.ncells <= 0) return 0;
  if (lc.engine == ENGINE_PLAIN) {
    if constexpr (qss_only<NS>()) return (int)cudaErrorNotSupported;
    PPB_CAT4(launch_plain_, PPB_NS, _p, 3)(M, o, method, b, dt, st);
    return (int)cudaGetLastError();
  }
  const bool fp32 = lc.lu_fp32 && method == METHOD_BDF;
  const int team = (lc.team == 16 || lc.team > 32) ? lc.team : 32;
  // a multi-warp team is one block
  const int wpb = team > 32 ? team / 32 : (lc.warps_per_block > 0 ? lc.warps_per_block : 4);
  TeamKernel kern = team_kernel<NS>(method, fp32, team, lc.minb, lc.rhsv, wpb);
  if (!kern) return (int)cudaErrorInvalidConfiguration;
  const int tpb = team > 32 ? 1 : wpb * (32 / team); // cells per block
  const size_t cb = fp32 ? team_bytes<float>(M.nsp, M.nrxn, M.nqss, M.nrq)
                         : team_bytes<double>(M.nsp, M.nrxn, M.nqss, M.nrq);
  const size_t shm = cb * tpb;
  cudaError_t e = cudaFuncSetAttribute((const void*)kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm);
  if (e != cudaSuccess) return (int)e;
  int blocks;
  if (lc.persistent) {
    int dev = 0, nsm = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)kern, wpb * 32, shm);
    if (e != cudaSuccess) return (int)e;
    if (per_sm < 1) return (int)cudaErrorInvalidConfiguration;
    blocks = nsm * per_sm;
    const int need = (b.ncells + tpb - 1) / tpb;
    if (blocks > need) blocks = need;
    e = cudaMemsetAsync(queue, 0, sizeof(int), st);
    if (e != cudaSuccess) return (int)e;
  } else {
    blocks = (b.ncells + tpb - 1) / tpb;
  }
  Options ob = o;
  ob.rendezvous = (o.rendezvous < 0 && lc.rv > 0) ? lc.rv : rendezvous_bound(o.rendezvous, wpb);
  kern<<<blocks, wpb * 32, shm, st>>>(M, ob, b, dt, queue, cb, lc.persistent);
  return (int)cudaGetLastError();
}

// Resident cells per SM of a configuration (0: does not fit).
template <int NS>
static int occupancy_ns(const DevMech& M, int method, const LaunchConfig& lc)
{
  const bool fp32 = lc.lu_fp32 && method == METHOD_BDF;
  const int team = (lc.team == 16 || lc.team > 32) ? lc.team : 32;
  const int wpb = team > 32 ? team / 32 : (lc.warps_per_block > 0 ? lc.warps_per_block : 4);
  TeamKernel kern = team_kernel<NS>(method, fp32, team, lc.minb, lc.rhsv, wpb);
  if (!kern) return 0;
  const int tpb = team > 32 ? 1 : wpb * (32 / team);
  const size_t cb = fp32 ? team_bytes<float>(M.nsp, M.nrxn, M.nqss, M.nrq)
                         : team_bytes<double>(M.nsp, M.nrxn, M.nqss, M.nrq);
  const size_t shm = cb * tpb;
  int dev = 0, smem_max = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&smem_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if (shm > (size_t)smem_max) return 0;
  if (cudaFuncSetAttribute((const void*)kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm) != cudaSuccess)
    return 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)kern, wpb * 32, shm) != cudaSuccess) return 0;
  return per_sm * tpb;
}

template <int TEAM, int PER>
__global__ void k_ajacobian(DevMech M, const double* sc, const double* T, int consP, double* J, int ncells)
{
  extern __shared__ __align__(16) double psm[];
  Team<TEAM> tm;
  const int N = M.nsp, n = N + 1;
  const int per_block = blockDim.x / TEAM;
  const int slot = threadIdx.x / TEAM;
  const int c = blockIdx.x * per_block + slot;
  if (TEAM == 1 && c >= ncells) return;
  const int cc = c < ncells ? c : ncells - 1;
  double local[8 * 96];
  double* base = (TEAM == 1) ? local : psm + (size_t)slot * point_doubles(N, M.nrxn, true);
  double* s_sc = base;
  double* s_g = base + n;
  double* s_w = base + 2 * n;
  double* h1 = base + 3 * n;
  double* h2 = base + 4 * n;
  double* h3 = base + 5 * n;
  double* h4 = base + 6 * n;
  // serial: accumulate straight into the output; team: into shared memory
  double* s_J = (TEAM == 1) ? J + (size_t)cc * n * n : base + 8 * n + 5 * M.nrxn;
  for (int s = tm.lane; s < N; s += TEAM) s_sc[s] = sc[(size_t)cc * N + s];
  if (tm.lane == 0) s_sc[N] = 1.0; // padding slot of the packed reaction records
  tm.sync();
  RateScratch rs{s_sc, s_g, TEAM > 1 ? base + 8 * n : nullptr, TEAM > 1 ? base + 8 * n + M.nrxn : nullptr};
  ajacobian<TEAM, PER>(tm, M, s_J, s_sc, T[cc], consP, rs, s_w, h1, h2, h3, h4);
  if (TEAM > 1 && c < ncells)
    for (int i = tm.lane; i < n * n; i += TEAM) J[(size_t)c * n * n + i] = s_J[i];
}

template <int NS>
static int launch_ajac_ns(const DevMech& M, const double* sc, const double* T, int consP, double* J, int ncells,
                          int team, cudaStream_t st)
{
  if (team == 1) {
    const int threads = 64;
    k_ajacobian<1, NS><<<(ncells + threads - 1) / threads, threads, 0, st>>>(M, sc, T, consP, J, ncells);
  } else {
    const int cells_per_block = 2;
    const size_t shm = point_doubles(M.nsp, M.nrxn, true) * 8 * cells_per_block;
    auto k = k_ajacobian<32, (NS + 31) / 32>;
    cudaError_t e = cudaFuncSetAttribute((const void*)k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm);
    if (e != cudaSuccess) return (int)e;
    k<<<(ncells + cells_per_block - 1) / cells_per_block, 32 * cells_per_block, shm, st>>>(M, sc, T, consP, J,
                                                                                          ncells);
  }
  return (int)cudaGetLastError();
}


int PPB_CAT(launch_react_, PPB_NS)(const DeviceMechanism& m, const Options& o, int method, const LaunchConfig& lc,
                                   Batch b, double dt, int* queue, cudaStream_t st)
{
  return launch_react_ns<PPB_NS>(m, o, method, lc, b, dt, queue, st);
}
int PPB_CAT(react_occupancy_, PPB_NS)(const DevMech& M, int method, const LaunchConfig& lc)
{
  return occupancy_ns<PPB_NS>(M, method, lc);
}
int PPB_CAT(launch_ajacobian_, PPB_NS)(const DevMech& M, const double* sc, const double* T, int consP, double* J,
                                       int ncells, int team, cudaStream_t st)
{
  // a QSS mechanism has no analytical Jacobian here
  if constexpr (qss_only<PPB_NS>()) return (int)cudaErrorNotSupported;
  else return launch_ajac_ns<PPB_NS>(M, sc, T, consP, J, ncells, team, st);
}
#endif // PPB_PART == 0

#if PPB_PART == 3
void PPB_CAT4(launch_plain_, PPB_NS, _p, 3)(const DevMech& M, const Options& o, int method, Batch b, double dt,
                                            cudaStream_t st)
{
  if constexpr (!qss_only<PPB_NS>()) {
    const int threads = 128;
    const int blocks = (b.ncells + threads - 1) / threads;
    if (method == METHOD_BDF)
      k_react_plain<PPB_NS, METHOD_BDF><<<blocks, threads, 0, st>>>(M, o, b, dt);
    else
      k_react_plain<PPB_NS, METHOD_RK64><<<blocks, threads, 0, st>>>(M, o, b, dt);
  }
}
#endif

#if defined(PPB_PHASE_TIMERS)
// this object's copy of the phase counters (each part has its own)
int PPB_CAT4(phase_cycles_, PPB_NS, _p, PPB_PART)(unsigned long long* out, int reset)
{
  cudaError_t e = cudaMemcpyFromSymbol(out, g_phase_cycles, sizeof(unsigned long long) * PH_COUNT);
  if (e == cudaSuccess && reset) {
    unsigned long long z[PH_COUNT] = {};
    e = cudaMemcpyToSymbol(g_phase_cycles, z, sizeof(z));
  }
  return (int)e;
}
#endif
} // namespace ppb
