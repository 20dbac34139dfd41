// The ARKODE-style explicit reactor kernel for one species count (compiled
// with -DPPB_NS=<N>); algorithm and batch coupling in ppb_ark.cuh.
//
// One cooperative launch integrates the batch: grid = every co-resident
// block, a warp per cell at a time, cells assigned c = warp, warp + W, ...
// for the whole call (so a cell's data is only ever touched by one warp and
// needs no cross-block visibility).  Per step each warp runs all stages of
// each of its cells with the cell's stage vectors in shared memory, writes
// y+ to the cell-major scratch and adds its squared weighted errors to a
// lane-local sum; the block sums the warps in order, one bounded grid
// barrier publishes the block sums, and every block adds them in the same
// order -- identical bits, identical decisions everywhere.
#include <cfloat>

#include "ppb_ark.cuh"
#include "ppb_engine.h"

#ifndef PPB_NS
#error "compile with -DPPB_NS=<species count>"
#endif

namespace ppb {
namespace {

constexpr int NS = PPB_NS;
constexpr int ARK_THREADS = 256;
constexpr int ARK_WARPS = ARK_THREADS / 32;

// per-warp shared workspace, doubles: y, yst, src, Y, sc, g, wdot, ei (n
// each), the stage vectors k[S][n], the reaction scratch qd[R]
__host__ __device__ inline size_t ark_warp_doubles(int N, int R, int S)
{
  const size_t n = N + 1;
  return n * (8 + (size_t)S) + (size_t)R;
}

struct ArkWs {
  double *y, *yst, *src, *Y, *sc, *g, *wdot, *ei, *k, *qd;
};

__device__ inline ArkWs ark_carve(double* p, int N, int R, int S)
{
  const int n = N + 1;
  ArkWs w;
  w.y = p; p += n;
  w.yst = p; p += n;
  w.src = p; p += n;
  w.Y = p; p += n;
  w.sc = p; p += n;
  w.g = p; p += n;
  w.wdot = p; p += n;
  w.ei = p; p += n;
  w.k = p; p += (size_t)S * n;
  w.qd = p;
  return w;
}

__device__ __forceinline__ void ark_f(const Team<32>& tm, const DevMech& M, int rtype, double t, const double* y,
                                      double* ydot, double rhoe, double rhoesrc, const ArkWs& w)
{
  reactor_rhs<32>(tm, M, rtype, t, y, ydot, rhoe, rhoesrc, w.src, w.Y, w.sc, w.g, w.qd, w.wdot, w.ei);
}

__device__ __forceinline__ double ark_atol(const ArkParams& P, const ArkBuffers& B, int i)
{
  return B.atolv ? B.atolv[i] : P.atol;
}

__global__ void __launch_bounds__(ARK_THREADS) k_ark(DevMech M, ArkParams P, ArkBuffers B)
{
  extern __shared__ __align__(16) double ark_sm[];
  __shared__ double wred[ARK_WARPS];
  __shared__ double gval;
  __shared__ ErkTable tb;
  Team<32> tm;
  for (int i = threadIdx.x; i < (int)(sizeof(ErkTable) / sizeof(double)); i += blockDim.x)
    reinterpret_cast<double*>(&tb)[i] = reinterpret_cast<const double*>(&P.tab)[i];
  __syncthreads();
  const int N = M.nsp, n = N + 1, R = M.nrxn, S = tb.stages;
  const int warp = threadIdx.x >> 5;
  const int nwarps = blockDim.x >> 5;
  const int gw = blockIdx.x * nwarps + warp;
  const int GW = gridDim.x * nwarps;
  const int rtype = P.reactor_type;
  ArkWs w = ark_carve(ark_sm + (size_t)warp * ark_warp_doubles(N, R, S), N, R, S);
  int par = 0;
  int* tmo = &B.info->barrier_timeout;
  bool broken = false;

  // Sum (or max) over every lane of the grid; the same bits in every block.
  auto grid_reduce = [&](double v, bool mx) -> double {
    v = mx ? tm.max(v) : tm.sum(v);
    if (tm.lane == 0) wred[warp] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
      double s = wred[0];
      for (int i = 1; i < nwarps; i++) s = mx ? fmax(s, wred[i]) : s + wred[i];
      B.partial[par * gridDim.x + blockIdx.x] = s;
    }
    if (!ark_grid_barrier(B.bar, tmo, P.barrier_ns)) {
      broken = true;
      return 0.0;
    }
    if (warp == 0) {
      double s = mx ? 0.0 : 0.0;
      for (int i = tm.lane; i < (int)gridDim.x; i += 32) {
        const double x = __ldcg(B.partial + par * gridDim.x + i);
        s = mx ? fmax(s, x) : s + x;
      }
      s = mx ? tm.max(s) : tm.sum(s);
      if (tm.lane == 0) gval = s;
    }
    __syncthreads();
    const double r = gval;
    __syncthreads();
    par ^= 1;
    return r;
  };
  auto active = [&](int c) { return !(B.mask && B.mask[c] == -1); };
  auto cell_y = [&](double* base, int c) { return base + (size_t)c * n; };

  // ---- load the batch (species-major -> cell-major), f(0, y0), h0 bound
  double cnt = 0.0, hub_inv = 0.0;
  for (int c = gw; c < B.ncells; c += GW) {
    double* y0 = cell_y(B.Y0, c);
    for (int i = tm.lane; i < n; i += 32) y0[i] = B.ysoa[(size_t)i * B.ld + c];
    for (int i = tm.lane; i < N; i += 32) B.S[(size_t)c * N + i] = B.srcsoa[(size_t)i * B.ld + c];
    if (!active(c)) continue;
    if (tm.lane == 0) cnt += 1.0;
    for (int i = tm.lane; i < n; i += 32) w.y[i] = y0[i];
    for (int i = tm.lane; i < N; i += 32) w.src[i] = B.S[(size_t)c * N + i];
    tm.sync();
    ark_f(tm, M, rtype, 0.0, w.y, w.k, B.rhoe[c], B.rhoesrc[c], w);
    double* f0 = cell_y(B.F0, c);
    for (int i = tm.lane; i < n; i += 32) {
      f0[i] = w.k[i];
      const double ewinv = P.rtol * fabs(w.y[i]) + ark_atol(P, B, i);
      hub_inv = fmax(hub_inv, fabs(w.k[i]) / (0.1 * fabs(w.y[i]) + ewinv));
    }
    tm.sync();
  }
  const double nact = grid_reduce(cnt, false);
  if (broken) return;
  hub_inv = grid_reduce(hub_inv, true);
  if (broken) return;
  const double ntot = nact * n;
  long long nfe = nact > 0.0 ? 1 : 0, nst = 0, netf = 0, attempts = 0;
  int status = ST_OK;
  double t = 0.0, h = 0.0;
  const double tout = P.tout;

  // wrms over the batch of (v - f0) / hg at y0 + hg f0: the second-derivative
  // estimate of the initial-step heuristic
  auto ydd_norm = [&](double hg) -> double {
    double acc = 0.0;
    for (int c = gw; c < B.ncells; c += GW) {
      if (!active(c)) continue;
      const double* y0 = cell_y(B.Y0, c);
      const double* f0 = cell_y(B.F0, c);
      for (int i = tm.lane; i < n; i += 32) w.yst[i] = hg * f0[i] + y0[i];
      for (int i = tm.lane; i < N; i += 32) w.src[i] = B.S[(size_t)c * N + i];
      tm.sync();
      ark_f(tm, M, rtype, hg, w.yst, w.k, B.rhoe[c], B.rhoesrc[c], w);
      for (int i = tm.lane; i < n; i += 32) {
        const double ewt = 1.0 / (P.rtol * fabs(y0[i]) + ark_atol(P, B, i));
        const double x = (w.k[i] - f0[i]) * (1.0 / hg) * ewt;
        acc += x * x;
      }
      tm.sync();
    }
    return sqrt(grid_reduce(acc, false) / ntot);
  };

  if (nact > 0.0) {
    // ---- initial step (the CVODE/ARKODE estimate)
    const double tround = DBL_EPSILON * tout;
    if (!(tout > 0.0) || tout < 2.0 * tround) {
      status = ST_TOO_CLOSE;
    } else {
      const double hlb = 100.0 * tround;
      double hub = 0.1 * tout;
      if (hub * hub_inv > 1.0) hub = 1.0 / hub_inv;
      double hg = sqrt(hlb * hub);
      if (hub < hlb) {
        h = hg;
      } else {
        double hnew = hg;
        for (int count1 = 1; count1 <= 4; count1++) {
          const double yddnrm = ydd_norm(hg);
          if (broken) return;
          nfe++;
          hnew = (yddnrm * hub * hub > 2.0) ? sqrt(2.0 / yddnrm) : sqrt(hg * hub);
          if (count1 == 4) break;
          const double hrat = hnew / hg;
          if (hrat > 0.5 && hrat < 2.0) break;
          if (count1 > 1 && hrat > 2.0) {
            hnew = hg;
            break;
          }
          hg = hnew;
        }
        h = 0.5 * hnew;
        if (h < hlb) h = hlb;
        if (h > hub) h = hub;
      }
    }
  }

  // ---- steps
  double* Yc = B.Y0; // y_n
  double* Yn = B.Y1; // y_{n+1} of the attempt
  double* Fc = B.F0; // f(t_n, y_n) (valid when f_ok)
  double* Fn = B.F1; // FSAL: f(t_{n+1}, y_{n+1})
  bool f_ok = true;  // f at y_n is stored in Fc
  double ep = 0.0, epp = 0.0, etamax = ArkAdapt::etamx1;
  int nacc = 0;
  bool done = (nact == 0.0) || status != ST_OK;
  if (nact == 0.0) t = tout;
  while (!done) {
    if (nst >= P.max_steps) {
      status = ST_TOO_MUCH_WORK;
      break;
    }
    int nef = 0;
    bool accepted = false;
    while (!accepted) {
      attempts++;
      double acc = 0.0;
      for (int c = gw; c < B.ncells; c += GW) {
        if (!active(c)) continue;
        const double* y0 = cell_y(Yc, c);
        double* f0 = cell_y(Fc, c);
        for (int i = tm.lane; i < n; i += 32) w.y[i] = y0[i];
        for (int i = tm.lane; i < N; i += 32) w.src[i] = B.S[(size_t)c * N + i];
        tm.sync();
        if (f_ok) {
          for (int i = tm.lane; i < n; i += 32) w.k[i] = f0[i];
        } else {
          ark_f(tm, M, rtype, t, w.y, w.k, B.rhoe[c], B.rhoesrc[c], w);
          for (int i = tm.lane; i < n; i += 32) f0[i] = w.k[i];
        }
        tm.sync();
        for (int s = 1; s < S; s++) {
          for (int i = tm.lane; i < n; i += 32) {
            double a = 0.0;
            for (int j = 0; j < s; j++) a += tb.A[s][j] * w.k[(size_t)j * n + i];
            w.yst[i] = w.y[i] + h * a;
          }
          tm.sync();
          ark_f(tm, M, rtype, t + tb.c[s] * h, w.yst, w.k + (size_t)s * n, B.rhoe[c], B.rhoesrc[c], w);
        }
        double* y1 = cell_y(Yn, c);
        for (int i = tm.lane; i < n; i += 32) {
          double a = 0.0, e = 0.0;
          for (int j = 0; j < S; j++) {
            const double kj = w.k[(size_t)j * n + i];
            a += tb.b[j] * kj;
            e += (tb.b[j] - tb.d[j]) * kj;
          }
          y1[i] = w.y[i] + h * a;
          const double ewt = 1.0 / (P.rtol * fabs(w.y[i]) + ark_atol(P, B, i));
          const double x = h * e * ewt;
          acc += x * x;
        }
        if (P.fsal) {
          double* f1 = cell_y(Fn, c);
          for (int i = tm.lane; i < n; i += 32) f1[i] = w.k[(size_t)(S - 1) * n + i];
        }
        tm.sync();
      }
      const double dsm = sqrt(grid_reduce(acc, false) / ntot);
      if (broken) return;
      nfe += (f_ok ? 0 : 1) + (S - 1);
      f_ok = true; // Fc holds f(t_n, y_n) now
      const int ord = tb.q;
      if (dsm <= 1.0) {
        const double eta = ark_eta(P.controller, ord, h, dsm, ep, epp, nacc, etamax);
        accepted = true;
        t += h;
        nst++;
        nacc++;
        epp = ep;
        ep = ArkAdapt::bias * dsm;
        double* tmp = Yc;
        Yc = Yn;
        Yn = tmp;
        if (P.fsal) {
          tmp = Fc;
          Fc = Fn;
          Fn = tmp;
        } else {
          tmp = Fc; // keep f(t_n, y_n) for the dense output in Fn
          Fc = Fn;
          Fn = tmp;
          f_ok = false;
        }
        if (t >= tout) {
          done = true;
        } else {
          h *= eta;
          etamax = ArkAdapt::growth;
        }
      } else {
        netf++;
        nef++;
        if (nef >= ArkAdapt::max_nef) {
          status = ST_ERR_FAILURE;
          done = true;
          break;
        }
        double eta = fmin(ark_eta(P.controller, ord, h, dsm, ep, epp, nacc, etamax), 1.0);
        etamax = 1.0;
        if (nef >= ArkAdapt::small_nef) eta = fmin(eta, ArkAdapt::etamxf);
        h *= eta;
        if (t + h == t) {
          status = ST_ERR_FAILURE;
          done = true;
          break;
        }
      }
    }
  }

  // ---- output: the cubic Hermite interpolant at tout after a step past it,
  // else the last state reached
  const bool interp = status == ST_OK && nact > 0.0 && t > tout;
  const double t_out = status == ST_OK ? tout : t;
  if (interp) {
    // y_n in Yn, f(t_n, y_n) in Fn; y_{n+1} in Yc, f(t_{n+1}) in Fc if FSAL
    const double hs = h, theta = (tout - (t - hs)) / hs;
    const double t2 = theta * theta, t3 = t2 * theta;
    const double h00 = 2.0 * t3 - 3.0 * t2 + 1.0, h10 = t3 - 2.0 * t2 + theta;
    const double h01 = -2.0 * t3 + 3.0 * t2, h11 = t3 - t2;
    for (int c = gw; c < B.ncells; c += GW) {
      if (!active(c)) continue;
      const double* ya = cell_y(Yn, c);
      const double* fa = cell_y(Fn, c);
      const double* yb = cell_y(Yc, c);
      for (int i = tm.lane; i < n; i += 32) w.y[i] = yb[i];
      for (int i = tm.lane; i < N; i += 32) w.src[i] = B.S[(size_t)c * N + i];
      tm.sync();
      const double* fb;
      if (P.fsal) {
        fb = cell_y(Fc, c);
      } else {
        ark_f(tm, M, rtype, t, w.y, w.k, B.rhoe[c], B.rhoesrc[c], w);
        fb = w.k;
      }
      for (int i = tm.lane; i < n; i += 32)
        B.ysoa[(size_t)i * B.ld + c] = h00 * ya[i] + h10 * hs * fa[i] + h01 * yb[i] + h11 * hs * fb[i];
      tm.sync();
    }
    if (!P.fsal) nfe++;
  } else if (nact > 0.0) {
    for (int c = gw; c < B.ncells; c += GW) {
      if (!active(c)) continue;
      const double* yb = cell_y(Yc, c);
      for (int i = tm.lane; i < n; i += 32) B.ysoa[(size_t)i * B.ld + c] = yb[i];
    }
  }
  // per-cell flags and counters; the energy update with the time reached
  for (int c = gw; c < B.ncells; c += GW) {
    const bool a = active(c);
    if (tm.lane == 0) {
      if (B.status) B.status[c] = a ? status : ST_SKIPPED;
      if (B.nfe) B.nfe[c] = a ? (int)nfe : 0;
      if (B.rhoe_out) B.rhoe_out[c] = B.rhoe[c] + t_out * B.rhoesrc[c];
    }
    if (B.stats && tm.lane < 7) {
      const long long v[7] = {nst, nfe, 0, 0, 0, netf, 0};
      B.stats[(size_t)c * 7 + tm.lane] = a ? (int)v[tm.lane] : 0;
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    B.info->t = t_out;
    B.info->h = h;
    B.info->nst = nst;
    B.info->nfe = nfe;
    B.info->netf = netf;
    B.info->attempts = attempts;
    B.info->status = status;
  }
}

} // namespace

#define PPB_CAT2(a, b) a##b
#define PPB_CAT(a, b) PPB_CAT2(a, b)

int PPB_CAT(launch_ark_, PPB_NS)(const DeviceMechanism& m, const ArkParams& P, const ArkBuffers& B,
                                               int* grid_out, cudaStream_t st)
{
  const DevMech& M = *m.dm;
  const size_t shm = ark_warp_doubles(M.nsp, M.nrxn, P.tab.stages) * 8 * ARK_WARPS;
  cudaError_t e = cudaFuncSetAttribute((const void*)k_ark, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm);
  if (e != cudaSuccess) return (int)e;
  int dev = 0, nsm = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)k_ark, ARK_THREADS, shm);
  if (e != cudaSuccess) return (int)e;
  if (per_sm < 1) return (int)cudaErrorInvalidConfiguration;
  int grid = nsm * per_sm;
  const int need = (B.ncells + ARK_WARPS - 1) / ARK_WARPS;
  if (grid > need) grid = need;
  if (grid_out && *grid_out > 0 && *grid_out < grid) grid = *grid_out; // caller's partial buffer bound
  if (grid_out) *grid_out = grid;
  e = cudaMemsetAsync(B.bar, 0, 2 * sizeof(unsigned), st);
  if (e != cudaSuccess) return (int)e;
  DevMech Mv = M;
  ArkParams Pv = P;
  ArkBuffers Bv = B;
  void* args[] = {&Mv, &Pv, &Bv};
  e = cudaLaunchCooperativeKernel((const void*)k_ark, dim3(grid), dim3(ARK_THREADS), args, shm, st);
  return (int)e;
}

} // namespace ppb
