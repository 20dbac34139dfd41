// Per-cell reactor model and stiff integrators for the B200 engine.
//
//  * reactor_rhs  : the reference's fKernelSpec (Source/Reactions/
//                   ReactorUtils.H:358-415) over the Fuego EOS wrappers
//  * reactor_jac  : the CPU dense analytical Jacobian callback
//                   (Source/Reactions/ReactorCvodeJacobian.cpp:86-152)
//  * bdf_cell     : variable-order (1..5) BDF in Nordsieck form with
//                   fixed-leading-coefficient coefficients, WRMS local error
//                   test, step/order selection and a modified Newton on
//                   I - gamma J: the CVODE algorithm with the options the
//                   reference sets (ReactorCvode.cpp:230-503)
//  * rk64_cell    : ReactorRK64.cpp:73-144
//
// One team of TEAM lanes integrates one cell; every lane holds the scalar
// integrator state, vectors are lane-strided over team-shared memory.
#pragma once
#include "ppb_mech.cuh"
#include "ppb_srk.cuh"

namespace ppb {

// Optional per-phase cycle counters (compile with -DPPB_PHASE_TIMERS): each
// team accumulates clock64() deltas per phase and adds them to
// g_phase_cycles at the end of a cell.  Off in the shipped library.
enum Phase { PH_RHS = 0, PH_JAC, PH_LU, PH_SOLVE, PH_NEWTON, PH_STEP, PH_TOTAL, PH_COUNT };
#ifdef PPB_PHASE_TIMERS
static __device__ unsigned long long g_phase_cycles[PH_COUNT]; // one copy per translation unit
#define PPB_TIC(ph) const long long _tic_##ph = clock64()
#define PPB_TOC(ph) s.phase[ph] += clock64() - _tic_##ph
#else
#define PPB_TIC(ph)
#define PPB_TOC(ph)
#endif

enum { ST_OK = 0, ST_TOO_MUCH_WORK = -1, ST_ERR_FAILURE = -3, ST_CONV_FAILURE = -4,
       ST_LSETUP_FAIL = -6, ST_TOO_CLOSE = -27, ST_SKIPPED = 1 };

struct Options {
  double rtol, atol;
  int max_order, max_steps, max_nls_iters, max_err_fails, jac_eval_freq;
  int reactor_type;      // 1: e / cv, 2: h / cp
  int lu_fp32;           // factor I - gamma J in FP32 and refine in FP64
  int refine_sweeps;     // iterative-refinement sweeps when lu_fp32
  int rk_guess, rk_min, rk_max;
  int use_typ_vals;
  int rendezvous;        // cycles a warp waits at a right-hand side for its block's other warps (0: off)
};

// The rendezvous bound a launch of `warps` warps per block runs with when
// the autotuner picked none; -1 picks it by block size: 300,000 SM clocks
// above 8 warps, 1,000,000 up to 8 (drm19 64^3 field: 16 warps 947k-959k
// cells/s at 300k against 894k-898k at 1M; 8 warps 425k-432k against
// 450k-454k).
inline int rendezvous_bound(int cycles, int warps)
{
  return cycles >= 0 ? cycles : (warps > 8 ? 300000 : 1000000);
}

// Team-shared per-cell workspace.  LT is the LU storage type.
template <typename LT>
struct Work {
  double* zn[6];
  double *ewt, *acor, *y, *tempv, *ftemp, *delta;
  double *src, *atolv;
  LT* J;        // saved Jacobian (the factor's precision)
  double* jtmp; // where the Jacobian is evaluated in FP64 (J itself for FP64)
  double* jx;   // per-reaction factors of the Jacobian evaluation
  LT* A;
  int* piv;
  int* perm;  // row order of the factored matrix: row i of PA is row perm[i] of A
  struct BdfArrays* ba; // the integrator's coefficient arrays (team-shared)
  // rate scratch
  double *Y, *sc, *g, *qd, *wdot, *ei, *h1, *h2, *h3;
  double* qco = nullptr; // QSS solve scratch (QSS mechanisms)
  // block-shared rendezvous counters {arrived, generation, active warps}, or nullptr
  int* rv = nullptr;
};

// Soft rendezvous of a block's warp teams before a right-hand side: the
// team's lane 0 counts itself in and waits (at most `cycles` SM clocks) until
// every active team of the block has arrived, so that the block's warps run
// the right-hand side's instruction stream together.  It changes no
// arithmetic: a team that times out just goes on alone.
//
// rv[0] packs the generation (high 16 bits) and the arrivals of that
// generation (low 16 bits), so an arrival learns its generation from the same
// atomic that counts it; rv[2] is the number of active teams.  A generation
// is released by one compare-and-swap that bumps the generation and clears
// the count only if no arrival landed in between, so no arrival is ever
// erased.  A team that timed out and arrives again early counts twice: that
// only releases a generation early.
__device__ __forceinline__ void rendezvous_try_release(int* rv)
{
  volatile int* v = rv;
  for (int i = 0; i < 64; i++) { // bounded: each failed CAS means another arrival landed
    const int cur = v[0];
    const int active = v[2];
    if (active <= 0 || (cur & 0xffff) < active) return;
    if (atomicCAS(&rv[0], cur, (int)(((unsigned)cur & 0xffff0000u) + 0x10000u)) == cur) return;
  }
}

__device__ __forceinline__ void rendezvous(int* rv, int cycles)
{
  if ((threadIdx.x & 31) == 0) {
    volatile int* v = rv;
    const unsigned g = (unsigned)atomicAdd(&rv[0], 1) >> 16;
    rendezvous_try_release(rv);
    const long long t0 = clock64();
    // polls back off from 32 to 256 ns: a waiting warp's polls take issue
    // slots from the warps still working
    unsigned ns = 32;
    while (((unsigned)v[0] >> 16) == g && clock64() - t0 < cycles) {
      __nanosleep(ns);
      if (ns < 256) ns <<= 1;
    }
  }
  __syncwarp();
}

// The block's counters for a persistent loop of `teams` warp teams; every
// thread of the block calls it.  nullptr (no rendezvous) when cycles <= 0.
__device__ __forceinline__ int* rendezvous_init(int* rv, int teams, int cycles)
{
  if (cycles <= 0) return nullptr;
  if (threadIdx.x == 0) {
    rv[0] = 0;
    rv[1] = 0;
    rv[2] = teams;
  }
  __syncthreads();
  return rv;
}

// A team leaves the persistent loop, or pauses for a stretch it runs alone:
// the others stop waiting for it.
__device__ __forceinline__ void rendezvous_leave(int* rv)
{
  if (rv && (threadIdx.x & 31) == 0) {
    atomicSub(&rv[2], 1);
    rendezvous_try_release(rv);
  }
}

// A paused team counts itself back in (it arrives at its next right-hand side).
__device__ __forceinline__ void rendezvous_resume(int* rv)
{
  if (rv && (threadIdx.x & 31) == 0) atomicAdd(&rv[2], 1);
}

// QSS: a QSS mechanism (sc and g then have its QSS slots, qco the QSS
// solve's scratch; the team path solves the QSS concentrations only when
// QSS is set, the one-lane path whenever the mechanism has QSS species).
template <int TEAM, bool QSS = false>
__device__ double reactor_rhs(
  const Team<TEAM>& tm, const DevMech& M, int rtype, double t, const double* y, double* ydot, double rhoe,
  double rhoesrc, const double* src, double* Y, double* sc, double* g, double* qd, double* wdot, double* ei,
  double* qco = nullptr)
{
  const int N = M.nsp;
  double a = 0.0;
  for (int s = tm.lane; s < N; s += TEAM) a += y[s];
  const double rho = tm.sum(a);
  const double rinv = 1.0 / rho;
  for (int s = tm.lane; s < N; s += TEAM) Y[s] = y[s] * rinv;
  tm.sync();
  const double nrg = (rhoe + rhoesrc * t) * rinv;
  double T = y[N];
  const int EH = (rtype == 2);
  t_from_energy(tm, M, EH, nrg, Y, T);
  const double invT = 1.0 / T;
  const double RT = RU * T;
  RateScratch rs{sc, g, qd, nullptr, qco};
  double cv;
  if constexpr (TEAM > 1) {
    // one pass over the species at the final T: the heat capacity (as
    // mix_c), the energies, the concentrations, their sum and g/RT (as
    // productionRate forms them), then the two sums together
    const double logT = ppb_log(T);
    const double refC = 101325 / 8.31446 * invT;
    const double refCinv = 1 / refC;
    double cvs = 0.0, mix = 0.0;
    for (int s = tm.lane; s < N; s += TEAM) {
      const double im = __ldg(M.imw + s);
      cvs += Y[s] * (EH ? cp_R(M, s, T) : cv_R(M, s, T)) * __ldg(M.imw + s);
      ei[s] = (EH ? h_RT(M, s, T, invT) : u_RT(M, s, T, invT)) * (RT * im);
      const double scs = (rho * Y[s] * im) * 1.0e6;
      sc[s] = scs;
      mix += scs;
      g[s] = g_RT(M, s, T, invT, logT);
    }
    cv = tm.sum(cvs) * RU;
    const double mixture = tm.sum(mix);
    if (tm.lane == 0) {
      sc[N] = 1.0; // padding slots of the packed reaction records
      g[N] = 0.0;
    }
    tm.sync();
    if constexpr (QSS) qss_solve<TEAM>(tm, M, sc, g, T, invT, logT, refC, refCinv, mixture, qco, qco + 2 * M.nrq);
    production_rate_core(tm, M, wdot, sc, T, invT, logT, refC, refCinv, mixture, rs);
  } else {
    cv = mix_c(tm, M, EH, T, Y);
    for (int s = tm.lane; s < N; s += TEAM) {
      const double im = __ldg(M.imw + s);
      ei[s] = (EH ? h_RT(M, s, T, invT) : u_RT(M, s, T, invT)) * (RT * im);
      sc[s] = (rho * Y[s] * im) * 1.0e6;
    }
    if (tm.lane == 0) sc[N] = 1.0; // padding slot of the packed reaction records
    tm.sync();
    production_rate(tm, M, wdot, sc, T, rs);
  }
  double acc = 0.0;
  for (int s = tm.lane; s < N; s += TEAM) {
    const double cd = wdot[s] * 1.0e-6 * __ldg(M.mw + s) + src[s];
    ydot[s] = cd;
    acc += cd * ei[s];
  }
  const double esrc = rhoesrc - tm.sum(acc);
  if (tm.lane == 0) ydot[N] = esrc * (rinv / cv);
  tm.sync();
  return T;
}

// The reference's fKernelSpec with the SRK EOS (reactor type 1): REY2T,
// RTY2Ei, RTY2Cv and the activities of RTY2WDOT (Source/Eos/SRK.H:446-487,
// 659-688, 413-427, 589-638) in place of the ideal-gas forms.
template <int TEAM>
__device__ double reactor_rhs_srk(
  const Team<TEAM>& tm, const DevMech& M, double t, const double* y, double* ydot, double rhoe, double rhoesrc,
  const double* src, double* Y, double* sc, double* g, double* qd, double* wdot, double* ei)
{
  const int N = M.nsp;
  double a = 0.0;
  for (int s = tm.lane; s < N; s += TEAM) a += y[s];
  const double rho = tm.sum(a);
  const double rinv = 1.0 / rho;
  for (int s = tm.lane; s < N; s += TEAM) Y[s] = y[s] * rinv;
  tm.sync();
  const double nrg = (rhoe + rhoesrc * t) * rinv;
  double T = y[N];
  SrkState k;
  srk_t_from_energy(tm, M, rho, nrg, Y, T, k);
  srk_sums(tm, M, T, rho, Y, k);
  const double cv = mix_c(tm, M, 0, T, Y) + T * k.d2AmdT2 * k.K1;
  const double invT = 1.0 / T, RT = RU * T, sqrtT = sqrt(T);
  double sy = 0.0;
  for (int s = tm.lane; s < N; s += TEAM) sy += Y[s] * __ldg(M.imw + s);
  const double wbar = 1.0 / tm.sum(sy);
  const double InvBm = 1.0 / k.bm, tau = 1.0 / rho;
  const double RmT = RU / wbar * T, InvRuT = 1.0 / (RU * T);
  const double d1 = 1.0 / (tau - k.bm), d3 = 1.0 / (tau + k.bm);
  const double* P = M.srk;
  for (int s = tm.lane; s < N; s += TEAM) {
    const double sOT = __ldg(P + s), sA = __ldg(P + N + s), B = __ldg(P + 2 * N + s), F = __ldg(P + 3 * N + s);
    const double al = (1.0 + F * (1.0 - sqrtT * sOT)) * sA;
    const double ad = -0.5 * F * sA * invT * sqrtT * sOT;
    const double dAmdY = 2.0 * al * k.S1, d2AmdTY = 2.0 * (al * k.S1p + ad * k.S1);
    const double im = __ldg(M.imw + s);
    ei[s] = u_RT(M, s, T, invT) * (RT * im) + (T * d2AmdTY - dAmdY) * k.K1 +
            (T * k.dAmdT - k.am) * B * (d3 - k.K1) * InvBm;
    const double act = ppb_exp((__ldg(M.mw + s) * InvRuT) *
                               (RmT * d1 * B - k.K1 * dAmdY + k.am * InvBm * k.K1 * B - k.am * d3 * B * InvBm)) *
                       Y[s] * im * d1;
    sc[s] = act * 1.0e6;
  }
  if (tm.lane == 0) sc[N] = 1.0; // padding slot of the packed reaction records
  tm.sync();
  RateScratch rs{sc, g, qd};
  production_rate(tm, M, wdot, sc, T, rs);
  double acc = 0.0;
  for (int s = tm.lane; s < N; s += TEAM) {
    const double cd = wdot[s] * 1.0e-6 * __ldg(M.mw + s) + src[s];
    ydot[s] = cd;
    acc += cd * ei[s];
  }
  const double esrc = rhoesrc - tm.sum(acc);
  if (tm.lane == 0) ydot[N] = esrc * (rinv / cv);
  tm.sync();
  return T;
}

// Reactor Jacobian, column-major n x n: J[i*n + k] = d f_k / d y_i.
template <int TEAM, int PER>
__device__ void reactor_jac(
  const Team<TEAM>& tm, const DevMech& M, int rtype, const double* y, double* J, double* sc, double* g,
  double* wdot, double* h1, double* h2, double* h3, double* h4, double* qd = nullptr, double* jx = nullptr)
{
  const int N = M.nsp, n = N + 1;
  double a = 0.0;
  for (int s = tm.lane; s < N; s += TEAM) a += y[s];
  const double rho = tm.sum(a);
  const double temp = y[N];
  for (int s = tm.lane; s < N; s += TEAM) {
    const double Ys = y[s] / rho;
    sc[s] = 1.e6 * (rho * Ys * __ldg(M.imw + s));
  }
  if (tm.lane == 0) sc[N] = 1.0; // padding slot of the packed reaction records
  tm.sync();
  RateScratch rs{sc, g, qd, jx};
  ajacobian<TEAM, PER>(tm, M, J, sc, temp, rtype == 2 ? 1 : 0, rs, wdot, h1, h2, h3, h4);
  // DWDOT unit rescaling followed by the cJac mw/imw scaling, column by column
  for (int i = tm.lane; i < n; i += TEAM) {
    double* col = J + i * n;
    if (i < N) {
      const double imi = __ldg(M.imw + i);
      for (int k = 0; k < N; k++) col[k] = col[k] * __ldg(M.mw + k) * imi;
      col[N] = (col[N] * 1.e6) * imi;
    } else {
      for (int k = 0; k < N; k++) col[k] = (col[k] * 1.e-6) * __ldg(M.mw + k);
      col[N] = 0.0;
    }
  }
  tm.sync();
}

// ---------------------------------------------------------------- dense LU
// Partial-pivoting LU of a column-major n x n matrix (first maximum wins, as
// the SUNDIALS dense GETRF).  Returns 0 or k+1 for a zero pivot.
template <int TEAM, typename LT>
__device__ int lu_factor(const Team<TEAM>& tm, LT* A, int n, int* piv)
{
  for (int k = 0; k < n; k++) {
    LT* colk = A + k * n;
    if constexpr (TEAM == 32) {
      if (n - k <= 32) {
        // one row per lane (row k + lane): the largest magnitude by a max
        // reduction, the first row holding it by a ballot (rows in lane
        // order), its value by one shuffle, so the reciprocal overlaps the
        // row swap; a NaN entry never wins (its lane stays at -1)
        const int i = k + tm.lane;
        const LT a = i < n ? colk[i] : (LT)0;
        const double v = fabs((double)a);
        const double mine = (i < n && v > -1.0) ? v : -1.0;
        double mx = mine;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        const unsigned hit = __ballot_sync(0xffffffffu, i < n && mine == mx);
        const int src = hit ? __ffs(hit) - 1 : 0;
        const LT pv = __shfl_sync(0xffffffffu, a, src);
        const int l = k + src;
        if (!(mx > 0.0) || !hit) {
          tm.sync();
          return k + 1;
        }
        if (tm.lane == 0) piv[k] = l;
        const LT mult = (LT)1.0 / pv;
        if (l != k) {
          for (int j = tm.lane; j < n; j += TEAM) {
            const LT t = A[j * n + l];
            A[j * n + l] = A[j * n + k];
            A[j * n + k] = t;
          }
        }
        tm.sync();
        if (i > k && i < n) {
          // the lane scales its own row's multiplier and keeps it
          const LT lik = colk[i] * mult;
          colk[i] = lik;
#pragma unroll 4
          for (int j = k + 1; j < n; j++) {
            const LT akj = A[j * n + k];
            if (akj != (LT)0) A[j * n + i] -= akj * lik;
          }
        }
        tm.sync();
        continue;
      }
    }
    double best = -1.0;
    int bi = n;
    for (int i = k + tm.lane; i < n; i += TEAM) {
      const double v = fabs((double)colk[i]);
      if (v > best) {
        best = v;
        bi = i;
      }
    }
    if constexpr (TEAM <= 32) {
#pragma unroll
      for (int o = TEAM / 2; o > 0; o >>= 1) {
        const double ob = __shfl_xor_sync(tm.mask, best, o, TEAM);
        const int oi = __shfl_xor_sync(tm.mask, bi, o, TEAM);
        if (ob > best || (ob == best && oi < bi)) {
          best = ob;
          bi = oi;
        }
      }
    } else {
      tm.argmax(best, bi);
    }
    const int l = bi;
    // a zero column is singular; an all-NaN column selects no row (bi == n)
    if (!(best > 0.0) || l >= n) {
      tm.sync();
      return k + 1;
    }
    if (tm.lane == 0) piv[k] = l;
    if (l != k) {
      for (int j = tm.lane; j < n; j += TEAM) {
        const LT t = A[j * n + l];
        A[j * n + l] = A[j * n + k];
        A[j * n + k] = t;
      }
    }
    tm.sync();
    const LT mult = (LT)1.0 / colk[k];
    for (int i = k + 1 + tm.lane; i < n; i += TEAM) colk[i] *= mult;
    tm.sync();
    for (int i = k + 1 + tm.lane; i < n; i += TEAM) {
      const LT lik = colk[i];
      for (int j = k + 1; j < n; j++) {
        const LT akj = A[j * n + k];
        if (akj != (LT)0) A[j * n + i] -= akj * lik;
      }
    }
    tm.sync();
  }
  return 0;
}

// Solve (LU) x = b in place (b team-shared, double).
template <int TEAM, typename LT>
__device__ void lu_solve(const Team<TEAM>& tm, const LT* A, int n, const int* piv, double* b)
{
  if (tm.lane == 0) {
    for (int k = 0; k < n; k++) {
      const int pk = piv[k];
      if (pk != k) {
        const double t = b[k];
        b[k] = b[pk];
        b[pk] = t;
      }
    }
  }
  tm.sync();
  for (int k = 0; k < n - 1; k++) {
    const double bk = b[k];
    const LT* colk = A + k * n;
    for (int i = k + 1 + tm.lane; i < n; i += TEAM) b[i] -= (double)colk[i] * bk;
    tm.sync();
  }
  for (int k = n - 1; k > 0; k--) {
    const LT* colk = A + k * n;
    const double bk = b[k] / (double)colk[k];
    tm.sync();
    if (tm.lane == k % TEAM) b[k] = bk;
    for (int i = tm.lane; i < k; i += TEAM) b[i] -= (double)colk[i] * bk;
    tm.sync();
  }
  if (tm.lane == 0) b[0] /= (double)A[0];
  tm.sync();
}

// Row order of a factored matrix from its LAPACK-style pivots: the
// interchanges k <-> piv[k], in order, applied to the identity, so that the
// pivoted right-hand side is b[perm[0..n-1]].  A pivot outside [0, n) (pivots
// of no factorisation yet, e.g. a checkpoint taken before the first step) is
// skipped, so perm is always a permutation of 0..n-1.
template <int TEAM>
__device__ __forceinline__ void perm_from_piv(const Team<TEAM>& tm, const int* piv, int* perm, int n)
{
  if (tm.lane == 0) {
    for (int i = 0; i < n; i++) perm[i] = i;
    for (int k = 0; k < n; k++) {
      const int p = piv[k];
      if (p != k && p >= 0 && p < n) {
        const int t = perm[k];
        perm[k] = perm[p];
        perm[p] = t;
      }
    }
  }
  tm.sync();
}

// lu_solve for a team of 16 or 32 lanes and n <= TEAM with the solution in
// registers, lane i holding entry i: the pivoted gather, then the two
// triangular sweeps with the running entry k broadcast by a shuffle instead of
// a shared-memory round trip and a team barrier per column.  Every entry is
// updated by the same operations in the same order as in lu_solve.
template <int TEAM, typename LT, int NN>
__device__ __forceinline__ void lu_solve_reg(const Team<TEAM>& tm, const LT* A, const int* perm, double* b)
{
  static_assert((TEAM == 16 || TEAM == 32) && NN <= TEAM, "one entry per lane");
  const int i = tm.lane;
  double x = (i < NN) ? b[perm[i]] : 0.0;
#pragma unroll
  for (int k = 0; k < NN - 1; k++) {
    const double bk = __shfl_sync(tm.mask, x, k, TEAM);
    if (i > k && i < NN) x -= (double)A[k * NN + i] * bk;
  }
#pragma unroll
  for (int k = NN - 1; k > 0; k--) {
    const double bk = __shfl_sync(tm.mask, x, k, TEAM) / (double)A[k * NN + k];
    if (i == k) {
      x = bk;
    } else if (i < k) {
      x -= (double)A[k * NN + i] * bk;
    }
  }
  if (i == 0) x /= (double)A[0];
  tm.sync(); // every lane has gathered its entry before any writes
  if (i < NN) b[i] = x;
  tm.sync();
}

// ---------------------------------------------------------------- BDF
// The integrator's coefficient arrays, indexed by order at run time (in
// registers they would force the integrator's whole state to local memory):
// one shared copy per warp of a cell's team.  The first lane of the warp
// writes them and the warp synchronises before they are read, so their
// read-modify-write updates never race.
struct BdfArrays {
  double tau[7], tq[6], l[6];
  // cold state, out of the registers: the last step size and the error
  // constant saved for an order increase; the statistics counters
  double hu, saved_tq5;
  int nje, nsetups, nni, ncfn, netf, pad;
};

// The scalar integrator state: every lane of the team holds the same values
// (in registers).
struct BdfScalars {
  double h, hprime, hscale, eta, etamax, tn, rl1, gamma, gammap, gamrat, crate, delp, acnrm;
  double gamma_lu; // gamma of the factored matrix I - gamma J
  int q, qprime, qwait, L, qmax, indx_acor, jcur;
  int nst, nstlp, nstlj, nfe;
#ifdef PPB_PHASE_TIMERS
  long long phase[PH_COUNT];
#endif
};

struct CellIn {
  double rhoe, rhoesrc;
};

// The integrator's right-hand side at (t, y) into fy (fKernelSpec).  A free
// function taking what it reads, so that no caller's state has to live in
// memory for the call.  Inlined at its call sites by default (drm19 64^3:
// 909k against 837k cells/s out of line, which keeps one copy of the
// right-hand side in the kernel; build with -DPPB_RHS_ATTR=__noinline__ for
// that form).
#ifndef PPB_RHS_ATTR
#define PPB_RHS_ATTR __forceinline__
#endif
// The right-hand side variants of the integrator (the RHSV template
// argument): the ideal-gas reactor, the SRK e-reactor, the ideal-gas reactor
// of a QSS mechanism.  The last two have no analytical Jacobian.
enum : int { RHS_IDEAL = 0, RHS_SRK = 1, RHS_QSS = 2 };

// The difference-quotient variants (SRK, QSS) evaluate the right-hand
// side from two call sites, the integrator and the Jacobian's n + 1
// columns: one out-of-line copy of it (drm19 SRK at 50 atm 39k -> 60k
// cells/s, CH4_lean_qss 294k -> 672k against the copy inlined at both).
template <int TEAM, int RHSV>
__device__ __noinline__ void bdf_rhs_dq(Team<TEAM> tm, const DevMech& M, int rtype, double t, const double* y,
                                        double* fy, double rhoe, double rhoesrc, const double* src, double* Y,
                                        double* sc, double* g, double* qd, double* wdot, double* ei, double* qco)
{
  if constexpr (RHSV == RHS_SRK) {
    reactor_rhs_srk<TEAM>(tm, M, t, y, fy, rhoe, rhoesrc, src, Y, sc, g, qd, wdot, ei);
  } else {
    reactor_rhs<TEAM, RHSV == RHS_QSS>(tm, M, rtype, t, y, fy, rhoe, rhoesrc, src, Y, sc, g, qd, wdot, ei, qco);
  }
}

template <int TEAM, int RHSV>
__device__ PPB_RHS_ATTR void bdf_rhs(Team<TEAM> tm, const DevMech& M, int rtype, double t, const double* y,
                                     double* fy, double rhoe, double rhoesrc, const double* src, double* Y,
                                     double* sc, double* g, double* qd, double* wdot, double* ei, double* qco)
{
  if constexpr (RHSV == RHS_IDEAL) {
    reactor_rhs<TEAM, false>(tm, M, rtype, t, y, fy, rhoe, rhoesrc, src, Y, sc, g, qd, wdot, ei, qco);
  } else {
    bdf_rhs_dq<TEAM, RHSV>(tm, M, rtype, t, y, fy, rhoe, rhoesrc, src, Y, sc, g, qd, wdot, ei, qco);
  }
}

// Recorder interface of the integrator: every operation that changes the
// Nordsieck history, with the coefficients it used, in execution order (the
// discrete adjoint and tangent-linear sweeps replay these).  NoRec records
// nothing and compiles away.
struct NoRec {
  static constexpr bool on = false;
};

template <int NS, int TEAM, typename LT, typename Rec = NoRec, int RHSV = RHS_IDEAL>
struct Bdf {
  static constexpr int n = NS + 1;
  static constexpr int PER = (NS + TEAM - 1) / TEAM;
  const Team<TEAM>& tm;
  const DevMech& M;
  const Options& o;
  Work<LT>& w;
  CellIn cin;
  BdfScalars s;
  BdfArrays& ar;
  Rec rec;

  __device__ Bdf(const Team<TEAM>& t, const DevMech& m, const Options& op, Work<LT>& wk, CellIn ci)
    : tm(t), M(m), o(op), w(wk), cin(ci), ar(wk.ba[TEAM > 32 ? (t.lane >> 5) : 0])
  {
  }

  // the lane that writes this warp's copy of the coefficient arrays
  __device__ __forceinline__ bool lead() const { return (tm.lane % Team<TEAM>::W) == 0; }
  // the warp (or the team's part of it) sees the copy's latest writes
  __device__ __forceinline__ void wsync() const
  {
    if constexpr (TEAM > 32) {
      __syncwarp();
    } else if constexpr (TEAM > 1) {
      __syncwarp(tm.mask);
    }
  }

  __device__ __forceinline__ double wrms(const double* v) const
  {
    double a = 0.0;
    for (int i = tm.lane; i < n; i += TEAM) {
      const double x = v[i] * w.ewt[i];
      a += x * x;
    }
    return sqrt(tm.sum(a) / n);
  }

  __device__ __forceinline__ void set_ewt(const double* y)
  {
    for (int i = tm.lane; i < n; i += TEAM) {
      const double at = o.use_typ_vals ? w.atolv[i] : o.atol;
      w.ewt[i] = 1.0 / (o.rtol * fabs(y[i]) + at);
    }
    tm.sync();
  }

  // the block rendezvous (when on), then the right-hand side
  __device__ __forceinline__ void f(double t, const double* y, double* fy)
  {
    if (w.rv) rendezvous(w.rv, o.rendezvous);
    PPB_TIC(PH_RHS);
    bdf_rhs<TEAM, RHSV>(tm, M, o.reactor_type, t, y, fy, cin.rhoe, cin.rhoesrc, w.src, w.Y, w.sc, w.g, w.qd, w.wdot,
                        w.ei, w.qco);
    s.nfe++;
    PPB_TOC(PH_RHS);
  }

  __device__ __forceinline__ void jac()
  {
    PPB_TIC(PH_JAC);
    if constexpr (RHSV != RHS_IDEAL) {
      jac_dq();
    } else {
      // the Newton matrix region is free while the Jacobian is formed: it
      // holds the per-reaction factors of the warp-cooperative evaluation
      reactor_jac<TEAM, PER>(tm, M, o.reactor_type, w.y, w.jtmp, w.sc, w.g, w.wdot, w.Y, w.ei, w.h1, w.h2,
                             TEAM > 1 ? w.qd : nullptr, TEAM > 1 ? w.jx : nullptr);
      if constexpr (sizeof(LT) != sizeof(double)) jac_to_lt();
    }
    PPB_TOC(PH_JAC);
  }

  // The FP64 Jacobian in w.jtmp, rounded to the factor's precision in
  // place: chunk by chunk, every lane holds its entries of a chunk in
  // registers before any lane writes, and an entry's FP32 slot lies at or
  // below the FP64 entries already read.
  __device__ __forceinline__ void jac_to_lt()
  {
    constexpr int CH = 8;
    const int nn = n * n;
    for (int base = 0; base < nn; base += CH * TEAM) {
      double v[CH];
#pragma unroll
      for (int q = 0; q < CH; q++) {
        const int i = base + q * TEAM + tm.lane;
        v[q] = (i < nn) ? w.jtmp[i] : 0.0;
      }
      tm.sync();
#pragma unroll
      for (int q = 0; q < CH; q++) {
        const int i = base + q * TEAM + tm.lane;
        if (i < nn) w.J[i] = (LT)v[q];
      }
      tm.sync();
    }
  }

  // Difference-quotient dense Jacobian at (tn, y) with f(tn, y) in ftemp:
  // the SRK EOS has no analytical Jacobian (SRK::RTY2JAC aborts,
  // Source/Eos/SRK.H:640-648), nor a QSS mechanism without CEPTR's symbolic
  // build (aJacobian_precond aborts in its mechanism.H), so the reference's
  // CVODE forms it by differences (cvode.solve_type = dense_direct);
  // restated from CVODE's dense difference-quotient Jacobian:
  // column j uses inc = max(sqrt(eps) |y_j|, min_inc / ewt_j), min_inc =
  // 1000 |h| eps n ||f||_WRMS (1 when ||f|| = 0).  Its RHS evaluations are
  // not counted in nfe (CVODE counts them separately).
  __device__ __forceinline__ void jac_dq()
  {
    const double fnorm = wrms(w.ftemp);
    const double eps = 2.220446049250313e-16;
    const double srur = sqrt(eps);
    const double min_inc = (fnorm != 0.0) ? (1000.0 * fabs(s.h) * eps * n * fnorm) : 1.0;
    for (int i = tm.lane; i < n; i += TEAM) w.tempv[i] = w.y[i];
    tm.sync();
    for (int j = 0; j < n; j++) {
      const double yj = w.tempv[j];
      const double inc = fmax(srur * fabs(yj), min_inc / w.ewt[j]);
      tm.sync();
      if (tm.lane == 0) w.tempv[j] = yj + inc;
      tm.sync();
      double* col = w.J + (size_t)j * n;
      bdf_rhs<TEAM, RHSV>(tm, M, o.reactor_type, s.tn, w.tempv, col, cin.rhoe, cin.rhoesrc, w.src, w.Y, w.sc, w.g,
                          w.qd, w.wdot, w.ei, w.qco);
      const double inc_inv = 1.0 / inc;
      for (int i = tm.lane; i < n; i += TEAM) col[i] = inc_inv * col[i] + (-inc_inv) * w.ftemp[i];
      if (tm.lane == 0) w.tempv[j] = yj;
      tm.sync();
    }
  }

  __device__ __forceinline__ int hin(double tout)
  {
    const double tdiff = tout - s.tn;
    if (tdiff == 0.0) return ST_TOO_CLOSE;
    const double tdist = fabs(tdiff);
    const double tround = 2.220446049250313e-16 * fmax(fabs(s.tn), fabs(tout));
    if (tdist < 2.0 * tround) return ST_TOO_CLOSE;
    const double hlb = 100.0 * tround;
    double hub_inv = 0.0;
    for (int i = tm.lane; i < n; i += TEAM) {
      const double t1 = 0.1 * fabs(w.zn[0][i]) + 1.0 / w.ewt[i];
      hub_inv = fmax(hub_inv, fabs(w.zn[1][i]) / t1);
    }
    hub_inv = tm.max(hub_inv);
    double hub = 0.1 * tdist;
    if (hub * hub_inv > 1.0) hub = 1.0 / hub_inv;
    double hg = sqrt(hlb * hub);
    if (hub < hlb) {
      s.h = hg;
      return ST_OK;
    }
    double hnew = hg;
    for (int count1 = 1; count1 <= 4; count1++) {
      for (int i = tm.lane; i < n; i += TEAM) w.y[i] = hg * w.zn[1][i] + w.zn[0][i];
      tm.sync();
      f(s.tn + hg, w.y, w.tempv);
      for (int i = tm.lane; i < n; i += TEAM) w.tempv[i] = (w.tempv[i] - w.zn[1][i]) * (1.0 / hg);
      tm.sync();
      const double yddnrm = wrms(w.tempv);
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
    double h0 = 0.5 * hnew;
    if (h0 < hlb) h0 = hlb;
    if (h0 > hub) h0 = hub;
    s.h = h0;
    return ST_OK;
  }

  __device__ __forceinline__ void rescale()
  {
    if constexpr (Rec::on) rec.rescale(tm, s.q, s.eta);
    double factor = s.eta;
    for (int j = 1; j <= s.q; j++) {
      for (int i = tm.lane; i < n; i += TEAM) w.zn[j][i] *= factor;
      factor *= s.eta;
    }
    tm.sync();
    s.h = s.hscale * s.eta;
    s.hscale = s.h;
  }

  __device__ __forceinline__ void predict()
  {
    s.tn += s.h;
    for (int i = tm.lane; i < n; i += TEAM) {
      for (int k = 1; k <= s.q; k++)
        for (int j = s.q; j >= k; j--) w.zn[j - 1][i] += w.zn[j][i];
    }
    tm.sync();
  }

  __device__ __forceinline__ void restore(double saved_t)
  {
    s.tn = saved_t;
    for (int i = tm.lane; i < n; i += TEAM) {
      for (int k = 1; k <= s.q; k++)
        for (int j = s.q; j >= k; j--) w.zn[j - 1][i] -= w.zn[j][i];
    }
    tm.sync();
  }

  // the coefficients of order q: written by the lead lane only
  __device__ __forceinline__ void set_bdf()
  {
    if (lead()) set_bdf_lead();
    wsync();
  }

  __device__ __forceinline__ void set_bdf_lead()
  {
    double alpha0, alpha0_hat, xi_inv, xistar_inv, hsum;
    const int q = s.q;
    ar.l[0] = ar.l[1] = xi_inv = xistar_inv = 1.0;
    for (int i = 2; i <= q; i++) ar.l[i] = 0.0;
    alpha0 = alpha0_hat = -1.0;
    hsum = s.h;
    if (q > 1) {
      for (int j = 2; j < q; j++) {
        hsum += ar.tau[j - 1];
        xi_inv = s.h / hsum;
        alpha0 -= 1.0 / j;
        for (int i = j; i >= 1; i--) ar.l[i] += ar.l[i - 1] * xi_inv;
      }
      alpha0 -= 1.0 / q;
      xistar_inv = -ar.l[1] - alpha0;
      hsum += ar.tau[q - 1];
      xi_inv = s.h / hsum;
      alpha0_hat = -ar.l[1] - xi_inv;
      for (int i = q; i >= 1; i--) ar.l[i] += ar.l[i - 1] * xistar_inv;
    }
    const double A1 = 1.0 - alpha0_hat + alpha0;
    const double A2 = 1.0 + q * A1;
    ar.tq[2] = fabs(A1 / (alpha0 * A2));
    ar.tq[5] = fabs(A2 * xistar_inv / (ar.l[q] * xi_inv));
    if (s.qwait == 1) {
      if (q > 1) {
        const double C = xistar_inv / ar.l[q];
        const double A3 = alpha0 + 1.0 / q;
        const double A4 = alpha0_hat + xi_inv;
        const double Cpinv = (1.0 - A4 + A3) / A3;
        ar.tq[1] = fabs(C * Cpinv);
      } else {
        ar.tq[1] = 1.0;
      }
      hsum += ar.tau[q];
      xi_inv = s.h / hsum;
      const double A5 = alpha0 - (1.0 / (q + 1));
      const double A6 = alpha0_hat - xi_inv;
      const double Cppinv = (1.0 - A6 + A5) / A2;
      ar.tq[3] = fabs(Cppinv / (xi_inv * (q + 2) * A5));
    }
    ar.tq[4] = 0.1 / ar.tq[2];
  }

  __device__ __forceinline__ void set()
  {
    set_bdf();
    s.rl1 = 1.0 / ar.l[1];
    s.gamma = s.h * s.rl1;
    if (s.nst == 0) s.gammap = s.gamma;
    s.gamrat = (s.nst > 0) ? s.gamma / s.gammap : 1.0;
  }

  // cvLsSetup: (re)use J, form I - gamma J, factor
  __device__ __forceinline__ int ls_setup(int convfail)
  {
    const double dgamma = fabs((s.gamma / s.gammap) - 1.0);
    const bool jbad = (s.nst == 0) || (s.nst >= s.nstlj + o.jac_eval_freq) || ((convfail == 1) && (dgamma < 0.2)) ||
                      (convfail == 2);
    if (!jbad) {
      s.jcur = 0;
    } else {
      if (lead()) ar.nje++;
      s.nstlj = s.nst;
      s.jcur = 1;
      // the Jacobian is the longest stretch a team runs alone (drm19: ~300k
      // SM clocks, against ~34k for a right-hand side and ~65k for a
      // factorisation): the team leaves the block rendezvous meanwhile, so
      // that the other teams' right-hand sides do not wait for it (drm19
      // 64^3: 1.047M cells/s against 0.96M; leaving it for the
      // factorisations too gave 0.55M, as the teams then drift apart)
      rendezvous_leave(w.rv);
      jac();
      rendezvous_resume(w.rv);
    }
    s.gamma_lu = s.gamma;
    PPB_TIC(PH_LU);
    for (int i = tm.lane; i < n; i += TEAM) {
      for (int j = 0; j < n; j++) {
        double v = -s.gamma * (double)w.J[j * n + i];
        if (i == j) v += 1.0;
        w.A[j * n + i] = (LT)v;
      }
    }
    tm.sync();
    const int ier = lu_factor<TEAM, LT>(tm, w.A, n, w.piv) ? 1 : 0;
    if constexpr ((TEAM == 16 || TEAM == 32) && n <= TEAM) {
      if (!ier) perm_from_piv(tm, w.piv, w.perm, n);
    }
    PPB_TOC(PH_LU);
    return ier;
  }

  // (LU) x = b in place with the current factor
  __device__ __forceinline__ void lsolve(double* b)
  {
    if constexpr ((TEAM == 16 || TEAM == 32) && n <= TEAM) {
      lu_solve_reg<TEAM, LT, n>(tm, w.A, w.perm, b);
    } else {
      lu_solve<TEAM, LT>(tm, w.A, n, w.piv, b);
    }
  }

  // x := (I - gamma J)^{-1} b, with FP64 iterative refinement when the
  // factor is FP32.  b and x are w.delta; w.tempv is scratch.
  __device__ __forceinline__ void ls_solve()
  {
    PPB_TIC(PH_SOLVE);
    ls_solve_impl();
    PPB_TOC(PH_SOLVE);
  }

  __device__ __forceinline__ void ls_solve_impl()
  {
    if (sizeof(LT) == sizeof(double) || o.refine_sweeps <= 0) {
      lsolve(w.delta);
      return;
    }
    // keep b in ftemp-sized scratch: w.h3 (length >= n)
    double* b = w.h3;
    for (int i = tm.lane; i < n; i += TEAM) b[i] = w.delta[i];
    tm.sync();
    lsolve(w.delta);
    for (int sweep = 0; sweep < o.refine_sweeps; sweep++) {
      // r = b - (I - gamma_lu J) x in FP64, against the matrix that was
      // factored (CVODE corrects a stale gamma afterwards, in nls)
      for (int i = tm.lane; i < n; i += TEAM) {
        double ax = w.delta[i];
        double jx = 0.0;
        for (int j = 0; j < n; j++) jx += (double)w.J[j * n + i] * w.delta[j];
        ax -= s.gamma_lu * jx;
        w.tempv[i] = b[i] - ax;
      }
      tm.sync();
      lsolve(w.tempv);
      for (int i = tm.lane; i < n; i += TEAM) w.delta[i] += w.tempv[i];
      tm.sync();
    }
  }

  __device__ __forceinline__ void nls_residual()
  {
    for (int i = tm.lane; i < n; i += TEAM) w.y[i] = w.zn[0][i] + w.acor[i];
    tm.sync();
    f(s.tn, w.y, w.ftemp);
    for (int i = tm.lane; i < n; i += TEAM) {
      const double r = s.rl1 * w.zn[1][i] + w.acor[i];
      w.delta[i] = -s.gamma * w.ftemp[i] + r;
    }
    tm.sync();
  }

  __device__ __forceinline__ int nls(int nflag)
  {
    PPB_TIC(PH_NEWTON);
    const int r = nls_impl(nflag);
    PPB_TOC(PH_NEWTON);
    return r;
  }

  __device__ __forceinline__ int nls_impl(int nflag)
  {
    const int convfail = ((nflag == 0) || (nflag == 2)) ? 0 : 2;
    bool callSetup = (nflag == 1) || (nflag == 2) || (s.nst == 0) || (s.nst >= s.nstlp + 20) ||
                     (fabs(s.gamrat - 1.0) > 0.3);
    for (int i = tm.lane; i < n; i += TEAM) w.acor[i] = 0.0;
    tm.sync();
    bool jbad = false;
    int retval = 0;
    for (;;) {
      nls_residual();
      if (callSetup) {
        const int ier = ls_setup(jbad ? 1 : convfail);
        if (lead()) ar.nsetups++;
        s.gamrat = 1.0;
        s.gammap = s.gamma;
        s.crate = 1.0;
        s.nstlp = s.nst;
        if (ier) return -1;
      }
      int m = 0;
      for (;;) {
        if (lead()) ar.nni++;
        for (int i = tm.lane; i < n; i += TEAM) w.delta[i] = -w.delta[i];
        tm.sync();
        ls_solve();
        if (s.gamrat != 1.0) {
          const double sc = 2.0 / (1.0 + s.gamrat);
          for (int i = tm.lane; i < n; i += TEAM) w.delta[i] *= sc;
        }
        for (int i = tm.lane; i < n; i += TEAM) w.acor[i] += w.delta[i];
        tm.sync();
        const double del = wrms(w.delta);
        if (m > 0) s.crate = fmax(0.3 * s.crate, del / s.delp);
        const double dcon = del * fmin(1.0, s.crate) / ar.tq[4];
        if (dcon <= 1.0) {
          s.acnrm = (m == 0) ? del : wrms(w.acor);
          s.jcur = 0;
          return 0;
        }
        if ((m >= 1) && (del > 2.0 * s.delp)) {
          retval = 1;
          break;
        }
        s.delp = del;
        m++;
        if (m >= o.max_nls_iters) {
          retval = 1;
          break;
        }
        nls_residual();
      }
      if (retval > 0 && !s.jcur) {
        callSetup = true;
        jbad = true;
        for (int i = tm.lane; i < n; i += TEAM) w.acor[i] = 0.0;
        tm.sync();
        continue;
      }
      break;
    }
    return retval;
  }

  __device__ __forceinline__ void increase_bdf()
  {
    double alpha0, alpha1, prod, xi, xiold, hsum, A1;
    const bool ld = lead();
    if (ld) {
      for (int i = 0; i <= s.qmax; i++) ar.l[i] = 0.0;
      ar.l[2] = 1.0;
    }
    alpha1 = prod = xiold = 1.0;
    alpha0 = -1.0;
    hsum = s.hscale;
    if (s.q > 1) {
      for (int j = 1; j < s.q; j++) {
        hsum += ar.tau[j + 1];
        xi = hsum / s.hscale;
        prod *= xi;
        alpha0 -= 1.0 / (j + 1);
        alpha1 += 1.0 / xi;
        if (ld)
          for (int i = j + 2; i >= 2; i--) ar.l[i] = ar.l[i] * xiold + ar.l[i - 1];
        xiold = xi;
      }
    }
    wsync();
    A1 = (-alpha0 - alpha1) / prod;
    for (int i = tm.lane; i < n; i += TEAM) {
      const double zL = A1 * w.zn[s.indx_acor][i];
      w.zn[s.L][i] = zL;
      for (int j = 2; j <= s.q; j++) w.zn[j][i] += ar.l[j] * zL;
    }
    tm.sync();
    if constexpr (Rec::on) rec.increase(tm, s.q, s.L, s.indx_acor, A1, ar.l);
  }

  __device__ __forceinline__ void decrease_bdf()
  {
    if (lead()) {
      for (int i = 0; i <= s.qmax; i++) ar.l[i] = 0.0;
      ar.l[2] = 1.0;
      double hsum = 0.0;
      for (int j = 1; j <= s.q - 2; j++) {
        hsum += ar.tau[j];
        const double xi = hsum / s.hscale;
        for (int i = j + 2; i >= 2; i--) ar.l[i] = ar.l[i] * xi + ar.l[i - 1];
      }
    }
    wsync();
    for (int i = tm.lane; i < n; i += TEAM)
      for (int j = 2; j < s.q; j++) w.zn[j][i] -= ar.l[j] * w.zn[s.q][i];
    tm.sync();
    if constexpr (Rec::on) rec.decrease(tm, s.q, ar.l);
  }

  __device__ __forceinline__ void adjust_order(int deltaq)
  {
    if ((s.q == 2) && (deltaq != 1)) return;
    if (deltaq == 1) increase_bdf();
    else if (deltaq == -1) decrease_bdf();
  }

  __device__ __forceinline__ int handle_nflag(int& nflag, double saved_t, int& ncf)
  {
    if (nflag == 0) return 2; // DO_ERROR_TEST
    if (lead()) ar.ncfn++;
    restore(saved_t);
    if (nflag < 0) return ST_LSETUP_FAIL;
    ncf++;
    s.etamax = 1.0;
    if (ncf == 10) return ST_CONV_FAILURE;
    s.eta = 0.25;
    nflag = 1;
    rescale();
    return 3; // PREDICT_AGAIN
  }

  __device__ __forceinline__ int do_error_test(int& nflag, double saved_t, int& nef, double& dsm)
  {
    dsm = s.acnrm * ar.tq[2];
    if (dsm <= 1.0) return ST_OK;
    nef++;
    if (lead()) ar.netf++;
    nflag = 2;
    restore(saved_t);
    if (nef == o.max_err_fails) return ST_ERR_FAILURE;
    s.etamax = 1.0;
    if (nef <= 3) {
      s.eta = 1.0 / (pow(6.0 * dsm, 1.0 / s.L) + 1.0e-6);
      s.eta = fmax(0.1, s.eta);
      if (nef >= 2) s.eta = fmin(s.eta, 0.2);
      rescale();
      return 5; // TRY_AGAIN
    }
    if (s.q > 1) {
      s.eta = 0.1;
      adjust_order(-1);
      s.L = s.q;
      s.q--;
      s.qwait = s.L;
      rescale();
      return 5;
    }
    s.eta = 0.1;
    s.h *= s.eta;
    s.hscale = s.h;
    s.qwait = 10;
    f(s.tn, w.zn[0], w.tempv);
    for (int i = tm.lane; i < n; i += TEAM) w.zn[1][i] = s.h * w.tempv[i];
    tm.sync();
    if constexpr (Rec::on) rec.freset(tm, s.tn, s.h, w.zn[0]);
    return 5;
  }

  __device__ __forceinline__ void complete_step()
  {
    s.nst++;
    const bool save = ((s.qwait - 1) == 1) && (s.q != s.qmax);
    if (lead()) {
      ar.hu = s.h;
      for (int i = s.q; i >= 2; i--) ar.tau[i] = ar.tau[i - 1];
      if ((s.q == 1) && (s.nst > 1)) ar.tau[2] = ar.tau[1];
      ar.tau[1] = s.h;
      if (save) ar.saved_tq5 = ar.tq[5];
    }
    wsync();
    if constexpr (Rec::on) {
      rec.predict(tm, s.q);
      rec.correct(tm, s.q, save, s.tn, s.gamma, s.rl1, ar.l, w.zn[0], w.acor);
    }
    for (int i = tm.lane; i < n; i += TEAM) {
      const double a = w.acor[i];
      for (int j = 0; j <= s.q; j++) w.zn[j][i] += ar.l[j] * a;
      if (save) w.zn[s.qmax][i] = a;
    }
    tm.sync();
    s.qwait--;
    if (save) s.indx_acor = s.qmax;
  }

  __device__ __forceinline__ void set_eta()
  {
    if ((s.eta > 0.0) && (s.eta < 1.5)) {
      s.eta = 1.0;
      s.hprime = s.h;
    } else {
      s.eta = fmin(s.eta, s.etamax);
      s.hprime = s.h * s.eta;
    }
  }

  __device__ __forceinline__ void prepare_next_step(double dsm)
  {
    if (s.etamax == 1.0) {
      s.qwait = s.qwait > 2 ? s.qwait : 2;
      s.qprime = s.q;
      s.hprime = s.h;
      s.eta = 1.0;
      return;
    }
    const double etaq = 1.0 / (pow(6.0 * dsm, 1.0 / s.L) + 1.0e-6);
    if (s.qwait != 0) {
      s.eta = etaq;
      s.qprime = s.q;
      set_eta();
      return;
    }
    s.qwait = 2;
    double etaqm1 = 0.0;
    if (s.q > 1) {
      const double ddn = wrms(w.zn[s.q]) * ar.tq[1];
      etaqm1 = 1.0 / (pow(6.0 * ddn, 1.0 / s.q) + 1.0e-6);
    }
    double etaqp1 = 0.0;
    if (s.q != s.qmax && ar.saved_tq5 != 0.0) {
      const double cquot = (ar.tq[5] / ar.saved_tq5) * pow(s.h / ar.tau[2], (double)s.L);
      for (int i = tm.lane; i < n; i += TEAM) w.tempv[i] = -cquot * w.zn[s.qmax][i] + w.acor[i];
      tm.sync();
      const double dup = wrms(w.tempv) * ar.tq[3];
      etaqp1 = 1.0 / (pow(10.0 * dup, 1.0 / (s.L + 1)) + 1.0e-6);
    }
    const double etam = fmax(etaqm1, fmax(etaq, etaqp1));
    if ((etam > 0.0) && (etam < 1.5)) {
      s.eta = 1.0;
      s.qprime = s.q;
    } else if (etam == etaq) {
      s.eta = etaq;
      s.qprime = s.q;
    } else if (etam == etaqm1) {
      s.eta = etaqm1;
      s.qprime = s.q - 1;
    } else {
      s.eta = etaqp1;
      s.qprime = s.q + 1;
      for (int i = tm.lane; i < n; i += TEAM) w.zn[s.qmax][i] = w.acor[i];
      tm.sync();
      if constexpr (Rec::on) rec.saveqmax(tm);
    }
    set_eta();
  }

  __device__ __forceinline__ void adjust_params()
  {
    if (s.qprime != s.q) {
      adjust_order(s.qprime - s.q);
      s.q = s.qprime;
      s.L = s.q + 1;
      s.qwait = s.L;
    }
    rescale();
  }

  __device__ __forceinline__ int step()
  {
    PPB_TIC(PH_STEP);
    const int r = step_impl();
    PPB_TOC(PH_STEP);
    return r;
  }

  __device__ __forceinline__ int step_impl()
  {
    const double saved_t = s.tn;
    int ncf = 0, nef = 0, nflag = 0;
    double dsm = 0.0;
    if ((s.nst > 0) && (s.hprime != s.h)) adjust_params();
    for (;;) {
      predict();
      set();
      nflag = nls(nflag);
      const int kflag = handle_nflag(nflag, saved_t, ncf);
      if (kflag == 3) continue;
      if (kflag != 2) return kflag;
      const int eflag = do_error_test(nflag, saved_t, nef, dsm);
      if (eflag == 5) continue;
      if (eflag != ST_OK) return eflag;
      break;
    }
    complete_step();
    prepare_next_step(dsm);
    s.etamax = 10.0;
    return ST_OK;
  }

  // Start of an integration of w.zn[0] (initial y, team-shared) towards
  // tout: history, error weights, initial step (cvInitialSetup, cvHin).
  __device__ __forceinline__ int start(double tout)
  {
    s = BdfScalars{};
    if (lead()) ar = BdfArrays{};
    // no factorisation yet: identity pivots and row order (a checkpoint taken
    // before the first step holds valid ones)
    for (int i = tm.lane; i < n; i += TEAM) {
      w.piv[i] = i;
      w.perm[i] = i;
    }
    tm.sync();
    s.qmax = o.max_order;
    s.q = 1;
    s.L = 2;
    s.qwait = 2;
    s.etamax = 10000.0;
    s.tn = 0.0;
    set_ewt(w.zn[0]);
    f(s.tn, w.zn[0], w.zn[1]);
    const int flag = hin(tout);
    if (flag == ST_OK) {
      s.hscale = s.h;
      s.hprime = s.h;
      for (int i = tm.lane; i < n; i += TEAM) w.zn[1][i] *= s.h;
      tm.sync();
      if constexpr (Rec::on) rec.init(tm, s.h, w.zn[0]);
    }
    return flag;
  }

  // Step until tout is passed (then interpolate to tout into w.y and set
  // done) or, with a recorder, until the recorder closes its segment.
  // nstloc counts the steps of this call to react.
  __device__ __forceinline__ int advance(double tout, int& nstloc, bool& done)
  {
    done = false;
    for (;;) {
      if (s.nst > 0) set_ewt(w.zn[0]);
      if (nstloc >= o.max_steps) return ST_TOO_MUCH_WORK;
      const int flag = step();
      if (flag != ST_OK) return flag;
      nstloc++;
      if ((s.tn - tout) * s.h >= 0.0) {
        const double sfac = (tout - s.tn) / s.h;
        for (int i = tm.lane; i < n; i += TEAM) {
          double v = w.zn[s.q][i];
          for (int j = s.q - 1; j >= 0; j--) v = w.zn[j][i] + sfac * v;
          w.y[i] = v;
        }
        tm.sync();
        if constexpr (Rec::on) rec.output(tm, s.q, sfac);
        done = true;
        return ST_OK;
      }
      if constexpr (Rec::on) {
        if (rec.segment_full()) return ST_OK;
      }
    }
  }

  // Integrate w.zn[0] (initial y, team-shared) over [0, tout]; result in w.y.
  __device__ __forceinline__ int run(double tout)
  {
    PPB_TIC(PH_TOTAL);
    int flag = start(tout);
    if (flag == ST_OK) {
      int nstloc = 0;
      bool done = false;
      flag = advance(tout, nstloc, done);
    }
    if (flag != ST_OK) {
      for (int i = tm.lane; i < n; i += TEAM) w.y[i] = w.zn[0][i];
      tm.sync();
    }
    PPB_TOC(PH_TOTAL);
#ifdef PPB_PHASE_TIMERS
    if (tm.lane == 0)
      for (int q = 0; q < PH_COUNT; q++) atomicAdd(&g_phase_cycles[q], (unsigned long long)s.phase[q]);
#endif
    return flag;
  }
};

// ReactorRK64.cpp:73-144 for one cell (team).  y (team-shared) in/out;
// returns the number of RK steps.
template <int TEAM, typename LT>
__device__ int rk64_cell(const Team<TEAM>& tm, const DevMech& M, const Options& o, Work<LT>& w, CellIn cin,
                         double dt)
{
  const double alpha[6] = {0.218150805229859, 0.256702469801519, 0.527402592007520,
                           0.0484864267224467, 1.24517071533530, 0.412366034843237};
  const double beta[6] = {-0.113554138044166, -0.215118587818400, -0.0510152146250577,
                          -1.07992686223881, -0.248664241213447, 0.0};
  const double err[6] = {-0.0554699315064507, 0.158481845574980, -0.0905918835751907,
                         -0.219084567203338, 0.164022338959433, 0.0426421977505659};
  const int neq = M.nsp + 1;
  double* soln = w.y;
  double* carry = w.zn[0];
  double* error = w.zn[1];
  double* ydot = w.ftemp;
  for (int i = tm.lane; i < neq; i += TEAM) carry[i] = soln[i];
  tm.sync();
  double t = 0.0;
  double dt_rk = dt / (double)o.rk_guess;
  const double dt_rk_min = dt / (double)o.rk_max;
  const double dt_rk_max = dt / (double)o.rk_min;
  int nsteps = 0;
  // the reference loop has no step cap; dt_rk >= dt / rk_max bounds it except
  // for round-off tails, which the cap below ends
  const int cap = 4 * o.rk_max + 1000;
  while (t < dt && nsteps < cap) {
    for (int i = tm.lane; i < neq; i += TEAM) error[i] = 0.0;
    tm.sync();
    for (int st = 0; st < 6; st++) {
      reactor_rhs<TEAM>(tm, M, o.reactor_type, t, soln, ydot, cin.rhoe, cin.rhoesrc, w.src, w.Y, w.sc, w.g, w.qd,
                        w.wdot, w.ei);
      for (int i = tm.lane; i < neq; i += TEAM) {
        error[i] += err[st] * dt_rk * ydot[i];
        soln[i] = carry[i] + alpha[st] * dt_rk * ydot[i];
        carry[i] = soln[i] + beta[st] * dt_rk * ydot[i];
      }
      tm.sync();
    }
    t += dt_rk;
    nsteps++;
    double me = 1e-50;
    for (int i = tm.lane; i < neq; i += TEAM) me = fabs(error[i]) > me ? fabs(error[i]) : me;
    me = tm.max(me);
    if (me < o.atol) {
      dt_rk = fmin(dt_rk_max, dt_rk * (1.0 * pow((o.atol / me), 0.25)));
    } else {
      dt_rk = fmax(dt_rk_min, dt_rk * (1.0 * pow((o.atol / me), 0.2)));
    }
    dt_rk = fmin(dt_rk, dt - t);
  }
  return nsteps;
}

} // namespace ppb
