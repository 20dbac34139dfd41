// Device-side mechanism arithmetic for the B200 chemistry engine.
//
// Every function here evaluates the same formulas as the reference's
// CEPTR-generated Mechanisms/<mech>/mechanism.H (productionRate, aJacobian,
// NASA-7 thermo, GET_T_GIVEN_EY/HY) from data tables instead of straight-line
// code, so one compiled kernel serves every mechanism of a given species
// count.  The functions are written for a "team" of TEAM lanes that share one
// cell: TEAM == 1 is one thread per cell (the plain path), TEAM == 32 is one
// warp per cell (the tuned path).  Per-cell vectors live in memory shared by
// the team (shared memory for TEAM > 1, thread-local memory for TEAM == 1);
// lane l owns entries l, l+TEAM, ...  Team reductions use xor-butterflies so
// every lane ends with a bitwise-identical scalar, which keeps the control
// flow of the integrator uniform across the team.
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "mech/mech_tables.h"

namespace ppb {
// Out-of-line exp / log / log10: one copy of each per kernel instead of one
// per call site, for kernels bound by instruction fetch (measured +8 % drm19
// throughput over the inlined forms without the block rendezvous).
#ifndef PPB_MATH_ATTR
#define PPB_MATH_ATTR __noinline__
#endif
static __device__ PPB_MATH_ATTR double ppb_exp(double x) { return ::exp(x); }
static __device__ PPB_MATH_ATTR double ppb_log(double x) { return ::log(x); }
static __device__ PPB_MATH_ATTR double ppb_log10(double x) { return ::log10(x); }


constexpr double RU = 8.31446261815324e7; // erg/(mol K), PhysicsConstants.H:11

// Device copy of PPBMechTables (same layout) plus the species-major gather
// lists used to sum reaction rates into species rates without atomics.
struct DevMech {
  int nsp, nrxn;
  int nqss, nrq; // QSS species and reactions with one (PPBMechTables)
  const double *mw, *imw, *tmid;
  const double *th_cv, *th_cp, *th_dcp, *th_u, *th_h, *th_g;
  const int *rx_kind, *rx_rev, *rx_kcpow;
  const double *rx_A, *rx_beta, *rx_EaR, *rx_sum_nuk;
  const int *fps_n, *fps_sp;
  const double* fps_c;
  const int *rps_n, *rps_sp;
  const double* rps_c;
  const int *kc_n, *kc_sp;
  const double* kc_c;
  const int *wup_n, *wup_sp;
  const double* wup_c;
  const int *jn_n, *jn_sp;
  const double* jn_c;
  const int *hr_n, *hr_sp;
  const double* hr_c;
  const int *hp_n, *hp_sp;
  const double* hp_c;
  const int *eff_off, *eff_sp;
  const double *eff_e, *eff_m1;
  const double* fo_d;
  const int* fo_i;
  // species-major gather of the productionRate updates: for species s,
  // entries g in [wg_off[s], wg_off[s+1]) add wg_c[g] * qdot[wg_rx[g]]
  const int *wg_off, *wg_rx;
  const double* wg_c;
  // packed per-reaction records (see RxPack) for the warp-cooperative paths
  const struct RxPack* rxp;
  const struct FoPack* fop;
  const unsigned* effmask; // 4 words per reaction: species with a listed efficiency
  const double* effd;      // [third-body reactions][nsp] efficiencies, 1 where unlisted
  // per species k, in reaction order, the reactions whose Jacobian row
  // d q_r / d c_k can be nonzero: every third-body / fall-off reaction and
  // the reactions with k in their forward or (reversible) reverse phase space
  const int* jc_off;
  const unsigned short* jc_rx;
  // per species k, in reaction order, the reactions with k in their forward
  // or (reversible) reverse phase space; and the third-body / fall-off
  // reactions (al_off = {0, count})
  const int* jm_off;
  const unsigned short* jm_rx;
  const int* al_off;
  const unsigned short* al_rx;
  // species-major gather of the aJacobian net stoichiometry (jn lists)
  const int *jg_off, *jg_rx;
  const double* jg_c;
  // SRK equation of state: [sqrt(1/Tc) | sqrt(a*) | B | F(omega)], N each
  const double* srk;
  // QSS balance (PPBMechTables: q_rx, q_off, q_term, q_role, q_coef,
  // rx_rmfwd); the thermo arrays then have an entry per concentration slot
  const int *q_rx, *q_off, *q_term, *q_role;
  const double* q_coef;
  const int* rx_rmfwd;
};

// One reaction in 80 bytes (5 x 16-byte loads).  Species lists are expanded
// by order and padded with the index nsp, whose concentration slot holds 1.0
// and whose g/RT and h/RT slots hold 0.
struct alignas(16) RxPack {
  double A, beta, EaR;     // SI pre-exponential, exponent, Ea/R
  unsigned char fsp[4];    // forward phase space (reactants + explicit collider)
  unsigned char rsp[8];    // reverse phase space
  unsigned char kcs[6];    // Gibbs terms of the equilibrium exponent
  signed char kcc[6];
  unsigned char jns[6];    // aJacobian net stoichiometry
  signed char jnc[6];
  unsigned char kind, rev; // PPB_RX_*, reversible
  signed char kcpow;       // power of 1/refC
  signed char sum_nuk;     // (#products - #reactants) incl. collider
  unsigned char fo;        // fall-off record, 255 = none
  unsigned char nf, nr, njn;
  unsigned short eff0, effn; // efficiency list
  unsigned short aslot;      // row of the dense efficiency table (effd)
  unsigned char rmf;         // forward rate removed by the QSS reduction (qdot = -q_r)
  unsigned char pad;
};
static_assert(sizeof(RxPack) == 80, "RxPack is five 16-byte words");

struct alignas(16) FoPack {
  double P0, k0, beta0, EaR0, prdim, a, T3, T1, T2, oma, iT3, iT1;
  unsigned char ntroe, p1, p2, j1, j2, j3, lindemann, pad[9];
};
static_assert(sizeof(FoPack) == 112, "FoPack is seven 16-byte words");

// A team of TEAM lanes integrates one cell: TEAM = 1 (one thread), 16 or 32
// (part of or a whole warp: shuffles and __syncwarp), or 64 / 128 (several
// warps, one team per block: warp shuffles, then the warps' partial results
// through a small shared scratch and __syncthreads).  Every reduction returns
// the same bits on every lane (fixed combination order).
// The block-shared scratch of a multi-warp team (2 * warps doubles); warp
// teams carry none.
template <int TEAM, bool MULTI = (TEAM > 32)>
struct TeamScratch {
  __device__ __forceinline__ TeamScratch(double*) {}
};
template <int TEAM>
struct TeamScratch<TEAM, true> {
  double* red;
  __device__ __forceinline__ TeamScratch(double* s) : red(s) {}
};

template <int TEAM>
struct Team : TeamScratch<TEAM> {
  static constexpr int W = TEAM < 32 ? TEAM : 32; // lanes per warp in the team
  static constexpr int NW = TEAM > 32 ? TEAM / 32 : 1;
  int lane;
  unsigned mask;
  __device__ __forceinline__ Team(double* scratch = nullptr) : TeamScratch<TEAM>(scratch)
  {
    lane = (TEAM == 1) ? 0 : (int)(threadIdx.x % TEAM);
    if (TEAM >= 32) {
      mask = 0xffffffffu;
    } else if (TEAM == 1) {
      mask = 1u << (threadIdx.x % 32);
    } else {
      mask = ((1u << (TEAM & 31)) - 1u) << ((threadIdx.x % 32) / TEAM * TEAM);
    }
  }
  __device__ __forceinline__ void sync() const
  {
    if (TEAM > 32) {
      __syncthreads();
    } else if (TEAM > 1) {
      __syncwarp(mask);
    }
  }
  template <typename T, typename Op>
  __device__ __forceinline__ T reduce(T x, Op op) const
  {
#pragma unroll
    for (int o = W / 2; o > 0; o >>= 1) x = op(x, __shfl_xor_sync(mask, x, o, W));
    if constexpr (TEAM > 32) {
      T* r = reinterpret_cast<T*>(this->red);
      if ((lane & 31) == 0) r[lane >> 5] = x;
      __syncthreads();
      x = r[0];
#pragma unroll
      for (int i = 1; i < NW; i++) x = op(x, r[i]);
      __syncthreads();
    }
    return x;
  }
  // warp teams: plain xor butterflies (the multi-warp path adds the
  // cross-warp step of reduce)
  __device__ __forceinline__ double sum(double x) const
  {
    if constexpr (TEAM <= 32) {
#pragma unroll
      for (int o = TEAM / 2; o > 0; o >>= 1) x += __shfl_xor_sync(mask, x, o, TEAM);
      return x;
    } else {
      return reduce(x, [](double a, double b) { return a + b; });
    }
  }
  __device__ __forceinline__ double max(double x) const
  {
    if constexpr (TEAM <= 32) {
#pragma unroll
      for (int o = TEAM / 2; o > 0; o >>= 1) x = fmax(x, __shfl_xor_sync(mask, x, o, TEAM));
      return x;
    } else {
      return reduce(x, [](double a, double b) { return fmax(a, b); });
    }
  }
  __device__ __forceinline__ int imax(int x) const
  {
    if constexpr (TEAM <= 32) {
#pragma unroll
      for (int o = TEAM / 2; o > 0; o >>= 1) x = ::max(x, __shfl_xor_sync(mask, x, o, TEAM));
      return x;
    } else {
      return reduce(x, [](int a, int b) { return ::max(a, b); });
    }
  }
  // broadcast from team lane src
  __device__ __forceinline__ double bcast(double x, int src) const
  {
    if constexpr (TEAM == 1) {
      return x;
    } else if constexpr (TEAM <= 32) {
      return __shfl_sync(mask, x, src, TEAM);
    } else {
      if (lane == src) this->red[0] = x;
      __syncthreads();
      const double v = this->red[0];
      __syncthreads();
      return v;
    }
  }
  __device__ __forceinline__ int bcast_int(int x, int src) const
  {
    if constexpr (TEAM == 1) {
      return x;
    } else if constexpr (TEAM <= 32) {
      return __shfl_sync(mask, x, src, TEAM);
    } else {
      int* r = reinterpret_cast<int*>(this->red);
      if (lane == src) r[0] = x;
      __syncthreads();
      const int v = r[0];
      __syncthreads();
      return v;
    }
  }
  // largest best over the team, ties to the smallest index bi
  __device__ __forceinline__ void argmax(double& best, int& bi) const
  {
    if constexpr (TEAM > 1) {
#pragma unroll
      for (int o = W / 2; o > 0; o >>= 1) {
        const double ob = __shfl_xor_sync(mask, best, o, W);
        const int oi = __shfl_xor_sync(mask, bi, o, W);
        if (ob > best || (ob == best && oi < bi)) {
          best = ob;
          bi = oi;
        }
      }
    }
    if constexpr (TEAM > 32) {
      int* ri = reinterpret_cast<int*>(this->red + NW);
      if ((lane & 31) == 0) {
        this->red[lane >> 5] = best;
        ri[lane >> 5] = bi;
      }
      __syncthreads();
      best = this->red[0];
      bi = ri[0];
#pragma unroll
      for (int i = 1; i < NW; i++) {
        if (this->red[i] > best || (this->red[i] == best && ri[i] < bi)) {
          best = this->red[i];
          bi = ri[i];
        }
      }
      __syncthreads();
    }
  }
};

__device__ __forceinline__ int nasa_range(const DevMech& M, int s, double T)
{
  const double tm = __ldg(M.tmid + s);
  return (tm >= 0.0 && T < tm) ? 0 : 1;
}

// mechanism.H cv_R (thermo.py:516-526)
__device__ __forceinline__ double cv_R(const DevMech& M, int s, double T)
{
  const double* c = M.th_cv + (2 * s + nasa_range(M, s, T)) * 5;
  const double T2 = T * T, T3 = T * T * T, T4 = T * T * T * T;
  return __ldg(c) + __ldg(c + 1) * T + __ldg(c + 2) * T2 + __ldg(c + 3) * T3 + __ldg(c + 4) * T4;
}
// mechanism.H cp_R (thermo.py:549-559)
__device__ __forceinline__ double cp_R(const DevMech& M, int s, double T)
{
  const double* c = M.th_cp + (2 * s + nasa_range(M, s, T)) * 5;
  const double T2 = T * T, T3 = T * T * T, T4 = T * T * T * T;
  return __ldg(c) + __ldg(c + 1) * T + __ldg(c + 2) * T2 + __ldg(c + 3) * T3 + __ldg(c + 4) * T4;
}
// mechanism.H dcvpRdT (thermo.py:561-570)
__device__ __forceinline__ double dcvpRdT(const DevMech& M, int s, double T)
{
  const double* c = M.th_dcp + (2 * s + nasa_range(M, s, T)) * 4;
  const double T2 = T * T, T3 = T * T * T;
  return __ldg(c) + __ldg(c + 1) * T + __ldg(c + 2) * T2 + __ldg(c + 3) * T3;
}
// mechanism.H speciesInternalEnergy, e/RT (thermo.py:625-646)
__device__ __forceinline__ double u_RT(const DevMech& M, int s, double T, double invT)
{
  const double* c = M.th_u + (2 * s + nasa_range(M, s, T)) * 6;
  const double T2 = T * T, T3 = T * T * T, T4 = T * T * T * T;
  return __ldg(c) + __ldg(c + 1) * T + __ldg(c + 2) * T2 + __ldg(c + 3) * T3 + __ldg(c + 4) * T4 +
         __ldg(c + 5) * invT;
}
// mechanism.H speciesEnthalpy, h/RT (thermo.py:649-669)
__device__ __forceinline__ double h_RT(const DevMech& M, int s, double T, double invT)
{
  const double* c = M.th_h + (2 * s + nasa_range(M, s, T)) * 6;
  const double T2 = T * T, T3 = T * T * T, T4 = T * T * T * T;
  return __ldg(c) + __ldg(c + 1) * T + __ldg(c + 2) * T2 + __ldg(c + 3) * T3 + __ldg(c + 4) * T4 +
         __ldg(c + 5) * invT;
}
// mechanism.H gibbs, g/RT (thermo.py:572-595)
__device__ __forceinline__ double g_RT(const DevMech& M, int s, double T, double invT, double logT)
{
  const double* c = M.th_g + (2 * s + nasa_range(M, s, T)) * 7;
  const double T2 = T * T, T3 = T * T * T, T4 = T * T * T * T;
  return __ldg(c) * invT + __ldg(c + 1) + __ldg(c + 2) * logT + __ldg(c + 3) * T + __ldg(c + 4) * T2 +
         __ldg(c + 5) * T3 + __ldg(c + 6) * T4;
}

// Mixture energy (EH=0: CKUBMS, erg/g) or enthalpy (EH=1: CKHBMS) and the
// matching heat capacity (CKCVBS / CKCPBS) of mass fractions Y (team-shared).
template <int TEAM>
__device__ __forceinline__ void mix_e_c(
  const Team<TEAM>& tm, const DevMech& M, int EH, double T, const double* Y, double& e, double& c)
{
  const double invT = 1.0 / T;
  double se = 0.0, sc = 0.0;
  for (int s = tm.lane; s < M.nsp; s += TEAM) {
    const double im = __ldg(M.imw + s);
    const double ys = Y[s];
    se += ys * (EH ? h_RT(M, s, T, invT) : u_RT(M, s, T, invT)) * im;
    sc += ys * (EH ? cp_R(M, s, T) : cv_R(M, s, T)) * im;
  }
  se = tm.sum(se);
  sc = tm.sum(sc);
  const double RT = RU * T;
  e = se * RT;
  c = sc * RU;
}

template <int TEAM>
__device__ __forceinline__ double mix_e(const Team<TEAM>& tm, const DevMech& M, int EH, double T, const double* Y)
{
  const double invT = 1.0 / T;
  double se = 0.0;
  for (int s = tm.lane; s < M.nsp; s += TEAM) {
    se += Y[s] * (EH ? h_RT(M, s, T, invT) : u_RT(M, s, T, invT)) * __ldg(M.imw + s);
  }
  se = tm.sum(se);
  return se * (RU * T);
}

template <int TEAM>
__device__ __forceinline__ double mix_c(const Team<TEAM>& tm, const DevMech& M, int EH, double T, const double* Y)
{
  double sc = 0.0;
  for (int s = tm.lane; s < M.nsp; s += TEAM) {
    sc += Y[s] * (EH ? cp_R(M, s, T) : cv_R(M, s, T)) * __ldg(M.imw + s);
  }
  sc = tm.sum(sc);
  return sc * RU;
}

// mechanism.H GET_T_GIVEN_EY / GET_T_GIVEN_HY: Newton from the supplied T,
// |step| <= 100 K, stop at |dT| < 1e-6 K, <= 200 iterations, linear
// extrapolation outside [90, 4000] K (returns 1 there).  When the supplied T
// lies in [90, 4000] K (the integrator's case: it is the previous T), the
// bounds' energies and the first Newton iterate's energy and heat capacity
// are summed in one pass over the species; every sum is formed in the order
// mix_e / mix_e_c form it.
template <int TEAM>
__device__ int t_from_energy(const Team<TEAM>& tm, const DevMech& M, int EH, double e, const double* Y, double& t)
{
  const double tmin = 90, tmax = 4000;
  double t1 = t;
  double emin, emax, e1 = 0.0, cv1 = 0.0;
  const bool fused = !(t1 < tmin || t1 > tmax);
  if (fused) {
    const double imin = 1.0 / tmin, imax = 1.0 / tmax, i1 = 1.0 / t1;
    double smin = 0.0, smax = 0.0, se = 0.0, sc = 0.0;
    for (int s = tm.lane; s < M.nsp; s += TEAM) {
      const double im = __ldg(M.imw + s);
      const double ys = Y[s];
      smin += Y[s] * (EH ? h_RT(M, s, tmin, imin) : u_RT(M, s, tmin, imin)) * im;
      smax += Y[s] * (EH ? h_RT(M, s, tmax, imax) : u_RT(M, s, tmax, imax)) * im;
      se += ys * (EH ? h_RT(M, s, t1, i1) : u_RT(M, s, t1, i1)) * im;
      sc += ys * (EH ? cp_R(M, s, t1) : cv_R(M, s, t1)) * im;
    }
    smin = tm.sum(smin);
    smax = tm.sum(smax);
    se = tm.sum(se);
    sc = tm.sum(sc);
    emin = smin * (RU * tmin);
    emax = smax * (RU * tmax);
    e1 = se * (RU * t1);
    cv1 = sc * RU;
  } else {
    emin = mix_e(tm, M, EH, tmin, Y);
    emax = mix_e(tm, M, EH, tmax, Y);
  }
  if (e < emin) {
    t = tmin - (emin - e) / mix_c(tm, M, EH, tmin, Y);
    return 1;
  }
  if (e > emax) {
    t = tmax - (emax - e) / mix_c(tm, M, EH, tmax, Y);
    return 1;
  }
  if (!fused) t1 = tmin + (tmax - tmin) / (emax - emin) * (e - emin);
  for (int i = 0; i < 200; ++i) {
    double ec, cv;
    if (i == 0 && fused) {
      ec = e1;
      cv = cv1;
    } else {
      mix_e_c(tm, M, EH, t1, Y, ec, cv);
    }
    double dt = (e - ec) / cv;
    if (dt > 100.) {
      dt = 100.;
    } else if (dt < -100.) {
      dt = -100.;
    } else if (fabs(dt) < 1.e-6) {
      break;
    }
    t1 += dt;
  }
  t = t1;
  return 0;
}

__device__ __forceinline__ double phase_space(const int* sp, const double* c, int n, const double* sc)
{
  double p = 1.0;
  for (int j = 0; j < n; j++) {
    const double x = sc[__ldg(sp + j)];
    const int o = (int)__ldg(c + j);
    double t = x;
    for (int q = 1; q < o; q++) t *= x;
    p *= t;
  }
  return p;
}

__device__ __forceinline__ double refc_pow(int p, double refC, double refCinv)
{
  double r = 1.0;
  for (int q = 0; q < p; q++) r *= refCinv;
  for (int q = 0; q < -p; q++) r *= refC;
  return r;
}

// Net rate of progress of reaction r as the reference's productionRate
// computes it (production.py:991-1435); optionally returns q_f and q_r.
__device__ __forceinline__ double rxn_qdot(
  const DevMech& M, int r, double T, double invT, double logT, double refC, double refCinv, double mixture,
  const double* sc, const double* g, double* qf_out = nullptr, double* qr_out = nullptr)
{
  const int kind = __ldg(M.rx_kind + r);
  const double k_f = __ldg(M.rx_A + r) * ppb_exp(__ldg(M.rx_beta + r) * logT - __ldg(M.rx_EaR + r) * invT);
  double Corr = 1.0;
  const bool corr = (kind == PPB_RX_THIRD || kind == PPB_RX_TROE || kind == PPB_RX_LINDEMANN);
  if (corr) {
    Corr = mixture;
    const int e1 = __ldg(M.eff_off + r + 1);
    for (int e = __ldg(M.eff_off + r); e < e1; e++) {
      const double m1 = __ldg(M.eff_m1 + e);
      if (m1 != 0.0) Corr += m1 * sc[__ldg(M.eff_sp + e)];
    }
  }
  if (kind == PPB_RX_TROE || kind == PPB_RX_LINDEMANN) {
    const double* fd = M.fo_d + r * PPB_NFOD;
    const int* fi = M.fo_i + r * PPB_NFOI;
    const double redP =
      Corr / k_f * __ldg(fd + PPB_FO_P0) * ppb_exp(__ldg(fd + PPB_FO_BETA0) * logT - __ldg(fd + PPB_FO_EAR0) * invT);
    const double F = redP / (1.0 + redP);
    if (kind == PPB_RX_TROE) {
      const double logPred = ppb_log10(redP);
      double fc = 0.0;
      if (__ldg(fi + PPB_FOI_P1)) fc = __ldg(fd + PPB_FO_OMA) * ppb_exp(-T * __ldg(fd + PPB_FO_IT3));
      if (__ldg(fi + PPB_FOI_P2)) fc += __ldg(fd + PPB_FO_A) * ppb_exp(-T * __ldg(fd + PPB_FO_IT1));
      if (__ldg(fi + PPB_FOI_NTROE) == 4) fc += ppb_exp(-__ldg(fd + PPB_FO_T2) * invT);
      const double logFcent = ppb_log10(fc);
      const double troe_c = -0.4 - 0.67 * logFcent;
      const double troe_n = 0.75 - 1.27 * logFcent;
      const double troe = (troe_c + logPred) / (troe_n - 0.14 * (troe_c + logPred));
      const double F_troe = ppb_exp(M_LN10 * logFcent / (1.0 + troe * troe));
      Corr = F * F_troe;
    } else {
      Corr = F;
    }
  }
  const double phf = phase_space(M.fps_sp + r * PPB_MAXPS, M.fps_c + r * PPB_MAXPS, __ldg(M.fps_n + r), sc);
  const double qf = corr ? Corr * k_f * phf : k_f * phf;
  double qr = 0.0;
  if (__ldg(M.rx_rev + r)) {
    double arg = 0.0;
    const int nk = __ldg(M.kc_n + r);
    for (int j = 0; j < nk; j++) arg += __ldg(M.kc_c + r * PPB_MAXKC + j) * g[__ldg(M.kc_sp + r * PPB_MAXKC + j)];
    const double phr = phase_space(M.rps_sp + r * PPB_MAXPS, M.rps_c + r * PPB_MAXPS, __ldg(M.rps_n + r), sc);
    qr = (corr ? Corr * k_f : k_f) * ppb_exp(-arg) * refc_pow(__ldg(M.rx_kcpow + r), refC, refCinv) * phr;
  }
  // a forward rate the QSS reduction removed counts 0 (qdot = -q_r)
  const double qfe = (M.nqss > 0 && __ldg(M.rx_rmfwd + r)) ? 0.0 : qf;
  if (qf_out) *qf_out = qfe;
  if (qr_out) *qr_out = qr;
  return qfe - qr;
}

__device__ __forceinline__ RxPack load_rx(const DevMech& M, int r)
{
  RxPack p;
  const int4* src = reinterpret_cast<const int4*>(M.rxp + r);
  int4* dst = reinterpret_cast<int4*>(&p);
#pragma unroll
  for (int i = 0; i < 5; i++) dst[i] = __ldg(src + i);
  return p;
}

__device__ __forceinline__ FoPack load_fo(const DevMech& M, int f)
{
  FoPack p;
  const int4* src = reinterpret_cast<const int4*>(M.fop + f);
  int4* dst = reinterpret_cast<int4*>(&p);
#pragma unroll
  for (int i = 0; i < 7; i++) dst[i] = __ldg(src + i);
  return p;
}

// Slot lists are sorted by species with repeats adjacent (a species of
// order o fills o slots); the helpers walk them run by run so that each
// product is formed exactly as from the (species, order) lists.  Every slot
// index is a compile-time constant (the loops unroll), so a packed record
// stays in registers.

// Phase space: product over runs of x^o, as phase_space() forms it.
template <int K>
__device__ __forceinline__ double slots_product(const unsigned char (&sp)[K], const double* sc)
{
  double p = 1.0, t = 1.0;
#pragma unroll
  for (int i = 0; i < K; i++) {
    const double x = sc[sp[i]];
    if (i == 0) {
      t = x;
    } else if (sp[i] != sp[i - 1]) {
      p *= t;
      t = x;
    } else {
      t *= x;
    }
  }
  return p * t;
}

// d(phase space)/d sc[k], as dphase() forms it (jacobian.py:1398-1515): a run
// of species k of order o multiplies by o and then o-1 times by x (nothing
// for o = 1), another run by x^o.
template <int K>
__device__ __forceinline__ double slots_dproduct(const unsigned char (&sp)[K], const double* sc, int k)
{
  double p = 1.0;
#pragma unroll
  for (int i = 0; i < K; i++) {
    if (i > 0 && sp[i] == sp[i - 1]) continue; // not the start of a run
    int c = 1;
#pragma unroll
    for (int q = i + 1; q < K; q++)
      if (q == i + c && sp[q] == sp[i]) c++;
    const double x = sc[sp[i]];
    if (sp[i] == k) {
      if (c > 1) {
        p *= (double)c;
        for (int q = 1; q < c; q++) p *= x;
      }
    } else {
      double t = x;
      for (int q = 1; q < c; q++) t *= x;
      p *= t;
    }
  }
  return p;
}

// Sum over runs of o * h[species] (the enthalpy sums of dKc/dT).
template <int K>
__device__ __forceinline__ double slots_hsum(const unsigned char (&sp)[K], const double* h)
{
  double s = 0.0, v = 0.0;
  int c = 0;
#pragma unroll
  for (int i = 0; i < K; i++) {
    const bool start = (i == 0) || (sp[i] != sp[i - 1]);
    if (start) {
      if (i > 0) s += (c == 1) ? v : (double)c * v;
      v = h[sp[i]];
      c = 1;
    } else {
      c++;
    }
  }
  return s + ((c == 1) ? v : (double)c * v);
}

template <int K>
__device__ __forceinline__ bool slots_has(const unsigned char (&sp)[K], int k)
{
  bool h = false;
#pragma unroll
  for (int j = 0; j < K; j++) h |= (sp[j] == k);
  return h;
}

// Rates of progress q_f, q_r from a packed record (same formulas as
// rxn_qdot).
__device__ __forceinline__ void rx_rates_packed(
  const DevMech& M, const RxPack& p, double T, double invT, double logT, double refC, double refCinv, double mixture,
  const double* sc, const double* g, double& qf_out, double& qr_out)
{
  const int kind = p.kind;
  const double k_f = p.A * ppb_exp(p.beta * logT - p.EaR * invT);
  double Corr = 1.0;
  const bool corr = (kind == PPB_RX_THIRD || kind == PPB_RX_TROE || kind == PPB_RX_LINDEMANN);
  if (corr) {
    Corr = mixture;
    for (int e = p.eff0; e < p.eff0 + p.effn; e++) {
      const double m1 = __ldg(M.eff_m1 + e);
      if (m1 != 0.0) Corr += m1 * sc[__ldg(M.eff_sp + e)];
    }
  }
  if (p.fo != 255) {
    const FoPack f = load_fo(M, p.fo);
    const double redP = Corr / k_f * f.P0 * ppb_exp(f.beta0 * logT - f.EaR0 * invT);
    const double F = redP / (1.0 + redP);
    if (!f.lindemann) {
      const double logPred = ppb_log10(redP);
      double fc = 0.0;
      if (f.p1) fc = f.oma * ppb_exp(-T * f.iT3);
      if (f.p2) fc += f.a * ppb_exp(-T * f.iT1);
      if (f.ntroe == 4) fc += ppb_exp(-f.T2 * invT);
      const double logFcent = ppb_log10(fc);
      const double troe_c = -0.4 - 0.67 * logFcent;
      const double troe_n = 0.75 - 1.27 * logFcent;
      const double troe = (troe_c + logPred) / (troe_n - 0.14 * (troe_c + logPred));
      const double F_troe = ppb_exp(M_LN10 * logFcent / (1.0 + troe * troe));
      Corr = F * F_troe;
    } else {
      Corr = F;
    }
  }
  const double phf = slots_product(p.fsp, sc);
  const double qf = corr ? Corr * k_f * phf : k_f * phf;
  double qr = 0.0;
  if (p.rev) {
    double arg = 0.0;
#pragma unroll
    for (int j = 0; j < 6; j++) arg += (double)p.kcc[j] * g[p.kcs[j]];
    const double phr = slots_product(p.rsp, sc);
    qr = (corr ? Corr * k_f : k_f) * ppb_exp(-arg) * refc_pow(p.kcpow, refC, refCinv) * phr;
  }
  qf_out = p.rmf ? 0.0 : qf;
  qr_out = qr;
}

// Net rate of progress from a packed record.
__device__ __forceinline__ double rx_qdot_packed(
  const DevMech& M, const RxPack& p, double T, double invT, double logT, double refC, double refCinv, double mixture,
  const double* sc, const double* g)
{
  double qf, qr;
  rx_rates_packed(M, p, T, invT, logT, refC, refCinv, mixture, sc, g, qf, qr);
  return qf - qr;
}

// Scratch doubles of the QSS solve: the coefficients q_f,k, q_r,k (2 nrq)
// and the balance matrix with its right-hand side (nqss (nqss + 1)).
__host__ __device__ inline size_t qss_scratch_doubles(int nqss, int nrq)
{
  return nqss > 0 ? 2 * (size_t)nrq + (size_t)nqss * (nqss + 1) : 0;
}

// The QSS concentrations of a QSS mechanism into the slots sc[nsp + 1 + q]
// (comp_qss_coeff and comp_sc_qss of the reference's generated QSS
// mechanism.H), given sc[0..nsp] (sc[nsp] = 1) and g[0..nsp] (g[nsp] = 0);
// it writes g/RT of the QSS slots too.  With the QSS slots at 1 the QSS
// reactions' rates are their coefficients q_f,k, q_r,k; per QSS species i,
// in reaction order, the production P_i = eps + sum, the loss D_i = eps -
// sum and the couplings C_ij = (eps + sum) / D_i (eps = 1e-12, where the
// generated code adds it); then x_i + sum_j C_ij x_j = -P_i / D_i is solved
// by elimination in species order without pivoting (the loss of a species
// includes its conversions into the others, so the matrix is
// column-diagonally dominant), one lane per row, and back substitution.
template <int TEAM>
__device__ void qss_solve(const Team<TEAM>& tm, const DevMech& M, double* sc, double* g, double T, double invT,
                          double logT, double refC, double refCinv, double mixture, double* co, double* A)
{
  const int N = M.nsp, Q = M.nqss, K = M.nrq, W = Q + 1;
  constexpr double eps = 1e-12;
  for (int q = tm.lane; q < Q; q += TEAM) {
    g[N + 1 + q] = g_RT(M, N + 1 + q, T, invT, logT);
    sc[N + 1 + q] = 1.0;
  }
  tm.sync();
  for (int k = tm.lane; k < K; k += TEAM) {
    const RxPack p = load_rx(M, __ldg(M.q_rx + k));
    double qf, qr;
    rx_rates_packed(M, p, T, invT, logT, refC, refCinv, mixture, sc, g, qf, qr);
    co[2 * k] = qf;
    co[2 * k + 1] = qr;
  }
  tm.sync();
  for (int i = tm.lane; i < Q; i += TEAM) {
    double* row = A + i * W;
    for (int j = 0; j < Q; j++) row[j] = 0.0;
    unsigned has = 0u; // couplings present (at most 32 QSS species)
    double P = eps, D = eps;
    const int t1 = __ldg(M.q_off + i + 1);
    for (int t = __ldg(M.q_off + i); t < t1; t++) {
      const double cf = __ldg(M.q_coef + t);
      const double v = cf == 1.0 ? co[__ldg(M.q_term + t)] : cf * co[__ldg(M.q_term + t)];
      const int role = __ldg(M.q_role + t);
      if (role == -1) {
        P += v;
      } else if (role == -2) {
        D -= v;
      } else {
        if (!((has >> role) & 1u)) {
          row[role] = eps;
          has |= 1u << role;
        }
        row[role] += v;
      }
    }
    for (int j = 0; j < Q; j++)
      if ((has >> j) & 1u) row[j] = row[j] / D;
    row[i] = 1.0;
    row[Q] = -P / D;
  }
  tm.sync();
  for (int c = 0; c < Q; c++) {
    for (int i = c + 1 + tm.lane; i < Q; i += TEAM) {
      const double f = A[i * W + c] / A[c * W + c];
      if (f != 0.0)
        for (int j = c; j <= Q; j++) A[i * W + j] -= f * A[c * W + j];
    }
    tm.sync();
  }
  if (tm.lane == 0) {
    for (int i = Q - 1; i >= 0; i--) {
      double x = A[i * W + Q];
      for (int j = i + 1; j < Q; j++) x -= A[i * W + j] * sc[N + 1 + j];
      sc[N + 1 + i] = x / A[i * W + i];
    }
  }
  tm.sync();
}

// Per-cell scratch for the rate evaluation (team-shared).
struct RateScratch {
  double* sc;           // [nsp + 1 (+ nqss)] SI concentrations (+ the unit slot, the QSS slots)
  double* g;            // [nsp + 1 (+ nqss)] g/RT (+ the unit slot, the QSS slots)
  double* qd;           // [nrxn] net rates (TEAM > 1)
  double* jx = nullptr; // [4 nrxn] per-reaction Jacobian factors (TEAM > 1)
  double* qco = nullptr; // QSS scratch (qss_scratch_doubles), for a QSS mechanism
};

// The reactions and the species gather of productionRate for a team of
// lanes (TEAM > 1), given g/RT in rs.g (0 in the padding slot), sc with 1 in
// its padding slot, and the temperature terms and mixture concentration.
template <int TEAM>
__device__ __forceinline__ void production_rate_core(const Team<TEAM>& tm, const DevMech& M, double* wdot,
                                                     const double* sc_in, double T, double invT, double logT,
                                                     double refC, double refCinv, double mixture, RateScratch& rs)
{
  for (int r = tm.lane; r < M.nrxn; r += TEAM) {
    const RxPack p = load_rx(M, r);
    rs.qd[r] = rx_qdot_packed(M, p, T, invT, logT, refC, refCinv, mixture, sc_in, rs.g);
  }
  tm.sync();
  for (int s = tm.lane; s < M.nsp; s += TEAM) {
    double w = 0.0;
    const int g1 = __ldg(M.wg_off + s + 1);
    for (int gi = __ldg(M.wg_off + s); gi < g1; gi++) w += __ldg(M.wg_c + gi) * rs.qd[__ldg(M.wg_rx + gi)];
    wdot[s] = w;
  }
  tm.sync();
}

// productionRate (SI): wdot[s] for s owned by the lane (team-shared wdot).
// sc_in[nsp] holds 1 (the unit slot); for a QSS mechanism the QSS slots of
// sc_in are solved first (qss_solve, with rs.qco as scratch).
template <int TEAM>
__device__ void production_rate(
  const Team<TEAM>& tm, const DevMech& M, double* wdot, double* sc_in, double T, RateScratch& rs)
{
  const double invT = 1.0 / T;
  const double logT = ppb_log(T);
  const double refC = 101325 / 8.31446 * invT;
  const double refCinv = 1 / refC;
  double mix = 0.0;
  for (int s = tm.lane; s < M.nsp; s += TEAM) {
    mix += sc_in[s];
    rs.g[s] = g_RT(M, s, T, invT, logT);
  }
  const double mixture = tm.sum(mix);
  tm.sync();
  if (M.nqss > 0) {
    if (tm.lane == 0) rs.g[M.nsp] = 0.0;
    tm.sync();
    qss_solve<TEAM>(tm, M, sc_in, rs.g, T, invT, logT, refC, refCinv, mixture, rs.qco, rs.qco + 2 * M.nrq);
  }
  if (TEAM == 1) {
    for (int s = 0; s < M.nsp; s++) wdot[s] = 0.0;
    for (int r = 0; r < M.nrxn; r++) {
      const double qdot = rxn_qdot(M, r, T, invT, logT, refC, refCinv, mixture, sc_in, rs.g);
      const int nw = __ldg(M.wup_n + r);
      for (int j = 0; j < nw; j++) {
        const int s = __ldg(M.wup_sp + r * PPB_MAXW + j);
        const double c = __ldg(M.wup_c + r * PPB_MAXW + j);
        if (c == -1.0) {
          wdot[s] -= qdot;
        } else if (c == 1.0) {
          wdot[s] += qdot;
        } else if (c < 0) {
          wdot[s] -= (-c) * qdot;
        } else {
          wdot[s] += c * qdot;
        }
      }
    }
  } else {
    // padding slots of the packed records: sc[nsp] = 1 (set by the caller),
    // g[nsp] = 0
    if (tm.lane == 0) rs.g[M.nsp] = 0.0;
    tm.sync();
    production_rate_core(tm, M, wdot, sc_in, T, invT, logT, refC, refCinv, mixture, rs);
    return;
  }
  tm.sync();
}

__device__ __forceinline__ bool has_sp(const int* sp, int n, int k)
{
  for (int j = 0; j < n; j++)
    if (__ldg(sp + j) == k) return true;
  return false;
}

__device__ __forceinline__ double dphase(const int* sp, const double* c, int n, const double* sc, int k)
{
  double p = 1.0;
  for (int j = 0; j < n; j++) {
    const double x = sc[__ldg(sp + j)];
    const int o = (int)__ldg(c + j);
    if (__ldg(sp + j) == k) {
      if (o > 1) {
        p *= (double)o;
        for (int q = 1; q < o; q++) p *= x;
      }
    } else {
      double t = x;
      for (int q = 1; q < o; q++) t *= x;
      p *= t;
    }
  }
  return p;
}

// Temperature row and column of the Jacobian (jacobian.py:203-281) from the
// species columns, wdot and the d/dT row.
template <int TEAM>
__device__ void ajacobian_trow(
  const Team<TEAM>& tm, const DevMech& M, double* J, const double* sc, double T, int consP, const double* wdot,
  const double* hrt, double* crt, double* dcrt, double* ehrt)
{
  const int N = M.nsp, n = N + 1;
  const double invT = 1.0 / T;
  double a_cmix = 0.0, a_ehmix = 0.0, a_dcmix = 0.0, a_dehmix = 0.0;
  for (int s = tm.lane; s < N; s += TEAM) {
    const double cr = consP ? cp_R(M, s, T) : cv_R(M, s, T);
    const double dc = dcvpRdT(M, s, T);
    const double eh = consP ? hrt[s] : u_RT(M, s, T, invT);
    crt[s] = cr;
    dcrt[s] = dc;
    ehrt[s] = eh;
    a_cmix += cr * sc[s];
    a_dcmix += dc * sc[s];
    a_ehmix += eh * wdot[s];
    a_dehmix += invT * (cr - eh) * wdot[s] + eh * J[N * n + s];
  }
  const double cmix = tm.sum(a_cmix);
  const double dcmixdT = tm.sum(a_dcmix);
  const double ehmix = tm.sum(a_ehmix);
  const double dehmixdT = tm.sum(a_dehmix);
  tm.sync();
  const double cmixinv = 1.0 / cmix;
  const double tmp1 = ehmix * cmixinv;
  const double tmp3 = cmixinv * T;
  const double tmp2 = tmp1 * tmp3;
  for (int k = tm.lane; k < N; k += TEAM) {
    double dehmixdc = 0.0;
    for (int m = 0; m < N; ++m) dehmixdc += ehrt[m] * J[k * n + m];
    J[k * n + N] = tmp2 * crt[k] - tmp3 * dehmixdc;
  }
  if (tm.lane == 0) J[N * n + N] = -tmp1 + tmp2 * dcmixdT - tmp3 * dehmixdT;
  tm.sync();
}

// Per-reaction factors of the analytical Jacobian (jacobian.py:546-1305)
// from a packed record: the net rate q, dq/dT, the forward and reverse rate
// constants with the third-body / fall-off factor folded in, and the factor
// that multiplies (efficiency - 1) in dq/dc.  Same formulas and operation
// order as the reaction loop of ajacobian().
struct RxJac {
  double q, dqdT, kf, kr, fac;
  double dlnk; // d ln q / d ln k_f at fixed concentrations and T (k_inf for fall-off)
};

__device__ __forceinline__ RxJac rx_jac_packed(
  const DevMech& M, const RxPack& p, double T, double invT, double invT2, double logT, double refC, double refCinv,
  double mixture, const double* sc, const double* g, const double* hrt)
{
  const double ln10 = M_LN10;
  const double log10e = 1.0 / M_LN10;
  const bool falloff = (p.fo != 255);
  const bool has_alpha = (p.kind == PPB_RX_THIRD) || falloff;
  const bool rev = p.rev != 0;
  double alpha = 0.0;
  if (has_alpha) {
    alpha = mixture;
    for (int e = p.eff0; e < p.eff0 + p.effn; e++) {
      const double em1 = __ldg(M.eff_e + e) - 1.0;
      if (em1 != 0.0) alpha += em1 * sc[__ldg(M.eff_sp + e)];
    }
  }
  const double phi_f = slots_product(p.fsp, sc);
  double k_f = p.A * ppb_exp(p.beta * logT - p.EaR * invT);
  const double dlnkfdT = p.beta * invT + p.EaR * invT2;
  double Pr = 0.0, fPr = 0.0, F = 1.0, dlogFdlogPr = 0.0, dlogFdT = 0.0, dlogfPrdT = 0.0;
  if (falloff) {
    const FoPack f = load_fo(M, p.fo);
    const double k_0 = f.k0 * ppb_exp(f.beta0 * logT - f.EaR0 * invT);
    Pr = f.prdim * alpha / k_f * k_0;
    fPr = Pr / (1.0 + Pr);
    const double dlnk0dT = f.beta0 * invT + f.EaR0 * invT2;
    const double dlogPrdT = log10e * (dlnk0dT - dlnkfdT);
    dlogfPrdT = dlogPrdT / (1.0 + Pr);
    if (!f.lindemann) {
      const double logPr = ppb_log10(Pr);
      const double Fcent1 = f.j1 ? (1. - f.a) * ppb_exp(-T / f.T3) : 0.;
      const double Fcent2 = f.j2 ? f.a * ppb_exp(-T / f.T1) : 0.;
      const double Fcent3 = (f.ntroe == 4) ? ppb_exp(-f.T2 * invT) : 0.;
      const double Fcent = Fcent1 + Fcent2 + Fcent3;
      const double logFcent = ppb_log10(Fcent);
      const double troe_c = -.4 - .67 * logFcent;
      const double troe_n = .75 - 1.27 * logFcent;
      const double troePr_den = 1.0 / (troe_n - .14 * (troe_c + logPr));
      const double troePr = (troe_c + logPr) * troePr_den;
      const double troe = 1.0 / (1.0 + troePr * troePr);
      F = ppb_exp(M_LN10 * logFcent * troe);
      double sm = 0.0;
      if (f.j1) sm += -Fcent1 / f.T3;
      if (f.j2) sm += -Fcent2 / f.T1;
      if (f.j3) sm += Fcent3 * f.T2 * invT2;
      const double dlogFcentdT = log10e / Fcent * (sm);
      const double dlogFdcn_fac = 2.0 * logFcent * troe * troe * troePr * troePr_den;
      const double dlogFdc = -troe_n * dlogFdcn_fac * troePr_den;
      const double dlogFdn = dlogFdcn_fac * troePr;
      dlogFdlogPr = dlogFdc;
      dlogFdT = dlogFcentdT * (troe - 0.67 * dlogFdc - 1.27 * dlogFdn) + dlogFdlogPr * dlogPrdT;
    }
  }
  double q, q_nocor = 0.0, Corr = 1.0, dqdT, k_r = 0.0;
  if (!rev) {
    if (!has_alpha) {
      q = k_f * phi_f;
    } else {
      q_nocor = k_f * phi_f;
      if (falloff) {
        Corr = fPr * F;
        q = Corr * q_nocor;
      } else {
        q = alpha * q_nocor;
      }
    }
    if (falloff) {
      dqdT = Corr * dlnkfdT * k_f * phi_f + ln10 * (dlogfPrdT + dlogFdT) * q;
    } else if (has_alpha) {
      dqdT = alpha * dlnkfdT * k_f * phi_f;
    } else {
      dqdT = dlnkfdT * k_f * phi_f;
    }
  } else {
    const double phi_r = slots_product(p.rsp, sc);
    double arg = 0.0;
#pragma unroll
    for (int j = 0; j < 6; j++)
      if (p.kcc[j]) arg += (double)p.kcc[j] * g[p.kcs[j]];
    const double Kc = refc_pow(-p.kcpow, refC, refCinv) * ppb_exp(arg);
    k_r = k_f / Kc;
    const double hsum_r = slots_hsum(p.fsp, hrt);
    const double hsum_p = slots_hsum(p.rsp, hrt);
    const double snk = p.sum_nuk;
    double inner = -(hsum_r) + (hsum_p);
    if (snk > 0) {
      inner -= snk;
    } else if (snk < 0) {
      inner += -snk;
    }
    const double dlnKcdT = invT * (inner);
    const double dkrdT = (dlnkfdT - dlnKcdT) * k_r;
    if (!has_alpha) {
      q = k_f * phi_f - k_r * phi_r;
    } else {
      q_nocor = k_f * phi_f - k_r * phi_r;
      if (falloff) {
        Corr = fPr * F;
        q = Corr * q_nocor;
      } else {
        q = alpha * q_nocor;
      }
    }
    if (falloff) {
      dqdT = Corr * (dlnkfdT * k_f * phi_f - dkrdT * phi_r) + ln10 * (dlogfPrdT + dlogFdT) * q;
    } else if (has_alpha) {
      dqdT = alpha * (dlnkfdT * k_f * phi_f - dkrdT * phi_r);
    } else {
      dqdT = (dlnkfdT * k_f * phi_f - dkrdT * phi_r);
    }
  }
  if (falloff) {
    k_f *= Corr;
    if (rev) k_r *= Corr;
  } else if (has_alpha) {
    k_f *= alpha;
    if (rev) k_r *= alpha;
  }
  RxJac o;
  o.q = q;
  o.dqdT = dqdT;
  o.kf = k_f;
  o.kr = k_r;
  o.fac = falloff ? q / alpha * (1.0 / (Pr + 1.0) + dlogFdlogPr) : q_nocor;
  // fall-off: Pr = alpha k_0 / k_inf, so d ln(Pr/(1+Pr) F(Pr)) / d ln k_inf
  // = -1/(1+Pr) - dlog F/dlog Pr
  o.dlnk = falloff ? Pr / (1.0 + Pr) - dlogFdlogPr : 1.0;
  return o;
}

// Warp-cooperative analytical Jacobian over the packed records, in three
// passes: (1) lanes over reactions compute each reaction's factors (the
// exp/log work) into jx and qd; (2) lanes over species gather wdot and the
// d/dT row in reaction order; (3) the reactions are walked in order while
// lane l updates columns l, l+TEAM, ... -- the same accumulation order into
// each J entry as ajacobian(), including the reuse of a stale dq/dc value
// for a zero-efficiency species without a rate term in the consP == 0 form.
template <int TEAM, int PER>
__device__ void ajacobian_packed(
  const Team<TEAM>& tm, const DevMech& M, double* J, const double* sc, double T, int consP, RateScratch& rs,
  double* wdot, double* hrt, double* crt, double* dcrt, double* ehrt)
{
  const int N = M.nsp, n = N + 1, R = M.nrxn;
  for (int i = tm.lane; i < n * n; i += TEAM) J[i] = 0.0;
  const double invT = 1.0 / T;
  const double invT2 = invT * invT;
  const double logT = ppb_log(T);
  const double refC = 101325 / 8.31446 / T;
  const double refCinv = 1.0 / refC;
  double mix = 0.0;
  for (int s = tm.lane; s < N; s += TEAM) {
    mix += sc[s];
    rs.g[s] = g_RT(M, s, T, invT, logT);
    hrt[s] = h_RT(M, s, T, invT);
  }
  if (tm.lane == 0) {
    rs.g[N] = 0.0;
    hrt[N] = 0.0;
  }
  const double mixture = tm.sum(mix);
  tm.sync();
  // (1) per-reaction factors
  double* jx = rs.jx;
  for (int r = tm.lane; r < R; r += TEAM) {
    const RxPack p = load_rx(M, r);
    const RxJac f = rx_jac_packed(M, p, T, invT, invT2, logT, refC, refCinv, mixture, sc, rs.g, hrt);
    rs.qd[r] = f.q;
    jx[4 * r + 0] = f.kf;
    jx[4 * r + 1] = f.kr;
    jx[4 * r + 2] = f.fac;
    jx[4 * r + 3] = f.dqdT;
  }
  tm.sync();
  // (2) wdot and the d/dT row, reaction order per species
  for (int s = tm.lane; s < N; s += TEAM) {
    double w = 0.0, d = 0.0;
    const int g1 = __ldg(M.jg_off + s + 1);
    for (int gi = __ldg(M.jg_off + s); gi < g1; gi++) {
      const int r = __ldg(M.jg_rx + gi);
      const double nu = __ldg(M.jg_c + gi);
      w += nu * rs.qd[r];
      d += nu * jx[4 * r + 3];
    }
    wdot[s] = w;
    J[N * n + s] = d;
  }
  // (3) species columns: lane l owns columns l, l+TEAM, ... and walks the
  // reactions that reach its column in reaction order (the per-entry
  // accumulation order of the generated code; dq carries the last dq/dc_k of
  // a third-body reaction, which the consP == 0 form reuses for a
  // zero-efficiency species without a rate term)
#pragma unroll
  for (int qq = 0; qq < PER; qq++) {
    const int k = tm.lane + qq * TEAM;
    if (k >= N) break;
    double dq = 0.0;
    double* Jk = J + k * n;
    const unsigned word_i = (unsigned)(k >> 5), bit = 1u << (k & 31);
    const int e1 = __ldg(M.jc_off + k + 1);
    for (int ei = __ldg(M.jc_off + k); ei < e1; ei++) {
      const int r = __ldg(M.jc_rx + ei);
      const RxPack p = load_rx(M, r);
      const bool falloff = (p.fo != 255);
      const bool has_alpha = (p.kind == PPB_RX_THIRD) || falloff;
      const bool rev = p.rev != 0;
      const double k_f = jx[4 * r + 0];
      const double k_r = jx[4 * r + 1];
      const double fac = jx[4 * r + 2];
      const bool inr = slots_has(p.fsp, k);
      const bool inp = rev && slots_has(p.rsp, k);
      double d = 0.0;
      bool apply = false;
      if (has_alpha) {
        const bool listed = (__ldg(M.effmask + 4 * r + word_i) & bit) != 0u;
        const double* ed = M.effd + (size_t)p.aslot * N;
        if (consP == 1) {
          if (listed) {
            d = (__ldg(ed + k) - 1) * fac;
            apply = true;
          }
          if (inr) {
            d += k_f * slots_dproduct(p.fsp, sc, k);
            apply = true;
          }
          if (inp) {
            d -= k_r * slots_dproduct(p.rsp, sc, k);
            apply = true;
          }
        } else {
          const double e = listed ? __ldg(ed + k) : 1.0;
          if (!(e == 0.0 && !inr && !inp)) {
            if (e == 0.0) {
              d = 0.0;
              if (inr) d = k_f * slots_dproduct(p.fsp, sc, k);
              if (inp) d = (inr ? d : 0.0) - k_r * slots_dproduct(p.rsp, sc, k);
            } else {
              d = (e == 1.0) ? fac : e * fac;
              if (inr) d += k_f * slots_dproduct(p.fsp, sc, k);
              if (inp) d -= k_r * slots_dproduct(p.rsp, sc, k);
            }
            dq = d;
          }
          d = dq;
          apply = true;
        }
      } else {
        if (inr) d += k_f * slots_dproduct(p.fsp, sc, k);
        if (inp) d -= k_r * slots_dproduct(p.rsp, sc, k);
        apply = inr || inp;
      }
      if (apply) {
        #pragma unroll
        for (int j = 0; j < 6; j++) { // static slot index: the record stays in registers
          if (j >= p.njn) break;
          const double nu = (double)p.jnc[j];
          if (nu != 0) Jk[p.jns[j]] += nu * d;
        }
      }
    }
  }
  tm.sync();
  ajacobian_trow<TEAM>(tm, M, J, sc, T, consP, wdot, hrt, crt, dcrt, ehrt);
}

// The reference's analytical Jacobian (jacobian.py:12-283, :546-1305), SI,
// column-major J[k*(N+1)+m] = d wdot_m / d sc_k with the temperature row and
// column.  Reactions are visited in order by the whole team; lane l owns
// columns k = l, l+TEAM, ...  The consP == 0 branch reproduces the generated
// code exactly, including its use of dqdc[k] values left over from an
// earlier reaction when a species has zero third-body efficiency and no rate
// term (the generated code never assigns dqdc[k] then but still reads it).
// wdot/hrt/crt/dcrt/ehrt are team-shared scratch of length nsp.
template <int TEAM, int PER>
__device__ void ajacobian(
  const Team<TEAM>& tm, const DevMech& M, double* J, const double* sc, double T, int consP, RateScratch& rs,
  double* wdot, double* hrt, double* crt, double* dcrt, double* ehrt)
{
  if constexpr (TEAM > 1) {
    if (rs.jx) {
      ajacobian_packed<TEAM, PER>(tm, M, J, sc, T, consP, rs, wdot, hrt, crt, dcrt, ehrt);
      return;
    }
  }
  const int N = M.nsp, n = N + 1;
  for (int i = tm.lane; i < n * n; i += TEAM) J[i] = 0.0;
  const double invT = 1.0 / T;
  const double invT2 = invT * invT;
  const double logT = ppb_log(T);
  const double refC = 101325 / 8.31446 / T;
  const double refCinv = 1.0 / refC;
  double mix = 0.0;
  for (int s = tm.lane; s < N; s += TEAM) {
    mix += sc[s];
    rs.g[s] = g_RT(M, s, T, invT, logT);
    hrt[s] = h_RT(M, s, T, invT);
    wdot[s] = 0.0;
  }
  const double mixture = tm.sum(mix);
  tm.sync();
  const double ln10 = M_LN10;
  const double log10e = 1.0 / M_LN10;
  double dq[PER]; // dqdc of the lane's species, carried across reactions
#pragma unroll
  for (int p = 0; p < PER; p++) dq[p] = 0.0;
  for (int r = 0; r < M.nrxn; r++) {
    const int kind = __ldg(M.rx_kind + r);
    const bool falloff = (kind == PPB_RX_TROE || kind == PPB_RX_LINDEMANN);
    const bool has_alpha = (kind == PPB_RX_THIRD) || falloff;
    const bool rev = __ldg(M.rx_rev + r) != 0;
    const int* fsp = M.fps_sp + r * PPB_MAXPS;
    const double* fc = M.fps_c + r * PPB_MAXPS;
    const int fn = __ldg(M.fps_n + r);
    const int* rsp = M.rps_sp + r * PPB_MAXPS;
    const double* rc = M.rps_c + r * PPB_MAXPS;
    const int rn = __ldg(M.rps_n + r);
    const int e0 = __ldg(M.eff_off + r), e1 = __ldg(M.eff_off + r + 1);
    double alpha = 0.0;
    if (has_alpha) {
      alpha = mixture;
      for (int e = e0; e < e1; e++) {
        const double em1 = __ldg(M.eff_e + e) - 1.0;
        if (em1 != 0.0) alpha += em1 * sc[__ldg(M.eff_sp + e)];
      }
    }
    const double phi_f = phase_space(fsp, fc, fn, sc);
    double k_f = __ldg(M.rx_A + r) * ppb_exp(__ldg(M.rx_beta + r) * logT - __ldg(M.rx_EaR + r) * invT);
    const double dlnkfdT = __ldg(M.rx_beta + r) * invT + __ldg(M.rx_EaR + r) * invT2;
    double Pr = 0.0, fPr = 0.0, F = 1.0, dlogFdlogPr = 0.0, dlogFdT = 0.0, dlogfPrdT = 0.0;
    if (falloff) {
      const double* fd = M.fo_d + r * PPB_NFOD;
      const int* fi = M.fo_i + r * PPB_NFOI;
      const double k_0 =
        __ldg(fd + PPB_FO_K0) * ppb_exp(__ldg(fd + PPB_FO_BETA0) * logT - __ldg(fd + PPB_FO_EAR0) * invT);
      Pr = __ldg(fd + PPB_FO_PRDIM) * alpha / k_f * k_0;
      fPr = Pr / (1.0 + Pr);
      const double dlnk0dT = __ldg(fd + PPB_FO_BETA0) * invT + __ldg(fd + PPB_FO_EAR0) * invT2;
      const double dlogPrdT = log10e * (dlnk0dT - dlnkfdT);
      dlogfPrdT = dlogPrdT / (1.0 + Pr);
      if (kind == PPB_RX_TROE) {
        const double a = __ldg(fd + PPB_FO_A), T3 = __ldg(fd + PPB_FO_T3);
        const double T1 = __ldg(fd + PPB_FO_T1), T2 = __ldg(fd + PPB_FO_T2);
        const double logPr = ppb_log10(Pr);
        const double Fcent1 = __ldg(fi + PPB_FOI_J1) ? (1. - a) * ppb_exp(-T / T3) : 0.;
        const double Fcent2 = __ldg(fi + PPB_FOI_J2) ? a * ppb_exp(-T / T1) : 0.;
        const double Fcent3 = (__ldg(fi + PPB_FOI_NTROE) == 4) ? ppb_exp(-T2 * invT) : 0.;
        const double Fcent = Fcent1 + Fcent2 + Fcent3;
        const double logFcent = ppb_log10(Fcent);
        const double troe_c = -.4 - .67 * logFcent;
        const double troe_n = .75 - 1.27 * logFcent;
        const double troePr_den = 1.0 / (troe_n - .14 * (troe_c + logPr));
        const double troePr = (troe_c + logPr) * troePr_den;
        const double troe = 1.0 / (1.0 + troePr * troePr);
        F = ppb_exp(M_LN10 * logFcent * troe);
        double s = 0.0;
        if (__ldg(fi + PPB_FOI_J1)) s += -Fcent1 / T3;
        if (__ldg(fi + PPB_FOI_J2)) s += -Fcent2 / T1;
        if (__ldg(fi + PPB_FOI_J3)) s += Fcent3 * T2 * invT2;
        const double dlogFcentdT = log10e / Fcent * (s);
        const double dlogFdcn_fac = 2.0 * logFcent * troe * troe * troePr * troePr_den;
        const double dlogFdc = -troe_n * dlogFdcn_fac * troePr_den;
        const double dlogFdn = dlogFdcn_fac * troePr;
        dlogFdlogPr = dlogFdc;
        dlogFdT = dlogFcentdT * (troe - 0.67 * dlogFdc - 1.27 * dlogFdn) + dlogFdlogPr * dlogPrdT;
      }
    }
    double q, q_nocor = 0.0, Corr = 1.0, dqdT, k_r = 0.0;
    if (!rev) {
      if (!has_alpha) {
        q = k_f * phi_f;
      } else {
        q_nocor = k_f * phi_f;
        if (falloff) {
          Corr = fPr * F;
          q = Corr * q_nocor;
        } else {
          q = alpha * q_nocor;
        }
      }
      if (falloff) {
        dqdT = Corr * dlnkfdT * k_f * phi_f + ln10 * (dlogfPrdT + dlogFdT) * q;
      } else if (has_alpha) {
        dqdT = alpha * dlnkfdT * k_f * phi_f;
      } else {
        dqdT = dlnkfdT * k_f * phi_f;
      }
    } else {
      const double phi_r = phase_space(rsp, rc, rn, sc);
      double arg = 0.0;
      const int nk = __ldg(M.kc_n + r);
      for (int j = 0; j < nk; j++) arg += __ldg(M.kc_c + r * PPB_MAXKC + j) * rs.g[__ldg(M.kc_sp + r * PPB_MAXKC + j)];
      const double Kc = refc_pow(-__ldg(M.rx_kcpow + r), refC, refCinv) * ppb_exp(arg);
      k_r = k_f / Kc;
      double hsum_r = 0.0, hsum_p = 0.0;
      const int nhr = __ldg(M.hr_n + r), nhp = __ldg(M.hp_n + r);
      for (int j = 0; j < nhr; j++) {
        const double c = __ldg(M.hr_c + r * PPB_MAXPS + j);
        const double h = hrt[__ldg(M.hr_sp + r * PPB_MAXPS + j)];
        hsum_r += (c == 1.0) ? h : c * h;
      }
      for (int j = 0; j < nhp; j++) {
        const double c = __ldg(M.hp_c + r * PPB_MAXPS + j);
        const double h = hrt[__ldg(M.hp_sp + r * PPB_MAXPS + j)];
        hsum_p += (c == 1.0) ? h : c * h;
      }
      const double snk = __ldg(M.rx_sum_nuk + r);
      double inner = -(hsum_r) + (hsum_p);
      if (snk > 0) {
        inner -= snk;
      } else if (snk < 0) {
        inner += -snk;
      }
      const double dlnKcdT = invT * (inner);
      const double dkrdT = (dlnkfdT - dlnKcdT) * k_r;
      if (!has_alpha) {
        q = k_f * phi_f - k_r * phi_r;
      } else {
        q_nocor = k_f * phi_f - k_r * phi_r;
        if (falloff) {
          Corr = fPr * F;
          q = Corr * q_nocor;
        } else {
          q = alpha * q_nocor;
        }
      }
      if (falloff) {
        dqdT = Corr * (dlnkfdT * k_f * phi_f - dkrdT * phi_r) + ln10 * (dlogfPrdT + dlogFdT) * q;
      } else if (has_alpha) {
        dqdT = alpha * (dlnkfdT * k_f * phi_f - dkrdT * phi_r);
      } else {
        dqdT = (dlnkfdT * k_f * phi_f - dkrdT * phi_r);
      }
    }
    const int jnn = __ldg(M.jn_n + r);
    const int* jsp = M.jn_sp + r * PPB_MAXJN;
    const double* jc = M.jn_c + r * PPB_MAXJN;
    // wdot (owned species only) and the d/dT row
    for (int j = 0; j < jnn; j++) {
      const int s = __ldg(jsp + j);
      const double nu = __ldg(jc + j);
      if (s % TEAM == tm.lane) {
        if (nu == 1) {
          wdot[s] += q;
        } else if (nu == -1) {
          wdot[s] -= q;
        } else if (nu > 0) {
          wdot[s] += nu * q;
        } else if (nu < 0) {
          wdot[s] -= (-nu) * q;
        }
        if (nu != 0) J[N * n + s] += nu * dqdT;
      }
    }
    if (falloff) {
      k_f *= Corr;
      if (rev) k_r *= Corr;
    } else if (has_alpha) {
      k_f *= alpha;
      if (rev) k_r *= alpha;
    }
    const double dcdc_fac = falloff ? q / alpha * (1.0 / (Pr + 1.0) + dlogFdlogPr) : 0.0;
    const int* hrs = M.hr_sp + r * PPB_MAXPS;
    const int hrn = __ldg(M.hr_n + r);
    const int* hps = M.hp_sp + r * PPB_MAXPS;
    const int hpn = __ldg(M.hp_n + r);
    const double fac = falloff ? dcdc_fac : q_nocor;
#pragma unroll
    for (int p = 0; p < PER; p++) {
      const int k = tm.lane + p * TEAM;
      if (k >= N) break;
      const bool inr = has_sp(hrs, hrn, k);
      const bool inp = rev && has_sp(hps, hpn, k);
      double d = 0.0;
      bool apply = false;
      if (has_alpha) {
        int ei = -1;
        for (int e = e0; e < e1; e++) {
          if (__ldg(M.eff_sp + e) == k) {
            ei = e;
            break;
          }
        }
        if (consP == 1) {
          if (ei >= 0) {
            d = (__ldg(M.eff_e + ei) - 1) * fac;
            apply = true;
          }
          if (inr) {
            d += k_f * dphase(fsp, fc, fn, sc, k);
            apply = true;
          }
          if (inp) {
            d -= k_r * dphase(rsp, rc, rn, sc, k);
            apply = true;
          }
        } else {
          const double e = (ei >= 0) ? __ldg(M.eff_e + ei) : 1.0;
          if (!(e == 0.0 && !inr && !inp)) {
            if (e == 0.0) {
              d = 0.0;
              if (inr) d = k_f * dphase(fsp, fc, fn, sc, k);
              if (inp) d = (inr ? d : 0.0) - k_r * dphase(rsp, rc, rn, sc, k);
            } else {
              d = (e == 1.0) ? fac : e * fac;
              if (inr) d += k_f * dphase(fsp, fc, fn, sc, k);
              if (inp) d -= k_r * dphase(rsp, rc, rn, sc, k);
            }
            dq[p] = d;
          }
          d = dq[p];
          apply = true;
        }
      } else {
        if (inr) d += k_f * dphase(fsp, fc, fn, sc, k);
        if (inp) d -= k_r * dphase(rsp, rc, rn, sc, k);
        apply = inr || inp;
      }
      if (apply) {
        for (int j = 0; j < jnn; j++) {
          const double nu = __ldg(jc + j);
          if (nu != 0) J[k * n + __ldg(jsp + j)] += nu * d;
        }
      }
    }
  }
  tm.sync();
  ajacobian_trow<TEAM>(tm, M, J, sc, T, consP, wdot, hrt, crt, dcrt, ehrt);
}

} // namespace ppb
