// Soave-Redlich-Kwong equation of state for the e-reactor, team-parallel
// (the reference's Source/Eos/SRK.H, struct SRK).
//
// The mixing rules are double sums over species pairs in the reference
// (MixingRuleAmBm, Calc_dAmdT, Calc_dAmdY, Calc_d2AmdTY, Calc_d2AmdT2,
// SRK.H:53-348); every one factors through two single sums,
//   S1 = sum Y_i a_i(T),  S1' = sum Y_i a_i'(T),
// with a_i = (1 + F_i (1 - sqrt(T / Tc_i))) sqrt(a*_i) and a_i' = da_i/dT:
//   a_m = S1^2, da_m/dT = 2 S1 S1', d2a_m/dT2 = -(1/2T)(-4T S1'^2 + 2 S1 S1'),
//   da_m/dY_i = 2 a_i S1,  d2a_m/dTdY_i = 2 (a_i S1' + a_i' S1),
// so the team evaluates them in O(N) with two reductions (the same values,
// summed in another order).
#pragma once
#include "ppb_mech.cuh"

namespace ppb {

struct SrkState {
  double S1, S1p, bm, am, dAmdT, d2AmdT2, K1;
};

// per-species parameters: M.srk = [sqrt(1/Tc) | sqrt(a*) | B | F(omega)]
template <int TEAM>
__device__ __forceinline__ void srk_sums(const Team<TEAM>& tm, const DevMech& M, double T, double R,
                                         const double* Y, SrkState& s)
{
  const int N = M.nsp;
  const double* P = M.srk;
  const double sqrtT = sqrt(T), oneOverT = 1.0 / T;
  double a1 = 0.0, a2 = 0.0, b = 0.0;
  for (int i = tm.lane; i < N; i += TEAM) {
    const double sOT = __ldg(P + i), sA = __ldg(P + N + i), B = __ldg(P + 2 * N + i), F = __ldg(P + 3 * N + i);
    a1 += Y[i] * ((1.0 + F * (1.0 - sqrtT * sOT)) * sA);
    a2 += Y[i] * (-0.5 * F * sA * oneOverT * sqrtT * sOT);
    b += Y[i] * B;
  }
  s.S1 = tm.sum(a1);
  s.S1p = tm.sum(a2);
  s.bm = tm.sum(b);
  s.am = s.S1 * s.S1;
  s.dAmdT = 2.0 * s.S1 * s.S1p;
  s.d2AmdT2 = (-0.5 * oneOverT) * (-4.0 * T * s.S1p * s.S1p + 2.0 * s.S1 * s.S1p);
  s.K1 = (1.0 / s.bm) * log1p(s.bm * R);
}

// REY2T (SRK.H:446-487): Newton from the supplied T on
// e(T) = e_ig(T) + (T da_m/dT - a_m) K1, |dT| < 1e-6 K, <= 2000 iterations.
// Returns 1 when the iteration cap was reached.
template <int TEAM>
__device__ int srk_t_from_energy(const Team<TEAM>& tm, const DevMech& M, double R, double E, const double* Y,
                                 double& T, SrkState& s)
{
  double Tn = T, dT = 100000.0;
  int it = 0;
  while (fabs(dT) > 1e-6 && it < 2000) {
    it++;
    srk_sums(tm, M, Tn, R, Y, s);
    double Eig, Cv;
    mix_e_c(tm, M, 0, Tn, Y, Eig, Cv);
    Cv += Tn * s.d2AmdT2 * s.K1;
    const double fzero = -E + Eig + (Tn * s.dAmdT - s.am) * s.K1;
    dT = fzero / Cv;
    Tn -= dT;
  }
  T = Tn;
  return it >= 2000;
}

} // namespace ppb
