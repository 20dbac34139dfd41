// ORACLE / TEST INFRASTRUCTURE ONLY: CPU restatement of the reference's
// Soave-Redlich-Kwong equation of state (Source/Eos/SRK.H) for the
// e-reactor: the mixing rules and their derivatives (SRK.H:53-348), REY2T
// (:446-487), RTY2Cv (:413-427), RTY2Ei (:659-688), RTY2E (:690-714), the
// activities RTY2C (:589-621) and RTY2WDOT (:623-638), and the reactor
// right-hand side of Source/Reactions/ReactorUtils.H:358-415 over them.
// The per-species parameters are the mechanism's GET_CRITPARAMS_SRK values
// (tables from pelephysics_b200/mechgen/transport_tables.py).
#include <math.h>
#include <string.h>

#include "oracle.h"

#define SRK_RU 8.31446261815324e7 // Source/PhysicsConstants.H:11

typedef struct Srk {
  const PPBMechTables* M;
  const double *sOT, *sA, *B, *F;
  int N;
} Srk;

static int srk_get(const char* mech, Srk* s)
{
  const double* p = ppo_srk(mech);
  s->M = ppo_mech(mech);
  if (!p || !s->M) return -100;
  s->N = s->M->nsp;
  s->sOT = p;
  s->sA = p + s->N;
  s->B = p + 2 * s->N;
  s->F = p + 3 * s->N;
  return 0;
}

static double amloc(const Srk* s, int i, double sqrtT)
{
  return (1.0 + s->F[i] * (1.0 - sqrtT * s->sOT[i])) * s->sA[i];
}

static double amlocder(const Srk* s, int i, double T, double sqrtT)
{
  return -0.5 * s->F[i] * s->sA[i] * (1.0 / T) * sqrtT * s->sOT[i];
}

static void mix_am_bm(const Srk* s, double T, const double* Y, double* am, double* bm)
{
  const double sqrtT = sqrt(T);
  double a[NMAX_TR];
  *am = 0.0;
  *bm = 0.0;
  for (int i = 0; i < s->N; i++) {
    a[i] = amloc(s, i, sqrtT);
    *bm += Y[i] * s->B[i];
  }
  for (int i = 0; i < s->N; i++)
    for (int j = 0; j < s->N; j++) *am += Y[i] * Y[j] * a[i] * a[j];
}

static double mix_bm(const Srk* s, const double* Y)
{
  double bm = 0.0;
  for (int i = 0; i < s->N; i++) bm += Y[i] * s->B[i];
  return bm;
}

static double d_am_dT(const Srk* s, double T, const double* Y)
{
  const double sqrtT = sqrt(T);
  double a[NMAX_TR], ad[NMAX_TR], r = 0.0;
  for (int i = 0; i < s->N; i++) {
    a[i] = amloc(s, i, sqrtT);
    ad[i] = amlocder(s, i, T, sqrtT);
  }
  for (int i = 0; i < s->N; i++)
    for (int j = 0; j < s->N; j++) r += Y[i] * Y[j] * (a[i] * ad[j] + a[j] * ad[i]);
  return r;
}

static void d_am_dY(const Srk* s, double T, const double* Y, double* out)
{
  const double sqrtT = sqrt(T);
  double a[NMAX_TR];
  for (int i = 0; i < s->N; i++) {
    out[i] = 0.0;
    a[i] = amloc(s, i, sqrtT);
  }
  for (int i = 0; i < s->N; i++)
    for (int j = 0; j < s->N; j++) out[i] += 2.0 * Y[j] * (a[i] * a[j]);
}

static void d2_am_dTY(const Srk* s, double T, const double* Y, double* out)
{
  const double sqrtT = sqrt(T);
  double a[NMAX_TR], ad[NMAX_TR];
  for (int i = 0; i < s->N; i++) {
    out[i] = 0.0;
    a[i] = amloc(s, i, sqrtT);
    ad[i] = amlocder(s, i, T, sqrtT);
  }
  for (int i = 0; i < s->N; i++)
    for (int j = 0; j < s->N; j++) out[i] += 2.0 * Y[j] * (a[i] * ad[j] + a[j] * ad[i]);
}

static double d2_am_dT2(const Srk* s, double T, const double* Y)
{
  const double sqrtT = sqrt(T), tmp1 = -0.5 * (1.0 / T);
  double a[NMAX_TR], ad[NMAX_TR], r = 0.0;
  for (int i = 0; i < s->N; i++) {
    a[i] = amloc(s, i, sqrtT);
    ad[i] = amlocder(s, i, T, sqrtT);
  }
  for (int i = 0; i < s->N; i++)
    for (int j = 0; j < s->N; j++) r += tmp1 * Y[i] * Y[j] * (-4.0 * T * ad[i] * ad[j] + a[i] * ad[j] + a[j] * ad[i]);
  return r;
}

// Calc_Am_and_derivs (SRK.H:292-348)
static void am_and_derivs(const Srk* s, double T, const double* Y, double* am, double* dAmdT, double* d2AmdT2)
{
  const double oneOverT = 1.0 / T, tmp1 = -0.5 * oneOverT, sqrtT = sqrt(T);
  double a[NMAX_TR], ad[NMAX_TR];
  for (int i = 0; i < s->N; i++) {
    a[i] = amloc(s, i, sqrtT);
    ad[i] = s->F[i] * s->sA[i] * s->sOT[i];
  }
  *am = *dAmdT = *d2AmdT2 = 0.0;
  if (s->N > 1) {
    for (int i = 0; i < s->N; i++)
      for (int j = i + 1; j < s->N; j++) {
        *am += Y[i] * Y[j] * a[i] * a[j];
        *dAmdT += Y[i] * Y[j] * (a[i] * ad[j] + a[j] * ad[i]);
        *d2AmdT2 += Y[i] * Y[j] * ad[i] * ad[j];
      }
    *am *= 2.0;
    *dAmdT *= 2.0;
    *d2AmdT2 *= 2.0;
  }
  for (int i = 0; i < s->N; i++) {
    *am += Y[i] * Y[i] * a[i] * a[i];
    *dAmdT += 2.0 * Y[i] * Y[i] * (a[i] * ad[i]);
    *d2AmdT2 += Y[i] * Y[i] * ad[i] * ad[i];
  }
  *dAmdT *= tmp1 * sqrtT;
  *d2AmdT2 = -*d2AmdT2;
  *d2AmdT2 += *dAmdT;
  *d2AmdT2 *= tmp1;
}

int ppo_srk_rey2t(const char* mech, double R, double E, const double* Y, double* T)
{
  Srk s;
  if (srk_get(mech, &s)) return -100;
  const double bm = mix_bm(&s, Y);
  const double K1 = (1.0 / bm) * log1p(bm * R);
  double Tn = *T, dT = 100000.0;
  int it = 0;
  while (fabs(dT) > 1e-6 && it < 2000) {
    it++;
    double am, dAmdT, d2AmdT2;
    am_and_derivs(&s, Tn, Y, &am, &dAmdT, &d2AmdT2);
    const double Eig = ppo_ckubms(s.M, Tn, Y);
    double Cv = ppo_ckcvbs(s.M, Tn, Y);
    Cv += Tn * d2AmdT2 * K1;
    const double fzero = -E + Eig + (Tn * dAmdT - am) * K1;
    dT = fzero / Cv;
    Tn -= dT;
  }
  *T = Tn;
  return it < 2000 ? 0 : -1;
}

double ppo_srk_rty2cv(const char* mech, double R, double T, const double* Y)
{
  Srk s;
  if (srk_get(mech, &s)) return NAN;
  double am, bm;
  mix_am_bm(&s, T, Y, &am, &bm);
  const double d2 = d2_am_dT2(&s, T, Y);
  double cv = ppo_ckcvbs(s.M, T, Y);
  return cv + T * d2 * (1.0 / bm) * log1p(bm * R);
}

void ppo_srk_rty2ei(const char* mech, double R, double T, const double* Y, double* Ei)
{
  Srk s;
  if (srk_get(mech, &s)) return;
  double am, bm, dY[NMAX_TR], dTY[NMAX_TR];
  ppo_ckums(s.M, T, Ei);
  mix_am_bm(&s, T, Y, &am, &bm);
  const double dAmdT = d_am_dT(&s, T, Y);
  d_am_dY(&s, T, Y, dY);
  d2_am_dTY(&s, T, Y, dTY);
  const double inv_bm = 1.0 / bm;
  const double K1 = inv_bm * log1p(bm * R);
  const double d3 = 1.0 / (1.0 / R + bm);
  for (int i = 0; i < s.N; i++) {
    Ei[i] += (T * dTY[i] - dY[i]) * K1;
    Ei[i] += (T * dAmdT - am) * s.B[i] * (d3 - K1) * inv_bm;
  }
}

double ppo_srk_rty2e(const char* mech, double R, double T, const double* Y)
{
  Srk s;
  if (srk_get(mech, &s)) return NAN;
  double Ei[NMAX_TR], E = 0.0, am, bm;
  ppo_ckums(s.M, T, Ei);
  for (int i = 0; i < s.N; i++) E += Ei[i] * Y[i];
  mix_am_bm(&s, T, Y, &am, &bm);
  const double dAmdT = d_am_dT(&s, T, Y);
  const double K1 = (1.0 / bm) * log1p(bm * R);
  return E + (T * dAmdT - am) * K1;
}

void ppo_srk_rty2c(const char* mech, double R, double T, const double* Y, double* C)
{
  Srk s;
  if (srk_get(mech, &s)) return;
  double am, bm, dY[NMAX_TR];
  mix_am_bm(&s, T, Y, &am, &bm);
  d_am_dY(&s, T, Y, dY);
  double sy = 0.0;
  for (int i = 0; i < s.N; i++) sy += Y[i] * s.M->imw[i];
  const double wbar = 1.0 / sy;
  const double InvBm = 1.0 / bm, tau = 1.0 / R;
  const double K1 = InvBm * log1p(bm * R);
  const double RmT = SRK_RU / wbar * T, InvRuT = 1.0 / (SRK_RU * T);
  const double d1 = 1.0 / (tau - bm), d3 = 1.0 / (tau + bm);
  for (int i = 0; i < s.N; i++)
    C[i] = exp((s.M->mw[i] * InvRuT) *
               (RmT * d1 * s.B[i] - K1 * dY[i] + am * InvBm * K1 * s.B[i] - am * d3 * s.B[i] * InvBm)) *
           Y[i] * s.M->imw[i] * d1;
}

void ppo_srk_rty2wdot(const char* mech, double R, double T, const double* Y, double* wdot)
{
  Srk s;
  if (srk_get(mech, &s)) return;
  double C[NMAX_TR];
  ppo_srk_rty2c(mech, R, T, Y, C);
  ppo_ckwc(s.M, T, C, wdot);
  for (int n = 0; n < s.N; n++) wdot[n] *= s.M->mw[n];
}

double ppo_reactor_rhs_srk(const char* mech, double t_rel, const double* y, double* ydot, double rhoe_init,
                           double rhoesrc, const double* rYsrc)
{
  const PPBMechTables* M = ppo_mech(mech);
  if (!M) return NAN;
  const int N = M->nsp;
  double rho = 0.0, Y[NMAX_TR], ei[NMAX_TR], cd[NMAX_TR];
  for (int n = 0; n < N; n++) rho += y[n];
  const double rinv = 1.0 / rho;
  for (int n = 0; n < N; n++) Y[n] = y[n] * rinv;
  const double nrg = (rhoe_init + rhoesrc * t_rel) * rinv;
  double T = y[N];
  ppo_srk_rey2t(mech, rho, nrg, Y, &T);
  ppo_srk_rty2ei(mech, rho, T, Y, ei);
  const double cv = ppo_srk_rty2cv(mech, rho, T, Y);
  ppo_srk_rty2wdot(mech, rho, T, Y, cd);
  double es = rhoesrc;
  for (int n = 0; n < N; n++) {
    const double c = cd[n] + rYsrc[n];
    ydot[n] = c;
    es -= c * ei[n];
  }
  ydot[N] = es * (rinv / cv);
  return T;
}
