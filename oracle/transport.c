// ORACLE / TEST INFRASTRUCTURE ONLY: CPU restatement of the reference's
// mixture-averaged transport (Source/Transport/Simple.H, ideal-gas EOS),
// the checker for the engine's transport kernel.
//
//   * SimpleTransport::transport (Simple.H:263-374): trace-amount floor on Y,
//     mole fractions, pure-species viscosities exp(fit(ln T)) mixed as
//     (sum X mu^6)^(1/6), conductivities (sum X lam^(1/4))^4, the bulk
//     viscosity of comp_pure_bulk (Simple.H:200-261) mixed as
//     (sum X xi^(3/4))^(4/3), and the light species' thermal diffusion ratios;
//   * BinaryDiff for the ideal gas (Simple.H:133-165): Ddiag_i =
//     W_i sum_{j != i} Y_j / sum_{j != i} X_j / D_ij * P_atm / (R T);
//   * the coefficients of the mechanism's generated header as
//     Source/Transport/TransportParams.H:228-258 loads them (tables from
//     pelephysics_b200/mechgen/transport_tables.py).
#include <math.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "oracle.h"
#include "../pelephysics_b200/csrc/mech/trans_LiDryer.h"
#include "../pelephysics_b200/csrc/mech/trans_drm19.h"
#include "../pelephysics_b200/csrc/mech/trans_dodecane_lu.h"
#include "../pelephysics_b200/csrc/mech/trans_heptane_lu_88sk.h"

#define TR_PATM 1.01325e+06           // Source/PhysicsConstants.H:14
#define TR_RU 8.31446261815324e7      // Source/PhysicsConstants.H:11
#define TR_PI 3.14159265358979323846

const PPBTransTables* ppo_trans(const char* name)
{
  if (!strcmp(name, "LiDryer")) return &ppbt_LiDryer;
  if (!strcmp(name, "drm19")) return &ppbt_drm19;
  if (!strcmp(name, "dodecane_lu")) return &ppbt_dodecane_lu;
  if (!strcmp(name, "heptane_lu_88sk")) return &ppbt_heptane_lu_88sk;
  return 0;
}

static double fit3(const double* c, const double* logT)
{
  return c[0] + c[1] * logT[0] + c[2] * logT[1] + c[3] * logT[2];
}

int ppo_transport(const char* mech, int flags, double T, double rho, const double* Yin, double* D, double* chi,
                  double* mu_out, double* xi_out, double* lam_out)
{
  (void)rho; // the ideal-gas path does not use the density
  const PPBTransTables* t = ppo_trans(mech);
  const PPBMechTables* M = ppo_mech(mech);
  if (!t || !M) return -100;
  const int N = t->nsp;
  const int get_xi = flags & 1, get_mu = flags & 2, get_lam = flags & 4, get_D = flags & 8, get_chi = flags & 16;
  double Y[NMAX_TR], X[NMAX_TR], muloc[NMAX_TR], chi_mix[NMAX_TR];
  double logT[3];
  logT[0] = log(T);
  logT[1] = logT[0] * logT[0];
  logT[2] = logT[0] * logT[1];
  double sum = 0.0;
  for (int i = 0; i < N; i++) sum += Yin[i];
  for (int i = 0; i < N; i++) Y[i] = Yin[i] + 1.e-15 * (sum / N - Yin[i]);
  double wbar = 0.0;
  for (int i = 0; i < N; i++) wbar += Y[i] * (1.0 / t->wt[i]);
  wbar = 1.0 / wbar;
  for (int i = 0; i < N; i++) X[i] = Y[i] * wbar * (1.0 / t->wt[i]);
  double mu = 0.0, xi = 0.0, lam = 0.0;
  if (get_mu) {
    for (int i = 0; i < N; i++) muloc[i] = exp(fit3(t->fitmu + 4 * i, logT));
    for (int i = 0; i < N; i++) {
      const double m = muloc[i];
      mu += X[i] * (m * m * m * m * m * m);
    }
    mu = cbrt(sqrt(mu));
    if (get_xi) {
      // comp_pure_bulk
      double cvk[NMAX_TR];
      ppo_cv_R(M, T, cvk);
      for (int i = 0; i < N; i++) cvk[i] *= t->cvms[i];
      const double pi3_2 = pow(TR_PI, 1.5);
      for (int i = 0; i < N; i++) {
        double xiloc = 0.0;
        if (t->nlin[i] != 0) {
          const double cvkint = cvk[i] * t->wt[i] / TR_RU - 1.50;
          const double cvkrot = t->nlin[i] == 1 ? 1.0 : 1.5;
          const double es = t->eps[i] / 298.0, et = t->eps[i] / T;
          const double Fnorm = 1.0 + 0.50 * pi3_2 * sqrt(es) + (2.0 + .50 * TR_PI * TR_PI) * es + pi3_2 * sqrt(es) * es;
          const double FofT = 1.0 + 0.50 * pi3_2 * sqrt(et) + (2.0 + .50 * TR_PI * TR_PI) * et + pi3_2 * sqrt(et) * et;
          xiloc = 0.250 * TR_PI * (cvkint / (cvkint + 1.50) * cvkint / (cvkint + 1.50)) * t->zrot[i] / cvkrot * Fnorm /
                  FofT * muloc[i];
        }
        xi += X[i] * sqrt(sqrt(xiloc * xiloc * xiloc));
      }
      xi = cbrt(xi * xi * xi * xi);
    }
  }
  if (get_lam) {
    for (int i = 0; i < N; i++) lam += X[i] * sqrt(sqrt(exp(fit3(t->fitlam + 4 * i, logT))));
    lam = lam * lam * lam * lam;
  }
  if (get_D) {
    const double scale = TR_PATM / (TR_RU * T);
    for (int i = 0; i < N; i++) {
      double term1 = 0.0, term2 = 0.0;
      for (int j = 0; j < N; j++) {
        if (i == j) continue;
        term1 += Y[j];
        term2 += X[j] * exp(-fit3(t->fitdbin + 4 * (i + N * j), logT));
      }
      D[i] = t->wt[i] * term1 / term2 * scale;
    }
  }
  if (get_chi) {
    for (int i = 0; i < N; i++) chi_mix[i] = 0.0;
    for (int n = 0; n < t->nlite; n++) {
      const int i = t->ktdif[n];
      for (int j = 0; j < N; j++) {
        if (j == i) continue;
        const double* c = t->fittdrat + 4 * (j + N * n);
        chi_mix[i] += X[j] * (c[0] + T * (c[1] + T * (c[2] + T * c[3])));
      }
      chi_mix[i] *= X[i];
    }
    if (chi) memcpy(chi, chi_mix, sizeof(double) * N);
  }
  if (mu_out) *mu_out = mu;
  if (xi_out) *xi_out = xi;
  if (lam_out) *lam_out = lam;
  return 0;
}

// The same over a batch of cells (cell-major Y, D, chi), OpenMP over cells:
// the CPU baseline of the transport benchmark.
int ppo_transport_batch(const char* mech, int flags, int ncells, const double* T, const double* rho, const double* Y,
                        double* D, double* chi, double* mu, double* xi, double* lam, int nthreads)
{
  const PPBTransTables* t = ppo_trans(mech);
  if (!t) return -100;
  const int N = t->nsp;
#ifdef _OPENMP
  if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(static) num_threads(nthreads)
#endif
  for (int c = 0; c < ncells; c++)
    ppo_transport(mech, flags, T[c], rho[c], Y + (long)c * N, D + (long)c * N, chi + (long)c * N, mu + c, xi + c,
                  lam + c);
  return 0;
}

// SRK parameters of a mechanism: [sqrt(1/Tc) | sqrt(a*) | B | F(omega)], N each.
const double* ppo_srk(const char* name)
{
  if (!strcmp(name, "LiDryer")) return ppbt_LiDryer_srk;
  if (!strcmp(name, "drm19")) return ppbt_drm19_srk;
  if (!strcmp(name, "dodecane_lu")) return ppbt_dodecane_lu_srk;
  if (!strcmp(name, "heptane_lu_88sk")) return ppbt_heptane_lu_88sk_srk;
  return 0;
}
