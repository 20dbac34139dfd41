// ORACLE / TEST INFRASTRUCTURE ONLY: table-driven restatement of the
// reference's generated mechanism arithmetic (Mechanisms/<mech>/mechanism.H,
// produced by Support/ceptr/ceptr/{thermo,production,jacobian}.py).  The
// tables come from pelephysics_b200/mechgen/ceptr_tables.py, which rounds
// every constant exactly as the generated source prints it.
#include <math.h>
#include <string.h>

#include "oracle.h"
#include "../pelephysics_b200/csrc/mech/mech_LiDryer.h"
#include "../pelephysics_b200/csrc/mech/mech_drm19.h"
#include "../pelephysics_b200/csrc/mech/mech_dodecane_lu.h"
#include "../pelephysics_b200/csrc/mech/mech_heptane_lu_88sk.h"
#include "../pelephysics_b200/csrc/mech/mech_CH4_lean_qss.h"
#include "../pelephysics_b200/csrc/mech/mech_C1-C2-NO_qss.h"
#include "../pelephysics_b200/csrc/mech/mech_LuEthylene_qss.h"
#include "../pelephysics_b200/csrc/mech/mech_grimech30.h"
#include "../pelephysics_b200/csrc/mech/mech_FFCM1_Red.h"
#include "../pelephysics_b200/csrc/mech/mech_chem-H.h"

const PPBMechTables* ppo_mech(const char* name)
{
  if (!strcmp(name, "LiDryer")) return &ppbm_LiDryer;
  if (!strcmp(name, "drm19")) return &ppbm_drm19;
  if (!strcmp(name, "dodecane_lu")) return &ppbm_dodecane_lu;
  if (!strcmp(name, "heptane_lu_88sk")) return &ppbm_heptane_lu_88sk;
  if (!strcmp(name, "CH4_lean_qss")) return &ppbm_CH4_lean_qss;
  if (!strcmp(name, "C1-C2-NO_qss")) return &ppbm_C1_C2_NO_qss;
  if (!strcmp(name, "LuEthylene_qss")) return &ppbm_LuEthylene_qss;
  if (!strcmp(name, "grimech30")) return &ppbm_grimech30;
  if (!strcmp(name, "FFCM1_Red")) return &ppbm_FFCM1_Red;
  if (!strcmp(name, "chem-H")) return &ppbm_chem_H;
  return 0;
}

int ppo_nqss(const char* name)
{
  const PPBMechTables* M = ppo_mech(name);
  return M ? M->nqss : -1;
}

const char* ppo_species_name(const char* name, int k)
{
  const PPBMechTables* M = ppo_mech(name);
  return (M && k >= 0 && k < M->nsp) ? M->species[k] : 0;
}

void ppo_mw(const char* name, double* mw)
{
  const PPBMechTables* M = ppo_mech(name);
  for (int k = 0; M && k < M->nsp; k++) mw[k] = M->mw[k];
}

int ppo_nsp(const char* name)
{
  const PPBMechTables* M = ppo_mech(name);
  return M ? M->nsp : -1;
}

// NASA-7 range: low below the species mid-point (thermo.py:317-345,
// "if (T < Tmid)"), high otherwise; a single-range species stores the same
// set twice.
static inline int rng(const PPBMechTables* M, int s, double T)
{
  return (M->tmid[s] >= 0.0 && T < M->tmid[s]) ? 0 : 1;
}

// thermo.py:516-526 cv_nasa7
void ppo_cv_R(const PPBMechTables* M, double T, double* out)
{
  const double T2 = T * T, T3 = T * T * T, T4 = T * T * T * T;
  for (int s = 0; s < M->nsp; s++) {
    const double* c = M->th_cv + (2 * s + rng(M, s, T)) * 5;
    out[s] = c[0] + c[1] * T + c[2] * T2 + c[3] * T3 + c[4] * T4;
  }
}

// thermo.py:549-559 cp_nasa7
void ppo_cp_R(const PPBMechTables* M, double T, double* out)
{
  const double T2 = T * T, T3 = T * T * T, T4 = T * T * T * T;
  for (int s = 0; s < M->nsp; s++) {
    const double* c = M->th_cp + (2 * s + rng(M, s, T)) * 5;
    out[s] = c[0] + c[1] * T + c[2] * T2 + c[3] * T3 + c[4] * T4;
  }
}

// thermo.py:561-570 dcpdtemp_nasa7
void ppo_dcvpRdT(const PPBMechTables* M, double T, double* out)
{
  const double T2 = T * T, T3 = T * T * T;
  for (int s = 0; s < M->nsp; s++) {
    const double* c = M->th_dcp + (2 * s + rng(M, s, T)) * 4;
    out[s] = c[0] + c[1] * T + c[2] * T2 + c[3] * T3;
  }
}

// thermo.py:625-646 internal_energy_nasa7
void ppo_species_internal_energy(const PPBMechTables* M, double T, double* out)
{
  const double T2 = T * T, T3 = T * T * T, T4 = T * T * T * T, invT = 1.0 / T;
  for (int s = 0; s < M->nsp; s++) {
    const double* c = M->th_u + (2 * s + rng(M, s, T)) * 6;
    out[s] = c[0] + c[1] * T + c[2] * T2 + c[3] * T3 + c[4] * T4 + c[5] * invT;
  }
}

// thermo.py:649-669 enthalpy_nasa7
void ppo_species_enthalpy(const PPBMechTables* M, double T, double* out)
{
  const double T2 = T * T, T3 = T * T * T, T4 = T * T * T * T, invT = 1.0 / T;
  for (int s = 0; s < M->nsp; s++) {
    const double* c = M->th_h + (2 * s + rng(M, s, T)) * 6;
    out[s] = c[0] + c[1] * T + c[2] * T2 + c[3] * T3 + c[4] * T4 + c[5] * invT;
  }
}

// thermo.py:572-595 gibbs_nasa7
void ppo_gibbs(const PPBMechTables* M, double T, double* out)
{
  const double T2 = T * T, T3 = T * T * T, T4 = T * T * T * T;
  const double invT = 1.0 / T, logT = log(T);
  for (int s = 0; s < M->nsp; s++) {
    const double* c = M->th_g + (2 * s + rng(M, s, T)) * 7;
    out[s] = c[0] * invT + c[1] + c[2] * logT + c[3] * T + c[4] * T2 + c[5] * T3 +
             c[6] * T4;
  }
}

// mechanism.H CKUBMS (LiDryer :1238-1356): sum y_k e_k/RT / W_k, times R T
double ppo_ckubms(const PPBMechTables* M, double T, const double* y)
{
  const double T2 = T * T, T3 = T * T * T, T4 = T * T * T * T, invT = 1.0 / T;
  double r = 0.0;
  for (int s = 0; s < M->nsp; s++) {
    const double* c = M->th_u + (2 * s + rng(M, s, T)) * 6;
    r += y[s] * (c[0] + c[1] * T + c[2] * T2 + c[3] * T3 + c[4] * T4 + c[5] * invT) *
         M->imw[s];
  }
  const double RT = PPO_RU * T;
  return r * RT;
}

double ppo_ckhbms(const PPBMechTables* M, double T, const double* y)
{
  const double T2 = T * T, T3 = T * T * T, T4 = T * T * T * T, invT = 1.0 / T;
  double r = 0.0;
  for (int s = 0; s < M->nsp; s++) {
    const double* c = M->th_h + (2 * s + rng(M, s, T)) * 6;
    r += y[s] * (c[0] + c[1] * T + c[2] * T2 + c[3] * T3 + c[4] * T4 + c[5] * invT) *
         M->imw[s];
  }
  const double RT = PPO_RU * T;
  return r * RT;
}

// mechanism.H CKCVBS (LiDryer :981-1080)
double ppo_ckcvbs(const PPBMechTables* M, double T, const double* y)
{
  const double T2 = T * T, T3 = T * T * T, T4 = T * T * T * T;
  double r = 0.0;
  for (int s = 0; s < M->nsp; s++) {
    const double* c = M->th_cv + (2 * s + rng(M, s, T)) * 5;
    r += y[s] * (c[0] + c[1] * T + c[2] * T2 + c[3] * T3 + c[4] * T4) * M->imw[s];
  }
  return r * PPO_RU;
}

double ppo_ckcpbs(const PPBMechTables* M, double T, const double* y)
{
  const double T2 = T * T, T3 = T * T * T, T4 = T * T * T * T;
  double r = 0.0;
  for (int s = 0; s < M->nsp; s++) {
    const double* c = M->th_cp + (2 * s + rng(M, s, T)) * 5;
    r += y[s] * (c[0] + c[1] * T + c[2] * T2 + c[3] * T3 + c[4] * T4) * M->imw[s];
  }
  return r * PPO_RU;
}

// mechanism.H CKUMS (LiDryer :2019-2029)
void ppo_ckums(const PPBMechTables* M, double T, double* u)
{
  const double RT = PPO_RU * T;
  ppo_species_internal_energy(M, T, u);
  for (int s = 0; s < M->nsp; s++) u[s] *= RT * M->imw[s];
}

void ppo_ckhms(const PPBMechTables* M, double T, double* h)
{
  const double RT = PPO_RU * T;
  ppo_species_enthalpy(M, T, h);
  for (int s = 0; s < M->nsp; s++) h[s] *= RT * M->imw[s];
}

// mechanism.H CKRHOY (LiDryer :1608-1622)
double ppo_ckrhoy(const PPBMechTables* M, double P, double T, const double* y)
{
  double YOW = 0.0;
  for (int s = 0; s < M->nsp; s++) YOW += y[s] * M->imw[s];
  return P / (PPO_RU * T * YOW);
}

// mechanism.H GET_T_GIVEN_EY (LiDryer :1419-1468): Newton on e(T) from the
// supplied T, steps clipped to +-100 K, stop when |dT| < 1e-6 K, at most 200
// iterations; linear extrapolation outside [90, 4000] K with ierr = 1.
static int t_from(const PPBMechTables* M, double e, const double* y, double* t,
                  double (*E)(const PPBMechTables*, double, const double*),
                  double (*C)(const PPBMechTables*, double, const double*))
{
  const int maxiter = 200;
  const double tol = 1.e-6;
  const double tmin = 90, tmax = 4000;
  const double emin = E(M, tmin, y), emax = E(M, tmax, y);
  if (e < emin) {
    const double cv = C(M, tmin, y);
    *t = tmin - (emin - e) / cv;
    return 1;
  }
  if (e > emax) {
    const double cv = C(M, tmax, y);
    *t = tmax - (emax - e) / cv;
    return 1;
  }
  double t1 = *t;
  if (t1 < tmin || t1 > tmax) t1 = tmin + (tmax - tmin) / (emax - emin) * (e - emin);
  for (int i = 0; i < maxiter; ++i) {
    const double e1 = E(M, t1, y);
    const double cv = C(M, t1, y);
    double dt = (e - e1) / cv;
    if (dt > 100.) {
      dt = 100.;
    } else if (dt < -100.) {
      dt = -100.;
    } else if (fabs(dt) < tol) {
      break;
    }
    t1 += dt;
  }
  *t = t1;
  return 0;
}

int ppo_get_t_given_ey(const PPBMechTables* M, double e, const double* y, double* T)
{
  return t_from(M, e, y, T, ppo_ckubms, ppo_ckcvbs);
}

int ppo_get_t_given_hy(const PPBMechTables* M, double h, const double* y, double* T)
{
  return t_from(M, h, y, T, ppo_ckhbms, ppo_ckcpbs);
}

static inline double phase_space(const int* sp, const double* c, int n, const double* sc)
{
  double p = 1.0;
  for (int j = 0; j < n; j++) {
    const double x = sc[sp[j]];
    const int o = (int)c[j];
    double t = x;
    for (int q = 1; q < o; q++) t *= x;
    p *= t;
  }
  return p;
}

static inline double refc_pow(int p, double refC, double refCinv)
{
  double r = 1.0;
  for (int q = 0; q < p; q++) r *= refCinv;
  for (int q = 0; q < -p; q++) r *= refC;
  return r;
}

// g/RT of thermo entry s (gibbs_nasa7 of thermo.py:572-595; for a QSS
// mechanism the QSS species' entries are those of gibbs_qss)
static double gibbs_one(const PPBMechTables* M, int s, double T, double invT, double logT)
{
  const double* c = M->th_g + (2 * s + rng(M, s, T)) * 7;
  return c[0] * invT + c[1] + c[2] * logT + c[3] * T + c[4] * (T * T) + c[5] * (T * T * T) +
         c[6] * (T * T * T * T);
}

// Rates of progress q_f, q_r of reaction r (production.py:991-1435) over
// the concentration slots sc and g/RT slots g.
static void rxn_rates(const PPBMechTables* M, int r, double T, double invT, double logT, double refC,
                      double refCinv, double mixture, const double* sc, const double* g_RT, double* qf_out,
                      double* qr_out)
{
  {
    const int kind = M->rx_kind[r];
    const double k_f =
      M->rx_A[r] * exp(M->rx_beta[r] * logT - M->rx_EaR[r] * invT);
    double Corr = 1.0;
    int corr = 0;
    if (kind == PPB_RX_THIRD || kind == PPB_RX_TROE || kind == PPB_RX_LINDEMANN) {
      Corr = mixture;
      for (int e = M->eff_off[r]; e < M->eff_off[r + 1]; e++) {
        if (M->eff_m1[e] != 0.0) Corr += M->eff_m1[e] * sc[M->eff_sp[e]];
      }
      corr = 1;
    }
    if (kind == PPB_RX_TROE || kind == PPB_RX_LINDEMANN) {
      const double* fd = M->fo_d + r * PPB_NFOD;
      const int* fi = M->fo_i + r * PPB_NFOI;
      const double redP = Corr / k_f * fd[PPB_FO_P0] *
                          exp(fd[PPB_FO_BETA0] * logT - fd[PPB_FO_EAR0] * invT);
      const double F = redP / (1.0 + redP);
      if (kind == PPB_RX_TROE) {
        const double logPred = log10(redP);
        double fc = 0.0;
        if (fi[PPB_FOI_P1]) fc = fd[PPB_FO_OMA] * exp(-T * fd[PPB_FO_IT3]);
        if (fi[PPB_FOI_P2]) fc += fd[PPB_FO_A] * exp(-T * fd[PPB_FO_IT1]);
        if (fi[PPB_FOI_NTROE] == 4) {
          fc += exp(-fd[PPB_FO_T2] * invT);
        } else {
          fc += 0.0;
        }
        const double logFcent = log10(fc);
        const double troe_c = -0.4 - 0.67 * logFcent;
        const double troe_n = 0.75 - 1.27 * logFcent;
        const double troe = (troe_c + logPred) / (troe_n - 0.14 * (troe_c + logPred));
        const double F_troe = exp(M_LN10 * logFcent / (1.0 + troe * troe));
        Corr = F * F_troe;
      } else {
        Corr = F;
      }
    }
    const int W = PPB_MAXPS;
    const double phf = phase_space(M->rx_fps_sp + r * W, M->rx_fps_c + r * W, M->rx_fps_n[r], sc);
    const double qf = corr ? Corr * k_f * phf : k_f * phf;
    double qr = 0.0;
    if (M->rx_rev[r]) {
      double arg = 0.0;
      for (int j = 0; j < M->rx_kc_n[r]; j++) {
        arg += M->rx_kc_c[r * PPB_MAXKC + j] * g_RT[M->rx_kc_sp[r * PPB_MAXKC + j]];
      }
      const double phr = phase_space(M->rx_rps_sp + r * W, M->rx_rps_c + r * W, M->rx_rps_n[r], sc);
      const double conv = refc_pow(M->rx_kcpow[r], refC, refCinv);
      qr = (corr ? Corr * k_f : k_f) * exp(-arg) * conv * phr;
    }
    // a forward rate the QSS reduction removed counts 0 (qdot = -q_r)
    *qf_out = (M->nqss > 0 && M->rx_rmfwd[r]) ? 0.0 : qf;
    *qr_out = qr;
  }
}

// The QSS concentrations (comp_qss_coeff, comp_sc_qss of the reference's
// generated QSS mechanism.H): with the QSS slots of sc at 1, the
// coefficients q_f,k and q_r,k of the QSS reactions; per QSS species i the
// production P_i = eps + sum, the loss D_i = eps - sum (of the loss
// coefficients, so negative) and the couplings C_ij = (eps + sum) / D_i, all
// summed in k order, eps = 1e-12 as the generated code adds it; then the
// linear balance x_i + sum_j C_ij x_j = -P_i / D_i, solved by Gaussian
// elimination in species order without pivoting (the generated code
// eliminates symbolically in an order of its own: the same system, solved to
// rounding).  No pivoting: the loss of species i includes every reaction
// that turns it into another QSS species, so the balance matrix is
// column-diagonally dominant and elimination on its unit diagonal is
// stable, while a row swap can mix a species of concentration 1e-17 with one
// of 1e-2 and lose the small one to cancellation.
static void qss_concentrations(const PPBMechTables* M, double T, double invT, double logT, double refC,
                               double refCinv, double mixture, double* sc, const double* g_RT, double* sys_out)
{
  const int N = M->nsp, Q = M->nqss, K = M->nrq;
  const double eps = 1e-12;
  double co[2 * 512];
  double A[32 * 33];
  for (int q = 0; q < Q; q++) sc[N + 1 + q] = 1.0;
  for (int k = 0; k < K; k++) rxn_rates(M, M->q_rx[k], T, invT, logT, refC, refCinv, mixture, sc, g_RT, &co[2 * k], &co[2 * k + 1]);
  for (int i = 0; i < Q; i++) {
    double* row = A + i * (Q + 1);
    unsigned char has[32];
    for (int j = 0; j < Q; j++) {
      row[j] = 0.0;
      has[j] = 0;
    }
    double P = eps, D = eps;
    for (int t = M->q_off[i]; t < M->q_off[i + 1]; t++) {
      const double c = M->q_coef[t];
      const double v = c == 1.0 ? co[M->q_term[t]] : c * co[M->q_term[t]];
      const int role = M->q_role[t];
      if (role == -1) {
        P += v;
      } else if (role == -2) {
        D -= v;
      } else {
        if (!has[role]) {
          row[role] = eps;
          has[role] = 1;
        }
        row[role] += v;
      }
    }
    for (int j = 0; j < Q; j++)
      if (has[j]) row[j] = row[j] / D;
    row[i] = 1.0;
    row[Q] = -P / D;
  }
  if (sys_out) {
    for (int i = 0; i < Q * (Q + 1); i++) sys_out[i] = A[i];
    return;
  }
  // forward elimination, then back substitution
  for (int c = 0; c < Q; c++) {
    for (int i = c + 1; i < Q; i++) {
      const double f = A[i * (Q + 1) + c] / A[c * (Q + 1) + c];
      if (f == 0.0) continue;
      for (int j = c; j <= Q; j++) A[i * (Q + 1) + j] -= f * A[c * (Q + 1) + j];
    }
  }
  for (int i = Q - 1; i >= 0; i--) {
    double x = A[i * (Q + 1) + Q];
    for (int j = i + 1; j < Q; j++) x -= A[i * (Q + 1) + j] * sc[N + 1 + j];
    sc[N + 1 + i] = x / A[i * (Q + 1) + i];
  }
}

// The QSS concentrations (SI) productionRate uses at (sc, T): out[nqss].
static void qss_eval(const PPBMechTables* M, const double* sc_in, double T, double* out, double* sys_out);

void ppo_qss_concentrations(const PPBMechTables* M, const double* sc_in, double T, double* out)
{
  qss_eval(M, sc_in, T, out, 0);
}

// The QSS balance system [C + I | -P/D] (nqss rows of nqss + 1) at (sc, T),
// for checks of the solve against exact arithmetic.
void ppo_qss_system(const PPBMechTables* M, const double* sc_in, double T, double* sys_out)
{
  qss_eval(M, sc_in, T, 0, sys_out);
}

static void qss_eval(const PPBMechTables* M, const double* sc_in, double T, double* out, double* sys_out)
{
  const int N = M->nsp, Q = M->nqss;
  const double invT = 1.0 / T, logT = log(T);
  const double refC = 101325 / 8.31446 * invT, refCinv = 1 / refC;
  double g_RT[160], sc[160];
  double mixture = 0.0;
  for (int i = 0; i < N; i++) mixture += sc_in[i];
  ppo_gibbs(M, T, g_RT);
  for (int i = 0; i < N; i++) sc[i] = sc_in[i];
  sc[N] = 1.0;
  g_RT[N] = 0.0;
  for (int q = 0; q < Q; q++) g_RT[N + 1 + q] = gibbs_one(M, N + 1 + q, T, invT, logT);
  qss_concentrations(M, T, invT, logT, refC, refCinv, mixture, sc, g_RT, sys_out);
  if (out)
    for (int q = 0; q < Q; q++) out[q] = sc[N + 1 + q];
}

// production.py:991-1435 (productionRate, SI units).  When absterm is not
// NULL it also receives, per species, sum over reactions of
// |nu| (|q_f| + |q_r|): the magnitude against which the rounding error of
// the (cancelling) sum wdot is measured.  For a QSS mechanism the QSS
// concentrations are solved first (qss_concentrations).
static void production_rate_impl(const PPBMechTables* M, double* wdot, const double* sc_in,
                                 double T, double* absterm)
{
  const int N = M->nsp, Q = M->nqss;
  const double invT = 1.0 / T;
  const double logT = log(T);
  const double refC = 101325 / 8.31446 * invT;
  const double refCinv = 1 / refC;
  double g_RT[160], sc[160];
  for (int i = 0; i < N; i++) wdot[i] = 0.0;
  double mixture = 0.0;
  for (int i = 0; i < N; i++) mixture += sc_in[i];
  ppo_gibbs(M, T, g_RT);
  for (int i = 0; i < N; i++) sc[i] = sc_in[i];
  sc[N] = 1.0;
  g_RT[N] = 0.0;
  if (Q > 0) {
    for (int q = 0; q < Q; q++) g_RT[N + 1 + q] = gibbs_one(M, N + 1 + q, T, invT, logT);
    qss_concentrations(M, T, invT, logT, refC, refCinv, mixture, sc, g_RT, 0);
  }
  for (int r = 0; r < M->nrxn; r++) {
    double qf, qr;
    rxn_rates(M, r, T, invT, logT, refC, refCinv, mixture, sc, g_RT, &qf, &qr);
    const double qdot = qf - qr;
    for (int j = 0; j < M->rx_wup_n[r]; j++) {
      const int s = M->rx_wup_sp[r * PPB_MAXW + j];
      const double c = M->rx_wup_c[r * PPB_MAXW + j];
      if (absterm) absterm[s] += fabs(c) * (fabs(qf) + fabs(qr));
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
}

void ppo_production_rate(const PPBMechTables* M, double* wdot, const double* sc, double T)
{
  production_rate_impl(M, wdot, sc, T, 0);
}

void ppo_production_rate_abs(const PPBMechTables* M, double* absterm, const double* sc, double T)
{
  double w[128];
  for (int i = 0; i < M->nsp; i++) absterm[i] = 0.0;
  production_rate_impl(M, w, sc, T, absterm);
}

// mechanism.H CKWC (LiDryer :2606-2622)
void ppo_ckwc(const PPBMechTables* M, double T, const double* C, double* wdot)
{
  double c[128];
  for (int i = 0; i < M->nsp; i++) c[i] = C[i] * 1.0e6;
  ppo_production_rate(M, wdot, c, T);
  for (int i = 0; i < M->nsp; i++) wdot[i] *= 1.0e-6;
}

// jacobian.py:1398-1515 dphase_space: d(phi)/d(sc[k]) for a species present
static inline double dphase(const int* sp, const double* c, int n, const double* sc, int k)
{
  double p = 1.0;
  for (int j = 0; j < n; j++) {
    const double x = sc[sp[j]];
    const int o = (int)c[j];
    if (sp[j] == k) {
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

static inline int has_sp(const int* sp, int n, int k)
{
  for (int j = 0; j < n; j++)
    if (sp[j] == k) return 1;
  return 0;
}

// jacobian.py:12-283 (ajac) and :546-1305 (ajac_reaction_d): the reference's
// analytical Jacobian, J[k*(N+1)+m] = d wdot_m / d sc_k, last row d/dT,
// last column dTdot/d sc_k, corner dTdot/dT; consP selects h/cp vs e/cv.
void ppo_ajacobian(const PPBMechTables* M, double* J, const double* sc, double T, int consP)
{
  const int N = M->nsp;
  const int n = N + 1;
  for (int i = 0; i < n * n; i++) J[i] = 0.0;
  double wdot[128];
  for (int i = 0; i < N; i++) wdot[i] = 0.0;
  const double invT = 1.0 / T;
  const double invT2 = invT * invT;
  const double logT = log(T);
  const double refC = 101325 / 8.31446 / T;
  const double refCinv = 1.0 / refC;
  double mixture = 0.0;
  for (int k = 0; k < N; k++) mixture += sc[k];
  double g_RT[128], h_RT[128];
  // carried across reactions on purpose: see the consP == 0 branch below
  double dqdc[128];
  for (int k = 0; k < N; k++) dqdc[k] = 0.0;
  ppo_gibbs(M, T, g_RT);
  ppo_species_enthalpy(M, T, h_RT);
  const double ln10 = log(10.0);
  const double log10e = 1.0 / log(10.0);
  const int W = PPB_MAXPS;
  for (int r = 0; r < M->nrxn; r++) {
    const int kind = M->rx_kind[r];
    const int falloff = (kind == PPB_RX_TROE || kind == PPB_RX_LINDEMANN);
    const int has_alpha = (kind == PPB_RX_THIRD) || falloff;
    const int rev = M->rx_rev[r];
    const int* fsp = M->rx_fps_sp + r * W;
    const double* fc = M->rx_fps_c + r * W;
    const int fn = M->rx_fps_n[r];
    const int* rsp = M->rx_rps_sp + r * W;
    const double* rc = M->rx_rps_c + r * W;
    const int rn = M->rx_rps_n[r];
    double alpha = 0.0;
    if (has_alpha) {
      alpha = mixture;
      for (int e = M->eff_off[r]; e < M->eff_off[r + 1]; e++) {
        const double em1 = M->eff_e[e] - 1.0;
        if (M->eff_e[e] - 1.0 != 0.0) alpha += em1 * sc[M->eff_sp[e]];
      }
    }
    const double phi_f = phase_space(fsp, fc, fn, sc);
    double k_f = M->rx_A[r] * exp(M->rx_beta[r] * logT - M->rx_EaR[r] * invT);
    const double dlnkfdT = M->rx_beta[r] * invT + M->rx_EaR[r] * invT2;
    double Pr = 0.0, fPr = 0.0, F = 1.0, dlogFdlogPr = 0.0, dlogFdT = 0.0, dlogfPrdT = 0.0;
    if (falloff) {
      const double* fd = M->fo_d + r * PPB_NFOD;
      const int* fi = M->fo_i + r * PPB_NFOI;
      const double k_0 = fd[PPB_FO_K0] * exp(fd[PPB_FO_BETA0] * logT - fd[PPB_FO_EAR0] * invT);
      Pr = fd[PPB_FO_PRDIM] * alpha / k_f * k_0;
      fPr = Pr / (1.0 + Pr);
      const double dlnk0dT = fd[PPB_FO_BETA0] * invT + fd[PPB_FO_EAR0] * invT2;
      const double dlogPrdT = log10e * (dlnk0dT - dlnkfdT);
      dlogfPrdT = dlogPrdT / (1.0 + Pr);
      if (kind == PPB_RX_TROE) {
        const double a = fd[PPB_FO_A], T3 = fd[PPB_FO_T3], T1 = fd[PPB_FO_T1], T2 = fd[PPB_FO_T2];
        const double logPr = log10(Pr);
        const double Fcent1 = fi[PPB_FOI_J1] ? (1. - a) * exp(-T / T3) : 0.;
        const double Fcent2 = fi[PPB_FOI_J2] ? a * exp(-T / T1) : 0.;
        const double Fcent3 = (fi[PPB_FOI_NTROE] == 4) ? exp(-T2 * invT) : 0.;
        const double Fcent = Fcent1 + Fcent2 + Fcent3;
        const double logFcent = log10(Fcent);
        const double troe_c = -.4 - .67 * logFcent;
        const double troe_n = .75 - 1.27 * logFcent;
        const double troePr_den = 1.0 / (troe_n - .14 * (troe_c + logPr));
        const double troePr = (troe_c + logPr) * troePr_den;
        const double troe = 1.0 / (1.0 + troePr * troePr);
        F = exp(M_LN10 * logFcent * troe);
        double s = 0.0;
        if (fi[PPB_FOI_J1]) s += -Fcent1 / T3;
        if (fi[PPB_FOI_J2]) s += -Fcent2 / T1;
        if (fi[PPB_FOI_J3]) s += Fcent3 * T2 * invT2;
        const double dlogFcentdT = log10e / Fcent * (s);
        const double dlogFdcn_fac = 2.0 * logFcent * troe * troe * troePr * troePr_den;
        const double dlogFdc = -troe_n * dlogFdcn_fac * troePr_den;
        const double dlogFdn = dlogFdcn_fac * troePr;
        dlogFdlogPr = dlogFdc;
        dlogFdT = dlogFcentdT * (troe - 0.67 * dlogFdc - 1.27 * dlogFdn) + dlogFdlogPr * dlogPrdT;
      } else {
        F = 1.0;
        dlogFdlogPr = 0.0;
        dlogFdT = 0.0;
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
        const double dlnCorrdT = ln10 * (dlogfPrdT + dlogFdT);
        dqdT = Corr * dlnkfdT * k_f * phi_f + dlnCorrdT * q;
      } else if (has_alpha) {
        dqdT = alpha * dlnkfdT * k_f * phi_f;
      } else {
        dqdT = dlnkfdT * k_f * phi_f;
      }
    } else {
      const double phi_r = phase_space(rsp, rc, rn, sc);
      double arg = 0.0;
      for (int j = 0; j < M->rx_kc_n[r]; j++) {
        arg += M->rx_kc_c[r * PPB_MAXKC + j] * g_RT[M->rx_kc_sp[r * PPB_MAXKC + j]];
      }
      // Kc = refC^(-kcpow) exp(arg); k_r = k_f / Kc (utilities.py:245-291)
      const double Kc = refc_pow(-M->rx_kcpow[r], refC, refCinv) * exp(arg);
      k_r = k_f / Kc;
      double hsum_r = 0.0, hsum_p = 0.0;
      for (int j = 0; j < M->rx_hr_n[r]; j++) {
        const double c = M->rx_hr_c[r * W + j];
        const double h = h_RT[M->rx_hr_sp[r * W + j]];
        hsum_r += (c == 1.0) ? h : c * h;
      }
      for (int j = 0; j < M->rx_hp_n[r]; j++) {
        const double c = M->rx_hp_c[r * W + j];
        const double h = h_RT[M->rx_hp_sp[r * W + j]];
        hsum_p += (c == 1.0) ? h : c * h;
      }
      const double snk = M->rx_sum_nuk[r];
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
        const double dlnCorrdT = ln10 * (dlogfPrdT + dlogFdT);
        dqdT = Corr * (dlnkfdT * k_f * phi_f - dkrdT * phi_r) + dlnCorrdT * q;
      } else if (has_alpha) {
        dqdT = alpha * (dlnkfdT * k_f * phi_f - dkrdT * phi_r);
      } else {
        dqdT = (dlnkfdT * k_f * phi_f - dkrdT * phi_r);
      }
    }
    const int jnn = M->rx_jn_n[r];
    const int* jsp = M->rx_jn_sp + r * PPB_MAXJN;
    const double* jc = M->rx_jn_c + r * PPB_MAXJN;
    for (int j = 0; j < jnn; j++) {
      const double nu = jc[j];
      if (nu == 1) {
        wdot[jsp[j]] += q;
      } else if (nu == -1) {
        wdot[jsp[j]] -= q;
      } else if (nu > 0) {
        wdot[jsp[j]] += nu * q;
      } else if (nu < 0) {
        wdot[jsp[j]] -= (-nu) * q;
      }
    }
    if (falloff) {
      k_f *= Corr;
      if (rev) k_r *= Corr;
    } else if (has_alpha) {
      k_f *= alpha;
      if (rev) k_r *= alpha;
    }
    double dcdc_fac = 0.0;
    if (falloff) dcdc_fac = q / alpha * (1.0 / (Pr + 1.0) + dlogFdlogPr);
    const int* hrs = M->rx_hr_sp + r * W; // reactant dict (with collider)
    const int hrn = M->rx_hr_n[r];
    const int* hps = M->rx_hp_sp + r * W; // product dict (with collider)
    const int hpn = M->rx_hp_n[r];
    if (has_alpha) {
      const double fac = falloff ? dcdc_fac : q_nocor;
      if (consP == 1) {
        for (int k = 0; k < N; k++) {
          int present = 0;
          double d = 0.0;
          for (int e = M->eff_off[r]; e < M->eff_off[r + 1]; e++) {
            if (M->eff_sp[e] == k) {
              d = (M->eff_e[e] - 1) * fac;
              present = 1;
              break;
            }
          }
          if (has_sp(hrs, hrn, k)) {
            d += k_f * dphase(fsp, fc, fn, sc, k);
            present = 1;
          }
          if (rev && has_sp(hps, hpn, k)) {
            d -= k_r * dphase(rsp, rc, rn, sc, k);
            present = 1;
          }
          if (!present) continue;
          for (int j = 0; j < jnn; j++) {
            if (jc[j] != 0) J[k * n + jsp[j]] += jc[j] * d;
          }
        }
      } else {
        for (int k = 0; k < N; k++) {
          double e = 1.0;
          for (int q2 = M->eff_off[r]; q2 < M->eff_off[r + 1]; q2++) {
            if (M->eff_sp[q2] == k) {
              e = M->eff_e[q2];
              break;
            }
          }
          const int inr = has_sp(hrs, hrn, k);
          const int inp = rev && has_sp(hps, hpn, k);
          // jacobian.py:1165-1197 with :1308-1362: a zero efficiency prints
          // as "0", which the generator treats as "no term"; with no rate
          // term either, dqdc[k] is not assigned and keeps the value of the
          // last reaction that assigned it (the loop below still reads it).
          if (e == 0.0 && !inr && !inp) continue;
          double d = (e == 0.0) ? 0.0 : ((e == 1.0) ? fac : e * fac);
          if (e == 0.0) {
            if (inr) d = k_f * dphase(fsp, fc, fn, sc, k);
            if (inp) d = (inr ? d : 0.0) - k_r * dphase(rsp, rc, rn, sc, k);
          } else {
            if (inr) d += k_f * dphase(fsp, fc, fn, sc, k);
            if (inp) d -= k_r * dphase(rsp, rc, rn, sc, k);
          }
          dqdc[k] = d;
        }
        for (int k = 0; k < N; k++) {
          for (int j = 0; j < jnn; j++) {
            if (jc[j] != 0) J[n * k + jsp[j]] += jc[j] * dqdc[k];
          }
        }
      }
      for (int j = 0; j < jnn; j++) {
        if (jc[j] != 0) J[N * n + jsp[j]] += jc[j] * dqdT;
      }
    } else {
      for (int k = 0; k < N; k++) {
        const int inr = has_sp(hrs, hrn, k);
        const int inp = rev && has_sp(hps, hpn, k);
        if (!inr && !inp) continue;
        double d = 0.0;
        if (inr) d += k_f * dphase(fsp, fc, fn, sc, k);
        if (inp) d -= k_r * dphase(rsp, rc, rn, sc, k);
        for (int j = 0; j < jnn; j++) {
          if (jc[j] != 0) J[k * n + jsp[j]] += jc[j] * d;
        }
      }
      for (int j = 0; j < jnn; j++) {
        if (jc[j] != 0) J[N * n + jsp[j]] += jc[j] * dqdT;
      }
    }
  }
  // temperature row and column (jacobian.py:203-281)
  double c_R[128], dcRdT[128], e_RT[128];
  const double* eh_RT;
  if (consP == 1) {
    ppo_cp_R(M, T, c_R);
    ppo_dcvpRdT(M, T, dcRdT);
    eh_RT = h_RT;
  } else {
    ppo_cv_R(M, T, c_R);
    ppo_dcvpRdT(M, T, dcRdT);
    ppo_species_internal_energy(M, T, e_RT);
    eh_RT = e_RT;
  }
  double cmix = 0.0, ehmix = 0.0, dcmixdT = 0.0, dehmixdT = 0.0;
  for (int k = 0; k < N; ++k) {
    cmix += c_R[k] * sc[k];
    dcmixdT += dcRdT[k] * sc[k];
    ehmix += eh_RT[k] * wdot[k];
    dehmixdT += invT * (c_R[k] - eh_RT[k]) * wdot[k] + eh_RT[k] * J[N * n + k];
  }
  const double cmixinv = 1.0 / cmix;
  const double tmp1 = ehmix * cmixinv;
  const double tmp3 = cmixinv * T;
  const double tmp2 = tmp1 * tmp3;
  for (int k = 0; k < N; ++k) {
    double dehmixdc = 0.0;
    for (int m = 0; m < N; ++m) dehmixdc += eh_RT[m] * J[k * n + m];
    J[k * n + N] = tmp2 * c_R[k] - tmp3 * dehmixdc;
  }
  J[N * n + N] = -tmp1 + tmp2 * dcmixdT - tmp3 * dehmixdT;
}

// mechanism.H DWDOT (LiDryer :5141-5160)
void ppo_dwdot(const PPBMechTables* M, double* J, const double* sc, double T, int consP)
{
  const int N = M->nsp;
  double c[128];
  for (int k = 0; k < N; k++) c[k] = 1.e6 * sc[k];
  ppo_ajacobian(M, J, c, T, consP);
  for (int k = 0; k < N; k++) {
    J[N * (N + 1) + k] *= 1.e-6;
    J[k * (N + 1) + N] *= 1.e6;
  }
}
