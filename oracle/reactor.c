// ORACLE / TEST INFRASTRUCTURE ONLY: CPU restatement of the reference's
// reactor path for one cell at a time.
//
//  * reactor right-hand side: Source/Reactions/ReactorUtils.H:358-415
//    (fKernelSpec) over Source/Eos/Fuego.H wrappers
//  * dense analytical Jacobian: Source/Reactions/ReactorCvodeJacobian.cpp:86-152
//  * BDF integrator: the algorithm of SUNDIALS CVODE (external dependency
//    Submodules/sundials, >= v7.1 by API use, absent from the reference tree)
//    as the reference configures it in ReactorCvode.cpp:230-503 -- variable
//    order 1..max_order Nordsieck BDF with fixed-leading-coefficient
//    coefficients, WRMS local error test, modified Newton on
//    I - gamma J with a dense partial-pivoting LU, step/order selection,
//    Jacobian reuse; restated from the published CVODE method description
//    (Hindmarsh et al., "SUNDIALS: Suite of nonlinear and
//    differential/algebraic equation solvers", ACM TOMS 31, 2005; CVODE user
//    guide, "Mathematical Considerations"), which the reference docs cite in
//    Docs/sphinx/IntroductionToCvode.rst:20-101
//  * RK64: Source/Reactions/ReactorRK64.H:9-40 and ReactorRK64.cpp:73-144
#include <dlfcn.h>
#include <float.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "oracle.h"

#define NMAX 96
#define QMAX 5

// ---------------------------------------------------------------- reference
// kernels loaded from oracle/_ref (optional)
typedef double (*ref_rhs_t)(int, double, const double*, double*, double, double, const double*);
typedef void (*ref_jac_t)(int, const double*, double*);
static struct {
  char mech[64];
  void* h;
  ref_rhs_t rhs;
  ref_jac_t jac;
} g_ref[8];

int ppo_load_ref(const char* mech, const char* path)
{
  for (int i = 0; i < 8; i++) {
    if (g_ref[i].h && !strcmp(g_ref[i].mech, mech)) return 0;
  }
  for (int i = 0; i < 8; i++) {
    if (!g_ref[i].h) {
      void* h = dlopen(path, RTLD_NOW | RTLD_LOCAL);
      if (!h) return -1;
      g_ref[i].rhs = (ref_rhs_t)dlsym(h, "ref_reactor_rhs");
      g_ref[i].jac = (ref_jac_t)dlsym(h, "ref_reactor_jac");
      if (!g_ref[i].rhs || !g_ref[i].jac) {
        dlclose(h);
        return -2;
      }
      snprintf(g_ref[i].mech, sizeof(g_ref[i].mech), "%s", mech);
      g_ref[i].h = h;
      return 0;
    }
  }
  return -3;
}

static int find_ref(const char* mech)
{
  for (int i = 0; i < 8; i++)
    if (g_ref[i].h && !strcmp(g_ref[i].mech, mech)) return i;
  return -1;
}

// ------------------------------------------------------------ reactor model
double ppo_reactor_rhs(
  const PPBMechTables* M, int reactor_type, double t_rel, const double* y,
  double* ydot, double rhoe_init, double rhoesrc, const double* rYsrc)
{
  const int N = M->nsp;
  double rho = 0.0;
  for (int n = 0; n < N; n++) rho += y[n];
  const double rinv = 1.0 / rho;
  double Y[NMAX], ei[NMAX], C[NMAX], wdot[NMAX];
  for (int n = 0; n < N; n++) Y[n] = y[n] * rinv;
  const double nrg = (rhoe_init + rhoesrc * t_rel) * rinv;
  double T = y[N];
  double cv;
  if (reactor_type == 1) {
    ppo_get_t_given_ey(M, nrg, Y, &T);
    ppo_ckums(M, T, ei);
    cv = ppo_ckcvbs(M, T, Y);
  } else {
    ppo_get_t_given_hy(M, nrg, Y, &T);
    ppo_ckhms(M, T, ei);
    cv = ppo_ckcpbs(M, T, Y);
  }
  for (int n = 0; n < N; n++) C[n] = rho * Y[n] * M->imw[n];
  ppo_ckwc(M, T, C, wdot);
  double esrc = rhoesrc;
  for (int n = 0; n < N; n++) {
    const double cd = wdot[n] * M->mw[n] + rYsrc[n];
    ydot[n] = cd;
    esrc -= cd * ei[n];
  }
  ydot[N] = esrc * (rinv / cv);
  return T;
}

void ppo_reactor_jac(const PPBMechTables* M, int reactor_type, const double* y, double* J)
{
  const int N = M->nsp, n = N + 1;
  double rho = 0.0;
  for (int i = 0; i < N; i++) rho = rho + y[i];
  const double temp = y[N];
  double Y[NMAX], C[NMAX];
  static __thread double Jm[NMAX * NMAX];
  for (int i = 0; i < N; i++) Y[i] = y[i] / rho;
  for (int i = 0; i < N; i++) C[i] = rho * Y[i] * M->imw[i];
  ppo_dwdot(M, Jm, C, temp, reactor_type == 2 ? 1 : 0);
  for (int i = 0; i < N; i++) {
    double* col = J + i * n;
    for (int k = 0; k < N; k++) col[k] = Jm[i * n + k] * M->mw[k] * M->imw[i];
    col[N] = Jm[i * n + N] * M->imw[i];
  }
  double* col = J + N * n;
  for (int i = 0; i < N; i++) col[i] = Jm[N * n + i] * M->mw[i];
  col[N] = 0.0; // never written by the reference; zeroed by SUNMatZero
}

typedef struct Sys {
  const PPBMechTables* M;
  int reactor_type, ref;
  const double* rYsrc;
  double rhoe_init, rhoesrc;
  int eos; // 0 ideal gas, 1 SRK (oracle/srk.c; difference-quotient Jacobian)
  unsigned long long* noise; // right-hand-side noise stream (rhs_noise_seed), or NULL
} Sys;

// splitmix64 (Steele, Lea, Flood, "Fast splittable pseudorandom number
// generators", OOPSLA 2014)
static unsigned long long mix64(unsigned long long* x)
{
  unsigned long long z = (*x += 0x9e3779b97f4a7c15ull);
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

static void sys_f(const Sys* s, double t, const double* y, double* f)
{
  if (s->eos == 1) {
    ppo_reactor_rhs_srk(s->M->name, t, y, f, s->rhoe_init, s->rhoesrc, s->rYsrc);
  } else if (s->ref >= 0) {
    g_ref[s->ref].rhs(s->reactor_type, t, y, f, s->rhoe_init, s->rhoesrc, s->rYsrc);
  } else {
    ppo_reactor_rhs(s->M, s->reactor_type, t, y, f, s->rhoe_init, s->rhoesrc, s->rYsrc);
  }
  if (s->noise) {
    for (int i = 0; i <= s->M->nsp; i++) {
      const unsigned long long r = mix64(s->noise) % 3;
      if (r == 1) f[i] = nextafter(f[i], INFINITY);
      if (r == 2) f[i] = nextafter(f[i], -INFINITY);
    }
  }
}

static void sys_j(const Sys* s, const double* y, double* J)
{
  if (s->ref >= 0) {
    g_ref[s->ref].jac(s->reactor_type, y, J);
  } else {
    ppo_reactor_jac(s->M, s->reactor_type, y, J);
  }
}

void ppo_default_options(PPOOptions* o)
{
  // ReactorCvode.H defaults: rtol 1e-6, atol 1e-10, max_order 2; hard-coded
  // CVODE settings of ReactorCvode.cpp:480-497; RK64 ReactorRK64.H:132-134
  o->rtol = 1e-6;
  o->atol = 1e-10;
  o->max_order = 2;
  o->max_steps = 10000;
  o->max_nls_iters = 3;
  o->max_err_fails = 100;
  o->jac_eval_freq = 100;
  o->use_ref_kernels = 0;
  o->rhs_noise_seed = 0;
  o->rk64_nsubsteps_guess = 10;
  o->rk64_nsubsteps_min = 5;
  o->rk64_nsubsteps_max = 500;
  o->typ_vals = 0;
  o->eos = 0;
}

// ------------------------------------------------------------ dense LU
// Partial-pivoting LU, column-major (the SUNDIALS dense GETRF/GETRS pair).
static int lu_factor(double* a, int n, int* p)
{
  for (int k = 0; k < n; k++) {
    double* colk = a + k * n;
    int l = k;
    for (int i = k + 1; i < n; i++)
      if (fabs(colk[i]) > fabs(colk[l])) l = i;
    p[k] = l;
    if (colk[l] == 0.0) return k + 1;
    if (l != k) {
      for (int i = 0; i < n; i++) {
        double t = a[i * n + l];
        a[i * n + l] = a[i * n + k];
        a[i * n + k] = t;
      }
    }
    const double mult = 1.0 / colk[k];
    for (int i = k + 1; i < n; i++) colk[i] *= mult;
    for (int j = k + 1; j < n; j++) {
      double* colj = a + j * n;
      const double a_kj = colj[k];
      if (a_kj != 0.0)
        for (int i = k + 1; i < n; i++) colj[i] -= a_kj * colk[i];
    }
  }
  return 0;
}

static void lu_solve(const double* a, int n, const int* p, double* b)
{
  for (int k = 0; k < n; k++) {
    const int pk = p[k];
    if (pk != k) {
      double t = b[k];
      b[k] = b[pk];
      b[pk] = t;
    }
  }
  for (int k = 0; k < n - 1; k++) {
    const double* colk = a + k * n;
    const double bk = b[k];
    for (int i = k + 1; i < n; i++) b[i] -= colk[i] * bk;
  }
  for (int k = n - 1; k > 0; k--) {
    const double* colk = a + k * n;
    b[k] /= colk[k];
    const double bk = b[k];
    for (int i = 0; i < k; i++) b[i] -= colk[i] * bk;
  }
  b[0] /= a[0];
}

// ------------------------------------------------------------ CVODE BDF
enum { FIRST_CALL = 0, PREV_CONV_FAIL = 1, PREV_ERR_FAIL = 2 };
enum { CV_SUCCESS = 0, CV_TOO_MUCH_WORK = -1, CV_ERR_FAILURE = -3, CV_CONV_FAILURE = -4,
       CV_LSETUP_FAIL = -6, CV_TOO_CLOSE = -27 };
enum { DO_ERROR_TEST = 2, PREDICT_AGAIN = 3, TRY_AGAIN = 5 };
enum { CV_NO_FAILURES = 0, CV_FAIL_BAD_J = 1, CV_FAIL_OTHER = 2 };
#define ETAMX1 10000.0
#define ETAMX2 10.0
#define ETAMX3 10.0
#define ETAMXF 0.2
#define ETAMIN 0.1
#define ETACF 0.25
#define ADDON 1.0e-6
#define BIAS1 6.0
#define BIAS2 6.0
#define BIAS3 10.0
#define ONEPSM 1.000001
#define SMALL_NST 10
#define MXNCF 10
#define MXNEF1 3
#define SMALL_NEF 2
#define LONG_WAIT 10
#define CRDOWN 0.3
#define DGMAX_LSETUP 0.3
#define RDIV 2.0
#define MSBP 20
#define CVLS_DGMAX 0.2
#define NLSCOEF 0.1
#define ETA_MAX_FX 1.5

typedef struct BDF {
  int n;
  double zn[QMAX + 1][NMAX];
  double ewt[NMAX], acor[NMAX], y[NMAX], tempv[NMAX], ftemp[NMAX], delta[NMAX];
  double savedJ[NMAX * NMAX], A[NMAX * NMAX];
  int piv[NMAX];
  double tau[QMAX + 2], tq[6], l[QMAX + 1];
  double h, hprime, hscale, eta, etamax, etaq, etaqm1, etaqp1, tn, rl1, gamma, gammap,
    gamrat, crate, delp, acnrm, saved_tq5, hu;
  int q, qprime, qwait, L, qmax, indx_acor;
  long nst, nstlp, nstlj, nscon, nfe, nje, nsetups, nni, ncfn, netf;
  int jcur; // Newton solver's notion of a current Jacobian
  double rtol;
  const double* atolv;
  double atol;
  int maxcor, maxnef, msbj;
  const Sys* sys;
} BDF;

static double wrms(const BDF* b, const double* v)
{
  double s = 0.0;
  for (int i = 0; i < b->n; i++) {
    const double x = v[i] * b->ewt[i];
    s += x * x;
  }
  return sqrt(s / b->n);
}

static void set_ewt(BDF* b, const double* y)
{
  for (int i = 0; i < b->n; i++) {
    const double at = b->atolv ? b->atolv[i] : b->atol;
    b->ewt[i] = 1.0 / (b->rtol * fabs(y[i]) + at);
  }
}

static void f_eval(BDF* b, double t, const double* y, double* f)
{
  sys_f(b->sys, t, y, f);
  b->nfe++;
}

static double upper_bound_h0(BDF* b, double tdist)
{
  double hub_inv = 0.0;
  for (int i = 0; i < b->n; i++) {
    const double t1 = 0.1 * fabs(b->zn[0][i]) + 1.0 / b->ewt[i];
    const double r = fabs(b->zn[1][i]) / t1;
    if (r > hub_inv) hub_inv = r;
  }
  double hub = 0.1 * tdist;
  if (hub * hub_inv > 1.0) hub = 1.0 / hub_inv;
  return hub;
}

static double ydd_norm(BDF* b, double hg)
{
  for (int i = 0; i < b->n; i++) b->y[i] = hg * b->zn[1][i] + b->zn[0][i];
  f_eval(b, b->tn + hg, b->y, b->tempv);
  for (int i = 0; i < b->n; i++) b->tempv[i] = (b->tempv[i] - b->zn[1][i]) * (1.0 / hg);
  return wrms(b, b->tempv);
}

static int cv_hin(BDF* b, double tout)
{
  const double tdiff = tout - b->tn;
  if (tdiff == 0.0) return CV_TOO_CLOSE;
  const double tdist = fabs(tdiff);
  const double tround = DBL_EPSILON * fmax(fabs(b->tn), fabs(tout));
  if (tdist < 2.0 * tround) return CV_TOO_CLOSE;
  const double hlb = 100.0 * tround;
  const double hub = upper_bound_h0(b, tdist);
  double hg = sqrt(hlb * hub);
  if (hub < hlb) {
    b->h = hg;
    return CV_SUCCESS;
  }
  double hnew = hg;
  for (int count1 = 1; count1 <= 4; count1++) {
    const double yddnrm = ydd_norm(b, hg);
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
  b->h = h0;
  return CV_SUCCESS;
}

static void cv_rescale(BDF* b)
{
  double factor = b->eta;
  for (int j = 1; j <= b->q; j++) {
    for (int i = 0; i < b->n; i++) b->zn[j][i] *= factor;
    factor *= b->eta;
  }
  b->h = b->hscale * b->eta;
  b->hscale = b->h;
  b->nscon = 0;
}

static void cv_predict(BDF* b)
{
  b->tn += b->h;
  for (int k = 1; k <= b->q; k++)
    for (int j = b->q; j >= k; j--)
      for (int i = 0; i < b->n; i++) b->zn[j - 1][i] += b->zn[j][i];
}

static void cv_restore(BDF* b, double saved_t)
{
  b->tn = saved_t;
  for (int k = 1; k <= b->q; k++)
    for (int j = b->q; j >= k; j--)
      for (int i = 0; i < b->n; i++) b->zn[j - 1][i] -= b->zn[j][i];
}

static void cv_set_bdf(BDF* b)
{
  double alpha0, alpha0_hat, xi_inv, xistar_inv, hsum;
  const int q = b->q;
  b->l[0] = b->l[1] = xi_inv = xistar_inv = 1.0;
  for (int i = 2; i <= q; i++) b->l[i] = 0.0;
  alpha0 = alpha0_hat = -1.0;
  hsum = b->h;
  if (q > 1) {
    for (int j = 2; j < q; j++) {
      hsum += b->tau[j - 1];
      xi_inv = b->h / hsum;
      alpha0 -= 1.0 / j;
      for (int i = j; i >= 1; i--) b->l[i] += b->l[i - 1] * xi_inv;
    }
    alpha0 -= 1.0 / q;
    xistar_inv = -b->l[1] - alpha0;
    hsum += b->tau[q - 1];
    xi_inv = b->h / hsum;
    alpha0_hat = -b->l[1] - xi_inv;
    for (int i = q; i >= 1; i--) b->l[i] += b->l[i - 1] * xistar_inv;
  }
  // tq (cvSetTqBDF)
  const double A1 = 1.0 - alpha0_hat + alpha0;
  const double A2 = 1.0 + q * A1;
  b->tq[2] = fabs(A1 / (alpha0 * A2));
  b->tq[5] = fabs(A2 * xistar_inv / (b->l[q] * xi_inv));
  if (b->qwait == 1) {
    if (q > 1) {
      const double C = xistar_inv / b->l[q];
      const double A3 = alpha0 + 1.0 / q;
      const double A4 = alpha0_hat + xi_inv;
      const double Cpinv = (1.0 - A4 + A3) / A3;
      b->tq[1] = fabs(C * Cpinv);
    } else {
      b->tq[1] = 1.0;
    }
    hsum += b->tau[q];
    xi_inv = b->h / hsum;
    const double A5 = alpha0 - (1.0 / (q + 1));
    const double A6 = alpha0_hat - xi_inv;
    const double Cppinv = (1.0 - A6 + A5) / A2;
    b->tq[3] = fabs(Cppinv / (xi_inv * (q + 2) * A5));
  }
  b->tq[4] = NLSCOEF / b->tq[2];
}

static void cv_set(BDF* b)
{
  cv_set_bdf(b);
  b->rl1 = 1.0 / b->l[1];
  b->gamma = b->h * b->rl1;
  if (b->nst == 0) b->gammap = b->gamma;
  b->gamrat = (b->nst > 0) ? b->gamma / b->gammap : 1.0;
}

// cvLsSetup with a matrix-based direct solver
// CVODE's dense difference-quotient Jacobian (the reference's path when
// the EOS has no analytical Jacobian, Source/Eos/SRK.H:640-648) at
// (tn, y) with f(tn, y) in ftemp: column j with inc = max(sqrt(eps)|y_j|,
// min_inc / ewt_j), min_inc = 1000 |h| eps n ||f||_WRMS (1 if ||f|| = 0).
// Its evaluations are not counted in nfe.
static void dq_jac(BDF* b)
{
  const int n = b->n;
  const double fnorm = wrms(b, b->ftemp);
  const double srur = sqrt(DBL_EPSILON);
  const double min_inc = (fnorm != 0.0) ? (1000.0 * fabs(b->h) * DBL_EPSILON * n * fnorm) : 1.0;
  double yp[NMAX];
  memcpy(yp, b->y, sizeof(double) * n);
  for (int j = 0; j < n; j++) {
    const double yj = yp[j];
    const double inc = fmax(srur * fabs(yj), min_inc / b->ewt[j]);
    yp[j] = yj + inc;
    double* col = b->savedJ + (long)j * n;
    sys_f(b->sys, b->tn, yp, col);
    const double inc_inv = 1.0 / inc;
    for (int i = 0; i < n; i++) col[i] = inc_inv * col[i] + (-inc_inv) * b->ftemp[i];
    yp[j] = yj;
  }
}

static int ls_setup(BDF* b, int convfail)
{
  const int n = b->n;
  const double dgamma = fabs((b->gamma / b->gammap) - 1.0);
  const int jbad = (b->nst == 0) || (b->nst >= b->nstlj + b->msbj) ||
                   ((convfail == CV_FAIL_BAD_J) && (dgamma < CVLS_DGMAX)) ||
                   (convfail == CV_FAIL_OTHER);
  if (!jbad) {
    b->jcur = 0;
  } else {
    b->nje++;
    b->nstlj = b->nst;
    b->jcur = 1;
    if (b->sys->eos == 1 || b->sys->M->nqss > 0) {
      // SRK, or a QSS mechanism (its analytical Jacobian needs CEPTR's
      // symbolic build; the reference's dense_direct solve differences f)
      dq_jac(b);
    } else {
      sys_j(b->sys, b->y, b->savedJ);
    }
  }
  for (int i = 0; i < n * n; i++) b->A[i] = -b->gamma * b->savedJ[i];
  for (int i = 0; i < n; i++) b->A[i * n + i] += 1.0;
  const int ier = lu_factor(b->A, n, b->piv);
  return ier ? 1 : 0;
}

// cvNlsResidual: res = rl1*zn[1] + ycor - gamma*f(tn, zn[0]+ycor)
static void nls_residual(BDF* b)
{
  for (int i = 0; i < b->n; i++) b->y[i] = b->zn[0][i] + b->acor[i];
  f_eval(b, b->tn, b->y, b->ftemp);
  for (int i = 0; i < b->n; i++) {
    const double r = b->rl1 * b->zn[1][i] + b->acor[i];
    b->delta[i] = -b->gamma * b->ftemp[i] + r;
  }
}

// cvNls + SUNNonlinSol_Newton: returns 0 on success, >0 recoverable
// convergence failure, <0 unrecoverable (linear setup failure).
static int cv_nls(BDF* b, int nflag)
{
  int convfail = ((nflag == FIRST_CALL) || (nflag == PREV_ERR_FAIL)) ? CV_NO_FAILURES : CV_FAIL_OTHER;
  int callSetup = (nflag == PREV_CONV_FAIL) || (nflag == PREV_ERR_FAIL) || (b->nst == 0) ||
                  (b->nst >= b->nstlp + MSBP) || (fabs(b->gamrat - 1.0) > DGMAX_LSETUP);
  for (int i = 0; i < b->n; i++) b->acor[i] = 0.0;
  int jbad = 0;
  int retval;
  for (;;) {
    nls_residual(b);
    if (callSetup) {
      int cf = jbad ? CV_FAIL_BAD_J : convfail;
      const int ier = ls_setup(b, cf);
      b->nsetups++;
      b->gamrat = 1.0;
      b->gammap = b->gamma;
      b->crate = 1.0;
      b->nstlp = b->nst;
      if (ier) return -1;
    }
    int m = 0;
    for (;;) {
      b->nni++;
      for (int i = 0; i < b->n; i++) b->delta[i] = -b->delta[i];
      lu_solve(b->A, b->n, b->piv, b->delta);
      if (b->gamrat != 1.0) {
        const double s = 2.0 / (1.0 + b->gamrat);
        for (int i = 0; i < b->n; i++) b->delta[i] *= s;
      }
      for (int i = 0; i < b->n; i++) b->acor[i] += b->delta[i];
      // cvNlsConvTest
      const double del = wrms(b, b->delta);
      if (m > 0) b->crate = fmax(CRDOWN * b->crate, del / b->delp);
      const double dcon = del * fmin(1.0, b->crate) / b->tq[4];
      if (dcon <= 1.0) {
        b->acnrm = (m == 0) ? del : wrms(b, b->acor);
        b->jcur = 0;
        for (int i = 0; i < b->n; i++) b->y[i] = b->zn[0][i] + b->acor[i];
        return 0;
      }
      if ((m >= 1) && (del > RDIV * b->delp)) {
        retval = 1;
        break;
      }
      b->delp = del;
      m++;
      if (m >= b->maxcor) {
        retval = 1;
        break;
      }
      nls_residual(b);
    }
    if (retval > 0 && !b->jcur) {
      callSetup = 1;
      jbad = 1;
      for (int i = 0; i < b->n; i++) b->acor[i] = 0.0;
      continue;
    }
    break;
  }
  for (int i = 0; i < b->n; i++) b->y[i] = b->zn[0][i] + b->acor[i];
  return retval;
}

static int cv_handle_nflag(BDF* b, int* nflag, double saved_t, int* ncf)
{
  if (*nflag == 0) return DO_ERROR_TEST;
  b->ncfn++;
  cv_restore(b, saved_t);
  if (*nflag < 0) return CV_LSETUP_FAIL;
  (*ncf)++;
  b->etamax = 1.0;
  if (*ncf == MXNCF) return CV_CONV_FAILURE;
  b->eta = ETACF;
  *nflag = PREV_CONV_FAIL;
  cv_rescale(b);
  return PREDICT_AGAIN;
}

static void cv_increase_bdf(BDF* b)
{
  double alpha0, alpha1, prod, xi, xiold, hsum, A1;
  for (int i = 0; i <= b->qmax; i++) b->l[i] = 0.0;
  b->l[2] = alpha1 = prod = xiold = 1.0;
  alpha0 = -1.0;
  hsum = b->hscale;
  if (b->q > 1) {
    for (int j = 1; j < b->q; j++) {
      hsum += b->tau[j + 1];
      xi = hsum / b->hscale;
      prod *= xi;
      alpha0 -= 1.0 / (j + 1);
      alpha1 += 1.0 / xi;
      for (int i = j + 2; i >= 2; i--) b->l[i] = b->l[i] * xiold + b->l[i - 1];
      xiold = xi;
    }
  }
  A1 = (-alpha0 - alpha1) / prod;
  for (int i = 0; i < b->n; i++) b->zn[b->L][i] = A1 * b->zn[b->indx_acor][i];
  for (int j = 2; j <= b->q; j++)
    for (int i = 0; i < b->n; i++) b->zn[j][i] += b->l[j] * b->zn[b->L][i];
}

static void cv_decrease_bdf(BDF* b)
{
  double hsum, xi;
  for (int i = 0; i <= b->qmax; i++) b->l[i] = 0.0;
  b->l[2] = 1.0;
  hsum = 0.0;
  for (int j = 1; j <= b->q - 2; j++) {
    hsum += b->tau[j];
    xi = hsum / b->hscale;
    for (int i = j + 2; i >= 2; i--) b->l[i] = b->l[i] * xi + b->l[i - 1];
  }
  for (int j = 2; j < b->q; j++)
    for (int i = 0; i < b->n; i++) b->zn[j][i] -= b->l[j] * b->zn[b->q][i];
}

static void cv_adjust_order(BDF* b, int deltaq)
{
  if ((b->q == 2) && (deltaq != 1)) return;
  if (deltaq == 1) cv_increase_bdf(b);
  else if (deltaq == -1) cv_decrease_bdf(b);
}

static int cv_do_error_test(BDF* b, int* nflag, double saved_t, int* nef, double* dsmp)
{
  const double dsm = b->acnrm * b->tq[2];
  *dsmp = dsm;
  if (dsm <= 1.0) return CV_SUCCESS;
  (*nef)++;
  b->netf++;
  *nflag = PREV_ERR_FAIL;
  cv_restore(b, saved_t);
  if (*nef == b->maxnef) return CV_ERR_FAILURE;
  b->etamax = 1.0;
  if (*nef <= MXNEF1) {
    b->eta = 1.0 / (pow(BIAS2 * dsm, 1.0 / b->L) + ADDON);
    b->eta = fmax(ETAMIN, b->eta);
    if (*nef >= SMALL_NEF) b->eta = fmin(b->eta, ETAMXF);
    cv_rescale(b);
    return TRY_AGAIN;
  }
  if (b->q > 1) {
    b->eta = ETAMIN;
    cv_adjust_order(b, -1);
    b->L = b->q;
    b->q--;
    b->qwait = b->L;
    cv_rescale(b);
    return TRY_AGAIN;
  }
  b->eta = ETAMIN;
  b->h *= b->eta;
  b->hscale = b->h;
  b->qwait = LONG_WAIT;
  b->nscon = 0;
  f_eval(b, b->tn, b->zn[0], b->tempv);
  for (int i = 0; i < b->n; i++) b->zn[1][i] = b->h * b->tempv[i];
  return TRY_AGAIN;
}

static void cv_complete_step(BDF* b)
{
  b->nst++;
  b->nscon++;
  b->hu = b->h;
  for (int i = b->q; i >= 2; i--) b->tau[i] = b->tau[i - 1];
  if ((b->q == 1) && (b->nst > 1)) b->tau[2] = b->tau[1];
  b->tau[1] = b->h;
  for (int j = 0; j <= b->q; j++)
    for (int i = 0; i < b->n; i++) b->zn[j][i] += b->l[j] * b->acor[i];
  b->qwait--;
  if ((b->qwait == 1) && (b->q != b->qmax)) {
    for (int i = 0; i < b->n; i++) b->zn[b->qmax][i] = b->acor[i];
    b->saved_tq5 = b->tq[5];
    b->indx_acor = b->qmax;
  }
}

static void cv_set_eta(BDF* b)
{
  if ((b->eta > 0.0) && (b->eta < ETA_MAX_FX)) {
    b->eta = 1.0;
    b->hprime = b->h;
  } else {
    b->eta = fmin(b->eta, b->etamax);
    b->hprime = b->h * b->eta;
  }
}

static void cv_prepare_next_step(BDF* b, double dsm)
{
  if (b->etamax == 1.0) {
    b->qwait = b->qwait > 2 ? b->qwait : 2;
    b->qprime = b->q;
    b->hprime = b->h;
    b->eta = 1.0;
    return;
  }
  b->etaq = 1.0 / (pow(BIAS2 * dsm, 1.0 / b->L) + ADDON);
  if (b->qwait != 0) {
    b->eta = b->etaq;
    b->qprime = b->q;
    cv_set_eta(b);
    return;
  }
  b->qwait = 2;
  // cvComputeEtaqm1
  b->etaqm1 = 0.0;
  if (b->q > 1) {
    const double ddn = wrms(b, b->zn[b->q]) * b->tq[1];
    b->etaqm1 = 1.0 / (pow(BIAS1 * ddn, 1.0 / b->q) + ADDON);
  }
  // cvComputeEtaqp1
  b->etaqp1 = 0.0;
  if (b->q != b->qmax && b->saved_tq5 != 0.0) {
    const double cquot = (b->tq[5] / b->saved_tq5) * pow(b->h / b->tau[2], (double)b->L);
    for (int i = 0; i < b->n; i++) b->tempv[i] = -cquot * b->zn[b->qmax][i] + b->acor[i];
    const double dup = wrms(b, b->tempv) * b->tq[3];
    b->etaqp1 = 1.0 / (pow(BIAS3 * dup, 1.0 / (b->L + 1)) + ADDON);
  }
  // cvChooseEta
  const double etam = fmax(b->etaqm1, fmax(b->etaq, b->etaqp1));
  if ((etam > 0.0) && (etam < ETA_MAX_FX)) {
    b->eta = 1.0;
    b->qprime = b->q;
  } else if (etam == b->etaq) {
    b->eta = b->etaq;
    b->qprime = b->q;
  } else if (etam == b->etaqm1) {
    b->eta = b->etaqm1;
    b->qprime = b->q - 1;
  } else {
    b->eta = b->etaqp1;
    b->qprime = b->q + 1;
    for (int i = 0; i < b->n; i++) b->zn[b->qmax][i] = b->acor[i];
  }
  cv_set_eta(b);
}

static void cv_adjust_params(BDF* b)
{
  if (b->qprime != b->q) {
    cv_adjust_order(b, b->qprime - b->q);
    b->q = b->qprime;
    b->L = b->q + 1;
    b->qwait = b->L;
  }
  cv_rescale(b);
}

static int cv_step(BDF* b)
{
  const double saved_t = b->tn;
  int ncf = 0, nef = 0, nflag = FIRST_CALL;
  double dsm = 0.0;
  if ((b->nst > 0) && (b->hprime != b->h)) cv_adjust_params(b);
  for (;;) {
    cv_predict(b);
    cv_set(b);
    nflag = cv_nls(b, nflag);
    const int kflag = cv_handle_nflag(b, &nflag, saved_t, &ncf);
    if (kflag == PREDICT_AGAIN) continue;
    if (kflag != DO_ERROR_TEST) return kflag;
    const int eflag = cv_do_error_test(b, &nflag, saved_t, &nef, &dsm);
    if (eflag == TRY_AGAIN) continue;
    if (eflag != CV_SUCCESS) return eflag;
    break;
  }
  cv_complete_step(b);
  cv_prepare_next_step(b, dsm);
  b->etamax = (b->nst <= SMALL_NST) ? ETAMX2 : ETAMX3;
  return CV_SUCCESS;
}

// CVodeGetDky(t, 0): Horner on the Nordsieck array
static void cv_dky0(const BDF* b, double t, double* out)
{
  const double s = (t - b->tn) / b->h;
  for (int i = 0; i < b->n; i++) {
    double v = b->zn[b->q][i];
    for (int j = b->q - 1; j >= 0; j--) v = b->zn[j][i] + s * v;
    out[i] = v;
  }
}

int ppo_bdf_cell(
  const PPBMechTables* M, int reactor_type, const PPOOptions* opt, double* y,
  const double* rYsrc, double rhoe_init, double rhoesrc, double dt, PPOStats* st)
{
  Sys sys = {M, reactor_type, -1, rYsrc, rhoe_init, rhoesrc, opt->eos, NULL};
  if (opt->use_ref_kernels) sys.ref = find_ref(M->name);
  unsigned long long noise = 0;
  if (opt->rhs_noise_seed) { // a stream per cell: the seed mixed with the cell's input bits
    noise = opt->rhs_noise_seed;
    for (int i = 0; i <= M->nsp; i++) {
      unsigned long long u;
      memcpy(&u, &y[i], sizeof(u));
      noise ^= u + 0x9e3779b97f4a7c15ull + (noise << 6) + (noise >> 2);
    }
    sys.noise = &noise;
  }
  BDF* b = (BDF*)calloc(1, sizeof(BDF));
  const int n = M->nsp + 1;
  double atolv[NMAX];
  b->n = n;
  b->sys = &sys;
  b->rtol = opt->rtol;
  b->atol = opt->atol;
  if (opt->typ_vals) {
    for (int i = 0; i < n; i++) atolv[i] = opt->typ_vals[i] * opt->atol;
    b->atolv = atolv;
  }
  b->maxcor = opt->max_nls_iters;
  b->maxnef = opt->max_err_fails;
  b->msbj = opt->jac_eval_freq;
  b->qmax = opt->max_order;
  b->q = 1;
  b->L = 2;
  b->qwait = b->L;
  b->etamax = ETAMX1;
  b->tn = 0.0;
  const double tout = dt;
  for (int i = 0; i < n; i++) b->zn[0][i] = y[i];
  set_ewt(b, b->zn[0]);
  f_eval(b, b->tn, b->zn[0], b->zn[1]);
  int flag = cv_hin(b, tout);
  if (flag == CV_SUCCESS) {
    b->hscale = b->h;
    b->hprime = b->h;
    for (int i = 0; i < n; i++) b->zn[1][i] *= b->h;
    long nstloc = 0;
    for (;;) {
      if (b->nst > 0) set_ewt(b, b->zn[0]);
      if (nstloc >= opt->max_steps) {
        flag = CV_TOO_MUCH_WORK;
        break;
      }
      flag = cv_step(b);
      if (flag != CV_SUCCESS) break;
      nstloc++;
      if ((b->tn - tout) * b->h >= 0.0) {
        cv_dky0(b, tout, y);
        break;
      }
    }
  }
  if (flag != CV_SUCCESS) {
    for (int i = 0; i < n; i++) y[i] = b->zn[0][i];
  }
  if (st) {
    st->nsteps = b->nst;
    st->nfe = b->nfe;
    st->nje = b->nje;
    st->nsetups = b->nsetups;
    st->nni = b->nni;
    st->ncfn = b->ncfn;
    st->netf = b->netf;
    st->status = flag;
    st->last_order = b->q;
    st->last_h = b->h;
  }
  free(b);
  return flag;
}

// ------------------------------------------------------------ RK64
int ppo_rk64_cell(
  const PPBMechTables* M, int reactor_type, const PPOOptions* opt, double* y,
  const double* rYsrc, double rhoe_init, double rhoesrc, double dt)
{
  static const double alpha[6] = {0.218150805229859, 0.256702469801519, 0.527402592007520,
                                  0.0484864267224467, 1.24517071533530, 0.412366034843237};
  static const double beta[6] = {-0.113554138044166, -0.215118587818400, -0.0510152146250577,
                                 -1.07992686223881, -0.248664241213447, 0.0};
  static const double err[6] = {-0.0554699315064507, 0.158481845574980, -0.0905918835751907,
                                -0.219084567203338, 0.164022338959433, 0.0426421977505659};
  Sys sys = {M, reactor_type, -1, rYsrc, rhoe_init, rhoesrc, opt->eos};
  if (opt->use_ref_kernels) sys.ref = find_ref(M->name);
  const int neq = M->nsp + 1;
  double soln[NMAX], carry[NMAX], error[NMAX], ydot[NMAX];
  const double time_init = 0.0, time_out = dt;
  double t = time_init;
  for (int i = 0; i < neq; i++) soln[i] = carry[i] = y[i];
  double dt_rk = dt / (double)opt->rk64_nsubsteps_guess;
  const double dt_rk_min = dt / (double)opt->rk64_nsubsteps_max;
  const double dt_rk_max = dt / (double)opt->rk64_nsubsteps_min;
  int nsteps = 0;
  while (t < time_out) {
    for (int i = 0; i < neq; i++) error[i] = 0.0;
    for (int s = 0; s < 6; s++) {
      sys_f(&sys, t - time_init, soln, ydot);
      for (int i = 0; i < neq; i++) {
        error[i] += err[s] * dt_rk * ydot[i];
        soln[i] = carry[i] + alpha[s] * dt_rk * ydot[i];
        carry[i] = soln[i] + beta[s] * dt_rk * ydot[i];
      }
    }
    t += dt_rk;
    nsteps++;
    double max_err = 1e-50;
    for (int i = 0; i < neq; i++) max_err = fabs(error[i]) > max_err ? fabs(error[i]) : max_err;
    if (max_err < opt->atol) {
      const double cf = 1.0 * pow((opt->atol / max_err), 0.25);
      dt_rk = fmin(dt_rk_max, dt_rk * cf);
    } else {
      const double cf = 1.0 * pow((opt->atol / max_err), 0.2);
      dt_rk = fmax(dt_rk_min, dt_rk * cf);
    }
    dt_rk = fmin(dt_rk, time_out - t);
  }
  for (int i = 0; i < neq; i++) y[i] = soln[i];
  return nsteps;
}

// ------------------------------------------------------------ flat react
int ppo_react_flat(
  const char* mech, int reactor_type, const PPOOptions* opt, int method,
  double* rY, const double* rYsrc, double* rX, const double* rX_src, double dt,
  int ncells, int nthreads, long* nfe_out, int* status_out)
{
  const PPBMechTables* M = ppo_mech(mech);
  if (!M) return -100;
  return ppo_react_flat_tables(M, reactor_type, opt, method, rY, rYsrc, rX, rX_src, dt, ncells, nthreads,
                               nfe_out, status_out);
}

PPBMechTables* ppo_mech_with_arrhenius(const char* name, const double* A, const double* beta, const double* EaR)
{
  const PPBMechTables* M = ppo_mech(name);
  if (!M) return 0;
  PPBMechTables* C = (PPBMechTables*)malloc(sizeof(PPBMechTables));
  double* buf = (double*)malloc(sizeof(double) * 3 * (size_t)M->nrxn);
  if (!C || !buf) {
    free(C);
    free(buf);
    return 0;
  }
  *C = *M;
  for (int r = 0; r < M->nrxn; r++) {
    buf[r] = A[r];
    buf[M->nrxn + r] = beta[r];
    buf[2 * M->nrxn + r] = EaR[r];
  }
  C->rx_A = buf;
  C->rx_beta = buf + M->nrxn;
  C->rx_EaR = buf + 2 * M->nrxn;
  return C;
}

void ppo_mech_free(PPBMechTables* M)
{
  if (!M) return;
  free((void*)M->rx_A);
  free(M);
}

static int react_flat_impl(
  const PPBMechTables* M, int reactor_type, const PPOOptions* opt, int method,
  double* rY, const double* rYsrc, double* rX, const double* rX_src, double dt,
  int ncells, int nthreads, long* nfe_out, int* status_out, long* stats_out)
{
  if (!M) return -100;
  const int N = M->nsp;
  int first_err = 0;
#ifdef _OPENMP
  if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
#endif
  for (int c = 0; c < ncells; c++) {
    double* y = rY + (long)c * (N + 1);
    const double* src = rYsrc + (long)c * N;
    if (method == 0) {
      PPOStats st;
      const int f = ppo_bdf_cell(M, reactor_type, opt, y, src, rX[c], rX_src[c], dt, &st);
      if (nfe_out) nfe_out[c] = st.nfe;
      if (status_out) status_out[c] = f;
      if (stats_out) {
        long* o = stats_out + (long)c * 7;
        o[0] = st.nsteps;
        o[1] = st.nfe;
        o[2] = st.nje;
        o[3] = st.nsetups;
        o[4] = st.nni;
        o[5] = st.netf;
        o[6] = st.ncfn;
      }
      if (f != 0) {
#ifdef _OPENMP
#pragma omp critical
#endif
        if (!first_err) first_err = f;
      }
    } else {
      const int ns = ppo_rk64_cell(M, reactor_type, opt, y, src, rX[c], rX_src[c], dt);
      if (nfe_out) nfe_out[c] = ns;
      if (status_out) status_out[c] = 0;
      if (stats_out) {
        long* o = stats_out + (long)c * 7;
        o[0] = ns;
        o[1] = 6L * ns;
        for (int q = 2; q < 7; q++) o[q] = 0;
      }
    }
    rX[c] = rX[c] + dt * rX_src[c];
  }
  return first_err;
}

int ppo_react_flat_tables(
  const PPBMechTables* M, int reactor_type, const PPOOptions* opt, int method,
  double* rY, const double* rYsrc, double* rX, const double* rX_src, double dt,
  int ncells, int nthreads, long* nfe_out, int* status_out)
{
  return react_flat_impl(M, reactor_type, opt, method, rY, rYsrc, rX, rX_src, dt, ncells, nthreads, nfe_out,
                         status_out, 0);
}

int ppo_react_flat_stats(
  const char* mech, int reactor_type, const PPOOptions* opt, int method,
  double* rY, const double* rYsrc, double* rX, const double* rX_src, double dt,
  int ncells, int nthreads, int* status_out, long* stats_out)
{
  return react_flat_impl(ppo_mech(mech), reactor_type, opt, method, rY, rYsrc, rX, rX_src, dt, ncells, nthreads,
                         0, status_out, stats_out);
}
