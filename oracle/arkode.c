// ORACLE / TEST INFRASTRUCTURE ONLY: CPU restatement of the reference's
// ReactorArkode path (Source/Reactions/ReactorArkode.cpp:134-398), the
// checker for the engine's "ReactorArkode" integrator.
//
// The reference integrates the whole batch as ONE ARKODE ERKStep/ARKStep
// problem: the state is the YCOrder vector of ncells * (N+1) entries, the
// right-hand side is fKernelSpec per cell (ReactorArkode.cpp:400-433,
// ReactorUtils.H:358-415), and the step size comes from one WRMS norm over
// all entries.  SUNDIALS (Submodules/sundials, >= v7.1 by API use) is absent
// from the reference tree, so the ERK integration is restated from ARKODE's
// published description ("ARKODE mathematical considerations": ERK methods,
// time step adaptivity, error norms, initial step size):
//   * explicit embedded tables by the reference's ode.rk_method number
//     (pelephysics_b200/csrc/ppb_erk_tables.h, exact rationals verified
//     against the Butcher order conditions);
//   * weights 1 / (rtol |y_n| + atol_i), dsm = WRMS of the embedded error
//     over the batch, accept when dsm <= 1;
//   * controllers (ReactorArkode.cpp:88-118): PID (0.58, 0.21, 0.1), PI
//     (0.8, 0.31), I (1), explicit Gustafsson (0.367, 0.268) on bias * dsm
//     (bias 1.5) with order q; safety 0.96; growth <= 1e4 on the first step,
//     20 after; no change for a proposed ratio in (1, 1.5); minimum ratio
//     0.1; after an error-test failure no growth for that step and, from the
//     second failure on, at most 0.3; 7 failures end the call;
//   * the CVODE/ARKODE initial-step estimate;
//   * ARK_NORMAL: step past tout, return the cubic Hermite interpolant at
//     tout; at most max_steps steps (ARKODE's default 500), else stop at the
//     last step reached.
#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../pelephysics_b200/csrc/ppb_erk_tables.h"
#include "oracle.h"

static const ErkTable* ark_table(int id)
{
  for (int i = 0; i < ppb_erk_ntables; i++)
    if (ppb_erk_tables[i].id == id) return &ppb_erk_tables[i];
  return ark_table(40);
}

static double ark_ctrl(int ctl, int ord, double h, double dsm, double ep, double epp, int nacc)
{
  const double e1 = fmax(1.5 * dsm, 1e-10), e2 = fmax(ep, 1e-10), e3 = fmax(epp, 1e-10);
  const double o = ord;
  switch (ctl) {
  case 2:
    return h * pow(e1, -1.0 / o);
  case 1:
    return nacc < 1 ? h * pow(e1, -0.8 / o) : h * pow(e1, -0.8 / o) * pow(e2, 0.31 / o);
  case 3:
    return nacc < 1 ? h * pow(e1, -0.367 / o) : h * pow(e1, -0.367 / o) * pow(e1 / e2, -0.268 / o);
  default:
    if (nacc < 1) return h * pow(e1, -0.58 / o);
    if (nacc < 2) return h * pow(e1, -0.58 / o) * pow(e2, 0.21 / o);
    return h * pow(e1, -0.58 / o) * pow(e2, 0.21 / o) * pow(e3, -0.1 / o);
  }
}

static double ark_eta(int ctl, int ord, double h, double dsm, double ep, double epp, int nacc, double etamax)
{
  double ha = ark_ctrl(ctl, ord, h, dsm, ep, epp, nacc) * 0.96;
  if (ha > etamax * h) ha = etamax * h;
  if (ha < 0.1 * h) ha = 0.1 * h;
  if (ha > h && ha < 1.5 * h) ha = h;
  return ha / h;
}

typedef struct ArkSys {
  const PPBMechTables* M;
  int rtype, ncells, n, N;
  const double *src, *rhoe, *rhoesrc, *atolv;
  double rtol, atol;
  const int* active;
  int nthreads;
  long nfe;
} ArkSys;

// f(t, y) for every active cell (the batch right-hand side)
static void ark_f(ArkSys* s, double t, const double* y, double* f)
{
#ifdef _OPENMP
#pragma omp parallel for schedule(static) num_threads(s->nthreads)
#endif
  for (int c = 0; c < s->ncells; c++) {
    if (!s->active[c]) continue;
    ppo_reactor_rhs(s->M, s->rtype, t, y + (long)c * s->n, f + (long)c * s->n, s->rhoe[c], s->rhoesrc[c],
                    s->src + (long)c * s->N);
  }
  s->nfe++;
}

static double ark_atol(const ArkSys* s, int i) { return s->atolv ? s->atolv[i] : s->atol; }

// sqrt(sum (v_i w_i)^2 / count) over active cells, weights from y
static double ark_wrms(const ArkSys* s, const double* v, const double* y, double scale, double ntot)
{
  double acc = 0.0;
  for (int c = 0; c < s->ncells; c++) {
    if (!s->active[c]) continue;
    for (int i = 0; i < s->n; i++) {
      const long k = (long)c * s->n + i;
      const double x = v[k] * scale / (s->rtol * fabs(y[k]) + ark_atol(s, i));
      acc += x * x;
    }
  }
  return sqrt(acc / ntot);
}

int ppo_react_arkode(
  const PPBMechTables* M, int reactor_type, const PPOArkOptions* opt, double* rY, const double* rYsrc, double* rX,
  const double* rX_src, const int* mask, double dt, int ncells, int nthreads, PPOArkStats* st)
{
  if (!M || !opt || ncells < 0) return -100;
  const int N = M->nsp, n = N + 1;
  const ErkTable* tb = ark_table(opt->rk_method);
  const int S = tb->stages;
  int fsal = tb->c[S - 1] == 1.0 && tb->b[S - 1] == 0.0;
  for (int j = 0; j < S - 1 && fsal; j++) fsal = tb->A[S - 1][j] == tb->b[j];
  const int ctl = (opt->rk_controller >= 0 && opt->rk_controller <= 3) ? opt->rk_controller : 0;
#ifdef _OPENMP
  if (nthreads <= 0) nthreads = omp_get_max_threads();
#else
  nthreads = 1;
#endif
  const long tot = (long)ncells * n;
  double* y = (double*)calloc(tot, sizeof(double));
  double* ynew = (double*)calloc(tot, sizeof(double));
  double* f0 = (double*)calloc(tot, sizeof(double));
  double* fnew = (double*)calloc(tot, sizeof(double));
  double* ytmp = (double*)calloc(tot, sizeof(double));
  double* err = (double*)calloc(tot, sizeof(double));
  double* k = (double*)calloc(tot * S, sizeof(double));
  int* active = (int*)calloc(ncells > 0 ? ncells : 1, sizeof(int));
  if (!y || !ynew || !f0 || !fnew || !ytmp || !err || !k || !active) {
    free(y), free(ynew), free(f0), free(fnew), free(ytmp), free(err), free(k), free(active);
    return -101;
  }
  memcpy(y, rY, tot * sizeof(double));
  int nact = 0;
  for (int c = 0; c < ncells; c++) {
    active[c] = !(mask && mask[c] == -1);
    nact += active[c];
  }
  ArkSys s = {M, reactor_type, ncells, n, N, rYsrc, rX, rX_src, opt->typ_vals_atol, opt->rtol, opt->atol,
              active, nthreads, 0};
  const double ntot = (double)nact * n;
  const double tout = dt;
  long nst = 0, netf = 0;
  int status = 0;
  double t = 0.0, h = 0.0;
  if (nact == 0) {
    t = tout;
    goto out;
  }
  ark_f(&s, 0.0, y, f0);
  {
    // initial step
    const double tround = DBL_EPSILON * tout;
    if (!(tout > 0.0) || tout < 2.0 * tround) {
      status = -27;
      goto out;
    }
    const double hlb = 100.0 * tround;
    double hub_inv = 0.0;
    for (int c = 0; c < ncells; c++) {
      if (!active[c]) continue;
      for (int i = 0; i < n; i++) {
        const long q = (long)c * n + i;
        const double r = fabs(f0[q]) / (0.1 * fabs(y[q]) + s.rtol * fabs(y[q]) + ark_atol(&s, i));
        if (r > hub_inv) hub_inv = r;
      }
    }
    double hub = 0.1 * tout;
    if (hub * hub_inv > 1.0) hub = 1.0 / hub_inv;
    double hg = sqrt(hlb * hub);
    if (hub < hlb) {
      h = hg;
    } else {
      double hnew = hg;
      for (int count1 = 1; count1 <= 4; count1++) {
        for (long q = 0; q < tot; q++) ytmp[q] = hg * f0[q] + y[q];
        ark_f(&s, hg, ytmp, err);
        for (long q = 0; q < tot; q++) err[q] = err[q] - f0[q];
        const double yddnrm = ark_wrms(&s, err, y, 1.0 / hg, ntot);
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
  {
    double ep = 0.0, epp = 0.0, etamax = 1.0e4;
    int nacc = 0, f_ok = 1, done = 0;
    while (!done) {
      if (nst >= opt->max_steps) {
        status = -1;
        break;
      }
      int nef = 0, accepted = 0;
      while (!accepted) {
        if (!f_ok) ark_f(&s, t, y, f0);
        f_ok = 1;
        memcpy(k, f0, tot * sizeof(double));
        for (int st_ = 1; st_ < S; st_++) {
          for (long q = 0; q < tot; q++) {
            double a = 0.0;
            for (int j = 0; j < st_; j++) a += tb->A[st_][j] * k[j * tot + q];
            ytmp[q] = y[q] + h * a;
          }
          ark_f(&s, t + tb->c[st_] * h, ytmp, k + st_ * tot);
        }
        for (long q = 0; q < tot; q++) {
          double a = 0.0, e = 0.0;
          for (int j = 0; j < S; j++) {
            a += tb->b[j] * k[j * tot + q];
            e += (tb->b[j] - tb->d[j]) * k[j * tot + q];
          }
          ynew[q] = y[q] + h * a;
          err[q] = e;
        }
        const double dsm = ark_wrms(&s, err, y, h, ntot);
        if (dsm <= 1.0) {
          const double eta = ark_eta(ctl, tb->q, h, dsm, ep, epp, nacc, etamax);
          accepted = 1;
          t += h;
          nst++;
          nacc++;
          epp = ep;
          ep = 1.5 * dsm;
          if (t >= tout) {
            // dense output at tout (cubic Hermite on [t - h, t])
            if (t > tout) {
              if (fsal) {
                memcpy(fnew, k + (S - 1) * tot, tot * sizeof(double));
              } else {
                ark_f(&s, t, ynew, fnew);
              }
              const double th = (tout - (t - h)) / h, t2 = th * th, t3 = t2 * th;
              const double h00 = 2 * t3 - 3 * t2 + 1, h10 = t3 - 2 * t2 + th, h01 = -2 * t3 + 3 * t2, h11 = t3 - t2;
              for (long q = 0; q < tot; q++)
                ytmp[q] = h00 * y[q] + h10 * h * f0[q] + h01 * ynew[q] + h11 * h * fnew[q];
              memcpy(y, ytmp, tot * sizeof(double));
            } else {
              memcpy(y, ynew, tot * sizeof(double));
            }
            t = tout;
            done = 1;
          } else {
            memcpy(y, ynew, tot * sizeof(double));
            if (fsal) {
              memcpy(f0, k + (S - 1) * tot, tot * sizeof(double));
            } else {
              f_ok = 0;
            }
            h *= eta;
            etamax = 20.0;
          }
        } else {
          netf++;
          nef++;
          if (nef >= 7) {
            status = -3;
            done = 1;
            break;
          }
          double eta = ark_eta(ctl, tb->q, h, dsm, ep, epp, nacc, etamax);
          if (eta > 1.0) eta = 1.0;
          etamax = 1.0;
          if (nef >= 2 && eta > 0.3) eta = 0.3;
          h *= eta;
          if (t + h == t) {
            status = -3;
            done = 1;
            break;
          }
        }
      }
    }
  }
out:
  for (int c = 0; c < ncells; c++) {
    if (!active[c]) continue;
    memcpy(rY + (long)c * n, y + (long)c * n, n * sizeof(double));
  }
  for (int c = 0; c < ncells; c++) rX[c] = rX[c] + t * rX_src[c];
  if (st) {
    st->t = t;
    st->h = h;
    st->nst = nst;
    st->nfe = s.nfe;
    st->netf = netf;
    st->status = status;
  }
  free(y), free(ynew), free(f0), free(fnew), free(ytmp), free(err), free(k), free(active);
  return status;
}
