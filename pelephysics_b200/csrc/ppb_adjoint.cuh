// Discrete adjoint and tangent-linear model of the BDF integration.
//
// The forward integration (Bdf in ppb_bdf.cuh, the CVODE algorithm) changes
// its Nordsieck history Z = (z_0 .. z_qmax) only through a short list of
// operations, which a recorder (AdjRec) writes to a per-warp tape with the
// coefficients they used:
//
//   INIT     z_0 = y0, z_1 = h0 f(0, y0)                      (cvInitialSetup)
//   FRESET   z_1 = h f(t_n, z_0)                  (cvDoErrorTest, q = 1 reset)
//   RESCALE  z_j *= eta^j, j = 1..q                                (cvRescale)
//   PREDICT  z_{j-1} += z_j (Pascal triangle)                      (cvPredict)
//   CORRECT  a solves a + rl1 z_1 = gamma f(t_n, z_0 + a); z_j += l_j a,
//            optionally z_qmax = a                    (cvNls + cvCompleteStep)
//   SAVEQMAX z_qmax = a of the last correction               (cvPrepareNextStep)
//   INCREASE z_L = A1 z_idx; z_j += l_j z_L               (cvIncreaseBDF)
//   DECREASE z_j -= l_j z_q                                (cvDecreaseBDF)
//   OUTPUT   y(tout) = sum_j s^j z_j                             (CVodeGetDky)
//
// Step sizes, orders and the coefficients are frozen at their forward
// values (the controller is not differentiated); rejected attempts leave no
// trace except their RESCALE / DECREASE / FRESET operations, because
// restore() undoes predict() exactly in exact arithmetic.  The correction
// is differentiated at its converged value by the implicit-function theorem
// with the exact Jacobian of the right-hand side, so the adjoint is the exact
// transpose of the tangent-linear model of the recorded scheme.
//
// The right-hand side differentiated is the reactor RHS as evaluated
// (fKernelSpec, ReactorUtils.H:358-415): T comes from the energy constraint
// sum_k y_k e_k(T) = E(t), E(t) = rhoe + rhoesrc t, so f does not depend on
// the T slot y_N, and dT/dy_k = -e_k / (rho c_v).  The production-rate
// derivatives are the exact partials (the consP = 0 form of the reference's
// analytical Jacobian, jacobian.py:546-1305, without its reuse of a stale
// dq/dc for zero-efficiency species).  Parameters: per reaction ln A, beta
// and Ea/R of the forward (for fall-off: high-pressure) Arrhenius rate.
#pragma once
#include "ppb_bdf.cuh"

namespace ppb {

enum { ST_ADJ_CAPACITY = -40, ST_ADJ_SINGULAR = -41, ST_ADJ_REPLAY = -42 };


enum TapeOp : int {
  TP_FRESET = 1,
  TP_RESCALE,
  TP_PREDICT,
  TP_CORRECT,
  TP_SAVEQMAX,
  TP_INCREASE,
  TP_DECREASE,
  TP_OUTPUT
};

// One tape record: 7 x 16 bytes.
struct alignas(16) TapeRec {
  int op, q, i1, i2;
  double c[12];
};
static_assert(sizeof(TapeRec) == 112, "TapeRec is seven 16-byte words");

// Integrator recorder writing one segment of operations to a per-warp tape
// in global memory.  All lanes of the team call every hook with the same
// arguments; lane 0 writes the record, the lanes write the vectors.
template <int TEAM>
struct AdjRec {
  static constexpr bool on = true;
  TapeRec* tape = nullptr;
  double* ys = nullptr;    // [cap_y][n] states at which f was differentiated
  double* yinfo = nullptr; // [cap_y][2] their time and gamma (0: no matrix), or nullptr
  int n = 0;
  int nrec = 0, ny = 0, nsteps = 0;
  int seg_steps = 16, close_rec = 0, close_y = 0;
  double h0 = 0.0;

  __device__ void begin()
  {
    nrec = 0;
    ny = 0;
    nsteps = 0;
  }
  __device__ bool segment_full() const { return nsteps >= seg_steps || nrec >= close_rec || ny >= close_y; }

  __device__ void put(const Team<TEAM>& tm, int op, int q, int i1, int i2, const double* c, int nc)
  {
    if (tm.lane == 0) {
      TapeRec* r = tape + nrec;
      r->op = op;
      r->q = q;
      r->i1 = i1;
      r->i2 = i2;
      for (int j = 0; j < nc; j++) r->c[j] = c[j];
    }
    nrec++;
  }

  __device__ void init(const Team<TEAM>&, double h, const double*) { h0 = h; }
  __device__ void rescale(const Team<TEAM>& tm, int q, double eta)
  {
    const double c[1] = {eta};
    put(tm, TP_RESCALE, q, 0, 0, c, 1);
  }
  __device__ void predict(const Team<TEAM>& tm, int q) { put(tm, TP_PREDICT, q, 0, 0, nullptr, 0); }
  __device__ void correct(const Team<TEAM>& tm, int q, bool save, double tn, double gamma, double rl1, const double* l,
                          const double* z0, const double* acor)
  {
    double* yv = ys + (size_t)ny * n;
    for (int i = tm.lane; i < n; i += TEAM) yv[i] = z0[i] + acor[i];
    double c[9] = {tn, gamma, rl1, 0, 0, 0, 0, 0, 0};
    for (int j = 0; j <= q; j++) c[3 + j] = l[j];
    put(tm, TP_CORRECT, q, save ? 1 : 0, ny, c, 9);
    if (yinfo && tm.lane == 0) {
      yinfo[2 * ny] = tn;
      yinfo[2 * ny + 1] = gamma;
    }
    ny++;
    nsteps++;
  }
  __device__ void saveqmax(const Team<TEAM>& tm) { put(tm, TP_SAVEQMAX, 0, 0, 0, nullptr, 0); }
  __device__ void increase(const Team<TEAM>& tm, int q, int L, int idx, double A1, const double* l)
  {
    double c[6] = {A1, 0, 0, 0, 0, 0};
    for (int j = 2; j <= q; j++) c[j - 1] = l[j];
    put(tm, TP_INCREASE, q, L, idx, c, 6);
  }
  __device__ void decrease(const Team<TEAM>& tm, int q, const double* l)
  {
    double c[6] = {0, 0, 0, 0, 0, 0};
    for (int j = 2; j < q; j++) c[j - 2] = l[j];
    put(tm, TP_DECREASE, q, 0, 0, c, 6);
  }
  __device__ void freset(const Team<TEAM>& tm, double tn, double h, const double* z0)
  {
    double* yv = ys + (size_t)ny * n;
    for (int i = tm.lane; i < n; i += TEAM) yv[i] = z0[i];
    const double c[2] = {tn, h};
    put(tm, TP_FRESET, 1, 0, ny, c, 2);
    if (yinfo && tm.lane == 0) {
      yinfo[2 * ny] = tn;
      yinfo[2 * ny + 1] = 0.0;
    }
    ny++;
  }
  __device__ void output(const Team<TEAM>& tm, int q, double sfac)
  {
    const double c[1] = {sfac};
    put(tm, TP_OUTPUT, q, 0, 0, c, 1);
  }
};

// Team-shared adjoint workspace of one cell.
struct AdjWork {
  double* lam;  // [6][n] adjoint (or tangent) of the Nordsieck history
  double* pend; // [n] adjoint (tangent) of the last correction
  double* mu;   // [n]
  double* v;    // [n + 1] species weights (padding slot nsp)
  double* fE;   // [n] df/dE
  double* fy;   // [n] f
  double* ek;   // [n] mass-specific e_k (h_k)
  double* cvk;  // [n] mass-specific c_v,k (c_p,k)
  double* dcvk; // [n] d c_v,k / dT
  double* ybuf; // [n]
  double* tmp;  // [n]
  double* Jc;   // [n * n] df/dy, column-major Jc[j*n + i] = d f_i / d y_j
  double* AT;   // [n * n] FP64 LU of I - gamma Jc or of its transpose
  double* jxa;  // [5R] per-reaction factors kf, kr, fac, dq/dT, dq/dlnk
  double* gacc; // [3R] parameter gradient of this warp's cells
  int* piv;     // [n]
};

__host__ __device__ inline size_t adj_bytes(int N, int R)
{
  const size_t n = N + 1;
  const size_t d = 6 * n + 10 * n + 1 + 2 * n * n + 6 * (size_t)R + 3 * (size_t)R;
  return ((d * 8 + 4 * n) + 15) & ~size_t(15);
}


__device__ inline void carve_adj(AdjWork& a, char* base, int N, int R)
{
  const int n = N + 1;
  double* p = (double*)base;
  a.lam = p; p += 6 * n;
  a.pend = p; p += n;
  a.mu = p; p += n;
  a.v = p; p += n + 1;
  a.fE = p; p += n;
  a.fy = p; p += n;
  a.ek = p; p += n;
  a.cvk = p; p += n;
  a.dcvk = p; p += n;
  a.ybuf = p; p += n;
  a.tmp = p; p += n;
  a.Jc = p; p += (size_t)n * n;
  a.AT = p; p += (size_t)n * n;
  a.jxa = p; p += 6 * (size_t)R;
  a.gacc = p; p += 3 * (size_t)R;
  a.piv = (int*)p;
}

// Point at which the right-hand side was differentiated.
struct AdjPoint {
  double T, invT, logT, Den, dDen;
};

// f, df/dy and df/dE of the reactor right-hand side at (t, y), plus the
// per-reaction factors for the parameter derivatives (a.jxa).  Uses the
// forward workspace's rate scratch (w.Y, w.sc, w.g, w.qd, w.wdot, w.h1).
template <int TEAM, int PER, typename LT>
__device__ AdjPoint rhs_exact_jacobian(const Team<TEAM>& tm, const DevMech& M, int rtype, double t, const double* y,
                                       double rhoe, double rhoesrc, const double* src, Work<LT>& w, AdjWork& a)
{
  const int N = M.nsp, n = N + 1, R = M.nrxn;
  double acc = 0.0;
  for (int s = tm.lane; s < N; s += TEAM) acc += y[s];
  const double rho = tm.sum(acc);
  const double rinv = 1.0 / rho;
  for (int s = tm.lane; s < N; s += TEAM) w.Y[s] = y[s] * rinv;
  tm.sync();
  const int EH = (rtype == 2);
  double T = y[N];
  t_from_energy(tm, M, EH, (rhoe + rhoesrc * t) * rinv, w.Y, T);
  AdjPoint pt;
  pt.T = T;
  pt.invT = 1.0 / T;
  pt.logT = ppb_log(T);
  const double RT = RU * T;
  double aden = 0.0, adden = 0.0, amix = 0.0;
  for (int s = tm.lane; s < N; s += TEAM) {
    const double im = __ldg(M.imw + s);
    a.ek[s] = (EH ? h_RT(M, s, T, pt.invT) : u_RT(M, s, T, pt.invT)) * (RT * im);
    a.cvk[s] = (EH ? cp_R(M, s, T) : cv_R(M, s, T)) * (RU * im);
    a.dcvk[s] = dcvpRdT(M, s, T) * (RU * im);
    w.sc[s] = (rho * w.Y[s] * im) * 1.0e6;
    w.g[s] = g_RT(M, s, T, pt.invT, pt.logT);
    w.h1[s] = h_RT(M, s, T, pt.invT);
    aden += y[s] * a.cvk[s];
    adden += y[s] * a.dcvk[s];
    amix += w.sc[s];
  }
  if (tm.lane == 0) {
    w.sc[N] = 1.0;
    w.g[N] = 0.0;
    w.h1[N] = 0.0;
  }
  for (int i = tm.lane; i < n * n; i += TEAM) a.Jc[i] = 0.0;
  pt.Den = tm.sum(aden); // rho c_v
  pt.dDen = tm.sum(adden);
  const double mixture = tm.sum(amix);
  tm.sync();
  const double refC = 101325 / 8.31446 * pt.invT;
  const double refCinv = 1.0 / refC;
  // per-reaction factors
  for (int r = tm.lane; r < R; r += TEAM) {
    const RxPack p = load_rx(M, r);
    const RxJac f =
      rx_jac_packed(M, p, T, pt.invT, pt.invT * pt.invT, pt.logT, refC, refCinv, mixture, w.sc, w.g, w.h1);
    w.qd[r] = f.q;
    a.jxa[5 * r + 0] = f.kf;
    a.jxa[5 * r + 1] = f.kr;
    a.jxa[5 * r + 2] = f.fac;
    a.jxa[5 * r + 3] = f.dqdT;
    a.jxa[5 * r + 4] = f.q * f.dlnk;
  }
  tm.sync();
  // wdot and d wdot / dT (held in column N until the assembly)
  for (int s = tm.lane; s < N; s += TEAM) {
    double wd = 0.0, d = 0.0;
    const int g1 = __ldg(M.jg_off + s + 1);
    for (int gi = __ldg(M.jg_off + s); gi < g1; gi++) {
      const int r = __ldg(M.jg_rx + gi);
      const double nu = __ldg(M.jg_c + gi);
      wd += nu * w.qd[r];
      d += nu * a.jxa[5 * r + 3];
    }
    w.wdot[s] = wd;
    a.Jc[N * n + s] = d;
  }
  tm.sync();
  // from here on qd holds dq/d ln k (the parameter derivatives outlive the
  // per-reaction factors, whose storage the Newton-matrix factor may reuse)
  for (int r = tm.lane; r < R; r += TEAM) w.qd[r] = a.jxa[5 * r + 4];
  // third-body / fall-off terms: a rank-one update e_k fac_r nu_r per
  // reaction, all lanes on the same reaction, lane l on columns l, l+TEAM, ..
  {
    const int na = __ldg(M.al_off + 1);
    for (int ai = 0; ai < na; ai++) {
      const int r = __ldg(M.al_rx + ai);
      const RxPack p = load_rx(M, r);
      const double fac = a.jxa[5 * r + 2];
      const double* ed = M.effd + (size_t)p.aslot * N;
#pragma unroll
      for (int qq = 0; qq < PER; qq++) {
        const int k = tm.lane + qq * TEAM;
        if (k >= N) break;
        const double d = __ldg(ed + k) * fac;
        if (d == 0.0) continue;
        double* Jk = a.Jc + k * n;
        #pragma unroll
        for (int j = 0; j < 6; j++) { // static slot index: the record stays in registers
          if (j >= p.njn) break;
          const double nu = (double)p.jnc[j];
          if (nu != 0) Jk[p.jns[j]] += nu * d;
        }
      }
    }
  }
  // phase-space terms: lane l owns columns l, l+TEAM, ... and walks the
  // reactions with its species in their phase space
#pragma unroll
  for (int qq = 0; qq < PER; qq++) {
    const int k = tm.lane + qq * TEAM;
    if (k >= N) break;
    double* Jk = a.Jc + k * n;
    const int e1 = __ldg(M.jm_off + k + 1);
    for (int ei = __ldg(M.jm_off + k); ei < e1; ei++) {
      const int r = __ldg(M.jm_rx + ei);
      const RxPack p = load_rx(M, r);
      const bool inr = slots_has(p.fsp, k);
      const bool inp = (p.rev != 0) && slots_has(p.rsp, k);
      double d = 0.0;
      if (inr) d += a.jxa[5 * r + 0] * slots_dproduct(p.fsp, w.sc, k);
      if (inp) d -= a.jxa[5 * r + 1] * slots_dproduct(p.rsp, w.sc, k);
      #pragma unroll
        for (int j = 0; j < 6; j++) { // static slot index: the record stays in registers
          if (j >= p.njn) break;
        const double nu = (double)p.jnc[j];
        if (nu != 0) Jk[p.jns[j]] += nu * d;
      }
    }
  }
  tm.sync();
  // f
  double ae = 0.0;
  for (int s = tm.lane; s < N; s += TEAM) {
    const double cd = w.wdot[s] * 1.0e-6 * __ldg(M.mw + s) + src[s];
    a.fy[s] = cd;
    ae += cd * a.ek[s];
  }
  const double num = rhoesrc - tm.sum(ae);
  if (tm.lane == 0) a.fy[N] = num / pt.Den;
  tm.sync();
  const double fyN = a.fy[N];
  // species columns: chain rule through T(E, y)
  for (int j = tm.lane; j < N; j += TEAM) {
    const double tau = -a.ek[j] / pt.Den;
    const double imj = __ldg(M.imw + j);
    double dnum = 0.0;
    for (int i = 0; i < N; i++) {
      const double mwi = __ldg(M.mw + i);
      const double v = mwi * imj * a.Jc[j * n + i] + 1.0e-6 * mwi * a.Jc[N * n + i] * tau;
      a.Jc[j * n + i] = v;
      dnum -= v * a.ek[i] + a.fy[i] * a.cvk[i] * tau;
    }
    const double dden = a.cvk[j] + tau * pt.dDen;
    a.Jc[j * n + N] = (dnum - fyN * dden) / pt.Den;
  }
  // df/dE (dT/dE = 1 / (rho c_v))
  double aE = 0.0;
  for (int i = tm.lane; i < N; i += TEAM) {
    const double fe = 1.0e-6 * __ldg(M.mw + i) * a.Jc[N * n + i] / pt.Den;
    a.fE[i] = fe;
    aE += fe * a.ek[i] + a.fy[i] * a.cvk[i] / pt.Den;
  }
  const double dnumE = -tm.sum(aE);
  tm.sync();
  if (tm.lane == 0) a.fE[N] = (dnumE - fyN * pt.dDen / pt.Den) / pt.Den;
  for (int i = tm.lane; i < n; i += TEAM) a.Jc[N * n + i] = 0.0; // f does not depend on the T slot
  tm.sync();
  return pt;
}

// out[j] += scale * sum_i Jc[j*n + i] v[i]   (out += scale Jc^T v)
template <int TEAM>
__device__ void jc_tmul_add(const Team<TEAM>& tm, int n, const double* Jc, const double* v, double scale, double* out)
{
  for (int j = tm.lane; j < n; j += TEAM) {
    double s = 0.0;
    const double* col = Jc + (size_t)j * n;
    for (int i = 0; i < n; i++) s += col[i] * v[i];
    out[j] += scale * s;
  }
  tm.sync();
}

// out[i] = sum_j Jc[j*n + i] x[j]   (out = Jc x)
template <int TEAM>
__device__ void jc_mul(const Team<TEAM>& tm, int n, const double* Jc, const double* x, double* out)
{
  for (int i = tm.lane; i < n; i += TEAM) {
    double s = 0.0;
    for (int j = 0; j < n; j++) s += Jc[(size_t)j * n + i] * x[j];
    out[i] = s;
  }
  tm.sync();
}

// FP64 LU of I - gamma Jc (transpose = false) or of its transpose (out of
// line, as the solve below: the sweeps keep one copy of each).
template <int TEAM>
__device__ __noinline__ int adj_factor(const Team<TEAM>& tm, int n, const double* Jc, double gamma, bool transpose, double* A,
                          int* piv)
{
  for (int i = tm.lane; i < n; i += TEAM) {
    for (int j = 0; j < n; j++) {
      const double jv = transpose ? Jc[(size_t)i * n + j] : Jc[(size_t)j * n + i];
      double v = -gamma * jv;
      if (i == j) v += 1.0;
      A[(size_t)j * n + i] = v;
    }
  }
  tm.sync();
  return lu_factor<TEAM, double>(tm, A, n, piv);
}

template <int TEAM>
__device__ __noinline__ void adj_solve(const Team<TEAM>& tm, const double* A, int n, const int* piv, double* b)
{
  lu_solve<TEAM, double>(tm, A, n, piv, b);
}

// Parameter vector-Jacobian product at the last rhs_exact_jacobian point:
// gacc += scale * (df/dp)^T u, p = (ln A_r, beta_r, Ea_r / R) per reaction.
template <int TEAM>
__device__ void param_vjp(const Team<TEAM>& tm, const DevMech& M, const AdjPoint& pt, AdjWork& a,
                          const double* dqdlnk, const double* u, double scale)
{
  const int N = M.nsp, R = M.nrxn;
  // species weights: d(u . f)/d wdot_k (f_N depends on wdot through the
  // energy sum)
  const double uN = u[N];
  for (int k = tm.lane; k < N; k += TEAM) a.v[k] = 1.0e-6 * __ldg(M.mw + k) * (u[k] - uN * a.ek[k] / pt.Den);
  if (tm.lane == 0) a.v[N] = 0.0;
  tm.sync();
  for (int r = tm.lane; r < R; r += TEAM) {
    const RxPack p = load_rx(M, r);
    double g = 0.0;
#pragma unroll
    for (int j = 0; j < 6; j++)
      if (p.jnc[j]) g += (double)p.jnc[j] * a.v[p.jns[j]];
    g *= scale * dqdlnk[r];
    a.gacc[r] += g;
    a.gacc[R + r] += g * pt.logT;
    a.gacc[2 * R + r] -= g * pt.invT;
  }
  tm.sync();
}

// Parameter Jacobian-vector product: out = (df/dp) dp at the last
// rhs_exact_jacobian point (dp = [d ln A | d beta | d Ea/R]).
template <int TEAM>
__device__ void param_jvp(const Team<TEAM>& tm, const DevMech& M, const AdjPoint& pt, AdjWork& a,
                          const double* dqdlnk, const double* dp, double* out)
{
  const int N = M.nsp, R = M.nrxn;
  // a.jxa is free once the Jacobian is assembled: the rate tangents
  for (int r = tm.lane; r < R; r += TEAM)
    a.jxa[r] = dqdlnk[r] * (__ldg(dp + r) + pt.logT * __ldg(dp + R + r) - pt.invT * __ldg(dp + 2 * R + r));
  tm.sync();
  double ae = 0.0;
  for (int k = tm.lane; k < N; k += TEAM) {
    double sk = 0.0;
    const int g1 = __ldg(M.jg_off + k + 1);
    for (int gi = __ldg(M.jg_off + k); gi < g1; gi++) sk += __ldg(M.jg_c + gi) * a.jxa[__ldg(M.jg_rx + gi)];
    const double ok = 1.0e-6 * __ldg(M.mw + k) * sk;
    out[k] = ok;
    ae += ok * a.ek[k];
  }
  const double oN = -tm.sum(ae) / pt.Den;
  tm.sync();
  if (tm.lane == 0) out[N] = oN;
  tm.sync();
}

// The transposes of the operations that do not touch f (output, saved
// correction, predict, rescale, order change) on the adjoint history lam and
// pending correction adjoint pend; false for TP_CORRECT / TP_FRESET.
template <int TEAM>
__device__ bool rev_linear(const Team<TEAM>& tm, int n, int qmax, const TapeRec& R, AdjWork& a, const double* lam_y)
{
  const int q = R.q;
  switch (R.op) {
  case TP_OUTPUT: {
    // y(tout) = sum_j s^j z_j
    for (int i = tm.lane; i < n; i += TEAM) {
      double pw = 1.0;
      for (int j = 0; j <= q; j++) {
        a.lam[j * n + i] += pw * lam_y[i];
        pw *= R.c[0];
      }
    }
    tm.sync();
    break;
  }
  case TP_SAVEQMAX: {
    for (int i = tm.lane; i < n; i += TEAM) {
      a.pend[i] += a.lam[qmax * n + i];
      a.lam[qmax * n + i] = 0.0;
    }
    tm.sync();
    break;
  }
  case TP_PREDICT: {
    // forward: for k = 1..q, j = q..k: z_{j-1} += z_j
    for (int i = tm.lane; i < n; i += TEAM)
      for (int kk = q; kk >= 1; kk--)
        for (int j = kk; j <= q; j++) a.lam[j * n + i] += a.lam[(j - 1) * n + i];
    tm.sync();
    break;
  }
  case TP_RESCALE: {
    for (int i = tm.lane; i < n; i += TEAM) {
      double f = R.c[0];
      for (int j = 1; j <= q; j++) {
        a.lam[j * n + i] *= f;
        f *= R.c[0];
      }
    }
    tm.sync();
    break;
  }
  case TP_INCREASE: {
    const int L = R.i1, idx = R.i2;
    for (int i = tm.lane; i < n; i += TEAM) {
      double lz = a.lam[L * n + i];
      for (int j = 2; j <= q; j++) lz += R.c[j - 1] * a.lam[j * n + i];
      a.lam[L * n + i] = 0.0;
      a.lam[idx * n + i] += R.c[0] * lz;
    }
    tm.sync();
    break;
  }
  case TP_DECREASE: {
    for (int i = tm.lane; i < n; i += TEAM) {
      double s = 0.0;
      for (int j = 2; j < q; j++) s += R.c[j - 2] * a.lam[j * n + i];
      a.lam[q * n + i] -= s;
    }
    tm.sync();
    break;
  }
  default:
    return false;
  }
  return true;
}

// Sweeps over one tape segment.  lam holds the adjoint (reverse) or the
// tangent (forward) of the Nordsieck history, pend that of the last
// correction.  lamE is the adjoint of E (reverse) and dE the tangent of E
// (forward).
template <int TEAM, int PER, typename LT>
struct AdjSweep {
  const Team<TEAM>& tm;
  const DevMech& M;
  const Options& o;
  Work<LT>& w;
  AdjWork& a;
  CellIn cin;
  int n, qmax;

  __device__ __noinline__ AdjPoint point(double t, const double* yg)
  {
    for (int i = tm.lane; i < n; i += TEAM) a.ybuf[i] = yg[i];
    tm.sync();
    return rhs_exact_jacobian<TEAM, PER, LT>(tm, M, o.reactor_type, t, a.ybuf, cin.rhoe, cin.rhoesrc, w.src, w, a);
  }

  // ---- forward (tangent-linear)
  // out = Jc z + fE dE + fp dp at the last point
  __device__ void tangent_rhs(const AdjPoint& pt, const double* z, double dE, const double* dp, double* out)
  {
    jc_mul(tm, n, a.Jc, z, a.tmp);
    param_jvp(tm, M, pt, a, w.qd, dp, out);
    for (int i = tm.lane; i < n; i += TEAM) out[i] += a.tmp[i] + a.fE[i] * dE;
    tm.sync();
  }

  __device__ __noinline__ void fwd_freset(double t, double h, const double* yg, double dE, const double* dp)
  {
    const AdjPoint pt = point(t, yg);
    tangent_rhs(pt, a.lam, dE, dp, a.mu);
    for (int i = tm.lane; i < n; i += TEAM) a.lam[n + i] = h * a.mu[i];
    tm.sync();
  }

  __device__ __noinline__ int forward(const TapeRec* tape, int nrec, const double* ys, double dE, const double* dp,
                                     double* dy_out)
  {
    for (int k = 0; k < nrec; k++) {
      const TapeRec R = tape[k];
      const int q = R.q;
      switch (R.op) {
      case TP_OUTPUT: {
        for (int i = tm.lane; i < n; i += TEAM) {
          double v = a.lam[q * n + i];
          for (int j = q - 1; j >= 0; j--) v = a.lam[j * n + i] + R.c[0] * v;
          dy_out[i] = v;
        }
        tm.sync();
        break;
      }
      case TP_CORRECT: {
        const double tn = R.c[0], gamma = R.c[1], rl1 = R.c[2];
        const AdjPoint pt = point(tn, ys + (size_t)R.i2 * n);
        tangent_rhs(pt, a.lam, dE, dp, a.mu);
        for (int i = tm.lane; i < n; i += TEAM) a.mu[i] = gamma * a.mu[i] - rl1 * a.lam[n + i];
        tm.sync();
        if (adj_factor(tm, n, a.Jc, gamma, false, a.AT, a.piv)) return ST_ADJ_SINGULAR;
        adj_solve<TEAM>(tm, a.AT, n, a.piv, a.mu);
        for (int i = tm.lane; i < n; i += TEAM) {
          const double d = a.mu[i];
          for (int j = 0; j <= q; j++) a.lam[j * n + i] += R.c[3 + j] * d;
          if (R.i1) a.lam[qmax * n + i] = d;
          a.pend[i] = d;
        }
        tm.sync();
        break;
      }
      case TP_SAVEQMAX: {
        for (int i = tm.lane; i < n; i += TEAM) a.lam[qmax * n + i] = a.pend[i];
        tm.sync();
        break;
      }
      case TP_PREDICT: {
        for (int i = tm.lane; i < n; i += TEAM)
          for (int kk = 1; kk <= q; kk++)
            for (int j = q; j >= kk; j--) a.lam[(j - 1) * n + i] += a.lam[j * n + i];
        tm.sync();
        break;
      }
      case TP_RESCALE: {
        for (int i = tm.lane; i < n; i += TEAM) {
          double f = R.c[0];
          for (int j = 1; j <= q; j++) {
            a.lam[j * n + i] *= f;
            f *= R.c[0];
          }
        }
        tm.sync();
        break;
      }
      case TP_INCREASE: {
        const int L = R.i1, idx = R.i2;
        for (int i = tm.lane; i < n; i += TEAM) {
          const double zL = R.c[0] * a.lam[idx * n + i];
          a.lam[L * n + i] = zL;
          for (int j = 2; j <= q; j++) a.lam[j * n + i] += R.c[j - 1] * zL;
        }
        tm.sync();
        break;
      }
      case TP_DECREASE: {
        for (int i = tm.lane; i < n; i += TEAM)
          for (int j = 2; j < q; j++) a.lam[j * n + i] -= R.c[j - 2] * a.lam[q * n + i];
        tm.sync();
        break;
      }
      case TP_FRESET: {
        fwd_freset(R.c[0], R.c[1], ys + (size_t)R.i2 * n, dE, dp);
        break;
      }
      default:
        break;
      }
    }
    return ST_OK;
  }
};

// ---------------------------------------------------------------- batched
// The batched reverse sweep evaluates, for every differentiated point of a
// segment of every cell at once, the exact Jacobian, df/dE, the rate
// derivatives and (for corrections) the FP64 factor of (I - gamma Jc)^T --
// none of which depends on the adjoint state -- and stores them per point;
// the sequential sweep then needs only solves and products.
struct ItemLayout {
  size_t at, fe, ek, dq, sc, piv, stride; // offsets in doubles
  __host__ __device__ ItemLayout(int N, int R)
  {
    const size_t n = N + 1;
    at = n * n;
    fe = 2 * n * n;
    ek = fe + n;
    dq = ek + n;
    sc = dq + (size_t)R;
    piv = sc + 4;
    stride = piv + (n + 1) / 2;
    stride = (stride + 1) & ~size_t(1);
  }
};

// shared memory of one item evaluation
__host__ __device__ inline size_t item_bytes(int N, int R)
{
  const size_t n = N + 1;
  return ((8 * (13 * n + 6 * (size_t)R + 2 * n * n) + 4 * n) + 15) & ~size_t(15);
}

template <int TEAM, int PER>
__device__ void eval_item(const Team<TEAM>& tm, const DevMech& M, int rtype, double t, double gamma, const double* yg,
                          double rhoe, double rhoesrc, const double* srcg, char* smem, double* item,
                          const ItemLayout& IL)
{
  const int N = M.nsp, n = N + 1, R = M.nrxn;
  double* p = (double*)smem;
  Work<double> w{};
  AdjWork a{};
  w.Y = p; p += n;
  w.sc = p; p += n;
  w.g = p; p += n;
  w.h1 = p; p += n;
  w.wdot = p; p += n;
  w.src = p; p += n;
  w.qd = p; p += R;
  a.ek = p; p += n;
  a.cvk = p; p += n;
  a.dcvk = p; p += n;
  a.fy = p; p += n;
  a.fE = p; p += n;
  a.ybuf = p; p += n;
  a.Jc = p; p += (size_t)n * n;
  a.AT = p; p += (size_t)n * n;
  a.jxa = p; p += 5 * (size_t)R;
  a.piv = (int*)p;
  for (int i = tm.lane; i < n; i += TEAM) {
    a.ybuf[i] = yg[i];
    w.src[i] = (i < N && srcg) ? srcg[i] : 0.0;
  }
  tm.sync();
  const AdjPoint pt = rhs_exact_jacobian<TEAM, PER, double>(tm, M, rtype, t, a.ybuf, rhoe, rhoesrc, w.src, w, a);
  int sing = 0;
  if (gamma != 0.0) sing = adj_factor(tm, n, a.Jc, gamma, true, a.AT, a.piv);
  for (int i = tm.lane; i < n * n; i += TEAM) item[i] = a.Jc[i];
  if (gamma != 0.0)
    for (int i = tm.lane; i < n * n; i += TEAM) item[IL.at + i] = a.AT[i];
  for (int i = tm.lane; i < n; i += TEAM) {
    item[IL.fe + i] = a.fE[i];
    item[IL.ek + i] = a.ek[i];
  }
  for (int r = tm.lane; r < R; r += TEAM) item[IL.dq + r] = w.qd[r];
  int* ip = reinterpret_cast<int*>(item + IL.piv);
  for (int i = tm.lane; i < n; i += TEAM) ip[i] = (sing && i == 0) ? -1 : a.piv[i];
  if (tm.lane == 0) {
    item[IL.sc + 0] = pt.Den;
    item[IL.sc + 1] = pt.logT;
    item[IL.sc + 2] = pt.invT;
    item[IL.sc + 3] = pt.T;
  }
}

// z_1 = h f(t, z_0) at a stored point: lam_0 += h Jc^T lam_1, lamE += h fE .
// lam_1, gradient, lam_1 = 0
template <int TEAM>
__device__ void rev_item_freset(const Team<TEAM>& tm, const DevMech& M, int n, AdjWork& a, const double* it,
                                const ItemLayout& IL, double h, double& lamE)
{
  double* l1 = a.lam + n;
  for (int i = tm.lane; i < n; i += TEAM) a.mu[i] = l1[i];
  tm.sync();
  for (int i = tm.lane; i < n; i += TEAM) l1[i] = 0.0;
  jc_tmul_add(tm, n, it, a.mu, h, a.lam);
  double s = 0.0;
  for (int i = tm.lane; i < n; i += TEAM) s += it[IL.fe + i] * a.mu[i];
  lamE += h * tm.sum(s);
  AdjPoint pt;
  pt.Den = it[IL.sc + 0];
  pt.logT = it[IL.sc + 1];
  pt.invT = it[IL.sc + 2];
  pt.T = it[IL.sc + 3];
  pt.dDen = 0.0;
  AdjWork av = a;
  av.ek = const_cast<double*>(it + IL.ek);
  param_vjp(tm, M, pt, av, it + IL.dq, a.mu, h);
}

// Reverse sweep of one tape segment with the segment's points evaluated
// beforehand (items: point k at items + k * IL.stride).  a.AT / a.piv are
// shared-memory copies of the factors.
template <int TEAM>
__device__ int sweep_items(const Team<TEAM>& tm, const DevMech& M, int n, int qmax, AdjWork& a, const TapeRec* tape,
                           int nrec, const double* items, const ItemLayout& IL, const double* lam_y, double& lamE)
{
  for (int k = nrec - 1; k >= 0; k--) {
    const TapeRec R = tape[k];
    if (rev_linear(tm, n, qmax, R, a, lam_y)) continue;
    const double* it = items + (size_t)R.i2 * IL.stride;
    if (R.op == TP_FRESET) {
      rev_item_freset(tm, M, n, a, it, IL, R.c[1], lamE);
      continue;
    }
    if (R.op != TP_CORRECT) continue;
    const int q = R.q;
    const double gamma = R.c[1], rl1 = R.c[2];
    for (int i = tm.lane; i < n; i += TEAM) {
      double la = a.pend[i];
      for (int j = 0; j <= q; j++) la += R.c[3 + j] * a.lam[j * n + i];
      if (R.i1) {
        la += a.lam[qmax * n + i];
        a.lam[qmax * n + i] = 0.0;
      }
      a.mu[i] = la;
      a.pend[i] = 0.0;
    }
    const int* ip = reinterpret_cast<const int*>(it + IL.piv);
    if (ip[0] < 0) return ST_ADJ_SINGULAR;
    for (int i = tm.lane; i < n * n; i += TEAM) a.AT[i] = it[IL.at + i];
    for (int i = tm.lane; i < n; i += TEAM) a.piv[i] = ip[i];
    tm.sync();
    adj_solve<TEAM>(tm, a.AT, n, a.piv, a.mu);
    jc_tmul_add(tm, n, it, a.mu, gamma, a.lam);
    double s = 0.0;
    for (int i = tm.lane; i < n; i += TEAM) {
      a.lam[n + i] -= rl1 * a.mu[i];
      s += it[IL.fe + i] * a.mu[i];
    }
    lamE += gamma * tm.sum(s);
    tm.sync();
    AdjPoint pt;
    pt.Den = it[IL.sc + 0];
    pt.logT = it[IL.sc + 1];
    pt.invT = it[IL.sc + 2];
    pt.T = it[IL.sc + 3];
    pt.dDen = 0.0;
    AdjWork av = a;
    av.ek = const_cast<double*>(it + IL.ek);
    param_vjp(tm, M, pt, av, it + IL.dq, a.mu, gamma);
  }
  return ST_OK;
}

} // namespace ppb
