// ORACLE / TEST INFRASTRUCTURE ONLY.
//
// Compiles the reference's own CEPTR-generated mechanism kernels
// (Mechanisms/<mech>/mechanism.H) on the host, against the two-file AMReX stub
// in oracle/amrex_stub, and exposes them through plain extern "C" symbols so
// that the tests, the golden-vector script and the CPU baseline can call the
// reference arithmetic directly.  Nothing in the product library links this.
//
// The reactor-level helpers at the bottom restate, around those compiled
// kernels, the composition the reference performs:
//   - ref_reactor_rhs   : Source/Reactions/ReactorUtils.H:358-415 (fKernelSpec)
//                         with the Fuego wrappers of Source/Eos/Fuego.H:31-39
//                         (RY2RRinvY), :163-192 (REY2T/RHY2T), :234-247
//                         (RTY2WDOT), :288-295/:392-399 (RTY2Ei/RTY2Hi),
//                         :72-98 (RTY2Cp/RTY2Cv)
//   - ref_reactor_jac   : Source/Reactions/ReactorCvodeJacobian.cpp:86-152
//                         (CPU dense cJac: RTY2JAC then mw/imw scaling)
// Built per mechanism by oracle/build_ref.sh into oracle/_ref/libref_<mech>.so.

#include <cstring>
#include "mechanism.H"

#define REF_API extern "C" __attribute__((visibility("default")))

REF_API int ref_nsp() { return NUM_SPECIES; }
REF_API int ref_nrxn() { return NUM_REACTIONS; }
REF_API void ref_mw(double* out) { get_mw(out); }
REF_API void ref_imw(double* out) { get_imw(out); }

// mechanism.H: productionRate (SI, mol/m^3/s from mol/m^3)
REF_API void ref_productionRate(double* wdot, const double* sc, double T)
{
  productionRate(wdot, sc, T);
}
#ifdef NUM_QSSA_GAS_SPECIES
// QSS mechanisms: the QSS concentrations productionRate solves first
// (SI; the first lines of productionRate in a QSS mechanism.H)
REF_API void ref_sc_qss(double* out, const double* sc_in, double T)
{
  const amrex::Real invT = 1.0 / T;
  const amrex::Real logT = log(T);
  amrex::Real sc[NUM_SPECIES];
  std::memcpy(sc, sc_in, sizeof(sc));
  amrex::Real g_RT[NUM_SPECIES];
  gibbs(g_RT, T);
  amrex::Real g_RT_qss[64], sc_qss[64];
  amrex::Real kf_qss[2048], qf_qss[2048], qr_qss[2048];
  gibbs_qss(g_RT_qss, T);
  comp_k_f_qss(T, invT, logT, kf_qss);
  comp_qss_coeff(kf_qss, qf_qss, qr_qss, sc, T, g_RT, g_RT_qss);
  comp_sc_qss(sc_qss, qf_qss, qr_qss);
  for (int q = 0; q < 64; q++) out[q] = sc_qss[q];
}
#endif

// mechanism.H: CKWC (CGS wrapper, mol/cm^3 in, mol/cm^3/s out)
REF_API void ref_CKWC(double T, const double* C, double* wdot)
{
  double c[NUM_SPECIES];
  std::memcpy(c, C, sizeof(c));
  CKWC(T, c, wdot);
}
// mechanism.H: aJacobian (SI concentrations)
REF_API void ref_aJacobian(double* J, const double* sc, double T, int consP)
{
  // a copy: the QSS mechanisms' aJacobian takes a non-const sc
  double c[NUM_SPECIES];
  std::memcpy(c, sc, sizeof(c));
  aJacobian(J, c, T, consP);
}
// mechanism.H: DWDOT (CGS concentrations, rescaled T row/column)
REF_API void ref_DWDOT(double* J, const double* sc, double T, int consP)
{
  DWDOT(J, sc, &T, &consP);
}
REF_API void ref_gibbs(double* g, double T) { gibbs(g, T); }
REF_API void ref_speciesInternalEnergy(double* e, double T)
{
  speciesInternalEnergy(e, T);
}
REF_API void ref_speciesEnthalpy(double* h, double T) { speciesEnthalpy(h, T); }
REF_API void ref_cv_R(double* c, double T) { cv_R(c, T); }
REF_API void ref_cp_R(double* c, double T) { cp_R(c, T); }
REF_API void ref_dcvpRdT(double* c, double T) { dcvpRdT(c, T); }
REF_API double ref_CKUBMS(double T, const double* y)
{
  double r;
  CKUBMS(T, y, r);
  return r;
}
REF_API double ref_CKHBMS(double T, const double* y)
{
  double r;
  CKHBMS(T, y, r);
  return r;
}
REF_API double ref_CKCVBS(double T, const double* y)
{
  double r;
  CKCVBS(T, y, r);
  return r;
}
REF_API double ref_CKCPBS(double T, const double* y)
{
  double r;
  CKCPBS(T, y, r);
  return r;
}
REF_API void ref_CKUMS(double T, double* u) { CKUMS(T, u); }
REF_API void ref_CKHMS(double T, double* h) { CKHMS(T, h); }
REF_API double ref_CKRHOY(double P, double T, const double* y)
{
  double r;
  CKRHOY(P, T, y, r);
  return r;
}
// mechanism.H: GET_T_GIVEN_EY / GET_T_GIVEN_HY (T in: initial guess; out: T)
REF_API int ref_GET_T_GIVEN_EY(double e, const double* y, double* T)
{
  int ierr = 0;
  GET_T_GIVEN_EY(e, y, *T, ierr);
  return ierr;
}
REF_API int ref_GET_T_GIVEN_HY(double h, const double* y, double* T)
{
  int ierr = 0;
  GET_T_GIVEN_HY(h, y, *T, ierr);
  return ierr;
}

// Reactor right-hand side for one cell in YCOrder: y = [rhoY_0..rhoY_{N-1}, T].
// t_rel is the time since the start of the react() call; the energy seen by
// the cell is rhoe_init + rhoesrc * t_rel.  Returns the T found by the
// temperature Newton (the value the Jacobian/flatten logic would use).
REF_API double ref_reactor_rhs(
  int reactor_type,
  double t_rel,
  const double* y,
  double* ydot,
  double rhoe_init,
  double rhoesrc,
  const double* rYsrc)
{
  double rho = 0.0;
  for (int n = 0; n < NUM_SPECIES; n++) {
    rho += y[n];
  }
  const double rinv = 1.0 / rho;
  double Y[NUM_SPECIES];
  for (int n = 0; n < NUM_SPECIES; n++) {
    Y[n] = y[n] * rinv;
  }
  const double nrg = (rhoe_init + rhoesrc * t_rel) * rinv;
  double T = y[NUM_SPECIES];
  double ei[NUM_SPECIES];
  double cv = 1.0;
  int ierr = 0;
  if (reactor_type == 1) {
    GET_T_GIVEN_EY(nrg, Y, T, ierr);
    CKUMS(T, ei);
    CKCVBS(T, Y, cv);
  } else {
    GET_T_GIVEN_HY(nrg, Y, T, ierr);
    CKHMS(T, ei);
    CKCPBS(T, Y, cv);
  }
  double C[NUM_SPECIES], wdot[NUM_SPECIES];
  CKYTCR(rho, T, Y, C);
  CKWC(T, C, wdot);
  double esrc = rhoesrc;
  for (int n = 0; n < NUM_SPECIES; n++) {
    const double cd = wdot[n] * mw(n) + rYsrc[n];
    ydot[n] = cd;
    esrc -= cd * ei[n];
  }
  ydot[NUM_SPECIES] = esrc * (rinv / cv);
  return T;
}

// Reactor Jacobian for one cell, dense column-major n x n (n = N+1), the
// layout SUNDenseMatrix uses: J[col*n + row].
REF_API void ref_reactor_jac(int reactor_type, const double* y, double* J)
{
  const int n = NUM_SPECIES + 1;
  double rho = 0.0;
  for (int i = 0; i < NUM_SPECIES; i++) {
    rho = rho + y[i];
  }
  const double temp = y[NUM_SPECIES];
  double Y[NUM_SPECIES];
  for (int i = 0; i < NUM_SPECIES; i++) {
    Y[i] = y[i] / rho;
  }
  double Jm[(NUM_SPECIES + 1) * (NUM_SPECIES + 1)];
  for (double& v : Jm) {
    v = 0.0;
  }
  const int consP = (reactor_type == 2) ? 1 : 0;
  double C[NUM_SPECIES];
  CKYTCR(rho, temp, Y, C);
  DWDOT(Jm, C, &temp, &consP);
  for (int i = 0; i < NUM_SPECIES; i++) {
    double* col = J + i * n;
    for (int k = 0; k < NUM_SPECIES; k++) {
      col[k] = Jm[i * n + k] * mw(k) * imw(i);
    }
    col[NUM_SPECIES] = Jm[i * n + NUM_SPECIES] * imw(i);
  }
  double* col = J + NUM_SPECIES * n;
  for (int i = 0; i < NUM_SPECIES; i++) {
    col[i] = Jm[NUM_SPECIES * n + i] * mw(i);
  }
  // The reference never writes the (T, T) entry; the matrix was zeroed by
  // SUNMatZero before the callback, so it stays 0.
  col[NUM_SPECIES] = 0.0;
}
