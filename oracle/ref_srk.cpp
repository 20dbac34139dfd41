// ORACLE / TEST INFRASTRUCTURE ONLY.
//
// Compiles the reference's own Soave-Redlich-Kwong equation of state
// (Source/Eos/SRK.H, struct SRK) with one mechanism's generated header on
// the host, against the AMReX stub in oracle/amrex_stub, and exposes the
// functions the e-reactor uses through extern "C" symbols: REY2T, RTY2E,
// RTY2Ei, RTY2Cv, RTY2C (activities) and RTY2WDOT, plus the reactor
// right-hand side of Source/Reactions/ReactorUtils.H:358-415 (fKernelSpec,
// reactor type 1) composed with them.  Built per mechanism by
// oracle/build_ref.sh into oracle/_ref/librefsrk_<mech>.so; nothing in the
// product library links it.

#include <cstring>

#include "mechanism.H"
#include "Eos/SRK.H"

using pele::physics::eos::SRK;

#define REF_API extern "C" __attribute__((visibility("default")))

REF_API int refsrk_nsp() { return NUM_SPECIES; }

REF_API void refsrk_rey2t(double R, double E, const double* Y, double* T)
{
  SRK eos;
  double y[NUM_SPECIES];
  std::memcpy(y, Y, sizeof(y));
  eos.REY2T(R, E, y, *T);
}

REF_API double refsrk_rty2e(double R, double T, const double* Y)
{
  SRK eos;
  double y[NUM_SPECIES], E = 0.0;
  std::memcpy(y, Y, sizeof(y));
  eos.RTY2E(R, T, y, E);
  return E;
}

REF_API void refsrk_rty2ei(double R, double T, const double* Y, double* Ei)
{
  SRK eos;
  double y[NUM_SPECIES];
  std::memcpy(y, Y, sizeof(y));
  eos.RTY2Ei(R, T, y, Ei);
}

REF_API double refsrk_rty2cv(double R, double T, const double* Y)
{
  SRK eos;
  double y[NUM_SPECIES], cv = 0.0;
  std::memcpy(y, Y, sizeof(y));
  eos.RTY2Cv(R, T, y, cv);
  return cv;
}

REF_API void refsrk_rty2c(double R, double T, const double* Y, double* C)
{
  SRK eos;
  double y[NUM_SPECIES];
  std::memcpy(y, Y, sizeof(y));
  eos.RTY2C(R, T, y, C);
}

REF_API void refsrk_rty2wdot(double R, double T, const double* Y, double* wdot)
{
  SRK eos;
  double y[NUM_SPECIES];
  std::memcpy(y, Y, sizeof(y));
  eos.RTY2WDOT(R, T, y, wdot);
}

// fKernelSpec (ReactorUtils.H:358-415), reactor type 1, with the SRK EOS:
// y = [rhoY_k, T] (T the Newton start), ydot out; returns the T used.
REF_API double refsrk_reactor_rhs(double t_rel, const double* y, double* ydot, double rhoe_init, double rhoesrc,
                                  const double* rYsrc)
{
  SRK eos;
  double rho = 0.0, rinv, Y[NUM_SPECIES], ei[NUM_SPECIES], cdots[NUM_SPECIES];
  double rY[NUM_SPECIES];
  std::memcpy(rY, y, sizeof(rY));
  eos.RY2RRinvY(rY, rho, rinv, Y);
  const double nrg = (rhoe_init + rhoesrc * t_rel) * rinv;
  double T = y[NUM_SPECIES], cv = 1.0;
  eos.REY2T(rho, nrg, Y, T);
  eos.RTY2Ei(rho, T, Y, ei);
  eos.RTY2Cv(rho, T, Y, cv);
  eos.RTY2WDOT(rho, T, Y, cdots);
  double es = rhoesrc;
  for (int n = 0; n < NUM_SPECIES; n++) {
    const double c = cdots[n] + rYsrc[n];
    ydot[n] = c;
    es -= c * ei[n];
  }
  ydot[NUM_SPECIES] = es * (rinv / cv);
  return T;
}
