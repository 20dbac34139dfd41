// ORACLE / TEST INFRASTRUCTURE ONLY.
//
// Compiles the reference's own mixture-averaged transport
// (Source/Transport/Simple.H: SimpleTransport::transport, BinaryDiff,
// comp_pure_bulk) with one mechanism's CEPTR transport fits
// (Mechanisms/<mech>/mechanism.H egtranset*) on the host, against the AMReX
// stub in oracle/amrex_stub plus the few AMReX types Simple.H names, and
// exposes one point evaluation through an extern "C" symbol.  The parameter
// struct is filled exactly as the reference's
// InitParm<TransParm<EOSType, SimpleTransport>>::host_initialize does
// (Source/Transport/TransportParams.H:228-258).  The reference's
// TransportParams.H itself is not included (it pulls in ParmParse and the
// whole EOS layer); its TransParm layout is declared here with the field
// names Simple.H reads.  Built per mechanism by oracle/build_ref.sh into
// oracle/_ref/libreftr_<mech>.so; nothing in the product library links it.

#include <array>
#include <cstring>

#include "mechanism.H"

// ---- the AMReX names Simple.H uses (host-only stand-ins)
namespace amrex {
template <class T, int N>
struct GpuArray {
  T arr[N];
  T& operator[](int i) { return arr[i]; }
  const T& operator[](int i) const { return arr[i]; }
  T* data() { return arr; }
};
struct Dim3 {
  int x, y, z;
};
struct Box {
  Dim3 lo, hi;
};
inline Dim3 lbound(const Box& b) { return b.lo; }
inline Dim3 ubound(const Box& b) { return b.hi; }
template <class T>
struct Array4 {
  T* p;
  long jstride, kstride, nstride;
  T& operator()(int i, int j, int k, int n = 0) const { return p[i + j * jstride + k * kstride + n * nstride]; }
};
} // namespace amrex

// ---- the EOS and transport-parameter declarations Simple.H expects
#define TRANSPORT_PARAMS_H
#include "PhysicsConstants.H"
namespace pele::physics {
namespace eos {
struct Fuego {};
struct SRK {};
} // namespace eos
using EosType = eos::Fuego;
namespace transport {
struct SimpleTransport;
template <typename EOSType, typename TransportType>
struct TransParm {
};
template <>
struct TransParm<eos::Fuego, SimpleTransport> {
  amrex::GpuArray<amrex::Real, NUM_SPECIES> wt, iwt, eps, sig, dip, pol, zrot;
  amrex::GpuArray<amrex::Real, NUM_SPECIES * NUM_FIT> fitmu, fitlam;
  amrex::GpuArray<amrex::Real, NUM_SPECIES * NUM_SPECIES * NUM_FIT> fitdbin;
  bool use_soret = false;
  int numLite = 3;
  amrex::GpuArray<int, NUM_SPECIES> liteSpec; // reference: 3 entries; NLITE <= N here
  amrex::GpuArray<amrex::Real, NUM_SPECIES * NUM_FIT * NUM_SPECIES> fittdrat;
  amrex::GpuArray<int, NUM_SPECIES> nlin;
};
// only compiled (Simple.H's SRK specialisations are non-template), never run
template <>
struct TransParm<eos::SRK, SimpleTransport> {
  const amrex::Real *wt, *iwt, *eps, *dip, *fitdbin, *Afac, *Bfac, *sqrtT2ij, *sqrtEpsilonij, *sqrtMWij,
    *sqrtKappaij, *Upsilonijk, *omega;
};
} // namespace transport
} // namespace pele::physics

#include "Transport/Simple.H"

using pele::physics::transport::SimpleTransport;
using TP = pele::physics::transport::TransParm<pele::physics::eos::Fuego, SimpleTransport>;

#define REF_API extern "C" __attribute__((visibility("default")))

static TP* parm(int use_soret)
{
  static TP p[2];
  static bool init[2] = {false, false};
  TP* t = &p[use_soret ? 1 : 0];
  if (!init[use_soret ? 1 : 0]) {
    std::memset(t, 0, sizeof(TP));
    egtransetWT(t->wt.data());
    egtransetEPS(t->eps.data());
    egtransetSIG(t->sig.data());
    egtransetDIP(t->dip.data());
    egtransetPOL(t->pol.data());
    egtransetZROT(t->zrot.data());
    egtransetNLIN(t->nlin.data());
    egtransetCOFETA(t->fitmu.data());
    egtransetCOFLAM(t->fitlam.data());
    egtransetCOFD(t->fitdbin.data());
    t->numLite = 3;
    t->use_soret = use_soret != 0;
    if (use_soret) {
      egtransetNLITE(&t->numLite);
      egtransetKTDIF(t->liteSpec.data());
      egtransetCOFTD(t->fittdrat.data());
    }
    for (int i = 0; i < NUM_SPECIES; ++i) t->iwt[i] = 1.0 / t->wt[i];
    init[use_soret ? 1 : 0] = true;
  }
  return t;
}

REF_API int reftr_nsp() { return NUM_SPECIES; }

// SimpleTransport::transport at one point: flags bit 0 xi, 1 mu, 2 lam,
// 3 Ddiag, 4 chi (chi also selects the Soret parameters).  Y is copied (the
// reference perturbs it in place by the trace amount).
REF_API void reftr_transport(int flags, double T, double rho, const double* Y, double* D, double* chi,
                             double* mu, double* xi, double* lam)
{
  const bool get_xi = flags & 1, get_mu = flags & 2, get_lam = flags & 4, get_D = flags & 8,
             get_chi = flags & 16;
  TP* t = parm(get_chi ? 1 : 0);
  double y[NUM_SPECIES], d[NUM_SPECIES] = {0.0}, c[NUM_SPECIES] = {0.0};
  std::memcpy(y, Y, sizeof(y));
  double m = 0.0, x = 0.0, l = 0.0;
  SimpleTransport::transport(get_xi, get_mu, get_lam, get_D, get_chi, T, rho, y, d, c, m, x, l, t);
  if (D) std::memcpy(D, d, sizeof(d));
  if (chi) std::memcpy(chi, c, sizeof(c));
  if (mu) *mu = m;
  if (xi) *xi = x;
  if (lam) *lam = l;
}
