// C++ mirror of the reference's reactor interface over the engine's C ABI.
//
// pele::physics::reactions::ReactorBase (Source/Reactions/ReactorBase.H:13-106)
// without AMReX: ReactorB200 / ReactorB200RK implement every member the
// reference's interface declares -- init, close, print_final_stats, the box
// react over Array4-style views, the flat react, flatten, unflatten and the
// non-virtual set_typ_vals_ode -- with the same argument lists and meaning,
// and report errors through return codes instead of amrex::Abort.  Inside the
// reference tree the same class derives from ReactorBase with amrex::Array4
// in place of Array4View (the binding is spelled out in INTEGRATION.md).
//
// Threading: one object may be shared by host threads that call react
// concurrently, as the reference's ReactEval driver does with OpenMP over
// tiles (Testing/Exec/ReactEval/main.cpp:478-520).  The engine keeps device
// scratch, cost order, captured graph and per-cell flags per calling thread.
// print_final_stats reports the calling thread's last call.
//
// Header-only; link pelephysics_b200/libppb200.so.
#pragma once

#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/pelephysics_b200.h"

namespace ppb_cpp {

// amrex::Array4<T>-compatible view: (i,j,k,n) -> p[(i-begin.x) +
// (j-begin.y)*jstride + (k-begin.z)*kstride + n*nstride], bounds [begin, end).
template <class T>
struct Array4View {
  T* p = nullptr;
  long jstride = 0, kstride = 0, nstride = 0;
  int begin[3] = {0, 0, 0};
  int end[3] = {1, 1, 1};
  int ncomp = 1;
};

struct Box {
  int lo[3], hi[3]; // inclusive, as amrex::Box smallEnd / bigEnd
  int numPts() const { return (hi[0] - lo[0] + 1) * (hi[1] - lo[1] + 1) * (hi[2] - lo[2] + 1); }
};

class ReactorB200
{
public:
  static std::string identifier() { return "ReactorB200"; }

  explicit ReactorB200(const std::string& mechanism, const char* integrator = "ReactorCvode")
  {
    if (ppb_create(mechanism.c_str(), integrator, &m_r) != 0) throw std::runtime_error(ppb_last_error());
    ppb_default_options(&m_opt);
  }
  virtual ~ReactorB200() { ppb_destroy(m_r); }
  ReactorB200(const ReactorB200&) = delete;
  ReactorB200& operator=(const ReactorB200&) = delete;

  // ParmParse-style options (ode.* / cvode.* keys of ReactorCvode::init)
  ppb_options& options() { return m_opt; }

  // ReactorBase::init(reactor_type, ncells) (ReactorBase.H:19)
  virtual int init(int reactor_type, int ncells)
  {
    m_reactor_type = reactor_type;
    return ppb_init(m_r, reactor_type, ncells, &m_opt);
  }

  // ReactorBase::close (ReactorBase.H:21)
  virtual void close() { ppb_close(m_r); }

  // ReactorBase::print_final_stats(void* sundials_mem) (ReactorBase.H:23):
  // the CVODE counters ReactorCvode::print_final_stats prints
  // (ReactorCvode.cpp:1838-1901), summed over the cells of the calling
  // thread's last call (there is no SUNDIALS memory; the argument is unused).
  virtual void print_final_stats(void* /*sundials_mem*/) { print_final_stats(ppb_last_ncells(m_r), stdout); }

  void print_final_stats(int ncells, FILE* out)
  {
    std::vector<int> st((size_t)ncells * 7);
    if (ncells <= 0 || ppb_get_cell_stats(m_r, st.data(), ncells) != 0) return;
    long s[7] = {0, 0, 0, 0, 0, 0, 0};
    for (int c = 0; c < ncells; c++)
      for (int q = 0; q < 7; q++) s[q] += st[(size_t)c * 7 + q];
    std::fprintf(out,
                 "-- Final stats: nSteps %ld nRHSeval %ld nJeval %ld nLinSetups %ld nNonlinIters %ld "
                 "nErrtf %ld nConvfail %ld\n",
                 s[0], s[1], s[2], s[3], s[4], s[5], s[6]);
  }

  // ReactorBase::set_typ_vals_ode (ReactorBase.H:82; N+1 typical values)
  int set_typ_vals_ode(const std::vector<double>& v) { return ppb_set_typ_vals(m_r, v.data(), (int)v.size()); }

  // ReactorBase::react(Box, Array4...) (ReactorBase.H:25-40) on device views
  virtual int react(const Box& box, Array4View<double> const& rY, Array4View<double> const& rYsrc,
                    Array4View<double> const& T, Array4View<double> const& rEner,
                    Array4View<double> const& rEner_src, Array4View<double> const& FC,
                    Array4View<int> const& mask, double& dt_react, double& time, void* stream = nullptr)
  {
    return ppb_react_box(m_r, box.lo, box.hi, view(rY), view(rYsrc), view(T), view(rEner), view(rEner_src),
                         view(FC), viewi(mask), &dt_react, &time, stream);
  }

  // ReactorBase::react(Real* ...) (ReactorBase.H:42-54) on flat YCOrder host
  // arrays; returns the cost as the reference does (RHS evaluations /
  // average RK steps), or 1 on an integration failure, or a negative
  // PPB_E_* code.
  virtual int react(double* rY, double* rYsrc, double* rX, double* rX_src, double& dt_react, double& time,
                    int ncells, void* stream = nullptr)
  {
    long cost = 0;
    const int rc = ppb_react_flat(m_r, rY, rYsrc, rX, rX_src, &dt_react, &time, ncells, stream, &cost);
    if (rc != 0) return rc;
    return (int)cost;
  }

  // ReactorBase::flatten (ReactorBase.H:56-67) on device views: the box into
  // component-major device vectors (the reference GPU build's CYOrder).
  virtual void flatten(const Box& box, const int ncells, Array4View<const double> const& rhoY,
                       Array4View<const double> const& frcExt, Array4View<const double> const& temperature,
                       Array4View<const double> const& rhoE, Array4View<const double> const& frcEExt,
                       double* y_vect, double* src_vect, double* vect_energy, double* src_vect_energy)
  {
    if (ncells != box.numPts()) {
      m_status = PPB_E_ARG;
      return;
    }
    m_status = ppb_flatten(m_r, box.lo, box.hi, view(rhoY), view(frcExt), view(temperature), view(rhoE),
                           view(frcEExt), y_vect, src_vect, vect_energy, src_vect_energy, nullptr);
  }

  // ReactorBase::unflatten (ReactorBase.H:69-80) on device views and vectors
  // (FCunt: per-cell costs, device memory).
  virtual void unflatten(const Box& box, const int ncells, Array4View<double> const& rhoY,
                         Array4View<double> const& temperature, Array4View<double> const& rhoE,
                         Array4View<double> const& frcEExt, Array4View<double> const& FC_in, double* y_vect,
                         double* vect_energy, long int* FCunt, double dt)
  {
    if (ncells != box.numPts()) {
      m_status = PPB_E_ARG;
      return;
    }
    m_status = ppb_unflatten(m_r, box.lo, box.hi, view(rhoY), view(temperature), view(rhoE), view(frcEExt),
                             view(FC_in), y_vect, vect_energy, FCunt, dt, nullptr);
  }

  // Status of the last flatten / unflatten (they return void, as in the
  // reference; the reference aborts on errors instead).
  int last_status() const { return m_status; }
  const char* last_error() const { return ppb_last_error(); }
  ppb_reactor* handle() { return m_r; }

protected:
  template <class T>
  static ppb_array4 view(Array4View<T> const& a)
  {
    ppb_array4 v;
    v.p = const_cast<double*>(a.p);
    v.jstride = a.jstride;
    v.kstride = a.kstride;
    v.nstride = a.nstride;
    for (int d = 0; d < 3; d++) {
      v.lo[d] = a.begin[d];
      v.hi[d] = a.end[d] - 1;
    }
    v.ncomp = a.ncomp;
    return v;
  }
  static ppb_array4i viewi(Array4View<int> const& a)
  {
    ppb_array4i v;
    v.p = a.p;
    v.jstride = a.jstride;
    v.kstride = a.kstride;
    v.nstride = a.nstride;
    for (int d = 0; d < 3; d++) {
      v.lo[d] = a.begin[d];
      v.hi[d] = a.end[d] - 1;
    }
    v.ncomp = a.ncomp;
    return v;
  }

  ppb_reactor* m_r = nullptr;
  ppb_options m_opt;
  int m_reactor_type = 1;
  int m_status = 0;
};

// The ReactorRK64 drop-in.
class ReactorB200RK : public ReactorB200
{
public:
  static std::string identifier() { return "ReactorB200RK"; }
  explicit ReactorB200RK(const std::string& mechanism) : ReactorB200(mechanism, "ReactorRK64") {}
};

} // namespace ppb_cpp
