// C++ mirror of the reference's reactor interface over the engine's C ABI.
//
// pele::physics::reactions::ReactorBase (Source/Reactions/ReactorBase.H:13-106)
// without AMReX: ReactorB200 / ReactorB200RK expose the same calls -- init,
// the box react over Array4-style views, the flat react, close,
// set_typ_vals_ode, print_final_stats -- with the same argument meaning, and
// report errors through return codes instead of amrex::Abort.  Header-only;
// link pelephysics_b200/libppb200.so.
#pragma once

#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/pelephysics_b200.h"

namespace ppb_cpp {

// amrex::Array4<T>-compatible view: (i,j,k,n) -> p[(i-lo.x) + (j-lo.y)*jstride
// + (k-lo.z)*kstride + n*nstride], bounds [begin, end).
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

  // ReactorBase::init(reactor_type, ncells)
  int init(int reactor_type, int ncells) { return ppb_init(m_r, reactor_type, ncells, &m_opt); }

  // ReactorBase::close
  void close() { ppb_close(m_r); }

  // ReactorBase::set_typ_vals_ode
  int set_typ_vals_ode(const std::vector<double>& v) { return ppb_set_typ_vals(m_r, v.data(), (int)v.size()); }

  // ReactorBase::react(Box, Array4...) on device views
  int react(const Box& box, Array4View<double> const& rY, Array4View<double> const& rYsrc,
            Array4View<double> const& T, Array4View<double> const& rEner, Array4View<double> const& rEner_src,
            Array4View<double> const& FC, Array4View<int> const& mask, double& dt_react, double& time,
            void* stream = nullptr)
  {
    return ppb_react_box(m_r, box.lo, box.hi, view(rY), view(rYsrc), view(T), view(rEner), view(rEner_src),
                         view(FC), viewi(mask), &dt_react, &time, stream);
  }

  // ReactorBase::react(Real* ...) on flat YCOrder host arrays; returns the
  // cost as the reference does (RHS evaluations / average RK steps), or 1 on
  // an integration failure, or a negative PPB_E_* code.
  int react(double* rY, double* rYsrc, double* rX, double* rX_src, double& dt_react, double& time, int ncells,
            void* stream = nullptr)
  {
    long cost = 0;
    const int rc = ppb_react_flat(m_r, rY, rYsrc, rX, rX_src, &dt_react, &time, ncells, stream, &cost);
    if (rc != 0) return rc;
    return (int)cost;
  }

  // ReactorBase::print_final_stats: sums of the per-cell counters
  void print_final_stats(int ncells, FILE* out = stdout)
  {
    std::vector<int> st((size_t)ncells * 7);
    if (ppb_get_cell_stats(m_r, st.data(), ncells) != 0) return;
    long s[7] = {0, 0, 0, 0, 0, 0, 0};
    for (int c = 0; c < ncells; c++)
      for (int q = 0; q < 7; q++) s[q] += st[(size_t)c * 7 + q];
    std::fprintf(out, "-- Final stats: nSteps %ld nRHSeval %ld nJeval %ld nLinSetups %ld nNonlinIters %ld "
                      "nErrtf %ld nConvfail %ld\n",
                 s[0], s[1], s[2], s[3], s[4], s[5], s[6]);
  }

  const char* last_error() const { return ppb_last_error(); }

protected:
  static ppb_array4 view(Array4View<double> const& a)
  {
    ppb_array4 v;
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
};

// The ReactorRK64 drop-in.
class ReactorB200RK : public ReactorB200
{
public:
  static std::string identifier() { return "ReactorB200RK"; }
  explicit ReactorB200RK(const std::string& mechanism) : ReactorB200(mechanism, "ReactorRK64") {}
};

} // namespace ppb_cpp
