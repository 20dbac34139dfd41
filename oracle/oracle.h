// ORACLE / TEST INFRASTRUCTURE ONLY -- the CPU checker for the B200 engine.
//
// A plain-C, FP64, table-driven restatement of the reference's per-cell
// chemistry path: the CEPTR-generated mechanism functions, the Fuego EOS
// wrappers, the reactor right-hand side and Jacobian, a CVODE-algorithm BDF
// integrator and the RK64 integrator.  Only tests/, __graft_entry__.smoke()
// and bench.py's CPU-baseline leg use it, always as the checker; the product
// library never links or calls it.  Each function cites the reference
// lines it restates.
#pragma once
#include "../pelephysics_b200/csrc/mech/mech_tables.h"
#include "../pelephysics_b200/csrc/mech/trans_tables.h"

#ifdef __cplusplus
extern "C" {
#endif

#define PPO_RU 8.31446261815324e7 // erg/mol/K (Source/Utility/PhysicsConstants.H:11)

const PPBMechTables* ppo_mech(const char* name);
int ppo_nsp(const char* name);
int ppo_nqss(const char* name); // QSS species of the mechanism (0: none)
const char* ppo_species_name(const char* name, int k);
void ppo_mw(const char* name, double* mw);

// thermo, per species (mechanism.H cv_R / cp_R / dcvpRdT /
// speciesInternalEnergy / speciesEnthalpy / gibbs)
void ppo_cv_R(const PPBMechTables* M, double T, double* out);
void ppo_cp_R(const PPBMechTables* M, double T, double* out);
void ppo_dcvpRdT(const PPBMechTables* M, double T, double* out);
void ppo_species_internal_energy(const PPBMechTables* M, double T, double* out);
void ppo_species_enthalpy(const PPBMechTables* M, double T, double* out);
void ppo_gibbs(const PPBMechTables* M, double T, double* out);
// mixture thermo (mechanism.H CKUBMS / CKHBMS / CKCVBS / CKCPBS / CKUMS / CKHMS / CKRHOY)
double ppo_ckubms(const PPBMechTables* M, double T, const double* y);
double ppo_ckhbms(const PPBMechTables* M, double T, const double* y);
double ppo_ckcvbs(const PPBMechTables* M, double T, const double* y);
double ppo_ckcpbs(const PPBMechTables* M, double T, const double* y);
void ppo_ckums(const PPBMechTables* M, double T, double* u);
void ppo_ckhms(const PPBMechTables* M, double T, double* h);
double ppo_ckrhoy(const PPBMechTables* M, double P, double T, const double* y);
// temperature from energy (mechanism.H GET_T_GIVEN_EY / GET_T_GIVEN_HY)
int ppo_get_t_given_ey(const PPBMechTables* M, double e, const double* y, double* T);
int ppo_get_t_given_hy(const PPBMechTables* M, double h, const double* y, double* T);
// rates and Jacobian (mechanism.H productionRate / aJacobian / DWDOT / CKWC)
void ppo_production_rate(const PPBMechTables* M, double* wdot, const double* sc, double T);
void ppo_qss_concentrations(const PPBMechTables* M, const double* sc, double T, double* out);
void ppo_qss_system(const PPBMechTables* M, const double* sc, double T, double* sys_out);
// per species sum |nu| (|q_f| + |q_r|): the scale of wdot's rounding error
void ppo_production_rate_abs(const PPBMechTables* M, double* absterm, const double* sc, double T);
void ppo_ckwc(const PPBMechTables* M, double T, const double* C, double* wdot);
void ppo_ajacobian(const PPBMechTables* M, double* J, const double* sc, double T, int consP);
void ppo_dwdot(const PPBMechTables* M, double* J, const double* sc, double T, int consP);

// Reactor right-hand side for one YCOrder cell (ReactorUtils.H:358-415) and
// the CPU dense Jacobian (ReactorCvodeJacobian.cpp:86-152, column-major).
double ppo_reactor_rhs(
  const PPBMechTables* M, int reactor_type, double t_rel, const double* y,
  double* ydot, double rhoe_init, double rhoesrc, const double* rYsrc);
void ppo_reactor_jac(const PPBMechTables* M, int reactor_type, const double* y, double* J);

// Per-cell integrator statistics.
typedef struct PPOStats {
  long nsteps, nfe, nje, nsetups, nni, ncfn, netf;
  int status; // 0 ok, <0 failure (CVODE flag values)
  int last_order;
  double last_h;
} PPOStats;

// Integrator options (ReactorCvode.cpp:18-35, :480-497; ReactorRK64.cpp:12-18)
typedef struct PPOOptions {
  double rtol, atol;
  int max_order;      // cvode.max_order
  long max_steps;     // CVodeSetMaxNumSteps
  int max_nls_iters;  // ode.max_nls_iters
  int max_err_fails;  // CVodeSetMaxErrTestFails
  int jac_eval_freq;  // CVodeSetJacEvalFrequency (msbj)
  int use_ref_kernels;// 1: the reference's compiled mechanism kernels; 0: tables
  int rk64_nsubsteps_guess, rk64_nsubsteps_min, rk64_nsubsteps_max;
  const double* typ_vals; // N+1 typical values or NULL
  int eos;                // 0 ideal gas (Fuego), 1 SRK (reactor type 1, difference-quotient Jacobian)
  // nonzero: every right-hand-side value is moved by at most one ulp (up,
  // down or not at all, from a per-cell stream of this seed): the algorithm
  // as an implementation whose arithmetic differs in the last bit runs it
  unsigned long long rhs_noise_seed;
} PPOOptions;

void ppo_default_options(PPOOptions* o);

// Mixture-averaged transport (Source/Transport/Simple.H, ideal gas) at one
// point: flags bit 0 bulk viscosity xi, 1 viscosity mu, 2 conductivity lam,
// 3 Ddiag, 4 thermal diffusion ratios chi (the light species; others 0).
#define NMAX_TR 96
const PPBTransTables* ppo_trans(const char* name);
int ppo_transport(const char* mech, int flags, double T, double rho, const double* Y, double* D, double* chi,
                  double* mu, double* xi, double* lam);
// Soave-Redlich-Kwong EOS (Source/Eos/SRK.H) for the e-reactor: the
// mechanism's GET_CRITPARAMS_SRK values, the EOS functions and the reactor
// right-hand side over them (reactor type 1).
const double* ppo_srk(const char* name);
int ppo_srk_rey2t(const char* mech, double R, double E, const double* Y, double* T);
double ppo_srk_rty2e(const char* mech, double R, double T, const double* Y);
void ppo_srk_rty2ei(const char* mech, double R, double T, const double* Y, double* Ei);
double ppo_srk_rty2cv(const char* mech, double R, double T, const double* Y);
void ppo_srk_rty2c(const char* mech, double R, double T, const double* Y, double* C);
void ppo_srk_rty2wdot(const char* mech, double R, double T, const double* Y, double* wdot);
double ppo_reactor_rhs_srk(const char* mech, double t_rel, const double* y, double* ydot, double rhoe_init,
                           double rhoesrc, const double* rYsrc);
int ppo_transport_batch(const char* mech, int flags, int ncells, const double* T, const double* rho, const double* Y,
                        double* D, double* chi, double* mu, double* xi, double* lam, int nthreads);

// ReactorArkode (ReactorArkode.cpp:10-20, :134-398): the whole batch as one
// explicit embedded RK integration with one adaptive step.
typedef struct PPOArkOptions {
  double rtol, atol;
  int rk_method;      // ode.rk_method (table number), 40
  int rk_controller;  // ode.rk_controller: 0 PID, 1 PI, 2 I, 3 explicit Gustafsson
  long max_steps;     // ARKODE's default 500
  const double* typ_vals_atol; // N+1 absolute tolerances or NULL
} PPOArkOptions;
typedef struct PPOArkStats {
  double t, h;        // time reached (tout on success), last step
  long nst, nfe, netf;
  int status;         // 0 ok, -1 too much work, -3 error-test failures, -27 too close
} PPOArkStats;
// rY[ncells*(N+1)] YCOrder in/out, rX advanced by the time reached; cells
// with mask == -1 are left untouched (mask may be NULL).
int ppo_react_arkode(
  const PPBMechTables* M, int reactor_type, const PPOArkOptions* opt, double* rY, const double* rYsrc, double* rX,
  const double* rX_src, const int* mask, double dt, int ncells, int nthreads, PPOArkStats* st);

// Integrate one cell (YCOrder y[N+1], in/out) over dt with the CVODE
// algorithm; returns the CVODE-style flag.
int ppo_bdf_cell(
  const PPBMechTables* M, int reactor_type, const PPOOptions* opt, double* y,
  const double* rYsrc, double rhoe_init, double rhoesrc, double dt, PPOStats* st);
// RK64 one cell (ReactorRK64.cpp:73-144); returns number of steps.
int ppo_rk64_cell(
  const PPBMechTables* M, int reactor_type, const PPOOptions* opt, double* y,
  const double* rYsrc, double rhoe_init, double rhoesrc, double dt);

// Flat react over ncells (ReactorBase.H:42-54 semantics: rY YCOrder with T in
// slot N, rYsrc [ncells*N], rX = rhoE, rX_src).  OpenMP over cells with
// nthreads (<=0: all).  method 0 = BDF, 1 = RK64.  Fills per-cell nfe (or RK
// steps) and status when the pointers are non-NULL.  Returns 0 or the first
// failing flag.
int ppo_react_flat(
  const char* mech, int reactor_type, const PPOOptions* opt, int method,
  double* rY, const double* rYsrc, double* rX, const double* rX_src, double dt,
  int ncells, int nthreads, long* nfe_out, int* status_out);

// Same over explicit mechanism tables (use_ref_kernels must be 0).
int ppo_react_flat_tables(
  const PPBMechTables* M, int reactor_type, const PPOOptions* opt, int method,
  double* rY, const double* rYsrc, double* rX, const double* rX_src, double dt,
  int ncells, int nthreads, long* nfe_out, int* status_out);
// Same as ppo_react_flat with the per-cell counters, 7 longs per cell: steps,
// RHS evaluations, Jacobian evaluations, factorisations of I - gamma J,
// Newton iterations, error-test failures, convergence failures (RK64: steps,
// 6 * steps, zeros).
int ppo_react_flat_stats(
  const char* mech, int reactor_type, const PPOOptions* opt, int method,
  double* rY, const double* rYsrc, double* rX, const double* rX_src, double dt,
  int ncells, int nthreads, int* status_out, long* stats_out);

// A copy of `name`'s tables with the forward Arrhenius parameters replaced
// (A in the tables' SI units, beta, Ea/R in K; arrays of R).  Free with
// ppo_mech_free.  Used for finite-difference derivatives.
PPBMechTables* ppo_mech_with_arrhenius(const char* name, const double* A, const double* beta, const double* EaR);
void ppo_mech_free(PPBMechTables* M);

// Select the reference kernels library (oracle/_ref/libref_<mech>.so) used
// when opt->use_ref_kernels is set.  Returns 0 when loaded.
int ppo_load_ref(const char* mech, const char* path);

#ifdef __cplusplus
}
#endif
