/*
 * pelephysics_b200 -- C ABI of the B200 stiff-chemistry engine.
 *
 * The entry points mirror the reference's reactor interface
 * (Source/Reactions/ReactorBase.H:13-106): a reactor is created by name
 * (Source/Factory.H:72-81), initialised with a reactor type and a cell count
 * (ReactorBase::init, ReactorBase.H:19), and advanced over a time step either
 * on flat per-cell arrays (ReactorBase::react, ReactorBase.H:42-54) or on a
 * box of Array4 views (ReactorBase::react, ReactorBase.H:25-40).  Plain
 * pointers and sizes only; no CUDA or C++ types cross the boundary (streams
 * are passed as void*, the value of a cudaStream_t).
 *
 * Every call returns 0 on success or a negative PPB_E* code; ppb_last_error()
 * gives a message.  No call aborts the process or traps the GPU.
 */
#ifndef PELEPHYSICS_B200_H
#define PELEPHYSICS_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define PPB_E_ARG (-1)      /* invalid argument */
#define PPB_E_CUDA (-2)     /* CUDA runtime error */
#define PPB_E_MECH (-3)     /* unknown mechanism */
#define PPB_E_STATE (-4)    /* call out of order (e.g. react before init) */
#define PPB_E_INTEGRATE (1) /* at least one cell failed to integrate (flat path of
                               ReactorCvode.cpp:1639-1641 returns 1 too); per-cell
                               flags via ppb_get_cell_status */

/* reactor types (Source/Reactions/ReactorTypes.H:10-11) */
#define PPB_REACTOR_E 1 /* internal energy / cv */
#define PPB_REACTOR_H 2 /* enthalpy / cp */

/* integration engine */
#define PPB_ENGINE_PLAIN 0 /* one thread per cell, FP64 */
#define PPB_ENGINE_TUNED 1 /* one warp per cell, persistent work queue */

typedef struct ppb_reactor ppb_reactor;

/* Options.  The first block carries the reference's ParmParse keys with the
 * reference defaults (ReactorCvode.cpp:18-35, ReactorCvode.H:187-197,
 * ReactorCvode.cpp:480-497, ReactorRK64.cpp:12-18); the second block is
 * engine tuning. */
typedef struct ppb_options {
  double rtol;              /* ode.rtol, 1e-6 */
  double atol;              /* ode.atol, 1e-10 */
  int max_order;            /* cvode.max_order, 2 */
  int max_steps;            /* CVodeSetMaxNumSteps, 10000 */
  int max_nls_iters;        /* ode.max_nls_iters, 3 */
  int max_err_fails;        /* CVodeSetMaxErrTestFails, 100 */
  int jac_eval_freq;        /* CVodeSetJacEvalFrequency, 100 */
  int clean_init_massfrac;  /* ode.clean_init_massfrac, 0 */
  int rk64_nsubsteps_guess; /* ode.rk64_nsubsteps_guess, 10 */
  int rk64_nsubsteps_min;   /* ode.rk64_nsubsteps_min, 5 */
  int rk64_nsubsteps_max;   /* ode.rk64_nsubsteps_max, 500 */
  int verbose;              /* ode.verbose, 0 */
  int engine;               /* PPB_ENGINE_TUNED */
  int lu_fp32;              /* factor I - gamma J in FP32 + FP64 refinement, 0 */
  int refine_sweeps;        /* refinement sweeps with lu_fp32, 1 */
  int warps_per_block;      /* tuned engine block size in warps (1, 2, 4, 8; 12 or 16 for the BDF, either LU
                               precision, with 32 lanes per cell and budget 2: one block per SM); 0 = autotune the block
                               size, lanes per cell and register budget on the first call (the SRK EOS and QSS
                               mechanisms, not autotuned: 16 warps where 16 cells fit one SM, else <= 8) */
  int use_graph;            /* replay react() as a captured CUDA graph, 1 */
  int adjoint_checkpoint_interval; /* accepted BDF steps between adjoint checkpoints, 16 */
  int adjoint_memory_mb;    /* device memory for adjoint checkpoints, tapes and points, 16384 */
  int team_lanes;           /* with warps_per_block > 0: lanes per cell, 32, 16 (<= 21 species), 64
                               (33..64 species) or 128 (65..128 species; one cell per block) */
  int register_budget;      /* with warps_per_block > 0: 2 (<= 128 registers) or 1 (<= 255) */
  /* ReactorArkode (ReactorArkode.cpp:10-20, ReactorArkode.H:131-137) */
  int rk_method;            /* ode.rk_method, 40 (ZONNEVELD_5_3_4); box path only, as in the reference */
  int rk_controller;        /* ode.rk_controller, 0 (PID), 1 PI, 2 I, 3 explicit Gustafsson; box path only */
  int use_erkstep;          /* ode.use_erkstep, 1 (ERKStep and an explicit-only ARKStep integrate alike) */
  int arkode_max_steps;     /* internal steps per react call, 500 (the ARKODE default; the reference sets none) */
  /* equation of state (the reference's build-time EOS choice, Source/Eos/EOS.H:20-27) */
  int eos;                  /* PPB_EOS_IDEAL (Fuego, default) or PPB_EOS_SRK (ReactorCvode, reactor type 1) */
  int cost_order;           /* tuned engine: hand cells to the work queue by descending cost of the previous
                               call on this reactor (longest first: no tail of a few slow cells), 1 */
  int rendezvous_cycles;    /* tuned engine, one warp per cell: before each right-hand side a cell's warp waits
                               up to this many SM clock cycles for the other warps of its block, so that they
                               run the right-hand side's instruction stream together (0: off; at most 1e7;
                               -1: for blocks of more than 8 warps the autotuner picks 300000 or 1000000, a
                               fixed launch takes 300000; 1000000 for smaller blocks and in the adjoint;
                               results are unchanged either way), -1 */
  int arkode_barrier_us;    /* ReactorArkode: longest wait of a block at the grid barrier of its one cooperative
                               launch, in microseconds (0..60000000; 0: a block that would have to wait gives up
                               at once); a wait that runs out ends the call with PPB_E_CUDA and the message
                               "grid barrier timed out" instead of hanging, 20000000 */
  int adjoint_keep_segments; /* adjoint: keep a copy of every recorded segment that fits in a third of what
                               adjoint_memory_mb leaves after the per-cell arrays, so that the reverse sweep
                               recomputes from a checkpoint only those that did not fit (0: recompute every
                               segment; the gradient is the same either way, bit for bit), 1 */
} ppb_options;

#define PPB_EOS_IDEAL 0 /* ideal gas: the mechanism's NASA-7 thermo (Source/Eos/Fuego.H) */
#define PPB_EOS_SRK 1   /* Soave-Redlich-Kwong real gas (Source/Eos/SRK.H): e-reactor only, BDF with a
                           difference-quotient Jacobian (SRK has no analytical one) */

/* An amrex::Array4<Real>-compatible view: element (i,j,k,n) lives at
 * p[(i-lo[0]) + (j-lo[1])*jstride + (k-lo[2])*kstride + n*nstride]. */
typedef struct ppb_array4 {
  double* p;
  long jstride, kstride, nstride;
  int lo[3], hi[3]; /* inclusive bounds of the allocation */
  int ncomp;
} ppb_array4;

typedef struct ppb_array4i {
  int* p;
  long jstride, kstride, nstride;
  int lo[3], hi[3];
  int ncomp;
} ppb_array4i;

/* Fill an options struct with the reference defaults. */
void ppb_default_options(ppb_options* opt);

/* Last error message of the calling thread. */
const char* ppb_last_error(void);

/* Mechanisms compiled into the library (LiDryer, drm19, dodecane_lu,
 * heptane_lu_88sk, grimech30, FFCM1_Red, chem-H, and the QSS mechanisms CH4_lean_qss, C1-C2-NO_qss and
 * LuEthylene_qss, whose species in quasi-steady state are not counted: their
 * productionRate solves them first, as their mechanism.H does): returns the
 * number of species and reactions of `mechanism`, or PPB_E_MECH. */
int ppb_mechanism_info(const char* mechanism, int* nspecies, int* nreactions);
/* Name of species k of `mechanism` (NULL when out of range). */
const char* ppb_species_name(const char* mechanism, int k);

/* Molecular weights (g/mol) of the species of `mechanism` (mechanism.H
 * get_mw), written to the HOST array mw[N]. */
int ppb_molecular_weights(const char* mechanism, double* mw);

/* ReactorBase::create (Factory.H:72-81).  integrator is "ReactorCvode"
 * (BDF, the ReactorCvode drop-in), "ReactorRK64" (explicit RK64) or
 * "ReactorArkode" (explicit embedded RK over the whole batch with one
 * adaptive step, the ReactorArkode drop-in: ReactorArkode.cpp:134-398; the
 * flat paths use the default order-4 table and PID controller, the box path
 * rk_method / rk_controller, as the reference does).  For ReactorArkode a
 * call that stops early (arkode_max_steps reached, repeated error-test
 * failures) returns PPB_E_INTEGRATE with *dt_react set to the interval
 * actually integrated (the reference's MOD_REACTOR bookkeeping,
 * ReactorArkode.cpp:223-226) and rX advanced by that interval. */
int ppb_create(const char* mechanism, const char* integrator, ppb_reactor** out);
/* ReactorBase::init(reactor_type, ncells) (ReactorBase.H:19) with options. */
int ppb_init(ppb_reactor* r, int reactor_type, int ncells, const ppb_options* opt);
/* ReactorBase::set_typ_vals_ode (ReactorBase.H:88, ReactorBase.cpp:6-31):
 * N+1 typical values; atol becomes typ_vals[i] * atol. */
int ppb_set_typ_vals(ppb_reactor* r, const double* typ_vals, int n);
/* ReactorBase::close (ReactorBase.H:21) and destruction. */
int ppb_close(ppb_reactor* r);
void ppb_destroy(ppb_reactor* r);

/* ReactorBase::react on flat YCOrder HOST arrays (ReactorBase.H:42-54;
 * ReactorCvode.cpp:1491-1689, ReactorRK64.cpp:22-164):
 *   rY[ncells*(N+1)]  rhoY_k then T per cell (in/out)
 *   rYsrc[ncells*N]   species sources (in)
 *   rX[ncells]        rho*e or rho*h (in/out: rX += dt*rX_src)
 *   rX_src[ncells]    energy source (in)
 * dt_react and time are in/out as in the reference (time += dt_react).
 * Returns the number of right-hand-side evaluations summed over cells (BDF)
 * or the average number of RK steps (RK64) as a non-negative value in *cost,
 * and 0 / PPB_E_INTEGRATE / an error code as the return value. */
int ppb_react_flat(ppb_reactor* r, double* rY, double* rYsrc, double* rX, double* rX_src, double* dt_react,
                   double* time, int ncells, void* stream, long* cost);

/* Same on DEVICE arrays in the same YCOrder layout. */
int ppb_react_flat_device(ppb_reactor* r, double* rY, double* rYsrc, double* rX, double* rX_src,
                          double* dt_react, double* time, int ncells, void* stream, long* cost);

/* Same on DEVICE arrays already in species-major (SoA) layout with leading
 * dimension ld >= ncells: y[i*ld + c] for i <= N, src[i*ld + c] for i < N. */
int ppb_react_soa_device(ppb_reactor* r, double* y, const double* src, double* rX, const double* rX_src, int ld,
                         double* dt_react, double* time, int ncells, void* stream, long* cost);

/* ReactorBase::react on a box of DEVICE Array4 views (ReactorBase.H:25-40;
 * ReactorCvode.cpp:1267-1489 with box_flatten/box_unflatten of
 * ReactorUtils.H:160-291): lo/hi are the box bounds (inclusive); rY has N
 * components, T, rEner, rEner_src and FC one; cells with mask == -1 are
 * skipped and get FC = 0. */
int ppb_react_box(ppb_reactor* r, const int lo[3], const int hi[3], ppb_array4 rY, ppb_array4 rYsrc, ppb_array4 T,
                  ppb_array4 rEner, ppb_array4 rEner_src, ppb_array4 FC, ppb_array4i mask, double* dt_react,
                  double* time, void* stream);

/* ReactorBase::flatten (ReactorBase.H:56-67; FlattenOps::flatten and
 * box_flatten of ReactorUtils.H:160-220, 302-324) on DEVICE arrays: the box's
 * cells (i fastest) into component-major vectors -- the reference GPU build's
 * CYOrder (ReactorCvode.H:65): y_vect[n*ncells + c] for n <= N (T from the
 * energy with the stored T as the Newton start, in slot N), src_vect[n*ncells
 * + c], vect_energy[c], src_vect_energy[c], ncells the box's cell count --
 * with the reactor's reactor type and clean_init_massfrac.  Stream-ordered. */
int ppb_flatten(ppb_reactor* r, const int lo[3], const int hi[3], ppb_array4 rhoY, ppb_array4 frcExt,
                ppb_array4 temperature, ppb_array4 rhoE, ppb_array4 frcEExt, double* y_vect, double* src_vect,
                double* vect_energy, double* src_vect_energy, void* stream);
/* ReactorBase::unflatten (ReactorBase.H:69-80; box_unflatten of
 * ReactorUtils.H:222-291) on DEVICE arrays: rhoY from y_vect (with
 * clean_init_massfrac the clipped increment is added to the old rhoY),
 * rhoE = vect_energy + dt * frcEExt, T from the new energy, FC = FCunt[c]. */
int ppb_unflatten(ppb_reactor* r, const int lo[3], const int hi[3], ppb_array4 rhoY, ppb_array4 temperature,
                  ppb_array4 rhoE, ppb_array4 frcEExt, ppb_array4 FC, const double* y_vect,
                  const double* vect_energy, const long* FCunt, double dt, void* stream);

/* Per-cell integrator flag (0 ok, 1 skipped by mask, <0 CVODE-style failure
 * code) and cost (RHS evaluations or RK steps) of the last react call. */
int ppb_get_cell_status(ppb_reactor* r, int* status, int* cost, int ncells);

/* Cell count of the calling thread's last react call on r (0 before one;
 * negative PPB_E_ARG for a null reactor). */
int ppb_last_ncells(ppb_reactor* r);

/* Per-cell integrator counters of the last react call, 7 ints per cell:
 * steps, RHS evaluations, Jacobian evaluations, matrix factorisations,
 * Newton iterations, error-test failures, convergence failures (the
 * statistics ReactorCvode::print_final_stats reports, ReactorCvode.cpp:
 * 1838-1901, kept per cell).  RK64: steps, 6*steps, then zeros. */
int ppb_get_cell_stats(ppb_reactor* r, int* stats, int ncells);

/* Measured FP64 FMA throughput of the current device in GFLOP/s (a short
 * probe kernel); the denominator of the engine's compute roofline.  No
 * counterpart in the reference. */
int ppb_probe_fp64_peak(double* gflops, void* stream);

/* Pointwise mechanism kernels on DEVICE arrays, one cell per row, for
 * parity checks; team = 1 (thread per cell) or 32 (warp per cell).
 * mechanism.H productionRate (SI: mol/m^3 in, mol/m^3/s out):
 *   sc[ncells*N], T[ncells] -> wdot[ncells*N] */
int ppb_production_rate(const char* mechanism, const double* sc, const double* T, double* wdot, int ncells, int team,
                        void* stream);
/* mechanism.H aJacobian (SI), J[ncells*(N+1)^2] with
 * J[k*(N+1)+m] = d wdot_m / d sc_k (not for a QSS mechanism: PPB_E_CUDA,
 * "operation not supported"; its reactor forms the Jacobian by differences) */
int ppb_ajacobian(const char* mechanism, const double* sc, const double* T, int consP, double* J, int ncells,
                  int team, void* stream);
/* mechanism.H GET_T_GIVEN_EY (eh = 0) / GET_T_GIVEN_HY (eh = 1): e[ncells],
 * Y[ncells*N], T[ncells] in (initial guess) / out. */
int ppb_t_from_energy(const char* mechanism, int eh, const double* e, const double* Y, double* T, int ncells,
                      int team, void* stream);
/* ReactorUtils.H fKernelSpec: y[ncells*(N+1)] YCOrder, rhoe/rhoesrc[ncells],
 * src[ncells*N] -> ydot[ncells*(N+1)] at time t since the start of react. */
int ppb_reactor_rhs(const char* mechanism, int reactor_type, double t, const double* y, const double* rhoe,
                    const double* rhoesrc, const double* src, double* ydot, int ncells, int team, void* stream);

/* Fuego::PYT2RE (Source/Eos/Fuego.H:313-327) on DEVICE arrays: rho from
 * CKRHOY(P, T, Y) and e = CKUBMS (eh = 0) or h = CKHBMS (eh = 1), erg/g. */
int ppb_pyt2re(const char* mechanism, int eh, const double* P, const double* T, const double* Y, double* rho,
               double* e, int ncells, void* stream);

/* Mixture-averaged transport coefficients: the reference's SimpleTransport
 * (Source/Transport/Simple.H) with the ideal-gas EOS and the mechanism's
 * CEPTR transport fits.  flags select the outputs as SimpleTransport::
 * transport's wtr_get_* switches do (Simple.H:263-270); xi is computed only
 * together with mu (else 0), as there. */
#define PPB_TR_XI 1   /* bulk viscosity xi, g/(cm s) */
#define PPB_TR_MU 2   /* shear viscosity mu, g/(cm s) */
#define PPB_TR_LAM 4  /* thermal conductivity lambda, erg/(cm s K) */
#define PPB_TR_DIAG 8 /* mixture-averaged Ddiag_k (rho D_k W_k / W), g/(cm s) */
#define PPB_TR_CHI 16 /* thermal diffusion ratios of the light species (others 0) */
/* SimpleTransport::transport per cell on DEVICE arrays: T, rho [ncells];
 * Y, D, chi species-major with leading dimension ld >= ncells
 * (Y[k*ld + c]); outputs not selected by flags may be NULL. */
int ppb_transport(const char* mechanism, int flags, const double* T, const double* rho, const double* Y, int ld,
                  double* D, double* chi, double* mu, double* xi, double* lam, int ncells, void* stream);
/* SimpleTransport::get_transport_coeffs (Simple.H:395-446) on a box of DEVICE
 * Array4 views: Y, D, chi N components, T, rho, mu, xi, lam one; chi is
 * written only with use_soret (transport.use_soret), as there. */
int ppb_transport_box(const char* mechanism, int use_soret, const int lo[3], const int hi[3], ppb_array4 Y,
                      ppb_array4 T, ppb_array4 rho, ppb_array4 D, ppb_array4 chi, ppb_array4 mu, ppb_array4 xi,
                      ppb_array4 lam, void* stream);

/* Allocation-free flat react on DEVICE YCOrder arrays (no counterpart in the
 * reference).  For callers that must not have a library allocate GPU memory,
 * e.g. applications whose device memory is owned by an arena allocator
 * (AMReX-based codes hand every device buffer out of the AMReX Arena).  It
 * runs the tuned engine out of one static device array of 32 MiB per GPU
 * holding the mechanism tables and the per-call scratch, and calls no
 * cudaMalloc/cudaFree.  Limits: at most
 * floor((30 MiB - 1 KiB) / (8 (2N+1) + 12)) cells per call (drm19: 88,360;
 * heptane_lu_88sk: 22,028); larger calls return PPB_E_ARG.  The first call on
 * a device (and the first use of each further mechanism there) does a
 * synchronous set-up -- resolving the array's address and copying the
 * mechanism tables -- and should come before any stream capture.  Every call
 * on a device shares the array and keeps the last call's contents; calls
 * that overlap on the GPU race and must not be issued.  integrator is
 * "ReactorCvode" or "ReactorRK64"; opt may be NULL (reference defaults); the
 * arrays are as in ppb_react_flat and rX += dt_react * rX_src.  Options:
 * the integrator keys, lu_fp32 / refine_sweeps, eos (SRK as ppb_init allows
 * it), rendezvous_cycles and a fixed launch (warps_per_block, team_lanes,
 * register_budget; warps_per_block = 0 takes the largest block of <= 8 warps
 * of one warp per cell, as there is no autotuner here) are honoured; a value
 * this path cannot honour returns PPB_E_ARG.  use_graph and cost_order only
 * schedule work and leave results unchanged; they are not used (no graph,
 * cells in index order).  There are no typical values (ppb_set_typ_vals
 * belongs to a reactor handle).  The results are bitwise those of
 * ppb_react_flat_device with the same launch and cost_order = 0.  When nfailed
 * is not NULL the call waits for the stream and stores the number of cells
 * that failed (returning PPB_E_INTEGRATE if any); with nfailed == NULL it
 * returns once the work is queued. */
int ppb_react_flat_device_noalloc(const char* mechanism, const char* integrator, int reactor_type,
                                  const ppb_options* opt, double* rY, double* rYsrc, double* rX, double* rX_src,
                                  double dt_react, int ncells, void* stream, int* nfailed);

/* Launch configuration of the tuned engine the reactor uses (after the
 * autotuner ran, when warps_per_block was 0): block size in warps, lanes per
 * cell, register budget, and the autotuner's measured time of the chosen
 * configuration on its sample (ms; 0 when not tuned).  No counterpart in the
 * reference. */
int ppb_get_launch_config(ppb_reactor* r, int* warps_per_block, int* team_lanes, int* register_budget,
                          double* tuned_ms);

/* The block rendezvous bound (SM clocks) the reactor's tuned BDF launches use:
 * rendezvous_cycles when set, else the autotuner's pick or the block-size
 * default; 0 when its launches have no rendezvous (rendezvous_cycles = 0,
 * RK64, the plain engine, teams of other than 32 lanes).  No counterpart in
 * the reference. */
int ppb_get_rendezvous_cycles(ppb_reactor* r, int* cycles);

/* ---- Differentiation (no counterpart in the reference; the ReactorBase
 * interface has no derivative entry points).
 *
 * Parameters are per reaction r: ln A_r, beta_r and Ea_r/R (K) of the
 * forward rate constant k = A T^beta exp(-(Ea/R)/T) as the mechanism tables
 * hold it (A in SI mol-m^3-s units; for fall-off reactions the high-pressure
 * limit).  Gradient vectors are [3][R]: d/d ln A, d/d beta, d/d (Ea/R).
 * dL/dEa in the mechanism's energy unit is dL/d(Ea/R) / R in that unit. */

/* Arrhenius parameters of the reactor's mechanism (HOST arrays of R). */
int ppb_get_arrhenius(ppb_reactor* r, double* A, double* beta, double* EaR);
/* Replace them for this reactor (its react() and adjoint calls use a
 * private copy of the mechanism tables from then on). */
int ppb_set_arrhenius(ppb_reactor* r, const double* A, const double* beta, const double* EaR);

/* Discrete adjoint of ppb_react_flat over dt_react for the BDF integrator
 * ("ReactorCvode"), tuned engine, on DEVICE arrays (YCOrder, as
 * ppb_react_flat_device; rX is not updated).  Given lam_y = dL/dy(dt) per
 * cell ([ncells][N+1], y = rhoY_k and the T slot as integrated), it returns
 * y(dt) in y_out, dL/dy0 in lam_y0 ([ncells][N+1]), dL/drX (the energy
 * rhoe or rhoh) in lam_e ([ncells], may be NULL) and dL/dp summed over the
 * cells in grad_params ([3R], may be NULL).  The step sizes and orders are
 * those of the forward integration (frozen); the forward states are
 * recomputed from checkpoints every opt.adjoint_checkpoint_interval accepted
 * steps.  Per-cell status / counters: ppb_get_cell_status / _stats. */
int ppb_adjoint_flat_device(ppb_reactor* r, const double* rY0, const double* rYsrc, const double* rX,
                            const double* rX_src, double dt_react, int ncells, const double* lam_y, double* y_out,
                            double* lam_y0, double* lam_e, double* grad_params, void* stream);
/* Tangent-linear model of the same integration: the derivative of y(dt) in
 * the direction (dy0 [ncells][N+1], drX [ncells], dparams [3R]); any
 * direction pointer may be NULL (zero). */
int ppb_tangent_flat_device(ppb_reactor* r, const double* rY0, const double* rYsrc, const double* rX,
                            const double* rX_src, double dt_react, int ncells, const double* dy0, const double* drX,
                            const double* dparams, double* y_out, double* dy_out, void* stream);
/* Pointwise exact derivatives of the reactor right-hand side (fKernelSpec,
 * with T from the energy constraint) on DEVICE arrays: f, df/dy
 * ([ncells][(N+1)^2], column-major: entry j*(N+1)+i = d f_i / d y_j),
 * df/drX, and for weights v ([ncells][N+1]) v^T df/dy, v^T df/drX and
 * v^T df/dp ([ncells][3R]).  Any output may be NULL. */
int ppb_rhs_exact(const char* mechanism, int reactor_type, double t, const double* y, const double* rhoe,
                  const double* rhoesrc, const double* src, const double* v, double* f, double* dfdy, double* dfde,
                  double* vjp_y, double* vjp_e, double* vjp_p, int ncells, void* stream);

#ifdef __cplusplus
}
#endif
#endif
