// Mechanism tables shared by the CUDA engine and the CPU oracle.
//
// One PPBMechTables describes a gas-phase mechanism the way the reference's
// generated Mechanisms/<mech>/mechanism.H hard-wires it: NASA-7 coefficient
// sets per thermo routine, Arrhenius data in SI units, third-body
// efficiencies, fall-off parameters and the stoichiometry the generated
// productionRate / aJacobian use.  Reactions are stored in the reference's
// evaluation order (Troe, SRI, Lindemann, third-body, elementary);
// rx_orig maps back to the mechanism file's reaction index.
// The tables are produced by pelephysics_b200/mechgen/ceptr_tables.py.
#pragma once

#ifdef __cplusplus
extern "C" {
#endif

enum {
  PPB_RX_SIMPLE = 0,    // k_f * phi_f - k_r * phi_r
  PPB_RX_THIRD = 1,     // (mixture + sum (eff-1) c) * (...)
  PPB_RX_COLLIDER = 2,  // explicit single collider folded into phi_f/phi_r
  PPB_RX_TROE = 3,      // fall-off, Troe broadening
  PPB_RX_LINDEMANN = 4, // fall-off, no broadening
  PPB_RX_SRI = 5        // fall-off, SRI broadening (rates only)
};

enum {
  PPB_MAXPS = 6, // phase-space entries per side
  PPB_MAXW = 8,  // production-rate wdot updates per reaction
  PPB_MAXKC = 10,
  PPB_MAXJN = 8,
  PPB_NFOD = 17, // doubles per fall-off record
  PPB_NFOI = 8   // ints per fall-off record
};

// fall-off double record layout
enum {
  PPB_FO_P0 = 0,    // low-pressure factor used by productionRate (redP)
  PPB_FO_K0 = 1,    // low-pressure factor used by aJacobian (k_0)
  PPB_FO_BETA0 = 2,
  PPB_FO_EAR0 = 3,
  PPB_FO_PRDIM = 4, // 10^(-6 dim) literal of the Jacobian's Pr
  PPB_FO_A = 5,     // Troe alpha
  PPB_FO_T3 = 6,
  PPB_FO_T1 = 7,
  PPB_FO_T2 = 8,
  PPB_FO_OMA = 9,   // 1 - alpha as printed for productionRate
  PPB_FO_IT3 = 10,  // 1/T3 as printed for productionRate
  PPB_FO_IT1 = 11,  // 1/T1 as printed for productionRate
  PPB_FO_SRI = 12   // 5 SRI parameters a, b, c, d, e
};
// fall-off int record layout
enum {
  PPB_FOI_NTROE = 0,
  PPB_FOI_P1 = 1, // productionRate writes the (1-a) exp(-T/T3) term
  PPB_FOI_P2 = 2, // productionRate writes the a exp(-T/T1) term
  PPB_FOI_J1 = 3, // aJacobian writes Fcent1
  PPB_FOI_J2 = 4, // aJacobian writes Fcent2
  PPB_FOI_J3 = 5, // aJacobian uses T2 in dlogFcent/dT
  PPB_FOI_NSRI = 6
};

typedef struct PPBMechTables {
  const char* name;
  int nsp;
  int nrxn;
  const char* const* species;
  const double* mw;   // g/mol, as printed (%f)
  const double* imw;  // 1/mw, as printed (%.16f)
  const double* tmid; // NASA-7 mid-point; < 0 for a single range
  // per species: [low range coefs][high range coefs]
  const double* th_cv;  // 5: cv/R
  const double* th_cp;  // 5: cp/R
  const double* th_dcp; // 4: d(cp/R)/dT
  const double* th_u;   // 6: e/RT (last one multiplies 1/T)
  const double* th_h;   // 6: h/RT (last one multiplies 1/T)
  const double* th_g;   // 7: g/RT: 1/T, 1, log T, T, T^2, T^3, T^4
  const int* rx_orig;
  const int* rx_kind;
  const int* rx_rev;
  const double* rx_A;    // SI pre-exponential
  const double* rx_beta;
  const double* rx_EaR;  // Ea/R in K
  const int* rx_kcpow;   // power of 1/refC (refC = P_atm/(R T)) in k_r = k_f exp(-arg) refC^-p
  const double* rx_sum_nuk;
  // lists padded to a fixed width per reaction: n[r], sp[r*W+j], c[r*W+j]
  const int* rx_fps_n;  // forward phase space (species, order)
  const int* rx_fps_sp;
  const double* rx_fps_c;
  const int* rx_rps_n;  // reverse phase space
  const int* rx_rps_sp;
  const double* rx_rps_c;
  const int* rx_kc_n;   // Gibbs terms: exponent arg = sum c * g_RT[sp]
  const int* rx_kc_sp;
  const double* rx_kc_c;
  const int* rx_wup_n;  // productionRate wdot updates: wdot[sp] += c * qdot
  const int* rx_wup_sp;
  const double* rx_wup_c;
  const int* rx_jn_n;   // aJacobian net stoichiometry
  const int* rx_jn_sp;
  const double* rx_jn_c;
  const int* rx_hr_n;   // aJacobian dlnKc/dT reactant terms
  const int* rx_hr_sp;
  const double* rx_hr_c;
  const int* rx_hp_n;   // aJacobian dlnKc/dT product terms
  const int* rx_hp_sp;
  const double* rx_hp_c;
  const int* eff_off;   // CSR offsets, nrxn+1
  const int* eff_sp;
  const double* eff_e;  // efficiency (aJacobian)
  const double* eff_m1; // efficiency - 1 (productionRate)
  const double* fo_d;   // PPB_NFOD per reaction
  const int* fo_i;      // PPB_NFOI per reaction
  // QSS mechanisms (the reference's QSSA mechanisms; zero / null otherwise).
  // The nqss species in steady state have no state entry and no rate: their
  // concentrations are solved per evaluation from their linear balance
  // (comp_sc_qss of the reference's generated mechanism.H).  Species slots of
  // the reaction lists: 0..nsp-1 transported species, nsp the unit slot
  // (concentration 1, g/RT 0), nsp+1+q the QSS species q; the thermo arrays
  // and tmid have an entry per slot (the unit slot's is empty), mw and imw
  // the transported species only.
  int nqss;
  int nrq;                          // reactions with a QSS species (k = 0..nrq-1)
  const char* const* qss_species;
  const int* q_rx;                  // [nrq] the reaction (evaluation order) of QSS reaction k
  const int* q_off;                 // [nqss + 1] each QSS species' balance terms, in k order:
  const int* q_term;                //   2 k + 0 (forward coefficient of k) or 2 k + 1 (reverse)
  const int* q_role;                //   -1 production, -2 loss, j >= 0 production from QSS species j
  const double* q_coef;             //   molecules of the species the term makes or uses (1 or 2)
  const int* rx_rmfwd;              // [nrxn] 1: forward rate removed by the QSS reduction (qdot = -q_r)
} PPBMechTables;

#ifdef __cplusplus
}
#endif
