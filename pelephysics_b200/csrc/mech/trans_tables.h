// Transport tables shared by the CUDA transport kernel and the CPU oracle.
//
// One PPBTransTables holds a mechanism's mixture-averaged transport data as
// the reference's SimpleTransport reads it from the generated mechanism.H
// (Source/Transport/TransportParams.H:228-258): molecular data, the CEPTR
// log-T polynomial fits of the pure-species viscosities and conductivities
// and of the binary diffusion coefficients, the light species and their
// thermal-diffusion-ratio fits, and CKCVMS's R / W_k factors (bulk
// viscosity).  Produced by pelephysics_b200/mechgen/transport_tables.py.
#pragma once

#ifdef __cplusplus
extern "C" {
#endif

typedef struct PPBTransTables {
  const char* name;
  int nsp;
  int nlite;
  const double* wt;       // egtransetWT, g/mol
  const double* eps;      // egtransetEPS, epsilon / k_B, K
  const double* sig;      // egtransetSIG, Angstrom
  const double* dip;      // egtransetDIP, Debye
  const double* pol;      // egtransetPOL, Angstrom^3
  const double* zrot;     // egtransetZROT
  const int* nlin;        // egtransetNLIN: 0 atom, 1 linear, 2 nonlinear
  const double* fitmu;    // egtransetCOFETA: 4 per species, ln(mu) in ln T
  const double* fitlam;   // egtransetCOFLAM: 4 per species, ln(lambda) in ln T
  const double* fitdbin;  // egtransetCOFD: 4 per (i + N j), ln(D_ij P) in ln T
  const int* ktdif;       // egtransetKTDIF: light species (0-based)
  const double* fittdrat; // egtransetCOFTD: 4 per (j + N n), thermal diffusion ratio in T
  const double* cvms;     // CKCVMS: R / W_k, erg/(g K)
} PPBTransTables;

#ifdef __cplusplus
}
#endif
