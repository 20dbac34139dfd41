// Empty stand-in for AMReX_Utility.H (test infrastructure only).
#ifndef PPB200_ORACLE_AMREX_UTILITY_STUB_H
#define PPB200_ORACLE_AMREX_UTILITY_STUB_H
#include "AMReX.H"
#endif
