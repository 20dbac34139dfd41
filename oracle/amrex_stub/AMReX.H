// Minimal host-only stand-in for AMReX.H (test infrastructure only): what the
// reference's Source/Eos/SRK.H needs to compile without AMReX.
#ifndef PPB200_ORACLE_AMREX_STUB_H
#define PPB200_ORACLE_AMREX_STUB_H
#include <cstdlib>
#include "AMReX_Gpu.H"
#include "AMReX_REAL.H"
#ifndef AMREX_ASSERT
#define AMREX_ASSERT(x) ((void)0)
#endif
namespace amrex {
inline void Error(const char* = "") { std::abort(); }
} // namespace amrex
#endif
