// Minimal host-only stand-in for AMReX_Gpu.H (test infrastructure only):
// the macros and types the reference's generated mechanism.H needs.
#ifndef PPB200_ORACLE_AMREX_GPU_STUB_H
#define PPB200_ORACLE_AMREX_GPU_STUB_H
#include <cmath>
#include <cstdlib>
#include <string>
#include <vector>
#define AMREX_GPU_HOST_DEVICE
#define AMREX_GPU_DEVICE
#define AMREX_FORCE_INLINE inline
#define AMREX_GPU_CONSTANT
namespace amrex {
template <class T>
using Vector = std::vector<T>;
inline void Abort(const char* = "") { std::abort(); }
} // namespace amrex
#endif
