// Minimal stand-in for the AMReX header that the reference's generated
// mechanism.H includes. Test infrastructure only: it lets oracle/ref_wrap.cpp
// compile the reference's own mechanism kernels on the host without AMReX.
#ifndef PPB200_ORACLE_AMREX_REAL_STUB_H
#define PPB200_ORACLE_AMREX_REAL_STUB_H
namespace amrex {
using Real = double;
}
#endif
