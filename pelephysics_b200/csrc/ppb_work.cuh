// Shared-memory workspace layout of one team-integrated cell.
#pragma once
#include "ppb_bdf.cuh"

namespace ppb {
// ------------------------------------------------------------ workspace
// FP64 factor (LT = double): the saved Jacobian J (FP64, n x n) among the
// vectors, then the Newton-matrix region -- the n x n factor, or the
// per-reaction factors of the warp-cooperative Jacobian evaluation (4 doubles
// per reaction; 5 in the adjoint's exact Jacobian), which use it while the
// factor is not live, whichever is larger.
// FP32 factor (LT = float): the per-reaction factors (4 doubles each) get a
// region of their own and the saved Jacobian is kept in FP32 next to the
// FP32 factor; the
// two (8 n^2 bytes) hold the FP64 Jacobian while it is evaluated, which is
// then rounded to FP32 in place.  The Jacobian only drives the modified
// Newton iteration, whose residual is the FP64 right-hand side, so its
// precision changes the convergence rate, not the converged step; the cell
// shrinks from 8 n^2 + max(4 n^2, 40 R) to 8 n^2 + 32 R bytes plus the
// vectors (heptane_lu_88sk: 117 KB -> 107 KB, two cells per SM instead of
// one; the FP64 factor takes 146 KB).
template <typename LT>
__host__ __device__ inline size_t a_region_bytes(int N, int R)
{
  const size_t n = N + 1;
  size_t a = n * n * sizeof(LT);
  const size_t jx = 40 * (size_t)R;
  if (sizeof(LT) == sizeof(double) && jx > a) a = jx;
  return (a + 15) & ~size_t(15);
}

template <typename LT>
__host__ __device__ inline size_t jx_region_bytes(int R)
{
  return sizeof(LT) == sizeof(double) ? 0 : ((32 * (size_t)R + 15) & ~size_t(15));
}

// The saved Jacobian's region, padded to 16 bytes so that the factor (and
// what follows it: pivots, row order, the doubles of the coefficient
// arrays) starts 8-byte aligned for an odd n^2 in FP32 too.
template <typename LT>
__host__ __device__ inline size_t j_region_bytes(int N)
{
  const size_t n = N + 1;
  return (n * n * sizeof(LT) + 15) & ~size_t(15);
}

// pivots and row permutation (2n ints), then the coefficient arrays; for a
// QSS mechanism (Q QSS species, K reactions with one) a tail with the
// concentrations and g/RT over all n + Q slots (in place of the n-long
// ones) and the QSS solve's scratch
template <typename LT>
__host__ __device__ inline size_t team_bytes(int N, int R, int Q = 0, int K = 0)
{
  const int n = N + 1;
  const size_t d = 22 * (size_t)n + (size_t)R;
  size_t b = d * 8 + j_region_bytes<LT>(N) + jx_region_bytes<LT>(R) + a_region_bytes<LT>(N, R) +
             ((8 * (size_t)n + 7) & ~size_t(7)) + sizeof(BdfArrays);
  b = (b + 15) & ~size_t(15);
  if (Q > 0) b += ((2 * ((size_t)n + Q) + qss_scratch_doubles(Q, K)) * 8 + 15) & ~size_t(15);
  return b;
}


template <typename LT>
__device__ inline void carve(Work<LT>& w, char* base, int N, int R, int Q = 0, int K = 0)
{
  const int n = N + 1;
  double* p = (double*)base;
  for (int j = 0; j < 6; j++) {
    w.zn[j] = p;
    p += n;
  }
  w.ewt = p; p += n;
  w.acor = p; p += n;
  w.y = p; p += n;
  w.tempv = p; p += n;
  w.ftemp = p; p += n;
  w.delta = p; p += n;
  w.src = p; p += n;
  w.atolv = p; p += n;
  w.Y = p; p += n;
  w.sc = p; p += n;
  w.g = p; p += n;
  w.wdot = p; p += n;
  w.ei = p; p += n;
  w.h1 = p; p += n;
  w.h2 = p; p += n;
  w.h3 = p; p += n;
  w.qd = p; p += R;
  char* q = (char*)p;
  if constexpr (sizeof(LT) == sizeof(double)) {
    w.J = (LT*)q;
    q += j_region_bytes<LT>(N);
    w.A = (LT*)q;
    w.jx = (double*)q; // shares the factor region
    w.jtmp = (double*)w.J;
  } else {
    w.jx = (double*)q;
    q += jx_region_bytes<LT>(R);
    w.J = (LT*)q;
    w.jtmp = (double*)q; // FP64 Jacobian over the FP32 J and factor (8 n^2 <= both regions)
    q += j_region_bytes<LT>(N);
    w.A = (LT*)q;
  }
  w.piv = (int*)((char*)w.A + a_region_bytes<LT>(N, R));
  w.perm = w.piv + n;
  w.ba = (BdfArrays*)((char*)w.piv + ((8 * (size_t)n + 7) & ~size_t(7)));
  if (Q > 0) {
    double* t = (double*)(base + team_bytes<LT>(N, R));
    w.sc = t;
    t += n + Q;
    w.g = t;
    t += n + Q;
    w.qco = t;
  }
}


// team-shared scratch for the pointwise kernels: per cell
//   sc[N+1], g[N+1], wdot[N+1], h[5][N+1], qd[R], then for the Jacobian
//   jx[4R], J[(N+1)^2]
__host__ __device__ inline size_t point_doubles(int N, int R, bool jac)
{
  const int n = N + 1;
  return (size_t)8 * n + R + (jac ? 4 * (size_t)R + (size_t)n * n : 0);
}

// the pointwise rate kernels' QSS tail: sc and g/RT over all n + Q slots,
// then the QSS solve's scratch
__host__ __device__ inline size_t point_qss_doubles(int N, int Q, int K)
{
  return Q > 0 ? 2 * ((size_t)N + 1 + Q) + qss_scratch_doubles(Q, K) : 0;
}
} // namespace ppb
