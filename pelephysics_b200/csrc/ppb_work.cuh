// Shared-memory workspace layout of one team-integrated cell.
#pragma once
#include "ppb_bdf.cuh"

namespace ppb {
// ------------------------------------------------------------ workspace
// Newton-matrix region: the n x n factor, or the per-reaction factors of
// the warp-cooperative Jacobian evaluations (4 doubles per reaction; 5 in the
// adjoint's exact Jacobian), which use it while the matrix is not live,
// whichever is larger.
template <typename LT>
__host__ __device__ inline size_t a_region_bytes(int N, int R)
{
  const size_t n = N + 1;
  size_t a = n * n * sizeof(LT);
  const size_t jx = 40 * (size_t)R;
  if (jx > a) a = jx;
  return (a + 15) & ~size_t(15);
}

// pivots and row permutation (2n ints), then the coefficient arrays
template <typename LT>
__host__ __device__ inline size_t team_bytes(int N, int R)
{
  const int n = N + 1;
  size_t d = (size_t)n * n + 22 * (size_t)n + (size_t)R;
  size_t b = d * 8 + a_region_bytes<LT>(N, R) + ((8 * (size_t)n + 7) & ~size_t(7)) + sizeof(BdfArrays);
  return (b + 15) & ~size_t(15);
}


template <typename LT>
__device__ inline void carve(Work<LT>& w, char* base, int N, int R)
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
  w.J = p; p += (size_t)n * n;
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
  w.A = (LT*)p;
  w.piv = (int*)((char*)p + a_region_bytes<LT>(N, R));
  w.perm = w.piv + n;
  w.ba = (BdfArrays*)((char*)w.piv + ((8 * (size_t)n + 7) & ~size_t(7)));
}


// team-shared scratch for the pointwise kernels: per cell
//   sc[N+1], g[N+1], wdot[N+1], h[5][N+1], qd[R], then for the Jacobian
//   jx[4R], J[(N+1)^2]
__host__ __device__ inline size_t point_doubles(int N, int R, bool jac)
{
  const int n = N + 1;
  return (size_t)8 * n + R + (jac ? 4 * (size_t)R + (size_t)n * n : 0);
}
} // namespace ppb
