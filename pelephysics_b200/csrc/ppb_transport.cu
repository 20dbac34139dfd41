// Mixture-averaged transport coefficients (the reference's SimpleTransport,
// Source/Transport/Simple.H, ideal-gas EOS) for a box or a flat batch.
//
// Per cell the work is dominated by the binary-diffusion sums: for every
// species i, sum_{j != i} X_j exp(-fit(ln T)_ij), so the kernel is FP64-bound
// (HBM moves only about 3N doubles a cell).  A warp integrates one cell at a
// time, lanes owning species; the fits are symmetric (D_ij = D_ji, checked
// when the tables are uploaded), so each exp serves both row sums:
//   * N <= 32: the warp evaluates each of the N (N - 1) / 2 exps once, from a
//     pair list whose coefficients are contiguous, into the cell's matrix E
//     in shared memory; lane i then forms its row sum in the reference's
//     order j = 0..N-1, reading E column-wise (conflict-free);
//   * N <= 96: species blocks of 32.  For a block pair I < J, at rotation
//     d = 0..31 lane l evaluates E_ij for i = 32 I + l, j = 32 J + (l + d)
//     mod 32, adds X_j E_ij to its row and passes X_i E_ij by one shuffle to
//     the lane owning row j; a diagonal block needs rotations 1..16 only.
//     The coefficients are stored in that (pair of blocks, rotation, lane)
//     order, so every load is coalesced; padding and duplicate entries carry
//     a constant term of 1000 (exp = 0).  No matrix is kept; the row sums'
//     order differs from the reference's in the last bits.
// Tiles of Y, T and rho are staged through shared memory with loads along
// the box's x rows, and the outputs leave the same way.  Mixture sums (mean
// weight, viscosity, conductivity, bulk viscosity, thermal diffusion) are
// warp reductions.
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "mech/trans_LiDryer.h"
#include "mech/trans_dodecane_lu.h"
#include "mech/trans_drm19.h"
#include "mech/trans_heptane_lu_88sk.h"
#include "ppb_engine.h"
#include "ppb_mech.cuh"

namespace ppb {

const PPBTransTables* find_transport(const char* name)
{
  static const PPBTransTables* all[] = {&ppbt_LiDryer, &ppbt_drm19, &ppbt_dodecane_lu, &ppbt_heptane_lu_88sk};
  for (const PPBTransTables* t : all)
    if (!strcmp(t->name, name)) return t;
  return nullptr;
}

const double* find_srk(const char* name)
{
  if (!strcmp(name, "LiDryer")) return ppbt_LiDryer_srk;
  if (!strcmp(name, "drm19")) return ppbt_drm19_srk;
  if (!strcmp(name, "dodecane_lu")) return ppbt_dodecane_lu_srk;
  if (!strcmp(name, "heptane_lu_88sk")) return ppbt_heptane_lu_88sk_srk;
  return nullptr;
}

// Device copy of one mechanism's transport tables (one allocation).
struct DevTrans {
  int nsp, nlite, npairs;
  const double *wt, *iwt, *eps, *zrot, *cvms, *fitmu, *fitlam, *tilec, *pairc, *fittdrat;
  const int *nlin, *ktdif, *pairs; // pairs: i | j << 16, i < j
};

namespace {
std::mutex g_tr_mu;
std::vector<DeviceTransport*> g_trans;

constexpr int TR_THREADS = 256;
constexpr int TR_WARPS = TR_THREADS / 32;
constexpr double TR_PATM = 1.01325e+06;     // Source/PhysicsConstants.H:14
constexpr double TR_RU = 8.31446261815324e7; // Source/PhysicsConstants.H:11
constexpr double TR_PI = 3.14159265358979323846;

__device__ __forceinline__ long view_off(const BoxView& v, int i, int j, int k)
{
  return (long)(i - v.lo[0]) + (long)(j - v.lo[1]) * v.jstride + (long)(k - v.lo[2]) * v.kstride;
}

__device__ __forceinline__ double fit3(const double* c, double L0, double L1, double L2)
{
  return c[0] + c[1] * L0 + c[2] * L1 + c[3] * L2;
}

// shared memory of a block: Y, D, chi tiles [N][TT]; per warp X, Y [NP]
// (NP = N, or 32 NB zero-padded) and, with NB == 0, the cell's E matrix
// [N][ld], ld = N rounded up to odd
__host__ __device__ inline int e_ld(int N) { return N | 1; }
__host__ __device__ inline size_t tr_smem_doubles(int N, int tt, int nb)
{
  const size_t np = nb ? 32 * (size_t)nb : (size_t)N;
  return (size_t)3 * N * tt + (size_t)TR_WARPS * (2 * np + (nb == 0 ? (size_t)N * e_ld(N) : 0));
}

// TT cells per block tile; NB = 0: the E-matrix form (N <= 32), else the
// species-block form with NB blocks of 32
template <int TT, int NB>
__global__ void __launch_bounds__(TR_THREADS) k_transport(DevMech M, DevTrans t, TrBox b, int flags, long ncells)
{
  constexpr int TEAM = 32, TEAMS = TR_WARPS;
  extern __shared__ __align__(16) double trs[];
  __shared__ double sT[TT], srho[TT], smu[TT], sxi[TT], slam[TT];
  const int N = t.nsp, ld = e_ld(N);
  double* Yt = trs;
  double* Dt = Yt + (size_t)N * TT;
  double* Ct = Dt + (size_t)N * TT;
  const int team = threadIdx.x / TEAM;
  const int NP = NB ? 32 * NB : N;
  double* X = Ct + (size_t)N * TT + (size_t)team * (2 * NP + (NB == 0 ? (size_t)N * ld : 0));
  double* Yw = X + NP;
  double* E = Yw + NP;
  const Team<TEAM> tm;
  const bool get_xi = flags & 1, get_mu = flags & 2, get_lam = flags & 4, get_D = flags & 8, get_chi = flags & 16;
  const int nx = b.hi[0] - b.lo[0] + 1, ny = b.hi[1] - b.lo[1] + 1;
  const long ntiles = (ncells + TT - 1) / TT;
  for (long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const long c0 = tile * TT;
    const int nc = (int)min((long)TT, ncells - c0);
    // ---- stage the tile (consecutive cells run along x)
    for (int q = threadIdx.x; q < (N + 2) * TT; q += blockDim.x) {
      const int s = q / TT, cc = q % TT;
      if (cc >= nc) continue;
      const long c = c0 + cc;
      const int i = b.lo[0] + (int)(c % nx), j = b.lo[1] + (int)((c / nx) % ny), k = b.lo[2] + (int)(c / ((long)nx * ny));
      if (s < N) {
        Yt[(size_t)s * TT + cc] = b.Y.p[view_off(b.Y, i, j, k) + (long)s * b.Y.nstride];
      } else if (s == N) {
        sT[cc] = b.T.p[view_off(b.T, i, j, k)];
      } else {
        srho[cc] = b.rho.p ? b.rho.p[view_off(b.rho, i, j, k)] : 0.0;
      }
    }
    __syncthreads();
    for (int cc = team; cc < nc; cc += TEAMS) {
      const double T = sT[cc];
      const double L0 = log(T), L1 = L0 * L0, L2 = L0 * L1;
      // trace-amount floor, mean molecular weight, mole fractions
      double a = 0.0;
      for (int s = tm.lane; s < N; s += TEAM) a += Yt[(size_t)s * TT + cc];
      const double sum = tm.sum(a);
      a = 0.0;
      for (int s = tm.lane; s < N; s += TEAM) {
        const double y = Yt[(size_t)s * TT + cc];
        const double yl = y + 1.e-15 * (sum / N - y);
        Yw[s] = yl;
        a += yl * t.iwt[s];
      }
      const double wbar = 1.0 / tm.sum(a);
      for (int s = tm.lane; s < N; s += TEAM) X[s] = Yw[s] * wbar * t.iwt[s];
      for (int s = N + tm.lane; s < NP; s += TEAM) X[s] = Yw[s] = 0.0;
      tm.sync();
      double mu = 0.0, xi = 0.0, lam = 0.0;
      if (get_mu) {
        a = 0.0;
        double ax = 0.0;
        const double pi3_2 = pow(TR_PI, 1.5);
        for (int s = tm.lane; s < N; s += TEAM) {
          const double m = exp(fit3(t.fitmu + 4 * s, L0, L1, L2));
          a += X[s] * (m * m * m * m * m * m);
          if (get_xi) {
            // comp_pure_bulk (Simple.H:200-261)
            double xl = 0.0;
            const int nl = t.nlin[s];
            if (nl != 0) {
              const double cvk = cv_R(M, s, T) * t.cvms[s];
              const double cvkint = cvk * t.wt[s] / TR_RU - 1.50;
              const double cvkrot = nl == 1 ? 1.0 : 1.5;
              const double es = t.eps[s] / 298.0, et = t.eps[s] / T;
              const double Fnorm =
                1.0 + 0.50 * pi3_2 * sqrt(es) + (2.0 + .50 * TR_PI * TR_PI) * es + pi3_2 * sqrt(es) * es;
              const double FofT =
                1.0 + 0.50 * pi3_2 * sqrt(et) + (2.0 + .50 * TR_PI * TR_PI) * et + pi3_2 * sqrt(et) * et;
              xl = 0.250 * TR_PI * (cvkint / (cvkint + 1.50) * cvkint / (cvkint + 1.50)) * t.zrot[s] / cvkrot *
                   Fnorm / FofT * m;
            }
            ax += X[s] * sqrt(sqrt(xl * xl * xl));
          }
        }
        mu = cbrt(sqrt(tm.sum(a)));
        if (get_xi) {
          const double xs = tm.sum(ax);
          xi = cbrt(xs * xs * xs * xs);
        }
      }
      if (get_lam) {
        a = 0.0;
        for (int s = tm.lane; s < N; s += TEAM) a += X[s] * sqrt(sqrt(exp(fit3(t.fitlam + 4 * s, L0, L1, L2))));
        const double l = tm.sum(a);
        lam = l * l * l * l;
      }
      if (get_D && NB > 0) {
        // BinaryDiff, ideal gas (Simple.H:133-165), species-block form
        double t2[NB > 0 ? NB : 1];
#pragma unroll
        for (int I = 0; I < NB; I++) t2[I] = 0.0;
        const double* c = t.tilec + 4 * tm.lane;
#pragma unroll
        for (int I = 0; I < NB; I++) {
          const double Xi = X[I * 32 + tm.lane];
#pragma unroll
          for (int J = I; J < NB; J++) {
            const int d0 = I == J ? 1 : 0, d1 = I == J ? 16 : 31;
            for (int d = d0; d <= d1; d++, c += 128) {
              const double e = exp(-fit3(c, L0, L1, L2));
              t2[I] += X[J * 32 + ((tm.lane + d) & 31)] * e;
              t2[J] += __shfl_sync(0xffffffffu, Xi * e, (tm.lane - d) & 31);
            }
          }
        }
        a = 0.0;
        for (int s = tm.lane; s < N; s += TEAM) a += Yw[s];
        const double ysum = tm.sum(a);
        const double scale = TR_PATM / (TR_RU * T);
#pragma unroll
        for (int I = 0; I < NB; I++) {
          const int i = I * 32 + tm.lane;
          if (i < N) Dt[(size_t)i * TT + cc] = t.wt[i] * (ysum - Yw[i]) / t2[I] * scale;
        }
      }
      if (get_D && NB == 0) {
        // BinaryDiff, ideal gas (Simple.H:133-165), E-matrix form: one exp
        // per unordered pair, then each row sum in the reference's order
        for (int p = tm.lane; p < t.npairs; p += TEAM) {
          const int ij = __ldg(t.pairs + p);
          const int i = ij & 0xffff, j = ij >> 16;
          const double e = exp(-fit3(t.pairc + 4 * (size_t)p, L0, L1, L2));
          E[(size_t)i * ld + j] = e;
          E[(size_t)j * ld + i] = e;
        }
        tm.sync();
        const double scale = TR_PATM / (TR_RU * T);
        for (int s = tm.lane; s < N; s += TEAM) {
          double term1 = 0.0, term2 = 0.0;
          for (int jj = 0; jj < N; jj++) {
            if (jj == s) continue;
            term1 += Yw[jj];
            term2 += X[jj] * E[(size_t)jj * ld + s];
          }
          Dt[(size_t)s * TT + cc] = t.wt[s] * term1 / term2 * scale;
        }
      }
      if (get_chi) {
        for (int s = tm.lane; s < N; s += TEAM) Ct[(size_t)s * TT + cc] = 0.0;
        tm.sync();
        for (int n = 0; n < t.nlite; n++) {
          const int i = t.ktdif[n];
          a = 0.0;
          for (int jj = tm.lane; jj < N; jj += TEAM) {
            if (jj == i) continue;
            const double* c = t.fittdrat + 4 * (jj + N * n);
            a += X[jj] * (c[0] + T * (c[1] + T * (c[2] + T * c[3])));
          }
          const double ch = tm.sum(a);
          if (tm.lane == 0) Ct[(size_t)i * TT + cc] = ch * X[i];
        }
      }
      if (tm.lane == 0) {
        smu[cc] = mu;
        sxi[cc] = xi;
        slam[cc] = lam;
      }
      tm.sync(); // X, Y, E are reused by the team's next cell
    }
    __syncthreads();
    // ---- write the tile back
    const int nout = (get_D ? N : 0) + (get_chi ? N : 0);
    for (int q = threadIdx.x; q < (nout + 3) * TT; q += blockDim.x) {
      const int s = q / TT, cc = q % TT;
      if (cc >= nc) continue;
      const long c = c0 + cc;
      const int i = b.lo[0] + (int)(c % nx), j = b.lo[1] + (int)((c / nx) % ny), k = b.lo[2] + (int)(c / ((long)nx * ny));
      if (s < nout) {
        const bool isD = get_D && s < N;
        const int sp = isD ? s : s - (get_D ? N : 0);
        const BoxView& v = isD ? b.D : b.chi;
        v.p[view_off(v, i, j, k) + (long)sp * v.nstride] = (isD ? Dt : Ct)[(size_t)sp * TT + cc];
      } else {
        const int w = s - nout;
        const BoxView& v = w == 0 ? b.mu : (w == 1 ? b.xi : b.lam);
        if (v.p) v.p[view_off(v, i, j, k)] = (w == 0 ? smu : (w == 1 ? sxi : slam))[cc];
      }
    }
    __syncthreads();
  }
}

int upload_transport(const PPBTransTables* t, DeviceTransport* out)
{
  const int N = t->nsp, L = t->nlite;
  std::vector<double> d;
  auto put = [&](const double* p, size_t n) {
    const size_t o = d.size();
    d.insert(d.end(), p, p + n);
    return o;
  };
  std::vector<double> iwt(N);
  for (int i = 0; i < N; i++) iwt[i] = 1.0 / t->wt[i];
  // unordered pairs i < j with their coefficients, contiguous; the fits
  // must be symmetric (D_ij = D_ji) for one exp to serve both sums
  std::vector<double> pc;
  std::vector<int> pr;
  for (int i = 0; i < N; i++)
    for (int j = i + 1; j < N; j++) {
      for (int q = 0; q < 4; q++) {
        const double a = t->fitdbin[4 * (i + N * j) + q];
        if (a != t->fitdbin[4 * (j + N * i) + q]) return (int)cudaErrorInvalidValue;
        pc.push_back(a);
      }
      pr.push_back(i | (j << 16));
    }
  // species-block form: per block pair I <= J, rotation d, lane l the
  // coefficients of (32 I + l, 32 J + (l + d) mod 32); padding species and
  // the duplicate half of rotation 16 of a diagonal block get exp = 0
  std::vector<double> tc;
  const int NB = (N + 31) / 32;
  for (int I = 0; I < NB; I++)
    for (int J = I; J < NB; J++)
      for (int dd = (I == J ? 1 : 0); dd <= (I == J ? 16 : 31); dd++)
        for (int l = 0; l < 32; l++) {
          const int i = 32 * I + l, j = 32 * J + ((l + dd) & 31);
          const bool ok = i < N && j < N && !(I == J && dd == 16 && l >= 16);
          for (int q = 0; q < 4; q++) tc.push_back(ok ? t->fitdbin[4 * (i + N * j) + q] : (q == 0 ? 1000.0 : 0.0));
        }
  const size_t o_wt = put(t->wt, N), o_iwt = put(iwt.data(), N), o_eps = put(t->eps, N), o_zrot = put(t->zrot, N),
               o_cvms = put(t->cvms, N), o_mu = put(t->fitmu, 4 * N), o_lam = put(t->fitlam, 4 * N),
               o_full = put(tc.data(), tc.size()), o_db = put(pc.data(), pc.size()),
               o_td = put(t->fittdrat, (size_t)4 * N * L);
  const size_t nd = d.size();
  std::vector<int> ii(t->nlin, t->nlin + N);
  ii.insert(ii.end(), t->ktdif, t->ktdif + L);
  ii.insert(ii.end(), pr.begin(), pr.end());
  void* blob = nullptr;
  cudaError_t e = cudaMalloc(&blob, nd * 8 + ii.size() * 4);
  if (e != cudaSuccess) return (int)e;
  e = cudaMemcpy(blob, d.data(), nd * 8, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy((char*)blob + nd * 8, ii.data(), ii.size() * 4, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    cudaFree(blob);
    return (int)e;
  }
  const double* db = (const double*)blob;
  const int* ib = (const int*)((char*)blob + nd * 8);
  auto* dt = new DevTrans{N, L, (int)pr.size(), db + o_wt, db + o_iwt, db + o_eps, db + o_zrot, db + o_cvms,
                          db + o_mu, db + o_lam, db + o_full, db + o_db, db + o_td, ib, ib + N, ib + N + L};
  out->host = t;
  cudaGetDevice(&out->device);
  out->blob = blob;
  out->dt = dt;
  return 0;
}

} // namespace

int device_transport(const PPBTransTables* t, DeviceTransport** out)
{
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return (int)e;
  std::lock_guard<std::mutex> lk(g_tr_mu);
  for (auto* m : g_trans) {
    if (m->host == t && m->device == dev) {
      *out = m;
      return 0;
    }
  }
  auto* m = new DeviceTransport();
  int r = upload_transport(t, m);
  if (r) {
    delete m;
    return r;
  }
  g_trans.push_back(m);
  *out = m;
  return 0;
}

template <int TT, int NB>
static int launch_transport_t(const DevMech& M, const DevTrans& t, int flags, const TrBox& b, long ncells,
                              cudaStream_t st)
{
  auto kern = k_transport<TT, NB>;
  const size_t shm = tr_smem_doubles(t.nsp, TT, NB) * 8;
  cudaError_t e = cudaFuncSetAttribute((const void*)kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm);
  if (e != cudaSuccess) return (int)e;
  int dev = 0, nsm = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)kern, TR_THREADS, shm);
  if (e != cudaSuccess) return (int)e;
  if (per_sm < 1) return (int)cudaErrorInvalidConfiguration;
  const long ntiles = (ncells + TT - 1) / TT;
  long grid = (long)nsm * per_sm;
  if (grid > ntiles) grid = ntiles;
  kern<<<(int)grid, TR_THREADS, shm, st>>>(M, t, b, flags, ncells);
  return (int)cudaGetLastError();
}

int launch_transport(const DeviceMechanism& m, const DeviceTransport& tr, int flags, const TrBox& b,
                     cudaStream_t st)
{
  const DevTrans& t = *tr.dt;
  long ncells = 1;
  for (int d = 0; d < 3; d++) ncells *= (long)(b.hi[d] - b.lo[d] + 1);
  if (ncells <= 0) return 0;
  if (t.nsp <= 32) return launch_transport_t<32, 0>(*m.dm, t, flags, b, ncells, st);
  if (t.nsp <= 64) return launch_transport_t<32, 2>(*m.dm, t, flags, b, ncells, st);
  if (t.nsp <= 96) return launch_transport_t<16, 3>(*m.dm, t, flags, b, ncells, st);
  return (int)cudaErrorNotSupported;
}

} // namespace ppb
