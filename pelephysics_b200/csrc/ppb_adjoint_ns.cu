// Discrete adjoint / tangent-linear kernels of the BDF integration for one
// species count (compiled once per mechanism size with -DPPB_NS=<N>).
//
// One warp integrates one cell at a time, pulling cells from a work queue.
// Adjoint: the forward integration saves a checkpoint of the whole integrator
// state (scalars, Nordsieck history, Jacobian, Newton-matrix factor) at the
// start of every segment of `seg_steps` accepted steps, recording each
// segment's operations on the warp's tape; the reverse sweep then walks the
// segments from last to first, restoring the segment's checkpoint and
// recomputing it (bit for bit: the same code path runs on the same state) to
// rebuild its tape, and applies the transposed operations in reverse order.
// Tangent: each segment's tape is swept forward right after it is recorded.
#include "ppb_adjoint.cuh"
#include "ppb_engine.h"
#include "ppb_work.cuh"

#ifndef PPB_NS
#error "compile with -DPPB_NS=<number of species>"
#endif

namespace ppb {

// checkpoint layout: [BdfScalars | nstloc][zn 6n][ewt n][J n*n][A n*n LT][piv n]
template <typename LT>
__host__ __device__ inline size_t cp_head_bytes()
{
  return (sizeof(BdfScalars) + 16 + 15) & ~size_t(15);
}

template <typename LT>
__host__ __device__ inline size_t cp_bytes(int N)
{
  const size_t n = N + 1;
  const size_t b = cp_head_bytes<LT>() + 8 * (7 * n + n * n) + sizeof(LT) * n * n + 4 * n;
  return (b + 15) & ~size_t(15);
}

template <int NS, typename LT, typename B>
__device__ void save_cp(const Team<32>& tm, char* dst, const B& bdf, const Work<LT>& w, int nstloc)
{
  constexpr int n = NS + 1;
  if (tm.lane == 0) {
    *reinterpret_cast<BdfScalars*>(dst) = bdf.s;
    *reinterpret_cast<int*>(dst + sizeof(BdfScalars)) = nstloc;
  }
  double* z = reinterpret_cast<double*>(dst + cp_head_bytes<LT>());
  for (int j = 0; j < 6; j++)
    for (int i = tm.lane; i < n; i += 32) z[j * n + i] = w.zn[j][i];
  for (int i = tm.lane; i < n; i += 32) z[6 * n + i] = w.ewt[i];
  double* J = z + 7 * n;
  for (int i = tm.lane; i < n * n; i += 32) J[i] = w.J[i];
  LT* A = reinterpret_cast<LT*>(J + n * n);
  for (int i = tm.lane; i < n * n; i += 32) A[i] = w.A[i];
  int* piv = reinterpret_cast<int*>(A + n * n);
  for (int i = tm.lane; i < n; i += 32) piv[i] = w.piv[i];
  tm.sync();
}

template <int NS, typename LT, typename B>
__device__ void restore_cp(const Team<32>& tm, const char* src, B& bdf, Work<LT>& w, int& nstloc)
{
  constexpr int n = NS + 1;
  bdf.s = *reinterpret_cast<const BdfScalars*>(src);
  nstloc = *reinterpret_cast<const int*>(src + sizeof(BdfScalars));
  const double* z = reinterpret_cast<const double*>(src + cp_head_bytes<LT>());
  for (int j = 0; j < 6; j++)
    for (int i = tm.lane; i < n; i += 32) w.zn[j][i] = z[j * n + i];
  for (int i = tm.lane; i < n; i += 32) w.ewt[i] = z[6 * n + i];
  const double* J = z + 7 * n;
  for (int i = tm.lane; i < n * n; i += 32) w.J[i] = J[i];
  const LT* A = reinterpret_cast<const LT*>(J + n * n);
  for (int i = tm.lane; i < n * n; i += 32) w.A[i] = A[i];
  const int* piv = reinterpret_cast<const int*>(A + n * n);
  for (int i = tm.lane; i < n; i += 32) w.piv[i] = piv[i];
  tm.sync();
}

template <int NS, typename LT, int MODE>
__device__ void adjoint_cell(const Team<32>& tm, const DevMech& M, const Options& o, Work<LT>& w, AdjWork& a,
                             const AdjBatch& b, const AdjLayout& L, char* cpb, TapeRec* tape, double* ys, int c,
                             double dt)
{
  constexpr int n = NS + 1;
  constexpr int PER = (NS + 31) / 32;
  const double* y0 = b.y0 + (size_t)c * n;
  for (int i = tm.lane; i < n; i += 32) {
    w.zn[0][i] = y0[i];
    w.y[i] = y0[i];
    w.src[i] = (i < NS && b.src) ? b.src[(size_t)c * NS + i] : 0.0;
    if (o.use_typ_vals) w.atolv[i] = b.atolv[i];
  }
  tm.sync();
  const CellIn cin{b.rhoe[c], b.rhoesrc ? b.rhoesrc[c] : 0.0};
  Bdf<NS, 32, LT, AdjRec<32>> bdf(tm, M, o, w, cin);
  bdf.rec.tape = tape;
  bdf.rec.ys = ys;
  bdf.rec.n = n;
  bdf.rec.seg_steps = L.seg_steps;
  bdf.rec.close_rec = L.close_rec;
  bdf.rec.close_y = L.close_y;
  bdf.rec.begin();
  AdjSweep<32, PER, LT> sw{tm, M, o, w, a, cin, n, o.max_order};
  int flag = bdf.start(dt);
  int nstloc = 0;
  bool done = false;
  double lamE = 0.0;
  int fst[7] = {0, 0, 0, 0, 0, 0, 0}; // counters of the forward integration
  const int R = M.nrxn;
  if (MODE != ADJ_TANGENT) {
    a.gacc = L.gw + (size_t)c * 3 * R; // this cell's parameter gradient
    for (int r = tm.lane; r < 3 * R; r += 32) a.gacc[r] = 0.0;
  }
  for (int i = tm.lane; i < 6 * n; i += 32) a.lam[i] = 0.0;
  for (int i = tm.lane; i < n; i += 32) a.pend[i] = 0.0;
  tm.sync();
  double* out_vec = b.lam_y0 ? b.lam_y0 + (size_t)c * n : nullptr;
  if (MODE == ADJ_TANGENT) {
    const double dE = b.dE ? b.dE[c] : 0.0;
    if (flag == ST_OK) {
      // z_0 = y0, z_1 = h0 f(0, y0)
      for (int i = tm.lane; i < n; i += 32) a.lam[i] = b.dy0 ? b.dy0[(size_t)c * n + i] : 0.0;
      tm.sync();
      sw.fwd_freset(0.0, bdf.rec.h0, y0, dE, b.dp);
      for (;;) {
        flag = bdf.advance(dt, nstloc, done);
        if (flag != ST_OK) break;
        flag = sw.forward(tape, bdf.rec.nrec, ys, dE, b.dp, a.tmp);
        if (flag != ST_OK || done) break;
        bdf.rec.begin();
      }
    }
    if (out_vec)
      for (int i = tm.lane; i < n; i += 32) out_vec[i] = (flag == ST_OK) ? a.tmp[i] : 0.0;
  } else {
    int ncp = 0, seg = 0;
    bool fwd = true;
    while (flag == ST_OK) {
      if (fwd) {
        if (ncp >= L.cap_cp) {
          flag = ST_ADJ_CAPACITY;
          break;
        }
        save_cp<NS, LT>(tm, cpb + (size_t)ncp * L.cp_stride, bdf, w, nstloc);
        ncp++;
      } else {
        restore_cp<NS, LT>(tm, cpb + (size_t)seg * L.cp_stride, bdf, w, nstloc);
      }
      bdf.rec.begin();
      flag = bdf.advance(dt, nstloc, done);
      if (flag != ST_OK) break;
      if (fwd) {
        if (!done) continue;
        fwd = false;
        seg = ncp - 1;
        fst[0] = bdf.s.nst;
        fst[1] = bdf.s.nfe;
        fst[2] = bdf.s.nje;
        fst[3] = bdf.s.nsetups;
        fst[4] = bdf.s.nni;
        fst[5] = bdf.s.netf;
        fst[6] = bdf.s.ncfn;
        if (b.y_out)
          for (int i = tm.lane; i < n; i += 32) b.y_out[(size_t)c * n + i] = w.y[i];
        tm.sync();
      }
      flag = sw.reverse(tape, bdf.rec.nrec, ys, b.lam_y + (size_t)c * n, lamE);
      if (flag != ST_OK) break;
      if (seg == 0) {
        sw.rev_freset(0.0, bdf.rec.h0, y0, lamE);
        break;
      }
      seg--;
    }
    if (out_vec)
      for (int i = tm.lane; i < n; i += 32) out_vec[i] = (flag == ST_OK) ? a.lam[i] : 0.0;
    if (b.lam_e && tm.lane == 0) b.lam_e[c] = (flag == ST_OK) ? lamE : 0.0;
    // the per-cell gradients are summed in cell order afterwards, so the
    // result does not depend on which warp ran which cell
    if (flag != ST_OK)
      for (int r = tm.lane; r < 3 * R; r += 32) a.gacc[r] = 0.0;
  }
  if (MODE == ADJ_TANGENT && b.y_out)
    for (int i = tm.lane; i < n; i += 32) b.y_out[(size_t)c * n + i] = (flag == ST_OK) ? w.y[i] : w.zn[0][i];
  if (MODE != ADJ_TANGENT && flag != ST_OK && b.y_out)
    for (int i = tm.lane; i < n; i += 32) b.y_out[(size_t)c * n + i] = w.zn[0][i];
  if (tm.lane == 0) {
    if (b.status) b.status[c] = flag;
    if (b.stats) {
      int* st = b.stats + (size_t)c * 7;
      if (MODE == ADJ_TANGENT) {
        fst[0] = bdf.s.nst;
        fst[1] = bdf.s.nfe;
        fst[2] = bdf.s.nje;
        fst[3] = bdf.s.nsetups;
        fst[4] = bdf.s.nni;
        fst[5] = bdf.s.netf;
        fst[6] = bdf.s.ncfn;
      }
      for (int q = 0; q < 7; q++) st[q] = fst[q];
    }
  }
  tm.sync();
}

template <int NS, typename LT, int MODE>
__global__ void __launch_bounds__(256) k_adjoint(DevMech M, Options o, AdjBatch b, AdjLayout L, double dt, int* queue)
{
  extern __shared__ __align__(16) char smem[];
  Team<32> tm;
  const int R = M.nrxn;
  const int warp = threadIdx.x / 32;
  const size_t gwarp = (size_t)blockIdx.x * (blockDim.x / 32) + warp;
  char* base = smem + (size_t)warp * L.warp_smem;
  Work<LT> w;
  carve<LT>(w, base, NS, R);
  AdjWork a;
  if (MODE == ADJ_TANGENT)
    carve_adj(a, base + team_bytes<LT>(NS, R), NS, R);
  else
    carve_adj_rev<LT>(a, base + team_bytes<LT>(NS, R), w, NS, R);
  char* cpb = L.cp + gwarp * (size_t)L.cap_cp * L.cp_stride;
  TapeRec* tape = reinterpret_cast<TapeRec*>(L.tape) + gwarp * (size_t)L.cap_rec;
  double* ys = L.ys + gwarp * (size_t)L.cap_y * (NS + 1);
  for (;;) {
    int c = 0;
    if (tm.lane == 0) c = atomicAdd(queue, 1);
    c = __shfl_sync(0xffffffffu, c, 0);
    if (c >= b.ncells) break;
    adjoint_cell<NS, LT, MODE>(tm, M, o, w, a, b, L, cpb, tape, ys, c, dt);
  }
}

// Pointwise: f, df/dy, df/dE and, for a weight vector v per cell,
// v^T df/dy, v^T df/dE and v^T df/dp (per cell) of the reactor RHS.
template <int NS>
__global__ void __launch_bounds__(128) k_rhs_exact(DevMech M, int rtype, double t, const double* y, const double* rhoe,
                                                   const double* rhoesrc, const double* src, const double* v,
                                                   double* f_out, double* J_out, double* fE_out, double* vy_out,
                                                   double* vE_out, double* vp_out, int ncells, size_t warp_smem)
{
  extern __shared__ __align__(16) char smem[];
  Team<32> tm;
  constexpr int n = NS + 1;
  constexpr int PER = (NS + 31) / 32;
  const int R = M.nrxn;
  const int warp = threadIdx.x / 32;
  const int c = blockIdx.x * (blockDim.x / 32) + warp;
  if (c >= ncells) return;
  char* base = smem + (size_t)warp * warp_smem;
  Work<double> w;
  carve<double>(w, base, NS, R);
  AdjWork a;
  carve_adj(a, base + team_bytes<double>(NS, R), NS, R);
  for (int i = tm.lane; i < n; i += 32) {
    a.ybuf[i] = y[(size_t)c * n + i];
    w.src[i] = (i < NS && src) ? src[(size_t)c * NS + i] : 0.0;
  }
  for (int r = tm.lane; r < 3 * R; r += 32) a.gacc[r] = 0.0;
  tm.sync();
  const AdjPoint pt = rhs_exact_jacobian<32, PER, double>(tm, M, rtype, t, a.ybuf, rhoe[c], rhoesrc ? rhoesrc[c] : 0.0,
                                                          w.src, w, a);
  for (int i = tm.lane; i < n; i += 32) {
    if (f_out) f_out[(size_t)c * n + i] = a.fy[i];
    if (fE_out) fE_out[(size_t)c * n + i] = a.fE[i];
  }
  if (J_out)
    for (int i = tm.lane; i < n * n; i += 32) J_out[(size_t)c * n * n + i] = a.Jc[i];
  if (v) {
    for (int i = tm.lane; i < n; i += 32) {
      a.mu[i] = v[(size_t)c * n + i];
      a.tmp[i] = 0.0;
    }
    tm.sync();
    jc_tmul_add(tm, n, a.Jc, a.mu, 1.0, a.tmp);
    double s = 0.0;
    for (int i = tm.lane; i < n; i += 32) {
      if (vy_out) vy_out[(size_t)c * n + i] = a.tmp[i];
      s += a.fE[i] * a.mu[i];
    }
    s = tm.sum(s);
    if (vE_out && tm.lane == 0) vE_out[c] = s;
    param_vjp(tm, M, pt, a, a.mu, 1.0);
    if (vp_out)
      for (int r = tm.lane; r < 3 * R; r += 32) vp_out[(size_t)c * 3 * R + r] = a.gacc[r];
  }
}

// out[p] (+)= sum over cells, in cell order, of gw[c][p]
static __global__ void k_sum_cells(const double* gw, int nc, int np, double* out, int accumulate)
{
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= np) return;
  double s = accumulate ? out[p] : 0.0;
  for (int c = 0; c < nc; c++) s += gw[(size_t)c * np + p];
  out[p] = s;
}

template <int NS, typename LT, int MODE>
static size_t adj_warp_smem(const DevMech& M)
{
  return team_bytes<LT>(NS, M.nrxn) +
         (MODE == ADJ_TANGENT ? adj_bytes(NS, M.nrxn) : adj_rev_bytes<LT>(NS, M.nrxn));
}

// Block size (warps) with the most resident warps per SM.
template <int NS, typename LT, int MODE>
static int plan_ns_t(const DevMech& M, AdjPlan* p)
{
  const size_t wb = adj_warp_smem<NS, LT, MODE>(M);
  auto kern = k_adjoint<NS, LT, MODE>;
  int dev = 0, nsm = 0, smem_max = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  cudaDeviceGetAttribute(&smem_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  int best_w = 0, best_blocks = 0, best_warps = 0;
  for (int wpb = 8; wpb >= 1; wpb--) {
    const size_t shm = wb * wpb;
    if (shm > (size_t)smem_max) continue;
    cudaError_t e = cudaFuncSetAttribute((const void*)kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm);
    if (e != cudaSuccess) return (int)e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)kern, wpb * 32, shm);
    if (e != cudaSuccess) return (int)e;
    if (per_sm * wpb > best_warps) {
      best_warps = per_sm * wpb;
      best_w = wpb;
      best_blocks = per_sm;
    }
  }
  if (best_warps < 1) return (int)cudaErrorInvalidConfiguration;
  p->wpb = best_w;
  p->blocks = nsm * best_blocks;
  p->warp_smem = wb;
  p->cp_stride = cp_bytes<LT>(NS);
  return 0;
}

template <int NS>
static int plan_ns(const DevMech& M, int mode, int lu_fp32, AdjPlan* p)
{
  if (mode == ADJ_TANGENT)
    return lu_fp32 ? plan_ns_t<NS, float, ADJ_TANGENT>(M, p) : plan_ns_t<NS, double, ADJ_TANGENT>(M, p);
  return lu_fp32 ? plan_ns_t<NS, float, ADJ_REVERSE>(M, p) : plan_ns_t<NS, double, ADJ_REVERSE>(M, p);
}

template <int NS>
static int launch_ns(const DevMech& M, const Options& o, int mode, int lu_fp32, const AdjPlan& p, const AdjBatch& b,
                     const AdjLayout& L, double dt, int* queue, double* grad, int accumulate, cudaStream_t st)
{
  if (b.ncells <= 0) return 0;
  cudaError_t e = cudaMemsetAsync(queue, 0, sizeof(int), st);
  if (e != cudaSuccess) return (int)e;
  const size_t shm = p.warp_smem * p.wpb;
  typedef void (*KT)(DevMech, Options, AdjBatch, AdjLayout, double, int*);
  KT kern = (mode == ADJ_TANGENT) ? (lu_fp32 ? (KT)k_adjoint<NS, float, ADJ_TANGENT> : (KT)k_adjoint<NS, double, ADJ_TANGENT>)
                                  : (lu_fp32 ? (KT)k_adjoint<NS, float, ADJ_REVERSE> : (KT)k_adjoint<NS, double, ADJ_REVERSE>);
  e = cudaFuncSetAttribute((const void*)kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm);
  if (e != cudaSuccess) return (int)e;
  kern<<<p.blocks, p.wpb * 32, shm, st>>>(M, o, b, L, dt, queue);
  e = cudaGetLastError();
  if (e != cudaSuccess) return (int)e;
  if (mode == ADJ_REVERSE && grad && L.gw) {
    const int np = 3 * M.nrxn;
    k_sum_cells<<<(np + 127) / 128, 128, 0, st>>>(L.gw, b.ncells, np, grad, accumulate);
    e = cudaGetLastError();
  }
  return (int)e;
}

template <int NS>
static int launch_rhs_exact_ns(const DevMech& M, int rtype, double t, const double* y, const double* rhoe,
                               const double* rhoesrc, const double* src, const double* v, double* f_out,
                               double* J_out, double* fE_out, double* vy_out, double* vE_out, double* vp_out,
                               int ncells, cudaStream_t st)
{
  if (ncells <= 0) return 0;
  const size_t wb = team_bytes<double>(NS, M.nrxn) + adj_bytes(NS, M.nrxn);
  int wpb = 4;
  while (wpb > 1 && wb * wpb > 200 * 1024) wpb--;
  const size_t shm = wb * wpb;
  cudaError_t e =
    cudaFuncSetAttribute((const void*)k_rhs_exact<NS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm);
  if (e != cudaSuccess) return (int)e;
  k_rhs_exact<NS><<<(ncells + wpb - 1) / wpb, wpb * 32, shm, st>>>(M, rtype, t, y, rhoe, rhoesrc, src, v, f_out,
                                                                   J_out, fE_out, vy_out, vE_out, vp_out, ncells, wb);
  return (int)cudaGetLastError();
}

#define PPB_CAT2(a, b) a##b
#define PPB_CAT(a, b) PPB_CAT2(a, b)
int PPB_CAT(plan_adjoint_, PPB_NS)(const DevMech& M, int mode, int lu_fp32, AdjPlan* p)
{
  return plan_ns<PPB_NS>(M, mode, lu_fp32, p);
}
int PPB_CAT(launch_adjoint_, PPB_NS)(const DevMech& M, const Options& o, int mode, int lu_fp32, const AdjPlan& p,
                                     const AdjBatch& b, const AdjLayout& L, double dt, int* queue, double* grad,
                                     int accumulate, cudaStream_t st)
{
  return launch_ns<PPB_NS>(M, o, mode, lu_fp32, p, b, L, dt, queue, grad, accumulate, st);
}
int PPB_CAT(launch_rhs_exact_, PPB_NS)(const DevMech& M, int rtype, double t, const double* y, const double* rhoe,
                                       const double* rhoesrc, const double* src, const double* v, double* f_out,
                                       double* J_out, double* fE_out, double* vy_out, double* vE_out,
                                       double* vp_out, int ncells, cudaStream_t st)
{
  return launch_rhs_exact_ns<PPB_NS>(M, rtype, t, y, rhoe, rhoesrc, src, v, f_out, J_out, fE_out, vy_out, vE_out,
                                     vp_out, ncells, st);
}
} // namespace ppb
