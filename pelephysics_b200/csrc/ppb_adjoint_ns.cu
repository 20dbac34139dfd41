// Discrete adjoint / tangent-linear kernels of the BDF integration for one
// species count (compiled once per mechanism size with -DPPB_NS=<N>).
//
// Adjoint (batched over the cells, segment by segment):
//   1. k_adj_seg (forward): one warp per cell integrates from y0, saving a
//      checkpoint of the whole integrator state (scalars, Nordsieck history,
//      error weights, Jacobian, Newton-matrix factor) at the start of every
//      segment of seg_steps accepted steps into a shared pool, and recording
//      each segment's operations on the cell's tape (the last one stays);
//   2. for each segment s, last first: k_adj_seg (replay) restores every
//      cell's checkpoint s and recomputes the segment through the same code
//      (bit for bit, checked against checkpoint s+1) to rebuild its tape;
//      k_adj_items evaluates, for every point of every cell's segment at
//      once, the exact Jacobian, df/dE, the rate derivatives and the FP64
//      factor of (I - gamma Jc)^T; k_adj_sweep applies the transposed
//      operations in reverse order with those stored factors.
// Tangent (k_adj_seg, tangent mode): each segment's tape (per warp) is swept
// forward right after it is recorded, one warp per cell.  The adjoint's
// forward run, its recomputations and the tangent all integrate through the
// one call site of the integrator in k_adj_seg: two kernels holding their own
// inlined copies of the integrator may contract multiply-adds differently,
// and the stiff cells' step sequences then part in the last bit.
#include <algorithm>
#include <vector>

#include "ppb_adjoint.cuh"
#include "ppb_engine.h"
#include "ppb_work.cuh"

#ifndef PPB_NS
#error "compile with -DPPB_NS=<number of species>"
#endif

namespace ppb {

// checkpoint layout: [BdfScalars | BdfArrays | CpTail][zn 6n][ewt n][J n*n][A n*n LT][piv n]
// The tail: the step count of the call at the checkpoint and where the
// compact copy of the segment that starts there lies (toff < 0: none).
struct CpTail {
  int nstloc, nrec, ny, pad;
  long long toff;
};

template <typename LT>
__host__ __device__ inline size_t cp_head_bytes()
{
  return (sizeof(BdfScalars) + sizeof(BdfArrays) + sizeof(CpTail) + 15) & ~size_t(15);
}

template <typename LT>
__host__ __device__ inline size_t cp_bytes(int N)
{
  const size_t n = N + 1;
  const size_t b = cp_head_bytes<LT>() + 8 * (7 * n + n * n) + sizeof(LT) * n * n + 4 * n;
  return (b + 15) & ~size_t(15);
}

__device__ __forceinline__ CpTail* cp_tail(char* cp)
{
  return reinterpret_cast<CpTail*>(cp + sizeof(BdfScalars) + sizeof(BdfArrays));
}
__device__ __forceinline__ const CpTail* cp_tail(const char* cp)
{
  return reinterpret_cast<const CpTail*>(cp + sizeof(BdfScalars) + sizeof(BdfArrays));
}

// Bytes of the compact copy of a segment: its records, then the states and
// their (t, gamma), each part 16-byte aligned.
__host__ __device__ inline size_t seg_copy_parts(int nrec, int ny, int n, size_t* ys_off, size_t* yi_off)
{
  const size_t tb = (size_t)nrec * sizeof(TapeRec);
  const size_t yb = ((size_t)ny * n * 8 + 15) & ~size_t(15);
  const size_t ib = ((size_t)ny * 16 + 15) & ~size_t(15);
  *ys_off = tb;
  *yi_off = tb + yb;
  return tb + yb + ib;
}

// The tape of cell c's current segment: its compact copy, or the cell's own
// recording area.
struct SegTape {
  const TapeRec* tape;
  const double* ys;
  const double* yinfo;
};
__device__ __forceinline__ SegTape seg_tape(const AdjCells& C, int c, int n)
{
  const long long to = C.toff ? C.toff[c] : -1;
  if (to >= 0) {
    size_t yo, io;
    seg_copy_parts(C.nrec[c], C.ny[c], n, &yo, &io);
    const char* p = C.tpool + to;
    return {reinterpret_cast<const TapeRec*>(p), reinterpret_cast<const double*>(p + yo),
            reinterpret_cast<const double*>(p + io)};
  }
  return {reinterpret_cast<const TapeRec*>(C.tape) + (size_t)c * C.cap_rec, C.ys + (size_t)c * C.cap_y * n,
          C.yinfo + (size_t)c * C.cap_y * 2};
}

template <int NS, typename LT, typename B>
__device__ __noinline__ void save_cp(const Team<32>& tm, char* dst, const B& bdf, const Work<LT>& w, int nstloc)
{
  constexpr int n = NS + 1;
  if (tm.lane == 0) {
    *reinterpret_cast<BdfScalars*>(dst) = bdf.s;
    *reinterpret_cast<BdfArrays*>(dst + sizeof(BdfScalars)) = bdf.ar;
    *cp_tail(dst) = CpTail{nstloc, 0, 0, 0, -1};
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
__device__ __noinline__ void restore_cp(const Team<32>& tm, const char* src, B& bdf, Work<LT>& w, int& nstloc)
{
  constexpr int n = NS + 1;
  bdf.s = *reinterpret_cast<const BdfScalars*>(src);
  {
    const double* a = reinterpret_cast<const double*>(src + sizeof(BdfScalars));
    for (int i = tm.lane; i < (int)(sizeof(BdfArrays) / sizeof(double)); i += 32)
      reinterpret_cast<double*>(&bdf.ar)[i] = a[i];
  }
  nstloc = cp_tail(src)->nstloc;
  const double* z = reinterpret_cast<const double*>(src + cp_head_bytes<LT>());
  for (int j = 0; j < 6; j++)
    for (int i = tm.lane; i < n; i += 32) w.zn[j][i] = z[j * n + i];
  for (int i = tm.lane; i < n; i += 32) w.ewt[i] = z[6 * n + i];
  const double* J = z + 7 * n;
  for (int i = tm.lane; i < n * n; i += 32) w.J[i] = (LT)J[i];
  const LT* A = reinterpret_cast<const LT*>(J + n * n);
  for (int i = tm.lane; i < n * n; i += 32) w.A[i] = A[i];
  const int* piv = reinterpret_cast<const int*>(A + n * n);
  for (int i = tm.lane; i < n; i += 32) w.piv[i] = piv[i];
  tm.sync();
  perm_from_piv(tm, w.piv, w.perm, n);
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
    param_vjp(tm, M, pt, a, w.qd, a.mu, 1.0);
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

// Copy a just-recorded segment (records, states, their (t, gamma)) into the
// next free bytes of the tape pool and note where in its checkpoint's tail;
// when the pool is full the segment is recomputed in the reverse sweep.
static __device__ __noinline__ void copy_segment(const Team<32>& tm, const AdjCells& C, char* cp, const TapeRec* tape,
                                                 const double* ys, const double* yinfo, int nrec, int ny, int n)
{
  size_t yo, io;
  const size_t bytes = seg_copy_parts(nrec, ny, n, &yo, &io);
  unsigned long long off = 0;
  if (tm.lane == 0) off = atomicAdd(C.tpool_next, (unsigned long long)bytes);
  off = __shfl_sync(0xffffffffu, off, 0);
  const bool fits = off + bytes <= C.tpool_bytes;
  __syncwarp(); // the records (lane 0) and states (all lanes) are visible
  if (fits) {
    char* p = C.tpool + off;
    const int4* ts = reinterpret_cast<const int4*>(tape);
    int4* td = reinterpret_cast<int4*>(p);
    for (int i = tm.lane; i < nrec * (int)(sizeof(TapeRec) / 16); i += 32) td[i] = ts[i];
    double* yd = reinterpret_cast<double*>(p + yo);
    for (int i = tm.lane; i < ny * n; i += 32) yd[i] = ys[i];
    double* id = reinterpret_cast<double*>(p + io);
    for (int i = tm.lane; i < 2 * ny; i += 32) id[i] = yinfo[i];
  }
  if (tm.lane == 0) {
    CpTail* tl = cp_tail(cp);
    tl->nrec = nrec;
    tl->ny = ny;
    tl->toff = fits ? (long long)off : -1;
  }
  __syncwarp();
}

// ---------------------------------------------------------------- batched
// The modes of k_adj_seg.
enum : int { SEG_FORWARD = 0, SEG_REPLAY = 1, SEG_TANGENT = 2 };

// SEG_FORWARD: every cell from its initial state, a checkpoint at the start
// of each segment, the last segment's tape left in place (tapes per cell).
// SEG_REPLAY: recomputation of segment seg of every cell that has an earlier
// segment; it must end where the forward run did (checked against the next
// checkpoint).
// SEG_TANGENT: every cell from its initial state, each segment's tape (per
// warp) swept forward by the tangent-linear model as soon as it is recorded;
// dy(t_end) goes to b.lam_y0.  Needs the adjoint workspace after the
// integrator's in each warp's shared memory.
// All modes share the one call site of start() and of advance(), so every
// mode integrates with the same compiled arithmetic and their trajectories
// agree bit for bit.
template <int NS, typename LT>
__global__ void __launch_bounds__(512, 1) k_adj_seg(const __grid_constant__ DevMech M, const __grid_constant__ Options o,
                                                 const __grid_constant__ AdjBatch b, const __grid_constant__ AdjCells C,
                                                 double dt, int* queue, int seg, int mode, size_t warp_smem)
{
  extern __shared__ __align__(16) char smem[];
  Team<32> tm;
  constexpr int n = NS + 1;
  const int R = M.nrxn;
  const int warp = threadIdx.x / 32;
  const bool replay = (mode == SEG_REPLAY);
  const bool tangent = (mode == SEG_TANGENT);
  const size_t gwarp = (size_t)blockIdx.x * (blockDim.x / 32) + warp;
  char* base = smem + (size_t)warp * warp_smem;
  Work<LT> w;
  carve<LT>(w, base, NS, R);
  AdjWork a;
  if (tangent) carve_adj(a, base + team_bytes<LT>(NS, R), NS, R);
  __shared__ int rv[3];
  w.rv = rendezvous_init(rv, blockDim.x / 32, o.rendezvous);
  for (;;) {
    int c = 0;
    if (tm.lane == 0) c = atomicAdd(queue, 1);
    c = __shfl_sync(0xffffffffu, c, 0);
    if (c >= b.ncells) break;
    if (replay) {
      // cells without a segment seg are idle; for a cell whose last segment
      // is seg, the forward run left the tape (and its counts) in place
      const int ns = C.nseg[c];
      if (seg >= ns - 1) continue;
      // a segment the forward run copied needs no recomputation
      const CpTail* tl = cp_tail(C.cp_pool + (size_t)C.cp_idx[(size_t)c * C.max_seg + seg] * C.cp_stride);
      if (tl->toff >= 0) {
        if (tm.lane == 0) {
          C.nrec[c] = tl->nrec;
          C.ny[c] = tl->ny;
          C.toff[c] = tl->toff;
        }
        continue;
      }
    }
    const double* y0 = b.y0 + (size_t)c * n;
    for (int i = tm.lane; i < n; i += 32) {
      w.src[i] = (i < NS && b.src) ? b.src[(size_t)c * NS + i] : 0.0;
      if (o.use_typ_vals) w.atolv[i] = b.atolv[i];
      if (!replay) {
        w.zn[0][i] = y0[i];
        w.y[i] = y0[i];
      }
    }
    tm.sync();
    const CellIn cin{b.rhoe[c], b.rhoesrc ? b.rhoesrc[c] : 0.0};
    Bdf<NS, 32, LT, AdjRec<32>> bdf(tm, M, o, w, cin);
    const size_t slot_t = tangent ? gwarp : (size_t)c; // the tape's owner
    TapeRec* tape = reinterpret_cast<TapeRec*>(C.tape) + slot_t * C.cap_rec;
    double* ys = C.ys + slot_t * C.cap_y * n;
    bdf.rec.tape = tape;
    bdf.rec.ys = ys;
    bdf.rec.yinfo = (tangent || !C.yinfo) ? nullptr : C.yinfo + (size_t)c * C.cap_y * 2;
    bdf.rec.n = n;
    bdf.rec.seg_steps = C.seg_steps;
    bdf.rec.close_rec = C.close_rec;
    bdf.rec.close_y = C.close_y;
    bdf.rec.begin();
    AdjSweep<32, (NS + 31) / 32, LT> sw{tm, M, o, w, a, cin, n, o.max_order};
    const double dE = (tangent && b.dE) ? b.dE[c] : 0.0;
    int nstloc = 0, ncp = 0, flag = ST_OK;
    bool done = false;
    int* cpi = C.cp_idx + (size_t)c * C.max_seg;
    if (!replay) {
      flag = bdf.start(dt);
      if (tangent) {
        for (int i = tm.lane; i < 6 * n; i += 32) a.lam[i] = 0.0;
        for (int i = tm.lane; i < n; i += 32) a.pend[i] = 0.0;
        tm.sync();
        if (flag == ST_OK) {
          // z_0 = y0, z_1 = h0 f(0, y0)
          for (int i = tm.lane; i < n; i += 32) a.lam[i] = b.dy0 ? b.dy0[(size_t)c * n + i] : 0.0;
          tm.sync();
          sw.fwd_freset(0.0, bdf.rec.h0, y0, dE, b.dp);
        }
      } else {
        for (int i = tm.lane; i < 7 * n; i += 32) C.lam[(size_t)c * 7 * n + i] = 0.0;
        for (int r = tm.lane; r < 3 * R; r += 32) C.gw[(size_t)c * 3 * R + r] = 0.0;
        if (b.lam_y0)
          for (int i = tm.lane; i < n; i += 32) b.lam_y0[(size_t)c * n + i] = 0.0;
        if (tm.lane == 0) {
          C.lamE[c] = 0.0;
          if (b.lam_e) b.lam_e[c] = 0.0;
        }
      }
    }
    for (;;) {
      if (flag != ST_OK) break;
      if (mode == SEG_FORWARD) {
        if (ncp >= C.max_seg) {
          flag = ST_ADJ_CAPACITY;
          break;
        }
        int slot = 0;
        if (tm.lane == 0) slot = atomicAdd(C.pool_next, 1);
        slot = __shfl_sync(0xffffffffu, slot, 0);
        if (slot >= C.pool_cap) {
          flag = ST_ADJ_CAPACITY;
          break;
        }
        if (tm.lane == 0) cpi[ncp] = slot;
        save_cp<NS, LT>(tm, C.cp_pool + (size_t)slot * C.cp_stride, bdf, w, nstloc);
        ncp++;
      } else if (replay) {
        restore_cp<NS, LT>(tm, C.cp_pool + (size_t)cpi[seg] * C.cp_stride, bdf, w, nstloc);
      }
      bdf.rec.begin();
      flag = bdf.advance(dt, nstloc, done);
      if (tangent && flag == ST_OK) flag = sw.forward(tape, bdf.rec.nrec, ys, dE, b.dp, a.tmp);
      if (mode == SEG_FORWARD && flag == ST_OK && !done && C.tpool)
        copy_segment(tm, C, C.cp_pool + (size_t)cpi[ncp - 1] * C.cp_stride, tape, ys, bdf.rec.yinfo, bdf.rec.nrec,
                     bdf.rec.ny, n);
      if (flag != ST_OK || done || replay) break;
    }
    if (!replay) {
      if (b.y_out)
        for (int i = tm.lane; i < n; i += 32) b.y_out[(size_t)c * n + i] = (flag == ST_OK) ? w.y[i] : w.zn[0][i];
      if (tangent && b.lam_y0)
        for (int i = tm.lane; i < n; i += 32) b.lam_y0[(size_t)c * n + i] = (flag == ST_OK) ? a.tmp[i] : 0.0;
      if (tm.lane == 0) {
        if (b.status) b.status[c] = flag;
        if (b.stats) {
          int* st = b.stats + (size_t)c * 7;
          st[0] = bdf.s.nst;
          st[1] = bdf.s.nfe;
          st[2] = bdf.ar.nje;
          st[3] = bdf.ar.nsetups;
          st[4] = bdf.ar.nni;
          st[5] = bdf.ar.netf;
          st[6] = bdf.ar.ncfn;
        }
        if (!tangent) {
          C.nseg[c] = (flag == ST_OK) ? ncp : 0;
          C.h0[c] = bdf.rec.h0;
          C.nrec[c] = bdf.rec.nrec;
          C.ny[c] = bdf.rec.ny;
          if (C.toff) C.toff[c] = -1; // the last segment stays in the cell's own area
        }
      }
    } else {
      if (flag == ST_OK) {
        // the recomputed segment must end where the forward run did
        const BdfScalars* nx = reinterpret_cast<const BdfScalars*>(C.cp_pool + (size_t)cpi[seg + 1] * C.cp_stride);
        if (nx->tn != bdf.s.tn || nx->nst != bdf.s.nst || nx->h != bdf.s.h) flag = ST_ADJ_REPLAY;
      }
      if (tm.lane == 0) {
        if (flag != ST_OK) {
          if (b.status) b.status[c] = flag;
          C.nseg[c] = 0;
          C.nrec[c] = 0;
          C.ny[c] = 0;
        } else {
          C.nrec[c] = bdf.rec.nrec;
          C.ny[c] = bdf.rec.ny;
          if (C.toff) C.toff[c] = -1;
        }
      }
    }
    tm.sync();
  }
  rendezvous_leave(w.rv);
}

template <int NS, typename LT>
static size_t adj_warp_smem(const DevMech& M)
{
  return team_bytes<LT>(NS, M.nrxn) + adj_bytes(NS, M.nrxn);
}

// Block size (warps) with the most resident warps per SM.
template <int NS, typename LT>
static int plan_ns_t(const DevMech& M, AdjPlan* p)
{
  const size_t wb = adj_warp_smem<NS, LT>(M);
  auto kern = k_adj_seg<NS, LT>;
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
  // the reverse integration runs batched (launch_adjoint_batched)
  if (mode != ADJ_TANGENT) return (int)cudaErrorNotSupported;
  return lu_fp32 ? plan_ns_t<NS, float>(M, p) : plan_ns_t<NS, double>(M, p);
}

template <int NS>
static int launch_ns(const DevMech& M, const Options& o, int mode, int lu_fp32, const AdjPlan& p, const AdjBatch& b,
                     const AdjLayout& L, double dt, int* queue, double* grad, int accumulate, cudaStream_t st)
{
  if (b.ncells <= 0) return 0;
  if (mode != ADJ_TANGENT) return (int)cudaErrorNotSupported;
  cudaError_t e = cudaMemsetAsync(queue, 0, sizeof(int), st);
  if (e != cudaSuccess) return (int)e;
  const size_t shm = p.warp_smem * p.wpb;
  // per-warp tapes; no checkpoints
  AdjCells C{};
  C.tape = L.tape;
  C.cap_rec = L.cap_rec;
  C.close_rec = L.close_rec;
  C.ys = L.ys;
  C.cap_y = L.cap_y;
  C.close_y = L.close_y;
  C.seg_steps = L.seg_steps;
  // the warps spend whole segments in the tangent sweep between right-hand
  // sides, so a block rendezvous would only wait out its bound
  Options ot = o;
  ot.rendezvous = 0;
  typedef void (*KT)(DevMech, Options, AdjBatch, AdjCells, double, int*, int, int, size_t);
  KT kern = lu_fp32 ? (KT)k_adj_seg<NS, float> : (KT)k_adj_seg<NS, double>;
  e = cudaFuncSetAttribute((const void*)kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm);
  if (e != cudaSuccess) return (int)e;
  kern<<<p.blocks, p.wpb * 32, shm, st>>>(M, ot, b, C, dt, queue, 0, SEG_TANGENT, p.warp_smem);
  return (int)cudaGetLastError();
}

// Every differentiated point of items [i0, i1) of segment seg (item i of
// cell c is slot i - item_off[c]; at seg 0 the slot after the last is the
// initial state).
template <int NS>
__global__ void __launch_bounds__(256) k_adj_items(DevMech M, int rtype, AdjBatch b, AdjCells C, int seg, int c0,
                                                   int c1, int i0, int i1, size_t warp_smem)
{
  extern __shared__ __align__(16) char smem[];
  Team<32> tm;
  constexpr int n = NS + 1;
  constexpr int PER = (NS + 31) / 32;
  const int warp = threadIdx.x / 32;
  const int i = i0 + blockIdx.x * (blockDim.x / 32) + warp;
  if (i >= i1) return;
  // the cell owning item i: the last c in [c0, c1) with item_off[c] <= i
  int lo = c0, hi = c1 - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) / 2;
    if (C.item_off[mid] <= i) lo = mid;
    else hi = mid - 1;
  }
  const int c = lo;
  const int slot = i - C.item_off[c];
  const double* yg;
  double t, gamma;
  if (seg == 0 && slot == C.ny[c]) {
    yg = b.y0 + (size_t)c * n;
    t = 0.0;
    gamma = 0.0;
  } else {
    const SegTape sg = seg_tape(C, c, n);
    yg = sg.ys + (size_t)slot * n;
    t = sg.yinfo[2 * slot];
    gamma = sg.yinfo[2 * slot + 1];
  }
  const ItemLayout IL(NS, M.nrxn);
  eval_item<32, PER>(tm, M, rtype, t, gamma, yg, b.rhoe[c], b.rhoesrc ? b.rhoesrc[c] : 0.0,
                     b.src ? b.src + (size_t)c * NS : nullptr, smem + (size_t)warp * warp_smem,
                     C.items + (size_t)(i - i0) * IL.stride, IL);
}

// The reverse sweep of segment seg for cells [c0, c1), whose items start at
// global item index i0 in C.items.
template <int NS>
__global__ void __launch_bounds__(256) k_adj_sweep(DevMech M, Options o, AdjBatch b, AdjCells C, int seg, int c0,
                                                   int c1, int i0, size_t warp_smem)
{
  extern __shared__ __align__(16) char smem[];
  Team<32> tm;
  constexpr int n = NS + 1;
  const int R = M.nrxn;
  const int warp = threadIdx.x / 32;
  const int c = c0 + blockIdx.x * (blockDim.x / 32) + warp;
  if (c >= c1) return;
  if (seg >= C.nseg[c]) return;
  double* p = reinterpret_cast<double*>(smem + (size_t)warp * warp_smem);
  AdjWork a{};
  a.lam = p; p += 6 * n;
  a.pend = p; p += n;
  a.mu = p; p += n;
  a.v = p; p += n + 1;
  a.AT = p; p += (size_t)n * n;
  a.piv = reinterpret_cast<int*>(p);
  a.gacc = C.gw + (size_t)c * 3 * R;
  double* lg = C.lam + (size_t)c * 7 * n;
  for (int i = tm.lane; i < 7 * n; i += 32) a.lam[i] = lg[i]; // lam then pend
  double lamE = C.lamE[c];
  tm.sync();
  const ItemLayout IL(NS, R);
  const double* items = C.items + (size_t)(C.item_off[c] - i0) * IL.stride;
  const TapeRec* tape = seg_tape(C, c, n).tape;
  int flag = sweep_items<32>(tm, M, n, o.max_order, a, tape, C.nrec[c], items, IL, b.lam_y + (size_t)c * n, lamE);
  if (flag == ST_OK && seg == 0) {
    // z_0 = y0, z_1 = h0 f(0, y0)
    rev_item_freset<32>(tm, M, n, a, items + (size_t)C.ny[c] * IL.stride, IL, C.h0[c], lamE);
    if (b.lam_y0)
      for (int i = tm.lane; i < n; i += 32) b.lam_y0[(size_t)c * n + i] = a.lam[i];
    if (b.lam_e && tm.lane == 0) b.lam_e[c] = lamE;
  }
  if (flag != ST_OK) {
    for (int r = tm.lane; r < 3 * R; r += 32) a.gacc[r] = 0.0;
    if (tm.lane == 0) {
      if (b.status) b.status[c] = flag;
      C.nseg[c] = 0;
    }
  }
  tm.sync();
  for (int i = tm.lane; i < 7 * n; i += 32) lg[i] = a.lam[i];
  if (tm.lane == 0) C.lamE[c] = lamE;
}

// Block size (warps) with the most resident warps per SM for a kernel with
// wb bytes of shared memory per warp.
static int best_blocks(const void* kern, size_t wb, int max_wpb, int* wpb_out, int* per_sm_out)
{
  int dev = 0, smem_max = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&smem_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  int best_w = 0, best_b = 0, best = 0;
  for (int wpb = max_wpb; wpb >= 1; wpb--) {
    const size_t shm = wb * wpb;
    if (shm > (size_t)smem_max) continue;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm);
    if (e != cudaSuccess) return (int)e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, wpb * 32, shm);
    if (e != cudaSuccess) return (int)e;
    if (per_sm * wpb > best) {
      best = per_sm * wpb;
      best_w = wpb;
      best_b = per_sm;
    }
  }
  if (best < 1) return (int)cudaErrorInvalidConfiguration;
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(wb * best_w));
  *wpb_out = best_w;
  *per_sm_out = best_b;
  return 0;
}

template <int NS, typename LT>
static int batched_ns_t(const DevMech& M, const Options& o, const AdjBatch& b, AdjCells& C, double dt, int* queue,
                        double* grad, int accumulate, AdjGrow grow, void* ctx, cudaStream_t st)
{
  constexpr int n = NS + 1;
  const int R = M.nrxn, nc = b.ncells;
  if (nc <= 0) return 0;
  int dev = 0, nsm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  cudaError_t e;
  // launch shapes
  const size_t seg_wb = team_bytes<LT>(NS, R);
  int seg_w = 0, seg_b = 0, it_w = 0, it_b = 0, sw_w = 0, sw_b = 0;
  int err = best_blocks((const void*)k_adj_seg<NS, LT>, seg_wb, 16, &seg_w, &seg_b);
  if (err) return err;
  const size_t it_wb = item_bytes(NS, R);
  if ((err = best_blocks((const void*)k_adj_items<NS>, it_wb, 8, &it_w, &it_b))) return err;
  const size_t sw_wb = ((8 * (9 * (size_t)n + 1 + (size_t)n * n) + 4 * n) + 15) & ~size_t(15);
  if ((err = best_blocks((const void*)k_adj_sweep<NS>, sw_wb, 8, &sw_w, &sw_b))) return err;
  const int seg_grid = std::min(nsm * seg_b, (nc + seg_w - 1) / seg_w);
  // the recording kernel waits up to 1e6 SM clocks unless the caller set a
  // bound (drm19, 65536 cells, 16 warps: adjoint 519 ms at 1e6 against 579
  // at 3e5)
  Options os = o;
  if (o.rendezvous < 0) os.rendezvous = 1000000;
  const ItemLayout IL(NS, R);
  // forward with checkpoints
  if ((e = cudaMemsetAsync(C.pool_next, 0, sizeof(int), st)) || (e = cudaMemsetAsync(queue, 0, sizeof(int), st)))
    return (int)e;
  if (C.tpool && (e = cudaMemsetAsync(C.tpool_next, 0, sizeof(unsigned long long), st))) return (int)e;
  k_adj_seg<NS, LT><<<seg_grid, seg_w * 32, seg_wb * seg_w, st>>>(M, os, b, C, dt, queue, 0, SEG_FORWARD, seg_wb);
  if ((e = cudaGetLastError())) return (int)e;
  std::vector<int> nseg(nc), ny(nc), off(nc + 1);
  if ((e = cudaMemcpyAsync(nseg.data(), C.nseg, nc * sizeof(int), cudaMemcpyDeviceToHost, st)) ||
      (e = cudaStreamSynchronize(st)))
    return (int)e;
  int maxseg = 0;
  for (int c = 0; c < nc; c++) maxseg = std::max(maxseg, nseg[c]);
  for (int s = maxseg - 1; s >= 0; s--) {
    if ((e = cudaMemsetAsync(queue, 0, sizeof(int), st))) return (int)e;
    k_adj_seg<NS, LT><<<seg_grid, seg_w * 32, seg_wb * seg_w, st>>>(M, os, b, C, dt, queue, s, SEG_REPLAY, seg_wb);
    if ((e = cudaGetLastError())) return (int)e;
    if ((e = cudaMemcpyAsync(nseg.data(), C.nseg, nc * sizeof(int), cudaMemcpyDeviceToHost, st)) ||
        (e = cudaMemcpyAsync(ny.data(), C.ny, nc * sizeof(int), cudaMemcpyDeviceToHost, st)) ||
        (e = cudaStreamSynchronize(st)))
      return (int)e;
    long tot = 0;
    int most = 0;
    for (int c = 0; c < nc; c++) {
      off[c] = (int)tot;
      const int k = (s < nseg[c]) ? ny[c] + (s == 0 ? 1 : 0) : 0;
      most = std::max(most, k);
      tot += k;
    }
    off[nc] = (int)tot;
    if (tot == 0) continue;
    if (C.items_cap < most) {
      void* pi = C.items;
      if ((err = grow(ctx, &pi, (size_t)most * IL.stride * 8))) return err;
      C.items = (double*)pi;
      C.items_cap = most;
    }
    if ((e = cudaMemcpyAsync(C.item_off, off.data(), (nc + 1) * sizeof(int), cudaMemcpyHostToDevice, st)))
      return (int)e;
    // groups of cells whose items fit the buffer
    int c0 = 0;
    while (c0 < nc) {
      int c1 = c0;
      while (c1 < nc && (long)off[c1 + 1] - off[c0] <= C.items_cap) c1++;
      if (c1 == c0) c1 = c0 + 1;
      const int i0 = off[c0], i1 = off[c1];
      if (i1 > i0) {
        const int ni = i1 - i0;
        k_adj_items<NS><<<(ni + it_w - 1) / it_w, it_w * 32, it_wb * it_w, st>>>(M, o.reactor_type, b, C, s, c0, c1,
                                                                               i0, i1, it_wb);
        if ((e = cudaGetLastError())) return (int)e;
        k_adj_sweep<NS><<<(c1 - c0 + sw_w - 1) / sw_w, sw_w * 32, sw_wb * sw_w, st>>>(M, o, b, C, s, c0, c1, i0,
                                                                                   sw_wb);
        if ((e = cudaGetLastError())) return (int)e;
      }
      c0 = c1;
    }
  }
  if (grad) {
    const int np = 3 * R;
    k_sum_cells<<<(np + 127) / 128, 128, 0, st>>>(C.gw, nc, np, grad, accumulate);
    if ((e = cudaGetLastError())) return (int)e;
  }
  return 0;
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
int PPB_CAT(launch_adjoint_batched_, PPB_NS)(const DevMech& M, const Options& o, int lu_fp32, const AdjBatch& b,
                                             AdjCells& C, double dt, int* queue, double* grad, int accumulate,
                                             AdjGrow grow, void* ctx, cudaStream_t st)
{
  return lu_fp32 ? batched_ns_t<PPB_NS, float>(M, o, b, C, dt, queue, grad, accumulate, grow, ctx, st)
                 : batched_ns_t<PPB_NS, double>(M, o, b, C, dt, queue, grad, accumulate, grow, ctx, st);
}
size_t PPB_CAT(adj_cp_bytes_, PPB_NS)(int lu_fp32) { return lu_fp32 ? cp_bytes<float>(PPB_NS) : cp_bytes<double>(PPB_NS); }
int PPB_CAT(launch_rhs_exact_, PPB_NS)(const DevMech& M, int rtype, double t, const double* y, const double* rhoe,
                                       const double* rhoesrc, const double* src, const double* v, double* f_out,
                                       double* J_out, double* fE_out, double* vy_out, double* vE_out,
                                       double* vp_out, int ncells, cudaStream_t st)
{
  return launch_rhs_exact_ns<PPB_NS>(M, rtype, t, y, rhoe, rhoesrc, src, v, f_out, J_out, fE_out, vy_out, vE_out,
                                     vp_out, ncells, st);
}
} // namespace ppb
