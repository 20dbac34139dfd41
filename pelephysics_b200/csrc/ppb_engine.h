// Host-side interface between the C-ABI layer and the CUDA kernels.
#pragma once
#include <cuda_runtime.h>

#include "mech/mech_tables.h"
#include "mech/trans_tables.h"
#include "ppb_erk_tables.h"

namespace ppb {
struct DevMech;
struct Options;

// A mechanism uploaded to one device.
struct DeviceMechanism {
  const PPBMechTables* host = nullptr;
  int device = -1;
  void* blob = nullptr; // one device allocation holding every table
  DevMech* dm = nullptr; // host copy of the device pointer struct
};

int upload_mechanism(const PPBMechTables* t, DeviceMechanism* out);
// Table image for caller-owned device memory: size, and packing into a host
// buffer with device pointers relocated to dev_base.
size_t packed_mechanism_bytes(const PPBMechTables* t);
int pack_mechanism(const PPBMechTables* t, char* buf, size_t cap, const void* dev_base, DevMech* out);
void free_mechanism(DeviceMechanism* m);
const PPBMechTables* find_mechanism(const char* name);

// Device-resident batch of cells, species-major (SoA): y[i * ld + c] for
// i < N+1, src[i * ld + c] for i < N, ld >= ncells.
struct Batch {
  double* y;
  double* src;
  const double* rhoe;
  const double* rhoesrc;
  const double* atolv; // N+1 absolute tolerances or nullptr
  const int* mask;     // per cell, -1 skips the cell; nullptr: all cells
  int* status;         // per cell integrator flag (may be nullptr)
  int* nfe;            // per cell RHS evaluations / RK steps (may be nullptr)
  int* stats;          // per cell [nsteps, nfe, nje, nsetups, nni, netf, ncfn] (may be nullptr)
  int ncells;
  int ld;
  const int* order;    // work-queue order of the cells (nullptr: index order)
};

enum Engine { ENGINE_PLAIN = 0, ENGINE_TUNED = 1 };
enum Method { METHOD_BDF = 0, METHOD_RK64 = 1, METHOD_ARK = 2 };

struct LaunchConfig {
  int engine = ENGINE_TUNED;
  int warps_per_block = 4;
  int lu_fp32 = 0;
  int persistent = 1; // work queue
  int team = 32;      // lanes per cell: 32; 16 for <= 21 species; 64 (33..64 species) or 128 (65..128): one
                      // multi-warp team per block
  int minb = 2;       // register budget: >= minb blocks of 256 threads per SM
  int rhsv = 0;       // right-hand side: 0 ideal gas, 1 the SRK e-reactor, 2 a QSS mechanism (the last two:
                      // warp teams, <= 128 registers, difference-quotient Jacobian)
  int rv = -1;        // rendezvous bound the autotuner picked, used when the option is -1 (-1: by block size)
};
// Resident cells per SM of the tuned kernel in configuration lc (0: the
// configuration does not fit or is not compiled).
int react_occupancy(const DeviceMechanism& m, int method, const LaunchConfig& lc);

// Integrate every cell of the batch over dt.  queue is a device int used by
// the persistent kernel (reset inside the call).  Returns a cudaError_t.
int launch_react(const DeviceMechanism& m, const Options& o, int method, const LaunchConfig& lc, Batch b,
                 double dt, int* queue, cudaStream_t st);

// Layout conversion kernels (HBM-bound): YCOrder AoS <-> species-major SoA.
int launch_aos_to_soa(const double* aos, int nc_aos, double* soa, int ld, int ncomp, int ncells, cudaStream_t st);
int launch_soa_to_aos(const double* soa, int ld, int ncomp, double* aos, int nc_aos, int ncells, cudaStream_t st);

// Pointwise kernels (AoS per cell), team = 1 or 32.
int launch_production_rate(const DeviceMechanism& m, const double* sc, const double* T, double* wdot, int ncells,
                           int team, cudaStream_t st);
int launch_ajacobian(const DeviceMechanism& m, const double* sc, const double* T, int consP, double* J, int ncells,
                     int team, cudaStream_t st);
int launch_t_from_energy(const DeviceMechanism& m, int eh, const double* e, const double* Y, double* T, int ncells,
                         int team, cudaStream_t st);
int launch_reactor_rhs(const DeviceMechanism& m, int reactor_type, double t, const double* y, const double* rhoe,
                       const double* rhoesrc, const double* src, double* ydot, int ncells, int team,
                       cudaStream_t st);

// Array4-style views (device memory) of one box.
struct BoxView {
  double* p;
  long jstride, kstride, nstride;
  int lo[3];
};
struct BoxViewI {
  int* p;
  long jstride, kstride, nstride;
  int lo[3];
};
struct BoxArgs {
  int lo[3], hi[3]; // box (inclusive)
  BoxView rY, rYsrc, T, rE, rEs, FC;
  BoxViewI mask;    // p == nullptr: every cell active
  const long* fcunt = nullptr; // unflatten: per-cell cost as the reference's FCunt (else the batch's nfe)
};
// box_flatten / box_unflatten; the batch's mask array (when not null)
// receives the Array4 mask values and must be writable device memory.
int launch_box_flatten(const DeviceMechanism& m, int rtype, int clean, const BoxArgs& a, Batch b, cudaStream_t st);
int launch_box_unflatten(const DeviceMechanism& m, int rtype, int clean, const BoxArgs& a, Batch b, double dt,
                         cudaStream_t st);

int launch_pyt2re(const DeviceMechanism& m, int eh, const double* P, const double* T, const double* Y, double* rho,
                  double* e, int ncells, cudaStream_t st);
// FP64 FMA throughput probe: returns GFLOP/s measured with CUDA events.
int probe_fp64_peak(double* gflops, cudaStream_t st);
int launch_energy_update(double* rX, const double* rX_src, double dt, int ncells, cudaStream_t st);

// Work-queue order by descending cost: order = cells sorted by cost (the
// previous call's per-cell RHS evaluations), ties in index order.  keys_tmp
// (n ints) and tmp (cost_order_tmp_bytes(n)) are scratch; iota holds 0..n-1.
size_t cost_order_tmp_bytes(int n);
int launch_cost_order(const int* cost, int* keys_tmp, const int* iota, int* order, void* tmp, size_t tmp_bytes,
                      int n, cudaStream_t st);
int launch_iota(int* a, int n, cudaStream_t st);

// Mixture-averaged transport (ppb_transport.cu).  A mechanism's transport
// tables uploaded to one device, and the views of one call: a box lo..hi
// (a flat batch is the box 0..ncells-1 x 0 x 0) with Y, D, chi holding N
// components nstride apart.  flags: 1 xi, 2 mu, 4 lam, 8 Ddiag, 16 chi.
struct DevTrans;
struct DeviceTransport {
  const PPBTransTables* host = nullptr;
  int device = -1;
  void* blob = nullptr;
  DevTrans* dt = nullptr;
};
struct TrBox {
  int lo[3], hi[3];
  BoxView Y, T, rho, D, chi, mu, xi, lam;
};
const PPBTransTables* find_transport(const char* name);
// SRK parameters of a mechanism ([sqrt(1/Tc) | sqrt(a*) | B | F], N each) or nullptr.
const double* find_srk(const char* name);
int device_transport(const PPBTransTables* t, DeviceTransport** out);
int launch_transport(const DeviceMechanism& m, const DeviceTransport& tr, int flags, const TrBox& b,
                     cudaStream_t st);

enum ArkController { ARK_PID = 0, ARK_PI = 1, ARK_I = 2, ARK_EXPGUS = 3 };

// The ARKODE-style reactor (ppb_ark.cuh): method, tolerances, end time.
struct ArkParams {
  ErkTable tab;
  double rtol, atol, tout;
  int reactor_type, controller, max_steps, fsal;
  unsigned long long barrier_ns; // longest wait at the grid barrier (global-timer ns)
};

// Batch result: time reached, last step, counters, flag.
struct ArkInfo {
  double t, h;
  long long nst, nfe, netf, attempts;
  int status, barrier_timeout;
};

// Device buffers of one call.
struct ArkBuffers {
  int ncells, ld;
  double* ysoa;          // in/out, species-major with leading dimension ld
  const double* srcsoa;  // species sources, species-major
  const double *rhoe, *rhoesrc;
  const int* mask;       // -1 skips a cell (nullable)
  const double* atolv;   // N+1 absolute tolerances (nullable: atol)
  double* rhoe_out;      // nullable: rhoe + t_reached * rhoesrc
  double *Y0, *Y1, *F0, *F1, *S; // cell-major scratch
  double* partial;       // 2 * gridDim.x doubles
  unsigned* bar;         // [arrivals, generation]
  ArkInfo* info;
  int *status, *nfe, *stats;
};

// Integrate the batch with one cooperative launch; *grid in: the capacity of
// B.partial / 2 (0: no bound), out: the grid used.
int launch_ark(const DeviceMechanism& m, const ArkParams& P, const ArkBuffers& B, int* grid, cudaStream_t st);


// Store the message ppb_last_error() returns for the calling thread (no
// allocation).
void set_error(const char* msg);

#ifdef PPB_PHASE_TIMERS
int phase_cycles(unsigned long long* out, int reset);
#endif

// Bytes of shared memory one team-integrated cell needs.
size_t team_cell_bytes(const PPBMechTables* t, int lu_fp32);

// ---------------------------------------------------------------- adjoint
enum AdjMode { ADJ_REVERSE = 0, ADJ_TANGENT = 1 };

// Cells of an adjoint or tangent-linear integration (device memory, YCOrder
// cell-major: y0 / lam_y / dy0 / y_out / lam_y0 are [ncells][N+1]).
struct AdjBatch {
  const double* y0;
  const double* src;     // [ncells][N] or nullptr
  const double* rhoe;    // [ncells]
  const double* rhoesrc; // [ncells] or nullptr
  const double* atolv;   // typical-value tolerances or nullptr
  const double* lam_y;   // reverse: dL/dy(t_end)
  const double* dy0;     // tangent: direction in y0 (or nullptr)
  const double* dE;      // tangent: direction in rhoe (or nullptr)
  const double* dp;      // tangent: direction in [ln A | beta | Ea/R] (3R)
  double* y_out;         // y(t_end)
  double* lam_y0;        // reverse: dL/dy0; tangent: dy(t_end)
  double* lam_e;         // reverse: dL/drhoe (or nullptr)
  int* status;           // [ncells]
  int* stats;            // [ncells][7] or nullptr
  int ncells;
};

// Per-warp global scratch of the adjoint kernel.
struct AdjLayout {
  char* cp;          // [warps][cap_cp] checkpoints of cp_stride bytes
  size_t cp_stride;
  int cap_cp;
  void* tape;        // [warps][cap_rec] tape records
  int cap_rec, close_rec;
  double* ys;        // [warps][cap_y][N+1]
  int cap_y, close_y;
  double* gw;        // [ncells][3R] per-cell parameter gradients
  int seg_steps;     // accepted steps per checkpoint segment
  size_t warp_smem;  // shared memory per warp
};

// Per-cell global state of the batched reverse sweep (one chunk of cells).
struct AdjCells {
  char* cp_pool;        // checkpoint slots of cp_stride bytes
  size_t cp_stride;
  int pool_cap;         // slots
  int* pool_next;       // slot counter (device)
  int* cp_idx;          // [cells][max_seg] slot of each segment's checkpoint
  int max_seg;
  void* tape;           // [cells][cap_rec] records
  int cap_rec, close_rec;
  double* ys;           // [cells][cap_y][N+1]
  double* yinfo;        // [cells][cap_y][2] time, gamma
  int cap_y, close_y;
  int *nrec, *ny, *nseg; // [cells]
  double* h0;           // [cells] initial step
  double* lam;          // [cells][7(N+1)] adjoint history and pending correction
  double* lamE;         // [cells]
  double* gw;           // [cells][3R] parameter gradient per cell
  double* items;        // [items][stride] evaluated points of one segment
  int* item_off;        // [cells + 1] first item of each cell
  int* item_cell;       // [items]
  long items_cap;       // items the buffer holds
  int seg_steps;
  // compact copies of the recorded segments (all but each cell's last), so
  // that the reverse sweep needs no recomputation while they fit; or nullptr
  char* tpool;
  unsigned long long tpool_bytes;
  unsigned long long* tpool_next; // bytes handed out (device)
  long long* toff;                // [cells] the current segment's copy: byte offset in tpool, or -1
};
// Host callback growing a device buffer (returns a cudaError_t).
typedef int (*AdjGrow)(void* ctx, void** p, size_t bytes);

struct AdjPlan {
  int wpb = 0, blocks = 0;
  size_t warp_smem = 0, cp_stride = 0;
};
enum : int { ADJ_TAPE_BYTES = 112 };

int plan_adjoint(const DeviceMechanism& m, int mode, int lu_fp32, AdjPlan* p);
// grad (3R) receives (accumulate = 0) or gains (1) the cells' summed
// parameter gradient, summed in cell order.
int launch_adjoint(const DeviceMechanism& m, const Options& o, int mode, int lu_fp32, const AdjPlan& p,
                   const AdjBatch& b, const AdjLayout& L, double dt, int* queue, double* grad, int accumulate,
                   cudaStream_t st);
// The reverse (adjoint) integration of one chunk of cells, batched over the
// cells segment by segment: forward with checkpoints, then per segment
// (last first) recomputation, evaluation of every point, and the sweeps.
// grow enlarges C.items (passing its capacity in C.items_cap) when a segment
// needs more; the item bytes per point are adj_item_bytes().
int launch_adjoint_batched(const DeviceMechanism& m, const Options& o, int lu_fp32, const AdjBatch& b, AdjCells& C,
                           double dt, int* queue, double* grad, int accumulate, AdjGrow grow, void* grow_ctx,
                           cudaStream_t st);
size_t adj_item_bytes(int N, int R);
size_t adj_cp_bytes(int N, int lu_fp32);

// Pointwise exact derivatives of the reactor RHS (any output may be null).
int launch_rhs_exact(const DeviceMechanism& m, int rtype, double t, const double* y, const double* rhoe,
                     const double* rhoesrc, const double* src, const double* v, double* f_out, double* J_out,
                     double* fE_out, double* vy_out, double* vE_out, double* vp_out, int ncells, cudaStream_t st);
} // namespace ppb
