// The ARKODE-style explicit reactor (ReactorArkode drop-in).
//
// The reference (Source/Reactions/ReactorArkode.cpp:134-398) hands the whole
// batch to ONE SUNDIALS ERKStep/ARKStep integrator: the state is a single
// vector of ncells * (N+1) entries, so every cell advances with the same time
// steps, chosen from one WRMS error norm over all entries.  That coupling is
// restated here, B200-first: one persistent, co-resident grid integrates the
// batch; each warp carries a fixed set of cells through all stages of a step
// (the stages of a cell only need that cell), and the one global quantity --
// the error norm -- is summed block by block in a fixed order and combined
// after one grid barrier per step, so every block takes the same
// accept/reject and step-size decision from the same bits.
//
// Algorithm (SUNDIALS ARKODE, external and absent from the reference tree;
// restated from its published description, "ARKODE mathematical
// considerations": time step adaptivity, error norms, initial step):
//   * explicit embedded RK table (ppb_erk_tables.h), stage k_i =
//     f(t + c_i h, y + h sum_j A_ij k_j), y+ = y + h sum b_i k_i, embedded
//     error h sum (b_i - d_i) k_i; FSAL tables reuse the last stage;
//   * error weights 1 / (rtol |y_n| + atol_i) from the step's start state,
//     dsm = WRMS over every entry of the batch, accept when dsm <= 1;
//   * step controllers I, PI, PID, explicit Gustafsson on bias * dsm with
//     order q (the method order), safety factor, growth bound (first step
//     1e4, then 20), no-change window (1, 1.5), after a failed test no
//     growth, and after 2 failures at most 0.3; at most 7 failures a step;
//   * initial step from the CVODE/ARKODE estimate (bounded second-derivative
//     norm, at most 4 iterations);
//   * ARK_NORMAL output: integrate past tout and return the cubic Hermite
//     interpolant at tout; at most max_steps internal steps per call (the
//     ARKODE default 500 -- the reference sets none), after which the call
//     stops at the last step reached.
#pragma once
#include "ppb_bdf.cuh"
#include "ppb_engine.h"

namespace ppb {

// Controller gains (ARKODE defaults) and adaptivity constants.
struct ArkAdapt {
  static constexpr double safety = 0.96, bias = 1.5, growth = 20.0, etamx1 = 1.0e4, etamxf = 0.3, etamin = 0.1;
  static constexpr double lb = 1.0, ub = 1.5, tiny = 1.0e-10;
  static constexpr int small_nef = 2, max_nef = 7;
};

// Step estimate of the controller from the current and the two previous
// accepted (biased) error estimates; nacc = accepted steps so far.
__host__ __device__ inline double ark_controller(int ctl, int ord, double h, double dsm, double ep, double epp,
                                                 int nacc)
{
  const double e1 = fmax(ArkAdapt::bias * dsm, ArkAdapt::tiny);
  const double e2 = fmax(ep, ArkAdapt::tiny), e3 = fmax(epp, ArkAdapt::tiny);
  const double o = (double)ord;
  switch (ctl) {
  case ARK_I:
    return h * pow(e1, -1.0 / o);
  case ARK_PI:
    if (nacc < 1) return h * pow(e1, -0.8 / o);
    return h * pow(e1, -0.8 / o) * pow(e2, 0.31 / o);
  case ARK_EXPGUS:
    if (nacc < 1) return h * pow(e1, -0.367 / o);
    return h * pow(e1, -0.367 / o) * pow(e1 / e2, -0.268 / o);
  default: // PID
    if (nacc < 1) return h * pow(e1, -0.58 / o);
    if (nacc < 2) return h * pow(e1, -0.58 / o) * pow(e2, 0.21 / o);
    return h * pow(e1, -0.58 / o) * pow(e2, 0.21 / o) * pow(e3, -0.1 / o);
  }
}

// eta = h_next / h from the controller with the growth bound etamax.
__host__ __device__ inline double ark_eta(int ctl, int ord, double h, double dsm, double ep, double epp, int nacc,
                                          double etamax)
{
  double ha = ark_controller(ctl, ord, h, dsm, ep, epp, nacc) * ArkAdapt::safety;
  ha = fmin(ha, etamax * h);
  ha = fmax(ha, ArkAdapt::etamin * h);
  if (ha > h * ArkAdapt::lb && ha < h * ArkAdapt::ub) ha = h;
  return ha / h;
}

// Bounded grid barrier for a co-resident (cooperative) grid: every block
// arrives once per call; the last one opens the next generation.  A wait
// gives up after limit_ns of global time (20 s by default) and raises
// *timeout (the kernel then returns), so a lost block can never hang the GPU.
__device__ inline bool ark_grid_barrier(unsigned* bar, int* timeout, unsigned long long limit_ns)
{
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned* gen = bar + 1;
    const unsigned g = *gen;
    __threadfence();
    const unsigned arrived = atomicAdd(bar, 1u) + 1u;
    ok = 1;
    if (arrived == gridDim.x) {
      bar[0] = 0;
      __threadfence();
      atomicAdd(bar + 1, 1u);
    } else {
      unsigned long long t0, t1;
      asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
      while (*gen == g) {
        __nanosleep(256);
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t1));
        if (t1 - t0 > limit_ns) {
          atomicExch(timeout, 1);
          ok = 0;
          break;
        }
      }
    }
    __threadfence();
  }
  __syncthreads();
  return ok != 0;
}

} // namespace ppb
