/*
 * rodas3_kernels.cu -- the batched Rodas3 solve on sm_100a.
 *
 * Two kernels share one per-cell state machine (`advance`), which performs
 * exactly the arithmetic of Integrate_Cell_S
 * (src/geos-chem/KPP/fullchem/gckpp_BatchIntegrator.F90:408-707) one
 * attempt (one pass of the UntilAccepted loop, :567-699) at a time:
 *
 *   rodas3_plain      one thread per cell for the whole solve, the mapping of
 *                     the reference's `!$acc parallel loop gang vector`
 *                     (gpulib/src/gc_gpu_batch_api.F90:202-209).
 *   rodas3_persistent a persistent grid sized to the resident thread count;
 *                     every thread drains cells from a device work queue in
 *                     the caller's (cost-sorted) order and refills its slot
 *                     as soon as its cell finishes, so cells with few steps no
 *                     longer idle behind long ones in the same warp.
 *
 * Flattening the reference's three nested loops (TimeLoop / UntilAccepted /
 * singular retry) into one attempt per iteration does not change any
 * floating-point operation: the new-step prologue (Fcn0, dFdT, Jac0) runs
 * only when the previous attempt was accepted, the singular retry halves H
 * and re-factors, and every counter is bumped where the reference bumps it.
 *
 * All arithmetic is FP64.  Built with --fmad=false the kernels reproduce the
 * CPU oracle bit for bit; the production build contracts a*b+c into FMA and,
 * in the persistent kernel, forms LU multipliers and backward-solve quotients
 * from one reciprocal per pivot row (GC_LU_RECIP, mech_lu.cu).
 */
#include <cuda_runtime.h>
#include <float.h>
#include <mutex>
#include "rodas3_device.cuh"
#include "gc_pow.h"
#include "rodas3_kernels.h"

/* LU sparsity (KppDecomp tables LU_CROW/LU_DIAG/LU_ICOL, 0-based).  Every
   thread walks the same pattern in the same order, so these reads are
   warp-uniform broadcasts from the constant cache. */
__constant__ int c_lu_crow[NVAR + 1] = MECH_LU_CROW_INIT;
__constant__ int c_lu_diag[NVAR] = MECH_LU_DIAG_INIT;
__constant__ int c_lu_icol[NNZ] = MECH_LU_ICOL_INIT;

/* Row primitives of the indexed KppDecomp (gckpp_LinearAlgebra.F90:46-84)
   on slot arrays (element stride LANES).  The loop bodies are independent:
   the columns of one row are distinct, so no two iterations touch the same
   entry of W.  Each primitive handles B iterations per pass by loading all
   of the pass's operands before storing any result.  The B loads are then in
   flight together instead of one round trip per entry.  Every entry gets
   exactly the scalar loop's operation.  Each returns the first index it left
   undone (fewer than B remain), for a narrower pass to finish. */
template <int B>
__device__ __forceinline__ int lu_row_load_neg(double* __restrict__ W,
                                               const double* __restrict__ A,
                                               const int* __restrict__ icol, int kk, int r1) {
  for (; kk + B <= r1; kk += B) {          /* W(icol(kk)) = -A(kk) */
    double v[B];
#pragma unroll
    for (int b = 0; b < B; ++b) v[b] = A[(kk + b) * LANES];
#pragma unroll
    for (int b = 0; b < B; ++b) W[icol[kk + b] * LANES] = -v[b];
  }
  return kk;
}

template <int B>
__device__ __forceinline__ int lu_row_store(double* __restrict__ A, const double* __restrict__ W,
                                            const int* __restrict__ icol, int kk, int r1) {
  for (; kk + B <= r1; kk += B) {          /* A(kk) = W(icol(kk)) */
    double v[B];
#pragma unroll
    for (int b = 0; b < B; ++b) v[b] = W[icol[kk + b] * LANES];
#pragma unroll
    for (int b = 0; b < B; ++b) A[(kk + b) * LANES] = v[b];
  }
  return kk;
}

template <int B>
__device__ __forceinline__ int lu_row_axpy(double* __restrict__ W, const double* __restrict__ U,
                                           const int* __restrict__ icol, double a, int jj,
                                           int u1) {
  for (; jj + B <= u1; jj += B) {          /* W(icol(jj)) = W(icol(jj)) + a*U(jj) */
    int c[B];
    double w[B], u[B];
#pragma unroll
    for (int b = 0; b < B; ++b) {
      c[b] = icol[jj + b];
      w[b] = W[c[b] * LANES];
      u[b] = U[(jj + b) * LANES];
    }
#pragma unroll
    for (int b = 0; b < B; ++b) W[c[b] * LANES] = w[b] + a * u[b];
  }
  return jj;
}

/* whole rows: passes of GC_DECOMP_BATCH iterations, then GC_DECOMP_TAIL,
   then one */
#ifndef GC_DECOMP_BATCH
#define GC_DECOMP_BATCH 16
#endif
#ifndef GC_DECOMP_TAIL
#define GC_DECOMP_TAIL 4
#endif
#define GC_TAIL_PASS (GC_DECOMP_TAIL > 1 && GC_DECOMP_TAIL < GC_DECOMP_BATCH)

__device__ __forceinline__ void lu_load_row_neg(double* __restrict__ W,
                                                const double* __restrict__ A,
                                                const int* __restrict__ icol, int kk, int r1) {
  kk = lu_row_load_neg<GC_DECOMP_BATCH>(W, A, icol, kk, r1);
  if (GC_TAIL_PASS) kk = lu_row_load_neg<GC_DECOMP_TAIL>(W, A, icol, kk, r1);
  lu_row_load_neg<1>(W, A, icol, kk, r1);
}

__device__ __forceinline__ void lu_store_row(double* __restrict__ A, const double* __restrict__ W,
                                             const int* __restrict__ icol, int kk, int r1) {
  kk = lu_row_store<GC_DECOMP_BATCH>(A, W, icol, kk, r1);
  if (GC_TAIL_PASS) kk = lu_row_store<GC_DECOMP_TAIL>(A, W, icol, kk, r1);
  lu_row_store<1>(A, W, icol, kk, r1);
}

__device__ __forceinline__ void lu_axpy_row(double* __restrict__ W, const double* __restrict__ U,
                                            const int* __restrict__ icol, double a, int jj,
                                            int u1) {
  jj = lu_row_axpy<GC_DECOMP_BATCH>(W, U, icol, a, jj, u1);
  if (GC_TAIL_PASS) jj = lu_row_axpy<GC_DECOMP_TAIL>(W, U, icol, a, jj, u1);
  lu_row_axpy<1>(W, U, icol, a, jj, u1);
}

/* ros_PrepareMatrix (gckpp_BatchIntegrator.F90:573-577) fused into
   KppDecomp (gckpp_LinearAlgebra.F90:46-84): each row of -J0 + ghinv*I is
   built in the dense row scratch W, eliminated with the finished rows of G
   and stored once into G, so J0 is read once and G written once per row
   instead of a separate copy pass over all NNZ entries.  Every entry gets the
   reference's operations: G = -J0, G(i,i) = G(i,i) + ghinv, then the row
   updates W = W + a*U with a = -(W(j)/U(j,j)).  KppDecomp tests row k's
   diagonal before row k is touched, so the test reads (-J0(k,k)) + ghinv;
   after a singular return G is not used.
   With GC_IRECIP (FMA build only) each finished row stores 1/U(k,k) in Rs,
   a scratch array the caller has free during the factorisation, and every
   multiplier is -(w * Rs(j)), as in the generated fused LU; on return W
   holds the reciprocals for mech_solve_recip. */
__device__ __noinline__ int kpp_prep_decomp(const double* __restrict__ J0,
                                            double* __restrict__ G,
                                            double* __restrict__ W,
                                            double* __restrict__ Rs, double ghinv) {
  for (int k = 0; k < NVAR; ++k) {
    const int d = c_lu_diag[k];
    const double dk = (-J0[d * LANES]) + ghinv;
    if (fabs(dk) < DBL_MIN) return k + 1;
    const int r0 = c_lu_crow[k], r1 = c_lu_crow[k + 1];
    lu_load_row_neg(W, J0, c_lu_icol, r0, r1);
    W[k * LANES] = dk;
    for (int kk = r0; kk < d; ++kk) {
      const int j = c_lu_icol[kk];
#if GC_IRECIP
      const double a = -(W[j * LANES] * Rs[j * LANES]);
#else
      const double a = -(W[j * LANES] / G[c_lu_diag[j] * LANES]);
#endif
      W[j * LANES] = -a;
      lu_axpy_row(W, G, c_lu_icol, a, c_lu_diag[j] + 1, c_lu_crow[j + 1]);
    }
#if GC_IRECIP
    Rs[k * LANES] = 1.0 / W[k * LANES];
#endif
    lu_store_row(G, W, c_lu_icol, r0, r1);
  }
#if GC_IRECIP
  for (int i = 0; i < NVAR; ++i) W[i * LANES] = Rs[i * LANES];
#else
  (void)Rs;
#endif
  return 0;
}

/* per-thread state of the cell being solved */
struct Lane {
  long col;          /* batch column (0-based) of the cell */
  CellOpts o;
  CellStat st;
  double T, H;
  int nsteps, ncons;
  int rej_last, rej_more, newstep;
  int ierr;          /* 0 while running */
  int ysel;          /* which of the slot's two state arrays holds Y (an accepted
                        step swaps their roles instead of copying Ynew into Y) */
  int attempt;       /* 0: first solve; 1: the retry of a cell whose first solve failed */
};

struct BatchArgs {
  int ncell;
  double tstart, tend;
  double* C;               /* (NSPEC, ncell) column-major, in/out */
  const double* RCONST;    /* (NREACT, ncell) */
  const double* ATOL;      /* (NVAR) */
  const double* RTOL;      /* (NVAR) */
  const int* ICNTRL;       /* (20, ncell) */
  const double* RCNTRL;    /* (20, ncell) */
  const int* order;        /* launch order: 0-based columns (Perm(ic)-1) */
  int* ISTAT;              /* (8, ncell) */
  double* RSTAT;           /* (3, ncell) */
  int* IERR;               /* (ncell) */
  double* ws;              /* warp-tiled workspace */
  unsigned int* qhead;     /* persistent kernel: next queue position */
  int* nfail;              /* retry protocol on (non-NULL): [0] cells whose first solve
                              failed, [1] cells that failed the retry too */
  const double* ATOLr;     /* retry tolerances (NVAR) */
  const double* RTOLr;
  double* ckpt;            /* adjoint checkpoints (y_n, h_n) per accepted step, or NULL */
  int ckpt_max;            /* accepted steps stored per cell */
};

/* gather the cell's column into the slot and set the integrator state;
   attempt 1 is the retry: RCNTRL(3) (Hstart) taken as 0 and the retry
   tolerances, fullchem_mod.F90:2436-2520 */
__device__ __forceinline__ void lane_start(Lane& L, const BatchArgs& a, double* ws, long slot,
                                           long col, int attempt = 0) {
  L.col = col;
  L.attempt = attempt;
  const double* c = a.C + col * NSPEC;
  const double* r = a.RCONST + col * NREACT;
  double* Y = slot_ptr(ws, slot, OFF_Y);
  double* F = slot_ptr(ws, slot, OFF_FIX);
  double* R = slot_ptr(ws, slot, OFF_RCT);
  for (int i = 0; i < NVAR; ++i) Y[i * LANES] = c[i];
  for (int i = 0; i < NFIX; ++i) F[i * LANES] = c[NVAR + i];
  for (int j = 0; j < NREACT; ++j) R[j * LANES] = r[j];
  L.o = decode_options(a.ICNTRL + col * 20, a.RCNTRL + col * 20, a.tstart, a.tend,
                       attempt);
  L.st.nfun = L.st.njac = L.st.nstp = L.st.nacc = 0;
  L.st.nrej = L.st.ndec = L.st.nsol = L.st.nsng = 0;
  L.st.texit = L.st.hexit = L.st.hnew = 0.0;
  L.ierr = L.o.ierr_early;
  L.T = a.tstart;
  double H = fminF(fmaxF(fabs(L.o.hmin), fabs(L.o.hstart)), fabs(L.o.hmax));
  if (fabs(H) <= 10.0 * ROUNDOFF) H = DELTAMIN;
  const double dir = (a.tend >= a.tstart) ? 1.0 : -1.0;
  L.H = dir * H;
  L.nsteps = 0;
  L.ncons = 0;
  L.rej_last = L.rej_more = 0;
  L.newstep = 1;
  L.ysel = 0;
}

/* the slot's current Y and Ynew arrays */
__device__ __forceinline__ double* y_array(double* ws, long slot, int ysel) {
  return slot_ptr(ws, slot, ysel ? OFF_YNEW : OFF_Y);
}
__device__ __forceinline__ double* ynew_array(double* ws, long slot, int ysel) {
  return slot_ptr(ws, slot, ysel ? OFF_Y : OFF_YNEW);
}

/* scatter results to column L.col (gc_gpu_batch_api.F90:204-208) */
__device__ __forceinline__ void lane_finish(const Lane& L, const BatchArgs& a, double* ws, long slot) {
  const long col = L.col;
  if (L.o.ierr_early == 0) {
    const double* Y = y_array(ws, slot, L.ysel);
    double* c = a.C + col * NSPEC;
    for (int i = 0; i < NVAR; ++i) c[i] = Y[i * LANES];
  }
  int* is = a.ISTAT + col * 8;
  if (L.attempt) {   /* the retry's counters add to the first solve's */
    is[0] += L.st.nfun; is[1] += L.st.njac; is[2] += L.st.nstp; is[3] += L.st.nacc;
    is[4] += L.st.nrej; is[5] += L.st.ndec; is[6] += L.st.nsol; is[7] += L.st.nsng;
    if (L.ierr < 0) atomicAdd(&a.nfail[1], 1);
  } else {
    is[0] = L.st.nfun; is[1] = L.st.njac; is[2] = L.st.nstp; is[3] = L.st.nacc;
    is[4] = L.st.nrej; is[5] = L.st.ndec; is[6] = L.st.nsol; is[7] = L.st.nsng;
  }
  double* rs = a.RSTAT + col * 3;
  rs[0] = L.st.texit; rs[1] = L.st.hexit; rs[2] = L.st.hnew;
  a.IERR[col] = L.ierr;
}

/* The end of a solve.  With the retry protocol on, a first solve that
   failed (IERR < 0) is not written back: its counters are stored, and the
   lane starts the cell again from its untouched input column as the retry
   (the model's protocol, fullchem_mod.F90:2436-2520: reset C, Hstart = 0,
   retry tolerances, ISTAT summed over both solves, RSTAT and IERR of the
   retry).  The retry runs while the other lanes carry on, instead of in a
   second launch after the whole batch.  Returns 1 when the cell is finished,
   0 when the lane now holds its retry. */
__device__ __forceinline__ int lane_end(Lane& L, const BatchArgs& a, double* ws, long slot) {
  if (a.nfail && L.attempt == 0 && L.ierr < 0) {
    int* is = a.ISTAT + L.col * 8;
    is[0] = L.st.nfun; is[1] = L.st.njac; is[2] = L.st.nstp; is[3] = L.st.nacc;
    is[4] = L.st.nrej; is[5] = L.st.ndec; is[6] = L.st.nsol; is[7] = L.st.nsng;
    atomicAdd(&a.nfail[0], 1);
    lane_start(L, a, ws, slot, L.col, 1);
    if (L.ierr == 0) return 0;
  }
  lane_finish(L, a, ws, slot);
  return 1;
}

/* One pass of the integrator loop for the thread's cell, statement for
   statement the body of TimeLoop/UntilAccepted in
   gckpp_BatchIntegrator.F90:535-704, in four pieces so that the persistent
   kernel can reconverge its warp between them:

     step_begin     new step only: the TimeLoop exit tests and the H clamp;
                    1 when the cell is finished (L.ierr holds IERR)
     step_prologue  new step only: Fcn0 [, dFdT], Jac0
     step_factor    ros_PrepareMatrix + factorisation; 0 factored, 1
                    singular and retried with H/2 (the attempt ends), 2
                    singular too often (IERR -8, finished)
     step_stages    the four stages, the error norm, accept or reject

   kFusedLU selects the generated register-blocked factorisation
   (mech_prep_decomp) instead of the indexed KppDecomp with its W scratch row;
   both perform the same operations in the same order. */
struct StepPtrs {
  double *Y, *Ynew, *Fcn0, *dFdT, *W, *K, *Jac0, *G;
  const double *F, *R;
};

/* Row-scratch placement.  The indexed KppDecomp reads and writes its dense
   row scratch W (NVAR doubles) at every update of the factorisation.  By
   default W is an array of the cell's workspace slot (HBM).  For mechanisms
   without the generated fused LU and with few species (the 120-species
   synthetic one), W can instead live in shared memory: warp w's lanes own a
   per-warp tile, element c of lane l at tile[c * 32 + l] (the workspace's
   element stride, conflict-free).  The arithmetic and its order are the same
   either way.  A launch with shared W provides blockDim.x * NVAR doubles of
   dynamic shared memory; the *_sw kernels below are those launches. */
#define SMEM_W_OK (MECH_FUSED_LU == 0 && NVAR <= 160)
extern __shared__ double s_w[];

template <bool kSharedW>
__device__ __forceinline__ StepPtrs step_ptrs(double* ws, long slot, int ysel) {
  StepPtrs p;
  p.Y = y_array(ws, slot, ysel & 1);
  p.F = slot_ptr(ws, slot, OFF_FIX);
  p.R = slot_ptr(ws, slot, OFF_RCT);
  p.Ynew = ynew_array(ws, slot, ysel & 1);
  p.Fcn0 = slot_ptr(ws, slot, OFF_FCN0);
  p.dFdT = slot_ptr(ws, slot, OFF_DFDT);
  if (kSharedW)
    p.W = s_w + (long)(threadIdx.x >> 5) * (NVAR * LANES) + (threadIdx.x & 31);
  else
    p.W = slot_ptr(ws, slot, OFF_W);
  p.K = slot_ptr(ws, slot, OFF_K);
  p.Jac0 = slot_ptr(ws, slot, OFF_JAC0);
  p.G = slot_ptr(ws, slot, OFF_GHIMJ);
  return p;
}

__device__ __forceinline__ int step_begin(Lane& L, const BatchArgs& a) {
  const double Tend = a.tend;
  const int direction = (Tend >= a.tstart) ? 1 : -1;
  const bool running = (direction > 0 && ((L.T - Tend) + ROUNDOFF <= 0.0)) ||
                       (direction < 0 && ((Tend - L.T) + ROUNDOFF <= 0.0));
  if (!running) { L.ierr = 1; return 1; }
  if (L.nsteps > L.o.max_steps) { L.ierr = -6; return 1; }
  if (((L.T + 0.1 * L.H) == L.T) || (L.H <= ROUNDOFF)) { L.ierr = -7; return 1; }
  L.H = fminF(L.H, fabs(Tend - L.T));
  return 0;
}

__device__ __forceinline__ void step_prologue(Lane& L, const StepPtrs& p) {
  mech_fun(p.Y, p.F, p.R, p.Fcn0);
  L.st.nfun += 1;
  if (!L.o.autonomous) {
    const double delta = sqrt(ROUNDOFF) * fmaxF(1.0e-6, fabs(L.T));
    mech_fun(p.Y, p.F, p.R, p.dFdT);
    L.st.nfun += 1;
    for (int k = 0; k < NVAR; ++k)
      p.dFdT[k * LANES] = (p.dFdT[k * LANES] - p.Fcn0[k * LANES]) / delta;
  }
  mech_jac(p.Y, p.F, p.R, p.Jac0);
  L.st.njac += 1;
  L.newstep = 0;
  L.ncons = 0;
}

/* ros_PrepareMatrix: Ghimj = -Jac0 + diag(1/(H*gamma1)); factor */
template <bool kFusedLU>
__device__ __forceinline__ int step_factor(Lane& L, const BatchArgs& a, const StepPtrs& p) {
  const double dir = (a.tend >= a.tstart) ? 1.0 : -1.0;
  const double ghinv = 1.0 / ((dir * L.H) * 0.5);
  int ising;
  if (kFusedLU) {
    ising = mech_prep_decomp(p.Jac0, p.G, p.W, ghinv);
  } else {
    /* Ynew is dead here: the stages write it after the factorisation */
    ising = kpp_prep_decomp(p.Jac0, p.G, p.W, p.Ynew, ghinv);
  }
  L.st.ndec += 1;
  if (ising != 0) {
    L.st.nsng += 1;
    L.ncons += 1;
    if (L.ncons <= 5) { L.H = L.H * 0.5; return 1; }
    L.ierr = -8;
    return 2;
  }
  return 0;
}

/* KppSolve for a stage.  After the FMA build's fused factorisation the
   slot's W array holds 1/U(i,i) and the backward sweep multiplies by it. */
template <bool kFusedLU>
__device__ __forceinline__ void stage_solve(const StepPtrs& p, double* X) {
#if defined(GC_LU_RECIP) && GC_LU_RECIP
  if (kFusedLU || GC_IRECIP) { mech_solve_recip(p.G, p.W, X); return; }
#endif
  mech_solve(p.G, X);
}

template <bool kFusedLU>
__device__ __forceinline__ void step_stages(Lane& L, const BatchArgs& a, const StepPtrs& p) {
  const double dir = (a.tend >= a.tstart) ? 1.0 : -1.0;
  double* Y = p.Y;
  double* Ynew = p.Ynew;
  const double* Fcn0 = p.Fcn0;
  const double* dFdT = p.dFdT;
  const double* F = p.F;
  const double* R = p.R;
  double* K = p.K;
  const double dH = dir * L.H;
  double* K2 = K + NVAR * LANES;
  double* K3 = K + 2 * NVAR * LANES;
  double* K4 = K + 3 * NVAR * LANES;
  /* Each stage's vector updates are done in one pass per array with the
     per-element operation sequence of the reference's separate loops
     (gckpp_BatchIntegrator.F90:595-632): K(s) = Fcn, then + HC_j*K(j) for
     j = 1..s-1 in order, then + HG*dFdT. */
  /* stage 1: K1 = Fcn0 [+ (dH*gamma1) dFdT] */
  if (L.o.autonomous) {
    for (int k = 0; k < NVAR; ++k) K[k * LANES] = Fcn0[k * LANES];
  } else {
    const double hg = dH * 0.5;
    for (int k = 0; k < NVAR; ++k) K[k * LANES] = Fcn0[k * LANES] + hg * dFdT[k * LANES];
  }
  stage_solve<kFusedLU>(p, K);
  L.st.nsol += 1;
  /* stage 2: ros_NewF(2) false, Fcn stays Fcn0: K2 = Fcn0 + (4/dH) K1 [+ (dH*gamma2) dFdT] */
  {
    const double hc = 4.0 / dH;
    if (L.o.autonomous) {
      for (int k = 0; k < NVAR; ++k) K2[k * LANES] = Fcn0[k * LANES] + hc * K[k * LANES];
    } else {
      const double hg = dH * 1.5;
      for (int k = 0; k < NVAR; ++k)
        K2[k * LANES] = (Fcn0[k * LANES] + hc * K[k * LANES]) + hg * dFdT[k * LANES];
    }
    stage_solve<kFusedLU>(p, K2);
    L.st.nsol += 1;
  }
  /* stage 3: Ynew = (Y + 2 K1) + 0 K2; K3 = F(Ynew); K3 = (K3 + (1/dH) K1) + (-1/dH) K2 */
  {
    for (int k = 0; k < NVAR; ++k)
      Ynew[k * LANES] = (Y[k * LANES] + 2.0 * K[k * LANES]) + 0.0 * K2[k * LANES];
    mech_fun(Ynew, F, R, K3);
    L.st.nfun += 1;
    const double hc1 = 1.0 / dH, hc2 = -1.0 / dH;
    for (int k = 0; k < NVAR; ++k)
      K3[k * LANES] = (K3[k * LANES] + hc1 * K[k * LANES]) + hc2 * K2[k * LANES];
    stage_solve<kFusedLU>(p, K3);
    L.st.nsol += 1;
  }
  /* stage 4: Ynew = ((Y + 2 K1) + 0 K2) + 1 K3; K4 = F(Ynew);
     K4 = ((K4 + (1/dH) K1) + (-1/dH) K2) + (-(8/3)/dH) K3.  Ynew still holds
     stage 3's (Y + 2 K1) + 0 K2, rounded exactly as this expression rounds
     it, so only the last term is added. */
  {
    for (int k = 0; k < NVAR; ++k)
      Ynew[k * LANES] = Ynew[k * LANES] + 1.0 * K3[k * LANES];
    mech_fun(Ynew, F, R, K4);
    L.st.nfun += 1;
    const double hc1 = 1.0 / dH, hc2 = -1.0 / dH, hc3 = -(8.0 / 3.0) / dH;
    for (int k = 0; k < NVAR; ++k)
      K4[k * LANES] = ((K4[k * LANES] + hc1 * K[k * LANES]) + hc2 * K2[k * LANES]) +
                      hc3 * K3[k * LANES];
    stage_solve<kFusedLU>(p, K4);
    L.st.nsol += 1;
  }

  /* Ynew = Y + sum ros_M(j) K(j); Yerr = sum ros_E(j) K(j); WRMS norm */
  const double* atol = L.attempt ? a.ATOLr : a.ATOL;
  const double* rtol = L.attempt ? a.RTOLr : a.RTOL;
  double err = 0.0;
  for (int i = 0; i < NVAR; ++i) {
    const double y = Y[i * LANES];
    const double k1 = K[i * LANES], k2 = K2[i * LANES], k3 = K3[i * LANES], k4 = K4[i * LANES];
    const double yn = (((y + 2.0 * k1) + 0.0 * k2) + 1.0 * k3) + 1.0 * k4;
    Ynew[i * LANES] = yn;
    const double ye = (((0.0 + 0.0 * k1) + 0.0 * k2) + 0.0 * k3) + 1.0 * k4;
    const double ymax = fmaxF(fabs(y), fabs(yn));
    const double scal = L.o.vectortol ? (__ldg(atol + i) + __ldg(rtol + i) * ymax)
                                      : (__ldg(atol) + __ldg(rtol) * ymax);
    const double q = ye / scal;
    err = err + q * q;
  }
  err = sqrt(err / (double)NVAR);
  err = fmaxF(err, 1.0e-10);
  const double fac = fminF(L.o.facmax,
                           fmaxF(L.o.facmin, L.o.facsafe / gc_pow(err, 1.0 / ROS_ELO)));
  double hnew = L.H * fac;

  L.nsteps += 1;
  L.st.nstp += 1;
  if ((err <= 1.0) || (L.H <= L.o.hmin)) {
    L.st.nacc += 1;
    if (a.ckpt && L.st.nacc <= a.ckpt_max) {
      /* checkpoint for the adjoint: the step's starting state and its size */
      double* ck = a.ckpt + ((long)L.col * a.ckpt_max + (L.st.nacc - 1)) * (NVAR + 1);
      for (int k = 0; k < NVAR; ++k) ck[k] = Y[k * LANES];
      ck[NVAR] = L.H;
    }
    /* Y = Ynew [clamped at 0]: the arrays swap roles instead of copying */
    if (L.o.clamp) {
      for (int k = 0; k < NVAR; ++k) Ynew[k * LANES] = fmaxF(Ynew[k * LANES], 0.0);
    }
    L.ysel ^= 1;
    L.T = L.T + dir * L.H;
    hnew = fmaxF(L.o.hmin, fminF(hnew, L.o.hmax));
    if (L.rej_last) hnew = fminF(hnew, L.H);
    L.st.hexit = L.H;
    L.st.hnew = hnew;
    L.st.texit = L.T;
    L.rej_last = 0;
    L.rej_more = 0;
    L.H = hnew;
    L.newstep = 1;
  } else {
    if (L.rej_more) hnew = L.H * L.o.facrej;
    L.rej_more = L.rej_last;
    L.rej_last = 1;
    L.H = hnew;
    if (L.st.nacc >= 1) L.st.nrej += 1;
    L.ncons = 0;
  }
}

/* one attempt; returns 1 when the cell is finished (L.ierr holds IERR) */
template <bool kFusedLU, bool kSharedW>
__device__ __forceinline__ int advance(Lane& L, const BatchArgs& a, double* ws, long slot) {
  const StepPtrs p = step_ptrs<kSharedW>(ws, slot, L.ysel);
  if (L.newstep) {
    if (step_begin(L, a)) return 1;
    step_prologue(L, p);
  }
  const int f = step_factor<kFusedLU>(L, a, p);
  if (f == 1) return 0;
  if (f == 2) return 1;
  step_stages<kFusedLU>(L, a, p);
  return 0;
}

/* ---------------------------------------------------------------------- */
template <bool kFusedLU, bool kSharedW>
__device__ __forceinline__ void plain_cell(const BatchArgs& a, int first, int count) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= count) return;
  const long col = a.order[first + t];
  const long slot = t;
  Lane L;
  lane_start(L, a, a.ws, slot, col);
  do {
    if (L.ierr == 0) {
      while (!advance<kFusedLU, kSharedW>(L, a, a.ws, slot)) {}
    }
  } while (!lane_end(L, a, a.ws, slot));
}

/* the reference's mapping: one thread per cell, indexed KppDecomp with its
   dense row scratch, the reference's divides */
__global__ void __launch_bounds__(256) rodas3_plain(BatchArgs a, int first, int count) {
  plain_cell<false, false>(a, first, count);
}

/* one thread per cell with the persistent kernel's arithmetic (generated
   fused factorisation; pivot reciprocals in the FMA build): the baseline
   that isolates what the queue and the cost order gain */
__global__ void __launch_bounds__(256) rodas3_plain_fused(BatchArgs a, int first, int count) {
  plain_cell<MECH_FUSED_LU != 0, false>(a, first, count);
}

/* The loop is warp-synchronous: every lane of a warp runs every iteration
   (blockDim is a multiple of 32 and no lane leaves early), the lanes without
   a cell take consecutive queue positions with one atomic per warp, and the
   full-mask ballot at the top of each iteration reconverges the warp before
   the attempt.  A per-lane refill with `continue`/`break` inside the loop
   left no reconvergence point before `advance`: measured with ncu on a case
   where all lanes step in lockstep, only 20 of 32 lanes were active per
   instruction (31.7 in the one-cell-per-thread kernel). */
template <bool kSharedW>
__device__ __forceinline__ void persistent_loop(const BatchArgs& a) {
  const long slot = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const unsigned int lane = threadIdx.x & 31u;
  const unsigned int FULL = 0xffffffffu;
  Lane L;
  L.ysel = 0;   /* lanes without a cell still form (unused) stage pointers */
  int have = 0;
  bool drained = false;  /* warp-uniform: the queue has no cell left */
  const unsigned int ncell = (unsigned int)a.ncell;
  for (;;) {
    const unsigned int need = __ballot_sync(FULL, !have);
    if (need != 0u && !drained) {
      const int leader = __ffs(need) - 1;
      const unsigned int take = (unsigned int)__popc(need);
      unsigned int base = 0u;
      if ((int)lane == leader) base = atomicAdd(a.qhead, take);
      base = __shfl_sync(FULL, base, leader);
      if (base >= ncell || ncell - base <= take) drained = true;
      if (!have) {
        const unsigned int p = base + (unsigned int)__popc(need & ((1u << lane) - 1u));
        if (p < ncell) {
          lane_start(L, a, a.ws, slot, a.order[p]);
          have = (L.ierr == 0) || !lane_end(L, a, a.ws, slot);
        }
      }
    }
    if (!__any_sync(FULL, have)) {
      if (drained) break;
      continue;
    }
    /* one attempt (advance), cut where lanes can part: only the lanes that
       start a new step run the TimeLoop tests and Fcn0/Jac0 (a rejected
       attempt is retried without them), and a singular factorisation ends
       the attempt early.  Every lane passes every __syncwarp. */
    const StepPtrs p = step_ptrs<kSharedW>(a.ws, slot, L.ysel);
    int go = have;
    if (go && L.newstep) {
      if (step_begin(L, a)) { have = !lane_end(L, a, a.ws, slot); go = 0; }
      else step_prologue(L, p);
    }
    __syncwarp(FULL);
    int f = 0;
    if (go) f = step_factor<MECH_FUSED_LU != 0>(L, a, p);
    __syncwarp(FULL);
    if (go && f == 2) have = !lane_end(L, a, a.ws, slot);
    if (go && f == 0) step_stages<MECH_FUSED_LU != 0>(L, a, p);
    __syncwarp(FULL);
  }
}

__global__ void __launch_bounds__(256) rodas3_persistent(BatchArgs a) {
  persistent_loop<false>(a);
}

#if SMEM_W_OK
/* the same kernels with the indexed factorisation's row scratch in shared
   memory (launched with blockDim.x * NVAR doubles of dynamic shared memory) */
__global__ void __launch_bounds__(256) rodas3_plain_sw(BatchArgs a, int first, int count) {
  plain_cell<false, true>(a, first, count);
}
__global__ void __launch_bounds__(256) rodas3_persistent_sw(BatchArgs a) {
  persistent_loop<true>(a);
}
#endif

/* Cost ordering: the model's pre-scan sort (fullchem_mod.F90:906-960), a
   STABLE counting sort of the cells by the previous step's ISTAT(3), most
   expensive first, ties kept in cell order, no bound on the key.

   On the device the same order is produced by sorting unique 64-bit
   composites  (~(key ^ 0x80000000)) << 32 | cell  in ascending order: the
   high word orders by descending key (any int32), the low word breaks ties
   by ascending cell index, so the result equals the stable sort exactly and
   does not depend on thread timing.  The sort is a bitonic network over the
   composites padded to a power of two with UINT64_MAX: tiles of
   COST_TILE composites are sorted and merged in shared memory, larger
   strides go through global memory (one launch per stride). */
#define COST_TILE 2048
typedef unsigned long long u64;

__device__ __forceinline__ void cmp_swap(u64& x, u64& y, bool up) {
  if ((x > y) == up) { const u64 t = x; x = y; y = t; }
}

__global__ void cost_fill(const int* keys, int n, long n2, u64* comp) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n2) return;
  if (i < n) {
    const unsigned int hi = ~((unsigned int)keys[i] ^ 0x80000000u);
    comp[i] = ((u64)hi << 32) | (u64)(unsigned int)i;
  } else {
    comp[i] = ~0ull;
  }
}

/* strides j = jstart .. 1 of the merge of size k, one tile per block; with
   k_from > 0 the block first sorts its tile completely (all sizes
   k_from .. COST_TILE) */
__global__ void __launch_bounds__(COST_TILE / 2) cost_tile(u64* comp, long k, long jstart,
                                                           int full_tile) {
  __shared__ u64 t[COST_TILE];
  const long base = (long)blockIdx.x * COST_TILE;
  const int tid = threadIdx.x;
  t[tid] = comp[base + tid];
  t[tid + COST_TILE / 2] = comp[base + tid + COST_TILE / 2];
  __syncthreads();
  if (full_tile) {
    for (long kk = 2; kk <= COST_TILE; kk <<= 1) {
      for (long j = kk >> 1; j > 0; j >>= 1) {
        const long i = (tid / j) * 2 * j + (tid % j);
        cmp_swap(t[i], t[i + j], ((base + i) & kk) == 0);
        __syncthreads();
      }
    }
  } else {
    for (long j = jstart; j > 0; j >>= 1) {
      const long i = (tid / j) * 2 * j + (tid % j);
      cmp_swap(t[i], t[i + j], ((base + i) & k) == 0);
      __syncthreads();
    }
  }
  comp[base + tid] = t[tid];
  comp[base + tid + COST_TILE / 2] = t[tid + COST_TILE / 2];
}

__global__ void cost_stride(u64* comp, long n2, long k, long j) {
  const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n2 / 2) return;
  const long i = (p / j) * 2 * j + (p % j);
  u64 x = comp[i], y = comp[i + j];
  const bool up = (i & k) == 0;
  if ((x > y) == up) { comp[i] = y; comp[i + j] = x; }
}

__global__ void cost_extract(const u64* comp, int n, int* order) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) order[i] = (int)(unsigned int)(comp[i] & 0xffffffffull);
}

/* composites the sort of n keys needs in its scratch buffer */
extern "C" long rodas3_cost_scratch(int n) {
  long n2 = COST_TILE;
  while (n2 < n) n2 <<= 1;
  return n2;
}

extern "C" cudaError_t rodas3_cost_order(const int* keys, int n, int* order,
                                         unsigned long long* scratch, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  const long n2 = rodas3_cost_scratch(n);
  u64* comp = scratch;
  cost_fill<<<(int)((n2 + 255) / 256), 256, 0, s>>>(keys, n, n2, comp);
  const int tiles = (int)(n2 / COST_TILE);
  cost_tile<<<tiles, COST_TILE / 2, 0, s>>>(comp, 0, 0, 1);
  for (long k = 2 * COST_TILE; k <= n2; k <<= 1) {
    for (long j = k >> 1; j >= COST_TILE; j >>= 1)
      cost_stride<<<(int)((n2 / 2 + 255) / 256), 256, 0, s>>>(comp, n2, k, j);
    cost_tile<<<tiles, COST_TILE / 2, 0, s>>>(comp, k, COST_TILE / 2, 0);
  }
  cost_extract<<<(n + 255) / 256, 256, 0, s>>>(comp, n, order);
  return cudaGetLastError();
}

/* Perm (1-based) -> 0-based order; rejects out-of-range entries */
__global__ void perm_to_order(const int* perm, int n, int* order, int* bad) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int p = perm[i];
  if (p < 1 || p > n) { atomicExch(bad, 1); order[i] = 0; return; }
  order[i] = p - 1;
}

/* ---------------------------------------------------------------------- */
extern "C" int rodas3_ws_elems(void) { return WS_ELEMS; }
extern "C" void rodas3_sizes(int* nvar, int* nfix, int* nreact, int* nnz) {
  *nvar = NVAR; *nfix = NFIX; *nreact = NREACT; *nnz = NNZ;
}

/* dynamic shared memory of a solver launch, and the largest block size the
   solver kernels accept, for the row-scratch placement sw (0 workspace, 1
   shared memory) */
static size_t solver_smem(int threads, int sw) {
  return sw ? (size_t)threads * NVAR * sizeof(double) : 0;
}

extern "C" int rodas3_shared_scratch_ok(void) { return SMEM_W_OK ? 1 : 0; }

extern "C" int rodas3_max_threads(int sw) {
  if (!sw) return 256;
  const int t = (int)((227 * 1024) / (NVAR * sizeof(double))) / 32 * 32;
  return t < 256 ? t : 256;
}

/* allow the shared-memory W tiles above the 48 KB default (a function
   attribute, not stream work: legal at any time, repeated calls are cheap) */
static cudaError_t solver_smem_attr(void) {
#if SMEM_W_OK
  const int bytes = (int)solver_smem(rodas3_max_threads(1), 1);
  cudaError_t e = cudaFuncSetAttribute(rodas3_persistent_sw,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(rodas3_plain_sw, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  return e;
#else
  return cudaSuccess;
#endif
}

extern "C" int rodas3_persistent_blocks_per_sm(int threads, int sw) {
  int nb = 0;
  if (sw && !SMEM_W_OK) return 0;
  if (threads > rodas3_max_threads(sw)) return 0;
  cudaError_t e;
#if SMEM_W_OK
  if (sw) {
    if (solver_smem_attr() != cudaSuccess) return 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, rodas3_persistent_sw, threads,
                                                      solver_smem(threads, 1));
  } else
#endif
  {
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, rodas3_persistent, threads, 0);
  }
  return e == cudaSuccess ? nb : 0;
}

extern "C" cudaError_t rodas3_launch(const Rodas3Launch* L, cudaStream_t s) {
  BatchArgs a;
  a.ncell = L->ncell; a.tstart = L->tstart; a.tend = L->tend;
  a.C = L->C; a.RCONST = L->RCONST; a.ATOL = L->ATOL; a.RTOL = L->RTOL;
  a.ICNTRL = L->ICNTRL; a.RCNTRL = L->RCNTRL; a.order = L->order;
  a.ISTAT = L->ISTAT; a.RSTAT = L->RSTAT; a.IERR = L->IERR;
  a.ws = L->ws; a.qhead = L->qhead;
  a.nfail = L->nfail; a.ATOLr = L->ATOLr; a.RTOLr = L->RTOLr;
  a.ckpt = L->ckpt; a.ckpt_max = L->ckpt_max;
  const int threads = L->threads > 0 ? L->threads : 128;
  const int sw = L->shared_scratch ? 1 : 0;
  if ((sw && !SMEM_W_OK) || threads > rodas3_max_threads(sw)) return cudaErrorInvalidValue;
  if (sw) {
    const cudaError_t ea = solver_smem_attr();
    if (ea != cudaSuccess) return ea;
  }
  const size_t smem = solver_smem(threads, sw);
  if (L->mode == RODAS3_PLAIN || L->mode == RODAS3_PLAIN_FUSED) {
    /* one thread per cell, chunked so the workspace holds `slots` cells */
    const long slots = L->slots;
    for (long first = 0; first < L->ncell; first += slots) {
      const int count = (int)((L->ncell - first) < slots ? (L->ncell - first) : slots);
      const int blocks = (count + threads - 1) / threads;
#if SMEM_W_OK
      if (sw)   /* no fused LU here: both plain modes are the indexed kernel */
        rodas3_plain_sw<<<blocks, threads, smem, s>>>(a, (int)first, count);
      else
#endif
      if (L->mode == RODAS3_PLAIN)
        rodas3_plain<<<blocks, threads, 0, s>>>(a, (int)first, count);
      else
        rodas3_plain_fused<<<blocks, threads, 0, s>>>(a, (int)first, count);
    }
  } else {
    cudaMemsetAsync(L->qhead, 0, sizeof(unsigned int), s);
    const int blocks = (int)(L->slots / threads);
#if SMEM_W_OK
    if (sw)
      rodas3_persistent_sw<<<blocks, threads, smem, s>>>(a);
    else
#endif
      rodas3_persistent<<<blocks, threads, 0, s>>>(a);
  }
  return cudaGetLastError();
}

extern "C" cudaError_t rodas3_perm_to_order(const int* perm, int n, int* order, int* bad,
                                            cudaStream_t s) {
  cudaMemsetAsync(bad, 0, sizeof(int), s);
  perm_to_order<<<(n + 255) / 256, 256, 0, s>>>(perm, n, order, bad);
  return cudaGetLastError();
}

/* ---------------------------------------------------------------------- */
/* FP64 throughput probe: every thread runs 8 independent FMA chains, so the
   FP64 pipe, not latency, is the limit.  Used to measure the FP64 peak that
   the solver's roofline fraction is quoted against. */
__global__ void __launch_bounds__(256) fp64_probe(double* out, int iters, double a, double b) {
  double x0 = threadIdx.x, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3;
  double x4 = x0 + 4, x5 = x0 + 5, x6 = x0 + 6, x7 = x0 + 7;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int u = 0; u < 16; ++u) {
      x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
      x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
    }
  }
  const double s = ((x0 + x1) + (x2 + x3)) + ((x4 + x5) + (x6 + x7));
  if (s == 12345.678) out[blockIdx.x] = s;   /* keeps the chains alive */
}

extern "C" double rodas3_fp64_peak_tflops(void) {
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return -1.0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return -1.0;
  double* out = nullptr;
  const int blocks = sms * 8;
  if (cudaMalloc(&out, blocks * sizeof(double)) != cudaSuccess) return -1.0;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int iters = 4096;
  fp64_probe<<<blocks, 256>>>(out, 64, 0.999999, 1e-9);   /* warm-up */
  float best = 1e30f;
  for (int r = 0; r < 5; ++r) {
    cudaEventRecord(e0);
    fp64_probe<<<blocks, 256>>>(out, iters, 0.999999, 1e-9);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms < best) best = ms;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  if (cudaGetLastError() != cudaSuccess) return -1.0;
  const double flops = 2.0 * 8 * 16 * (double)iters * blocks * 256;
  return flops / (best * 1e-3) / 1e12;
}

/* ---------------------------------------------------------------------- */
/* Phase micro-benchmark: `reps` calls of one building block per thread on
   the warp-tiled workspace (filled with benign values first), so the cost
   of Fun / Jac / factorisation / solve can be measured separately.
   phase: 0 Fun, 1 Jac, 2 fused prep+LU (-2: not generated), 3 solve,
   4 indexed prep+KppDecomp. */
__global__ void __launch_bounds__(128) phase_fill(double* ws, long slots) {
  const long slot = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (slot >= slots) return;
  double* Y = slot_ptr(ws, slot, OFF_Y);
  for (int i = 0; i < NVAR + NFIX; ++i) Y[i * LANES] = 1.0e6 * (1.0 + 0.001 * (i % 7));
  double* R = slot_ptr(ws, slot, OFF_RCT);
  for (int j = 0; j < NREACT; ++j) R[j * LANES] = 1.0e-12 * (1.0 + 0.01 * (j % 13));
}

__global__ void __launch_bounds__(128) phase_run(double* ws, long slots, int phase, int reps) {
  const long slot = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (slot >= slots) return;
  double* Y = slot_ptr(ws, slot, OFF_Y);
  const double* F = slot_ptr(ws, slot, OFF_FIX);
  const double* R = slot_ptr(ws, slot, OFF_RCT);
  double* K = slot_ptr(ws, slot, OFF_K);
  double* J0 = slot_ptr(ws, slot, OFF_JAC0);
  double* G = slot_ptr(ws, slot, OFF_GHIMJ);
  double* W = slot_ptr(ws, slot, OFF_W);
  for (int r = 0; r < reps; ++r) {
    if (phase == 0) mech_fun(Y, F, R, K);
    else if (phase == 1) mech_jac(Y, F, R, J0);
    else if (phase == 2) mech_prep_decomp(J0, G, W, 1.0e-3);
#if defined(GC_LU_RECIP) && GC_LU_RECIP && MECH_FUSED_LU
    else if (phase == 3) mech_solve_recip(G, W, K);  /* W: 1/U(i,i) from phase 2 */
#else
    else if (phase == 3) mech_solve(G, K);
#endif
    else kpp_prep_decomp(J0, G, W, slot_ptr(ws, slot, OFF_YNEW), 1.0e-3);
  }
}

extern "C" double rodas3_phase_ms(int phase, long slots, int reps, double* ws) {
  const int threads = 128;
  const int blocks = (int)((slots + threads - 1) / threads);
  phase_fill<<<blocks, threads>>>(ws, slots);
  /* prime J0/G/K so the factorisation and solves see finite data */
  phase_run<<<blocks, threads>>>(ws, slots, 1, 1);
#if MECH_FUSED_LU
  phase_run<<<blocks, threads>>>(ws, slots, 2, 1);
#else
  if (phase == 2) return -2.0;    /* no fused LU generated for this mechanism */
  phase_run<<<blocks, threads>>>(ws, slots, 4, 1);
#endif
  phase_run<<<blocks, threads>>>(ws, slots, 0, 1);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0);
  phase_run<<<blocks, threads>>>(ws, slots, phase, reps);
  cudaEventRecord(e1);
  cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (cudaGetLastError() != cudaSuccess) return -1.0;
  return ms;
}

/* ---------------------------------------------------------------------- */
/* Allocation-free solve.
   Some callers cannot allocate device memory at the moment they need the
   chemistry solved: a model whose GPU memory is handed out up front by its
   own pool, or a host thread that must not call cudaMalloc/cudaFree (they
   synchronise the whole device and stall every other stream).  For them
   this entry point solves up to NOALLOC_MAX_CELLS cells with the
   one-thread-per-cell kernel, its solver workspace taken from a fixed array
   in the library's device image instead of the per-device pool.  The array
   is held on every GPU that loads the library, for as long as the process
   lives: NOALLOC_MAX_CELLS * WS_ELEMS doubles (about 32 MB for fullchem).
   All calls on a device share that one array, which keeps the previous
   call's contents: calls whose work overlaps on the GPU (for instance on two
   streams) race and corrupt each other, so order them on one stream.  Every
   workspace entry the kernel reads it has written earlier in the same call,
   so nothing needs clearing between calls. */
#define NOALLOC_MAX_CELLS 256
static __device__ __align__(256) double g_noalloc_ws[(size_t)NOALLOC_MAX_CELLS * WS_ELEMS];

/* device address of g_noalloc_ws, looked up once per device (in host code the
   symbol itself is only a host-side stand-in, not a device address).  Each
   device's entry is written and read under that device's mutex, so host
   threads making their first call on one device at the same time do not
   race.  The cached address belongs to the device's primary context: after
   cudaDeviceReset on that device it is stale, and a process that resets a
   device must not call this entry point on it again. */
static std::mutex g_noalloc_mu[64];
static double* g_noalloc_addr[64];

static double* noalloc_workspace(int dev) {
  std::lock_guard<std::mutex> lock(g_noalloc_mu[dev]);
  if (g_noalloc_addr[dev] == nullptr) {
    /* first call on this device: resolve the array's device address with the
       device current (make this first call before any stream capture) */
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_ws) != cudaSuccess || p == nullptr) {
      cudaGetLastError();
      return nullptr;
    }
    g_noalloc_addr[dev] = (double*)p;
  }
  return g_noalloc_addr[dev];
}

extern "C" int gcchem_b200_integrate_device_noalloc(
    int nCell, double Tstart, double Tend, double* C, const double* RCONST,
    const double* ATOL, const double* RTOL, const int* ICNTRL, const double* RCNTRL,
    const int* order, int* ISTAT, double* RSTAT, int* IERR, void* stream) {
  if (nCell <= 0) return 0;
  if (nCell > NOALLOC_MAX_CELLS) return -4;   /* more cells than the fixed workspace holds */
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return -1;
  double* ws = noalloc_workspace(dev);
  if (ws == nullptr) return -1;
  BatchArgs a;
  a.ncell = nCell; a.tstart = Tstart; a.tend = Tend;
  a.C = C; a.RCONST = RCONST; a.ATOL = ATOL; a.RTOL = RTOL;
  a.ICNTRL = ICNTRL; a.RCNTRL = RCNTRL; a.order = order;
  a.ISTAT = ISTAT; a.RSTAT = RSTAT; a.IERR = IERR;
  a.ws = ws;
  a.qhead = nullptr;
  a.nfail = nullptr;
  a.ATOLr = nullptr;
  a.RTOLr = nullptr;
  a.ckpt = nullptr;
  a.ckpt_max = 0;
  const int threads = 128;
  rodas3_plain<<<(nCell + threads - 1) / threads, threads, 0, (cudaStream_t)stream>>>(a, 0, nCell);
  /* peek, not get: an error left pending by the caller's earlier work is
     reported here as -3 too, but stays pending for the caller to read */
  return cudaPeekAtLastError() == cudaSuccess ? 0 : -3;
}
