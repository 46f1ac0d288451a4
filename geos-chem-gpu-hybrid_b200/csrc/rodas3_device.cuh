/*
 * rodas3_device.cuh -- device-side layout and building blocks of the batched
 * Rodas3 solve (one CUDA thread per grid cell).
 *
 * Workspace layout ("warp-tiled interleaved"): every solver thread owns one
 * workspace slot.  The slots of one warp form a contiguous region; inside it
 * element e of every per-cell array sits at a fixed offset, the 32 lanes'
 * copies of that element side by side:
 *
 *     addr(slot s, array off_a, element e) =
 *         ws + ((s / 32) * WS_ELEMS + off_a + e) * 32 + (s % 32)
 *
 * so a warp touching the same element of its 32 cells issues one 256-byte
 * coalesced access, and the element stride is the compile-time constant 32.
 * The generated statement lists (fun.inc, jac.inc, solve.inc, lu.inc) address
 * arrays through the accessor macros defined here.
 *
 * Sizes: NVAR variable species, NFIX fixed, NREACT reactions, NNZ entries of
 * the LU pattern (with fill-in), NB Jacobian partials -- all from mech.h.
 */
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "mech.h"

#define NVAR MECH_NVAR
#define NFIX MECH_NFIX
#define NSPEC MECH_NSPEC
#define NREACT MECH_NREACT
#define NNZ MECH_NNZ
#define NB MECH_NB

#define LANES 32

/* compiler-only memory barrier placed by the code generator between groups
   of statements: bounds register live ranges, emits no instruction */
#define GC_FENCE() asm volatile("" ::: "memory")
#define GC_ROW_FENCE() GC_FENCE()

/* Global loads with a cache hint, for workspace arrays that a thread reads
   once per call and that its L1 share cannot keep between calls:
   kind 0 a plain load, 1 cache-global (L2 only, __ldcg), 2 streaming
   (__ldcs), 3 last use (__ldlu).  The value loaded is the same. */
#define GC_LD(kind, p) ((kind) == 1 ? __ldcg(p) : (kind) == 2 ? __ldcs(p) : \
                        (kind) == 3 ? __ldlu(p) : *(p))

/* per-slot workspace (in elements) -------------------------------------- */
#define OFF_Y      0                        /* Y(NVAR): current solution   */
#define OFF_FIX    (OFF_Y + NVAR)           /* FIX(NFIX)                   */
#define OFF_RCT    (OFF_FIX + NFIX)         /* RCONST(NREACT)              */
#define OFF_YNEW   (OFF_RCT + NREACT)       /* Ynew(NVAR)                  */
#define OFF_FCN0   (OFF_YNEW + NVAR)        /* Fcn0(NVAR)                  */
#define OFF_DFDT   (OFF_FCN0 + NVAR)        /* dFdT(NVAR)                  */
#define OFF_W      (OFF_DFDT + NVAR)        /* KppDecomp row scratch W     */
#define OFF_K      (OFF_W + NVAR)           /* Kw(4*NVAR): stage vectors   */
#define OFF_JAC0   (OFF_K + 4 * NVAR)       /* Jac0(NNZ)                   */
#define OFF_GHIMJ  (OFF_JAC0 + NNZ)         /* Ghimj(NNZ): LU factors      */
#define WS_ELEMS   (OFF_GHIMJ + NNZ)

/* pointer to element 0 of array `off` of the calling thread's slot */
__device__ __forceinline__ double* slot_ptr(double* ws, long slot, int off) {
  return ws + ((slot >> 5) * (long)WS_ELEMS + off) * LANES + (slot & 31);
}

/* Fortran MAX/MIN on REAL: IEEE maxNum/minNum (gfortran >= 8 behaviour) */
__device__ __forceinline__ double fmaxF(double a, double b) { return fmax(a, b); }
__device__ __forceinline__ double fminF(double a, double b) { return fmin(a, b); }

/* Rodas3 tableau (gckpp_BatchIntegrator.F90:443-452) */
#define ROS_ELO 3.0
#define ROUNDOFF 2.220446049250313080847263336181640625e-16 /* 2**-52 */
#define DELTAMIN 1.0e-5

/* generated mechanism routines (one translation unit each) ---------------- */
/* Fun_SPLIT(V, F, RCT, Vdot): arrays are slot pointers (element stride 32) */
extern __device__ __noinline__ void mech_fun(const double* __restrict__ V,
                                             const double* __restrict__ F,
                                             const double* __restrict__ RCT,
                                             double* __restrict__ Vdot);
/* Jac_SP(V, F, RCT, JVS) */
extern __device__ __noinline__ void mech_jac(const double* __restrict__ V,
                                             const double* __restrict__ F,
                                             const double* __restrict__ RCT,
                                             double* __restrict__ JVS);
/* ros_PrepareMatrix + KppDecomp: G = LU(-J0 + ghinv I); returns KppDecomp's
   IER (0 = factored).  W: an NVAR scratch array of the slot (pivot
   reciprocals in the FMA build) */
extern __device__ __noinline__ int mech_prep_decomp(const double* __restrict__ J0,
                                                    double* __restrict__ G,
                                                    double* __restrict__ W,
                                                    double ghinv);
/* ros_PrepareMatrix + KppDecomp on the LU tables (the indexed form, every
   mechanism): G = LU(-J0 + ghinv*I), W the row scratch, Rs an NVAR array
   free during the call.  Returns 0, or k+1 when the k-th diagonal of
   -J0 + ghinv is below DBL_MIN.  With GC_IRECIP the multipliers use
   reciprocal pivots and W returns 1/U(i,i). */
#ifndef GC_INDEXED_RECIP
#define GC_INDEXED_RECIP 1
#endif
#if defined(GC_LU_RECIP) && GC_LU_RECIP && GC_INDEXED_RECIP
#define GC_IRECIP 1
#else
#define GC_IRECIP 0
#endif
extern __device__ __noinline__ int kpp_prep_decomp(const double* __restrict__ J0,
                                                   double* __restrict__ G,
                                                   double* __restrict__ W,
                                                   double* __restrict__ Rs, double ghinv);
/* KppSolve(JVS, X) */
extern __device__ __noinline__ void mech_solve(const double* __restrict__ JVS,
                                               double* __restrict__ X);
/* KppSolve with the backward divides replaced by products with R = 1/U(i,i),
   which the FMA build's factorisation leaves in the slot's W array */
extern __device__ __noinline__ void mech_solve_recip(const double* __restrict__ JVS,
                                                     const double* __restrict__ R,
                                                     double* __restrict__ X);

/* per-cell status kept by the solver (ISTAT(1:8), RSTAT(1:3) semantics of
   gckpp_BatchIntegrator.F90:413-420) */
struct CellStat {
  int nfun, njac, nstp, nacc, nrej, ndec, nsol, nsng;
  double texit, hexit, hnew;
};

/* options after the gpu_solve_cell merge (gc_gpu_batch_api.F90:79-86) and
   the Integrate_Cell_S decode (gckpp_BatchIntegrator.F90:467-518) */
struct CellOpts {
  int ierr_early;   /* 0, or -90 / -2 when the options are rejected */
  int autonomous, vectortol, clamp, max_steps;
  double hmin, hmax, hstart, facmin, facmax, facrej, facsafe;
};

/* zero_hstart: ignore the caller's RCNTRL(3) (the retry protocol zeroes
   Hstart before the second launch, fullchem_mod.F90:2467) */
__device__ __forceinline__ CellOpts decode_options(const int* icntrl_u,
                                                   const double* rcntrl_u,
                                                   double Tstart, double Tend,
                                                   int zero_hstart = 0) {
  int ic[20];
  double rc[20];
#pragma unroll
  for (int k = 0; k < 20; ++k) { ic[k] = 0; rc[k] = 0.0; }
  ic[14] = 5;
#pragma unroll
  for (int k = 0; k < 20; ++k) {
    const int iu = icntrl_u[k];
    const double ru = rcntrl_u[k];
    if (iu != 0) ic[k] = iu;
    if (ru > 0.0) rc[k] = ru;
  }
  if (zero_hstart) rc[2] = 0.0;
  CellOpts o;
  o.ierr_early = 0;
  if (ic[11] == 1) o.ierr_early = -90;
  else if (!(ic[2] == 0 || ic[2] == 4)) o.ierr_early = -2;
  o.autonomous = !(ic[0] == 0);
  o.vectortol = (ic[1] == 0);
  o.clamp = (ic[15] == 1);
  o.max_steps = (ic[3] == 0) ? 200000 : ic[3];
  const double span = fabs(Tend - Tstart);
  o.hmin = (rc[0] > 0.0) ? rc[0] : 0.0;
  o.hmax = (rc[1] > 0.0) ? fminF(fabs(rc[1]), span) : span;
  o.hstart = (rc[2] > 0.0) ? fminF(fabs(rc[2]), span) : fmaxF(o.hmin, DELTAMIN);
  o.facmin = (rc[3] > 0.0) ? rc[3] : 0.2;
  o.facmax = (rc[4] > 0.0) ? rc[4] : 6.0;
  o.facrej = (rc[5] > 0.0) ? rc[5] : 0.1;
  o.facsafe = (rc[6] > 0.0) ? rc[6] : 0.9;
  return o;
}
