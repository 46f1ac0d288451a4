/*
 * mech_lu.cu -- ros_PrepareMatrix + KppDecomp fused and unrolled over the
 * mechanism's LU pattern (gckpp_BatchIntegrator.F90:573-577 and
 * gckpp_LinearAlgebra.F90:46-84), one cell per thread on the warp-tiled
 * workspace.  lu_fused.inc is generated: each row of the factor is built in
 * registers (blocks of consecutive entries) from -Jac0 (+ghinv on the
 * diagonal), eliminated with the already-final U rows in the reference's
 * pivot order, and stored once.
 *
 * Returns 0, or k+1 when the k-th diagonal of -Jac0 + ghinv is below TINY
 * (DBL_MIN) -- the value KppDecomp's IER would report; nothing is factored
 * in that case.
 *
 * Multipliers: by default a = -(w / U(j,j)), the reference's divide, one per
 * L entry (2,773 in fullchem).  Built with GC_LU_RECIP=1 (the FMA library),
 * each finished row stores R(j) = 1/U(j,j) in the slot's NVAR scratch array
 * W and every multiplier is -(w * R(j)): 353 divides instead of 2,773, and a
 * multiply instead of a divide on the row's dependency chain.  The two forms
 * differ by at most about one rounding per multiplier, so only the bit-exact
 * (--fmad=false) build keeps the divide.
 */
#include <float.h>
#include "rodas3_device.cuh"

#define J0_(k) J0[(k) * LANES]
#define G_(k) G[(k) * LANES]
/* Finished factor entries (U rows, stored multipliers) are read through
   the L2 only: each is re-read by later rows of the same cell, long after
   its L1 line would have been evicted by the other 255 cells of the SM, and
   allocating it in L1 only displaced useful lines.  Full 4x5 grid solve:
   4.10 s with plain loads, 3.95 s cache-global, 3.99 s streaming, 4.02 s
   last-use; bit-identical results.  (The same hint on the solves' factor
   reads made the solve 15% slower: those reads do hit in L1.) */
#ifndef GC_HINT_LU
#define GC_HINT_LU 1
#endif
#define GU_(k) GC_LD(GC_HINT_LU, G + (k) * LANES)
#define R_(j) W[(j) * LANES]
#if defined(GC_LU_RECIP) && GC_LU_RECIP
#define GC_PIVOT(w, d, j) (-((w) * R_(j)))
#define GC_RECIP(j, dv) (R_(j) = 1.0 / (dv))
#else
#define GC_PIVOT(w, d, j) (-((w) / (d)))
#define GC_RECIP(j, dv) ((void)0)
#endif

__constant__ int c_diag_lu[NVAR] = MECH_LU_DIAG_INIT;

__device__ __noinline__ int mech_prep_decomp(const double* __restrict__ J0,
                                             double* __restrict__ G,
                                             double* __restrict__ W,
                                             double ghinv) {
  for (int i = 0; i < NVAR; ++i) {
    const int d = c_diag_lu[i];
    if (fabs((-J0[d * LANES]) + ghinv) < DBL_MIN) return i + 1;
  }
#if MECH_FUSED_LU
#include "lu_fused.inc"
  return 0;
#else
  /* not generated for this mechanism (the kernels use the indexed
     KppDecomp); never called */
  (void)G;
  (void)W;
  return -1;
#endif
}
