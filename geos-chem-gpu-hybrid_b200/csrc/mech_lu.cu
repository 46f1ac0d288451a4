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
 */
#include <float.h>
#include "rodas3_device.cuh"

#define J0_(k) J0[(k) * LANES]
#define G_(k) G[(k) * LANES]

__constant__ int c_diag_lu[NVAR] = MECH_LU_DIAG_INIT;

__device__ __noinline__ int mech_prep_decomp(const double* __restrict__ J0,
                                             double* __restrict__ G,
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
  return -1;
#endif
}
