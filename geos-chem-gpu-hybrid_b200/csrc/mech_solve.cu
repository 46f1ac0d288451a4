/*
 * mech_solve.cu -- KppSolve (gckpp_LinearAlgebra.F90:645-2311) for one cell
 * per thread on the warp-tiled workspace: forward unit-lower sweep, then the
 * backward upper sweep with the diagonal divide, term order of the
 * reference's generated code.
 */
#include "rodas3_device.cuh"

#define JVS_(k) JVS[(k) * LANES]
#define X_(i) X[(i) * LANES]
#define R_(i) R[(i) * LANES]

/* the reference's backward divide X(i) = (...)/JVS(diag i) */
#define GC_SDIV(x, d, i) ((x) / (d))
__device__ __noinline__ void mech_solve(const double* __restrict__ JVS,
                                        double* __restrict__ X) {
#include "solve.inc"
}
#undef GC_SDIV

#if defined(GC_LU_RECIP) && GC_LU_RECIP
/* FMA build after the reciprocal-pivot factorisation: R holds 1/JVS(diag i)
   for every row, and the backward sweep multiplies by it (one rounding
   apart from the divide) */
#define GC_SDIV(x, d, i) ((x) * R_(i))
__device__ __noinline__ void mech_solve_recip(const double* __restrict__ JVS,
                                              const double* __restrict__ R,
                                              double* __restrict__ X) {
#include "solve.inc"
}
#undef GC_SDIV
#endif
