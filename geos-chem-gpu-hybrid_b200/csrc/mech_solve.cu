/*
 * mech_solve.cu -- KppSolve (gckpp_LinearAlgebra.F90:645-2311) for one cell
 * per thread on the warp-tiled workspace: forward unit-lower sweep, then the
 * backward upper sweep with the diagonal divide, term order of the
 * reference's generated code.
 */
#include "rodas3_device.cuh"

#define JVS_(k) JVS[(k) * LANES]
#define X_(i) X[(i) * LANES]

__device__ __noinline__ void mech_solve(const double* __restrict__ JVS,
                                        double* __restrict__ X) {
#include "solve.inc"
}
