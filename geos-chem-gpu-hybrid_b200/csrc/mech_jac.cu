/*
 * mech_jac.cu -- Jac_SP (gckpp_Jacobian.F90:47-20887) for one cell per
 * thread on the warp-tiled workspace.  jac.inc is generated from the
 * reference's expression trees: each partial B(m) is a scalar declared just
 * before the first JVS(k) sum of its column that uses it.
 */
#include "rodas3_device.cuh"

#define V_(i) V[(i) * LANES]
#define F_(i) F[(i) * LANES]
#define RCT_(j) RCT[(j) * LANES]
#define JVS_(k) JVS[(k) * LANES]
#define B_(k) b##k

__device__ __noinline__ void mech_jac(const double* __restrict__ V,
                                      const double* __restrict__ F,
                                      const double* __restrict__ RCT,
                                      double* __restrict__ JVS) {
#include "jac.inc"
}
