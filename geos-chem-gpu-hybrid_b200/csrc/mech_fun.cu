/*
 * mech_fun.cu -- Fun_SPLIT (gckpp_Function.F90:2170-5060) for one cell per
 * thread, on the warp-tiled workspace (element stride 32).  The statement
 * list fun.inc is generated from the reference's expression trees with the
 * Fortran association order preserved: the rates A(j) are scalars declared
 * next to the species that consume them, P_VAR and D_VAR are written inline
 * in each Vdot statement.
 */
#include "rodas3_device.cuh"

#define V_(i) V[(i) * LANES]
#define F_(i) F[(i) * LANES]
#define RCT_(j) RCT[(j) * LANES]
#define VDOT_(i) Vdot[(i) * LANES]
#define A_(j) a##j

__device__ __noinline__ void mech_fun(const double* __restrict__ V,
                                      const double* __restrict__ F,
                                      const double* __restrict__ RCT,
                                      double* __restrict__ Vdot) {
#include "fun.inc"
}
