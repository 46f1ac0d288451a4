/*
 * gencheck.cpp -- TEST INFRASTRUCTURE ONLY.
 *
 * Compiles the product-side generated statement lists that have no
 * counterpart in the oracle (the fused, register-blocked factorisation
 * lu_fused.inc) with plain host arrays, so the tests can compare them bit
 * for bit against the oracle's indexed KppDecomp on the CPU before any GPU
 * run.  Built with the oracle's flags (-O2 -ffp-contract=off).
 *
 * gencheck_prep_decomp_recip compiles the same statements with the FMA
 * library's multiplier form (one reciprocal 1/U(j,j) per row, stored in W),
 * so the tests can bound how far that form moves the factors.
 */
#include <math.h>
#include <float.h>
#include "mech.h"

#define NVAR MECH_NVAR
#define LANES 1
#define J0_(k) J0[k]
#define G_(k) G[k]
#define GU_(k) G[k]
#define GC_FENCE()
#define GC_ROW_FENCE()
#define GC_PIVOT(w, d, j) (-((w) / (d)))   /* the reference's divide */
#define GC_RECIP(j, dv) ((void)0)

extern "C" int gencheck_prep_decomp(const double* J0, double* G, double ghinv) {
  static const int diag[NVAR] = MECH_LU_DIAG_INIT;
  for (int i = 0; i < NVAR; ++i)
    if (fabs((-J0[diag[i]]) + ghinv) < DBL_MIN) return i + 1;
#if MECH_FUSED_LU
#include "lu_fused.inc"
  return 0;
#else
  (void)G;
  return -1;   /* this mechanism has no fused factorisation */
#endif
}

#undef GC_PIVOT
#undef GC_RECIP
#define R_(j) W[j]
#define GC_PIVOT(w, d, j) (-((w) * R_(j)))
#define GC_RECIP(j, dv) (R_(j) = 1.0 / (dv))

extern "C" int gencheck_prep_decomp_recip(const double* J0, double* G, double* W,
                                          double ghinv) {
  static const int diag[NVAR] = MECH_LU_DIAG_INIT;
  for (int i = 0; i < NVAR; ++i)
    if (fabs((-J0[diag[i]]) + ghinv) < DBL_MIN) return i + 1;
#if MECH_FUSED_LU
#include "lu_fused.inc"
  return 0;
#else
  (void)G;
  (void)W;
  return -1;
#endif
}
