/*
 * rodas3_oracle.cpp -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of the reference's batched Rodas3 solve, used as the
 * parity oracle by tests/, by __graft_entry__.smoke() and as the timed CPU
 * baseline by bench.py.  Nothing in the product path links or calls it.
 *
 * What it restates (paths relative to the reference checkout):
 *   - gpu_solve_cell option merging     gpulib/src/gc_gpu_batch_api.F90:54-110
 *   - Integrate_Cell_S (Rodas3 driver)  src/geos-chem/KPP/fullchem/gckpp_BatchIntegrator.F90:408-707
 *   - AddGhinvDiag                      gckpp_BatchIntegrator.F90:784-795
 *   - KppDecomp (indexed sparse LU)     src/geos-chem/KPP/fullchem/gckpp_LinearAlgebra.F90:46-84
 *   - Fun_SPLIT / Jac_SP / KppSolve     generated statement lists included below,
 *     emitted from the expression trees of gckpp_Function.F90:2170-5060,
 *     gckpp_Jacobian.F90:47-20887, gckpp_LinearAlgebra.F90:645-2311.
 *
 * Build: g++ -O2 -ffp-contract=off (no -ffast-math), which rounds like the
 * reference's gfortran -O2 x86-64 build (no FMA, left-to-right evaluation).
 * Fortran MAX/MIN are taken with IEEE maxNum/minNum semantics (fmax/fmin),
 * the behaviour of gfortran >= 8 for REAL arguments.  Err**(1/3) uses the
 * project's gc_pow (gc_pow.h), the same function the CUDA kernels use.
 *
 * The mechanism is selected by the include path: the directory holding its
 * generated mech.h, fun.inc, jac.inc and solve.inc.
 *
 * Parity status: weakly pinned.  The reference's Fortran cannot be compiled
 * here (no Fortran compiler), so the oracle is pinned by the reference's
 * one known answer (gc_gpu_selftest: rc = 1, 12 internal steps) and by its
 * parsed expression trees, evaluated independently in Python
 * (tests/golden/), not by running the reference itself.
 */
#include <math.h>
#include <stdint.h>
#include <string.h>
#include <stdlib.h>
#include <float.h>
#include <vector>
#include <omp.h>

#include "gc_pow.h"

/* Err**(1/ros_ELO) (gckpp_BatchIntegrator.F90:667).  The oracle uses the
   project's correctly rounded gc_pow, the function the CUDA kernels use.
   Built with -DORACLE_LIBM_POW it calls the host C library's pow instead,
   the function the reference's gfortran build calls there; that variant
   only measures how many cells the choice of pow changes. */
#ifdef ORACLE_LIBM_POW
static inline double step_pow(double x, double y) { return pow(x, y); }
#else
static inline double step_pow(double x, double y) { return gc_pow(x, y); }
#endif

#include "mech.h"

#define NVAR MECH_NVAR
#define NFIX MECH_NFIX
#define NSPEC MECH_NSPEC
#define NREACT MECH_NREACT
#define NNZ MECH_NNZ
#define NB MECH_NB
#define LU_CROW MECH_LU_CROW
#define LU_DIAG MECH_LU_DIAG
#define LU_ICOL MECH_LU_ICOL

#define V_(i) V[i]
#define F_(i) F[i]
#define RCT_(j) RCT[j]
#define A_(j) a##j
#define B_(k) b##k
#define VDOT_(i) Vdot[i]
#define JVS_(k) JVS[k]
#define X_(i) X[i]
#define GC_FENCE()
#define GC_ROW_FENCE()
#define GC_SDIV(x, d, i) ((x) / (d))   /* the reference's divide */

/* Fun_SPLIT(V, F, RCT, Vdot): the generated statements compute P_VAR and
   D_VAR inline in each Vdot(i) and hold the rates as scalars */
static void fun_split(const double* V, const double* F, const double* RCT,
                      double* Vdot) {
#include "fun.inc"
}

/* Jac_SP(V, F, RCT, JVS) */
static void jac_sp(const double* V, const double* F, const double* RCT,
                   double* JVS) {
#include "jac.inc"
}

/* KppSolve(JVS, X) */
static void kpp_solve(const double* JVS, double* X) {
#include "solve.inc"
}

/* KppDecomp(JVS, IER): gckpp_LinearAlgebra.F90:46-84, loop for loop */
static int kpp_decomp(double* JVS) {
  double W[NVAR];
  double a;
  for (int k = 0; k < NVAR; ++k) {
    if (fabs(JVS[LU_DIAG[k]]) < DBL_MIN) return k + 1; /* TINY(a) */
    for (int kk = LU_CROW[k]; kk < LU_CROW[k + 1]; ++kk) W[LU_ICOL[kk]] = JVS[kk];
    for (int kk = LU_CROW[k]; kk < LU_DIAG[k]; ++kk) {
      int j = LU_ICOL[kk];
      a = -(W[j] / JVS[LU_DIAG[j]]);
      W[j] = -a;
      for (int jj = LU_DIAG[j] + 1; jj < LU_CROW[j + 1]; ++jj)
        W[LU_ICOL[jj]] = W[LU_ICOL[jj]] + a * JVS[jj];
    }
    for (int kk = LU_CROW[k]; kk < LU_CROW[k + 1]; ++kk) JVS[kk] = W[LU_ICOL[kk]];
  }
  return 0;
}

static inline double fmaxF(double a, double b) { return fmax(a, b); }
static inline double fminF(double a, double b) { return fmin(a, b); }

/* Integrate_Cell_S: gckpp_BatchIntegrator.F90:408-707.  Workspace is
   routine-local (the Integrate_Cell_L / gpu_solve_cell pattern). */
static void integrate_cell_s(double* Y, const double* FIXc, const double* RCT,
                             double Tstart, double Tend, const double* AbsTol,
                             const double* RelTol, const int* ICNTRL,
                             const double* RCNTRL, int* ISTAT, double* RSTAT,
                             int* IERR_out) {
  static const double ros_A[6] = {0.0, 2.0, 0.0, 2.0, 0.0, 1.0};
  static const double ros_C[6] = {4.0, 1.0, -1.0, 1.0, -1.0, -(8.0 / 3.0)};
  static const int ros_NewF[4] = {1, 0, 1, 1};
  static const double ros_M[4] = {2.0, 0.0, 1.0, 1.0};
  static const double ros_E[4] = {0.0, 0.0, 0.0, 1.0};
  static const double ros_ELO = 3.0;
  static const double ros_Gamma[4] = {0.5, 1.5, 0.0, 0.0};
  const double ROUNDOFF = 2.220446049250313080847263336181640625e-16; /* 2**-52 */
  const double DELTAMIN = 1.0e-5;
  const double ZERO = 0.0, ONE = 1.0, HALF = 0.5;

  std::vector<double> ws(4 * NVAR + 2 * NNZ + 5 * NVAR);
  double* Kw = ws.data();
  double* Ghimj = Kw + 4 * NVAR;
  double* Jac0 = Ghimj + NNZ;
  double* Ynew = Jac0 + NNZ;
  double* Fcn0 = Ynew + NVAR;
  double* Fcn = Fcn0 + NVAR;
  double* dFdT = Fcn + NVAR;
  double* Yerr = dFdT + NVAR;

  int IERR = 0, Nsteps = 0;
  for (int s = 0; s < 8; ++s) ISTAT[s] = 0;
  for (int s = 0; s < 3; ++s) RSTAT[s] = ZERO;

  if (ICNTRL[11] == 1) { *IERR_out = -90; return; }
  const bool Autonomous = !(ICNTRL[0] == 0);
  const bool VectorTol = (ICNTRL[1] == 0);
  if (!(ICNTRL[2] == 0 || ICNTRL[2] == 4)) { *IERR_out = -2; return; }
  const int Max_no_steps = (ICNTRL[3] == 0) ? 200000 : ICNTRL[3];
  const double Hmin = (RCNTRL[0] > ZERO) ? RCNTRL[0] : ZERO;
  const double Hmax = (RCNTRL[1] > ZERO) ? fminF(fabs(RCNTRL[1]), fabs(Tend - Tstart))
                                         : fabs(Tend - Tstart);
  const double Hstart = (RCNTRL[2] > ZERO) ? fminF(fabs(RCNTRL[2]), fabs(Tend - Tstart))
                                           : fmaxF(Hmin, DELTAMIN);
  const double FacMin = (RCNTRL[3] > ZERO) ? RCNTRL[3] : 0.2;
  const double FacMax = (RCNTRL[4] > ZERO) ? RCNTRL[4] : 6.0;
  const double FacRej = (RCNTRL[5] > ZERO) ? RCNTRL[5] : 0.1;
  const double FacSafe = (RCNTRL[6] > ZERO) ? RCNTRL[6] : 0.9;

  double T = Tstart;
  double H = fminF(fmaxF(fabs(Hmin), fabs(Hstart)), fabs(Hmax));
  if (fabs(H) <= 10.0 * ROUNDOFF) H = DELTAMIN;
  const int Direction = (Tend >= Tstart) ? +1 : -1;
  const double Dir = (double)Direction;
  H = Dir * H;
  bool RejectLastH = false, RejectMoreH = false;

  while ((Direction > 0 && ((T - Tend) + ROUNDOFF <= ZERO)) ||
         (Direction < 0 && ((Tend - T) + ROUNDOFF <= ZERO))) {
    if (Nsteps > Max_no_steps) { *IERR_out = -6; return; }
    if (((T + 0.1 * H) == T) || (H <= ROUNDOFF)) { *IERR_out = -7; return; }
    H = fminF(H, fabs(Tend - T));

    fun_split(Y, FIXc, RCT, Fcn0);
    ISTAT[0] += 1;
    if (!Autonomous) {
      const double Delta = sqrt(ROUNDOFF) * fmaxF(1.0e-6, fabs(T));
      fun_split(Y, FIXc, RCT, dFdT);
      ISTAT[0] += 1;
      for (int k = 0; k < NVAR; ++k) dFdT[k] = (dFdT[k] - Fcn0[k]) / Delta;
    }
    jac_sp(Y, FIXc, RCT, Jac0);
    ISTAT[1] += 1;

    for (;;) { /* UntilAccepted */
      int Nconsecutive = 0;
      bool Singular = true;
      while (Singular) {
        for (int k = 0; k < NNZ; ++k) Ghimj[k] = -Jac0[k];
        const double ghinv = ONE / ((Dir * H) * ros_Gamma[0]);
        for (int i = 0; i < NVAR; ++i) Ghimj[LU_DIAG[i]] = Ghimj[LU_DIAG[i]] + ghinv;
        const int ising = kpp_decomp(Ghimj);
        ISTAT[5] += 1;
        if (ising == 0) {
          Singular = false;
        } else {
          ISTAT[7] += 1;
          Nconsecutive += 1;
          if (Nconsecutive <= 5) {
            H = H * HALF;
          } else {
            *IERR_out = -8;
            return;
          }
        }
      }

      for (int istage = 1; istage <= 4; ++istage) {
        const int ioffset = NVAR * (istage - 1);
        if (istage == 1) {
          for (int k = 0; k < NVAR; ++k) Fcn[k] = Fcn0[k];
        } else if (ros_NewF[istage - 1]) {
          for (int k = 0; k < NVAR; ++k) Ynew[k] = Y[k];
          for (int j = 1; j <= istage - 1; ++j) {
            const double aa = ros_A[(istage - 1) * (istage - 2) / 2 + j - 1];
            for (int k = 0; k < NVAR; ++k) Ynew[k] = Ynew[k] + aa * Kw[NVAR * (j - 1) + k];
          }
          fun_split(Ynew, FIXc, RCT, Fcn);
          ISTAT[0] += 1;
        }
        for (int k = 0; k < NVAR; ++k) Kw[ioffset + k] = Fcn[k];
        for (int j = 1; j <= istage - 1; ++j) {
          const double HC = ros_C[(istage - 1) * (istage - 2) / 2 + j - 1] / (Dir * H);
          for (int k = 0; k < NVAR; ++k)
            Kw[ioffset + k] = Kw[ioffset + k] + HC * Kw[NVAR * (j - 1) + k];
        }
        if (!Autonomous && ros_Gamma[istage - 1] != ZERO) {
          const double HG = (Dir * H) * ros_Gamma[istage - 1];
          for (int k = 0; k < NVAR; ++k) Kw[ioffset + k] = Kw[ioffset + k] + HG * dFdT[k];
        }
        kpp_solve(Ghimj, Kw + ioffset);
        ISTAT[6] += 1;
      }

      for (int k = 0; k < NVAR; ++k) Ynew[k] = Y[k];
      for (int j = 1; j <= 4; ++j)
        for (int k = 0; k < NVAR; ++k) Ynew[k] = Ynew[k] + ros_M[j - 1] * Kw[NVAR * (j - 1) + k];
      for (int k = 0; k < NVAR; ++k) Yerr[k] = ZERO;
      for (int j = 1; j <= 4; ++j)
        for (int k = 0; k < NVAR; ++k) Yerr[k] = Yerr[k] + ros_E[j - 1] * Kw[NVAR * (j - 1) + k];

      double Err = ZERO;
      for (int i = 0; i < NVAR; ++i) {
        const double Ymax = fmaxF(fabs(Y[i]), fabs(Ynew[i]));
        const double Scal = VectorTol ? AbsTol[i] + RelTol[i] * Ymax
                                      : AbsTol[0] + RelTol[0] * Ymax;
        const double q = Yerr[i] / Scal;
        Err = Err + q * q;
      }
      Err = sqrt(Err / (double)NVAR);
      Err = fmaxF(Err, 1.0e-10);

      const double Fac = fminF(FacMax, fmaxF(FacMin, FacSafe / step_pow(Err, ONE / ros_ELO)));
      double Hnew = H * Fac;

      Nsteps += 1;
      ISTAT[2] += 1;
      if ((Err <= ONE) || (H <= Hmin)) {
        ISTAT[3] += 1;
        if (ICNTRL[15] == 1) {
          for (int k = 0; k < NVAR; ++k) Y[k] = fmaxF(Ynew[k], ZERO);
        } else {
          for (int k = 0; k < NVAR; ++k) Y[k] = Ynew[k];
        }
        T = T + Dir * H;
        Hnew = fmaxF(Hmin, fminF(Hnew, Hmax));
        if (RejectLastH) Hnew = fminF(Hnew, H);
        RSTAT[1] = H;
        RSTAT[2] = Hnew;
        RSTAT[0] = T;
        RejectLastH = false;
        RejectMoreH = false;
        H = Hnew;
        break;
      } else {
        if (RejectMoreH) Hnew = H * FacRej;
        RejectMoreH = RejectLastH;
        RejectLastH = true;
        H = Hnew;
        if (ISTAT[3] >= 1) ISTAT[4] += 1;
      }
    }
  }
  (void)IERR;
  *IERR_out = 1;
}

/* gpu_solve_cell (gc_gpu_batch_api.F90:54-110): zeroed controls, default
   ICNTRL(15)=5, merge ICNTRL_U/=0 and RCNTRL_U>0, local copies, solve. */
static void solve_cell(double* Ycol, const double* FIXc, const double* RCT,
                       double Tstart, double Tend, const double* ATOL,
                       const double* RTOL, const int* ICNTRL_U,
                       const double* RCNTRL_U, int* ISTAT, double* RSTAT,
                       int* IERR) {
  int ICNTRL[20];
  double RCNTRL[20];
  for (int kk = 0; kk < 20; ++kk) { ICNTRL[kk] = 0; RCNTRL[kk] = 0.0; }
  ICNTRL[14] = 5;
  for (int kk = 0; kk < 20; ++kk) {
    if (ICNTRL_U[kk] != 0) ICNTRL[kk] = ICNTRL_U[kk];
    if (RCNTRL_U[kk] > 0.0) RCNTRL[kk] = RCNTRL_U[kk];
  }
  double Yl[NVAR], FIXl[NFIX > 0 ? NFIX : 1];
  for (int kk = 0; kk < NVAR; ++kk) Yl[kk] = Ycol[kk];
  for (int kk = 0; kk < NFIX; ++kk) FIXl[kk] = FIXc[kk];
  integrate_cell_s(Yl, FIXl, RCT, Tstart, Tend, ATOL, RTOL, ICNTRL, RCNTRL,
                   ISTAT, RSTAT, IERR);
  for (int kk = 0; kk < NVAR; ++kk) Ycol[kk] = Yl[kk];
}

extern "C" {

int oracle_sizes(int* nvar, int* nfix, int* nreact, int* nnz) {
  *nvar = NVAR; *nfix = NFIX; *nreact = NREACT; *nnz = NNZ;
  return 0;
}

/* gc_gpu_integrate_batch semantics on the host (Fortran layout: C(NSPEC,n),
   RCONST(NREACT,n), ICNTRL(20,n), RCNTRL(20,n), 1-based Perm; outputs at
   column Perm(ic)).  nthreads<=0 uses every OpenMP thread. */
void oracle_integrate_batch(int nCell, double Tstart, double Tend, double* C,
                            const double* RCONST, const double* ATOL,
                            const double* RTOL, const int* ICNTRL,
                            const double* RCNTRL, const int* Perm, int* ISTAT,
                            double* RSTAT, int* IERR, int nthreads) {
  if (nCell <= 0) return;
  if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 16) num_threads(nthreads)
  for (int ic = 0; ic < nCell; ++ic) {
    const long idx = (long)Perm[ic] - 1;
    solve_cell(C + idx * NSPEC, C + idx * NSPEC + NVAR, RCONST + idx * NREACT,
               Tstart, Tend, ATOL, RTOL, ICNTRL + idx * 20, RCNTRL + idx * 20,
               ISTAT + idx * 8, RSTAT + idx * 3, IERR + idx);
  }
}

/* Rodas3 over a frozen sequence of step sizes (no error control): the map
   whose exact derivatives the GPU adjoint computes.  Stage arithmetic as in
   integrate_cell_s (gckpp_BatchIntegrator.F90:595-650), autonomous form.
   Returns 0, or the 1-based step whose factorisation was singular. */
int oracle_integrate_frozen(const double* Y0, const double* FIXc, const double* RCT,
                            const double* hs, int nsteps, double* Yout) {
  std::vector<double> ws(4 * NVAR + 2 * NNZ + 2 * NVAR);
  double* Kw = ws.data();
  double* Jac0 = Kw + 4 * NVAR;
  double* G = Jac0 + NNZ;
  double* Ynew = G + NNZ;
  double* Fcn = Ynew + NVAR;
  std::vector<double> Y(Y0, Y0 + NVAR);
  for (int n = 0; n < nsteps; ++n) {
    const double H = hs[n];
    fun_split(Y.data(), FIXc, RCT, Fcn);
    jac_sp(Y.data(), FIXc, RCT, Jac0);
    for (int k = 0; k < NNZ; ++k) G[k] = -Jac0[k];
    const double ghinv = 1.0 / (H * 0.5);
    for (int i = 0; i < NVAR; ++i) G[LU_DIAG[i]] = G[LU_DIAG[i]] + ghinv;
    if (kpp_decomp(G) != 0) return n + 1;
    double* K1 = Kw; double* K2 = Kw + NVAR; double* K3 = Kw + 2 * NVAR; double* K4 = Kw + 3 * NVAR;
    for (int k = 0; k < NVAR; ++k) K1[k] = Fcn[k];
    kpp_solve(G, K1);
    for (int k = 0; k < NVAR; ++k) K2[k] = Fcn[k] + (4.0 / H) * K1[k];
    kpp_solve(G, K2);
    for (int k = 0; k < NVAR; ++k) Ynew[k] = (Y[k] + 2.0 * K1[k]) + 0.0 * K2[k];
    fun_split(Ynew, FIXc, RCT, K3);
    for (int k = 0; k < NVAR; ++k) K3[k] = (K3[k] + (1.0 / H) * K1[k]) + (-1.0 / H) * K2[k];
    kpp_solve(G, K3);
    for (int k = 0; k < NVAR; ++k) Ynew[k] = ((Y[k] + 2.0 * K1[k]) + 0.0 * K2[k]) + 1.0 * K3[k];
    fun_split(Ynew, FIXc, RCT, K4);
    for (int k = 0; k < NVAR; ++k)
      K4[k] = ((K4[k] + (1.0 / H) * K1[k]) + (-1.0 / H) * K2[k]) + (-(8.0 / 3.0) / H) * K3[k];
    kpp_solve(G, K4);
    for (int k = 0; k < NVAR; ++k)
      Y[k] = (((Y[k] + 2.0 * K1[k]) + 0.0 * K2[k]) + 1.0 * K3[k]) + 1.0 * K4[k];
  }
  for (int k = 0; k < NVAR; ++k) Yout[k] = Y[k];
  return 0;
}

void oracle_fun(const double* V, const double* F, const double* RCT, double* Vdot) {
  fun_split(V, F, RCT, Vdot);
}
void oracle_jac(const double* V, const double* F, const double* RCT, double* JVS) {
  jac_sp(V, F, RCT, JVS);
}
int oracle_decomp(double* JVS) { return kpp_decomp(JVS); }
void oracle_solve(const double* JVS, double* X) { kpp_solve(JVS, X); }
double oracle_pow(double x, double y) { return gc_pow(x, y); }
void oracle_lu_tables(int* crow, int* diag, int* icol) {
  for (int i = 0; i <= NVAR; ++i) crow[i] = LU_CROW[i];
  for (int i = 0; i < NVAR; ++i) diag[i] = LU_DIAG[i];
  for (int k = 0; k < NNZ; ++k) icol[k] = LU_ICOL[k];
}

}  /* extern "C" */
