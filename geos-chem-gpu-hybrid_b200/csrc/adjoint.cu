/*
 * adjoint.cu -- discrete adjoint of the Rodas3 solve (one thread per cell).
 *
 * The reference has no adjoint; its building blocks are KppSolveTR
 * (gckpp_LinearAlgebra.F90:2327-3701, column-oriented as KppSolveTRIndirect
 * :204-230), JacTR_SP_Vec (gckpp_Jacobian.F90:21793-22738) and the
 * stoichiometric matrix of CalcStoichNum (gckpp_Function.F90:7271-12790).
 *
 * The forward solve (gcchem_b200_integrate_device_ckpt) checkpoints, for every
 * accepted step n, the state y_n at the start of the step and the accepted
 * step size h_n.  With that step sequence frozen, one Rodas3 step is the map
 *     G = I/(h*gamma1) - J(y)
 *     G K1 = f(y)                         G K2 = f(y) + (c21/h) K1
 *     G K3 = f(Y3) + (c31 K1 + c32 K2)/h  G K4 = f(Y4) + (c41 K1 + c42 K2 + c43 K3)/h
 *     Y3 = y + a31 K1 + a32 K2,  Y4 = y + a41 K1 + a42 K2 + a43 K3
 *     y_{n+1} = y + m1 K1 + m2 K2 + m3 K3 + m4 K4
 * (gckpp_BatchIntegrator.F90:595-650, tableau :443-452).  Its exact adjoint,
 * given lambda = dL/dy_{n+1}: W_s = m_s lambda; for s = 4..1
 *     U_s   = G^{-T} W_s
 *     lambda_n += J(Y_s)^T U_s + d/dy [U_s^T J(y) K_s]
 *     W_j  += a_sj J(Y_s)^T U_s + (c_sj/h) U_s           (j < s)
 *     dL/dln k_j += (U_s . S_j) (A_j(Y_s) + dA_j(y) . K_s)
 * plus lambda_n += lambda (y_{n+1} = y_n + ...).  (Y_1 = Y_2 = y.)
 * For mass action A_j = c_j prod y_v, so J^T u, the Hessian term and the
 * rate-constant term come from one pass over the reactions with
 * t_j = u . S_j.
 */
#include <float.h>
#include "rodas3_device.cuh"
#include "adj.inc"
#include "rodas3_kernels.h"

__device__ const int d_adj_rct[NREACT] = ADJ_RCT_INIT;
__device__ const double d_adj_lit[NREACT] = ADJ_LIT_INIT;
__device__ const int d_adj_nv[NREACT] = ADJ_NV_INIT;
__device__ const int d_adj_v[3 * NREACT] = ADJ_V_INIT;
__device__ const int d_adj_f[2 * NREACT] = ADJ_F_INIT;
__device__ const int d_adj_sptr[NREACT + 1] = ADJ_SPTR_INIT;
__device__ const int d_adj_ssp[ADJ_NSTO] = ADJ_SSP_INIT;
__device__ const double d_adj_sval[ADJ_NSTO] = ADJ_SVAL_INIT;

/* adjoint workspace per slot (elements) */
#define A_Y    0
#define A_FIX  (A_Y + NVAR)
#define A_RCT  (A_FIX + NFIX)
#define A_J0   (A_RCT + NREACT)
#define A_G    (A_J0 + NNZ)
#define A_W    (A_G + NNZ)
#define A_K    (A_W + NVAR)
#define A_YS   (A_K + 4 * NVAR)
#define A_U    (A_YS + NVAR)
#define A_WV   (A_U + NVAR)
#define A_LAM  (A_WV + 4 * NVAR)
#define A_LAMN (A_LAM + NVAR)
#define A_VT   (A_LAMN + NVAR)
#define A_MU   (A_VT + NVAR)
#define A_ELEMS (A_MU + NREACT)

__device__ __forceinline__ double* aslot(double* ws, long slot, int off) {
  return ws + ((slot >> 5) * (long)A_ELEMS + off) * LANES + (slot & 31);
}

/* With the FMA build's fused factorisation, R (the slot's W array) holds
   1/U(i,i) and the U^T sweep multiplies by it, as the forward solves do;
   otherwise the reference's divide. */
#if defined(GC_LU_RECIP) && GC_LU_RECIP && (MECH_FUSED_LU || GC_IRECIP)
#define GC_SDIV(x, d, i) ((x) * R[(i) * LANES])
#else
#define GC_SDIV(x, d, i) ((x) / (d))
#endif
#define JVS_(k) JVS[(k) * LANES]
#define X_(i) X[(i) * LANES]
__device__ __noinline__ void adj_solve_tr(const double* __restrict__ JVS,
                                          const double* __restrict__ R,
                                          double* __restrict__ X) {
  (void)R;
#include "solve_tr.inc"
}
#undef JVS_
#undef X_
#undef GC_SDIV

/* forward stage solve of the recomputed step: the same KppSolve form as the
   forward kernel's, so the adjoint differentiates the map that ran */
__device__ __forceinline__ void adj_stage_solve(const double* G, const double* W, double* X) {
#if defined(GC_LU_RECIP) && GC_LU_RECIP && (MECH_FUSED_LU || GC_IRECIP)
  mech_solve_recip(G, W, X);
#else
  (void)W;
  mech_solve(G, X);
#endif
}

/* One pass over the reactions for stage s:
     VT   = J(Yev)^T U                       (VT overwritten)
     LAMN += d/dy [U^T J(Yb) K]             (Hessian term at the step start)
     MU_j += (U.S_j) (A_j(Yev) + dA_j(Yb).K) (rate-constant gradient) */
__device__ __noinline__ void adj_react(const double* __restrict__ Yev, const double* __restrict__ Yb,
                                       const double* __restrict__ Ks, const double* __restrict__ U,
                                       const double* __restrict__ F, const double* __restrict__ R,
                                       double* __restrict__ VT, double* __restrict__ LAMN,
                                       double* __restrict__ MU) {
  for (int i = 0; i < NVAR; ++i) VT[i * LANES] = 0.0;
  for (int j = 0; j < NREACT; ++j) {
    double t = 0.0;
    const int q1 = d_adj_sptr[j + 1];
    for (int q = d_adj_sptr[j]; q < q1; ++q) t += d_adj_sval[q] * U[d_adj_ssp[q] * LANES];
    const int rj = d_adj_rct[j];
    double c = (rj >= 0) ? R[rj * LANES] : 1.0;
    c *= d_adj_lit[j];
    const int f0 = d_adj_f[2 * j], f1 = d_adj_f[2 * j + 1];
    if (f0 >= 0) c *= F[f0 * LANES];
    if (f1 >= 0) c *= F[f1 * LANES];
    const int nv = d_adj_nv[j];
    double a_ev, dak;
    if (nv == 0) {
      a_ev = c;
      dak = 0.0;
    } else if (nv == 1) {
      const int v0 = d_adj_v[3 * j];
      a_ev = c * Yev[v0 * LANES];
      dak = c * Ks[v0 * LANES];
      VT[v0 * LANES] += t * c;
    } else if (nv == 2) {
      const int v0 = d_adj_v[3 * j], v1 = d_adj_v[3 * j + 1];
      const double ea = Yev[v0 * LANES], eb = Yev[v1 * LANES];
      a_ev = c * ea * eb;
      VT[v0 * LANES] += t * c * eb;
      VT[v1 * LANES] += t * c * ea;
      const double za = Yb[v0 * LANES], zb = Yb[v1 * LANES];
      const double ka = Ks[v0 * LANES], kb = Ks[v1 * LANES];
      dak = c * (ka * zb + kb * za);
      LAMN[v1 * LANES] += t * c * ka;
      LAMN[v0 * LANES] += t * c * kb;
    } else {
      const int v0 = d_adj_v[3 * j], v1 = d_adj_v[3 * j + 1], v2 = d_adj_v[3 * j + 2];
      const double ea = Yev[v0 * LANES], eb = Yev[v1 * LANES], ec = Yev[v2 * LANES];
      a_ev = c * ea * eb * ec;
      VT[v0 * LANES] += t * c * eb * ec;
      VT[v1 * LANES] += t * c * ea * ec;
      VT[v2 * LANES] += t * c * ea * eb;
      const double za = Yb[v0 * LANES], zb = Yb[v1 * LANES], zc = Yb[v2 * LANES];
      const double ka = Ks[v0 * LANES], kb = Ks[v1 * LANES], kc = Ks[v2 * LANES];
      dak = c * (ka * zb * zc + kb * za * zc + kc * za * zb);
      /* d/dy of dak: d/dza = c(kb zc + kc zb), d/dzb = c(ka zc + kc za), d/dzc = c(ka zb + kb za) */
      LAMN[v0 * LANES] += t * c * (kb * zc + kc * zb);
      LAMN[v1 * LANES] += t * c * (ka * zc + kc * za);
      LAMN[v2 * LANES] += t * c * (ka * zb + kb * za);
    }
    if (rj >= 0) MU[j * LANES] += t * (a_ev + dak);
  }
}

struct AdjArgs {
  int ncell;
  const double* C0;      /* (NSPEC, n): initial concentrations (FIX rows used) */
  const double* RCONST;  /* (NREACT, n) */
  const int* ISTAT;      /* (8, n): forward counters, ISTAT(4) = accepted steps */
  const double* ckpt;    /* (ckpt_max*(NVAR+1), n): y_n and h_n per accepted step */
  int ckpt_max;
  const double* lam;     /* (NSPEC, n): dL/dC at the end of the step */
  double* gC0;           /* (NSPEC, n): dL/dC0 (FIX rows 0) */
  double* gK;            /* (NREACT, n): dL/d ln RCONST */
  int* ierr;             /* (n): 1, or -101 checkpoint overflow, -8 singular */
  double* ws;
  const int* order;      /* cells in launch order (descending accepted steps), or NULL */
};

__global__ void __launch_bounds__(128) rodas3_adjoint(AdjArgs a, int first, int count) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= count) return;
  /* with the cells in descending order of accepted steps, the lanes of a
     warp walk back similar step counts instead of idling behind the longest
     cell of a random group of 32 */
  const long col = a.order ? a.order[first + t] : first + t;
  const long slot = t;
  double* ws = a.ws;
  double* Y = aslot(ws, slot, A_Y);
  double* F = aslot(ws, slot, A_FIX);
  double* R = aslot(ws, slot, A_RCT);
  double* J0 = aslot(ws, slot, A_J0);
  double* G = aslot(ws, slot, A_G);
  double* W = aslot(ws, slot, A_W);
  double* K1 = aslot(ws, slot, A_K);
  double* K2 = K1 + NVAR * LANES;
  double* K3 = K1 + 2 * NVAR * LANES;
  double* K4 = K1 + 3 * NVAR * LANES;
  double* YS = aslot(ws, slot, A_YS);
  double* U = aslot(ws, slot, A_U);
  double* W1 = aslot(ws, slot, A_WV);
  double* W2 = W1 + NVAR * LANES;
  double* W3 = W1 + 2 * NVAR * LANES;
  double* W4 = W1 + 3 * NVAR * LANES;
  double* LAM = aslot(ws, slot, A_LAM);
  double* LAMN = aslot(ws, slot, A_LAMN);
  double* VT = aslot(ws, slot, A_VT);
  double* MU = aslot(ws, slot, A_MU);

  const double* c0 = a.C0 + col * NSPEC;
  for (int i = 0; i < NFIX; ++i) F[i * LANES] = c0[NVAR + i];
  const double* r = a.RCONST + col * NREACT;
  for (int j = 0; j < NREACT; ++j) { R[j * LANES] = r[j]; MU[j * LANES] = 0.0; }
  const double* lam = a.lam + col * NSPEC;
  for (int i = 0; i < NVAR; ++i) LAM[i * LANES] = lam[i];
  int ierr = 1;
  const int nacc = a.ISTAT[col * 8 + 3];
  if (nacc > a.ckpt_max) ierr = -101;
  for (int n = (ierr == 1 ? nacc - 1 : -1); n >= 0; --n) {
    const double* ck = a.ckpt + ((long)col * a.ckpt_max + n) * (NVAR + 1);
    for (int i = 0; i < NVAR; ++i) Y[i * LANES] = ck[i];
    const double h = ck[NVAR];
    /* forward stages of the accepted step */
    mech_jac(Y, F, R, J0);
    const double ghinv = 1.0 / (h * 0.5);
#if MECH_FUSED_LU
    const int ising = mech_prep_decomp(J0, G, W, ghinv);
#else
    const int ising = kpp_prep_decomp(J0, G, W, YS, ghinv);   /* YS is written later */
#endif
    if (ising != 0) { ierr = -8; break; }
    mech_fun(Y, F, R, K1);
    for (int k = 0; k < NVAR; ++k) K2[k * LANES] = K1[k * LANES];    /* K2 <- f(y) for now */
    adj_stage_solve(G, W, K1);
    const double hc21 = 4.0 / h;
    for (int k = 0; k < NVAR; ++k) K2[k * LANES] = K2[k * LANES] + hc21 * K1[k * LANES];
    adj_stage_solve(G, W, K2);
    for (int k = 0; k < NVAR; ++k)
      YS[k * LANES] = (Y[k * LANES] + 2.0 * K1[k * LANES]) + 0.0 * K2[k * LANES];
    mech_fun(YS, F, R, K3);
    const double hc1 = 1.0 / h, hc2 = -1.0 / h, hc3 = -(8.0 / 3.0) / h;
    for (int k = 0; k < NVAR; ++k)
      K3[k * LANES] = (K3[k * LANES] + hc1 * K1[k * LANES]) + hc2 * K2[k * LANES];
    adj_stage_solve(G, W, K3);
    for (int k = 0; k < NVAR; ++k)
      YS[k * LANES] = ((Y[k * LANES] + 2.0 * K1[k * LANES]) + 0.0 * K2[k * LANES]) + 1.0 * K3[k * LANES];
    mech_fun(YS, F, R, K4);
    for (int k = 0; k < NVAR; ++k)
      K4[k * LANES] = ((K4[k * LANES] + hc1 * K1[k * LANES]) + hc2 * K2[k * LANES]) + hc3 * K3[k * LANES];
    adj_stage_solve(G, W, K4);

    /* adjoint of the step: W_s = m_s lambda, m = (2, 0, 1, 1) */
    for (int k = 0; k < NVAR; ++k) {
      const double l = LAM[k * LANES];
      W1[k * LANES] = 2.0 * l;
      W2[k * LANES] = 0.0;
      W3[k * LANES] = l;
      W4[k * LANES] = l;
      LAMN[k * LANES] = l;
    }
    /* stage 4 (YS holds Y4) */
    for (int k = 0; k < NVAR; ++k) U[k * LANES] = W4[k * LANES];
    adj_solve_tr(G, W, U);
    adj_react(YS, Y, K4, U, F, R, VT, LAMN, MU);
    for (int k = 0; k < NVAR; ++k) {
      const double v = VT[k * LANES], u = U[k * LANES];
      LAMN[k * LANES] += v;
      W1[k * LANES] += 2.0 * v + hc1 * u;
      W2[k * LANES] += hc2 * u;
      W3[k * LANES] += v + hc3 * u;
    }
    /* stage 3 (Y3 = y + 2 K1) */
    for (int k = 0; k < NVAR; ++k)
      YS[k * LANES] = (Y[k * LANES] + 2.0 * K1[k * LANES]) + 0.0 * K2[k * LANES];
    for (int k = 0; k < NVAR; ++k) U[k * LANES] = W3[k * LANES];
    adj_solve_tr(G, W, U);
    adj_react(YS, Y, K3, U, F, R, VT, LAMN, MU);
    for (int k = 0; k < NVAR; ++k) {
      const double v = VT[k * LANES], u = U[k * LANES];
      LAMN[k * LANES] += v;
      W1[k * LANES] += 2.0 * v + hc1 * u;
      W2[k * LANES] += hc2 * u;
    }
    /* stage 2 (right-hand side f(y) + (4/h) K1) */
    for (int k = 0; k < NVAR; ++k) U[k * LANES] = W2[k * LANES];
    adj_solve_tr(G, W, U);
    adj_react(Y, Y, K2, U, F, R, VT, LAMN, MU);
    for (int k = 0; k < NVAR; ++k) {
      LAMN[k * LANES] += VT[k * LANES];
      W1[k * LANES] += hc21 * U[k * LANES];
    }
    /* stage 1 (right-hand side f(y)) */
    for (int k = 0; k < NVAR; ++k) U[k * LANES] = W1[k * LANES];
    adj_solve_tr(G, W, U);
    adj_react(Y, Y, K1, U, F, R, VT, LAMN, MU);
    for (int k = 0; k < NVAR; ++k) LAM[k * LANES] = LAMN[k * LANES] + VT[k * LANES];
  }
  double* g = a.gC0 + col * NSPEC;
  for (int i = 0; i < NVAR; ++i) g[i] = (ierr == 1) ? LAM[i * LANES] : NAN;
  for (int i = 0; i < NFIX; ++i) g[NVAR + i] = 0.0;
  double* gk = a.gK + col * NREACT;
  for (int j = 0; j < NREACT; ++j) gk[j] = (ierr == 1) ? MU[j * LANES] : NAN;
  a.ierr[col] = ierr;
}

extern "C" int rodas3_adjoint_ws_elems(void) { return A_ELEMS; }

/* sort keys: ISTAT(4), the accepted steps the backward sweep walks */
__global__ void adj_keys(const int* ISTAT, int n, int* keys) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) keys[i] = ISTAT[(long)i * 8 + 3];
}

extern "C" cudaError_t rodas3_adjoint_launch(int ncell, const double* C0, const double* RCONST,
                                             const int* ISTAT, const double* ckpt, int ckpt_max,
                                             const double* lam, double* gC0, double* gK,
                                             int* ierr, double* ws, long slots,
                                             int* sortbuf, unsigned long long* sortscratch,
                                             cudaStream_t s) {
  AdjArgs a;
  a.ncell = ncell; a.C0 = C0; a.RCONST = RCONST; a.ISTAT = ISTAT; a.ckpt = ckpt;
  a.ckpt_max = ckpt_max; a.lam = lam; a.gC0 = gC0; a.gK = gK; a.ierr = ierr; a.ws = ws;
  a.order = nullptr;
  if (sortbuf && sortscratch) {
    /* sortbuf: ncell keys, then ncell order entries */
    adj_keys<<<(ncell + 255) / 256, 256, 0, s>>>(ISTAT, ncell, sortbuf);
    const cudaError_t e = rodas3_cost_order(sortbuf, ncell, sortbuf + ncell, sortscratch, s);
    if (e != cudaSuccess) return e;
    a.order = sortbuf + ncell;
  }
  const int threads = 128;
  for (long first = 0; first < ncell; first += slots) {
    const int count = (int)((ncell - first) < slots ? (ncell - first) : slots);
    rodas3_adjoint<<<(count + threads - 1) / threads, threads, 0, s>>>(a, (int)first, count);
  }
  return cudaGetLastError();
}
