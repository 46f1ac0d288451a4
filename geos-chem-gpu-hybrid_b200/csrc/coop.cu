/*
 * coop.cu -- the cooperative Rodas3 kernel: one thread block per cell, the
 * whole cell state in shared memory.
 *
 * The one-thread-per-cell kernels stream every cell's workspace (the LU
 * factors, the Jacobian, the stage vectors) through HBM, because 256 cells
 * per SM cannot keep 50-125 KB each on chip.  Here a block of 128 or 256
 * threads owns one cell at a time and keeps its factors G (NNZ doubles), the
 * state and stage vectors, the rate constants and a scratch array in shared
 * memory (69 KB for the 120-species synthetic mechanism, 94 KB for
 * fullchem), so the solve reads HBM only to load a cell and store its
 * result.  The block drains the same cost-ordered work queue as the
 * persistent kernel: thread 0 takes the next queue position, and the block
 * solves that cell to the end (with the in-place retry), then takes the next.
 *
 * Parallelism inside a cell comes from tables generated from the mechanism
 * (coop.inc, mechanism/coop.py):
 *   Fun      rates A(j) one per thread, then P_VAR/D_VAR/Vdot one species per
 *            thread (gckpp_Function.F90:2170-5060 expressions, same rounding);
 *   Jac      partials B(m), then entries JVS(k), written straight into the
 *            factor array as -JVS (+ 1/(H*gamma) on the diagonal); the
 *            Jacobian is recomputed at every attempt instead of being stored
 *            (Y is unchanged after a rejection, so it is the same Jacobian);
 *   KppDecomp right-looking: step j forms column j's multipliers, then
 *            applies pivot row j to every row below it at once; each entry
 *            gets its updates in the reference's order
 *            (gckpp_LinearAlgebra.F90:46-84), so the factors are identical;
 *   KppSolve forward sweep by columns, each row's terms in the reference's
 *            order (:645-2311); backward sweep by levels of rows in the
 *            reference's order (--fmad=false build), or by columns (FMA
 *            build: 120 parallel steps instead of a chain of every row's
 *            terms, the per-row order reversed).
 * Step-size control, counters, options and the retry protocol are the
 * arithmetic of Integrate_Cell_S (gckpp_BatchIntegrator.F90:408-707) and of
 * the model's retry (fullchem_mod.F90:2436-2520), computed redundantly by
 * every thread of the block so that every branch is block-uniform; the one
 * sequential sum (the error norm, in species order) is taken by thread 0.
 *
 * Built with --fmad=false this kernel reproduces the CPU oracle bit for bit,
 * as the one-thread-per-cell kernels do; the FMA build contracts into FMA
 * and forms the multipliers and the backward quotients from one reciprocal
 * per pivot (GC_IRECIP).
 *
 * Every __syncthreads() is reached by all threads of the block: loop bounds
 * come from the tables, and every branch around a barrier depends only on
 * values all threads hold identically (shared-memory words read after a
 * barrier, or scalars computed redundantly from them).  Nothing waits on
 * another block.
 */
#include <cuda_runtime.h>
#include <float.h>
#include <limits.h>
#include "rodas3_device.cuh"
#include "gc_pow.h"
#include "rodas3_kernels.h"
#include "coop.inc"

#if MECH_COOP

static __device__ const int coop_diag[NVAR] = MECH_LU_DIAG_INIT;
static __constant__ int coop_diag_c[NVAR] = MECH_LU_DIAG_INIT;   /* block-uniform reads */
static __device__ const int coop_crow[NVAR + 1] = MECH_LU_CROW_INIT;
static __device__ const int coop_icol[NNZ] = MECH_LU_ICOL_INIT;

/* shared-memory layout of one cell (in doubles) */
#define COOP_NFIX1 (NFIX > 0 ? NFIX : 1)
#define COOP_MAX2(a, b) ((a) > (b) ? (a) : (b))
#define COOP_NSCR COOP_MAX2(COOP_MAX2(NREACT, NB), NVAR)
#define SO_G     0
#define SO_Y0    (SO_G + NNZ)
#define SO_Y1    (SO_Y0 + NVAR)
#define SO_FCN0  (SO_Y1 + NVAR)
#define SO_DFDT  (SO_FCN0 + NVAR)
#define SO_K     (SO_DFDT + NVAR)
#define SO_R     (SO_K + 4 * NVAR)
#define SO_FIX   (SO_R + NVAR)
#define SO_RCT   (SO_FIX + COOP_NFIX1)
#define SO_S     (SO_RCT + NREACT)
#define SO_END   (SO_S + COOP_NSCR)

struct CoopArgs {
  int ncell;
  double tstart, tend;
  double* C;
  const double* RCONST;
  const double* ATOL;
  const double* RTOL;
  const int* ICNTRL;
  const double* RCNTRL;
  const int* order;
  int* ISTAT;
  double* RSTAT;
  int* IERR;
  unsigned int* qhead;
  int* nfail;
  const double* ATOLr;
  const double* RTOLr;
};

/* the cell's integrator state; every thread of the block holds the same */
struct CoopCell {
  long col;
  CellOpts o;
  CellStat st;
  double T, H;
  int nsteps, ncons, rej_last, rej_more, newstep, ierr, ysel, attempt;
};

/* one factor of a term: V, F, RCT, scratch (rates / partials) or a literal */
__device__ __forceinline__ double coop_factor(unsigned int code, const double* V,
                                              const double* F, const double* K,
                                              const double* S) {
  const unsigned int idx = code & 0x1FFFu;
  switch (code >> 13) {
    case 0: return V[idx];
    case 1: return F[idx];
    case 2: return K[idx];
    case 3: return S[idx];
    default: return __ldg(&coop_const[idx]);
  }
}

/* value of the terms q0 .. q1-1 of the tables: a signed left-to-right sum
   of products */
__device__ __forceinline__ double coop_terms(int q0, int q1, const double* V, const double* F,
                                             const double* K, const double* S) {
  const ushort4* fac = reinterpret_cast<const ushort4*>(coop_term_fac);
  double s = 0.0;
  for (int q = q0; q < q1; ++q) {
    const ushort4 f = __ldg(fac + q);
    const int op = __ldg(&coop_term_op[q]);
    double v = coop_factor(f.x, V, F, K, S);
    if (f.y != 0xFFFFu) v = v * coop_factor(f.y, V, F, K, S);
    if (f.z != 0xFFFFu) v = v * coop_factor(f.z, V, F, K, S);
    if (f.w != 0xFFFFu) v = v * coop_factor(f.w, V, F, K, S);
    s = (op == 0) ? v : (op == 1) ? -v : (op == 2) ? s + v : s - v;
  }
  return s;
}

/* value `sid` of the tables */
__device__ __forceinline__ double coop_sum(int sid, const double* V, const double* F,
                                           const double* K, const double* S) {
  return coop_terms(__ldg(&coop_sum_off[sid]), __ldg(&coop_sum_off[sid + 1]), V, F, K, S);
}

/* Fun_SPLIT: out = P_VAR - D_VAR*V */
__device__ __forceinline__ void coop_fun(const double* V, double* out, const double* F,
                                         const double* K, double* S) {
  for (int j = threadIdx.x; j < NREACT; j += blockDim.x)
    S[j] = coop_sum(COOP_SID_RATE + j, V, F, K, S);
  __syncthreads();
  for (int i = threadIdx.x; i < NVAR; i += blockDim.x) {
    const double p = coop_sum(COOP_SID_PROD + i, V, F, K, S);
    const double d = coop_sum(COOP_SID_DEST + i, V, F, K, S);
    out[i] = p - (d * V[i]);
  }
  __syncthreads();
}

/* Jac_SP straight into ros_PrepareMatrix's form: G = -JVS, plus ghinv on
   the diagonal.  KppDecomp's singularity test reads each prepared diagonal
   before its row is eliminated, so it is taken here: *ising becomes the
   lowest failing row + 1 (it holds INT_MAX on entry). */
__device__ __forceinline__ void coop_jac_prep(const double* V, const double* F,
                                              const double* K, double* S, double* G,
                                              double ghinv, int* ising) {
  for (int m = threadIdx.x; m < NB; m += blockDim.x)
    S[m] = coop_sum(COOP_SID_B + m, V, F, K, S);
  __syncthreads();
  /* the next entry's term range is loaded while the current one is summed */
  int q0 = 0, q1 = 0;
  if (threadIdx.x < NNZ) {
    q0 = __ldg(&coop_sum_off[COOP_SID_JVS + threadIdx.x]);
    q1 = __ldg(&coop_sum_off[COOP_SID_JVS + threadIdx.x + 1]);
  }
  for (int k = threadIdx.x; k < NNZ; k += blockDim.x) {
    const int c0 = q0, c1 = q1;
    if (k + blockDim.x < NNZ) {
      q0 = __ldg(&coop_sum_off[COOP_SID_JVS + k + blockDim.x]);
      q1 = __ldg(&coop_sum_off[COOP_SID_JVS + k + blockDim.x + 1]);
    }
    double g = -coop_terms(c0, c1, V, F, K, S);
    const int row = __ldg(&coop_kdiag[k]);
    if (row >= 0) {
      g = g + ghinv;
      if (fabs(g) < DBL_MIN) atomicMin(ising, row + 1);
    }
    G[k] = g;
  }
  __syncthreads();
}

/* KppDecomp, right-looking; R receives 1/U(i,i) in the FMA build.
   Table loads are the latency to hide: each step first issues the loads of
   its multiplier positions and of its first COOP_UB update entries per
   thread, then forms the multipliers, so the update entries arrive while
   the multipliers are computed and the block synchronises.  Updates are
   applied COOP_UG at a time, all operand loads of a group before its stores
   (the targets of one step are distinct and are neither multipliers nor
   pivot row entries).  The update table streams through (evict-first
   loads). */
#define COOP_UB 8     /* update entries loaded ahead per thread */
#define COOP_UG 4     /* updates whose operands are loaded before their stores */
__device__ __forceinline__ void coop_decomp(double* G, double* R) {
  const ushort4* upd = reinterpret_cast<const ushort4*>(coop_upd);
  const int tid = threadIdx.x, nt = blockDim.x;
  for (int j = 0; j < NVAR; ++j) {
    const int m0 = coop_mul_off[j], m1 = coop_mul_off[j + 1];
    if (m0 == m1) continue;                 /* no multipliers, no updates */
    const int u0 = coop_upd_off[j], u1 = coop_upd_off[j + 1];
    ushort4 e[COOP_UB];
#pragma unroll
    for (int b = 0; b < COOP_UB; ++b) {
      const int q = u0 + tid + b * nt;
      e[b] = (q < u1) ? __ldcs(upd + q) : make_ushort4(0, 0, 0, 1);
    }
    const double dj = G[coop_diag_c[j]];
#if GC_IRECIP
    const double rj = 1.0 / dj;
#endif
    for (int q = m0 + tid; q < m1; q += nt) {
      const int p = __ldg(&coop_mul_pos[q]);
#if GC_IRECIP
      const double a = -(G[p] * rj);
#else
      const double a = -(G[p] / dj);
#endif
      G[p] = -a;
    }
    if (u0 == u1) continue;
    __syncthreads();
    for (int q0 = u0 + tid;;) {
#pragma unroll
      for (int b0 = 0; b0 < COOP_UB; b0 += COOP_UG) {
        double ga[COOP_UG], gu[COOP_UG], gt[COOP_UG];
#pragma unroll
        for (int b = b0; b < b0 + COOP_UG; ++b) {
          if (e[b].w == 0) { ga[b - b0] = G[e[b].y]; gu[b - b0] = G[e[b].z]; gt[b - b0] = G[e[b].x]; }
        }
#pragma unroll
        for (int b = b0; b < b0 + COOP_UG; ++b) {
          if (e[b].w == 0) {
            const double a = -ga[b - b0];
            G[e[b].x] = gt[b - b0] + a * gu[b - b0];
          }
        }
      }
      q0 += COOP_UB * nt;
      if (q0 >= u1) break;
#pragma unroll
      for (int b = 0; b < COOP_UB; ++b) {
        const int q = q0 + b * nt;
        e[b] = (q < u1) ? __ldcs(upd + q) : make_ushort4(0, 0, 0, 1);
      }
    }
    __syncthreads();
  }
  __syncthreads();
#if GC_IRECIP
  for (int i = tid; i < NVAR; i += nt) R[i] = 1.0 / G[__ldg(&coop_diag[i])];
  __syncthreads();
#else
  (void)R;
#endif
}

/* KppSolve in place on X (the caller has synchronised after writing X).
   Forward sweep by columns: a thread's entry of the next column is loaded
   while the current column is applied.  Backward sweep: in the FMA build by
   columns as well (the per-row order reversed, within the tolerance); in the
   --fmad=false build by levels, each row's terms in the reference order,
   their operands loaded COOP_SB at a time ahead of the dependent
   subtractions. */
#define COOP_SB 4
__device__ __forceinline__ void coop_solve(const double* G, const double* R, double* X) {
  const ushort2* fwd = reinterpret_cast<const ushort2*>(coop_fwd);
  const int tid = threadIdx.x, nt = blockDim.x;
  ushort2 nxt = make_ushort2(0, 0);
  int nxt_ok = 0;
  {
    const int f0 = coop_fwd_off[0], f1 = coop_fwd_off[1];
    if (f0 + tid < f1) { nxt = __ldg(fwd + f0 + tid); nxt_ok = 1; }
  }
  for (int j = 0; j < NVAR; ++j) {
    const int f0 = coop_fwd_off[j], f1 = coop_fwd_off[j + 1];
    const ushort2 cur = nxt;
    const int cur_ok = nxt_ok;
    if (j + 1 < NVAR) {            /* the next column's first entry for this thread */
      const int g0 = coop_fwd_off[j + 1], g1 = coop_fwd_off[j + 2];
      nxt_ok = (g0 + tid < g1);
      if (nxt_ok) nxt = __ldg(fwd + g0 + tid);
    }
    if (f0 == f1) continue;
    const double xj = X[j];
    if (cur_ok) X[cur.x] = X[cur.x] - G[cur.y] * xj;
    for (int q = f0 + tid + nt; q < f1; q += nt) {
      const ushort2 e = __ldg(fwd + q);    /* row, L position */
      X[e.x] = X[e.x] - G[e.y] * xj;
    }
    __syncthreads();
  }
#if GC_IRECIP
  /* backward sweep by columns, from the last: at step i every thread forms
     x(i) = acc(i)/U(i,i) (a product with R(i)) and the rows r < i with
     U(r,i) subtract their term; thread 0 stores x(i) at the next step, when
     no thread reads or updates X(i) any more */
  {
    const ushort2* bwc = reinterpret_cast<const ushort2*>(coop_bwc);
    double pend = 0.0;
    for (int s = 0; s < NVAR; ++s) {
      const int i = NVAR - 1 - s;
      const int b0 = coop_bwc_off[s], b1 = coop_bwc_off[s + 1];
      const double xi = X[i] * R[i];
      if (tid == 0 && s > 0) X[i + 1] = pend;
      pend = xi;
      if (b0 == b1) continue;
      for (int q = b0 + tid; q < b1; q += nt) {
        const ushort2 e = __ldg(bwc + q);    /* row, U position */
        X[e.x] = X[e.x] - G[e.y] * xi;
      }
      __syncthreads();
    }
    if (tid == 0) X[0] = pend;
    __syncthreads();
  }
#else
  for (int l = 0; l < COOP_NLEV; ++l) {
    const int r0 = coop_bwd_off[l], r1 = coop_bwd_off[l + 1];
    for (int q = r0 + tid; q < r1; q += nt) {
      const int i = __ldg(&coop_bwd_rows[q]);
      const int d = __ldg(&coop_diag[i]), e = __ldg(&coop_crow[i + 1]);
      double s = X[i];
      for (int jj = d + 1; jj < e; jj += COOP_SB) {
        double g[COOP_SB], x[COOP_SB];
#pragma unroll
        for (int b = 0; b < COOP_SB; ++b) {
          if (jj + b < e) { g[b] = G[jj + b]; x[b] = X[__ldg(&coop_icol[jj + b])]; }
        }
#pragma unroll
        for (int b = 0; b < COOP_SB; ++b) {
          if (jj + b < e) s = s - g[b] * x[b];
        }
      }
      X[i] = s / G[d];
    }
    __syncthreads();
  }
#endif
}

/* load the cell's column and set the integrator state (lane_start of the
   one-thread-per-cell kernels); attempt 1 is the retry: Hstart taken as 0
   and the retry tolerances */
__device__ __forceinline__ void coop_start(CoopCell& c, const CoopArgs& a, double* sm, long col,
                                           int attempt) {
  c.col = col;
  c.attempt = attempt;
  const double* cc = a.C + col * NSPEC;
  const double* rr = a.RCONST + col * NREACT;
  for (int i = threadIdx.x; i < NVAR; i += blockDim.x) sm[SO_Y0 + i] = cc[i];
  for (int i = threadIdx.x; i < NFIX; i += blockDim.x) sm[SO_FIX + i] = cc[NVAR + i];
  for (int j = threadIdx.x; j < NREACT; j += blockDim.x) sm[SO_RCT + j] = rr[j];
  c.o = decode_options(a.ICNTRL + col * 20, a.RCNTRL + col * 20, a.tstart, a.tend, attempt);
  c.st.nfun = c.st.njac = c.st.nstp = c.st.nacc = 0;
  c.st.nrej = c.st.ndec = c.st.nsol = c.st.nsng = 0;
  c.st.texit = c.st.hexit = c.st.hnew = 0.0;
  c.ierr = c.o.ierr_early;
  c.T = a.tstart;
  double H = fminF(fmaxF(fabs(c.o.hmin), fabs(c.o.hstart)), fabs(c.o.hmax));
  if (fabs(H) <= 10.0 * ROUNDOFF) H = DELTAMIN;
  const double dir = (a.tend >= a.tstart) ? 1.0 : -1.0;
  c.H = dir * H;
  c.nsteps = 0;
  c.ncons = 0;
  c.rej_last = c.rej_more = 0;
  c.newstep = 1;
  c.ysel = 0;
  __syncthreads();
}

__device__ __forceinline__ void coop_store_istat(const CoopCell& c, const CoopArgs& a, int add) {
  int* is = a.ISTAT + c.col * 8;
  const int v[8] = {c.st.nfun, c.st.njac, c.st.nstp, c.st.nacc,
                    c.st.nrej, c.st.ndec, c.st.nsol, c.st.nsng};
#pragma unroll
  for (int k = 0; k < 8; ++k) is[k] = add ? is[k] + v[k] : v[k];
}

/* the end of a solve (lane_end / lane_finish of the other kernels): with the
   retry protocol on, a failed first solve stores its counters and restarts
   from the untouched input column; returns 1 when the cell is finished */
__device__ __forceinline__ int coop_end(CoopCell& c, const CoopArgs& a, double* sm) {
  if (a.nfail && c.attempt == 0 && c.ierr < 0) {
    if (threadIdx.x == 0) {
      coop_store_istat(c, a, 0);
      atomicAdd(&a.nfail[0], 1);
    }
    __syncthreads();
    coop_start(c, a, sm, c.col, 1);
    if (c.ierr == 0) return 0;
  }
  if (c.o.ierr_early == 0) {
    const double* Y = sm + (c.ysel ? SO_Y1 : SO_Y0);
    double* cc = a.C + c.col * NSPEC;
    for (int i = threadIdx.x; i < NVAR; i += blockDim.x) cc[i] = Y[i];
  }
  if (threadIdx.x == 0) {
    coop_store_istat(c, a, c.attempt);
    if (c.attempt && c.ierr < 0) atomicAdd(&a.nfail[1], 1);
    double* rs = a.RSTAT + c.col * 3;
    rs[0] = c.st.texit; rs[1] = c.st.hexit; rs[2] = c.st.hnew;
    a.IERR[c.col] = c.ierr;
  }
  return 1;
}

/* One pass of TimeLoop/UntilAccepted (gckpp_BatchIntegrator.F90:535-704)
   for the block's cell; returns 1 when the cell is finished (c.ierr holds
   IERR).  The statement-level arithmetic is that of step_begin,
   step_prologue, step_factor and step_stages in rodas3_kernels.cu. */
__device__ __forceinline__ int coop_attempt(CoopCell& c, const CoopArgs& a, double* sm,
                                            int* s_ising, double* s_err) {
  const int tid = threadIdx.x, nt = blockDim.x;
  const double Tend = a.tend;
  const double dir = (Tend >= a.tstart) ? 1.0 : -1.0;
  double* G = sm + SO_G;
  double* Y = sm + (c.ysel ? SO_Y1 : SO_Y0);
  double* Ynew = sm + (c.ysel ? SO_Y0 : SO_Y1);
  double* Fcn0 = sm + SO_FCN0;
  double* dFdT = sm + SO_DFDT;
  double* K1 = sm + SO_K;
  double* K2 = K1 + NVAR;
  double* K3 = K1 + 2 * NVAR;
  double* K4 = K1 + 3 * NVAR;
  double* R = sm + SO_R;
  const double* F = sm + SO_FIX;
  const double* RC = sm + SO_RCT;
  double* S = sm + SO_S;

  if (c.newstep) {
    /* TimeLoop exit tests and the H clamp */
    const int direction = (Tend >= a.tstart) ? 1 : -1;
    const bool running = (direction > 0 && ((c.T - Tend) + ROUNDOFF <= 0.0)) ||
                         (direction < 0 && ((Tend - c.T) + ROUNDOFF <= 0.0));
    if (!running) { c.ierr = 1; return 1; }
    if (c.nsteps > c.o.max_steps) { c.ierr = -6; return 1; }
    if (((c.T + 0.1 * c.H) == c.T) || (c.H <= ROUNDOFF)) { c.ierr = -7; return 1; }
    c.H = fminF(c.H, fabs(Tend - c.T));
    /* Fcn0 [, dFdT]; the Jacobian is formed below, at every attempt */
    coop_fun(Y, Fcn0, F, RC, S);
    c.st.nfun += 1;
    if (!c.o.autonomous) {
      const double delta = sqrt(ROUNDOFF) * fmaxF(1.0e-6, fabs(c.T));
      coop_fun(Y, dFdT, F, RC, S);
      c.st.nfun += 1;
      for (int k = tid; k < NVAR; k += nt) dFdT[k] = (dFdT[k] - Fcn0[k]) / delta;
    }
    c.st.njac += 1;
    c.newstep = 0;
    c.ncons = 0;
  }

  /* ros_PrepareMatrix + KppDecomp */
  const double ghinv = 1.0 / ((dir * c.H) * 0.5);
  if (tid == 0) *s_ising = INT_MAX;
  coop_jac_prep(Y, F, RC, S, G, ghinv, s_ising);
  const int ising = (*s_ising == INT_MAX) ? 0 : *s_ising;
  if (ising == 0) coop_decomp(G, R);
  c.st.ndec += 1;
  if (ising != 0) {
    c.st.nsng += 1;
    c.ncons += 1;
    __syncthreads();      /* every thread has read *s_ising */
    if (c.ncons <= 5) { c.H = c.H * 0.5; return 0; }
    c.ierr = -8;
    return 1;
  }

  /* the four stages (per-element operation order of :595-632) */
  const double dH = dir * c.H;
  if (c.o.autonomous) {
    for (int k = tid; k < NVAR; k += nt) K1[k] = Fcn0[k];
  } else {
    const double hg = dH * 0.5;
    for (int k = tid; k < NVAR; k += nt) K1[k] = Fcn0[k] + hg * dFdT[k];
  }
  __syncthreads();
  coop_solve(G, R, K1);
  c.st.nsol += 1;
  {
    const double hc = 4.0 / dH;
    if (c.o.autonomous) {
      for (int k = tid; k < NVAR; k += nt) K2[k] = Fcn0[k] + hc * K1[k];
    } else {
      const double hg = dH * 1.5;
      for (int k = tid; k < NVAR; k += nt) K2[k] = (Fcn0[k] + hc * K1[k]) + hg * dFdT[k];
    }
    __syncthreads();
    coop_solve(G, R, K2);
    c.st.nsol += 1;
  }
  const double hc1 = 1.0 / dH, hc2 = -1.0 / dH;
  {
    for (int k = tid; k < NVAR; k += nt) Ynew[k] = (Y[k] + 2.0 * K1[k]) + 0.0 * K2[k];
    __syncthreads();
    coop_fun(Ynew, K3, F, RC, S);
    c.st.nfun += 1;
    for (int k = tid; k < NVAR; k += nt) K3[k] = (K3[k] + hc1 * K1[k]) + hc2 * K2[k];
    __syncthreads();
    coop_solve(G, R, K3);
    c.st.nsol += 1;
  }
  {
    /* Ynew still holds stage 3's (Y + 2 K1) + 0 K2, rounded as this
       expression rounds it, so only the last term is added */
    for (int k = tid; k < NVAR; k += nt) Ynew[k] = Ynew[k] + 1.0 * K3[k];
    __syncthreads();
    coop_fun(Ynew, K4, F, RC, S);
    c.st.nfun += 1;
    const double hc3 = -(8.0 / 3.0) / dH;
    for (int k = tid; k < NVAR; k += nt)
      K4[k] = ((K4[k] + hc1 * K1[k]) + hc2 * K2[k]) + hc3 * K3[k];
    __syncthreads();
    coop_solve(G, R, K4);
    c.st.nsol += 1;
  }

  /* Ynew, Yerr and the scaled error terms in parallel; the WRMS sum in
     species order by thread 0 */
  const double* atol = c.attempt ? a.ATOLr : a.ATOL;
  const double* rtol = c.attempt ? a.RTOLr : a.RTOL;
  for (int i = tid; i < NVAR; i += nt) {
    const double y = Y[i];
    const double k1 = K1[i], k2 = K2[i], k3 = K3[i], k4 = K4[i];
    const double yn = (((y + 2.0 * k1) + 0.0 * k2) + 1.0 * k3) + 1.0 * k4;
    Ynew[i] = yn;
    const double ye = (((0.0 + 0.0 * k1) + 0.0 * k2) + 0.0 * k3) + 1.0 * k4;
    const double ymax = fmaxF(fabs(y), fabs(yn));
    const double scal = c.o.vectortol ? (__ldg(atol + i) + __ldg(rtol + i) * ymax)
                                      : (__ldg(atol) + __ldg(rtol) * ymax);
    S[i] = ye / scal;
  }
  __syncthreads();
  if (tid == 0) {
    double err = 0.0;
    for (int i = 0; i < NVAR; ++i) {
      const double q = S[i];
      err = err + q * q;
    }
    *s_err = err;
  }
  __syncthreads();
  double err = *s_err;
  err = sqrt(err / (double)NVAR);
  err = fmaxF(err, 1.0e-10);
  const double fac = fminF(c.o.facmax,
                           fmaxF(c.o.facmin, c.o.facsafe / gc_pow(err, 1.0 / ROS_ELO)));
  double hnew = c.H * fac;

  c.nsteps += 1;
  c.st.nstp += 1;
  if ((err <= 1.0) || (c.H <= c.o.hmin)) {
    c.st.nacc += 1;
    if (c.o.clamp) {
      for (int k = tid; k < NVAR; k += nt) Ynew[k] = fmaxF(Ynew[k], 0.0);
    }
    c.ysel ^= 1;              /* Y = Ynew: the arrays swap roles */
    c.T = c.T + dir * c.H;
    hnew = fmaxF(c.o.hmin, fminF(hnew, c.o.hmax));
    if (c.rej_last) hnew = fminF(hnew, c.H);
    c.st.hexit = c.H;
    c.st.hnew = hnew;
    c.st.texit = c.T;
    c.rej_last = 0;
    c.rej_more = 0;
    c.H = hnew;
    c.newstep = 1;
  } else {
    if (c.rej_more) hnew = c.H * c.o.facrej;
    c.rej_more = c.rej_last;
    c.rej_last = 1;
    c.H = hnew;
    if (c.st.nacc >= 1) c.st.nrej += 1;
    c.ncons = 0;
  }
  __syncthreads();            /* *s_err read by all; the clamp is complete */
  return 0;
}

template <int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB) rodas3_coop(CoopArgs a) {
  extern __shared__ double sm[];
  __shared__ unsigned int s_pos;
  __shared__ int s_ising;
  __shared__ double s_err;
  for (;;) {
    if (threadIdx.x == 0) s_pos = atomicAdd(a.qhead, 1u);
    __syncthreads();
    const unsigned int p = s_pos;
    __syncthreads();          /* s_pos read by all before thread 0 rewrites it */
    if (p >= (unsigned int)a.ncell) break;
    CoopCell c;
    coop_start(c, a, sm, (long)a.order[p], 0);
    do {
      if (c.ierr == 0) {
        while (!coop_attempt(c, a, sm, &s_ising, &s_err)) {}
      }
    } while (!coop_end(c, a, sm));
    __syncthreads();          /* the result is stored before the next cell loads */
  }
}

static size_t coop_smem_bytes(void) { return (size_t)SO_END * sizeof(double); }

/* the kernel instance for a block size (128 or 256 threads) */
static const void* coop_kernel(int threads) {
  if (threads == 128) return (const void*)rodas3_coop<128, 3>;
  if (threads == 256) return (const void*)rodas3_coop<256, 2>;
  return nullptr;
}

static cudaError_t coop_attr(int threads) {
  const void* k = coop_kernel(threads);
  if (!k) return cudaErrorInvalidValue;
  return cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)coop_smem_bytes());
}

extern "C" int rodas3_coop_ok(void) {
  return coop_smem_bytes() <= 227 * 1024 ? 1 : 0;
}

extern "C" size_t rodas3_coop_smem_bytes(void) { return coop_smem_bytes(); }

extern "C" int rodas3_coop_blocks_per_sm(int threads) {
  if (!rodas3_coop_ok() || coop_attr(threads) != cudaSuccess) return 0;
  int nb = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, coop_kernel(threads), threads,
                                                    coop_smem_bytes()) != cudaSuccess)
    return 0;
  return nb;
}

/* blocks: resident blocks of the launch (the caller's SM count x blocks per
   SM, at most one per cell) */
extern "C" cudaError_t rodas3_coop_launch(const Rodas3Launch* L, int blocks, cudaStream_t s) {
  if (!rodas3_coop_ok() || L->ckpt != nullptr) return cudaErrorInvalidValue;
  const int threads = L->threads;
  const cudaError_t ea = coop_attr(threads);
  if (ea != cudaSuccess) return ea;
  if (blocks > L->ncell) blocks = L->ncell;
  if (blocks <= 0) return cudaSuccess;
  CoopArgs a;
  a.ncell = L->ncell; a.tstart = L->tstart; a.tend = L->tend;
  a.C = L->C; a.RCONST = L->RCONST; a.ATOL = L->ATOL; a.RTOL = L->RTOL;
  a.ICNTRL = L->ICNTRL; a.RCNTRL = L->RCNTRL; a.order = L->order;
  a.ISTAT = L->ISTAT; a.RSTAT = L->RSTAT; a.IERR = L->IERR;
  a.qhead = L->qhead; a.nfail = L->nfail; a.ATOLr = L->ATOLr; a.RTOLr = L->RTOLr;
  cudaMemsetAsync(L->qhead, 0, sizeof(unsigned int), s);
  const size_t smem = coop_smem_bytes();
  if (threads == 128)
    rodas3_coop<128, 3><<<blocks, 128, smem, s>>>(a);
  else
    rodas3_coop<256, 2><<<blocks, 256, smem, s>>>(a);
  return cudaGetLastError();
}

#else  /* no tables for this mechanism */

extern "C" int rodas3_coop_ok(void) { return 0; }
extern "C" size_t rodas3_coop_smem_bytes(void) { return 0; }
extern "C" int rodas3_coop_blocks_per_sm(int) { return 0; }
extern "C" cudaError_t rodas3_coop_launch(const Rodas3Launch*, int, cudaStream_t) {
  return cudaErrorInvalidValue;
}

#endif
