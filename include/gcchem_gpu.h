/*
 * gcchem_gpu.h -- C-ABI of libgcchemgpu.so, the B200 batched Rodas3
 * gas-phase chemistry solver.
 *
 * The five gc_gpu_* entry points are drop-in replacements for the symbols
 * GEOS-Chem's fullchem_mod.F90 binds through ISO_C_BINDING
 * (src/geos-chem/GeosCore/fullchem_mod.F90:153-212).  Fortran BIND(C) rules
 * apply: VALUE arguments are passed by value, every other argument by
 * address; arrays are column-major with the cell index last; Perm is 1-based.
 *
 * The gcchem_b200_* entry points are additions: a device-resident,
 * stream-ordered variant of the same solve (all pointers are device
 * pointers), the launch knobs, and workspace control.  They keep the
 * per-cell semantics of the legacy symbols exactly.
 *
 * Per-cell IERR codes (gckpp_BatchIntegrator.F90:128-142,538-545,588 and
 * gc_gpu_batch_api.F90:183-187):
 *     1 success            -2 ICNTRL(3) not Rodas3 (0 or 4)
 *    -6 more than ICNTRL(4) steps (default 200000)
 *    -7 step size too small   -8 more than 5 consecutive singular matrices
 *   -90 ICNTRL(12)=1 (auto-reduce) requested
 *   -99 device selection failed (every IERR of the call)
 *  -100 the library could not run the solve (device memory, launch error);
 *       reported in every IERR of the call, which the caller's retry path
 *       treats like any other failure
 */
#ifndef GCCHEM_GPU_H
#define GCCHEM_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

/* Replaces gc_gpu_integrate_batch (gpulib/src/gc_gpu_batch_api.F90:115-136;
 * model interface fullchem_mod.F90:155-171).  Solves nCell independent cells
 * over [Tstart, Tend] on the calling host thread's current device.
 *   C      (NSPEC, nCell)  in/out: VAR = rows 1..NVAR, FIX = NVAR+1..NSPEC
 *   RCONST (NREACT, nCell) in
 *   ATOL, RTOL (NVAR)      in, shared by every cell
 *   ICNTRL (20, nCell) in, RCNTRL (20, nCell) in: merged per cell exactly as
 *          gpu_solve_cell does (zeroed, ICNTRL(15)=5, then ICNTRL_U/=0 and
 *          RCNTRL_U>0 override)
 *   Perm   (nCell)         launch slot ic solves column Perm(ic) (1-based)
 *          and writes that column's outputs
 *   ISTAT  (8, nCell) out: Nfun Njac Nstp Nacc Nrej Ndec Nsol Nsng
 *   RSTAT  (3, nCell) out: Texit Hexit Hnew
 *   IERR   (nCell)    out
 *   tTotal, tKernel   out: seconds for the whole call / the solve kernels */
void gc_gpu_integrate_batch(int nCell, double Tstart, double Tend, double* C,
                            const double* RCONST, const double* ATOL,
                            const double* RTOL, const int* ICNTRL,
                            const double* RCNTRL, const int* Perm, int* ISTAT,
                            double* RSTAT, int* IERR, double* tTotal,
                            double* tKernel);

/* Replaces gc_gpu_integrate_batch_dev (gc_gpu_batch_api.F90:147-216; model
 * interface fullchem_mod.F90:172-191).  dev >= 0 makes device `dev` current
 * for the calling host thread first (IERR(1:nCell) = -99 if that fails);
 * dev < 0 keeps the current device.  Different host threads may call this
 * concurrently on different devices. */
void gc_gpu_integrate_batch_dev(int dev, int nCell, double Tstart,
                                double Tend, double* C, const double* RCONST,
                                const double* ATOL, const double* RTOL,
                                const int* ICNTRL, const double* RCNTRL,
                                const int* Perm, int* ISTAT, double* RSTAT,
                                int* IERR, double* tTotal, double* tKernel);

/* Replaces gc_gpu_selftest (gc_gpu_batch_api.F90:349-376; interface
 * fullchem_mod.F90:206-211): one cell with C = 1e6, RCONST = 0,
 * ATOL = 1e-2, RTOL = 0.5e-2, ICNTRL(1,2,3,7,15) = (1,0,4,1,-1), over
 * [0, 1200] s.  rc = IERR of that cell (1), nsteps = its ISTAT(3) (12). */
void gc_gpu_selftest(int* rc, int* nsteps, double* tTotal);

/* Replaces gc_gpu_info (gpulib/src/gc_gpu_devinfo.c, lines 23-50 of the
 * file; interface fullchem_mod.F90:192-198): number of CUDA devices and
 * the name of device 0 (NUL-terminated, at most nameLen-1 characters).
 * nDev = 0 when no driver or device is present. */
void gc_gpu_info(int* nDev, char* devName, int nameLen);

/* Replaces gc_gpu_set_device (gc_gpu_devinfo.c, lines 67-86 of the file;
 * interface fullchem_mod.F90:199-203): make device d current for the
 * calling host thread; returns the current device afterwards, -1 on
 * failure. */
int gc_gpu_set_device(int d);

/* ---- additions (no counterpart in the reference) ----------------------- */

/* Mechanism sizes compiled into this library. */
void gcchem_b200_sizes(int* nvar, int* nfix, int* nreact, int* nnz);

/* Solver variants: 0 = plain (one thread per cell for the whole solve),
 * 1 = persistent (cost-ordered device work queue, slot refill). */
#define GCCHEM_B200_PLAIN 0
#define GCCHEM_B200_PERSISTENT 1

/* Launch knobs for subsequent calls on the calling thread's device.
 * threads: block size (multiple of 32, at most 256; 0 = default 128);
 * blocks_per_sm: resident blocks the persistent grid assumes
 * (0 = the occupancy calculator's maximum).  Returns 0, or -1 for invalid
 * values.  The environment variables GCCHEM_B200_MODE (plain|persistent),
 * GCCHEM_B200_THREADS and GCCHEM_B200_BLOCKS_PER_SM set the defaults. */
int gcchem_b200_set_launch(int mode, int threads, int blocks_per_sm);

/* Device-resident, stream-ordered solve.  Same layouts and per-cell
 * semantics as gc_gpu_integrate_batch, but every array is a DEVICE pointer
 * of the current device, `order` holds the launch order as 0-based columns
 * (the device form of Perm), and the call only enqueues work on `stream`
 * (a cudaStream_t; NULL = the legacy default stream).  The workspace is the
 * library's per-device pool (grown on demand, outside stream capture).
 * Calls on one device share that workspace and the queue counter, so calls
 * that could overlap on the GPU must be ordered (one stream, or events).
 * Returns 0 on success, a negative code if the launch could not be made. */
int gcchem_b200_integrate_device(int nCell, double Tstart, double Tend,
                                 double* C, const double* RCONST,
                                 const double* ATOL, const double* RTOL,
                                 const int* ICNTRL, const double* RCNTRL,
                                 const int* order, int* ISTAT, double* RSTAT,
                                 int* IERR, void* stream);

/* Device-resident solve with the model's retry protocol (replaces the host
 * retry of fullchem_mod.F90:2436-2520; the reference library itself has no
 * retry).  After the first launch, every cell with IERR < 0 gets its
 * pre-solve concentrations back, RCNTRL(3) (Hstart) treated as 0, and is
 * solved again with the retry tolerances ATOLr/RTOLr in a second persistent
 * launch whose queue length stays on the device (no host round trip).  For
 * retried cells ISTAT accumulates both attempts, RSTAT and IERR come from the
 * second.  nfail: device array of 2 ints, set to (cells that failed the
 * first attempt, cells that failed both).  Unlike the model, which stops at
 * the first cell that fails twice, every retried cell is merged; the caller
 * decides what a nonzero nfail[1] means.  Stream-ordered; returns 0 or a
 * negative code. */
int gcchem_b200_integrate_device_retry(int nCell, double Tstart, double Tend,
                                       double* C, const double* RCONST,
                                       const double* ATOL, const double* RTOL,
                                       const double* ATOLr, const double* RTOLr,
                                       const int* ICNTRL, const double* RCNTRL,
                                       const int* order, int* ISTAT, double* RSTAT,
                                       int* IERR, int* nfail, void* stream);

/* Discrete adjoint (no counterpart in the reference, which has only the
 * building blocks KppSolveTR, JacTR_SP_Vec and CalcStoichNum).
 *
 * gcchem_b200_integrate_device_ckpt: gcchem_b200_integrate_device that also
 * stores, for each accepted step n < ckpt_max of every cell, the state at
 * the start of the step and the accepted step size in
 * ckpt[(col*ckpt_max + n)*(NVAR+1) + 0..NVAR] (device, n*ckpt_max*(NVAR+1)
 * doubles).
 *
 * gcchem_b200_adjoint_device: given lam = dL/dC at the end of the step
 * (NSPEC, n), returns the exact derivatives of L through the recorded
 * (frozen) step sequence: gC0 = dL/dC0 (NSPEC, n; fixed-species rows 0) and
 * gK = dL/d ln RCONST (NREACT, n).  ISTAT and ckpt come from the
 * checkpointed forward call; ierr per cell: 1, -101 (more accepted steps
 * than ckpt_max), -8 (singular factor).  Autonomous cells without clamping
 * (ICNTRL(1)=1, ICNTRL(16)/=1, the model's settings).  Stream-ordered;
 * returns 0 or a negative code. */
int gcchem_b200_integrate_device_ckpt(int nCell, double Tstart, double Tend, double* C,
                                      const double* RCONST, const double* ATOL,
                                      const double* RTOL, const int* ICNTRL,
                                      const double* RCNTRL, const int* order, int* ISTAT,
                                      double* RSTAT, int* IERR, double* ckpt, int ckpt_max,
                                      void* stream);
int gcchem_b200_adjoint_device(int nCell, const double* C0, const double* RCONST,
                               const int* ISTAT, const double* ckpt, int ckpt_max,
                               const double* lam, double* gC0, double* gK, int* ierr,
                               void* stream);

/* Device-side cost ordering for the persistent queue: writes to `order`
 * (device, nCell ints) the columns 0..nCell-1 sorted by descending cost key
 * (device, nCell ints; keys are clamped to 0..4095).  With the previous
 * chemistry step's ISTAT(3) as keys this is the model's pre-scan sort
 * (fullchem_mod.F90:906-960) done on the device; ties keep no particular
 * order.  Stream-ordered on `stream`.  Returns 0 or a negative code. */
int gcchem_b200_cost_order(const int* keys, int nCell, int* order, void* stream);

/* Allocation-free solve (no counterpart in the reference).  For callers that
 * cannot allocate device memory when they solve: a model whose GPU memory
 * comes from its own pool, or a thread that must not call cudaMalloc/cudaFree
 * because they synchronise the whole device.  Same arguments and per-cell
 * results as gcchem_b200_integrate_device (one thread per cell), but the
 * solver workspace is a fixed array inside the library's device image, so a
 * call takes at most 256 cells; nCell > 256 returns -4 and does nothing.
 * The array (about 32 MB) is held on every GPU that loads the library until
 * the process exits.  The first call on a device looks up the array's device
 * address (make that first call before any stream capture).  All calls on a
 * device share the array: calls that overlap on the GPU race, so keep them on
 * one stream.  Returns 0, -4 (too many cells), or another negative code. */
int gcchem_b200_integrate_device_noalloc(int nCell, double Tstart, double Tend,
                                         double* C, const double* RCONST,
                                         const double* ATOL, const double* RTOL,
                                         const int* ICNTRL, const double* RCNTRL,
                                         const int* order, int* ISTAT, double* RSTAT,
                                         int* IERR, void* stream);

/* Make sure the current device's workspace pool can serve nCell cells with
 * the current launch settings (call before capturing a CUDA graph). Returns
 * 0 or a negative code. */
int gcchem_b200_reserve(int nCell);

/* Free the current device's workspace pool. */
void gcchem_b200_release(void);

/* Slots the next launch of nCell cells would use, and bytes per slot. */
long gcchem_b200_workspace_slots(int nCell);
long gcchem_b200_workspace_bytes_per_slot(void);

/* Measured FP64 FMA throughput of the current device in TFLOP/s (a short
 * probe kernel; the denominator of the solver's roofline fraction), or a
 * negative value on error. */
double gcchem_b200_fp64_peak_tflops(void);

/* Diagnostic: milliseconds for `reps` calls of one solver building block
 * (0 Fun, 1 Jac, 2 prepare+factorise, 3 solve, 4 indexed KppDecomp) by
 * `slots` threads (a multiple of 32) on synthetic data; negative on error. */
double gcchem_b200_phase_ms(int phase, long slots, int reps);

#ifdef __cplusplus
}
#endif
#endif /* GCCHEM_GPU_H */
