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

/* Solver variants: 0 = plain (one thread per cell for the whole solve, the
 * reference's indexed KppDecomp), 1 = persistent (cost-ordered device work
 * queue, slot refill, generated fused factorisation), 2 = plain with the
 * persistent kernel's arithmetic (one thread per cell, generated fused
 * factorisation: the baseline that isolates what the queue gains),
 * 3 = cooperative (one block of 128 or 256 threads per cell, the cell's
 * factors and vectors in shared memory, the same cost-ordered queue; no
 * solver workspace; for mechanisms whose state fits in shared memory --
 * gcchem_b200_set_launch returns -1 otherwise). */
#define GCCHEM_B200_PLAIN 0
#define GCCHEM_B200_PERSISTENT 1
#define GCCHEM_B200_PLAIN_FUSED 2
#define GCCHEM_B200_COOP 3

/* Launch knobs for subsequent calls on the calling thread's device.
 * threads: block size (multiple of 32, at most 256 -- at most 224 with the
 * row scratch in shared memory for the 120-species synthetic mechanism, see
 * gcchem_b200_set_row_scratch; 0 = default 128);
 * blocks_per_sm: resident blocks the persistent and cooperative grids assume
 * (0 = the occupancy calculator's maximum).  Returns 0, or -1 for invalid
 * values.  With the cooperative kernel selected, the checkpointing forward
 * solve of the adjoint runs on the persistent kernel.  The environment
 * variables GCCHEM_B200_MODE (plain|persistent|plain_fused|coop),
 * GCCHEM_B200_THREADS and GCCHEM_B200_BLOCKS_PER_SM set the defaults. */
int gcchem_b200_set_launch(int mode, int threads, int blocks_per_sm);

/* Where the indexed factorisation (KppDecomp, used by mechanisms without the
 * generated fused LU) keeps its dense row scratch: 0 = in the cell's
 * workspace slot (HBM, the default), 1 = in shared memory, one tile per warp
 * (mechanisms with at most 160 variable species, e.g. the synthetic one;
 * blocks of at most 224 threads for 120 species).  Same arithmetic either
 * way.  Returns 0, or -1 where the mechanism or the current block size does
 * not allow it.  GCCHEM_B200_ROW_SCRATCH=shared sets it by default. */
int gcchem_b200_set_row_scratch(int shared);

/* Plain (one-thread-per-cell) launches: solve at most `cells` cells per
 * launch, each launch's workspace reused by the next -- the reference's
 * low-memory global-workspace mode (gc_gpu_batch_api.F90:292-343) with the
 * chunk size as a launch setting.  0 = GC_GPU_WORKSPACE=global with
 * GC_GPU_CHUNK from the environment, else the whole batch in one launch
 * (memory permitting).  Returns 0 or -1. */
int gcchem_b200_set_chunk(int cells);

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
 * retry).  Every cell whose first solve ends with IERR < 0 is solved again
 * from its pre-solve concentrations, with RCNTRL(3) (Hstart) treated as 0
 * and the retry tolerances ATOLr/RTOLr.  For retried cells ISTAT sums both
 * solves, and RSTAT, IERR and C come from the retry.  The retry runs in the
 * same launch: the solver thread that saw the failure starts it at once,
 * while the rest of the batch is still being solved, so a few retried cells
 * add no serial tail.  nfail: device array of 2 ints, set to (cells that
 * failed the first solve, cells that failed the retry too).  Unlike the
 * model, which stops at the first cell that fails twice, every cell is
 * retried; the caller decides what a nonzero nfail[1] means.
 * Stream-ordered; returns 0 or a negative code. */
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
 * (device, nCell ints, any int32 value), cells with equal keys in increasing
 * column order.  With the previous chemistry step's ISTAT(3) as keys this is
 * exactly the model's stable pre-scan counting sort (fullchem_mod.F90:906-960)
 * done on the device, and the result does not vary from run to run.  The
 * first call for a larger nCell grows a per-device scratch buffer (make it
 * before any stream capture).  Stream-ordered on `stream`.  Returns 0 or a
 * negative code. */
int gcchem_b200_cost_order(const int* keys, int nCell, int* order, void* stream);

/* Allocation-free solve (no counterpart in the reference).  For callers that
 * cannot allocate device memory when they solve: a model whose GPU memory
 * comes from its own pool, or a thread that must not call cudaMalloc/cudaFree
 * because they synchronise the whole device.  Same arguments as
 * gcchem_b200_integrate_device, and bit for bit the same per-cell results as
 * its one-thread-per-cell launch (mode 0); the default persistent launch
 * factorises with pivot reciprocals in the FMA build and may differ from it
 * in the last bits.  The solver workspace is a fixed array inside the
 * library's device image, so a call takes at most 256 cells; nCell > 256
 * returns -4 and does nothing.
 * The array (about 32 MB) is held on every GPU that loads the library until
 * the process exits.  The first call on a device looks up the array's device
 * address (make that first call before any stream capture).  All calls on a
 * device share the array: calls that overlap on the GPU race, so keep them on
 * one stream.  Returns 0, -4 (too many cells), -1 (no device or symbol
 * lookup failed) or -3 (launch error; an error left pending by earlier work
 * on the thread is reported as -3 too, and is not cleared). */
int gcchem_b200_integrate_device_noalloc(int nCell, double Tstart, double Tend,
                                         double* C, const double* RCONST,
                                         const double* ATOL, const double* RTOL,
                                         const int* ICNTRL, const double* RCNTRL,
                                         const int* order, int* ISTAT, double* RSTAT,
                                         int* IERR, void* stream);

/* ---- batch bookkeeping on the device (state resident in HBM) ----------
 * Grid arrays are DEVICE arrays in Fortran order (NX, NY, NZ[, k]); cell
 * (I,J,L) is element (I-1) + NX*((J-1) + NY*(L-1)).  BatchMap is the
 * model's (3, nCell) int array of 1-based (I,J,L) per slot.  All three are
 * stream-ordered on `stream` and return 0 or a negative code. */

/* Replaces the model's pre-scan (fullchem_mod.F90:906-993): the chemistry
 * cells (InChem != 0, or every cell when InChem is NULL) sorted by
 * descending PrevNsteps, ties in L,J,I order -- the model's stable counting
 * sort -- or in L,J,I order alone when sort == 0 (GC_BATCH_SORT=0).  nCell
 * must be the number of chemistry cells; BatchMap receives nCell slots.
 * The first call for a larger grid grows a per-device scratch buffer (make
 * it before any stream capture). */
int gcchem_b200_batch_map(int NX, int NY, int NZ, const int* PrevNsteps, const int* InChem,
                          int sort, int nCell, int* BatchMap, void* stream);

/* Replaces the model's gather (fullchem_mod.F90:1538-1543 and :1749-1756):
 * C(N,slot) = Conc(I,J,L,MapKppSpc(N)) for KPP species N that are model
 * species (MapKppSpc(N) > 0, 1-based), 0 for the others.  Conc is
 * (NX,NY,NZ,nSpc).  With RconstGrid (NX,NY,NZ,NREACT) the batch RCONST
 * columns are gathered too (both pointers NULL: RCONST is left alone).
 * With KPPHvalue (NX,NY,NZ) the warm start RCNTRL(3,slot) = KPPHvalue(I,J,L)
 * is set in the (20, nCell) RCNTRL, as the model's integrator options do
 * (the other RCNTRL entries are left alone). */
int gcchem_b200_gather(int nCell, int NX, int NY, int NZ, const int* BatchMap,
                       const double* Conc, const int* MapKppSpc, double* C,
                       const double* RconstGrid, double* RCONST, const double* KPPHvalue,
                       double* RCNTRL, void* stream);

/* Replaces the model's scatter (fullchem_mod.F90:2878-3000): for mapped
 * species Conc(I,J,L,MapKppSpc(N)) = max(C(N,slot), 0); KPPHvalue(I,J,L) =
 * RSTAT(3,slot) (:2922) and PrevNsteps(I,J,L) = ISTAT(3,slot) (:2868, the
 * next step's sort key) when those arrays are given; KppDiag, when given,
 * is (NX,NY,NZ,9) float: ISTAT(1:8) (the KppDiags counters, :2926-2970)
 * and the number of mapped species that came back negative (KppNegatives,
 * :2983-2989). */
int gcchem_b200_scatter(int nCell, int NX, int NY, int NZ, const int* BatchMap, double* Conc,
                        const int* MapKppSpc, const double* C, const int* ISTAT,
                        const double* RSTAT, double* KPPHvalue, int* PrevNsteps,
                        float* KppDiag, void* stream);

/* ---- hybrid CPU/GPU split of one chemistry step ------------------------
 * Replaces the GC_BATCH_CHEM=3 scheduler of fullchem_mod.F90: the work
 * model (:997-1005, cost = max(previous Nstp, 1), prefix sums over the
 * cost-ordered slots), the GPU/CPU split from measured rates (:1006-1019),
 * the work-balanced contiguous device slices (:1020-1055) and the rate
 * updates, exponential moving averages of work per second (:2678-2706).
 * A GcHybrid carries that state from one chemistry step to the next; it is
 * not thread-safe (one per model process, used by one host thread). */
typedef struct GcHybrid GcHybrid;

/* ndev: devices to spread the GPU share over (GC_GPU_NDEV, at most the
 * devices present); frac: initial GPU share of the work (GC_GPU_FRAC, in
 * [0,1]); fixed_frac != 0 keeps it (GC_GPU_FRAC_FIXED=1).  NULL on bad
 * arguments. */
GcHybrid* gcchem_b200_hybrid_create(int ndev, double frac, int fixed_frac);
void gcchem_b200_hybrid_destroy(GcHybrid* h);

/* Plan one step over nCell cost-ordered cells whose previous internal step
 * counts are prevNsteps (host, nCell ints, in slot order): the head of
 * *nGpu slots goes to the GPUs, cut into *nDevUse slices
 * devLo[d]..devHi[d] (1-based, inclusive; arrays of at least ndev ints).
 * No CUDA call: runs without a GPU.  Returns 0 or -1. */
int gcchem_b200_hybrid_plan(GcHybrid* h, int nCell, const int* prevNsteps, int* nGpu,
                            int* nDevUse, int* devLo, int* devHi);

/* After the planned step: devTw[d] = wall seconds of device d's launch
 * (nDevUse values), tCpu = wall seconds the host took for the tail.
 * Updates the per-device, GPU and CPU rates.  Returns 0 or -1. */
int gcchem_b200_hybrid_update(GcHybrid* h, const double* devTw, double tCpu);

/* Current GPU share and rates (work units per second; devRate: ndev
 * values; NULL pointers are skipped). */
int gcchem_b200_hybrid_state(const GcHybrid* h, double* frac, double* rateGpu,
                             double* rateCpu, double* devRate);

/* One whole hybrid step on HOST arrays in the legacy layouts, already in
 * cost order (slot ic = column ic): plan; one host thread per device slice
 * calls gc_gpu_integrate_batch_dev on its columns while the calling thread
 * runs cpu_tail(first, count, user) for the tail (0-based first slot; the
 * caller's own CPU integrator writes C, ISTAT, RSTAT, IERR of those
 * columns); then the rates are updated.  The threads exist only during the
 * call.  nGpu, tGpu (slowest device) and tCpu report the step.  Returns 0,
 * or -1 for bad arguments (a tail without a cpu_tail). */
int gcchem_b200_hybrid_step(GcHybrid* h, int nCell, double Tstart, double Tend, double* C,
                            const double* RCONST, const double* ATOL, const double* RTOL,
                            const int* ICNTRL, const double* RCNTRL, const int* prevNsteps,
                            int* ISTAT, double* RSTAT, int* IERR,
                            void (*cpu_tail)(int first, int count, void* user), void* user,
                            int* nGpu, double* tGpu, double* tCpu);

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
 * (0 Fun, 1 Jac, 2 generated prepare+factorise, 3 solve, 4 indexed
 * prepare+KppDecomp) by `slots` threads (a multiple of 32) on synthetic
 * data; -2.0 for phase 2 when the mechanism has no generated factorisation,
 * -1.0 on error. */
double gcchem_b200_phase_ms(int phase, long slots, int reps);

#ifdef __cplusplus
}
#endif
#endif /* GCCHEM_GPU_H */
