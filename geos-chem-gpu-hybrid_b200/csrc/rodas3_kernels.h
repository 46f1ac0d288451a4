/* rodas3_kernels.h -- host-side launch interface of the Rodas3 kernels
   (internal to libgcchemgpu; the public C-ABI is include/gcchem_gpu.h). */
#pragma once
#include <cuda_runtime.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { RODAS3_PLAIN = 0, RODAS3_PERSISTENT = 1, RODAS3_PLAIN_FUSED = 2, RODAS3_COOP = 3 };

typedef struct {
  int mode;              /* RODAS3_PLAIN, RODAS3_PERSISTENT, RODAS3_PLAIN_FUSED or RODAS3_COOP */
  int ncell;
  double tstart, tend;
  double* C;             /* device, (NSPEC, ncell) column-major */
  const double* RCONST;  /* device, (NREACT, ncell) */
  const double* ATOL;    /* device, (NVAR) */
  const double* RTOL;    /* device, (NVAR) */
  const int* ICNTRL;     /* device, (20, ncell) */
  const double* RCNTRL;  /* device, (20, ncell) */
  const int* order;      /* device, launch order as 0-based columns */
  int* ISTAT;            /* device, (8, ncell) */
  double* RSTAT;         /* device, (3, ncell) */
  int* IERR;             /* device, (ncell) */
  double* ws;            /* device workspace: slots * rodas3_ws_elems() doubles */
  long slots;            /* workspace slots (multiple of 32) */
  unsigned int* qhead;   /* device counter for the persistent queue */
  int threads;           /* threads per block */
  int* nfail;            /* retry protocol (or NULL): device [2] counters, zeroed by the
                            caller: first solves failed, retries failed */
  const double* ATOLr;   /* device, (NVAR): retry tolerances */
  const double* RTOLr;
  double* ckpt;          /* adjoint checkpoints, or NULL */
  int ckpt_max;
  int shared_scratch;    /* indexed LU row scratch in shared memory (small mechanisms) */
} Rodas3Launch;

int rodas3_ws_elems(void);
void rodas3_sizes(int* nvar, int* nfix, int* nreact, int* nnz);
int rodas3_persistent_blocks_per_sm(int threads, int shared_scratch);
int rodas3_max_threads(int shared_scratch);
int rodas3_shared_scratch_ok(void);
cudaError_t rodas3_launch(const Rodas3Launch* L, cudaStream_t s);
/* the cooperative kernel (coop.cu): one block of 128 or 256 threads per cell,
   the cell state in shared memory, no workspace */
int rodas3_coop_ok(void);
size_t rodas3_coop_smem_bytes(void);
int rodas3_coop_blocks_per_sm(int threads);
cudaError_t rodas3_coop_launch(const Rodas3Launch* L, int blocks, cudaStream_t s);
double rodas3_fp64_peak_tflops(void);
long rodas3_cost_scratch(int n);
cudaError_t rodas3_cost_order(const int* keys, int n, int* order,
                              unsigned long long* scratch, cudaStream_t s);
double rodas3_phase_ms(int phase, long slots, int reps, double* ws);
int rodas3_adjoint_ws_elems(void);
cudaError_t rodas3_adjoint_launch(int ncell, const double* C0, const double* RCONST,
                                  const int* ISTAT, const double* ckpt, int ckpt_max,
                                  const double* lam, double* gC0, double* gK, int* ierr,
                                  double* ws, long slots, int* sortbuf,
                                  unsigned long long* sortscratch, cudaStream_t s);
cudaError_t rodas3_perm_to_order(const int* perm, int n, int* order, int* bad,
                                 cudaStream_t s);

cudaError_t rodas3_batch_keys(int ncells, const int* prev, const int* mask, int sort, int* keys,
                              cudaStream_t st);
cudaError_t rodas3_batch_decode(int ncell, int NX, int NY, const int* order, int* map,
                                cudaStream_t st);
cudaError_t rodas3_gather(int ncell, int NX, int NY, int NZ, const int* map, const double* conc,
                          const int* kmap, double* C, const double* rgrid, double* R,
                          const double* hval, double* RC, cudaStream_t st);
cudaError_t rodas3_scatter(int ncell, int NX, int NY, int NZ, const int* map, double* conc,
                           const int* kmap, const double* C, const int* ISTAT,
                           const double* RSTAT, double* hval, int* prev, float* diag,
                           cudaStream_t st);

#ifdef __cplusplus
}
#endif
