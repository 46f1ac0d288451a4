/*
 * gc_api.cu -- host side of libgcchemgpu.so (declarations and the reference
 * interfaces they replace: include/gcchem_gpu.h).
 *
 * Per call of the legacy entry (gc_gpu_integrate_batch_dev,
 * gpulib/src/gc_gpu_batch_api.F90:147-216) the library
 *   1. selects the device when dev >= 0 (IERR(:) = -99 on failure),
 *   2. returns at once when nCell <= 0,
 *   3. checks Perm on the host (IERR(:) = -100 for an entry outside 1..nCell)
 *      and copies C, RCONST, ATOL, RTOL, ICNTRL, RCNTRL and Perm to the device,
 *   4. runs the solve (persistent queue kernel by default; GCCHEM_B200_MODE=
 *      plain selects the one-thread-per-cell kernel),
 *   5. copies C, ISTAT, RSTAT and IERR back,
 * and reports tTotal (whole call) and tKernel (solve kernels, CUDA events).
 * Unlike the reference, device buffers and the solver workspace are cached
 * per device between calls (grown on demand) instead of being allocated and
 * freed every call; gcchem_b200_release() frees them.
 *
 * Threading: each device has its own mutex, stream and buffers, so host
 * threads working on different devices run concurrently (the model's
 * one-OpenMP-thread-per-device pattern, fullchem_mod.F90:1229-1268); calls on
 * the same device are serialised.  The library prints nothing and starts no
 * threads of its own.
 */
#include <cuda_runtime.h>
#include <stdlib.h>
#include <string.h>
#include <chrono>
#include <mutex>
#include <algorithm>

#include "rodas3_kernels.h"
#include "../../include/gcchem_gpu.h"

namespace {

const int kMaxDev = 64;

struct DevState {
  std::mutex mu;
  bool init = false;
  int sm_count = 0;
  int mode = RODAS3_PERSISTENT;
  int threads = 128;
  int bps = 0;               /* persistent blocks per SM, 0 = occupancy max */
  int chunk = 0;             /* plain kernels: cells per launch, 0 = env / whole batch */
  int scratch = 0;           /* indexed LU row scratch: 0 workspace, 1 shared memory */
  cudaStream_t stream = nullptr;
  double* ws = nullptr;
  long ws_slots = 0;
  unsigned int* qhead = nullptr;
  int* bad = nullptr;
  unsigned long long* sortc = nullptr;   /* cost-sort composites */
  long sortc_n = 0;
  int* gkeys = nullptr;      /* batch map: per-cell keys + order, 2 ints per grid cell */
  long gkeys_n = 0;
  /* staging buffers of the legacy (host-array) entry */
  char* buf = nullptr;
  size_t buf_bytes = 0;
  /* adjoint workspace */
  double* aws = nullptr;
  long aws_slots = 0;
  int* asort = nullptr;      /* adjoint launch order: keys + order, 2 ints per cell */
  long asort_n = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};

DevState g_dev[kMaxDev];

int env_int(const char* name, int dflt) {
  const char* v = getenv(name);
  if (!v || !*v) return dflt;
  char* end = nullptr;
  long x = strtol(v, &end, 10);
  if (end == v || *end != '\0' || x <= 0) return dflt;
  return (int)x;
}

bool env_is(const char* name, const char* val) {
  const char* v = getenv(name);
  if (!v) return false;
  return strncasecmp(v, val, strlen(val)) == 0;
}

/* caller holds s.mu */
int ensure_init(DevState& s, int dev) {
  if (s.init) return 0;
  if (cudaDeviceGetAttribute(&s.sm_count, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return -1;
  if (env_is("GCCHEM_B200_MODE", "coop") && rodas3_coop_ok()) s.mode = RODAS3_COOP;
  else if (env_is("GCCHEM_B200_MODE", "plain_fused")) s.mode = RODAS3_PLAIN_FUSED;
  else if (env_is("GCCHEM_B200_MODE", "plain")) s.mode = RODAS3_PLAIN;
  int t = env_int("GCCHEM_B200_THREADS", 128);
  /* kernels are built for <= 256 threads (fewer when their W row scratch is
     in shared memory) */
  if (t <= 0 || t % 32 != 0 || t > 256) t = 128;
  if (env_is("GCCHEM_B200_ROW_SCRATCH", "shared") && rodas3_shared_scratch_ok()) s.scratch = 1;
  if (t > rodas3_max_threads(s.scratch)) t = 128;
  if (s.mode == RODAS3_COOP && t != 128 && t != 256) t = 128;  /* its two block sizes */
  s.threads = t;
  s.bps = env_int("GCCHEM_B200_BLOCKS_PER_SM", 0);
  if (cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking) != cudaSuccess) return -1;
  if (cudaEventCreate(&s.ev0) != cudaSuccess || cudaEventCreate(&s.ev1) != cudaSuccess) return -1;
  if (cudaMalloc(&s.qhead, sizeof(unsigned int)) != cudaSuccess) return -1;
  if (cudaMalloc(&s.bad, sizeof(int)) != cudaSuccess) return -1;
  s.init = true;
  return 0;
}

long round_up(long x, long m) { return (x + m - 1) / m * m; }

/* slots the launch of nCell cells uses in `mode` (-1: the device's mode);
   the cooperative kernel keeps each cell in shared memory and uses none */
long slots_for(const DevState& s, int nCell, int mode = -1) {
  if (mode < 0) mode = s.mode;
  if (mode == RODAS3_COOP) return 0;
  const long bytes_per_slot = (long)rodas3_ws_elems() * 8;
  if (mode == RODAS3_PLAIN || mode == RODAS3_PLAIN_FUSED) {
    long chunk = nCell;
    if (s.chunk > 0) {
      chunk = std::min((long)s.chunk, (long)nCell);
    } else if (env_is("GC_GPU_WORKSPACE", "global")) {
      /* low-memory mode of the reference: chunked launches
         (gc_gpu_batch_api.F90:307-313) */
      chunk = env_int("GC_GPU_CHUNK", 32768);
      chunk = std::max(1024L, std::min(chunk, (long)nCell));
    }
    /* never plan more than 3/4 of the device's free memory */
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) == cudaSuccess) {
      long cap = (long)((double)fr * 0.75 / (double)bytes_per_slot);
      cap = std::max(1024L, cap / 1024 * 1024);
      chunk = std::min(chunk, cap);
    }
    return round_up(chunk, 32);
  }
  int bps = s.bps;
  if (bps <= 0) bps = rodas3_persistent_blocks_per_sm(s.threads, s.scratch);
  if (bps <= 0) bps = 1;
  long slots = (long)s.sm_count * bps * s.threads;
  const long need = round_up(nCell, s.threads);
  return std::min(slots, need);
}

/* caller holds s.mu */
int ensure_ws(DevState& s, long slots) {
  if (slots <= s.ws_slots) return 0;
  if (s.ws) { cudaFree(s.ws); s.ws = nullptr; s.ws_slots = 0; }
  const size_t bytes = (size_t)slots * rodas3_ws_elems() * sizeof(double);
  if (cudaMalloc(&s.ws, bytes) != cudaSuccess) { cudaGetLastError(); return -1; }
  s.ws_slots = slots;
  return 0;
}

/* caller holds s.mu; scratch of the device cost sort for n keys */
int ensure_sortc(DevState& s, int n) {
  const long need = rodas3_cost_scratch(n);
  if (need <= s.sortc_n) return 0;
  if (s.sortc) { cudaFree(s.sortc); s.sortc = nullptr; s.sortc_n = 0; }
  if (cudaMalloc(&s.sortc, (size_t)need * sizeof(unsigned long long)) != cudaSuccess) {
    cudaGetLastError();
    return -1;
  }
  s.sortc_n = need;
  return 0;
}

int ensure_buf(DevState& s, size_t bytes) {
  if (bytes <= s.buf_bytes) return 0;
  if (s.buf) { cudaFree(s.buf); s.buf = nullptr; s.buf_bytes = 0; }
  if (cudaMalloc(&s.buf, bytes) != cudaSuccess) { cudaGetLastError(); return -1; }
  s.buf_bytes = bytes;
  return 0;
}

int current_device() {
  int d = -1;
  if (cudaGetDevice(&d) != cudaSuccess) return -1;
  return (d >= 0 && d < kMaxDev) ? d : -1;
}

void fill_ierr(int* IERR, int n, int code) {
  for (int i = 0; i < n; ++i) IERR[i] = code;
}

int launch_on(DevState& s, int nCell, double Tstart, double Tend, double* C,
              const double* RCONST, const double* ATOL, const double* RTOL,
              const int* ICNTRL, const double* RCNTRL, const int* order,
              int* ISTAT, double* RSTAT, int* IERR, cudaStream_t st,
              int* nfail = nullptr, const double* ATOLr = nullptr,
              const double* RTOLr = nullptr, double* ckpt = nullptr, int ckpt_max = 0) {
  /* the checkpointing forward of the adjoint runs on the persistent kernel
     when the cooperative kernel is selected (it stores no checkpoints) */
  const int mode = (s.mode == RODAS3_COOP && ckpt != nullptr) ? RODAS3_PERSISTENT : s.mode;
  const long slots = slots_for(s, nCell, mode);
  if (ensure_ws(s, slots) != 0) return -2;
  Rodas3Launch L;
  L.mode = mode;
  L.shared_scratch = s.scratch;
  L.nfail = nfail;
  L.ATOLr = ATOLr;
  L.RTOLr = RTOLr;
  L.ckpt = ckpt;
  L.ckpt_max = ckpt_max;
  L.ncell = nCell;
  L.tstart = Tstart; L.tend = Tend;
  L.C = C; L.RCONST = RCONST; L.ATOL = ATOL; L.RTOL = RTOL;
  L.ICNTRL = ICNTRL; L.RCNTRL = RCNTRL; L.order = order;
  L.ISTAT = ISTAT; L.RSTAT = RSTAT; L.IERR = IERR;
  L.ws = s.ws; L.slots = slots; L.qhead = s.qhead; L.threads = s.threads;
  if (mode == RODAS3_COOP) {
    /* resident blocks: SMs x blocks per SM (the occupancy limit, or fewer
       when set_launch asked for fewer) */
    const int occ = rodas3_coop_blocks_per_sm(s.threads);
    const int bps = (s.bps > 0 && s.bps < occ) ? s.bps : occ;
    if (bps <= 0) return -3;
    return rodas3_coop_launch(&L, s.sm_count * bps, st) == cudaSuccess ? 0 : -3;
  }
  if (rodas3_launch(&L, st) != cudaSuccess) return -3;
  return 0;
}

}  // namespace

extern "C" {

void gc_gpu_integrate_batch_dev(int dev, int nCell, double Tstart, double Tend,
                                double* C, const double* RCONST,
                                const double* ATOL, const double* RTOL,
                                const int* ICNTRL, const double* RCNTRL,
                                const int* Perm, int* ISTAT, double* RSTAT,
                                int* IERR, double* tTotal, double* tKernel) {
  const auto t0 = std::chrono::steady_clock::now();
  *tTotal = 0.0;
  *tKernel = 0.0;
  if (dev >= 0) {
    if (gc_gpu_set_device(dev) != dev) {
      fill_ierr(IERR, nCell, -99);
      return;
    }
  }
  if (nCell <= 0) return;
  const int d = current_device();
  if (d < 0) { fill_ierr(IERR, nCell, -99); return; }
  DevState& s = g_dev[d];
  std::lock_guard<std::mutex> lock(s.mu);
  if (ensure_init(s, d) != 0) { fill_ierr(IERR, nCell, -100); return; }

  /* every launch slot must name a column 1..nCell */
  for (int i = 0; i < nCell; ++i) {
    if (Perm[i] < 1 || Perm[i] > nCell) { fill_ierr(IERR, nCell, -100); return; }
  }
  int nvar, nfix, nreact, nnz;
  rodas3_sizes(&nvar, &nfix, &nreact, &nnz);
  const int nspec = nvar + nfix;
  const size_t n = (size_t)nCell;
  /* one device buffer, 256-byte aligned sub-arrays */
  size_t off = 0;
  auto take = [&](size_t bytes) { size_t o = off; off += (bytes + 255) / 256 * 256; return o; };
  const size_t oC = take(n * nspec * 8), oR = take(n * nreact * 8);
  const size_t oA = take((size_t)nvar * 8), oT = take((size_t)nvar * 8);
  const size_t oIC = take(n * 20 * 4), oRC = take(n * 20 * 8), oP = take(n * 4);
  const size_t oO = take(n * 4), oIS = take(n * 8 * 4), oRS = take(n * 3 * 8);
  const size_t oE = take(n * 4);
  if (ensure_buf(s, off) != 0) { fill_ierr(IERR, nCell, -100); return; }
  char* b = s.buf;
  double* dC = (double*)(b + oC);
  cudaStream_t st = s.stream;
  cudaMemcpyAsync(dC, C, n * nspec * 8, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(b + oR, RCONST, n * nreact * 8, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(b + oA, ATOL, (size_t)nvar * 8, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(b + oT, RTOL, (size_t)nvar * 8, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(b + oIC, ICNTRL, n * 20 * 4, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(b + oRC, RCNTRL, n * 20 * 8, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(b + oP, Perm, n * 4, cudaMemcpyHostToDevice, st);
  /* Perm was checked on the host above, so the conversion, the solve and
     the copies back are enqueued without waiting in between */
  rodas3_perm_to_order((const int*)(b + oP), nCell, (int*)(b + oO), s.bad, st);
  cudaEventRecord(s.ev0, st);
  int rc = launch_on(s, nCell, Tstart, Tend, dC, (const double*)(b + oR),
                     (const double*)(b + oA), (const double*)(b + oT),
                     (const int*)(b + oIC), (const double*)(b + oRC),
                     (const int*)(b + oO), (int*)(b + oIS), (double*)(b + oRS),
                     (int*)(b + oE), st);
  cudaEventRecord(s.ev1, st);
  if (rc != 0) {
    cudaStreamSynchronize(st);
    cudaGetLastError();
    fill_ierr(IERR, nCell, -100);
    return;
  }
  cudaMemcpyAsync(C, dC, n * nspec * 8, cudaMemcpyDeviceToHost, st);
  cudaMemcpyAsync(ISTAT, b + oIS, n * 8 * 4, cudaMemcpyDeviceToHost, st);
  cudaMemcpyAsync(RSTAT, b + oRS, n * 3 * 8, cudaMemcpyDeviceToHost, st);
  cudaMemcpyAsync(IERR, b + oE, n * 4, cudaMemcpyDeviceToHost, st);
  if (cudaStreamSynchronize(st) != cudaSuccess) {
    cudaGetLastError();
    fill_ierr(IERR, nCell, -100);
    return;
  }
  float ms = 0.f;
  cudaEventElapsedTime(&ms, s.ev0, s.ev1);
  *tKernel = ms * 1e-3;
  *tTotal = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

void gc_gpu_integrate_batch(int nCell, double Tstart, double Tend, double* C,
                            const double* RCONST, const double* ATOL,
                            const double* RTOL, const int* ICNTRL,
                            const double* RCNTRL, const int* Perm, int* ISTAT,
                            double* RSTAT, int* IERR, double* tTotal,
                            double* tKernel) {
  gc_gpu_integrate_batch_dev(-1, nCell, Tstart, Tend, C, RCONST, ATOL, RTOL,
                             ICNTRL, RCNTRL, Perm, ISTAT, RSTAT, IERR, tTotal,
                             tKernel);
}

void gc_gpu_selftest(int* rc, int* nsteps, double* tTotal) {
  int nvar, nfix, nreact, nnz;
  rodas3_sizes(&nvar, &nfix, &nreact, &nnz);
  const int nspec = nvar + nfix;
  double* C = (double*)malloc(sizeof(double) * nspec);
  double* R = (double*)calloc(nreact, sizeof(double));
  double* atol = (double*)malloc(sizeof(double) * nvar);
  double* rtol = (double*)malloc(sizeof(double) * nvar);
  int ic[20] = {0};
  double rcn[20] = {0};
  int istat[8] = {0}, ierr = 0, perm = 1;
  double rstat[3] = {0}, tk = 0.0;
  *rc = 0; *nsteps = 0; *tTotal = 0.0;
  if (!C || !R || !atol || !rtol) { free(C); free(R); free(atol); free(rtol); return; }
  for (int i = 0; i < nspec; ++i) C[i] = 1.0e6;
  for (int i = 0; i < nvar; ++i) { atol[i] = 1.0e-2; rtol[i] = 0.5e-2; }
  ic[0] = 1; ic[1] = 0; ic[2] = 4; ic[6] = 1; ic[14] = -1;
  gc_gpu_integrate_batch(1, 0.0, 1200.0, C, R, atol, rtol, ic, rcn, &perm,
                         istat, rstat, &ierr, tTotal, &tk);
  *rc = ierr;
  *nsteps = istat[2];
  free(C); free(R); free(atol); free(rtol);
}

void gc_gpu_info(int* nDev, char* devName, int nameLen) {
  *nDev = 0;
  if (nameLen > 0) devName[0] = '\0';
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) { cudaGetLastError(); return; }
  *nDev = n;
  if (n > 0 && nameLen > 1) {
    cudaDeviceProp p;
    if (cudaGetDeviceProperties(&p, 0) == cudaSuccess) {
      int m = (int)strnlen(p.name, sizeof(p.name));
      if (m > nameLen - 1) m = nameLen - 1;
      memcpy(devName, p.name, (size_t)m);
      devName[m] = '\0';
    }
  }
}

int gc_gpu_set_device(int d) {
  if (cudaSetDevice(d) != cudaSuccess) { cudaGetLastError(); return -1; }
  int cur = -1;
  if (cudaGetDevice(&cur) != cudaSuccess) { cudaGetLastError(); return -1; }
  return cur;
}

void gcchem_b200_sizes(int* nvar, int* nfix, int* nreact, int* nnz) {
  rodas3_sizes(nvar, nfix, nreact, nnz);
}

int gcchem_b200_set_launch(int mode, int threads, int blocks_per_sm) {
  if (mode != RODAS3_PLAIN && mode != RODAS3_PERSISTENT && mode != RODAS3_PLAIN_FUSED &&
      mode != RODAS3_COOP) return -1;
  if (threads < 0 || threads % 32 != 0 || threads > 256 || blocks_per_sm < 0) return -1;
  /* the cooperative kernel: 128 or 256 threads per cell, tables generated */
  if (mode == RODAS3_COOP && (!rodas3_coop_ok() || (threads != 0 && threads != 128 &&
                                                     threads != 256))) return -1;
  const int d = current_device();
  if (d < 0) return -1;
  DevState& s = g_dev[d];
  std::lock_guard<std::mutex> lock(s.mu);
  if (ensure_init(s, d) != 0) return -1;
  if ((threads > 0 ? threads : 128) > rodas3_max_threads(s.scratch)) return -1;
  s.mode = mode;
  s.threads = threads > 0 ? threads : 128;
  s.bps = blocks_per_sm;
  return 0;
}

int gcchem_b200_integrate_device(int nCell, double Tstart, double Tend,
                                 double* C, const double* RCONST,
                                 const double* ATOL, const double* RTOL,
                                 const int* ICNTRL, const double* RCNTRL,
                                 const int* order, int* ISTAT, double* RSTAT,
                                 int* IERR, void* stream) {
  if (nCell <= 0) return 0;
  const int d = current_device();
  if (d < 0) return -1;
  DevState& s = g_dev[d];
  std::lock_guard<std::mutex> lock(s.mu);
  if (ensure_init(s, d) != 0) return -1;
  return launch_on(s, nCell, Tstart, Tend, C, RCONST, ATOL, RTOL, ICNTRL,
                   RCNTRL, order, ISTAT, RSTAT, IERR, (cudaStream_t)stream);
}

int gcchem_b200_integrate_device_retry(int nCell, double Tstart, double Tend,
                                       double* C, const double* RCONST,
                                       const double* ATOL, const double* RTOL,
                                       const double* ATOLr, const double* RTOLr,
                                       const int* ICNTRL, const double* RCNTRL,
                                       const int* order, int* ISTAT, double* RSTAT,
                                       int* IERR, int* nfail, void* stream) {
  if (nCell <= 0) return 0;
  const int d = current_device();
  if (d < 0) return -1;
  DevState& s = g_dev[d];
  std::lock_guard<std::mutex> lock(s.mu);
  if (ensure_init(s, d) != 0) return -1;
  /* one launch: a lane whose first solve fails starts the retry at once */
  cudaStream_t st = (cudaStream_t)stream;
  if (cudaMemsetAsync(nfail, 0, 2 * sizeof(int), st) != cudaSuccess) return -3;
  return launch_on(s, nCell, Tstart, Tend, C, RCONST, ATOL, RTOL, ICNTRL, RCNTRL, order,
                   ISTAT, RSTAT, IERR, st, nfail, ATOLr, RTOLr);
}

int gcchem_b200_integrate_device_ckpt(int nCell, double Tstart, double Tend, double* C,
                                      const double* RCONST, const double* ATOL,
                                      const double* RTOL, const int* ICNTRL,
                                      const double* RCNTRL, const int* order, int* ISTAT,
                                      double* RSTAT, int* IERR, double* ckpt, int ckpt_max,
                                      void* stream) {
  if (nCell <= 0) return 0;
  if (!ckpt || ckpt_max <= 0) return -1;
  const int d = current_device();
  if (d < 0) return -1;
  DevState& s = g_dev[d];
  std::lock_guard<std::mutex> lock(s.mu);
  if (ensure_init(s, d) != 0) return -1;
  return launch_on(s, nCell, Tstart, Tend, C, RCONST, ATOL, RTOL, ICNTRL, RCNTRL, order,
                   ISTAT, RSTAT, IERR, (cudaStream_t)stream, nullptr, nullptr, nullptr, ckpt,
                   ckpt_max);
}

int gcchem_b200_adjoint_device(int nCell, const double* C0, const double* RCONST,
                               const int* ISTAT, const double* ckpt, int ckpt_max,
                               const double* lam, double* gC0, double* gK, int* ierr,
                               void* stream) {
  if (nCell <= 0) return 0;
  const int d = current_device();
  if (d < 0) return -1;
  DevState& s = g_dev[d];
  std::lock_guard<std::mutex> lock(s.mu);
  if (ensure_init(s, d) != 0) return -1;
  const long per = (long)rodas3_adjoint_ws_elems() * 8;
  long slots = round_up(nCell, 32);
  size_t fr = 0, tot = 0;
  if (cudaMemGetInfo(&fr, &tot) == cudaSuccess) {
    long cap = (long)((double)fr * 0.5 / (double)per) / 32 * 32;
    if (cap < 32) cap = 32;
    if (slots > cap) slots = cap;
  }
  if (slots > s.aws_slots) {
    if (s.aws) { cudaFree(s.aws); s.aws = nullptr; s.aws_slots = 0; }
    if (cudaMalloc(&s.aws, (size_t)slots * per) != cudaSuccess) { cudaGetLastError(); return -2; }
    s.aws_slots = slots;
  }
  if (nCell > s.asort_n) {
    if (s.asort) { cudaFree(s.asort); s.asort = nullptr; s.asort_n = 0; }
    if (cudaMalloc(&s.asort, (size_t)nCell * 2 * sizeof(int)) != cudaSuccess) {
      cudaGetLastError();
      return -2;
    }
    s.asort_n = nCell;
  }
  if (ensure_sortc(s, nCell) != 0) return -2;
  return rodas3_adjoint_launch(nCell, C0, RCONST, ISTAT, ckpt, ckpt_max, lam, gC0, gK, ierr,
                               s.aws, s.aws_slots, s.asort, s.sortc,
                               (cudaStream_t)stream) == cudaSuccess ? 0 : -3;
}

int gcchem_b200_cost_order(const int* keys, int nCell, int* order, void* stream) {
  if (nCell <= 0) return 0;
  const int d = current_device();
  if (d < 0) return -1;
  DevState& s = g_dev[d];
  std::lock_guard<std::mutex> lock(s.mu);
  if (ensure_init(s, d) != 0) return -1;
  if (ensure_sortc(s, nCell) != 0) return -2;
  return rodas3_cost_order(keys, nCell, order, s.sortc, (cudaStream_t)stream) == cudaSuccess ? 0 : -1;
}

int gcchem_b200_reserve(int nCell) {
  const int d = current_device();
  if (d < 0) return -1;
  DevState& s = g_dev[d];
  std::lock_guard<std::mutex> lock(s.mu);
  if (ensure_init(s, d) != 0) return -1;
  return ensure_ws(s, slots_for(s, std::max(nCell, 1)));
}

void gcchem_b200_release(void) {
  const int d = current_device();
  if (d < 0) return;
  DevState& s = g_dev[d];
  std::lock_guard<std::mutex> lock(s.mu);
  if (s.ws) cudaFree(s.ws);
  if (s.buf) cudaFree(s.buf);
  if (s.aws) cudaFree(s.aws);
  if (s.asort) cudaFree(s.asort);
  if (s.sortc) cudaFree(s.sortc);
  s.sortc = nullptr; s.sortc_n = 0;
  if (s.gkeys) cudaFree(s.gkeys);
  s.gkeys = nullptr; s.gkeys_n = 0;
  s.aws = nullptr; s.aws_slots = 0;
  s.asort = nullptr; s.asort_n = 0;
  s.ws = nullptr; s.ws_slots = 0;
  s.buf = nullptr; s.buf_bytes = 0;
}

int gcchem_b200_set_row_scratch(int shared) {
  if (shared != 0 && shared != 1) return -1;
  if (shared && !rodas3_shared_scratch_ok()) return -1;
  const int d = current_device();
  if (d < 0) return -1;
  DevState& s = g_dev[d];
  std::lock_guard<std::mutex> lock(s.mu);
  if (ensure_init(s, d) != 0) return -1;
  if (s.threads > rodas3_max_threads(shared)) return -1;
  s.scratch = shared;
  return 0;
}

int gcchem_b200_set_chunk(int cells) {
  if (cells < 0) return -1;
  const int d = current_device();
  if (d < 0) return -1;
  DevState& s = g_dev[d];
  std::lock_guard<std::mutex> lock(s.mu);
  if (ensure_init(s, d) != 0) return -1;
  s.chunk = cells;
  return 0;
}

long gcchem_b200_workspace_slots(int nCell) {
  const int d = current_device();
  if (d < 0) return -1;
  DevState& s = g_dev[d];
  std::lock_guard<std::mutex> lock(s.mu);
  if (ensure_init(s, d) != 0) return -1;
  return slots_for(s, std::max(nCell, 1));
}

double gcchem_b200_phase_ms(int phase, long slots, int reps) {
  const int d = current_device();
  if (d < 0 || slots <= 0 || slots % 32 != 0) return -1.0;
  DevState& s = g_dev[d];
  std::lock_guard<std::mutex> lock(s.mu);
  if (ensure_init(s, d) != 0 || ensure_ws(s, slots) != 0) return -1.0;
  return rodas3_phase_ms(phase, slots, reps, s.ws);
}

double gcchem_b200_fp64_peak_tflops(void) {
  return rodas3_fp64_peak_tflops();
}

long gcchem_b200_workspace_bytes_per_slot(void) {
  return (long)rodas3_ws_elems() * 8;
}

int gcchem_b200_batch_map(int NX, int NY, int NZ, const int* PrevNsteps, const int* InChem,
                          int sort, int nCell, int* BatchMap, void* stream) {
  if (NX <= 0 || NY <= 0 || NZ <= 0 || !PrevNsteps || !BatchMap) return -1;
  const long ncells = (long)NX * NY * NZ;
  if (ncells > 2147483647L || nCell < 0 || nCell > ncells) return -1;
  const int d = current_device();
  if (d < 0) return -1;
  DevState& s = g_dev[d];
  std::lock_guard<std::mutex> lock(s.mu);
  if (ensure_init(s, d) != 0) return -1;
  if (ncells > s.gkeys_n) {
    if (s.gkeys) { cudaFree(s.gkeys); s.gkeys = nullptr; s.gkeys_n = 0; }
    if (cudaMalloc(&s.gkeys, (size_t)ncells * 2 * sizeof(int)) != cudaSuccess) {
      cudaGetLastError();
      return -2;
    }
    s.gkeys_n = ncells;
  }
  if (ensure_sortc(s, (int)ncells) != 0) return -2;
  cudaStream_t st = (cudaStream_t)stream;
  int* keys = s.gkeys;
  int* order = s.gkeys + ncells;
  if (rodas3_batch_keys((int)ncells, PrevNsteps, InChem, sort, keys, st) != cudaSuccess) return -3;
  if (rodas3_cost_order(keys, (int)ncells, order, s.sortc, st) != cudaSuccess) return -3;
  return rodas3_batch_decode(nCell, NX, NY, order, BatchMap, st) == cudaSuccess ? 0 : -3;
}

int gcchem_b200_gather(int nCell, int NX, int NY, int NZ, const int* BatchMap,
                       const double* Conc, const int* MapKppSpc, double* C,
                       const double* RconstGrid, double* RCONST, const double* KPPHvalue,
                       double* RCNTRL, void* stream) {
  if (nCell <= 0) return 0;
  if (NX <= 0 || NY <= 0 || NZ <= 0 || !BatchMap || !Conc || !MapKppSpc || !C) return -1;
  if ((RconstGrid == nullptr) != (RCONST == nullptr)) return -1;
  if ((KPPHvalue == nullptr) != (RCNTRL == nullptr)) return -1;
  return rodas3_gather(nCell, NX, NY, NZ, BatchMap, Conc, MapKppSpc, C, RconstGrid, RCONST,
                       KPPHvalue, RCNTRL, (cudaStream_t)stream) == cudaSuccess ? 0 : -3;
}

int gcchem_b200_scatter(int nCell, int NX, int NY, int NZ, const int* BatchMap, double* Conc,
                        const int* MapKppSpc, const double* C, const int* ISTAT,
                        const double* RSTAT, double* KPPHvalue, int* PrevNsteps,
                        float* KppDiag, void* stream) {
  if (nCell <= 0) return 0;
  if (NX <= 0 || NY <= 0 || NZ <= 0 || !BatchMap || !Conc || !MapKppSpc || !C || !ISTAT ||
      !RSTAT)
    return -1;
  return rodas3_scatter(nCell, NX, NY, NZ, BatchMap, Conc, MapKppSpc, C, ISTAT, RSTAT,
                        KPPHvalue, PrevNsteps, KppDiag, (cudaStream_t)stream) == cudaSuccess
             ? 0 : -3;
}

}  /* extern "C" */
