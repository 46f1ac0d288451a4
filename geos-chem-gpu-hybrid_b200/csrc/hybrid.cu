/*
 * hybrid.cu -- the hybrid CPU/GPU split of one chemistry step (host code).
 *
 * The model's GC_BATCH_CHEM=3 mode (src/geos-chem/GeosCore/fullchem_mod.F90)
 * solves the most expensive cells of a cost-ordered batch on the GPU(s) and
 * the rest on the host cores at the same time:
 *
 *   work model  (:997-1005)  cost(slot) = max(previous Nstp, 1); HybWork =
 *               prefix sums over the cost-ordered slots
 *   split       (:1006-1019) once both rates are measured (and the fraction
 *               is not fixed), frac = rate_gpu / (rate_gpu + rate_cpu)
 *               clamped to [0.01, 0.99]; the head is the longest prefix whose
 *               work does not exceed frac * total work
 *   devices     (:1020-1055) the head is cut into contiguous slices of equal
 *               weighted work, one per device; weights are the measured
 *               per-device rates once every device has one, else equal
 *   rates       (:2678-2706) exponential moving averages (weight 1/2) of
 *               work per second: per device (its slice / its launch wall
 *               time), GPU (head / slowest device), CPU (tail / CPU time)
 *
 * GcHybrid holds that state between chemistry steps.  gcchem_b200_hybrid_plan
 * and gcchem_b200_hybrid_update are the bookkeeping alone (no CUDA call, so
 * they run without a GPU); gcchem_b200_hybrid_step runs a whole step: one
 * host thread per device slice issues the legacy blocking launch
 * (gc_gpu_integrate_batch_dev, as the model's OpenMP threads do) while the
 * calling thread solves the tail through the caller's CPU integrator
 * callback, then the rates are updated.  Slices use 1-based inclusive slot
 * ranges, as the model's devLo/devHi.
 */
#include <algorithm>
#include <chrono>
#include <thread>
#include <vector>

#include "rodas3_kernels.h"
#include "../../include/gcchem_gpu.h"

struct GcHybrid {
  int ndev_max = 1;           /* GC_GPU_NDEV */
  double frac = 0.5;          /* HybWorkFrac: GPU share of the work */
  int fixed = 0;              /* GC_GPU_FRAC_FIXED */
  double rate_gpu = 0.0;      /* HybRateGpu, work per second */
  double rate_cpu = 0.0;      /* HybRateCpu */
  std::vector<double> dev_rate;   /* HybDevRate(0:ndev_max-1) */
  /* the last plan */
  std::vector<long long> work;    /* HybWork(0:n) */
  int n = 0, ngpu = 0, ndev_use = 0;
  std::vector<int> lo, hi;        /* devLo/devHi, 1-based inclusive */
};

namespace {

void ema(double& r, double x) { r = (r > 0.0) ? 0.5 * r + 0.5 * x : x; }

}  // namespace

extern "C" {

GcHybrid* gcchem_b200_hybrid_create(int ndev, double frac, int fixed_frac) {
  if (ndev < 1 || ndev > 64 || !(frac >= 0.0 && frac <= 1.0)) return nullptr;
  GcHybrid* h = new GcHybrid;
  h->ndev_max = ndev;
  h->frac = frac;
  h->fixed = fixed_frac ? 1 : 0;
  h->dev_rate.assign(ndev, 0.0);
  return h;
}

void gcchem_b200_hybrid_destroy(GcHybrid* h) { delete h; }

int gcchem_b200_hybrid_plan(GcHybrid* h, int nCell, const int* prevNsteps, int* nGpu,
                            int* nDevUse, int* devLo, int* devHi) {
  if (!h || nCell < 0 || (nCell > 0 && !prevNsteps)) return -1;
  const int n = nCell;
  h->n = n;
  h->work.assign((size_t)n + 1, 0);
  for (int ic = 1; ic <= n; ++ic)
    h->work[ic] = h->work[ic - 1] + std::max(prevNsteps[ic - 1], 1);
  const double wtot = (double)h->work[n];
  if (!h->fixed && h->rate_gpu > 0.0 && h->rate_cpu > 0.0) {
    h->frac = h->rate_gpu / (h->rate_gpu + h->rate_cpu);
    h->frac = std::min(std::max(h->frac, 0.01), 0.99);
  }
  h->frac = std::min(std::max(h->frac, 0.0), 1.0);
  double target = h->frac * wtot;
  int ngpu = 0;
  for (int ic = 1; ic <= n; ++ic) {
    if ((double)h->work[ic] > target) break;
    ngpu = ic;
  }
  h->ngpu = ngpu;
  int nd = h->ndev_max;
  if (ngpu < nd) nd = std::max(ngpu, 1);
  h->ndev_use = nd;
  /* device weights: the measured rates once every device has one */
  std::vector<double> w(nd, 1.0);
  bool all = true;
  for (int d = 0; d < nd; ++d) all = all && h->dev_rate[d] > 0.0;
  if (all)
    for (int d = 0; d < nd; ++d) w[d] = h->dev_rate[d];
  double wsum = 0.0;
  for (int d = 0; d < nd; ++d) wsum += w[d];
  h->lo.assign(nd, 1);
  h->hi.assign(nd, 0);
  int idx = 0;
  double cum = 0.0;
  for (int d = 0; d < nd; ++d) {
    h->lo[d] = idx + 1;
    if (d == nd - 1) {
      h->hi[d] = ngpu;
    } else {
      cum += w[d];
      target = (double)h->work[ngpu] * cum / wsum;
      for (int ic = idx + 1; ic <= ngpu; ++ic) {
        if ((double)h->work[ic] > target) break;
        idx = ic;
      }
      h->hi[d] = idx;
    }
    idx = h->hi[d];
  }
  if (nGpu) *nGpu = ngpu;
  if (nDevUse) *nDevUse = nd;
  for (int d = 0; d < nd; ++d) {
    if (devLo) devLo[d] = h->lo[d];
    if (devHi) devHi[d] = h->hi[d];
  }
  return 0;
}

int gcchem_b200_hybrid_update(GcHybrid* h, const double* devTw, double tCpu) {
  if (!h || (h->ndev_use > 0 && !devTw)) return -1;
  double gpu_tw = 0.0;
  for (int d = 0; d < h->ndev_use; ++d) {
    gpu_tw = std::max(gpu_tw, devTw[d]);
    if (h->hi[d] >= h->lo[d] && devTw[d] > 0.0)
      ema(h->dev_rate[d], (double)(h->work[h->hi[d]] - h->work[h->lo[d] - 1]) / devTw[d]);
  }
  if (h->ngpu > 0 && gpu_tw > 0.0) ema(h->rate_gpu, (double)h->work[h->ngpu] / gpu_tw);
  const int ncpu = h->n - h->ngpu;
  if (ncpu > 0 && tCpu > 0.0)
    ema(h->rate_cpu, (double)(h->work[h->n] - h->work[h->ngpu]) / tCpu);
  return 0;
}

int gcchem_b200_hybrid_state(const GcHybrid* h, double* frac, double* rateGpu,
                             double* rateCpu, double* devRate) {
  if (!h) return -1;
  if (frac) *frac = h->frac;
  if (rateGpu) *rateGpu = h->rate_gpu;
  if (rateCpu) *rateCpu = h->rate_cpu;
  if (devRate)
    for (int d = 0; d < h->ndev_max; ++d) devRate[d] = h->dev_rate[d];
  return 0;
}

int gcchem_b200_hybrid_step(GcHybrid* h, int nCell, double Tstart, double Tend, double* C,
                            const double* RCONST, const double* ATOL, const double* RTOL,
                            const int* ICNTRL, const double* RCNTRL, const int* prevNsteps,
                            int* ISTAT, double* RSTAT, int* IERR,
                            void (*cpu_tail)(int first, int count, void* user), void* user,
                            int* nGpu, double* tGpu, double* tCpu) {
  if (!h || nCell <= 0) return nCell == 0 ? 0 : -1;
  int nvar, nfix, nreact, nnz;
  rodas3_sizes(&nvar, &nfix, &nreact, &nnz);
  const long nspec = nvar + nfix;
  if (gcchem_b200_hybrid_plan(h, nCell, prevNsteps, nullptr, nullptr, nullptr, nullptr) != 0)
    return -1;
  const int ngpu = h->ngpu, nd = h->ndev_use;
  if (ngpu < nCell && !cpu_tail) return -1;     /* the tail needs a CPU integrator */
  std::vector<double> dev_tw(nd, 0.0);
  std::vector<std::vector<int>> perms(nd);
  std::vector<std::thread> pool;
  for (int d = 0; d < nd; ++d) {
    const int lo = h->lo[d], hi = h->hi[d];
    if (hi < lo) continue;
    const int cnt = hi - lo + 1;
    perms[d].resize(cnt);
    for (int i = 0; i < cnt; ++i) perms[d][i] = i + 1;   /* slice-local identity Perm */
    const long o = lo - 1;
    pool.emplace_back([=, &dev_tw, &perms]() {
      const auto t0 = std::chrono::steady_clock::now();
      double ta = 0.0, tk = 0.0;
      gc_gpu_integrate_batch_dev(d, cnt, Tstart, Tend, C + o * nspec, RCONST + o * nreact,
                                 ATOL, RTOL, ICNTRL + o * 20, RCNTRL + o * 20,
                                 perms[d].data(), ISTAT + o * 8, RSTAT + o * 3, IERR + o,
                                 &ta, &tk);
      dev_tw[d] = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    });
  }
  double tc = 0.0;
  if (ngpu < nCell) {
    const auto t0 = std::chrono::steady_clock::now();
    cpu_tail(ngpu, nCell - ngpu, user);
    tc = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
  for (auto& t : pool) t.join();
  gcchem_b200_hybrid_update(h, dev_tw.data(), tc);
  double tg = 0.0;
  for (int d = 0; d < nd; ++d) tg = std::max(tg, dev_tw[d]);
  if (nGpu) *nGpu = ngpu;
  if (tGpu) *tGpu = tg;
  if (tCpu) *tCpu = tc;
  return 0;
}

}  /* extern "C" */
