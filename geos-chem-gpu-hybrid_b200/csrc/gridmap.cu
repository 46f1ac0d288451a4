/*
 * gridmap.cu -- the model's batch bookkeeping on the device: the cost-ordered
 * slot map, the gather of grid fields into the batch arrays and the scatter
 * of the solved batch back to the grid, so that a chemistry step can run
 * with its state resident in HBM and no host staging
 * (src/geos-chem/GeosCore/fullchem_mod.F90).
 *
 * Grid arrays are Fortran-ordered (NX, NY, NZ[, k]): cell (I,J,L), 1-based,
 * sits at c = (I-1) + NX*((J-1) + NY*(L-1)), so increasing c is the model's
 * L,J,I loop order.  BatchMap is (3, nCell) int, 1-based (I,J,L) per slot,
 * as the model's BatchMap.
 *
 *   batch_map  the pre-scan (:906-993): chemistry cells sorted by descending
 *              previous-step Nstp, ties in L,J,I order (stable), or in L,J,I
 *              order alone when sorting is off; cells outside the chemistry
 *              grid (mask 0) are left out.
 *   gather     (:1538-1543, :1749-1756) C(N,slot) = Conc(I,J,L,Map(N)) for
 *              KPP species that are model species (Map(N) > 0), 0 for the
 *              others; optionally RCONST(:,slot) from a grid-resident
 *              rate-constant field, and the warm start RCNTRL(3,slot) =
 *              KPPHvalue(I,J,L) (the step size the previous chemistry step
 *              predicted, which the model's integrator options carry).
 *   scatter    (:2878-3000) Conc(I,J,L,Map(N)) = max(C(N,slot), 0) for mapped
 *              species; KPPHvalue(I,J,L) = RSTAT(3,slot) (:2922);
 *              PrevNsteps(I,J,L) = ISTAT(3,slot) (:2868, the next pre-scan's
 *              sort key); optionally the KppDiags counters ISTAT(1:8) and
 *              the count of mapped species that came back negative
 *              (KppNegatives, :2983-2989) into a (NX,NY,NZ,9) float field.
 */
#include <cuda_runtime.h>
#include <limits.h>

#include "rodas3_device.cuh"
#include "rodas3_kernels.h"

__global__ void gm_keys(int ncells, const int* prev, const int* mask, int sort, int* keys) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncells) return;
  const bool in = mask ? (mask[c] != 0) : true;
  keys[c] = in ? (sort ? prev[c] : 0) : INT_MIN;
}

__global__ void gm_decode(int ncell, int NX, int NY, const int* order, int* map) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= ncell) return;
  const int c = order[s];
  const int i = c % NX, j = (c / NX) % NY, l = c / (NX * NY);
  map[3 * s] = i + 1;
  map[3 * s + 1] = j + 1;
  map[3 * s + 2] = l + 1;
}

__device__ __forceinline__ long gm_cell(const int* map, int s, int NX, int NY) {
  return (long)(map[3 * s] - 1) + (long)NX * ((long)(map[3 * s + 1] - 1) +
                                              (long)NY * (long)(map[3 * s + 2] - 1));
}

/* one thread per (species, slot), species fastest: C's columns are written
   contiguously; the grid reads follow the cost order */
__global__ void gm_gather(int ncell, int NX, int NY, long ncells, const int* map,
                          const double* conc, const int* kmap, double* C,
                          const double* rgrid, double* R, const double* hval, double* RC) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long)ncell * NSPEC) return;
  const int s = (int)(t / NSPEC), n = (int)(t % NSPEC);
  const long c = gm_cell(map, s, NX, NY);
  const int spc = kmap[n];
  C[(long)s * NSPEC + n] = (spc > 0) ? conc[(long)(spc - 1) * ncells + c] : 0.0;
  if (R) {
    for (int j = n; j < NREACT; j += NSPEC)
      R[(long)s * NREACT + j] = rgrid[(long)j * ncells + c];
  }
  if (RC && n == 0) RC[(long)s * 20 + 2] = hval[c];
}

__global__ void gm_scatter(int ncell, int NX, int NY, long ncells, const int* map,
                           double* conc, const int* kmap, const double* C, const int* ISTAT,
                           const double* RSTAT, double* hval, int* prev, float* diag) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= ncell) return;
  const long c = gm_cell(map, s, NX, NY);
  const double* cs = C + (long)s * NSPEC;
  int neg = 0;
  for (int n = 0; n < NSPEC; ++n) {
    const int spc = kmap[n];
    if (spc <= 0) continue;
    const double v = cs[n];
    if (v < 0.0) ++neg;
    conc[(long)(spc - 1) * ncells + c] = fmax(v, 0.0);
  }
  if (hval) hval[c] = RSTAT[(long)s * 3 + 2];
  if (prev) prev[c] = ISTAT[(long)s * 8 + 2];
  if (diag) {
    for (int k = 0; k < 8; ++k) diag[(long)k * ncells + c] = (float)ISTAT[(long)s * 8 + k];
    diag[8L * ncells + c] = (float)neg;
  }
}

extern "C" cudaError_t rodas3_batch_keys(int ncells, const int* prev, const int* mask, int sort,
                                         int* keys, cudaStream_t st) {
  gm_keys<<<(ncells + 255) / 256, 256, 0, st>>>(ncells, prev, mask, sort, keys);
  return cudaGetLastError();
}

extern "C" cudaError_t rodas3_batch_decode(int ncell, int NX, int NY, const int* order, int* map,
                                           cudaStream_t st) {
  if (ncell > 0) gm_decode<<<(ncell + 255) / 256, 256, 0, st>>>(ncell, NX, NY, order, map);
  return cudaGetLastError();
}

extern "C" cudaError_t rodas3_gather(int ncell, int NX, int NY, int NZ, const int* map,
                                     const double* conc, const int* kmap, double* C,
                                     const double* rgrid, double* R, const double* hval,
                                     double* RC, cudaStream_t st) {
  const long ncells = (long)NX * NY * NZ;
  const long work = (long)ncell * NSPEC;
  if (work > 0)
    gm_gather<<<(int)((work + 255) / 256), 256, 0, st>>>(ncell, NX, NY, ncells, map, conc,
                                                         kmap, C, rgrid, R, hval, RC);
  return cudaGetLastError();
}

extern "C" cudaError_t rodas3_scatter(int ncell, int NX, int NY, int NZ, const int* map,
                                      double* conc, const int* kmap, const double* C,
                                      const int* ISTAT, const double* RSTAT, double* hval,
                                      int* prev, float* diag, cudaStream_t st) {
  const long ncells = (long)NX * NY * NZ;
  if (ncell > 0)
    gm_scatter<<<(ncell + 127) / 128, 128, 0, st>>>(ncell, NX, NY, ncells, map, conc, kmap, C,
                                                    ISTAT, RSTAT, hval, prev, diag);
  return cudaGetLastError();
}
