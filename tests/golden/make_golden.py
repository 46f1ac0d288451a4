"""Writes the golden fixtures in this directory (run from the repository root):

    python tests/golden/make_golden.py

* ``selftest_kat.json`` -- the reference's own known answer for
  gc_gpu_selftest (gpulib/src/gc_gpu_batch_api.F90:349-376, reported as
  rc = 1, nsteps = 12 in the reference's docs/GPU_IN_MODEL_RESULTS.md:181-186),
  with the full ISTAT/RSTAT the oracle produces for it.
* ``fun_jac_interp.npz`` -- Fun_SPLIT and Jac_SP values of the reference's
  parsed expression trees, evaluated by a plain Python interpreter (IEEE
  double, one operation at a time, Fortran association), for two seeded
  states.  Independent of the C code generator.
* ``oracle_cells.npz`` -- oracle solutions of 8 seeded cells (regression
  fixture for the oracle and, bit for bit, for the --fmad=false library).
"""
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path[:0] = [ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "geos-chem-gpu-hybrid_b200"),
                os.path.join(ROOT, "tests")]

import oracle  # noqa: E402
import workloads  # noqa: E402
from mechanism import codegen  # noqa: E402
from test_generated import _interp_fun, _interp_jac, _state  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))


def selftest_batch():
    nspec, nreact, nvar = 356, 1058, 353
    b = workloads.Batch(np.full((nspec, 1), 1.0e6, order="F"),
                        np.zeros((nreact, 1), order="F"), np.full(nvar, 1e-2),
                        np.full(nvar, 0.5e-2), np.zeros((20, 1), np.int32, order="F"),
                        np.zeros((20, 1), order="F"))
    b.ICNTRL[[0, 1, 2, 6, 14], 0] = [1, 0, 4, 1, -1]
    return b


def main():
    mech = codegen.load("fullchem")
    C, ist, rst, ierr = oracle.integrate_batch(selftest_batch())
    with open(os.path.join(HERE, "selftest_kat.json"), "w") as fh:
        json.dump({"reference_rc": 1, "reference_nsteps": 12, "ierr": int(ierr[0]),
                   "istat": ist[:, 0].tolist(), "rstat": [float(x) for x in rst[:, 0]]}, fh,
                  indent=1)
    arrs = {}
    for seed in (0, 1):
        V, F, R = _state(mech, seed)
        arrs[f"V{seed}"], arrs[f"F{seed}"], arrs[f"R{seed}"] = V, F, R
        arrs[f"fun{seed}"] = _interp_fun(mech, V, F, R)
        arrs[f"jac{seed}"] = _interp_jac(mech, V, F, R)
    np.savez_compressed(os.path.join(HERE, "fun_jac_interp.npz"), **arrs)
    b = workloads.plain_small(8, seed=77)
    C, ist, rst, ierr = oracle.integrate_batch(b)
    np.savez_compressed(os.path.join(HERE, "oracle_cells.npz"), C0=b.C, RCONST=b.RCONST,
                        ICNTRL=b.ICNTRL, RCNTRL=b.RCNTRL, ATOL=b.ATOL, RTOL=b.RTOL, C=C,
                        ISTAT=ist, RSTAT=rst, IERR=ierr)
    print("golden fixtures written")


if __name__ == "__main__":
    main()
