"""bench.py's per-cell parity block (host logic only): it compares the
sampled columns of the GPU state with the oracle's, with both denominator
floors, and counts cells over the tolerance and failures on either side."""
import importlib
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    if ROOT not in sys.path:
        sys.path.insert(0, ROOT)
    return importlib.import_module("bench")


def test_parity_report_floors_and_counts():
    b = _bench()
    nvar, nspec, n = 4, 5, 6
    rng = np.random.default_rng(0)
    ref_C = rng.uniform(1.0, 10.0, (nspec, 3))
    ref_C[1, 2] = 1e-8                              # tiny species: floor matters
    idx = np.array([1, 3, 5])
    gpu_C = np.zeros((n, nspec))
    gpu_C[idx] = ref_C.T
    gpu_C[3, 0] *= 1 + 3e-6                         # one cell over 1e-6
    gpu_C[5, 1] = 2e-8                              # 1e-8 abs: tiny against 1e-2, huge against 1e-20
    rist = np.ones((8, 3), np.int32)
    rierr = np.ones(3, np.int32)
    gpu_ist = np.ones((n, 8), np.int32)
    gpu_ist[5, 2] = 7
    gpu_ierr = np.ones(n, np.int32)
    out = b.parity_report(nvar, idx, (ref_C, rist, None, rierr), gpu_C, gpu_ist, gpu_ierr)
    assert out["cells"] == 3
    assert out["floor_1e-2"]["cells_over_tol"] == 1
    assert abs(out["floor_1e-2"]["max_rel"] - 3e-6) < 1e-12
    assert out["floor_1e-20"]["cells_over_tol"] == 2
    assert out["floor_1e-20"]["max_rel"] > 0.9
    assert out["gpu_failures"] == 0 and out["oracle_failures"] == 0 and out["ierr_equal"]
    assert out["istat_equal_cells"] == 2


def test_chain_cpu_baseline_is_the_chained_oracle(pkg, orc):
    """The chained workload's CPU leg runs `chain` oracle steps with the
    device chain's clamp and warm start; fed its own end state as the GPU's,
    the parity block reports no difference."""
    b = _bench()
    batch = pkg.workloads.plain_small(40, seed=3)
    batch.ICNTRL[3, :] = 5000

    class Args:
        chain = 2
        cpu_step_seconds = 0.2

    # the chain's end state, computed the way the CPU leg computes it
    sub = pkg.workloads.subset(batch, np.arange(batch.n))
    for _ in range(Args.chain):
        C, ist, rst, ierr = orc.integrate_batch(sub)
        sub.C = np.asfortranarray(np.maximum(C, 0.0))
        sub.RCNTRL[2, :] = rst[2]
    cpu, par = b.chain_cpu_baseline(pkg, batch, Args, sub.C.T.copy(), ierr.copy(),
                                    orc.load().sizes[0])
    assert cpu["unit"] == "cells/s per chemistry step" and cpu["value"] > 0
    assert par["steps"] == 2 and par["cells"] >= 1
    assert par["floor_1e-20"]["max_rel"] == 0.0 and par["gpu_failures"] == 0


def test_cpu_single_thread_and_model(pkg, orc):
    """The one-thread oracle figure reported beside the all-core baseline."""
    b = _bench()
    batch = pkg.workloads.plain_small(64, seed=3)
    batch.ICNTRL[3, :] = 40
    out = b.cpu_single_thread(orc, batch, 0.2)
    assert out["cores"] == 1 and out["value"] > 0 and "cells strided" in out["sample"]
    assert isinstance(b.cpu_model(), str) and b.cpu_model()
