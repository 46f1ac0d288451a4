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
