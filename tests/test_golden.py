"""The oracle against the committed golden fixtures (tests/golden/)."""
import json
import os

import numpy as np
import pytest

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _batch(pkg, g):
    return pkg.workloads.Batch(np.asfortranarray(g["C0"]), np.asfortranarray(g["RCONST"]),
                               g["ATOL"], g["RTOL"], np.asfortranarray(g["ICNTRL"]),
                               np.asfortranarray(g["RCNTRL"]))


def test_selftest_known_answer(orc):
    import sys
    sys.path.insert(0, HERE)
    from make_golden import selftest_batch
    kat = json.load(open(os.path.join(HERE, "selftest_kat.json")))
    C, ist, rst, ierr = orc.integrate_batch(selftest_batch())
    # the reference's documented answer
    assert ierr[0] == kat["reference_rc"] == 1
    assert ist[2, 0] == kat["reference_nsteps"] == 12
    assert ist[:, 0].tolist() == kat["istat"]
    assert rst[:, 0].tolist() == kat["rstat"]


def test_fun_jac_against_interpreter_fixture(orc):
    g = np.load(os.path.join(HERE, "fun_jac_interp.npz"))
    for seed in (0, 1):
        V, F, R = g[f"V{seed}"], g[f"F{seed}"], g[f"R{seed}"]
        assert np.array_equal(orc.fun(V, F, R).view(np.uint64), g[f"fun{seed}"].view(np.uint64))
        assert np.array_equal(orc.jac(V, F, R).view(np.uint64), g[f"jac{seed}"].view(np.uint64))


def test_oracle_cells_fixture(pkg, orc):
    g = np.load(os.path.join(HERE, "oracle_cells.npz"))
    C, ist, rst, ierr = orc.integrate_batch(_batch(pkg, g))
    assert np.array_equal(C.view(np.uint64), g["C"].view(np.uint64))
    assert np.array_equal(ist, g["ISTAT"]) and np.array_equal(ierr, g["IERR"])


@pytest.mark.gpu
@pytest.mark.timeout(120)
def test_gpu_nofma_against_fixture(pkg):
    g = np.load(os.path.join(HERE, "oracle_cells.npz"))
    s = pkg.solver("fullchem", "nofma")
    s.set_launch(pkg.PERSISTENT)
    C, ist, rst, ierr, *_ = s.integrate_batch(_batch(pkg, g))
    assert np.array_equal(C.view(np.uint64), g["C"].view(np.uint64))
    assert np.array_equal(ist, g["ISTAT"]) and np.array_equal(ierr, g["IERR"])
