"""GPU parity of the CUDA solver against the CPU oracle, through the C-ABI.

--fmad=false library: bit-exact per cell (C, ISTAT, RSTAT, IERR).
Production (FMA) library: every species within RTOL_PARITY relative of the
oracle, with the denominator floored at ATOL (1e-2 molecule cm^-3, the
solver's own absolute tolerance), and zero solver failures.
"""
import numpy as np
import pytest

pytestmark = [pytest.mark.gpu, pytest.mark.timeout(300)]

RTOL_PARITY = 1e-6
FLOOR = 1e-2


def _solver(pkg, variant, mode):
    s = pkg.solver("fullchem", variant)
    s.set_launch(mode)
    return s


def _bits(a):
    return np.ascontiguousarray(a).view(np.uint64 if a.dtype == np.float64 else np.uint32)


def _capped(b, max_steps=5000):
    """At most 5000 internal steps per cell (natural maximum ~200): a broken
    kernel then fails fast with IERR=-6 instead of running 200000 steps."""
    b.ICNTRL[3, :] = max_steps
    return b


@pytest.fixture(scope="module")
def batch256(pkg):
    return _capped(pkg.workloads.plain_small(256, seed=3))


@pytest.fixture(scope="module")
def ref256(orc, batch256):
    return orc.integrate_batch(batch256)


@pytest.mark.parametrize("mode", [0, 1, 3], ids=["plain", "persistent", "coop"])
@pytest.mark.parametrize("variant", ["nofma", "fma"])
def test_selftest_kat(pkg, variant, mode):
    s = _solver(pkg, variant, mode)
    rc, nsteps, tt = s.selftest()
    assert rc == 1 and nsteps == 12


@pytest.mark.parametrize("mode", [0, 1, 3], ids=["plain", "persistent", "coop"])
def test_bitexact_nofma(pkg, batch256, ref256, mode):
    s = _solver(pkg, "nofma", mode)
    C, ist, rst, ierr, tt, tk = s.integrate_batch(batch256)
    rC, rist, rrst, rierr = ref256
    assert np.array_equal(ierr, rierr)
    assert np.array_equal(ist, rist)
    assert np.array_equal(_bits(rst), _bits(rrst))
    assert np.array_equal(_bits(C), _bits(rC))


@pytest.mark.parametrize("mode", [0, 1, 3], ids=["plain", "persistent", "coop"])
def test_fma_tolerance(pkg, batch256, ref256, mode):
    s = _solver(pkg, "fma", mode)
    C, ist, rst, ierr, tt, tk = s.integrate_batch(batch256)
    rC, rist, rrst, rierr = ref256
    assert (ierr == 1).all() and (rierr == 1).all()
    n = s.nvar
    rel = np.abs(C[:n] - rC[:n]) / np.maximum(np.abs(rC[:n]), FLOOR)
    assert rel.max() <= RTOL_PARITY, rel.max()
    assert np.isfinite(C).all()


@pytest.mark.parametrize("mode", [0, 1, 3], ids=["plain", "persistent", "coop"])
def test_perm_columns(pkg, orc, mode):
    """Launch slot ic solves column Perm(ic) and writes that column."""
    b = _capped(pkg.workloads.plain_small(97, seed=5))
    perm = np.random.default_rng(0).permutation(b.n).astype(np.int32) + 1
    s = _solver(pkg, "nofma", mode)
    C, ist, rst, ierr, *_ = s.integrate_batch(b, perm=perm)
    rC, rist, rrst, rierr = orc.integrate_batch(b)
    assert np.array_equal(_bits(C), _bits(rC))
    assert np.array_equal(ist, rist) and np.array_equal(ierr, rierr)


def test_ncell_zero_is_noop(pkg):
    s = _solver(pkg, "fma", 1)
    b = pkg.workloads.plain_small(4, seed=1)
    import ctypes
    C = np.array(b.C, order="F")
    C0 = C.copy()
    ierr = np.full(4, 7, np.int32)
    tt, tk = ctypes.c_double(), ctypes.c_double()
    p = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    z = np.zeros(64)
    s.lib.gc_gpu_integrate_batch(0, 0.0, 1200.0, p(C), p(b.RCONST), p(b.ATOL), p(b.RTOL),
                                 p(b.ICNTRL), p(b.RCNTRL), p(np.arange(1, 5, dtype=np.int32)),
                                 p(np.zeros(32, np.int32)), p(z), p(ierr), ctypes.byref(tt),
                                 ctypes.byref(tk))
    assert np.array_equal(C, C0) and (ierr == 7).all()


@pytest.mark.parametrize("mode", [0, 1, 3], ids=["plain", "persistent", "coop"])
def test_option_errors_match_oracle(pkg, orc, mode):
    """Rejected options (-2, -90), step limit (-6) and clamping, per cell."""
    b = _capped(pkg.workloads.plain_small(40, seed=8))
    b.ICNTRL[2, 0:4] = 2          # not Rodas3 -> -2
    b.ICNTRL[11, 4:8] = 1         # auto-reduce -> -90
    b.ICNTRL[3, 8:14] = 3         # at most 3 steps -> -6
    b.ICNTRL[15, 14:20] = 1       # clamp negatives on accept
    b.ICNTRL[1, 20:24] = 1        # scalar tolerances
    b.RCNTRL[2, 24:28] = 50.0     # warm start H
    b.RCNTRL[4, 28:30] = 3.0      # FacMax
    b.ICNTRL[0, 30:34] = 0        # non-autonomous (dFdT path)
    s = _solver(pkg, "nofma", mode)
    C, ist, rst, ierr, *_ = s.integrate_batch(b)
    rC, rist, rrst, rierr = orc.integrate_batch(b)
    assert (rierr[0:4] == -2).all() and (rierr[4:8] == -90).all() and (rierr[8:14] == -6).all()
    assert np.array_equal(ierr, rierr)
    assert np.array_equal(ist, rist)
    assert np.array_equal(_bits(rst), _bits(rrst))
    assert np.array_equal(_bits(C), _bits(rC))


def test_cost_order_is_the_stable_descending_sort(pkg):
    """The device cost order equals the model's stable counting sort
    (fullchem_mod.F90:906-960): descending key, ties in column order, no
    bound on the key -- bit for bit against numpy's stable argsort, and the
    same on every run."""
    import torch
    s = _solver(pkg, "fma", 1)
    rng = np.random.default_rng(2)
    for n in (1, 31, 2048, 2049, 100003, 262144):
        keys = rng.integers(0, 6000, n).astype(np.int32)
        keys[: n // 3] = rng.integers(0, 12, n // 3)       # many ties
        if n > 4:
            keys[:4] = [2 ** 31 - 1, 0, 200001, 4096]      # keys beyond any bin count
        kd = torch.from_numpy(keys).cuda()
        want = np.argsort(-keys.astype(np.int64), kind="stable")
        for _ in range(2):
            order = s.cost_order(kd).cpu().numpy()
            assert np.array_equal(order, want), n


def test_invalid_perm_fails_every_cell(pkg):
    """A Perm entry outside 1..nCell is rejected on the host before any
    device work: IERR = -100 for every cell, C untouched."""
    b = _capped(pkg.workloads.plain_small(16, seed=9))
    s = _solver(pkg, "fma", 1)
    perm = np.arange(1, 17, dtype=np.int32)
    perm[5] = 17
    C, ist, rst, ierr, *_ = s.integrate_batch(b, perm=perm)
    assert (ierr == -100).all()
    assert np.array_equal(_bits(C), _bits(np.asfortranarray(b.C)))
