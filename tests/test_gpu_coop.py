"""The cooperative kernel (one thread block per cell, the cell state in
shared memory) against the oracle, through the C-ABI.

Its Fun, Jac, factorisation and solves walk generated tables in the
reference's per-entry operation order, so the --fmad=false library must
match the oracle bit for bit; the production library must stay within 1e-6
relative (denominator floored at 1e-2) with no failure.  Both block sizes
are covered, on the synthetic stiff mechanism (the kernel's target) and on
fullchem.  The option paths, Perm, the retry protocol and the 4x5 grid
sample are covered for this kernel by the parametrised tests of
test_gpu_parity.py, test_gpu_retry.py and test_gpu_config_parity.py.
"""
import numpy as np
import pytest

pytestmark = [pytest.mark.gpu, pytest.mark.timeout(600)]


def _bits(a):
    return np.ascontiguousarray(a).view(np.uint64 if a.dtype == np.float64 else np.uint32)


@pytest.fixture(scope="module")
def synth(pkg):
    b = pkg.workloads.synthetic_stiff(300, seed=5)
    b.ICNTRL[3, :] = 20000
    return b


@pytest.fixture(scope="module")
def synth_ref(synth):
    import oracle
    r = oracle.integrate_batch(synth, mech="synth120")
    assert (r[3] == 1).all()
    return r


@pytest.mark.parametrize("threads", [128, 256])
def test_coop_synthetic_bitexact_nofma(pkg, synth, synth_ref, threads):
    s = pkg.solver("synth120", "nofma")
    s.set_row_scratch(False)
    s.set_launch(pkg.COOP, threads)
    C, ist, rst, ierr, *_ = s.integrate_batch(synth)
    s.set_launch(pkg.PERSISTENT)
    rC, rist, rrst, rierr = synth_ref
    assert np.array_equal(ierr, rierr) and np.array_equal(ist, rist)
    assert np.array_equal(_bits(C), _bits(rC))
    assert np.array_equal(_bits(rst), _bits(rrst))


@pytest.mark.parametrize("threads", [128, 256])
def test_coop_synthetic_fma_tolerance(pkg, synth, synth_ref, threads):
    s = pkg.solver("synth120", "fma")
    s.set_row_scratch(False)
    s.set_launch(pkg.COOP, threads)
    C, ist, rst, ierr, *_ = s.integrate_batch(synth)
    s.set_launch(pkg.PERSISTENT)
    rC, rist, rrst, rierr = synth_ref
    assert (ierr == 1).all()
    n = s.nvar
    rel = np.abs(C[:n] - rC[:n]) / np.maximum(np.abs(rC[:n]), 1e-2)
    assert rel.max() <= 1e-6, rel.max()


def test_coop_synthetic_matches_persistent_fma_build(pkg, synth):
    """Same arithmetic as the indexed factorisation's FMA build (reciprocal
    pivots, same per-entry order): the two kernels agree to rounding."""
    s = pkg.solver("synth120", "fma")
    s.set_row_scratch(False)
    s.set_launch(pkg.COOP, 128)
    C1, ist1, _, ierr1, *_ = s.integrate_batch(synth)
    s.set_launch(pkg.PERSISTENT, 128)
    C2, ist2, _, ierr2, *_ = s.integrate_batch(synth)
    assert (ierr1 == 1).all() and (ierr2 == 1).all()
    n = s.nvar
    rel = np.abs(C1[:n] - C2[:n]) / np.maximum(np.abs(C2[:n]), 1e-2)
    assert rel.max() <= 1e-6, rel.max()


@pytest.mark.parametrize("threads", [128, 256])
def test_coop_fullchem_bitexact_nofma(pkg, orc, threads):
    b = pkg.workloads.plain_small(200, seed=13)
    b.ICNTRL[3, :] = 5000
    rC, rist, rrst, rierr = orc.integrate_batch(b)
    s = pkg.solver("fullchem", "nofma")
    s.set_launch(pkg.COOP, threads)
    C, ist, rst, ierr, *_ = s.integrate_batch(b)
    s.set_launch(pkg.PERSISTENT)
    assert np.array_equal(ierr, rierr) and np.array_equal(ist, rist)
    assert np.array_equal(_bits(C), _bits(rC))
    assert np.array_equal(_bits(rst), _bits(rrst))


def test_coop_needs_no_workspace_and_rejects_other_block_sizes(pkg):
    s = pkg.solver("synth120", "fma")
    s.set_launch(pkg.COOP, 128)
    assert s.lib.gcchem_b200_workspace_slots(100000) == 0
    with pytest.raises(ValueError):
        s.set_launch(pkg.COOP, 192)
    s.set_launch(pkg.PERSISTENT)
