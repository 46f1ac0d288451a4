"""The seeded synthetic stiff mechanism (120 species, 360 reactions)."""
import numpy as np
import pytest

from mechanism import codegen, synthetic

from test_generated import _interp_fun, _interp_jac


@pytest.fixture(scope="module")
def smech():
    return codegen.load("synth120")


def test_committed_tables_match_generator(smech):
    fresh = codegen.finalize(synthetic.generate())
    for key in ("nvar", "nreact", "nnz", "lu_irow", "lu_icol", "rates", "prod", "dest",
                "jac_b", "jvs"):
        assert fresh[key] == smech[key], key


def test_shape_and_pattern(smech):
    assert (smech["nvar"], smech["nfix"], smech["nreact"]) == (120, 0, 360)
    for e in smech["rates"]:          # 1-2 reactants
        assert str(e).count("'v'") in (1, 2)
    assert not codegen.fused_lu(smech)


def _state(m, seed):
    rng = np.random.default_rng(seed)
    V = 10.0 ** rng.uniform(-6, 0, m["nvar"])
    R = 10.0 ** rng.uniform(-20, 4, m["nreact"])
    return V, np.zeros(1), R


def test_oracle_matches_interpreter(smech):
    import oracle
    V, F, R = _state(smech, 0)
    ref = _interp_fun(smech, V, F, R)
    assert np.array_equal(oracle.fun(V, F, R, mech="synth120").view(np.uint64), ref.view(np.uint64))
    refj = _interp_jac(smech, V, F, R)
    assert np.array_equal(oracle.jac(V, F, R, mech="synth120").view(np.uint64), refj.view(np.uint64))


def test_jacobian_is_derivative_of_fun(smech):
    import oracle
    V, F, R = _state(smech, 1)
    J = oracle.jac(V, F, R, mech="synth120")
    irow, icol = np.array(smech["lu_irow"]), np.array(smech["lu_icol"])
    for c in (0, 57, 119):
        h = 1e-7 * V[c]
        vp, vm = V.copy(), V.copy()
        vp[c] += h
        vm[c] -= h
        fp, fm = oracle.fun(vp, F, R, mech="synth120"), oracle.fun(vm, F, R, mech="synth120")
        fd = (fp - fm) / (2 * h)
        col = np.zeros(smech["nvar"])
        sel = icol == c
        col[irow[sel]] = J[sel]
        noise = 1e-12 * (np.abs(fp) + np.abs(fm)) / (2 * h)
        assert (np.abs(col - fd) <= 1e-5 * np.abs(col) + noise + 1e-300).all()


@pytest.mark.gpu
@pytest.mark.timeout(300)
@pytest.mark.parametrize("scratch", ["global", "shared"])
@pytest.mark.parametrize("mode", [0, 1], ids=["plain", "persistent"])
def test_gpu_bitexact_synthetic(pkg, mode, scratch):
    """Both kernels, with the indexed factorisation's row scratch in the
    workspace or in shared memory, bit for bit against the oracle."""
    import oracle
    b = pkg.workloads.synthetic_stiff(300, seed=5)
    b.ICNTRL[3, :] = 20000
    rC, rist, rrst, rierr = oracle.integrate_batch(b, mech="synth120")
    assert (rierr == 1).all()
    s = pkg.solver("synth120", "nofma")
    s.set_row_scratch(False)
    s.set_launch(mode, 224 if scratch == "shared" else 128)
    s.set_row_scratch(scratch == "shared")
    C, ist, rst, ierr, *_ = s.integrate_batch(b)
    s.set_row_scratch(False)
    s.set_launch(pkg.PERSISTENT)
    assert np.array_equal(ierr, rierr) and np.array_equal(ist, rist)
    assert np.array_equal(C.view(np.uint64), rC.view(np.uint64))
    assert np.array_equal(rst.view(np.uint64), rrst.view(np.uint64))


@pytest.mark.gpu
@pytest.mark.timeout(300)
@pytest.mark.parametrize("mode", [0, 1], ids=["plain", "persistent"])
def test_gpu_fma_synthetic_within_tolerance(pkg, mode):
    """The production build (FMA contraction, reciprocal pivots in the
    indexed factorisation) keeps every variable species within 1e-6 relative
    of the oracle (denominator floored at 1e-2), with the same step counts on
    these cells and no failure."""
    import oracle
    b = pkg.workloads.synthetic_stiff(300, seed=5)
    b.ICNTRL[3, :] = 20000
    rC, rist, rrst, rierr = oracle.integrate_batch(b, mech="synth120")
    s = pkg.solver("synth120", "fma")
    s.set_row_scratch(False)
    s.set_launch(mode, 128)
    C, ist, rst, ierr, *_ = s.integrate_batch(b)
    s.set_launch(pkg.PERSISTENT)
    assert (ierr == 1).all() and (rierr == 1).all()
    n = s.nvar
    rel = np.abs(C[:n] - rC[:n]) / np.maximum(np.abs(rC[:n]), 1e-2)
    assert rel.max() <= 1e-6, rel.max()
