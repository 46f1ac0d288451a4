"""The oracle pinned to reference code that does not pass through the
project's expression parser.

tests/golden/reference_pins.json.gz (written by tests/golden/make_pins.py
with its own minimal reader) holds other generated routines of the same
fullchem KPP mechanism:

* CalcStoichNum (gckpp_Function.F90:7271-12790): the stoichiometric matrix;
* the aggregate Fun (gckpp_Function.F90:47-2150): rates and Vdot as sums of
  coefficient * rate;
* Jac_SP_Vec / JacTR_SP_Vec (gckpp_Jacobian.F90:20903-22738): the sparse
  Jacobian-vector products;
* KppSolveTR (gckpp_LinearAlgebra.F90:2327-3701): the transposed solve.

The oracle's Fun (from Fun_SPLIT), Jac (from Jac_SP) and the adjoint's
transposed solve are checked against them: structurally where the two
renderings must agree exactly, numerically (to rounding) where they sum the
same terms in a different order.
"""
import gzip
import json
import os

import numpy as np
import pytest

from mechanism import codegen

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def pins():
    with gzip.open(os.path.join(GOLDEN, "reference_pins.json.gz"), "rt") as fh:
        return json.load(fh)


def _num(text):
    return float(codegen.literal(text))


def _state(mech, seed):
    rng = np.random.default_rng(seed)
    V = 10.0 ** rng.uniform(2, 13, mech["nvar"])
    F = 10.0 ** rng.uniform(15, 19, mech["nfix"])
    R = 10.0 ** rng.uniform(-20, -1, mech["nreact"])
    return V, F, R


def _rates(pins, V, F, R):
    """A(j) of the aggregate Fun, left to right as written."""
    A = np.empty(len(pins["rates"]))
    for j, r in enumerate(pins["rates"]):
        a = R[r["rct"]] if r["rct"] >= 0 else _num(r["lit"])
        if r["rct"] >= 0 and r["lit"] != "1":
            a = a * _num(r["lit"])
        for v in r["v"]:
            a = a * V[v]
        for f in r["f"]:
            a = a * F[f]
        A[j] = a
    return A


def _aggregate_fun(pins, V, F, R):
    """Vdot of the aggregate Fun and the sum of |terms| (the rounding scale)."""
    A = _rates(pins, V, F, R)
    out = np.zeros(len(pins["vdot"]))
    mag = np.zeros(len(pins["vdot"]))
    for i, terms in enumerate(pins["vdot"]):
        for j, c in terms:
            t = _num(c) * A[j]
            out[i] += t
            mag[i] += abs(t)
    return out, mag


def test_sources_recorded(pins):
    assert set(pins["source"]) == {"CalcStoichNum", "Fun", "Jac_SP_Vec", "JacTR_SP_Vec",
                                   "KppSolveTR"}


def test_stoichiometry_matches_calcstoichnum(mech, pins):
    """The stoichiometric matrix the adjoint uses is CalcStoichNum's."""
    ours = {(i, j): _num(v) for i, j, v in mech["stoich"]}
    ref = {(i, j): _num(v) for i, j, v in pins["stoich"]}
    assert ours == ref


def test_aggregate_fun_is_calcstoichnum(pins):
    """Two renderings in the reference agree: Vdot(i) = sum_j S(i,j) A(j)."""
    S = {}
    for i, j, v in pins["stoich"]:
        S.setdefault(i, {})[j] = _num(v)
    for i, terms in enumerate(pins["vdot"]):
        agg = {}
        for j, c in terms:
            agg[j] = agg.get(j, 0.0) + _num(c)
        assert agg == S.get(i, {}), i


def test_rates_match_fun_split(mech, pins):
    """Every rate of the parsed Fun_SPLIT has the aggregate Fun's factors."""
    def factors(e, acc):
        if e[0] == "*":
            factors(e[1], acc)
            factors(e[2], acc)
        else:
            acc.append(e)
        return acc

    assert len(mech["rates"]) == len(pins["rates"])
    for j, (e, r) in enumerate(zip(mech["rates"], pins["rates"])):
        fs = factors(e, [])
        rct = [f[1] for f in fs if f[0] == "k"]
        lit = [_num(f[1]) for f in fs if f[0] == "n"]
        assert rct == ([r["rct"]] if r["rct"] >= 0 else []), j
        assert sorted(f[1] for f in fs if f[0] == "v") == sorted(r["v"]), j
        assert sorted(f[1] for f in fs if f[0] == "f") == sorted(r["f"]), j
        assert np.prod(lit) == _num(r["lit"]), j


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_oracle_fun_matches_aggregate_fun(mech, orc, pins, seed):
    """Fun_SPLIT (P_VAR - D_VAR*V) and the aggregate Fun sum the same terms in
    different orders: equal to rounding of the largest term."""
    V, F, R = _state(mech, seed)
    agg, mag = _aggregate_fun(pins, V, F, R)
    got = orc.fun(V, F, R)
    assert (np.abs(got - agg) <= 1e-13 * mag + 1e-300).all()


def test_jac_sp_vec_pattern(mech, pins):
    """Every JVS(p)*UV(c) term of JUV(i) sits at (i, c) of the LU pattern, and
    JacTR_SP_Vec holds exactly the transposed terms."""
    irow, icol = mech["lu_irow"], mech["lu_icol"]
    jv = set()
    for i, terms in enumerate(pins["jac_sp_vec"]):
        for p, c in terms:
            assert (irow[p], icol[p]) == (i, c)
            jv.add(p)
    jt = set()
    for c, terms in enumerate(pins["jactr_sp_vec"]):
        for p, i in terms:
            assert (irow[p], icol[p]) == (i, c)
            jt.add(p)
    assert jv == jt


def test_jac_zero_outside_jac_sp_vec(mech, orc, pins):
    """The entries Jac_SP_Vec leaves out are the pattern's fill-in: Jac_SP
    sets them to zero at every state.  Inside, Jac_SP sets every entry
    except the diagonals of species that no reaction consumes (Jac_SP writes
    a literal 0 there; Jac_SP_Vec keeps every diagonal)."""
    inside = {p for terms in pins["jac_sp_vec"] for p, _ in terms}
    outside = np.array(sorted(set(range(mech["nnz"])) - inside))
    lit0 = {p for p, e in enumerate(mech["jvs"]) if e == ["n", "0"]}
    diag = set(mech["lu_diag"])
    assert set(outside) <= lit0
    assert (lit0 - set(outside)) <= diag
    live = np.array(sorted(inside - lit0))
    for seed in (0, 1):
        J = orc.jac(*_state(mech, seed))
        assert (J[outside] == 0.0).all()
        assert (J[live] != 0.0).all()


@pytest.mark.parametrize("seed", [3, 4])
def test_jacobian_matches_fd_of_aggregate_fun(mech, orc, pins, seed):
    """J u through the reference's Jac_SP_Vec pattern, with the oracle's Jac,
    against central differences of the aggregate Fun (not Fun_SPLIT): the
    Jacobian is pinned to an independent rendering of the right-hand side."""
    V, F, R = _state(mech, seed)
    J = orc.jac(V, F, R)
    u = np.random.default_rng(seed).standard_normal(mech["nvar"]) * V
    Ju = np.array([sum(J[p] * u[c] for p, c in terms) for terms in pins["jac_sp_vec"]])
    h = 1e-6
    fp, mp = _aggregate_fun(pins, V + h * u, F, R)
    fm, mm = _aggregate_fun(pins, V - h * u, F, R)
    fd = (fp - fm) / (2 * h)
    noise = 1e-13 * (mp + mm) / (2 * h)
    assert (np.abs(Ju - fd) <= 1e-6 * np.abs(Ju) + noise + 1e-300).all()


def test_transposed_solve_is_kppsolvetr(mech, pins):
    """The adjoint's transposed solve is KppSolveTR statement for statement."""
    assert codegen.solve_tr_stmts(mech) == pins["kppsolvetr"]


def test_transposed_solve_solves_the_transpose(mech, orc):
    """KppSolveTR's statements, interpreted here, solve (LU)^T x = b."""
    V, F, R = _state(mech, 5)
    G = -orc.jac(V, F, R)
    for d in mech["lu_diag"]:
        G[d] += 1.0 / 30.0
    LU, ier = orc.decomp(G)
    assert ier == 0
    n = mech["nvar"]
    b = np.random.default_rng(1).standard_normal(n)
    x = b.copy()
    for i, src, terms, d in codegen.solve_tr_stmts(mech):
        s = x[i]
        for p, j in terms:
            s = s - LU[p] * x[j]
        x[i] = s / LU[d] if d >= 0 else s
    A = np.zeros((n, n))
    A[mech["lu_irow"], mech["lu_icol"]] = G
    r = np.abs(A.T @ x - b).max()
    xd = np.linalg.solve(A.T, b)
    assert r <= max(10 * np.abs(A.T @ xd - b).max(), 1e-15 * np.abs(A).max() * np.abs(x).max() * n)


def test_libm_pow_changes_no_step_and_stays_within_tolerance(pkg, orc):
    """The reference's CPU build takes Err**(1/3) from the C library's pow
    (gckpp_BatchIntegrator.F90:667); the oracle and the kernels use the
    project's correctly rounded gc_pow.  On config-0 cells the two oracles
    take the same steps, and the final states differ far below the 1e-6
    parity tolerance (the last bits of about 5% of the cells move; on all
    4,096 cells the largest difference is 7e-11 relative)."""
    b = pkg.workloads.plain_small(1024, seed=0)
    C, ist, rst, ierr = orc.integrate_batch(b)
    C2, ist2, rst2, ierr2 = orc.integrate_batch(b, pow_="libm")
    nv = orc.load().sizes[0]
    assert np.array_equal(ierr, ierr2) and np.array_equal(ist, ist2)
    rel = np.abs(C[:nv] - C2[:nv]) / np.maximum(np.abs(C[:nv]), 1e-20)
    assert rel.max() <= 1e-8
    assert (C[:nv] != C2[:nv]).any(axis=0).sum() > 0     # the two pows do differ


def test_libm_pow_on_the_synthetic_mechanism(pkg, orc):
    """The same check on config 1's synthetic cells, which take ~200 internal
    steps each and so give a last-bit difference in Err**(1/3) many more
    chances to change a step sequence: none does (identical ISTAT), and the
    final states differ by at most ~1e-12 relative (73 of 512 cells move in
    the last bits)."""
    b = pkg.workloads.synthetic_stiff(256, seed=7)
    b.ICNTRL[3, :] = 20000
    C, ist, rst, ierr = orc.integrate_batch(b, mech="synth120")
    C2, ist2, rst2, ierr2 = orc.integrate_batch(b, mech="synth120", pow_="libm")
    nv = 120
    assert (ierr == 1).all() and np.array_equal(ierr, ierr2) and np.array_equal(ist, ist2)
    rel = np.abs(C[:nv] - C2[:nv]) / np.maximum(np.abs(C[:nv]), 1e-20)
    assert rel.max() <= 1e-10
