"""CPU checks of the mechanism translator, the generated code and the oracle.

The oracle's faithfulness to the reference rests on the translator, so it is
checked three ways here: the parser's association order on hand-written
Fortran, statement counts against the reference's generated files
(gckpp_Function.F90 / gckpp_Jacobian.F90 / gckpp_LinearAlgebra.F90), and an
independent Python interpreter of the parsed expression trees that must
agree bit for bit with the compiled oracle.
"""
import ctypes

import numpy as np
import pytest

from mechanism import fortran_ir as fir
from mechanism import codegen


# ---------------------------------------------------------------- parser
def test_parse_left_association():
    assert fir.parse_expr("RCT(1)*V(2)*V(3)") == \
        ["*", ["*", ["k", 0], ["v", 1]], ["v", 2]]
    # leading unary minus binds to the first multiplication chain only
    assert fir.parse_expr("-B(1)-B(2)+0.5*B(3)") == \
        ["+", ["-", ["neg", ["b", 0]], ["b", 1]], ["*", ["n", "0.5"], ["b", 2]]]
    assert fir.parse_expr("-2*B(4)") == ["neg", ["*", ["n", "2"], ["b", 3]]]
    assert fir.parse_expr("(X(1)-JVS(2)*X(3))/(JVS(4))") == \
        ["/", ["-", ["x", 0], ["*", ["j", 1], ["x", 2]]], ["j", 3]]
    assert fir.parse_expr("RCT(196)*2*V(351)") == \
        ["*", ["*", ["k", 195], ["n", "2"]], ["v", 350]]


def test_literals_are_doubles():
    assert codegen.literal("2") == "2.0"
    assert codegen.literal("4.51e-12") == "4.51e-12"
    assert codegen.literal("1.0d-3") == "1.0e-3"
    assert codegen.literal("7e5") == "7.0e5"


def test_statement_joining_and_guards():
    lines = ["IF (DO_JVS(7)) &", "! JVS(7) = Jac_FULL(4,55)",
             "  JVS(7) = 2*B(1579)+B(3)&", "     &-0.25*B(9)"]
    (lhs, idx, ast, com), = list(fir.assignments(lines))
    assert (lhs, idx) == ("JVS", 6)
    assert fir.jac_full_position(com) == (6, 3, 54)
    assert ast[0] == "-"


# ------------------------------------------------------- extracted tables
def test_fullchem_counts(mech):
    # gckpp_Parameters values quoted by the reference (mgpu_test.F90:11,
    # gckpp_Jacobian.F90:31): NVAR=353, NFIX=3, NREACT=1058, LU_NONZERO=5683
    assert (mech["nvar"], mech["nfix"], mech["nreact"], mech["nnz"]) == (353, 3, 1058, 5683)
    assert len(mech["rates"]) == 1058
    assert len(mech["prod"]) == 353 and len(mech["dest"]) == 353
    assert mech["nb"] == 1817 and len(mech["jac_b"]) == 1805
    assert len(mech["jvs"]) == 5683


def test_lu_pattern(mech):
    n = mech["nvar"]
    crow, diag = mech["lu_crow"], mech["lu_diag"]
    assert crow[0] == 0 and crow[n] == mech["nnz"]
    assert all(crow[i] <= diag[i] < crow[i + 1] for i in range(n))
    # divisions and updates of one factorisation
    ndiv = sum(diag[k] - crow[k] for k in range(n))
    assert ndiv == 2773
    assert codegen.flop_counts(mech)["lu"] == 44353


def test_solve_order_matches_reference(mech):
    """The parsed reference KppSolve (505 statements) is exactly the
    pattern-driven forward/backward sweep the code generator emits."""
    assert mech["solve"] == codegen.solve_stmts(mech)
    assert len(mech["solve"]) == 505


# -------------------------------------------- independent interpreter
def _ev(node, env):
    tag = node[0]
    if tag == "n":
        return float(codegen.literal(node[1]))
    if tag in env:
        return env[tag][node[1]]
    if tag == "neg":
        return -_ev(node[1], env)
    a = _ev(node[1], env)
    b = _ev(node[2], env)
    if tag == "+":
        return a + b
    if tag == "-":
        return a - b
    if tag == "*":
        return a * b
    return a / b


def _state(mech, seed):
    rng = np.random.default_rng(seed)
    V = 10.0 ** rng.uniform(2, 13, mech["nvar"])
    F = 10.0 ** rng.uniform(15, 19, mech["nfix"])
    R = 10.0 ** rng.uniform(-20, -1, mech["nreact"])
    return V, F, R


def _interp_fun(mech, V, F, R):
    env = {"v": list(V), "f": list(F), "k": list(R)}
    env["a"] = [_ev(e, env) for e in mech["rates"]]
    P = [_ev(e, env) for e in mech["prod"]]
    D = [_ev(e, env) for e in mech["dest"]]
    return np.array([P[i] - D[i] * V[i] for i in range(mech["nvar"])])


def _interp_jac(mech, V, F, R):
    env = {"v": list(V), "f": list(F), "k": list(R)}
    B = [0.0] * mech["nb"]
    for k, e in mech["jac_b"]:
        B[k] = _ev(e, env)
    env["b"] = B
    return np.array([_ev(e, env) for e in mech["jvs"]])


@pytest.mark.parametrize("seed", [0, 1])
def test_oracle_fun_matches_interpreter(mech, orc, seed):
    V, F, R = _state(mech, seed)
    ref = _interp_fun(mech, V, F, R)
    got = orc.fun(V, F, R)
    assert np.array_equal(got.view(np.uint64), ref.view(np.uint64))


@pytest.mark.parametrize("seed", [0, 1])
def test_oracle_jac_matches_interpreter(mech, orc, seed):
    V, F, R = _state(mech, seed)
    ref = _interp_jac(mech, V, F, R)
    got = orc.jac(V, F, R)
    assert np.array_equal(got.view(np.uint64), ref.view(np.uint64))


def test_jacobian_is_derivative_of_fun(mech, orc):
    """Jac_SP against central differences of Fun_SPLIT on a few columns."""
    V, F, R = _state(mech, 2)
    J = orc.jac(V, F, R)
    irow, icol = np.array(mech["lu_irow"]), np.array(mech["lu_icol"])
    for c in (0, 100, 344, 352):
        h = 1e-6 * V[c]
        vp, vm = V.copy(), V.copy()
        vp[c] += h
        vm[c] -= h
        fp, fm = orc.fun(vp, F, R), orc.fun(vm, F, R)
        fd = (fp - fm) / (2 * h)
        col = np.zeros(mech["nvar"])
        sel = icol == c
        col[irow[sel]] = J[sel]
        # rounding noise of the difference quotient, row by row
        noise = 1e-12 * (np.abs(fp) + np.abs(fm)) / (2 * h)
        assert (np.abs(col - fd) <= 1e-5 * np.abs(col) + noise + 1e-300).all()


@pytest.mark.parametrize("seed,h", [(0, 1e-3), (1, 10.0), (2, 1200.0)])
def test_fused_lu_bitexact(mech, orc, seed, h):
    """Generated register-blocked factorisation == indexed KppDecomp."""
    V, F, R = _state(mech, seed)
    J0 = orc.jac(V, F, R)
    ghinv = 1.0 / (h * 0.5)
    G = -J0
    for d in mech["lu_diag"]:
        G[d] = G[d] + ghinv
    ref, ier = orc.decomp(G)
    got = np.zeros_like(J0)
    ier2 = orc.gencheck().gencheck_prep_decomp(
        J0.ctypes.data_as(ctypes.c_void_p), got.ctypes.data_as(ctypes.c_void_p), ghinv)
    assert ier == ier2 == 0
    assert np.array_equal(got.view(np.uint64), ref.view(np.uint64))


@pytest.mark.parametrize("seed,h", [(0, 1e-3), (1, 10.0), (2, 1200.0), (3, 60.0)])
def test_fused_lu_reciprocal_form(mech, orc, seed, h):
    """The FMA library's multiplier form (one reciprocal 1/U(j,j) per row, no
    divide per multiplier) solves as well as the reference's divides.

    On these deliberately ill-conditioned random states single factor
    entries can move by up to ~1e-3 relative through cancellation, as they
    do under FMA contraction, so the check is the backward error of a solve
    with each factorisation, plus the stored reciprocals themselves."""
    V, F, R = _state(mech, seed)
    J0 = orc.jac(V, F, R)
    ghinv = 1.0 / (h * 0.5)
    G = -J0
    for d in mech["lu_diag"]:
        G[d] = G[d] + ghinv
    ref, ier = orc.decomp(G)
    got = np.zeros_like(J0)
    W = np.zeros(mech["nvar"])
    ier2 = orc.gencheck().gencheck_prep_decomp_recip(
        J0.ctypes.data_as(ctypes.c_void_p), got.ctypes.data_as(ctypes.c_void_p),
        W.ctypes.data_as(ctypes.c_void_p), ghinv)
    assert ier == ier2 == 0
    diag = np.array(mech["lu_diag"])
    assert np.abs(W * got[diag] - 1.0).max() <= 4 * np.finfo(float).eps
    A = np.zeros((mech["nvar"], mech["nvar"]))
    A[mech["lu_irow"], mech["lu_icol"]] = G
    b = np.random.default_rng(seed).standard_normal(mech["nvar"])
    r_ref = np.abs(A @ orc.solve(ref, b) - b).max()
    r_got = np.abs(A @ orc.solve(got, b) - b).max()
    assert r_got <= 10 * r_ref + 1e-300


def test_lu_solve_matches_dense(mech, orc):
    V, F, R = _state(mech, 4)
    J0 = orc.jac(V, F, R)
    ghinv = 1.0 / (60.0 * 0.5)
    G = -J0
    for d in mech["lu_diag"]:
        G[d] += ghinv
    A = np.zeros((mech["nvar"], mech["nvar"]))
    A[mech["lu_irow"], mech["lu_icol"]] = G
    LU, ier = orc.decomp(G)
    assert ier == 0
    b = np.random.default_rng(0).standard_normal(mech["nvar"])
    x = orc.solve(LU, b)
    # backward error: the system is badly conditioned (random stiff rates),
    # so compare residuals with LAPACK's rather than solutions
    xd = np.linalg.solve(A, b)
    scale = np.abs(A).max() * np.abs(x).max() * A.shape[0]
    assert np.abs(A @ x - b).max() <= max(10 * np.abs(A @ xd - b).max(), 1e-15 * scale)


def test_singular_diagonal_detected(mech, orc):
    """KppDecomp reports the first row whose diagonal is below TINY."""
    V, F, R = _state(mech, 5)
    G = -orc.jac(V, F, R)
    ghinv = 1.0
    for d in mech["lu_diag"]:
        G[d] += ghinv
    k = 17
    G[mech["lu_diag"][k]] = 0.0
    _, ier = orc.decomp(G)
    assert ier == k + 1
