"""The cooperative kernel's tables, checked on the CPU before any GPU run.

The cooperative kernel (one thread block per cell) evaluates Fun, Jac, the
factorisation and the solves by walking tables (mechanism/coop.py) instead
of straight-line statements.  These tests walk the same tables in the same
order with Python floats (IEEE double, no FMA contraction) and require the
oracle's results bit for bit: Fun_SPLIT, Jac_SP, ros_PrepareMatrix +
KppDecomp in the right-looking order, and KppSolve (forward by columns,
backward by levels).
"""
import numpy as np
import pytest

from mechanism import codegen, coop

MECHS = ("synth120", "fullchem")


@pytest.fixture(scope="module", params=MECHS)
def case(request):
    import oracle
    m = codegen.load(request.param)
    oracle.load(request.param)
    return request.param, m, coop.compile_tables(m)


def _fac(code, V, F, K, S, consts):
    kind, idx = code >> 13, code & 0x1FFF
    return (V, F, K, S, consts)[kind][idx]


def _eval(t, sid, V, F, K, S):
    s = 0.0
    fac, ops, consts = t["term_fac"], t["term_op"], t["consts"]
    for q in range(t["sum_off"][sid], t["sum_off"][sid + 1]):
        codes = fac[4 * q:4 * q + 4]
        v = _fac(codes[0], V, F, K, S, consts)
        for c in codes[1:]:
            if c != coop.NONE:
                v = v * _fac(c, V, F, K, S, consts)
        op = ops[q]
        s = v if op == 0 else (-v if op == 1 else (s + v if op == 2 else s - v))
    return s


def _fun(m, t, V, F, K):
    S = [_eval(t, t["sid_rate"] + j, V, F, K, None) for j in range(m["nreact"])]
    out = []
    for i in range(m["nvar"]):
        p = _eval(t, t["sid_prod"] + i, V, F, K, S)
        d = _eval(t, t["sid_dest"] + i, V, F, K, S)
        out.append(p - (d * V[i]))
    return np.array(out)


def _jac(m, t, V, F, K):
    S = [_eval(t, t["sid_b"] + b, V, F, K, None) for b in range(m["nb"])]
    return np.array([_eval(t, t["sid_jvs"] + k, V, F, K, S) for k in range(m["nnz"])])


def _prep_decomp(m, t, J, ghinv):
    """G = -J (+ ghinv on the diagonal), then the right-looking steps."""
    G = [-x for x in J]
    for k, row in enumerate(t["kdiag"]):
        if row >= 0:
            G[k] = G[k] + ghinv
    diag = m["lu_diag"]
    for j in range(m["nvar"]):
        dj = G[diag[j]]
        for q in range(t["mul_off"][j], t["mul_off"][j + 1]):
            p = t["mul_pos"][q]
            a = -(G[p] / dj)
            G[p] = -a
        for q in range(t["upd_off"][j], t["upd_off"][j + 1]):
            tt, p, u = t["upd"][q]
            G[tt] = G[tt] + (-G[p]) * G[u]
    return np.array(G)


def _solve(m, t, G, X):
    X = list(X)
    crow, diag, icol = m["lu_crow"], m["lu_diag"], m["lu_icol"]
    for j in range(m["nvar"]):
        xj = X[j]
        for q in range(t["fwd_off"][j], t["fwd_off"][j + 1]):
            i, p = t["fwd"][q]
            X[i] = X[i] - G[p] * xj
    for lev in range(t["nlev"]):
        for q in range(t["bwd_off"][lev], t["bwd_off"][lev + 1]):
            i = t["bwd_rows"][q]
            s = X[i]
            for jj in range(diag[i] + 1, crow[i + 1]):
                s = s - G[jj] * X[icol[jj]]
            X[i] = s / G[diag[i]]
    return np.array(X)


def _solve_columns(m, t, G, X):
    """The FMA build's sweeps: forward by columns, backward by columns
    (x(i) = acc(i)/U(i,i), then every row r < i subtracts U(r,i)*x(i))."""
    X = list(X)
    diag = m["lu_diag"]
    n = m["nvar"]
    for j in range(n):
        xj = X[j]
        for q in range(t["fwd_off"][j], t["fwd_off"][j + 1]):
            i, p = t["fwd"][q]
            X[i] = X[i] - G[p] * xj
    for s in range(n):
        i = n - 1 - s
        X[i] = X[i] / G[diag[i]]
        for q in range(t["bwc_off"][s], t["bwc_off"][s + 1]):
            r, p = t["bwc"][q]
            assert r < i
            X[r] = X[r] - G[p] * X[i]
    return np.array(X)


def _state(m, seed):
    rng = np.random.default_rng(seed)
    V = 10.0 ** rng.uniform(-6, 0, m["nvar"]) * 1e6
    F = 10.0 ** rng.uniform(15, 19, max(m["nfix"], 1))
    K = 10.0 ** rng.uniform(-18, 2, m["nreact"])
    return V, F, K


def _bits(a):
    return np.asarray(a, dtype=np.float64).view(np.uint64)


def test_tables_exist_and_are_in_range(case):
    name, m, t = case
    assert t is not None, name
    nnz, n = m["nnz"], m["nvar"]
    assert len(t["sum_off"]) == t["nsum"] + 1
    assert t["nsum"] == m["nreact"] + 2 * n + m["nb"] + nnz
    for tt, p, u in t["upd"]:
        assert 0 <= tt < nnz and 0 <= p < nnz and 0 <= u < nnz
    assert all(0 <= p < nnz for p in t["mul_pos"])
    assert all(0 <= i < n and 0 <= p < nnz for i, p in t["fwd"])
    assert sorted(t["bwd_rows"]) == list(range(n))
    # every factor index lies inside the array its kind names
    sizes = (n, max(m["nfix"], 1), m["nreact"], max(m["nreact"], m["nb"]), len(t["consts"]))
    for c in t["term_fac"]:
        if c != coop.NONE:
            assert (c & 0x1FFF) < sizes[c >> 13]
    # one update per entry per step, and steps apply pivots in increasing order
    for j in range(n):
        tg = [u[0] for u in t["upd"][t["upd_off"][j]:t["upd_off"][j + 1]]]
        assert len(tg) == len(set(tg))


def test_fun_and_jac_match_oracle(case):
    import oracle
    name, m, t = case
    V, F, K = _state(m, 3)
    ref = oracle.fun(V, F[:m["nfix"]] if m["nfix"] else F, K, mech=name)
    got = _fun(m, t, list(V), list(F), list(K))
    assert np.array_equal(_bits(got), _bits(ref))
    refj = oracle.jac(V, F[:m["nfix"]] if m["nfix"] else F, K, mech=name)
    gotj = _jac(m, t, list(V), list(F), list(K))
    assert np.array_equal(_bits(gotj), _bits(refj))


def test_right_looking_factorisation_and_solves_match_oracle(case):
    import oracle
    name, m, t = case
    V, F, K = _state(m, 4)
    J = oracle.jac(V, F[:m["nfix"]] if m["nfix"] else F, K, mech=name)
    ghinv = 1.0 / (30.0 * 0.5)
    G0 = -J
    G0[np.array(m["lu_diag"])] += ghinv
    ref, ier = oracle.decomp(G0, mech=name)
    assert ier == 0
    got = _prep_decomp(m, t, list(J), ghinv)
    assert np.array_equal(_bits(got), _bits(ref))
    rng = np.random.default_rng(5)
    b = rng.standard_normal(m["nvar"]) * 1e5
    refx = oracle.solve(ref, b, mech=name)
    gotx = _solve(m, t, list(got), list(b))
    assert np.array_equal(_bits(gotx), _bits(refx))
    # the FMA build's column-wise backward sweep: the same terms, each row's
    # in the reverse order, so the solution agrees to rounding
    colx = _solve_columns(m, t, list(got), list(b))
    assert np.abs(colx - refx).max() <= 1e-9 * np.abs(refx).max()
    U = [(r, p) for r, p in t["bwc"]]
    assert len(U) == sum(m["lu_crow"][i + 1] - m["lu_diag"][i] - 1 for i in range(m["nvar"]))


def test_coop_inc_emits_macros(case):
    name, m, t = case
    txt = coop.coop_inc(m)
    assert "#define MECH_COOP 1" in txt
    assert f"#define COOP_NUPD {len(t['upd'])}" in txt


def test_unsupported_shapes_get_no_tables():
    """A rate that is not a product chain (here a quotient) or a product of
    more than four factors leaves the mechanism without cooperative tables:
    the generated coop.inc then defines MECH_COOP 0 and the library reports
    the kernel unavailable."""
    m = codegen.load("synth120")
    bad = dict(m)
    bad["rates"] = list(m["rates"])
    bad["rates"][0] = ["/", ["k", 0], ["v", 1]]
    assert coop.compile_tables(bad) is None
    assert "#define MECH_COOP 0" in coop.coop_inc(bad)
    long_prod = ["k", 0]
    for v in range(4):
        long_prod = ["*", long_prod, ["v", v]]
    bad["rates"][0] = long_prod
    assert coop.compile_tables(bad) is None


def test_column_backward_tables_cover_every_u_entry_once():
    m = codegen.load("synth120")
    t = coop.compile_tables(m)
    n, crow, diag = m["nvar"], m["lu_crow"], m["lu_diag"]
    want = {jj for i in range(n) for jj in range(diag[i] + 1, crow[i + 1])}
    got = [q for _, q in t["bwc"]]
    assert len(got) == len(set(got)) and set(got) == want
    # step s handles column n-1-s: every entry's column is that column
    icol = m["lu_icol"]
    for s in range(n):
        for r, q in t["bwc"][t["bwc_off"][s]:t["bwc_off"][s + 1]]:
            assert icol[q] == n - 1 - s and r < n - 1 - s
