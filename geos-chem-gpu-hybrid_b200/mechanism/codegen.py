"""Emit C++ / CUDA statement lists from a mechanism IR.

One IR (see ``fortran_ir``) drives every consumer: the CPU oracle (g++),
the plain CUDA kernel and the batched CUDA kernel.  Every expression is
emitted fully parenthesised in the Fortran association order, so the C
compiler cannot re-associate anything; with FMA contraction disabled
(``-ffp-contract=off`` / ``--fmad=false``) the emitted code rounds exactly
like the reference's gfortran build.

Array accesses go through accessor macros (``V_(i)``, ``RCT_(j)``,
``JVS_(k)`` ...) so the same text compiles against plain per-cell arrays
(oracle) and against the warp-tiled interleaved workspace (CUDA).

Generated files (written by ``generate`` into one directory per mechanism,
selected by the include path of the consumer):

``mech.h``      sizes (MECH_NVAR ...) and the LU sparsity tables
                (MECH_LU_CROW/LU_DIAG/LU_ICOL/LU_IROW, 0-based)
``fun.inc``     Fun_SPLIT body: scalar rates A_(j) at first use, VDOT_(i)
``jac.inc``     Jac_SP body: scalar partials B_(k) at first use, JVS_(k)
``solve.inc``   KppSolve body (forward L, backward U with divide), long rows
                in pieces
``lu_fused.inc`` straight-line KppDecomp (the operation order of the indexed
                loop of gckpp_LinearAlgebra.F90:46-84) fused with the
                -Jac0 + ghinv preparation, rows held in registers in column
                blocks; generated only for factorisations of at most
                FUSED_LU_MAX_FLOPS (mech.h: MECH_FUSED_LU)
"""
from __future__ import annotations

import json
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))

_ACC = {"v": "V_", "f": "F_", "k": "RCT_", "a": "A_", "b": "B_", "x": "X_",
        "j": "JVS_"}


def load(name: str) -> dict:
    path = name if name.endswith(".json") else os.path.join(HERE, f"{name}.json")
    with open(path) as fh:
        mech = json.load(fh)
    return finalize(mech)


def finalize(mech: dict) -> dict:
    """Derive LU_CROW/LU_DIAG from LU_IROW/LU_ICOL and check the pattern."""
    n, nnz = mech["nvar"], mech["nnz"]
    irow, icol = mech["lu_irow"], mech["lu_icol"]
    if irow != sorted(irow):
        raise ValueError("LU pattern is not stored row by row")
    crow = [0] * (n + 1)
    for r in irow:
        crow[r + 1] += 1
    for i in range(n):
        crow[i + 1] += crow[i]
    diag = [-1] * n
    where = {}
    for k in range(nnz):
        where[(irow[k], icol[k])] = k
        if irow[k] == icol[k]:
            diag[irow[k]] = k
    if min(diag) < 0:
        raise ValueError("missing diagonal entry")
    for i in range(n):
        if icol[crow[i]:crow[i + 1]] != sorted(icol[crow[i]:crow[i + 1]]):
            raise ValueError(f"row {i} columns not sorted")
    for k in range(n):  # pattern must already contain the LU fill-in
        for kk in range(crow[k], diag[k]):
            j = icol[kk]
            for jj in range(diag[j] + 1, crow[j + 1]):
                if (k, icol[jj]) not in where:
                    raise ValueError(f"fill-in ({k},{icol[jj]}) missing")
    mech["lu_crow"] = crow
    mech["lu_diag"] = diag
    mech["lu_where"] = where
    return mech


def literal(text: str) -> str:
    t = text.lower().replace("d", "e")
    if re.fullmatch(r"\d+", t):
        return t + ".0"
    if t.startswith("."):
        t = "0" + t
    if re.fullmatch(r"\d+e[-+]?\d+", t):
        m, e = t.split("e")
        t = m + ".0e" + e
    return t


def cexpr(node) -> str:
    tag = node[0]
    if tag == "n":
        return literal(node[1])
    if tag in _ACC:
        return f"{_ACC[tag]}({node[1]})"
    if tag == "neg":
        return f"(-{cexpr(node[1])})"
    if tag in "+-*/":
        return f"({cexpr(node[1])}{tag}{cexpr(node[2])})"
    raise ValueError(f"bad node {node}")


def _strip(s: str) -> str:
    # drop one redundant outer pair of parentheses for readability
    if s.startswith("(") and s.endswith(")"):
        depth = 0
        for i, ch in enumerate(s):
            depth += ch == "("
            depth -= ch == ")"
            if depth == 0 and i != len(s) - 1:
                return s
        return s[1:-1]
    return s


FENCE_EVERY = 24


def _fenced(lines, every=FENCE_EVERY):
    """Insert GC_FENCE() every ``every`` statements.  In CUDA builds the fence
    is a compiler-only memory barrier that bounds how long a loaded value is
    carried in registers (otherwise the whole state vector stays live and
    spills); the oracle defines it as nothing.  Fences never reorder or
    change an arithmetic operation."""
    out = []
    for i, ln in enumerate(lines):
        if i and i % every == 0:
            out.append("GC_FENCE();")
        out.append(ln)
    return out


def _refs(node, tag: str, acc=None) -> list:
    """Indices of the ``tag`` leaves of an expression, in reading order."""
    acc = [] if acc is None else acc
    if isinstance(node, list):
        if node[0] == tag:
            acc.append(node[1])
        elif node[0] not in _ACC and node[0] != "n":
            for x in node[1:]:
                _refs(x, tag, acc)
    return acc


SUM_CHUNK = 8


def _chain(node) -> list:
    """A left-associated chain ``((t0 op1 t1) op2 t2) ...`` of binary + and -
    as [(None, t0), (op1, t1), ...]; any other node is a chain of one."""
    terms = []
    while isinstance(node, list) and node[0] in ("+", "-"):
        terms.append((node[0], node[2]))
        node = node[1]
    terms.append((None, node))
    return terms[::-1]


def _sum_stmts(name: str, node, defs: dict, done: set, chunk: int = SUM_CHUNK):
    """Statements that evaluate ``node`` into the scalar ``name``.

    A long left-associated sum is split after every ``chunk`` terms:
    ``s = (t0+t1)+...; s = (s+t8)+...`` performs the same additions in the
    same order as the single expression, so the rounding is unchanged, but
    the compiler no longer has to hold the loads of hundreds of terms at
    once.  Before each piece, the scalars it reads that are not yet defined
    (rates A, partials B: ``defs`` maps (tag, index) to its declaration) are
    declared, so that each is computed next to its first consumer."""
    out = []

    def declare(t):
        for tag in ("a", "b"):
            for x in _refs(t, tag):
                if (tag, x) not in done:
                    done.add((tag, x))
                    out.append(defs[(tag, x)])

    ts = _chain(node)
    for c0 in range(0, len(ts), chunk):
        piece = ts[c0:c0 + chunk]
        for _, t in piece:
            declare(t)
        expr = name if c0 else cexpr(piece[0][1])
        for op, t in (piece if c0 else piece[1:]):
            expr = f"({expr}{op}{cexpr(t)})"
        out.append(f"{'' if c0 else 'double '}{name} = {_strip(expr)};")
    return out


def fun_species_order(mech: dict) -> list:
    """The order in which fun_body emits the species: greedy, each next
    species the one that leaves the fewest rates live (a rate is live from
    the first species that reads it to the last).  Rates are shared by 3.7
    species on average; in index order ~530 are live at a time for
    fullchem, far more than registers hold, and each spilled rate is
    reloaded per use.  This order keeps ~150 live.  Any order computes the
    same expressions, so rounding is unchanged."""
    n = mech["nvar"]
    uses = [set(_refs(mech["prod"][i], "a")) for i in range(n)]
    left = {}
    for u in uses:
        for j in u:
            left[j] = left.get(j, 0) + 1
    live, order, remaining = set(), [], set(range(n))
    while remaining:
        best, best_key = None, None
        for i in sorted(remaining):
            u = uses[i]
            after = len(live | u) - sum(1 for j in u if left[j] == 1)
            key = (after, -len(u & live), i)
            if best_key is None or key < best_key:
                best, best_key = i, key
        order.append(best)
        remaining.remove(best)
        for j in uses[best]:
            live.add(j)
            left[j] -= 1
            if left[j] == 0:
                live.discard(j)
    return order


def fun_body(mech: dict) -> str:
    """Fun_SPLIT species by species: ``Vdot(i) = P_VAR(i) - D_VAR(i)*V(i)``,
    each rate A(j) declared as a scalar just before the first piece of a
    P_VAR sum that needs it, the species in ``fun_species_order``.

    Every value is the expression of the reference (gckpp_Function.F90:
    2170-5060, A(j) then P_VAR/D_VAR then Vdot) with its association kept;
    only the evaluation order differs, which changes no rounding.  Computing
    a rate next to its consumers keeps most of the 1,058 rates of fullchem
    in registers instead of a stack array that is written once and re-read
    per use (~3.7 reads per rate).  Rates that feed no variable species are
    not computed (they reach no output)."""
    defs = {("a", j): f"const double A_({j}) = {_strip(cexpr(e))};"
            for j, e in enumerate(mech["rates"])}
    done, st = set(), []
    for i in fun_species_order(mech):
        st += _sum_stmts(f"p{i}", mech["prod"][i], defs, done)
        st += _sum_stmts(f"d{i}", mech["dest"][i], defs, done)
        st.append(f"VDOT_({i}) = p{i} - (d{i}*V_({i}));")
    return "/* rates A(j) at first use; Vdot = P_VAR - D_VAR*V per species */\n" + \
        "\n".join(_fenced(st)) + "\n"


def jac_body(mech: dict) -> str:
    """Jac_SP in column-major order of the LU pattern: each partial B(m) =
    dA(j)/dV(s) feeds only entries of column s, so emitting the JVS entries
    column by column, with every partial declared as a scalar just before
    its first use, keeps it live for one column instead of the whole
    Jacobian.  Expressions and association are the reference's
    (gckpp_Jacobian.F90:47-20887); only the evaluation order differs."""
    defs = {("b", m): f"const double B_({m}) = {_strip(cexpr(e))};"
            for m, e in mech["jac_b"]}
    irow, icol = mech["lu_irow"], mech["lu_icol"]
    done, st = set(), []
    for k in sorted(range(len(mech["jvs"])), key=lambda p: (icol[p], irow[p])):
        st += _sum_stmts(f"j{k}", mech["jvs"][k], defs, done)
        st.append(f"JVS_({k}) = j{k};")
    return "/* partials B(m) at first use; JVS(k) column by column */\n" + \
        "\n".join(_fenced(st)) + "\n"


def solve_stmts(mech: dict):
    """KppSolve statement list (target, ast): forward unit-lower sweep over
    rows with sub-diagonal entries, then backward upper sweep with the
    diagonal divide -- the order of KppSolveIndirect
    (gckpp_LinearAlgebra.F90:175-200), which the generated KppSolve
    (:645-2311) follows term by term."""
    n = mech["nvar"]
    crow, diag, icol = mech["lu_crow"], mech["lu_diag"], mech["lu_icol"]
    st = []
    for i in range(n):
        if diag[i] > crow[i]:
            t = ["x", i]
            for j in range(crow[i], diag[i]):
                t = ["-", t, ["*", ["j", j], ["x", icol[j]]]]
            st.append([i, t])
    for i in range(n - 1, -1, -1):
        t = ["x", i]
        for j in range(diag[i] + 1, crow[i + 1]):
            t = ["-", t, ["*", ["j", j], ["x", icol[j]]]]
        st.append([i, ["/", t, ["j", diag[i]]]])
    return st


def solve_tr_stmts(mech: dict):
    """KppSolveTR statement list (gckpp_LinearAlgebra.F90:2327-3701), the
    transposed solve (LU)^T x = b on the same factors, in the generated
    routine's pull form and term order:

    * U^T sweep, i = 1..NVAR: ``XX(i) = (X(i) - JVS(p)*XX(j) - ...)/JVS(d_i)``
      over the entries U(j,i), j < i, in increasing j;
    * unit L^T sweep, i = NVAR..1: ``XX(i) = XX(i) - JVS(p)*XX(j) - ...``
      over the entries L(j,i), j > i, in increasing j.

    Each statement is ``[i, source, [[p, j], ...], d]`` with source "X" or
    "XX" and d = -1 when there is no divide."""
    n = mech["nvar"]
    crow, diag, icol = mech["lu_crow"], mech["lu_diag"], mech["lu_icol"]
    upper = [[] for _ in range(n)]   # column i <- [(p, row j)] of U, j < i
    lower = [[] for _ in range(n)]   # column i <- [(p, row j)] of L, j > i
    for j in range(n):
        for p in range(crow[j], crow[j + 1]):
            if p > diag[j]:
                upper[icol[p]].append([p, j])
            elif p < diag[j]:
                lower[icol[p]].append([p, j])
    st = [[i, "X", upper[i], diag[i]] for i in range(n)]
    st += [[i, "XX", lower[i], -1] for i in range(n - 1, -1, -1)]
    return st


def solve_tr_body(mech: dict, chunk: int = SUM_CHUNK) -> str:
    """Transposed solve for the adjoint, the statements of KppSolveTR in
    their order (``solve_tr_stmts``), in place on X (the U^T sweep reads
    X(i) once before writing it, so input and output can share storage).
    Long sums are evaluated in left-to-right pieces as in ``solve_body``;
    the divide is ``GC_SDIV(x, U(i,i), i)``."""
    st = []
    for n_st, (i, _, terms, d) in enumerate(solve_tr_stmts(mech)):
        if not terms and d < 0:
            continue                                  # XX(i) = XX(i)
        parts = [f"X_({i})"] + [f"(JVS_({p})*X_({j}))" for p, j in terms]
        if len(parts) <= chunk + 1:
            expr = parts[0]
            for t in parts[1:]:
                expr = f"({expr}-{t})"
        else:
            name = f"t{n_st}"
            expr = parts[0]
            for k, t in enumerate(parts[1:]):
                expr = f"({expr}-{t})"
                if (k + 1) % chunk == 0:
                    st.append(f"{'double ' if k + 1 == chunk else ''}{name} = {_strip(expr)};")
                    expr = name
            if expr != name:
                st.append(f"{name} = {_strip(expr)};")
            expr = name
        rhs = expr if d < 0 else f"GC_SDIV({expr}, JVS_({d}), {i})"
        st.append(f"X_({i}) = {_strip(rhs)};")
    return "\n".join(_fenced(st, 8)) + "\n"


# compiler fence spacing of the forward solve: measured on a B200 (37,888
# threads, ms per call): every 4 statements 0.881, 8 0.587, 16 0.534,
# 32 0.542, none 0.584
SOLVE_FENCE = 16
# terms per left-to-right piece of a long solve row (same B200 case, ms per
# call): 4 terms 0.580, 8 0.527, 12 0.527, 16 0.522
SOLVE_CHUNK = 16


def solve_body(mech: dict, chunk: int = SOLVE_CHUNK) -> str:
    """KppSolve statements.  A row whose sum has more than ``chunk`` terms is
    evaluated in left-to-right pieces into a scalar (``s = (x-a*b)-...;
    s = (s-c*d)-...;``), the same subtractions in the same order, and the
    backward sweep's diagonal divide is applied to the final value.  Long rows
    (up to 266 terms in fullchem) otherwise make the compiler hold every load
    of the row at once and spill.

    The divide is ``GC_SDIV(x, U(i,i), i)``: ``x/U(i,i)`` as in the reference,
    or, where the factorisation left ``R(i) = 1/U(i,i)`` (FMA build), ``x*R(i)``."""
    st = []
    for n_st, (i, e) in enumerate(solve_stmts(mech)):
        div = None
        if e[0] == "/":
            div, e = e[2], e[1]
        ts = _chain(e)
        if len(ts) <= chunk:
            rhs = cexpr(e) if div is None else f"GC_SDIV({cexpr(e)}, {cexpr(div)}, {i})"
            st.append(f"X_({i}) = {_strip(rhs)};")
            continue
        name = f"s{n_st}"
        for c0 in range(0, len(ts), chunk):
            piece = ts[c0:c0 + chunk]
            expr = name if c0 else cexpr(piece[0][1])
            for op, t in (piece if c0 else piece[1:]):
                expr = f"({expr}{op}{cexpr(t)})"
            st.append(f"{'' if c0 else 'double '}{name} = {_strip(expr)};")
        st.append(f"X_({i}) = {name if div is None else f'GC_SDIV({name}, {cexpr(div)}, {i})'};")
    return "\n".join(_fenced(st, SOLVE_FENCE)) + "\n"


def lu_fused_body(mech: dict, block: int = 40) -> str:
    """Straight-line KppDecomp fused with ros_PrepareMatrix, rows held in
    registers.

    Reads the Jacobian J0_(p) and writes the factors G_(p); finished
    factors are read back through GU_(p):
    ``G = -J0`` plus ``ghinv`` on the diagonal (gckpp_BatchIntegrator.F90:
    573-577), then the row-wise elimination of gckpp_LinearAlgebra.F90:46-84.
    Row k is processed in blocks of at most ``block`` consecutive entries,
    held in local variables.  For a block, every sub-diagonal pivot j of the
    row below the block's last column is visited in increasing order: a pivot
    inside the block forms ``a = -(w_j / G(diag j))`` and stores
    ``w_j = -a``; a pivot of an earlier block re-reads its stored value
    ``-a``; then ``w_c = w_c + a*G(j,c)`` for the block's columns c of U row
    j.  Each entry therefore receives exactly the reference's updates in the
    reference's order (increasing j), only the dense scratch row W becomes
    registers.  The singularity test (any original diagonal below TINY)
    is done by the caller before this code runs.

    Multipliers go through ``GC_PIVOT(w, diag, j)``, which is the
    reference's ``-(w/U(j,j))``.  A build may instead define it as
    ``-(w*R(j))`` with ``R(j) = 1/U(j,j)`` stored once per row by
    ``GC_RECIP(j, U(j,j))``: one divide per row instead of one per
    multiplier, which rounds differently (not for the bit-exact build).
    """
    n = mech["nvar"]
    crow, diag, icol = mech["lu_crow"], mech["lu_diag"], mech["lu_icol"]
    out = []
    for k in range(n):
        r0, r1 = crow[k], crow[k + 1]
        if diag[k] == r0:
            # no pivots: the row is only negated (+ ghinv on the diagonal)
            for p in range(r0, r1):
                if p == diag[k]:
                    out.append(f"{{ const double dv = (-J0_({p})) + ghinv; G_({p}) = dv; "
                               f"GC_RECIP({k}, dv); }}")
                else:
                    out.append(f"G_({p}) = -J0_({p});")
            continue
        out.append(f"/* row {k} */")
        out.append("GC_ROW_FENCE();")
        ents = list(range(r0, r1))
        for b0 in range(0, len(ents), block):
            blk = ents[b0:b0 + block]
            cmin, cmax = icol[blk[0]], icol[blk[-1]]
            pos_of = {icol[p]: p for p in blk}
            out.append("{")
            for p in blk:
                init = f"(-J0_({p})) + ghinv" if p == diag[k] else f"-J0_({p})"
                out.append(f"  double w{p} = {init};")
            for kk in range(r0, diag[k]):
                j = icol[kk]
                if j > cmax:   # pivot j only updates columns c > j
                    break
                targets = [(jj, pos_of[icol[jj]]) for jj in range(diag[j] + 1, crow[j + 1])
                           if icol[jj] in pos_of]
                if j >= cmin:  # pivot inside this block
                    out.append(f"  {{ const double a = GC_PIVOT(w{kk}, GU_({diag[j]}), {j});")
                    out.append(f"    w{kk} = -a;")
                elif targets:
                    out.append(f"  {{ const double a = -GU_({kk});")
                else:
                    continue
                for jj, p in targets:
                    out.append(f"    w{p} = w{p} + (a*GU_({jj}));")
                out.append("  }")
            for p in blk:
                out.append(f"  G_({p}) = w{p};")
                if p == diag[k]:
                    out.append(f"  GC_RECIP({k}, w{p});")
            out.append("}")
    return "\n".join(out) + "\n"


def _rate_factors(e):
    """Factors of a rate A(j) (a left-associated product chain)."""
    if e[0] == "*":
        return _rate_factors(e[1]) + _rate_factors(e[2])
    return [e]


def adjoint_tables(mech: dict) -> str:
    """Per-reaction tables for the discrete adjoint: the factors of each rate
    A(j) = const * V(v1)*V(v2)*V(v3) (const = RCT(j) or a literal, times
    fixed species F), and the net stoichiometric matrix S (reaction-major
    CSR; CalcStoichNum, gckpp_Function.F90:7271-12790, for fullchem)."""
    n = mech["nreact"]
    rct, lit, nv, vv, ff = [], [], [], [], []
    for j, e in enumerate(mech["rates"]):
        r, l, vs, fs = -1, 1.0, [], []
        for f in _rate_factors(e):
            if f[0] == "k":
                r = f[1]
            elif f[0] == "n":
                l *= float(literal(f[1]))
            elif f[0] == "v":
                vs.append(f[1])
            elif f[0] == "f":
                fs.append(f[1])
            else:
                raise ValueError(f"unexpected factor {f} in A({j + 1})")
        if len(vs) > 3 or len(fs) > 2 or (r >= 0 and r != j):
            raise ValueError(f"rate A({j + 1}) outside the adjoint's forms")
        rct.append(r)
        lit.append(l)
        nv.append(len(vs))
        vv += vs + [0] * (3 - len(vs))
        ff += fs + [-1] * (2 - len(fs))
    by_r = [[] for _ in range(n)]
    for i, j, v in mech["stoich"]:
        by_r[j].append((i, float(literal(v))))
    ptr, sp, sv = [0], [], []
    for j in range(n):
        for i, v in sorted(by_r[j]):
            sp.append(i)
            sv.append(v)
        ptr.append(len(sp))

    def arr(name, vals):
        return f"#define {name}_INIT {{{','.join(repr(x) for x in vals)}}}"

    return "\n".join([
        "/* generated adjoint tables; do not edit */",
        "#pragma once",
        f"#define ADJ_NSTO {len(sp)}",
        arr("ADJ_RCT", rct), arr("ADJ_LIT", lit), arr("ADJ_NV", nv),
        arr("ADJ_V", vv), arr("ADJ_F", ff),
        arr("ADJ_SPTR", ptr), arr("ADJ_SSP", sp), arr("ADJ_SVAL", sv), ""])


def mech_header(mech: dict, name: str) -> str:
    n = mech["nvar"]

    def arr(cname, vals, ctype="int"):
        body = ",".join(str(v) for v in vals)
        return (f"#define {cname}_INIT {{{body}}}\n"
                f"static const {ctype} {cname}[{len(vals)}] = {cname}_INIT;")

    return "\n".join([
        f"/* generated from the {name} mechanism tables; do not edit */",
        "#pragma once",
        f"#define MECH_NAME \"{name}\"",
        f"#define MECH_NVAR {n}",
        f"#define MECH_NFIX {mech['nfix']}",
        f"#define MECH_NSPEC {n + mech['nfix']}",
        f"#define MECH_NREACT {mech['nreact']}",
        f"#define MECH_NNZ {mech['nnz']}",
        f"#define MECH_NB {mech['nb']}",
        arr("MECH_LU_CROW", mech["lu_crow"]),
        arr("MECH_LU_DIAG", mech["lu_diag"]),
        arr("MECH_LU_ICOL", mech["lu_icol"]),
        arr("MECH_LU_IROW", mech["lu_irow"]),
        "",
    ])


def flop_counts(mech: dict) -> dict:
    """Floating-point operations per call of each generated routine (every
    +, -, *, / counted once; unary minus not counted)."""
    def ops(e):
        if e[0] in _ACC or e[0] == "n":
            return 0
        if e[0] == "neg":
            return ops(e[1])
        return 1 + ops(e[1]) + ops(e[2])
    n = mech["nvar"]
    crow, diag, icol = mech["lu_crow"], mech["lu_diag"], mech["lu_icol"]
    fun = sum(ops(e) for e in mech["rates"]) + \
        sum(ops(e) for e in mech["prod"]) + \
        sum(ops(e) for e in mech["dest"]) + 2 * n
    jac = sum(ops(e) for _, e in mech["jac_b"]) + \
        sum(ops(e) for e in mech["jvs"])
    ndiv = sum(diag[k] - crow[k] for k in range(n))
    nupd = sum(crow[icol[kk] + 1] - diag[icol[kk]] - 1
               for k in range(n) for kk in range(crow[k], diag[k]))
    lu = ndiv + 2 * nupd
    solve = sum(ops(e) for _, e in solve_stmts(mech))
    prep = mech["nnz"] + n  # negation of Jac0 + diagonal add (counted as ops)
    return {"fun": fun, "jac": jac, "lu": lu, "solve": solve, "prep": prep,
            "vec": 12 * n}


# factorisations above this many flops are left to the indexed KppDecomp:
# straight-line code for them compiles for many minutes and fills the
# instruction cache (dense-ish patterns such as random mechanisms)
FUSED_LU_MAX_FLOPS = 120000


def fused_lu(mech: dict) -> bool:
    return flop_counts(mech)["lu"] <= FUSED_LU_MAX_FLOPS


def generate(mech: dict, name: str, outdir: str) -> dict:
    from . import coop  # the cooperative kernel's tables (coop.py imports this module)
    os.makedirs(outdir, exist_ok=True)
    fused = fused_lu(mech)
    files = {
        "mech.h": mech_header(mech, name) + f"#define MECH_FUSED_LU {1 if fused else 0}\n",
        "fun.inc": fun_body(mech),
        "jac.inc": jac_body(mech),
        "solve.inc": solve_body(mech),
        "adj.inc": adjoint_tables(mech),
        "solve_tr.inc": solve_tr_body(mech),
        "lu_fused.inc": lu_fused_body(mech) if fused else
        "/* not generated: this mechanism uses the indexed KppDecomp */\n",
        "coop.inc": coop.coop_inc(mech),
    }
    for fn, txt in files.items():
        path = os.path.join(outdir, fn)
        old = None
        if os.path.exists(path):
            with open(path) as fh:
                old = fh.read()
        if old != txt:  # keep mtimes stable so make does not rebuild
            with open(path, "w") as fh:
                fh.write(txt)
    return files
