"""Tables for the cooperative kernel (one thread block per cell).

The one-thread-per-cell kernels run straight-line statement lists.  In the
cooperative kernel the threads of a block share one cell, so every thread
runs the same instructions on different entries: Fun, Jac, the
factorisation and the solves become loops over tables.  This module turns
the mechanism IR into those tables; ``coop_inc`` emits them as C arrays.

Expressions.  Every rate A(j), production P_VAR(i), destruction D_VAR(i),
Jacobian partial B(m) and entry JVS(k) of the IR is a left-associated
signed sum ``((t0 op t1) op t2) ...`` (the first term possibly negated) of
left-associated products ``((f0*f1)*f2)*f3`` whose factors are variable
species V, fixed species F, rate constants RCT, rates A / partials B (one
scratch array) or literals.  A term is stored as four 16-bit factor codes
(kind << 13 | index, 0xFFFF for none) and an operation code (0 first term,
1 first term negated, 2 add, 3 subtract).  Evaluated in table order, each
value gets exactly the operations of the generated Fun_SPLIT / Jac_SP
statements (gckpp_Function.F90:2170-5060, gckpp_Jacobian.F90:47-20887), so
the --fmad=false build rounds like them.  A mechanism with any other
expression shape gets no tables (``compile_tables`` returns None) and no
cooperative kernel.

Factorisation (KppDecomp, gckpp_LinearAlgebra.F90:46-84), right-looking.
The reference eliminates row by row: row k receives, in increasing pivot
order j, ``W(c) = W(c) + a*U(j,c)`` with ``a = -(W(j)/U(j,j))``, and stores
``-a`` as L(k,j).  Step j of the right-looking form first forms the
multipliers of column j (every row i > j with L(i,j) in the pattern) and
then applies pivot row j to all those rows at once.  Each entry still
receives its updates in increasing pivot order and the same operations, so
the result is the same bit for bit; the parallelism is the rows and columns
of one step instead of one row's columns.

Solves (KppSolve, gckpp_LinearAlgebra.F90:645-2311).  The forward sweep
``X(i) = X(i) - L(i,j)*X(j)`` over increasing j is run column by column:
at step j, X(j) is final and every row i with L(i,j) subtracts its term --
the same per-row order.  The backward sweep subtracts U(i,c)*X(c) in
increasing c and then divides; its rows are grouped into levels (a row's
level is one more than the highest level among its columns), rows of one
level run in parallel, each row's terms in the reference order.  That
order makes the sweep a chain of every row's terms (2,452 dependent
subtractions for the synthetic mechanism), so the FMA build, which need
not round like the reference, runs the backward sweep by columns too
(``bwc``: at step i, X(i) = acc(i)/U(i,i) and every row r < i with U(r,i)
subtracts its term), in the reverse of the reference's per-row order.
"""
from __future__ import annotations

from . import codegen

KIND_V, KIND_F, KIND_K, KIND_S, KIND_N = 0, 1, 2, 3, 4
NONE = 0xFFFF
OP_FIRST, OP_NEG, OP_ADD, OP_SUB = 0, 1, 2, 3
MAX_FACTORS = 4
MAX_INDEX = 1 << 13


class Unsupported(ValueError):
    pass


def _factors(node, consts):
    """Factor codes of a left-associated product chain."""
    out = []
    while isinstance(node, list) and node[0] == "*":
        out.append(node[2])
        node = node[1]
    out.append(node)
    out.reverse()
    codes = []
    for f in out:
        tag = f[0]
        if tag == "v":
            kind, idx = KIND_V, f[1]
        elif tag == "f":
            kind, idx = KIND_F, f[1]
        elif tag == "k":
            kind, idx = KIND_K, f[1]
        elif tag in ("a", "b"):
            kind, idx = KIND_S, f[1]
        elif tag == "n":
            val = float(codegen.literal(f[1]))
            if val not in consts:
                consts[val] = len(consts)
            kind, idx = KIND_N, consts[val]
        else:
            raise Unsupported(f"factor {f}")
        if not 0 <= idx < MAX_INDEX:
            raise Unsupported(f"index {idx}")
        codes.append((kind << 13) | idx)
    if len(codes) > MAX_FACTORS:
        raise Unsupported("product of more than four factors")
    return codes + [NONE] * (MAX_FACTORS - len(codes))


def _sum_terms(node, consts):
    """(op, factor codes) of a left-associated signed sum of products."""
    terms = []
    for i, (op, t) in enumerate(codegen._chain(node)):
        if i == 0:
            code = OP_FIRST
            if t[0] == "neg":
                code, t = OP_NEG, t[1]
        else:
            code = OP_ADD if op == "+" else OP_SUB
        terms.append((code, _factors(t, consts)))
    return terms


def compile_tables(mech: dict):
    """All tables of the cooperative kernel, or None when some expression
    falls outside the supported shapes."""
    n, nnz = mech["nvar"], mech["nnz"]
    nreact, nb = mech["nreact"], mech["nb"]
    crow, diag, icol = mech["lu_crow"], mech["lu_diag"], mech["lu_icol"]
    where = mech["lu_where"]
    if nnz >= 1 << 16 or n >= 1 << 16:
        return None
    consts: dict = {}
    sums = []
    try:
        for e in mech["rates"]:                       # A(j): ids 0 .. NREACT-1
            sums.append(_sum_terms(e, consts))
        for e in mech["prod"]:                        # P_VAR(i)
            sums.append(_sum_terms(e, consts))
        for e in mech["dest"]:                        # D_VAR(i)
            sums.append(_sum_terms(e, consts))
        bexpr = [["n", "0"]] * nb                     # indices no entry reads
        for m, e in mech["jac_b"]:
            bexpr[m] = e
        for e in bexpr:                               # B(m)
            sums.append(_sum_terms(e, consts))
        for e in mech["jvs"]:                         # JVS(k)
            sums.append(_sum_terms(e, consts))
    except Unsupported:
        return None
    off, ops, fac = [0], [], []
    for s in sums:
        for op, codes in s:
            ops.append(op)
            fac.extend(codes)
        off.append(len(ops))

    # right-looking factorisation: per pivot j, the L(i,j) positions and the
    # updates (target (i,c), multiplier (i,j), source (j,c))
    mul = [[] for _ in range(n)]
    upd = [[] for _ in range(n)]
    for i in range(n):
        for kk in range(crow[i], diag[i]):
            j = icol[kk]
            mul[j].append(kk)
            for jj in range(diag[j] + 1, crow[j + 1]):
                upd[j].append((where[(i, icol[jj])], kk, jj))
    mul_off, mul_pos, upd_off, upd_ent = [0], [], [0], []
    for j in range(n):
        mul_pos += mul[j]
        mul_off.append(len(mul_pos))
        upd_ent += upd[j]
        upd_off.append(len(upd_ent))

    # forward sweep by columns: per j, the (row, L position) pairs
    fwd = [[] for _ in range(n)]
    for i in range(n):
        for kk in range(crow[i], diag[i]):
            fwd[icol[kk]].append((i, kk))
    fwd_off, fwd_ent = [0], []
    for j in range(n):
        fwd_ent += fwd[j]
        fwd_off.append(len(fwd_ent))

    # backward sweep by levels
    lev = [0] * n
    for i in range(n - 1, -1, -1):
        lev[i] = max([lev[icol[jj]] + 1 for jj in range(diag[i] + 1, crow[i + 1])] + [0])
    nlev = max(lev) + 1 if n else 0
    bwd_rows, bwd_off = [], [0]
    for level in range(nlev):
        bwd_rows += [i for i in range(n) if lev[i] == level]
        bwd_off.append(len(bwd_rows))

    # backward sweep by columns (FMA build): per column i, from the last, the
    # (row r < i, U(r,i) position) pairs
    bwc = [[] for _ in range(n)]
    for r in range(n):
        for jj in range(diag[r] + 1, crow[r + 1]):
            bwc[icol[jj]].append((r, jj))
    bwc_off, bwc_ent = [0], []
    for i in range(n - 1, -1, -1):
        bwc_ent += bwc[i]
        bwc_off.append(len(bwc_ent))

    kdiag = [-1] * nnz
    for i in range(n):
        kdiag[diag[i]] = i

    cvals = [0.0] * len(consts)
    for v, k in consts.items():
        cvals[k] = v
    return {
        "nsum": len(sums), "sum_off": off, "term_op": ops, "term_fac": fac,
        "consts": cvals or [0.0],
        "mul_off": mul_off, "mul_pos": mul_pos or [0],
        "upd_off": upd_off, "upd": upd_ent,
        "fwd_off": fwd_off, "fwd": fwd_ent,
        "bwd_off": bwd_off, "bwd_rows": bwd_rows, "nlev": nlev,
        "bwc_off": bwc_off, "bwc": bwc_ent,
        "kdiag": kdiag,
        "sid_rate": 0, "sid_prod": nreact, "sid_dest": nreact + n,
        "sid_b": nreact + 2 * n, "sid_jvs": nreact + 2 * n + nb,
    }


def coop_inc(mech: dict) -> str:
    """coop.inc: MECH_COOP and, when the tables exist, their C arrays
    (device-side ``static __device__ const`` definitions, included by one
    translation unit)."""
    t = compile_tables(mech)
    if t is None:
        return "/* no cooperative-kernel tables: unsupported expression shape */\n" \
               "#define MECH_COOP 0\n"

    def arr(ctype, name, vals, align="", space="__device__ const"):
        body = ",".join(str(v) for v in vals) if vals else "0"
        n = max(len(vals), 1)
        return f"static {space} {align}{ctype} {name}[{n}] = {{{body}}};"

    # per-step offsets are read by every thread of a block at the same index:
    # constant memory broadcasts them
    const = "__constant__"

    upd_flat = []
    for tt, p, u in t["upd"]:
        upd_flat += [tt, p, u, 0]
    fwd_flat = []
    for i, p in t["fwd"]:
        fwd_flat += [i, p]
    bwc_flat = []
    for r, q in t["bwc"]:
        bwc_flat += [r, q]
    lines = [
        "/* generated cooperative-kernel tables; do not edit */",
        "#pragma once",
        "#define MECH_COOP 1",
        f"#define COOP_NSUM {t['nsum']}",
        f"#define COOP_SID_RATE {t['sid_rate']}",
        f"#define COOP_SID_PROD {t['sid_prod']}",
        f"#define COOP_SID_DEST {t['sid_dest']}",
        f"#define COOP_SID_B {t['sid_b']}",
        f"#define COOP_SID_JVS {t['sid_jvs']}",
        f"#define COOP_NLEV {t['nlev']}",
        f"#define COOP_NUPD {len(t['upd'])}",
        arr("int", "coop_sum_off", t["sum_off"]),
        arr("unsigned char", "coop_term_op", t["term_op"]),
        arr("unsigned short", "coop_term_fac", t["term_fac"], "__align__(8) "),
        "static __device__ const double coop_const[%d] = {%s};" % (
            len(t["consts"]), ",".join(repr(float(c)) for c in t["consts"])),
        arr("int", "coop_mul_off", t["mul_off"], space=const),
        arr("unsigned short", "coop_mul_pos", t["mul_pos"]),
        arr("int", "coop_upd_off", t["upd_off"], space=const),
        arr("unsigned short", "coop_upd", upd_flat, "__align__(8) "),
        arr("int", "coop_fwd_off", t["fwd_off"], space=const),
        arr("unsigned short", "coop_fwd", fwd_flat, "__align__(4) "),
        arr("int", "coop_bwd_off", t["bwd_off"], space=const),
        arr("unsigned short", "coop_bwd_rows", t["bwd_rows"]),
        arr("int", "coop_bwc_off", t["bwc_off"], space=const),
        arr("unsigned short", "coop_bwc", bwc_flat, "__align__(4) "),
        arr("short", "coop_kdiag", t["kdiag"]),
        "",
    ]
    return "\n".join(lines)
