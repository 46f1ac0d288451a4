"""Freeze the reference's independent renderings of the fullchem mechanism
into tests/golden/reference_pins.json.gz (run in a checkout that has the
reference; the tests read only the fixture).

The oracle's Fun_SPLIT / Jac_SP / KppSolve come from the project's own
expression parser (mechanism/fortran_ir.py).  To pin them to the reference
without trusting that parser, this script reads OTHER generated routines of
the same KPP mechanism with a separate, deliberately minimal reader (fixed
regular expressions for the few statement forms these routines use; no
expression trees):

* ``CalcStoichNum`` (src/geos-chem/KPP/fullchem/gckpp_Function.F90:7271-12790):
  ``StoichNum(i,j) = c`` -- the net stoichiometric matrix S;
* the aggregate ``Fun`` (gckpp_Function.F90:47-2150): the rates
  ``A(j) = RCT(j)*V(a)*...*F(b)`` and ``Vdot(i) = c1*A(j1)+c2*A(j2)-...``;
* ``Jac_SP_Vec`` and ``JacTR_SP_Vec`` (gckpp_Jacobian.F90:20903-22738):
  ``JUV(i) = JVS(p)*UV(c)+...`` and ``JTUV(c) = JVS(p)*UV(i)+...``;
* ``KppSolveTR`` (gckpp_LinearAlgebra.F90:2327-3701): the transposed solve,
  ``XX(i) = (X(i)-JVS(p)*XX(j)-...)/(JVS(d))`` then ``XX(i) = XX(i)-...``.

Usage:  python tests/golden/make_pins.py [reference root]
"""
from __future__ import annotations

import gzip
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
KPP = os.path.join("src", "geos-chem", "KPP", "fullchem")


def _routine(path: str, name: str) -> tuple[int, list[str]]:
    """(first line, logical statements) of SUBROUTINE name; continuation
    lines (trailing '&', leading '&') are joined, comments dropped."""
    lines = open(path).read().split("\n")
    start = next(i for i, l in enumerate(lines)
                 if re.match(rf"\s*SUBROUTINE\s+{name}\s*\(", l))
    end = next(i for i in range(start, len(lines))
               if re.match(rf"\s*END\s+SUBROUTINE\s+{name}\b", lines[i]))
    stmts, cur = [], ""
    for raw in lines[start + 1:end]:
        s = raw.split("!")[0].rstrip()
        if not s.strip():
            continue
        s = s.strip()
        if s.startswith("&"):
            s = s[1:]
        if s.endswith("&"):
            cur += s[:-1]
            continue
        stmts.append(cur + s)
        cur = ""
    return start + 1, stmts


_NUM = r"[0-9]*\.?[0-9]+(?:[eEdD][-+]?[0-9]+)?"


def stoich(path):
    at, st = _routine(path, "CalcStoichNum")
    out = []
    for s in st:
        m = re.fullmatch(rf"StoichNum\((\d+),(\d+)\)\s*=\s*(-?{_NUM})", s.replace(" ", ""))
        if m:
            out.append([int(m.group(1)) - 1, int(m.group(2)) - 1, m.group(3)])
    return at, out


def aggregate_fun(path):
    """Rates as factor lists and Vdot(i) as signed coefficient lists, in the
    reference's term order."""
    at, st = _routine(path, "Fun")
    rates, vdot = {}, {}
    for s in st:
        s = s.replace(" ", "")
        if s.startswith("IF(DO_FUN("):
            s = s[s.index(")") + 2:]        # guard: "IF (DO_FUN(i)) Vdot(i) = ..."
        m = re.fullmatch(r"A\((\d+)\)=(.*)", s)
        if m:
            j = int(m.group(1)) - 1
            fac = m.group(2).split("*")
            r = {"rct": -1, "lit": "1", "v": [], "f": []}
            for f in fac:
                g = re.fullmatch(r"(RCT|V|F)\((\d+)\)", f)
                if g:
                    key = {"RCT": "rct", "V": "v", "F": "f"}[g.group(1)]
                    if key == "rct":
                        r["rct"] = int(g.group(2)) - 1
                    else:
                        r[key].append(int(g.group(2)) - 1)
                elif re.fullmatch(_NUM, f):
                    r["lit"] = f
                else:
                    raise ValueError(f"A({j + 1}): factor {f}")
            rates[j] = r
            continue
        m = re.fullmatch(r"Vdot\((\d+)\)=(.*)", s)
        if m:
            i = int(m.group(1)) - 1
            terms = []
            for sign, coef, j in re.findall(rf"([-+]?)(?:({_NUM})\*)?A\((\d+)\)", m.group(2)):
                c = coef if coef else "1"
                terms.append([int(j) - 1, ("-" if sign == "-" else "") + c])
            rebuilt = "".join(("" if (k == 0 and not t[1].startswith("-")) else
                               ("-" if t[1].startswith("-") else "+")) +
                              ("" if t[1].lstrip("-") == "1" else t[1].lstrip("-") + "*") +
                              f"A({t[0] + 1})" for k, t in enumerate(terms))
            if rebuilt != m.group(2) and not _same_terms(rebuilt, m.group(2)):
                raise ValueError(f"Vdot({i + 1}) not read completely")
            vdot[i] = terms
    n = max(rates) + 1
    return at, [rates[j] for j in range(n)], [vdot.get(i, []) for i in range(max(vdot) + 1)]


def _same_terms(a: str, b: str) -> bool:
    # "1*A(j)" may be written with an explicit coefficient in the source
    return a.replace("1*A", "A") == b.replace("1*A", "A")


def jac_vec(path, name, out_name, uv="UV"):
    at, st = _routine(path, name)
    rows = {}
    for s in st:
        s = s.replace(" ", "")
        m = re.fullmatch(rf"{out_name}\((\d+)\)=(.*)", s)
        if not m:
            continue
        terms = [[int(p) - 1, int(c) - 1]
                 for p, c in re.findall(rf"JVS\((\d+)\)\*{uv}\((\d+)\)", m.group(2))]
        if len(terms) != m.group(2).count("JVS("):
            raise ValueError(f"{name}: {s}")
        rows[int(m.group(1)) - 1] = terms
    return at, [rows.get(i, []) for i in range(max(rows) + 1)]


def solve_tr(path):
    """KppSolveTR statements: [target, rhs source ('X' or 'XX'),
    [[p, j], ...] subtracted terms in order, diagonal position or -1]."""
    at, st = _routine(path, "KppSolveTR")
    out = []
    for s in st:
        s = s.replace(" ", "")
        m = re.fullmatch(r"XX\((\d+)\)=(.*)", s)
        if not m:
            continue
        i, rhs = int(m.group(1)) - 1, m.group(2)
        div = -1
        d = re.fullmatch(r"\((.*)\)/\(JVS\((\d+)\)\)", rhs) or \
            re.fullmatch(r"(X\(\d+\))/JVS\((\d+)\)", rhs)
        if d:
            rhs, div = d.group(1), int(d.group(2)) - 1
        h = re.match(r"(XX|X)\((\d+)\)", rhs)
        if not h or int(h.group(2)) - 1 != i:
            raise ValueError(f"KppSolveTR: {s}")
        terms = [[int(p) - 1, int(j) - 1] for p, j in re.findall(r"-JVS\((\d+)\)\*XX\((\d+)\)",
                                                                 rhs[h.end():])]
        if len(terms) != rhs.count("JVS("):
            raise ValueError(f"KppSolveTR: {s}")
        out.append([i, h.group(1), terms, div])
    return at, out


def main(ref_root: str) -> str:
    kdir = os.path.join(ref_root, KPP)
    fun = os.path.join(kdir, "gckpp_Function.F90")
    jac = os.path.join(kdir, "gckpp_Jacobian.F90")
    la = os.path.join(kdir, "gckpp_LinearAlgebra.F90")
    s_at, S = stoich(fun)
    f_at, rates, vdot = aggregate_fun(fun)
    jv_at, jv = jac_vec(jac, "Jac_SP_Vec", "JUV")
    jt_at, jt = jac_vec(jac, "JacTR_SP_Vec", "JTUV")
    tr_at, tr = solve_tr(la)
    data = {
        "source": {"CalcStoichNum": f"{KPP}/gckpp_Function.F90:{s_at}",
                   "Fun": f"{KPP}/gckpp_Function.F90:{f_at}",
                   "Jac_SP_Vec": f"{KPP}/gckpp_Jacobian.F90:{jv_at}",
                   "JacTR_SP_Vec": f"{KPP}/gckpp_Jacobian.F90:{jt_at}",
                   "KppSolveTR": f"{KPP}/gckpp_LinearAlgebra.F90:{tr_at}"},
        "stoich": S, "rates": rates, "vdot": vdot,
        "jac_sp_vec": jv, "jactr_sp_vec": jt, "kppsolvetr": tr,
    }
    out = os.path.join(HERE, "reference_pins.json.gz")
    with gzip.open(out, "wt") as fh:
        json.dump(data, fh, separators=(",", ":"))
    return out


if __name__ == "__main__":
    print(main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference"))
