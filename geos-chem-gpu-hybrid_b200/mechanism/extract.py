"""Extract the fullchem mechanism tables from the reference's generated KPP code.

The reference does not vendor gckpp_Parameters / gckpp_JacobianSP (the
sizes and the LU sparsity tables), so everything is recovered from the three
generated kernel files:

* sizes NVAR/NREACT from the highest V()/RCT() index used, NFIX from F(),
  LU_NONZERO from the JVS assignments (gckpp_Jacobian.F90:31 declares 5683);
* LU_IROW/LU_ICOL from the ``! JVS(k) = Jac_FULL(i,j)`` comments
  (gckpp_Jacobian.F90:3675-20886), LU_CROW/LU_DIAG derived from them;
* the ordered expression trees of Fun_SPLIT (gckpp_Function.F90:2170-5060),
  Jac_SP (gckpp_Jacobian.F90:47-20887) and KppSolve
  (gckpp_LinearAlgebra.F90:645-2311).

Run as a script to (re)write ``fullchem.json`` next to this file:

    python -m mechanism.extract /path/to/reference   (from the package dir)

The JSON file is the mechanism *data* (reaction network, stoichiometric
coefficients, sparsity); all code that evaluates it is generated by
``codegen.py``.
"""
from __future__ import annotations

import json
import os
import re
import sys

try:
    from . import fortran_ir as fir
except ImportError:  # executed as a plain script
    import fortran_ir as fir  # type: ignore

KPP_DIR = os.path.join("src", "geos-chem", "KPP", "fullchem")


def _subroutine(lines: list[str], name: str) -> tuple[int, list[str]]:
    """Return (1-based first line, body lines) of SUBROUTINE ``name``."""
    start = end = None
    for i, l in enumerate(lines):
        s = l.strip()
        if start is None and s.startswith("SUBROUTINE") and \
                s.split()[1].split("(")[0] == name:
            start = i
        elif start is not None and s.startswith("END SUBROUTINE") and \
                s.split()[2] == name:
            end = i
            break
    if start is None or end is None:
        raise ValueError(f"subroutine {name} not found")
    return start + 1, lines[start:end + 1]


def _max_index(node, kind, best=-1):
    if node[0] == kind:
        return max(best, node[1])
    if node[0] in ("n",) or isinstance(node[1], int):
        return best
    for ch in node[1:]:
        best = _max_index(ch, kind, best)
    return best


def extract(ref_root: str) -> dict:
    kdir = os.path.join(ref_root, KPP_DIR)
    fun_lines = open(os.path.join(kdir, "gckpp_Function.F90")).read().split("\n")
    jac_lines = open(os.path.join(kdir, "gckpp_Jacobian.F90")).read().split("\n")
    la_lines = open(os.path.join(kdir, "gckpp_LinearAlgebra.F90")).read().split("\n")

    fun_at, fun = _subroutine(fun_lines, "Fun_SPLIT")
    jac_at, jac = _subroutine(jac_lines, "Jac_SP")
    slv_at, slv = _subroutine(la_lines, "KppSolve")

    rates: dict[int, list] = {}
    prod: dict[int, list] = {}
    dest: dict[int, list] = {}
    for lhs, idx, ast, _ in fir.assignments(fun):
        tgt = {"A": rates, "P_VAR": prod, "D_VAR": dest}[lhs]
        if idx in tgt:
            raise ValueError(f"{lhs}({idx + 1}) assigned twice")
        tgt[idx] = ast

    bpart: dict[int, list] = {}
    jvs: dict[int, list] = {}
    pos: dict[int, tuple[int, int]] = {}
    for lhs, idx, ast, comment in fir.assignments(jac):
        if lhs == "B":
            bpart[idx] = ast
        elif lhs == "JVS":
            jp = fir.jac_full_position(comment)
            if jp is None or jp[0] != idx:
                raise ValueError(f"JVS({idx + 1}) has no Jac_FULL comment")
            pos[idx] = (jp[1], jp[2])
            jvs[idx] = ast
        else:
            raise ValueError(f"unexpected {lhs} in Jac_SP")

    solve = [[idx, ast] for lhs, idx, ast, _ in fir.assignments(slv)
             if lhs == "X"]

    # net stoichiometric numbers StoichNum(i,j) (CalcStoichNum,
    # gckpp_Function.F90:7271-12790), kept as decimal text
    sto_at, sto = _subroutine(fun_lines, "CalcStoichNum")
    stoich = []
    for line in sto:
        m = re.match(r"\s*StoichNum\((\d+),(\d+)\)\s*=\s*(\S+)\s*$", line)
        if m:
            stoich.append([int(m.group(1)) - 1, int(m.group(2)) - 1, m.group(3)])

    nreact = len(rates)
    nvar = len(prod)
    nnz = len(jvs)
    # B partials with respect to fixed species are declared but never
    # assigned (e.g. B(436) = dA(227)/dF(2) is skipped), so B is sparse.
    nb = 1 + max(bpart)
    for d, n, what in ((rates, nreact, "A"), (prod, nvar, "P_VAR"),
                       (dest, nvar, "D_VAR"), (jvs, nnz, "JVS")):
        if sorted(d) != list(range(n)):
            raise ValueError(f"{what} indices are not 1..{n}")
    nfix = 1 + max(_max_index(e, "f") for e in list(rates.values()) +
                   list(bpart.values()) + list(dest.values()))
    maxv = max(_max_index(e, "v") for e in rates.values())
    maxk = max(_max_index(e, "k") for e in rates.values())
    if maxv + 1 > nvar or maxk + 1 != nreact:
        raise ValueError("inconsistent sizes")

    return {
        "name": "fullchem",
        "source": {
            "Fun_SPLIT": f"src/geos-chem/KPP/fullchem/gckpp_Function.F90:{fun_at}",
            "Jac_SP": f"src/geos-chem/KPP/fullchem/gckpp_Jacobian.F90:{jac_at}",
            "KppSolve": f"src/geos-chem/KPP/fullchem/gckpp_LinearAlgebra.F90:{slv_at}",
            "CalcStoichNum": f"src/geos-chem/KPP/fullchem/gckpp_Function.F90:{sto_at}",
        },
        "nvar": nvar, "nfix": nfix, "nreact": nreact, "nnz": nnz, "nb": nb,
        "lu_irow": [pos[k][0] for k in range(nnz)],
        "lu_icol": [pos[k][1] for k in range(nnz)],
        "rates": [rates[j] for j in range(nreact)],
        "prod": [prod[i] for i in range(nvar)],
        "dest": [dest[i] for i in range(nvar)],
        "jac_b": [[k, bpart[k]] for k in sorted(bpart)],
        "jvs": [jvs[k] for k in range(nnz)],
        "solve": solve,
        "stoich": stoich,
    }


def main(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    ref = argv[0] if argv else os.environ.get("GCCHEM_REFERENCE", "")
    if not ref or not os.path.isdir(ref):
        raise SystemExit("usage: extract.py <reference checkout>")
    mech = extract(ref)
    out = argv[1] if len(argv) > 1 else os.path.join(
        os.path.dirname(os.path.abspath(__file__)), "fullchem.json")
    with open(out, "w") as fh:
        json.dump(mech, fh, separators=(",", ":"))
    print(f"wrote {out}: NVAR={mech['nvar']} NFIX={mech['nfix']} "
          f"NREACT={mech['nreact']} NNZ={mech['nnz']} NB={mech['nb']}")


if __name__ == "__main__":
    main()
