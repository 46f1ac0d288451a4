"""Seeded synthetic stiff mass-action mechanism in the fullchem IR format.

120 species and 360 reactions, each with 1-2 reactants and 1-3 products
(no species appears on both sides).  The generated kernels follow KPP's
conventions for Fun_SPLIT / Jac_SP (the forms of
src/geos-chem/KPP/fullchem/gckpp_Function.F90:2170-5060 and
gckpp_Jacobian.F90:47-20887):

* ``A(j) = RCT(j)*V(a)[*V(b)]``;
* ``P_VAR(i)`` = sum over producing reactions, in reaction order, of
  ``A(j)`` or ``c*A(j)`` (c = the product multiplicity);
* ``D_VAR(i)`` = sum over consuming reactions of ``RCT(j)`` (unimolecular),
  ``RCT(j)*V(other)`` (bimolecular) or ``RCT(j)*2*V(i)`` (self reaction),
  so that Vdot = P_VAR - D_VAR*V;
* ``B(m) = dA(j)/dV(s)``: ``RCT(j)``, ``RCT(j)*V(other)`` or ``RCT(j)*2*V(s)``;
* ``JVS(k) = Jac(i,s)`` = signed sum of ``c*B(m)`` over the reactions in
  which s is a reactant, in reaction order; structural fill-in entries are 0.

The species are renumbered by a greedy Markowitz ordering of the Jacobian
pattern (symmetric pivoting on the diagonal, as KPP's fixed-pattern LU
requires), and the LU pattern is the symbolic factorisation in that order.
"""
from __future__ import annotations

import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def _draw_reactions(rng, nspec, nreact):
    reacts = []
    for _ in range(nreact):
        nr = 1 if rng.random() < 0.35 else 2
        r = [int(x) for x in rng.choice(nspec, nr, replace=(nr == 2 and rng.random() < 0.05))]
        pool = [s for s in range(nspec) if s not in r]
        npd = int(rng.integers(1, 4))
        prods = [int(x) for x in rng.choice(pool, npd, replace=False)]
        mult = {p: (2 if rng.random() < 0.1 else 1) for p in prods}
        reacts.append((sorted(r), prods, mult))
    return reacts


def _markowitz(nspec, pattern):
    """Greedy Markowitz order for symmetric diagonal pivoting on a pattern
    given as set of (row, col); returns the elimination order."""
    rows = {i: {c for (r, c) in pattern if r == i} | {i} for i in range(nspec)}
    cols = {j: {r for (r, c) in pattern if c == j} | {j} for j in range(nspec)}
    left = set(range(nspec))
    order = []
    while left:
        best = min(left, key=lambda p: ((len(rows[p] & left) - 1) * (len(cols[p] & left) - 1), p))
        order.append(best)
        left.discard(best)
        rr = [r for r in cols[best] if r in left]
        cc = [c for c in rows[best] if c in left]
        for r in rr:            # fill-in of eliminating `best`
            for c in cc:
                rows[r].add(c)
                cols[c].add(r)
    return order


def generate(seed: int = 20240, nspec: int = 120, nreact: int = 360) -> dict:
    rng = np.random.default_rng(seed)
    reacts = _draw_reactions(rng, nspec, nreact)
    # Jacobian pattern in the original numbering
    pat = set()
    for r, prods, mult in reacts:
        for s in set(r):
            for t in set(r):
                pat.add((t, s))
            for p in prods:
                pat.add((p, s))
    order = _markowitz(nspec, pat)
    new = {old: k for k, old in enumerate(order)}
    reacts = [([new[x] for x in sorted(r)], [new[p] for p in prods],
               {new[p]: m for p, m in mult.items()}) for r, prods, mult in reacts]
    for i, (r, prods, mult) in enumerate(reacts):
        reacts[i] = (sorted(r), prods, mult)

    V = lambda i: ["v", i]
    K = lambda j: ["k", j]
    A = lambda j: ["a", j]
    num = lambda x: ["n", str(x)]

    def prod(*fs):
        e = fs[0]
        for f in fs[1:]:
            e = ["*", e, f]
        return e

    rates, P, D = [], [[] for _ in range(nspec)], [[] for _ in range(nspec)]
    for j, (r, prods, mult) in enumerate(reacts):
        rates.append(prod(K(j), *[V(x) for x in r]))
        for p in prods:
            P[p].append(A(j) if mult[p] == 1 else prod(num(mult[p]), A(j)))
        if len(r) == 1:
            D[r[0]].append(K(j))
        elif r[0] == r[1]:
            D[r[0]].append(prod(K(j), num(2), V(r[0])))
        else:
            D[r[0]].append(prod(K(j), V(r[1])))
            D[r[1]].append(prod(K(j), V(r[0])))

    def plain_sum(ts):
        if not ts:
            return num(0)
        e = ts[0]
        for t in ts[1:]:
            e = ["+", e, t]
        return e

    # Jacobian partials and entries
    jac_b, contrib = [], {}
    for j, (r, prods, mult) in enumerate(reacts):
        for s in sorted(set(r)):
            m = len(jac_b)
            if len(r) == 1:
                b = K(j)
            elif r[0] == r[1]:
                b = prod(K(j), num(2), V(s))
            else:
                other = r[1] if s == r[0] else r[0]
                b = prod(K(j), V(other))
            jac_b.append([m, b])
            # reactant loss: -B per reactant removed (a self reaction removes
            # two X per event and its B = 2kX is dA/dX, so it counts -2*B)
            c = 2 if (len(r) == 2 and r[0] == r[1]) else 1
            for t in sorted(set(r)):
                contrib.setdefault((t, s), []).append(("-", c, m))
            for p in prods:
                contrib.setdefault((p, s), []).append(("+", mult[p], m))

    # symbolic LU pattern in the Markowitz order (already renumbered)
    struct = {(i, s) for (i, s) in contrib} | {(i, i) for i in range(nspec)}
    rows = [set(c for (r, c) in struct if r == i) for i in range(nspec)]
    # row-wise fill: eliminating row k with pivots j<k adds U row j's columns
    for k in range(nspec):
        changed = True
        while changed:
            changed = False
            for j in sorted(c for c in rows[k] if c < k):
                extra = {c for c in rows[j] if c > j} - rows[k]
                if extra:
                    rows[k] |= extra
                    changed = True
    irow, icol = [], []
    for i in range(nspec):
        for c in sorted(rows[i]):
            irow.append(i)
            icol.append(c)
    jvs = []
    for i, c in zip(irow, icol):
        terms = contrib.get((i, c), [])
        if not terms:
            jvs.append(num(0))
            continue
        e = None
        for sign, coef, m in terms:
            t = ["b", m] if coef == 1 else prod(num(coef), ["b", m])
            if e is None:
                e = ["neg", t] if sign == "-" else t
            else:
                e = [sign, e, t]
        jvs.append(e)

    stoich = []
    for j, (r, prods, mult) in enumerate(reacts):
        net = {}
        for p in prods:
            net[p] = net.get(p, 0) + mult[p]
        for x in r:
            net[x] = net.get(x, 0) - 1
        for i in sorted(net):
            if net[i] != 0:
                stoich.append([i, j, str(net[i])])
    stoich.sort()

    return {
        "name": "synth120",
        "source": {"generator": f"mechanism/synthetic.py seed={seed}"},
        "nvar": nspec, "nfix": 0, "nreact": nreact, "nnz": len(irow), "nb": len(jac_b),
        "lu_irow": irow, "lu_icol": icol,
        "rates": rates,
        "prod": [plain_sum(t) for t in P],
        "dest": [plain_sum(t) for t in D],
        "jac_b": jac_b,
        "jvs": jvs,
        "solve": [],
        "stoich": stoich,
    }


def main():
    mech = generate()
    out = os.path.join(HERE, "synth120.json")
    with open(out, "w") as fh:
        json.dump(mech, fh, separators=(",", ":"))
    print(f"wrote {out}: NVAR={mech['nvar']} NREACT={mech['nreact']} NNZ={mech['nnz']} "
          f"NB={mech['nb']}")


if __name__ == "__main__":
    main()
