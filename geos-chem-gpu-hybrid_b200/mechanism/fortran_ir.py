"""Order-preserving reader for KPP-generated Fortran kernels.

KPP writes each mechanism kernel as straight-line Fortran assignments:

* ``Fun_SPLIT``  (src/geos-chem/KPP/fullchem/gckpp_Function.F90:2170-5060):
  ``A(j) = RCT(j)*V(a)*V(b)``, ``P_VAR(i) = ... + 0.27*A(j) + ...``,
  ``D_VAR(i) = RCT(j)*V(a) + ...`` and ``Vdot = P_VAR - D_VAR*V``.
* ``Jac_SP``     (src/geos-chem/KPP/fullchem/gckpp_Jacobian.F90:47-20887):
  ``B(k) = RCT(j)*V(a)`` partials followed by ``JVS(k) = -B(m)+0.5*B(n)``,
  each JVS assignment preceded by the comment ``! JVS(k) = Jac_FULL(i,j)``.
* ``KppSolve``   (src/geos-chem/KPP/fullchem/gckpp_LinearAlgebra.F90:645-2311):
  ``X(i) = X(i)-JVS(p)*X(c)`` forward sweep and
  ``X(i) = (X(i)-JVS(p)*X(c))/(JVS(d))`` backward sweep.

The reference library is built with ``-fdefault-real-8`` (KPP CMakeLists.txt
lines 87-92), so every real literal is a REAL(8) value converted directly
from its decimal text, and integer literals such as ``2`` are converted to
REAL(8) before they multiply.  Without ``-ffast-math`` gfortran evaluates
each expression in the Fortran association order: ``*`` and ``/`` are left
associative, binary ``+``/``-`` are left associative, and a leading unary
minus applies to the first multiplication operand chain only
(``-a*b-c`` is ``(-(a*b))-c``).  The parser below builds exactly that tree,
so code emitted from it (C++ for the oracle, CUDA for the kernels) rounds
every intermediate the same way the reference does.

AST nodes are nested lists (JSON friendly, 0-based indices):

    ["n", "0.44"]      numeric literal (text kept verbatim)
    ["v", i]           V(i+1)       variable species
    ["f", i]           F(i+1)       fixed species
    ["k", j]           RCT(j+1)     rate constant
    ["a", j]           A(j+1)       reaction rate (Fun_SPLIT temporaries)
    ["b", k]           B(k+1)       Jacobian partials (Jac_SP temporaries)
    ["x", i]           X(i+1)       solve vector
    ["j", p]           JVS(p+1)     sparse matrix entry
    ["neg", e]         unary minus
    ["+", l, r] ["-", l, r] ["*", l, r] ["/", l, r]
"""
from __future__ import annotations

import re
from typing import Iterator

_REF_KIND = {"V": "v", "F": "f", "RCT": "k", "A": "a", "B": "b", "X": "x",
             "JVS": "j"}

_TOKEN = re.compile(
    r"\s*(?:(?P<ref>[A-Za-z_][A-Za-z_0-9]*)\((?P<idx>\d+)\)"
    r"|(?P<num>\d+\.\d*(?:[eEdD][-+]?\d+)?|\.\d+(?:[eEdD][-+]?\d+)?"
    r"|\d+[eEdD][-+]?\d+|\d+)"
    r"|(?P<op>[-+*/()]))")


def tokenize(text: str) -> list[tuple[str, object]]:
    out: list[tuple[str, object]] = []
    pos = 0
    text = text.rstrip()
    while pos < len(text):
        m = _TOKEN.match(text, pos)
        if m is None or m.end() == pos:
            raise ValueError(f"cannot tokenise {text[pos:pos + 40]!r}")
        pos = m.end()
        if m.group("ref"):
            name = m.group("ref")
            if name not in _REF_KIND:
                raise ValueError(f"unknown array {name} in {text!r}")
            out.append(("ref", (_REF_KIND[name], int(m.group("idx")) - 1)))
        elif m.group("num"):
            out.append(("num", m.group("num")))
        else:
            out.append(("op", m.group("op")))
    return out


class _Parser:
    """Fortran level-2 expression grammar restricted to + - * / and ()."""

    def __init__(self, toks):
        self.t = toks
        self.i = 0

    def peek(self):
        return self.t[self.i] if self.i < len(self.t) else (None, None)

    def take(self):
        tok = self.t[self.i]
        self.i += 1
        return tok

    def expr(self):
        # level-2-expr: [sign] add-operand { add-op add-operand }
        kind, val = self.peek()
        if kind == "op" and val in "+-":
            self.take()
            node = self.term()
            if val == "-":
                node = ["neg", node]
        else:
            node = self.term()
        while True:
            kind, val = self.peek()
            if kind == "op" and val in "+-":
                self.take()
                node = [val, node, self.term()]
            else:
                return node

    def term(self):
        node = self.primary()
        while True:
            kind, val = self.peek()
            if kind == "op" and val in "*/":
                self.take()
                node = [val, node, self.primary()]
            else:
                return node

    def primary(self):
        kind, val = self.take()
        if kind == "ref":
            return [val[0], val[1]]
        if kind == "num":
            return ["n", val]
        if kind == "op" and val == "(":
            node = self.expr()
            k2, v2 = self.take()
            if (k2, v2) != ("op", ")"):
                raise ValueError("unbalanced parentheses")
            return node
        raise ValueError(f"unexpected token {kind} {val}")


def parse_expr(text: str):
    p = _Parser(tokenize(text))
    node = p.expr()
    if p.i != len(p.t):
        raise ValueError(f"trailing tokens in {text!r}")
    return node


def statements(lines: list[str]) -> Iterator[tuple[str, str]]:
    """Join Fortran continuation lines; yield (kind, text).

    kind is "comment" for a full-line comment (text without the "!"),
    "stmt" for an executable or declaration statement.  A comment that sits
    between an ``IF (...) &`` line and its continuation (the ``Jac_SP``
    layout) is yielded before the joined statement.
    """
    cur = ""
    for raw in lines:
        s = raw.strip()
        if not s:
            continue
        if s.startswith("!"):
            yield "comment", s[1:].strip()
            continue
        if s.startswith("&"):
            s = s[1:]
        if s.endswith("&"):
            cur += s[:-1]
            continue
        cur += s
        yield "stmt", cur.strip()
        cur = ""
    if cur:
        yield "stmt", cur.strip()


_GUARD = re.compile(r"^IF\s*\(\s*DO_\w+\(\d+\)\s*\)\s*")
_ASSIGN = re.compile(r"^(?P<lhs>[A-Za-z_]+)\((?P<idx>\d+)\)\s*=\s*(?P<rhs>.+)$")
_JACFULL = re.compile(r"JVS\((\d+)\)\s*=\s*Jac_FULL\((\d+),(\d+)\)")


def assignments(lines: list[str]):
    """Yield (lhs_name, lhs_index0, ast, last_comment) for every indexed
    assignment; the constant ``DO_FUN``/``DO_JVS``/``DO_SLV`` guards (all
    ``.TRUE.`` PARAMETERs or SAVE variables that are never changed on the
    batched path) are dropped."""
    last_comment = None
    for kind, text in statements(lines):
        if kind == "comment":
            last_comment = text
            continue
        text = _GUARD.sub("", text)
        m = _ASSIGN.match(text)
        if not m:
            continue
        yield (m.group("lhs"), int(m.group("idx")) - 1,
               parse_expr(m.group("rhs")), last_comment)
        last_comment = None


def jac_full_position(comment: str | None):
    if not comment:
        return None
    m = _JACFULL.search(comment)
    if not m:
        return None
    return int(m.group(1)) - 1, int(m.group(2)) - 1, int(m.group(3)) - 1
