"""ctypes binding of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs load
this module; the product path never does.  The oracle restates the
reference's Rodas3 batch solve (see rodas3_oracle.cpp for the citations).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIBS: dict = {}


def lib_path(mech: str = "fullchem", pow_: str = "gc") -> str:
    """pow_="gc": the oracle proper (the project's correctly rounded pow, as
    in the kernels); "libm": the host C library's pow at the step-size
    factor, the function the reference's CPU build calls there."""
    tail = "_libmpow" if pow_ == "libm" else ""
    return os.path.join(HERE, "_build", f"liboracle_{mech}{tail}.so")


def load(mech: str = "fullchem", pow_: str = "gc"):
    key = mech if pow_ == "gc" else (mech, pow_)
    if key in _LIBS:
        return _LIBS[key]
    path = lib_path(mech, pow_)
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is not built (run __graft_entry__.build())")
    lib = ctypes.CDLL(path)
    vp, ci, cd = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
    lib.oracle_integrate_batch.argtypes = [ci, cd, cd] + [vp] * 10 + [ci]
    lib.oracle_integrate_batch.restype = None
    lib.oracle_fun.argtypes = [vp] * 4
    lib.oracle_jac.argtypes = [vp] * 4
    lib.oracle_decomp.argtypes = [vp]
    lib.oracle_decomp.restype = ci
    lib.oracle_solve.argtypes = [vp, vp]
    lib.oracle_pow.argtypes = [cd, cd]
    lib.oracle_pow.restype = cd
    lib.oracle_lu_tables.argtypes = [vp, vp, vp]
    lib.oracle_integrate_frozen.argtypes = [vp, vp, vp, vp, ci, vp]
    lib.oracle_integrate_frozen.restype = ci
    sizes = [ci() for _ in range(4)]
    lib.oracle_sizes(*[ctypes.byref(x) for x in sizes])
    lib.sizes = tuple(x.value for x in sizes)   # NVAR, NFIX, NREACT, NNZ
    _LIBS[key] = lib
    return lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def integrate_batch(batch, perm=None, nthreads: int = 0, mech: str = "fullchem",
                    pow_: str = "gc"):
    """Solve a workloads.Batch on the host; returns (C, ISTAT, RSTAT, IERR)
    in the Fortran layouts of gc_gpu_integrate_batch."""
    lib = load(mech, pow_)
    n = batch.n
    C = np.array(batch.C, order="F", copy=True)
    R = np.asfortranarray(batch.RCONST)
    IC = np.asfortranarray(batch.ICNTRL, dtype=np.int32)
    RC = np.asfortranarray(batch.RCNTRL)
    perm = np.arange(1, n + 1, dtype=np.int32) if perm is None else \
        np.ascontiguousarray(perm, dtype=np.int32)
    ist = np.zeros((8, n), np.int32, order="F")
    rst = np.zeros((3, n), np.float64, order="F")
    ierr = np.zeros(n, np.int32)
    atol = np.ascontiguousarray(batch.ATOL)
    rtol = np.ascontiguousarray(batch.RTOL)
    lib.oracle_integrate_batch(n, batch.Tstart, batch.Tend, _p(C), _p(R), _p(atol),
                               _p(rtol), _p(IC), _p(RC), _p(perm), _p(ist), _p(rst),
                               _p(ierr), int(nthreads))
    return C, ist, rst, ierr


def fun(V, F, RCT, mech="fullchem"):
    lib = load(mech)
    out = np.zeros(lib.sizes[0])
    lib.oracle_fun(_p(np.ascontiguousarray(V, dtype=np.float64)),
                   _p(np.ascontiguousarray(F, dtype=np.float64)),
                   _p(np.ascontiguousarray(RCT, dtype=np.float64)), _p(out))
    return out


def jac(V, F, RCT, mech="fullchem"):
    lib = load(mech)
    out = np.zeros(lib.sizes[3])
    lib.oracle_jac(_p(np.ascontiguousarray(V, dtype=np.float64)),
                   _p(np.ascontiguousarray(F, dtype=np.float64)),
                   _p(np.ascontiguousarray(RCT, dtype=np.float64)), _p(out))
    return out


def decomp(JVS, mech="fullchem"):
    lib = load(mech)
    a = np.array(JVS, dtype=np.float64, copy=True)
    ier = lib.oracle_decomp(_p(a))
    return a, ier


def solve(LU, X, mech="fullchem"):
    lib = load(mech)
    x = np.array(X, dtype=np.float64, copy=True)
    lib.oracle_solve(_p(np.ascontiguousarray(LU, dtype=np.float64)), _p(x))
    return x


def gc_pow(x, y, mech="fullchem"):
    return load(mech).oracle_pow(float(x), float(y))


def lu_tables(mech="fullchem"):
    lib = load(mech)
    nvar, _, _, nnz = lib.sizes
    crow = np.zeros(nvar + 1, np.int32)
    diag = np.zeros(nvar, np.int32)
    icol = np.zeros(nnz, np.int32)
    lib.oracle_lu_tables(_p(crow), _p(diag), _p(icol))
    return crow, diag, icol


def gencheck(mech: str = "fullchem"):
    """The generated fused factorisation compiled for the host (gencheck.cpp)."""
    key = ("gencheck", mech)
    if key not in _LIBS:
        lib = ctypes.CDLL(os.path.join(HERE, "_build", f"libgencheck_{mech}.so"))
        lib.gencheck_prep_decomp.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double]
        lib.gencheck_prep_decomp.restype = ctypes.c_int
        lib.gencheck_prep_decomp_recip.argtypes = [ctypes.c_void_p] * 3 + [ctypes.c_double]
        lib.gencheck_prep_decomp_recip.restype = ctypes.c_int
        _LIBS[key] = lib
    return _LIBS[key]


def build(mech: str, gen_dir: str) -> str:
    """Compile liboracle_<mech>.so from the generated sources in gen_dir."""
    subprocess.run(["make", "-s", "-j2", "-C", HERE, f"MECH={mech}",
                    f"GEN={os.path.abspath(gen_dir)}"], check=True)
    return lib_path(mech)


def integrate_with_retry(batch, atol_r, rtol_r, nthreads: int = 0, mech: str = "fullchem"):
    """The model's GPU-mode retry protocol on the host
    (src/geos-chem/GeosCore/fullchem_mod.F90:2384-2520): solve; cells with
    IERR < 0 are reset to their pre-solve concentrations, RCNTRL(3) = 0, and
    solved again with the retry tolerances; ISTAT accumulates both attempts,
    RSTAT and IERR come from the second.  Returns (C, ISTAT, RSTAT, IERR,
    nfail_first, nfail_both)."""
    import copy
    C, ist, rst, ierr = integrate_batch(batch, nthreads=nthreads, mech=mech)
    fail = np.flatnonzero(ierr < 0)
    if fail.size == 0:
        return C, ist, rst, ierr, 0, 0
    sub = copy.copy(batch)
    sub.C = np.asfortranarray(batch.C[:, fail])
    sub.RCONST = np.asfortranarray(batch.RCONST[:, fail])
    sub.ICNTRL = np.asfortranarray(batch.ICNTRL[:, fail])
    sub.RCNTRL = np.array(batch.RCNTRL[:, fail], order="F")
    sub.RCNTRL[2, :] = 0.0
    sub.ATOL = np.ascontiguousarray(atol_r)
    sub.RTOL = np.ascontiguousarray(rtol_r)
    C2, ist2, rst2, ierr2 = integrate_batch(sub, nthreads=nthreads, mech=mech)
    C[:, fail] = C2
    ist[:, fail] += ist2
    rst[:, fail] = rst2
    ierr[fail] = ierr2
    return C, ist, rst, ierr, int(fail.size), int((ierr2 < 0).sum())


def integrate_frozen(y0, fix, rct, hs, mech="fullchem"):
    """Rodas3 over the given step sizes without error control (the map the
    adjoint differentiates); returns the final state."""
    lib = load(mech)
    out = np.zeros(lib.sizes[0])
    fix = np.ascontiguousarray(fix if len(fix) else np.zeros(1), dtype=np.float64)
    rc = lib.oracle_integrate_frozen(_p(np.ascontiguousarray(y0, dtype=np.float64)), _p(fix),
                                     _p(np.ascontiguousarray(rct, dtype=np.float64)),
                                     _p(np.ascontiguousarray(hs, dtype=np.float64)),
                                     int(len(hs)), _p(out))
    if rc != 0:
        raise RuntimeError(f"singular factorisation at step {rc}")
    return out
