"""Seeded synthetic chemistry states for the batched Rodas3 solve.

The reference's harvested KPP-Standalone cells, its species database and
its rate-law routines (gckpp_Rates / fullchem_RateLawFuncs) are not in the
reference checkout, so the solver inputs are synthesised here from a seed.
The arrays come out exactly as the model hands them to
``gc_gpu_integrate_batch`` (gpulib/src/gc_gpu_batch_api.F90:147-162):
Fortran column-major, one column per cell.

Surrogates (documented because the names are missing):

* Species identities are assigned by reaction-graph degree: the variable
  species consumed by the most reactions stands in for OH, the next for
  HO2, then O3, NO, NO2, CO, CH4 and H2O (``SURROGATE_ORDER``).
* Fixed species: the most used fixed index stands in for O2 (0.2095 M),
  the next for N2 (0.7808 M), the last for H2 (0.5e-6 M).
* RCONST comes from a per-reaction-class model keyed by the factor
  structure of each rate in Fun_SPLIT: first order (RCT*V, treated as the
  photolytic class for the day/night mask), second order (RCT*V*V, with a
  per-reaction Arrhenius temperature factor), third order (RCT*V*V*V),
  pseudo-first order with a fixed species (RCT*V*F) and zero order in the
  variables (RCT*F).  Every rate constant is drawn log-uniform inside a
  per-class range in molecule cm^-3 s^-1 units.

Cell states follow the plain small workload: T ~ U(190, 310) K, P
log-uniform 10-1013 hPa, air density from the ideal gas law, H2O vmr
log-uniform 1e-6 - 3e-2, species vmr log-uniform 1e-15 - 1e-6 with O3
1e-8 - 1e-5, CO 5e-8 - 3e-7, CH4 1.8e-6; half the cells at night (all
photolysis zero), the rest with photolysis scaled by U(0,1)*cos(SZA).
The grid workloads build the same quantities on a (lon, lat, lev) grid with
a lapse-rate temperature profile, a hypsometric pressure profile, a
day/night split by longitude and stratospheric O3.
"""
from __future__ import annotations

import json
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
KB = 1.380649e-23           # J/K
SURROGATE_ORDER = ("OH", "HO2", "O3", "NO", "NO2", "CO", "CH4", "H2O")
FIXED_ORDER = (("O2", 0.2095), ("N2", 0.7808), ("H2", 0.5e-6))

# model defaults: fullchem_mod.F90:5244-5250
ATOL_DEFAULT = 1.0e-2
RTOL_DEFAULT = 0.5e-2


def _factors(e, out):
    if e[0] == "*":
        _factors(e[1], out)
        _factors(e[2], out)
    else:
        out.append(e)
    return out


@dataclass
class MechanismInfo:
    name: str
    nvar: int
    nfix: int
    nreact: int
    nnz: int
    klass: np.ndarray        # per reaction: 0 none/literal, 1 first, 2 second, 3 third, 4 V*F, 5 F only
    species: dict            # surrogate name -> variable index (0-based)
    fixed: list              # per fixed index: (name, fraction of M)


def mechanism_info(mech_json: str = "fullchem") -> MechanismInfo:
    path = mech_json if mech_json.endswith(".json") else \
        os.path.join(HERE, "mechanism", f"{mech_json}.json")
    with open(path) as fh:
        m = json.load(fh)
    nvar, nfix, nreact = m["nvar"], m["nfix"], m["nreact"]
    klass = np.zeros(nreact, np.int8)
    consumed = np.zeros(nvar, np.int64)
    fuse = np.zeros(max(nfix, 1), np.int64)
    for j, e in enumerate(m["rates"]):
        fs = _factors(e, [])
        kinds = sorted(f[0] for f in fs)
        nv = kinds.count("v")
        nf = kinds.count("f")
        for f in fs:
            if f[0] == "v":
                consumed[f[1]] += 1
            elif f[0] == "f":
                fuse[f[1]] += 1
        if "k" not in kinds:
            klass[j] = 0
        elif nf == 1 and nv == 0:
            klass[j] = 5
        elif nf >= 1:
            klass[j] = 4
        else:
            klass[j] = {0: 5, 1: 1, 2: 2}.get(nv, 3)
    order = sorted(range(nvar), key=lambda i: (-consumed[i], i))
    species = {name: order[r] for r, name in enumerate(SURROGATE_ORDER)
               if r < nvar}
    forder = sorted(range(nfix), key=lambda i: (-fuse[i], i))
    fixed = [None] * nfix
    for r, i in enumerate(forder):
        fixed[i] = FIXED_ORDER[r % len(FIXED_ORDER)]
    return MechanismInfo(m.get("name", "mech"), nvar, nfix, nreact, m["nnz"],
                         klass, species, fixed)


# per-class log10 ranges of the rate constant (molecule cm^-3 s^-1 units)
_K_RANGE = {1: (-6.0, -2.0),     # photolysis J at overhead sun, s^-1
            2: (-17.0, -10.0),   # bimolecular, cm^3 s^-1 at 298 K
            3: (-34.0, -31.0),   # termolecular, cm^6 s^-1
            4: (-17.0, -11.0),   # with a fixed species, cm^3 s^-1
            5: (-25.0, -20.0)}   # zero order in variables, cm^3 s^-1


@dataclass
class Batch:
    """One batch in the layout of gc_gpu_integrate_batch (Fortran order)."""
    C: np.ndarray        # (NSPEC, n) float64, F-contiguous
    RCONST: np.ndarray   # (NREACT, n)
    ATOL: np.ndarray     # (NVAR,)
    RTOL: np.ndarray     # (NVAR,)
    ICNTRL: np.ndarray   # (20, n) int32
    RCNTRL: np.ndarray   # (20, n)
    Tstart: float = 0.0
    Tend: float = 1200.0

    @property
    def n(self) -> int:
        return self.C.shape[1]


def _default_controls(n, rng, warm_h):
    ic = np.zeros((20, n), np.int32, order="F")
    ic[0, :] = 1      # autonomous
    ic[1, :] = 0      # vector tolerances
    ic[2, :] = 4      # Rodas3
    ic[6, :] = 1
    ic[14, :] = -1    # no Update_* calls
    rc = np.zeros((20, n), np.float64, order="F")
    if warm_h:
        rc[2, :] = 10.0 ** rng.uniform(1.0, np.log10(1200.0), n)
    return ic, rc


def _rate_constants(info: MechanismInfo, rng_mech, rng, T, jscale):
    """RCONST (NREACT, n) from the per-class model."""
    n = T.shape[0]
    k0 = np.zeros(info.nreact)
    ea = np.zeros(info.nreact)
    for c, (lo, hi) in _K_RANGE.items():
        sel = info.klass == c
        k0[sel] = 10.0 ** rng_mech.uniform(lo, hi, sel.sum())
    sel2 = info.klass == 2
    ea[sel2] = rng_mech.uniform(-500.0, 2000.0, sel2.sum())   # E/R in K
    # cells x reactions, C order == (NREACT, n) Fortran order; built in
    # chunks of cells with dense broadcasts (E/R is 0 outside the second-order
    # class, so its Arrhenius factor is 1 there)
    Rt = np.empty((n, info.nreact))
    sel1 = (info.klass == 1).astype(np.float32)[None, :]
    keep = (info.klass != 0).astype(np.float32)[None, :]
    mea = (-ea).astype(np.float32)[None, :]
    lo = np.float32(-0.1 * np.log(10.0))
    span = np.float32(0.2 * np.log(10.0))
    for c0 in range(0, n, 8192):
        c1 = min(n, c0 + 8192)
        invT = (1.0 / T[c0:c1] - 1.0 / 298.0).astype(np.float32)[:, None]
        # small per-cell jitter (10**U(-0.1, 0.1)) so no two cells share constants
        f = rng.random((c1 - c0, info.nreact), dtype=np.float32)
        f *= span
        f += lo
        f += mea * invT
        np.exp(f, out=f)
        f *= sel1 * (jscale[c0:c1, None].astype(np.float32) - 1.0) + 1.0
        f *= keep
        np.multiply(k0[None, :], f, out=Rt[c0:c1])
    return Rt.T


def _concentrations(info, rng, n, M, h2o_vmr, o3_vmr=None):
    NSPEC = info.nvar + info.nfix
    C = np.empty((NSPEC, n), order="F")
    vmr = 10.0 ** rng.uniform(-15.0, -6.0, (info.nvar, n))
    sp = info.species
    if "O3" in sp:
        vmr[sp["O3"]] = 10.0 ** rng.uniform(-8.0, -5.0, n) if o3_vmr is None else o3_vmr
    if "CO" in sp:
        vmr[sp["CO"]] = 10.0 ** rng.uniform(np.log10(5e-8), np.log10(3e-7), n)
    if "CH4" in sp:
        vmr[sp["CH4"]] = 1.8e-6
    if "H2O" in sp:
        vmr[sp["H2O"]] = h2o_vmr
    C[: info.nvar] = vmr * M[None, :]
    for i, (_, frac) in enumerate(info.fixed):
        C[info.nvar + i] = frac * M
    return C


def plain_small(n: int = 4096, seed: int = 0, mech: str = "fullchem",
                warm_h: bool = False) -> Batch:
    """Independent cells: the 4,096-cell plain workload (and, with n=65,536,
    the adjoint workload's states)."""
    info = mechanism_info(mech)
    rng_mech = np.random.default_rng(1234567)   # rate-constant table: fixed
    rng = np.random.default_rng(seed)
    T = rng.uniform(190.0, 310.0, n)
    P = 10.0 ** rng.uniform(np.log10(10.0), np.log10(1013.0), n) * 100.0  # Pa
    M = P / (KB * T) * 1e-6                       # molecule cm^-3
    h2o = 10.0 ** rng.uniform(-6.0, np.log10(3e-2), n)
    night = rng.uniform(size=n) < 0.5
    jscale = rng.uniform(size=n) * rng.uniform(size=n)   # U(0,1)*cos(SZA)
    jscale[night] = 0.0
    C = _concentrations(info, rng, n, M, h2o)
    R = _rate_constants(info, rng_mech, rng, T, jscale)
    ic, rc = _default_controls(n, rng, warm_h)
    return Batch(C, R, np.full(info.nvar, ATOL_DEFAULT),
                 np.full(info.nvar, RTOL_DEFAULT), ic, rc)


def grid(nlon: int, nlat: int, nlev: int = 72, seed: int = 0,
         mech: str = "fullchem", warm_h: bool = False, subsolar_lon: float = 0.0) -> Batch:
    """Vertically structured grid: 72x46x72 (4x5) or 144x91x72 (2x2.5).

    Cells are ordered level-fastest within each column, columns by latitude
    then longitude (n = nlon*nlat*nlev).  ``subsolar_lon`` (degrees east)
    places the sun: the same seed with ``subsolar_lon = 5`` is the grid one
    1200 s chemistry step earlier (the Earth turns 5 degrees in 1200 s), which
    moves the day/night terminator and nothing else."""
    info = mechanism_info(mech)
    rng_mech = np.random.default_rng(1234567)
    rng = np.random.default_rng(seed)
    lon = (np.arange(nlon) + 0.5) / nlon * 360.0 - 180.0
    lat = (np.arange(nlat) + 0.5) / nlat * 180.0 - 90.0
    LON, LAT, LEV = np.meshgrid(lon, lat, np.arange(nlev), indexing="ij")
    LON, LAT, LEV = LON.ravel(), LAT.ravel(), LEV.ravel()
    n = LON.size
    ncol = nlon * nlat
    # column properties
    t_sfc = 300.0 - 40.0 * (np.abs(LAT) / 90.0) ** 1.5 + rng.uniform(-3, 3, ncol).repeat(nlev)
    z_trop = (16.0 - 4.0 * np.abs(LAT) / 90.0 + rng.uniform(-0.5, 0.5, ncol).repeat(nlev))
    z = 0.06 + 79.9 * (LEV / (nlev - 1)) ** 2.2             # level height, km
    T = np.where(z < z_trop, t_sfc - 6.5 * z, t_sfc - 6.5 * z_trop + 1.0 * (z - z_trop))
    T = np.clip(T, 185.0, 320.0)
    # hypsometric pressure with the column's mean temperature
    H = 29.3 * 0.5 * (t_sfc + T) / 1000.0                 # scale height, km
    P = 101325.0 * np.exp(-z / H)                         # Pa
    M = P / (KB * T) * 1e-6
    h2o = np.where(z < z_trop, 10.0 ** (np.log10(2e-2) - 4.0 * z / z_trop), 5e-6)
    h2o = np.clip(h2o * 10.0 ** rng.uniform(-0.3, 0.3, n), 1e-6, 3e-2)
    o3 = np.where(z < z_trop, 10.0 ** rng.uniform(-8.0, -7.0, n),
                  10.0 ** rng.uniform(-6.0, -5.0, n))
    coszen = np.clip(np.cos(np.radians(LAT)) * np.cos(np.radians(LON - subsolar_lon)), 0.0, 1.0)
    jscale = coszen * rng.uniform(0.5, 1.0, n)           # night: lon half with coszen=0
    C = _concentrations(info, rng, n, M, h2o, o3_vmr=o3)
    R = _rate_constants(info, rng_mech, rng, T, jscale)
    ic, rc = _default_controls(n, rng, warm_h)
    return Batch(C, R, np.full(info.nvar, ATOL_DEFAULT),
                 np.full(info.nvar, RTOL_DEFAULT), ic, rc)


def grid_4x5(seed: int = 0, **kw) -> Batch:
    return grid(72, 46, 72, seed=seed, **kw)


def grid_2x25(seed: int = 0, **kw) -> Batch:
    return grid(144, 91, 72, seed=seed, **kw)


def subset(b: Batch, idx) -> Batch:
    idx = np.asarray(idx)
    return Batch(np.asfortranarray(b.C[:, idx]), np.asfortranarray(b.RCONST[:, idx]),
                 b.ATOL.copy(), b.RTOL.copy(), np.asfortranarray(b.ICNTRL[:, idx]),
                 np.asfortranarray(b.RCNTRL[:, idx]), b.Tstart, b.Tend)


def synthetic_stiff(n: int = 262144, seed: int = 0, mech: str = "synth120",
                    atol: float = 1e-8, rtol: float = 1e-3) -> Batch:
    """Cells of the seeded synthetic stiff mechanism (mechanism/synthetic.py):
    rate constants log-uniform 1e-20 .. 1e4 (per reaction, in the normalised
    concentration units of the initial state, which is log-uniform in
    [1e-6, 1]), every cell's rates scaled by one log-uniform 1e-2 .. 1e2
    factor, so cells differ widely in stiffness and step count."""
    info = mechanism_info(mech)
    rng_mech = np.random.default_rng(7654321)
    rng = np.random.default_rng(seed)
    k0 = 10.0 ** rng_mech.uniform(-20.0, 4.0, info.nreact)
    scale = 10.0 ** rng.uniform(-2.0, 2.0, n)
    jit = 10.0 ** rng.uniform(-0.05, 0.05, (n, info.nreact))
    Rt = k0[None, :] * scale[:, None] * jit
    Ct = 10.0 ** rng.uniform(-6.0, 0.0, (n, info.nvar + info.nfix))
    ic, rc = _default_controls(n, rng, False)
    return Batch(Ct.T, Rt.T, np.full(info.nvar, atol), np.full(info.nvar, rtol), ic, rc)
