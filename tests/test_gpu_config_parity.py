"""Parity on the configurations that are benchmarked, through the C-ABI.

* The plain small workload at its stated size: 4,096 independent fullchem
  cells, stock solver settings (no step cap), one 1200 s step.
* Cells of the 4x5 grid workload (72x46x72) taken where its vertical
  structure makes the chemistry differ most: the stratosphere (high O3, low
  pressure), the levels around the tropopause, and the night side (every
  photolysis rate zero).

The --fmad=false library must match the oracle bit for bit in C, ISTAT,
RSTAT and IERR; the production library must keep every variable species
within 1e-6 relative of the oracle, with the denominator floored at ATOL
(1e-2 molecule cm^-3), with no solver failure.
"""
import numpy as np
import pytest

pytestmark = [pytest.mark.gpu, pytest.mark.timeout(600)]

RTOL_PARITY = 1e-6
FLOOR = 1e-2
MODES = [0, 1, 2, 3]
MODE_IDS = ["plain", "persistent", "plain_fused", "coop"]
NLON, NLAT, NLEV = 72, 46, 72


def _bits(a):
    return np.ascontiguousarray(a).view(np.uint64 if a.dtype == np.float64 else np.uint32)


def _strata_columns():
    """Grid columns (0-based) of three groups, strided over the globe:
    stratosphere (levels 40-71, day side), tropopause (levels 26-36) and
    night side (|longitude| > 90 deg, all levels)."""
    lon = (np.arange(NLON) + 0.5) / NLON * 360.0 - 180.0
    cells = []
    for ilon in range(0, NLON, 5):
        for ilat in range(1, NLAT, 7):
            base = (ilon * NLAT + ilat) * NLEV
            if abs(lon[ilon]) > 90.0:
                cells += [base + lev for lev in range(0, NLEV, 3)]
            else:
                cells += [base + lev for lev in range(40, NLEV, 2)]
                cells += [base + lev for lev in range(26, 37)]
    return np.array(sorted(set(cells)), np.int64)


@pytest.fixture(scope="module")
def config0(pkg):
    return pkg.workloads.plain_small(4096, seed=0)


@pytest.fixture(scope="module")
def config0_ref(orc, config0):
    return orc.integrate_batch(config0)


@pytest.fixture(scope="module")
def strata(pkg):
    g = pkg.workloads.grid_4x5(seed=0)
    idx = _strata_columns()
    return pkg.workloads.subset(g, idx)


@pytest.fixture(scope="module")
def strata_ref(orc, strata):
    return orc.integrate_batch(strata)


def _check_bitexact(s, batch, ref):
    C, ist, rst, ierr, *_ = s.integrate_batch(batch)
    rC, rist, rrst, rierr = ref
    assert np.array_equal(ierr, rierr)
    assert np.array_equal(ist, rist)
    assert np.array_equal(_bits(rst), _bits(rrst))
    assert np.array_equal(_bits(C), _bits(rC))


def _check_tolerance(s, batch, ref):
    C, ist, rst, ierr, *_ = s.integrate_batch(batch)
    rC, rist, rrst, rierr = ref
    assert (rierr == 1).all() and (ierr == 1).all()
    n = s.nvar
    rel = np.abs(C[:n] - rC[:n]) / np.maximum(np.abs(rC[:n]), FLOOR)
    assert rel.max() <= RTOL_PARITY, rel.max()
    assert np.isfinite(C).all()


@pytest.mark.parametrize("mode", MODES, ids=MODE_IDS)
def test_config0_4096_bitexact_nofma(pkg, config0, config0_ref, mode):
    s = pkg.solver("fullchem", "nofma")
    s.set_launch(mode)
    _check_bitexact(s, config0, config0_ref)
    s.set_launch(pkg.PERSISTENT)


@pytest.mark.parametrize("mode", MODES, ids=MODE_IDS)
def test_config0_4096_fma_tolerance(pkg, config0, config0_ref, mode):
    s = pkg.solver("fullchem", "fma")
    s.set_launch(mode)
    _check_tolerance(s, config0, config0_ref)
    s.set_launch(pkg.PERSISTENT)


def test_strata_selection_covers_the_profile(strata):
    """The grid sample holds a few thousand cells of the three groups."""
    idx = _strata_columns()
    lev = idx % NLEV
    ilon = idx // (NLAT * NLEV)
    night = np.abs((ilon + 0.5) / NLON * 360.0 - 180.0) > 90.0
    assert strata.n == idx.size and 2000 <= idx.size <= 4000
    assert (~night & (lev >= 40)).sum() > 500          # stratosphere, day side
    assert (~night & (lev >= 26) & (lev <= 36)).sum() > 300
    assert night.sum() > 700


@pytest.mark.parametrize("mode", MODES, ids=MODE_IDS)
def test_grid4x5_strata_bitexact_nofma(pkg, strata, strata_ref, mode):
    s = pkg.solver("fullchem", "nofma")
    s.set_launch(mode)
    _check_bitexact(s, strata, strata_ref)
    s.set_launch(pkg.PERSISTENT)


@pytest.mark.parametrize("mode", MODES, ids=MODE_IDS)
def test_grid4x5_strata_fma_tolerance(pkg, strata, strata_ref, mode):
    s = pkg.solver("fullchem", "fma")
    s.set_launch(mode)
    _check_tolerance(s, strata, strata_ref)
    s.set_launch(pkg.PERSISTENT)
