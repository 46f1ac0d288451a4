"""The device-resident chemistry step (gridstep.GridChemistry: device
BatchMap, gather, solve with retry, scatter) against the model's host path
restated here in numpy around the oracle: the pre-scan sort
(fullchem_mod.F90:906-993), the gather (:1538-1543) with the warm start
RCNTRL(3) = KPPHvalue, the GPU-mode retry
(:2436-2520) and the scatter with its clamp, KPPHvalue, PrevNsteps and
KppDiags (:2878-3000).  The --fmad=false library must reproduce it bit for
bit, over two consecutive steps (the second sorted by the first's counts),
eager and replayed from a CUDA graph."""
import importlib

import numpy as np
import pytest

pytestmark = [pytest.mark.gpu, pytest.mark.timeout(600)]

NX, NY, NZ = 7, 5, 6


def _bits(a):
    return np.ascontiguousarray(a).view(np.uint64 if a.dtype == np.float64 else np.uint32)


def _fields(pkg):
    """Grid fields: model species = KPP species in a shuffled numbering plus
    4 species KPP does not use; 3 KPP variable species are not model species
    (the gather gives them 0)."""
    nc = NX * NY * NZ
    b = pkg.workloads.plain_small(nc, seed=71)
    b.ICNTRL[3, :] = 5000
    nspec = b.C.shape[0]
    rng = np.random.default_rng(7)
    nspc = nspec + 4
    perm = rng.permutation(nspc)[:nspec] + 1               # KPP N -> model species
    kmap = perm.astype(np.int32)
    kmap[[5, 77, 200]] = 0
    conc = rng.uniform(1e3, 1e9, (nspc, nc))
    for n in range(nspec):
        if kmap[n] > 0:
            conc[kmap[n] - 1] = b.C[n]
    mask = np.ones(nc, np.int32)
    mask[rng.choice(nc, 9, replace=False)] = 0              # cells outside the chemistry grid
    return b, conc, kmap, mask


def _host_step(orc, b, conc, kmap, rgrid, prev, kpph, diag, mask, sort=True):
    nc = NX * NY * NZ
    keys = np.where(mask != 0, prev if sort else 0, np.iinfo(np.int32).min).astype(np.int64)
    order = np.argsort(-keys, kind="stable")[: int(mask.sum())]
    nspec = len(kmap)
    C = np.zeros((nspec, order.size), order="F")
    for n in range(nspec):
        if kmap[n] > 0:
            C[n] = conc[kmap[n] - 1, order]
    rc = np.zeros((20, order.size), order="F")
    rc[2] = kpph[order]                     # warm start: Hstart = KPPHvalue
    bb = importlib.import_module("geos-chem-gpu-hybrid_b200.workloads").Batch(
        C, np.asfortranarray(rgrid[:, order]), b.ATOL, b.RTOL,
        np.asfortranarray(b.ICNTRL[:, :order.size]), rc)
    C, ist, rst, ierr, _, _ = orc.integrate_with_retry(bb, b.ATOL, b.RTOL)
    for n in range(nspec):
        if kmap[n] > 0:
            conc[kmap[n] - 1, order] = np.maximum(C[n], 0.0)
    neg = np.zeros(order.size)
    for n in range(nspec):
        if kmap[n] > 0:
            neg += C[n] < 0.0
    kpph[order] = rst[2]
    prev[order] = ist[2]
    diag[:8, order] = ist.astype(np.float32)
    diag[8, order] = neg.astype(np.float32)
    return ierr


@pytest.mark.parametrize("graph", [False, True], ids=["eager", "graph"])
def test_gridstep_matches_host_path(pkg, orc, graph):
    import torch
    gs = importlib.import_module("geos-chem-gpu-hybrid_b200.gridstep")
    b, conc, kmap, mask = _fields(pkg)
    s = pkg.solver("fullchem", "nofma")
    s.set_launch(pkg.PERSISTENT)
    dev = torch.device("cuda:0")
    shape = (NZ, NY, NX)
    tconc = torch.from_numpy(conc.reshape(-1, *shape).copy()).to(dev)
    trg = torch.from_numpy(np.ascontiguousarray(b.RCONST).reshape(-1, *shape).copy()).to(dev)
    g = gs.GridChemistry(s, tconc, kmap, trg, b.ATOL, b.RTOL, icntrl=b.ICNTRL[:, 0],
                         in_chem=mask.reshape(shape))
    hconc = conc.copy()
    prev = np.zeros(NX * NY * NZ, np.int32)
    kpph = np.zeros(NX * NY * NZ)
    diag = np.zeros((9, NX * NY * NZ), np.float32)
    nsteps = 2
    if graph:
        g.step()                           # eager step: sizes the buffers
        torch.cuda.synchronize()
        _host_step(orc, b, hconc, kmap, b.RCONST, prev, kpph, diag, mask)
        g.capture(nsteps)
        g.replay()
    else:
        for _ in range(nsteps):
            g.step()
    torch.cuda.synchronize()
    for _ in range(nsteps):
        ierr = _host_step(orc, b, hconc, kmap, b.RCONST, prev, kpph, diag, mask)
        assert (ierr == 1).all()
    got = g.conc.cpu().numpy().reshape(hconc.shape)
    assert np.array_equal(_bits(got), _bits(hconc))
    assert np.array_equal(g.prev.cpu().numpy().ravel(), prev)
    assert np.array_equal(_bits(g.kpph.cpu().numpy().ravel()), _bits(kpph))
    assert np.array_equal(g.diag.cpu().numpy().reshape(9, -1), diag)
    # cells outside the chemistry grid are untouched
    out = np.flatnonzero(mask == 0)
    assert np.array_equal(_bits(got[:, out]), _bits(conc[:, out]))
