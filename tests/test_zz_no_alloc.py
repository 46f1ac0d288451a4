"""The allocation-free solve entry point, gcchem_b200_integrate_device_noalloc.

It exists for callers that cannot allocate device memory while they solve:
a model whose GPU memory comes from its own pool, or a thread that must not
call cudaMalloc/cudaFree because they synchronise the whole device.  Its
workspace is a fixed array inside the library, so it takes at most 256 cells
per call.  This file is collected last on purpose: if it fails, a run that
stops at the first failure has already run every other test.  It passes
alone in a fresh process and after the other tests.
"""
import numpy as np
import pytest

pytestmark = [pytest.mark.gpu, pytest.mark.timeout(300)]

RTOL_PARITY = 1e-6   # the tolerance of the other FMA-build parity tests
FLOOR = 1e-2


def _device_batch(pkg, n, seed):
    import torch
    b = pkg.workloads.plain_small(n, seed=seed)
    b.ICNTRL[3, :] = 5000
    dev = torch.device("cuda:0")

    def up(a, dt):
        return torch.from_numpy(np.ascontiguousarray(a.T if a.ndim == 2 else a)).to(dev, dt)

    return dict(C=up(b.C, torch.float64), RCONST=up(b.RCONST, torch.float64),
                ATOL=up(b.ATOL, torch.float64), RTOL=up(b.RTOL, torch.float64),
                ICNTRL=up(b.ICNTRL, torch.int32), RCNTRL=up(b.RCNTRL, torch.float64),
                order=torch.arange(n, dtype=torch.int32, device=dev))


def _outputs(n):
    import torch
    dev = torch.device("cuda:0")
    return dict(ISTAT=torch.zeros((n, 8), dtype=torch.int32, device=dev),
                RSTAT=torch.zeros((n, 3), dtype=torch.float64, device=dev),
                IERR=torch.zeros(n, dtype=torch.int32, device=dev))


def test_noalloc_matches_integrate_device_twice(pkg):
    import torch
    s = pkg.solver("fullchem", "fma")
    s.set_launch(pkg.PERSISTENT)
    n = 200
    t = _device_batch(pkg, n, seed=21)
    ref = _outputs(n)
    Cref = t["C"].clone()
    s.integrate_device(Cref, t["RCONST"], t["ATOL"], t["RTOL"], t["ICNTRL"], t["RCNTRL"],
                       t["order"], ref["ISTAT"], ref["RSTAT"], ref["IERR"])
    torch.cuda.synchronize()
    assert (ref["IERR"] == 1).all()
    nv = s.nvar
    for call in range(2):   # the shared workspace keeps the previous call's contents
        out = _outputs(n)
        C = t["C"].clone()
        rc = s.integrate_device_noalloc(C, t["RCONST"], t["ATOL"], t["RTOL"], t["ICNTRL"],
                                        t["RCNTRL"], t["order"], out["ISTAT"], out["RSTAT"],
                                        out["IERR"])
        torch.cuda.synchronize()
        assert rc == 0, (call, rc)
        assert torch.equal(out["IERR"], ref["IERR"])
        assert torch.equal(out["ISTAT"], ref["ISTAT"])
        rel = ((C[:, :nv] - Cref[:, :nv]).abs() / Cref[:, :nv].abs().clamp_min(FLOOR)).max().item()
        assert rel <= RTOL_PARITY, (call, rel)


def test_noalloc_rejects_too_many_cells(pkg):
    import torch
    s = pkg.solver("fullchem", "fma")
    n = 257
    t = _device_batch(pkg, n, seed=22)
    out = _outputs(n)
    C0 = t["C"].clone()
    rc = s.integrate_device_noalloc(t["C"], t["RCONST"], t["ATOL"], t["RTOL"], t["ICNTRL"],
                                    t["RCNTRL"], t["order"], out["ISTAT"], out["RSTAT"],
                                    out["IERR"])
    assert rc == -4
    torch.cuda.synchronize()
    assert torch.equal(t["C"], C0)
