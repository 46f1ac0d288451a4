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
    """Two calls in a row give exactly what gcchem_b200_integrate_device gives
    with the same one-thread-per-cell kernel (bit for bit: same arithmetic,
    only the workspace differs), and the second call changes the device's
    free memory by nothing."""
    import torch
    s = pkg.solver("fullchem", "fma")
    s.set_launch(pkg.PLAIN)
    n = 200
    t = _device_batch(pkg, n, seed=21)
    ref = _outputs(n)
    Cref = t["C"].clone()
    s.integrate_device(Cref, t["RCONST"], t["ATOL"], t["RTOL"], t["ICNTRL"], t["RCNTRL"],
                       t["order"], ref["ISTAT"], ref["RSTAT"], ref["IERR"])
    torch.cuda.synchronize()
    s.set_launch(pkg.PERSISTENT)
    assert (ref["IERR"] == 1).all()
    outs = [_outputs(n) for _ in range(2)]
    Cs = [t["C"].clone() for _ in range(2)]
    free = []
    for call in range(2):   # the shared workspace keeps the previous call's contents
        out, C = outs[call], Cs[call]
        if call == 1:
            s.release()                 # the pooled entry points' buffers are gone
            torch.cuda.synchronize()
            free.append(torch.cuda.mem_get_info()[0])
        rc = s.integrate_device_noalloc(C, t["RCONST"], t["ATOL"], t["RTOL"], t["ICNTRL"],
                                        t["RCNTRL"], t["order"], out["ISTAT"], out["RSTAT"],
                                        out["IERR"])
        torch.cuda.synchronize()
        assert rc == 0, (call, rc)
        if call == 1:
            free.append(torch.cuda.mem_get_info()[0])
        assert torch.equal(out["IERR"], ref["IERR"]), call
        assert torch.equal(out["ISTAT"], ref["ISTAT"]), call
        assert torch.equal(out["RSTAT"], ref["RSTAT"]), call
        assert torch.equal(C, Cref), call
    assert free[0] == free[1], free


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
