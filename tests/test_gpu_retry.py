"""Device-side retry protocol (gcchem_b200_integrate_device_retry) against the
model's host protocol restated on the oracle (fullchem_mod.F90:2436-2520).

Failures are produced on the host, by the inputs: a tight first-attempt RTOL
and a small ICNTRL(4) make some cells exceed the step limit (IERR = -6); the
retry runs with the model's default tolerances and Hstart = 0.  Every kernel
runs the retry in the lane that saw the failure, inside the one launch."""
import numpy as np
import pytest

pytestmark = [pytest.mark.gpu, pytest.mark.timeout(300)]


def _to_dev(pkg, b):
    import torch
    dev = torch.device("cuda:0")

    def up(a, dt):
        return torch.from_numpy(np.ascontiguousarray(a.T if a.ndim == 2 else a)).to(dev, dt)

    return dict(C=up(b.C, torch.float64), RCONST=up(b.RCONST, torch.float64),
                ATOL=up(b.ATOL, torch.float64), RTOL=up(b.RTOL, torch.float64),
                ICNTRL=up(b.ICNTRL, torch.int32), RCNTRL=up(b.RCNTRL, torch.float64))


@pytest.mark.parametrize("max_steps,rtol,want_both", [(140, 2e-3, 0), (120, 3e-3, 7)])
@pytest.mark.parametrize("mode", [0, 1, 2, 3], ids=["plain", "persistent", "plain_fused", "coop"])
def test_retry_bitexact(pkg, orc, max_steps, rtol, want_both, mode):
    import torch
    b = pkg.workloads.plain_small(64, seed=31, warm_h=True)
    b.ICNTRL[3, :] = max_steps
    b.RTOL[:] = rtol
    atol_r = np.full(b.ATOL.shape, 1e-2)
    rtol_r = np.full(b.RTOL.shape, 0.5e-2)
    rC, rist, rrst, rierr, nf1, nf2 = orc.integrate_with_retry(b, atol_r, rtol_r)
    assert nf1 > 0 and nf2 == want_both

    s = pkg.solver("fullchem", "nofma")
    s.set_launch(mode)
    t = _to_dev(pkg, b)
    n = b.n
    dev = t["C"].device
    ist = torch.zeros((n, 8), dtype=torch.int32, device=dev)
    rst = torch.zeros((n, 3), dtype=torch.float64, device=dev)
    ierr = torch.zeros(n, dtype=torch.int32, device=dev)
    nfail = torch.zeros(2, dtype=torch.int32, device=dev)
    order = s.cost_order(torch.full((n,), 5, dtype=torch.int32, device=dev))
    s.integrate_device_retry(t["C"], t["RCONST"], t["ATOL"], t["RTOL"],
                             torch.from_numpy(atol_r).to(dev), torch.from_numpy(rtol_r).to(dev),
                             t["ICNTRL"], t["RCNTRL"], order, ist, rst, ierr, nfail)
    torch.cuda.synchronize()
    s.set_launch(1)
    assert nfail.tolist() == [nf1, nf2]
    assert np.array_equal(ierr.cpu().numpy(), rierr)
    assert np.array_equal(ist.cpu().numpy().T, rist)
    assert np.array_equal(rst.cpu().numpy().T.view(np.uint64), rrst.view(np.uint64))
    assert np.array_equal(t["C"].cpu().numpy().T.view(np.uint64), rC.view(np.uint64))
