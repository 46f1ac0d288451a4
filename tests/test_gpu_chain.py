"""Consecutive chemistry steps on the device, eager and CUDA-graph captured,
against the same chain on the oracle (negatives clamped, Hnew warm start)."""
import numpy as np
import pytest

pytestmark = [pytest.mark.gpu, pytest.mark.timeout(300)]


def _oracle_chain(orc, b, nsteps):
    import copy
    b = copy.deepcopy(b)
    for _ in range(nsteps):
        C, ist, rst, ierr = orc.integrate_batch(b)
        b.C = np.asfortranarray(np.maximum(C, 0.0))
        b.RCNTRL = np.array(b.RCNTRL, order="F")
        b.RCNTRL[2, :] = rst[2, :]
    return b.C, ist, rst, ierr


def test_chain_eager_graph_oracle(pkg, orc):
    import torch
    from chain import Chain
    b = pkg.workloads.plain_small(96, seed=41)
    b.ICNTRL[3, :] = 5000
    s = pkg.solver("fullchem", "nofma")
    s.set_launch(pkg.PERSISTENT)
    nsteps = 3
    rC, rist, rrst, rierr = _oracle_chain(orc, b, nsteps)

    eager = Chain(s, b)
    for _ in range(nsteps):
        eager.step()
    torch.cuda.synchronize()
    assert np.array_equal(eager.C.cpu().numpy().T.view(np.uint64), rC.view(np.uint64))
    assert np.array_equal(eager.ISTAT.cpu().numpy().T, rist)
    assert np.array_equal(eager.RSTAT.cpu().numpy().T.view(np.uint64), rrst.view(np.uint64))

    graphed = Chain(s, b)
    graphed.step()                     # eager first step (setup), then 2 captured
    graphed.capture(nsteps - 1)
    graphed.replay()
    torch.cuda.synchronize()
    assert torch.equal(graphed.C, eager.C)
    assert torch.equal(graphed.ISTAT, eager.ISTAT)
    assert torch.equal(graphed.RSTAT, eager.RSTAT)
