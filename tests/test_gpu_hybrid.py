"""One hybrid CPU/GPU chemistry step through gcchem_b200_hybrid_step: the
GPU head, launched from the scheduler's device thread through the legacy
entry, and the tail, solved by the caller's CPU integrator callback (here
the oracle, standing in for the model's stock CPU solve), together give
every cell the oracle's result; the measured times update the rates and the
next step's GPU share."""
import numpy as np
import pytest

pytestmark = [pytest.mark.gpu, pytest.mark.timeout(600)]


def _bits(a):
    return np.ascontiguousarray(a).view(np.uint64 if a.dtype == np.float64 else np.uint32)


def test_hybrid_step_matches_oracle(pkg, orc):
    wl = pkg.workloads
    b = wl.plain_small(400, seed=61)
    b.ICNTRL[3, :] = 5000
    rC, rist, rrst, rierr = orc.integrate_batch(b)
    # cost order from the (here: same) previous step's counts, stable descending
    order = np.argsort(-rist[2].astype(np.int64), kind="stable")
    cb = wl.subset(b, order)
    prev = rist[2][order]
    s = pkg.solver("fullchem", "nofma")
    s.set_launch(pkg.PERSISTENT)
    h = pkg.Hybrid(s, ndev=1, frac=0.6)
    seen = []

    def cpu_tail(first, count, C, ist, rst, ierr):
        seen.append((first, count))
        sub = wl.subset(cb, np.arange(first, first + count))
        tc, ti, tr, te = orc.integrate_batch(sub)
        C[:, first:first + count] = tc
        ist[:, first:first + count] = ti
        rst[:, first:first + count] = tr
        ierr[first:first + count] = te

    for step in range(2):
        st = h.state()
        frac = st["frac"]
        if st["rate_gpu"] > 0 and st["rate_cpu"] > 0:     # the share the step will use
            frac = min(max(st["rate_gpu"] / (st["rate_gpu"] + st["rate_cpu"]), 0.01), 0.99)
        ng_plan, _ = pkg.Hybrid(s, ndev=1, frac=frac, fixed=True).plan(prev)
        C, ist, rst, ierr, info = h.step(cb, prev, cpu_tail)
        assert info["n_gpu"] == ng_plan and 0 < info["n_gpu"] < b.n, info
        assert seen[-1] == (info["n_gpu"], b.n - info["n_gpu"])
        assert np.array_equal(ierr, rierr[order])
        assert np.array_equal(ist, rist[:, order])
        assert np.array_equal(_bits(rst), _bits(rrst[:, order]))
        assert np.array_equal(_bits(C), _bits(rC[:, order]))
        st = h.state()
        assert st["rate_gpu"] > 0 and st["rate_cpu"] > 0 and st["dev_rate"][0] > 0
    # after the first step the share follows the measured rates
    assert 0.01 <= st["frac"] <= 0.99
