"""The hybrid CPU/GPU scheduler (gcchem_b200_hybrid_*) against a statement
by statement restatement of the model's GC_BATCH_CHEM=3 bookkeeping
(src/geos-chem/GeosCore/fullchem_mod.F90: work model and split :997-1019,
device slices :1020-1055, rate updates :2678-2706).  The plan and update
entry points make no CUDA call, so these run on the CPU; the whole step
with GPU launches is in test_gpu_hybrid.py."""
import numpy as np
import pytest


class RefHybrid:
    """The model's variables HybWorkFrac, HybRateGpu/Cpu, HybDevRate."""

    def __init__(self, ndev, frac, fixed):
        self.ndev, self.frac, self.fixed = ndev, frac, fixed
        self.rate_gpu = self.rate_cpu = 0.0
        self.dev_rate = [0.0] * ndev

    def plan(self, prev):
        n = len(prev)
        work = [0] * (n + 1)
        for ic in range(1, n + 1):
            work[ic] = work[ic - 1] + max(int(prev[ic - 1]), 1)
        wtot = float(work[n])
        if not self.fixed and self.rate_gpu > 0.0 and self.rate_cpu > 0.0:
            self.frac = self.rate_gpu / (self.rate_gpu + self.rate_cpu)
            self.frac = min(max(self.frac, 0.01), 0.99)
        self.frac = min(max(self.frac, 0.0), 1.0)
        target = self.frac * wtot
        ngpu = 0
        for ic in range(1, n + 1):
            if float(work[ic]) > target:
                break
            ngpu = ic
        nd = self.ndev
        if ngpu < nd:
            nd = max(ngpu, 1)
        w = [1.0] * nd
        if all(self.dev_rate[d] > 0.0 for d in range(nd)):
            w = self.dev_rate[:nd]
        wsum = sum(w)
        lo, hi = [1] * nd, [0] * nd
        idx, cum = 0, 0.0
        for d in range(nd):
            lo[d] = idx + 1
            if d == nd - 1:
                hi[d] = ngpu
            else:
                cum += w[d]
                t = float(work[ngpu]) * cum / wsum
                for ic in range(idx + 1, ngpu + 1):
                    if float(work[ic]) > t:
                        break
                    idx = ic
                hi[d] = idx
            idx = hi[d]
        self.work, self.n, self.ngpu, self.lo, self.hi = work, n, ngpu, lo, hi
        return ngpu, list(zip(lo, hi))

    def update(self, dev_tw, tcpu):
        def ema(old, new):
            return 0.5 * old + 0.5 * new if old > 0.0 else new
        gtw = 0.0
        for d in range(len(self.lo)):
            gtw = max(gtw, dev_tw[d])
            if self.hi[d] >= self.lo[d] and dev_tw[d] > 0.0:
                self.dev_rate[d] = ema(self.dev_rate[d],
                                       (self.work[self.hi[d]] - self.work[self.lo[d] - 1])
                                       / dev_tw[d])
        if self.ngpu > 0 and gtw > 0.0:
            self.rate_gpu = ema(self.rate_gpu, self.work[self.ngpu] / gtw)
        if self.n - self.ngpu > 0 and tcpu > 0.0:
            self.rate_cpu = ema(self.rate_cpu, (self.work[self.n] - self.work[self.ngpu]) / tcpu)


@pytest.fixture(scope="module")
def solver(pkg):
    return pkg.binding.Solver("fullchem", "fma")


@pytest.mark.parametrize("ndev,frac,fixed", [(1, 0.5, False), (4, 0.7, False), (8, 0.3, True),
                                             (3, 1.0, False), (2, 0.0, False)])
def test_plan_and_rates_follow_the_model(pkg, solver, ndev, frac, fixed):
    rng = np.random.default_rng(ndev)
    h = pkg.Hybrid(solver, ndev=ndev, frac=frac, fixed=fixed)
    ref = RefHybrid(ndev, frac, fixed)
    for step in range(6):
        n = int(rng.integers(1, 4000))
        prev = np.sort(rng.integers(0, 300, n))[::-1]        # cost order: descending
        prev[rng.random(n) < 0.05] = 0                       # first-step keys
        got = h.plan(prev)
        want = ref.plan(prev)
        assert got == want, step
        nd = len(want[1])
        tw = rng.uniform(0.1, 2.0, nd)
        tc = float(rng.uniform(0.1, 3.0))
        h.update(tw, tc)
        ref.update(tw, tc)
        st = h.state()
        assert st["frac"] == ref.frac
        assert st["rate_gpu"] == ref.rate_gpu and st["rate_cpu"] == ref.rate_cpu
        assert st["dev_rate"] == ref.dev_rate


def test_measured_rates_set_the_share(pkg, solver):
    """With a GPU 3x as fast as the host cores the head takes ~3/4 of the work."""
    h = pkg.Hybrid(solver, ndev=1, frac=0.5)
    prev = np.full(1000, 10)
    ng, slices = h.plan(prev)
    assert ng == 500 and slices == [(1, 500)]
    h.update([1.0], 3.0)          # GPU: 5000 work/s; CPU: 5000/3 work/s
    ng, _ = h.plan(prev)
    assert ng == 750


def test_slices_balance_weighted_work(pkg, solver):
    h = pkg.Hybrid(solver, ndev=2, frac=1.0, fixed=True)
    prev = np.full(100, 5)
    ng, slices = h.plan(prev)
    assert ng == 100 and slices == [(1, 50), (51, 100)]
    h.update([1.0, 3.0], 0.0)     # device 0 three times as fast per work unit
    ng, slices = h.plan(prev)
    assert slices == [(1, 75), (76, 100)]


def test_bad_settings_rejected(pkg, solver):
    with pytest.raises(ValueError):
        pkg.Hybrid(solver, ndev=0)
    with pytest.raises(ValueError):
        pkg.Hybrid(solver, ndev=1, frac=1.5)
