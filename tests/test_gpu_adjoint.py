"""Discrete adjoint on the GPU against the oracle.

1. The checkpoints of the forward solve are right: replaying the recorded
   step sizes with the oracle's frozen-step integrator reproduces the GPU's
   --fmad=false result bit for bit.
2. dL/dC0 and dL/d ln RCONST match FP64 central finite differences
   (h = 1e-6 relative) of that frozen-step CPU integrator to 1e-5 relative,
   on 64 cells of the adjoint workload's generator (and on 10 cells of the
   synthetic mechanism, whose factorisation is the indexed one), for every
   sampled component whose difference quotient is not swamped by rounding
   noise (the noise estimate is printed with any failure).
3. A cell without a gradient (more accepted steps than the checkpoint
   capacity) makes the backward pass raise, or, when asked, get a zero
   gradient and a flag."""
import importlib

import numpy as np
import pytest

pytestmark = [pytest.mark.gpu, pytest.mark.timeout(600)]

CKMAX = 400
# a difference quotient is compared only where it is at least this many times
# its rounding noise, i.e. known to 1e-6 relative: ten times finer than the
# 1e-5 tolerance of the comparison
FD_MARGIN = 1e6


def _setup(pkg, n, seed, variant, mech="fullchem"):
    import torch
    adj = importlib.import_module("geos-chem-gpu-hybrid_b200.adjoint")
    Controls, loss_weights = adj.Controls, adj.loss_weights
    if mech == "fullchem":
        b = pkg.workloads.plain_small(n, seed=seed)
    else:
        b = pkg.workloads.synthetic_stiff(n, seed=seed)
    s = pkg.solver(mech, variant)
    s.set_launch(pkg.PERSISTENT)
    dev = torch.device("cuda:0")
    ctl = Controls(b, dev)
    C0 = torch.from_numpy(np.ascontiguousarray(b.C.T)).to(dev)
    logk = torch.from_numpy(np.ascontiguousarray(np.log(np.maximum(b.RCONST.T, 1e-300)))).to(dev)
    w = loss_weights(n, s.nvar, seed=seed, mech=mech)
    return b, s, ctl, C0, logk, w


def _forward_ckpt(s, ctl, C0, R, ckmax=CKMAX):
    import torch
    n = ctl.n
    dev = C0.device
    C = C0.clone()
    IST = torch.zeros((n, 8), dtype=torch.int32, device=dev)
    RST = torch.zeros((n, 3), dtype=torch.float64, device=dev)
    IE = torch.zeros(n, dtype=torch.int32, device=dev)
    ck = torch.zeros(n * ckmax * (s.nvar + 1), dtype=torch.float64, device=dev)
    s.integrate_device_ckpt(C, R, ctl.ATOL, ctl.RTOL, ctl.ICNTRL, ctl.RCNTRL,
                            torch.arange(n, dtype=torch.int32, device=dev), IST, RST, IE, ck, ckmax)
    torch.cuda.synchronize()
    return C, IST.cpu().numpy(), IE.cpu().numpy(), ck.cpu().numpy().reshape(n, ckmax, s.nvar + 1)


def test_checkpoints_replay_bitexact(pkg, orc):
    import torch
    b, s, ctl, C0, logk, w = _setup(pkg, 8, 51, "nofma")
    R = torch.from_numpy(np.ascontiguousarray(b.RCONST.T)).to(C0.device)
    C, ist, ierr, ck = _forward_ckpt(s, ctl, C0, R)
    assert (ierr == 1).all()
    nv = s.nvar
    for c in range(ctl.n):
        nacc = ist[c, 3]
        hs = ck[c, :nacc, nv]
        y = orc.integrate_frozen(b.C[:nv, c], b.C[nv:, c], b.RCONST[:, c], hs)
        assert np.array_equal(y.view(np.uint64), C[c, :nv].cpu().numpy().view(np.uint64))
        assert np.array_equal(ck[c, 0, :nv].view(np.uint64), b.C[:nv, c].view(np.uint64))


# fullchem: the 64 cells of the adjoint configuration.  The synthetic
# mechanism (indexed factorisation with reciprocal pivots, ~200 steps per
# cell): 10 cells, which keep the CPU difference quotients to seconds.
FD_CASES = {"fullchem": (64, 52, CKMAX, 100), "synth120": (10, 9, 2000, 40)}


@pytest.mark.parametrize("mech", list(FD_CASES))
def test_adjoint_matches_finite_differences(pkg, orc, mech):
    import torch
    chemistry_step = importlib.import_module("geos-chem-gpu-hybrid_b200.adjoint").chemistry_step
    ncell, seed, ckmax, min_checked = FD_CASES[mech]
    b, s, ctl, C0, logk, w = _setup(pkg, ncell, seed, "fma", mech)
    C0.requires_grad_(True)
    logk.requires_grad_(True)
    Cf = chemistry_step(C0, logk, s, ctl, ckmax)
    nv = s.nvar
    W = torch.zeros_like(Cf)
    W[:, :nv] = torch.from_numpy(w).to(Cf.device)
    L = (Cf * W).sum()
    L.backward()
    gy = C0.grad.cpu().numpy()
    gk = logk.grad.cpu().numpy()
    # recorded step sizes (a second checkpointed forward of the same cells)
    R = torch.exp(logk.detach())
    _, ist, ierr, ck = _forward_ckpt(s, ctl, C0.detach(), R, ckmax)
    assert (ierr == 1).all()
    rng = np.random.default_rng(3)
    checked = 0
    bad = []
    for c in range(ncell):
        hs = ck[c, :ist[c, 3], nv]
        y0 = b.C[:nv, c].copy()
        fix = b.C[nv:, c]
        rct = b.RCONST[:, c].copy()
        wc = w[c]

        def loss(y, r):
            return float(np.dot(wc, orc.integrate_frozen(y, fix, r, hs, mech=mech)))

        base = abs(np.dot(wc, np.abs(orc.integrate_frozen(y0, fix, rct, hs, mech=mech))))
        big_y = np.argsort(-np.abs(y0 * wc))[:40]
        for i in rng.choice(big_y, 8, replace=False):
            d = 1e-6 * y0[i]
            yp, ym = y0.copy(), y0.copy()
            yp[i] += d
            ym[i] -= d
            fd = (loss(yp, rct) - loss(ym, rct)) / (2 * d)
            noise = 1e-14 * base / (2 * d)
            if abs(fd) > FD_MARGIN * noise:
                checked += 1
                if abs(gy[c, i] - fd) > 1e-5 * abs(fd):
                    bad.append(("y", c, i, gy[c, i], fd, noise))
        active = np.flatnonzero(rct > 0)
        for j in rng.choice(active, 8, replace=False):
            rp, rm = rct.copy(), rct.copy()
            rp[j] *= np.exp(1e-6)
            rm[j] *= np.exp(-1e-6)
            fd = (loss(y0, rp) - loss(y0, rm)) / 2e-6
            noise = 1e-14 * base / 2e-6
            if abs(fd) > FD_MARGIN * noise:
                checked += 1
                if abs(gk[c, j] - fd) > 1e-5 * abs(fd):
                    bad.append(("lnk", c, j, gk[c, j], fd, noise))
    assert checked >= min_checked, checked
    assert not bad, bad


def _backward_with_capacity(pkg, ckmax, on_error):
    import torch
    adj = importlib.import_module("geos-chem-gpu-hybrid_b200.adjoint")
    b, s, ctl, C0, logk, w = _setup(pkg, 16, 53, "fma")
    C0.requires_grad_(True)
    logk.requires_grad_(True)
    Cf = adj.chemistry_step(C0, logk, s, ctl, ckmax, on_error=on_error)
    Cf.sum().backward()
    return adj, C0.grad, logk.grad


def test_checkpoint_overflow_raises(pkg):
    """Cold cells take tens of accepted steps; 3 checkpoints cannot hold them."""
    with pytest.raises(RuntimeError, match="ckpt_max=3"):
        _backward_with_capacity(pkg, 3, "raise")


def test_checkpoint_overflow_masks(pkg):
    adj, gC0, gK = _backward_with_capacity(pkg, 3, "mask")
    bad = adj.LAST_FAILED[0]
    assert bool(bad.all())
    assert float(gC0.abs().sum()) == 0.0 and float(gK.abs().sum()) == 0.0
