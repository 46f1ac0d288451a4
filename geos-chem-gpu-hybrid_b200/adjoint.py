"""Gradients of a chemistry step through torch.autograd.

``ChemistryStep.apply(C0, log_rconst, solver, controls)`` solves one
chemistry step of every cell on the GPU (forward: checkpointed persistent
solve) and returns the final concentrations; ``backward`` runs the discrete
adjoint kernel (csrc/adjoint.cu) through the recorded step sequence and
returns dL/dC0 (variable species; fixed species get 0) and
dL/d log RCONST.  Tensors use the device layout of the C-ABI: C (n, NSPEC),
RCONST (n, NREACT), float64 on the GPU.

The step sizes are frozen at the values the forward solve accepted, so the
gradient is the exact derivative of that discrete map (the step-size control
itself is not differentiated) -- the usual discrete adjoint of a Rosenbrock
method.
"""
from __future__ import annotations

import numpy as np

from . import workloads


class Controls:
    """Per-batch solver inputs that are not differentiated."""

    def __init__(self, batch, device):
        import torch

        def up(a, dt):
            return torch.from_numpy(np.ascontiguousarray(a.T if a.ndim == 2 else a)).to(device, dt)

        self.ATOL = up(batch.ATOL, torch.float64)
        self.RTOL = up(batch.RTOL, torch.float64)
        self.ICNTRL = up(batch.ICNTRL, torch.int32)
        self.RCNTRL = up(batch.RCNTRL, torch.float64)
        self.Tstart, self.Tend = float(batch.Tstart), float(batch.Tend)
        self.n = batch.n


def _function():
    import torch

    class ChemistryStep(torch.autograd.Function):
        @staticmethod
        def forward(ctx, C0, log_rconst, solver, ctl, ckpt_max, on_error):
            n = ctl.n
            dev = C0.device
            R = torch.exp(log_rconst).contiguous()
            C = C0.detach().clone().contiguous()
            order = torch.arange(n, dtype=torch.int32, device=dev)
            IST = torch.zeros((n, 8), dtype=torch.int32, device=dev)
            RST = torch.zeros((n, 3), dtype=torch.float64, device=dev)
            IE = torch.zeros(n, dtype=torch.int32, device=dev)
            ckpt = torch.empty(n * ckpt_max * (solver.nvar + 1), dtype=torch.float64, device=dev)
            solver.integrate_device_ckpt(C, R, ctl.ATOL, ctl.RTOL, ctl.ICNTRL, ctl.RCNTRL, order,
                                         IST, RST, IE, ckpt, ckpt_max, ctl.Tstart, ctl.Tend)
            ctx.save_for_backward(C0.detach(), R, IST, ckpt, IE)
            ctx.solver, ctx.ckpt_max, ctx.on_error = solver, ckpt_max, on_error
            return C

        @staticmethod
        def backward(ctx, grad_C):
            C0, R, IST, ckpt, IE = ctx.saved_tensors
            s = ctx.solver
            n = C0.shape[0]
            gC0 = torch.empty_like(C0)
            gK = torch.empty_like(R)
            ierr = torch.zeros(n, dtype=torch.int32, device=C0.device)
            s.adjoint_device(C0, R, IST, ckpt, ctx.ckpt_max, grad_C.contiguous(), gC0, gK, ierr)
            # a cell whose forward solve failed (IERR /= 1) has no complete
            # step sequence to differentiate; one with more accepted steps
            # than ckpt_max (-101) or a singular factor (-8) has no adjoint
            bad = (IE != 1) | (ierr != 1)
            nbad = int(bad.sum().item())
            if nbad:
                if ctx.on_error == "raise":
                    raise RuntimeError(
                        f"chemistry_step backward: {nbad} of {n} cells have no gradient "
                        f"(forward IERR /= 1: {int((IE != 1).sum().item())}, adjoint ierr "
                        f"-101 (more accepted steps than ckpt_max={ctx.ckpt_max}): "
                        f"{int((ierr == -101).sum().item())}, other: "
                        f"{int(((ierr != 1) & (ierr != -101)).sum().item())})")
                gC0[bad] = 0.0
                gK[bad] = 0.0
            LAST_FAILED[0] = bad
            return gC0, gK, None, None, None, None

    return ChemistryStep


_FN = None
# bool mask (n,) of the cells the last backward pass could not differentiate
LAST_FAILED = [None]


def chemistry_step(C0, log_rconst, solver, ctl, ckpt_max: int = 512, on_error: str = "raise"):
    """Differentiable chemistry step (see the module docstring).

    Cells without a gradient -- a forward solve that failed (IERR /= 1),
    more accepted steps than ``ckpt_max``, or a singular factor in the
    backward sweep -- make the backward pass raise RuntimeError
    (``on_error="raise"``), or get zero gradients with ``on_error="mask"``;
    either way ``LAST_FAILED[0]`` holds the mask of those cells."""
    global _FN
    if on_error not in ("raise", "mask"):
        raise ValueError("on_error must be 'raise' or 'mask'")
    if _FN is None:
        _FN = _function()
    return _FN.apply(C0, log_rconst, solver, ctl, ckpt_max, on_error)


def loss_weights(n: int, nvar: int, seed: int = 0, mech: str = "fullchem") -> np.ndarray:
    """Seeded positive weights of the final concentrations (n, NVAR); the
    surrogate O3, NO, NO2, OH, HO2 and CO species weighted x10."""
    rng = np.random.default_rng(seed)
    w = rng.uniform(0.1, 1.0, (n, nvar))
    info = workloads.mechanism_info(mech)
    for name in ("O3", "NO", "NO2", "OH", "HO2", "CO"):
        if name in info.species:
            w[:, info.species[name]] *= 10.0
    return w
