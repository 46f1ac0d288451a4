"""Consecutive chemistry steps with the state resident on the device.

One chemistry step of the model's batched GPU path, done entirely on the
device and stream-ordered, so that several steps can be captured into one
CUDA graph and replayed:

1. solve every cell (gcchem_b200_integrate_device, persistent queue);
2. clamp negative concentrations to zero, as the model's scatter does
   (``C(N) = MAX(C(N), 0)``, src/geos-chem/GeosCore/fullchem_mod.F90:2995);
3. warm start: RCNTRL(3) <- RSTAT(3) (Hnew; the model keeps it in
   State_Chm%KPPHvalue, fullchem_mod.F90:2922, and passes it back as Hstart);
4. the next step's queue order: cells sorted by this step's ISTAT(3),
   most expensive first (the model's pre-scan, fullchem_mod.F90:906-960).

Between steps the model would also update RCONST and the photolysis
fields; here RCONST stays fixed, so consecutive steps continue the same
chemistry from the evolved state.
"""
from __future__ import annotations

import numpy as np


class Chain:
    def __init__(self, solver, batch, device="cuda:0"):
        import torch
        self.torch = torch
        self.s = solver
        dev = torch.device(device)
        self.dev = dev

        def up(a, dt):
            return torch.from_numpy(np.ascontiguousarray(a.T if a.ndim == 2 else a)).to(dev, dt)

        self.n = batch.n
        self.tstart, self.tend = float(batch.Tstart), float(batch.Tend)
        self.C = up(batch.C, torch.float64)
        self.RCONST = up(batch.RCONST, torch.float64)
        self.ATOL = up(batch.ATOL, torch.float64)
        self.RTOL = up(batch.RTOL, torch.float64)
        self.ICNTRL = up(batch.ICNTRL, torch.int32)
        self.RCNTRL = up(batch.RCNTRL, torch.float64)
        self.order = torch.arange(self.n, dtype=torch.int32, device=dev)
        self.ISTAT = torch.zeros((self.n, 8), dtype=torch.int32, device=dev)
        self.RSTAT = torch.zeros((self.n, 3), dtype=torch.float64, device=dev)
        self.IERR = torch.zeros(self.n, dtype=torch.int32, device=dev)
        self.keys = torch.zeros(self.n, dtype=torch.int32, device=dev)
        self.graph = None
        solver.reserve(self.n)

    def step(self, stream=None) -> None:
        """Enqueue one chemistry step on `stream` (default: current)."""
        t = self.torch
        stream = stream or t.cuda.current_stream()
        self.s.integrate_device(self.C, self.RCONST, self.ATOL, self.RTOL, self.ICNTRL,
                                self.RCNTRL, self.order, self.ISTAT, self.RSTAT, self.IERR,
                                self.tstart, self.tend, stream=stream)
        with t.cuda.stream(stream):
            self.C.clamp_(min=0.0)
            self.RCNTRL[:, 2].copy_(self.RSTAT[:, 2])
            self.keys.copy_(self.ISTAT[:, 2])
        self.s.cost_order(self.keys, self.order, stream=stream)

    def capture(self, nsteps: int) -> None:
        """Capture `nsteps` consecutive steps into one CUDA graph.  One
        eager step must have run first (workspace and launch setup)."""
        t = self.torch
        s = t.cuda.Stream()
        s.wait_stream(t.cuda.current_stream())
        g = t.cuda.CUDAGraph()
        with t.cuda.stream(s):
            with t.cuda.graph(g, stream=s):
                for _ in range(nsteps):
                    self.step(stream=s)
        t.cuda.current_stream().wait_stream(s)
        self.graph = g
        self.graph_steps = nsteps

    def replay(self) -> None:
        self.graph.replay()
