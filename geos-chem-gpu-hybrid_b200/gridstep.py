"""A chemistry step of the model's batched GPU path with the model's grid
fields resident on the device.

``GridChemistry`` holds, on the GPU, what fullchem_mod.F90 keeps between
chemistry steps -- the species concentrations on the grid, the KPP step
size KPPHvalue and the previous internal step counts PrevNsteps -- and one
``step`` does the model's whole batch path without host staging:

1. the pre-scan: BatchMap = chemistry cells sorted by descending PrevNsteps
   (stable; L,J,I order on the first step) (gcchem_b200_batch_map,
   fullchem_mod.F90:906-993);
2. the gather of the grid concentrations (and the rate constants) into the
   cost-ordered batch, with the warm start Hstart = KPPHvalue
   (gcchem_b200_gather, :1538-1543, :1749-1756);
3. the solve with the model's retry protocol for failed cells
   (gcchem_b200_integrate_device_retry, :2436-2520);
4. the scatter: negatives clamped, KPPHvalue, PrevNsteps and the KPP
   diagnostics written per cell (gcchem_b200_scatter, :2878-3000).

Every call is stream-ordered, so steps can be captured into a CUDA graph.
Grid tensors use the model's Fortran order: a field (NX, NY, NZ, k) is a
contiguous torch tensor of shape (k, NZ, NY, NX).
"""
from __future__ import annotations

import ctypes

import numpy as np


class GridChemistry:
    def __init__(self, solver, conc, map_kpp_spc, rconst_grid, atol, rtol,
                 icntrl=None, in_chem=None, sort: bool = True, tstart: float = 0.0,
                 tend: float = 1200.0, atol_retry=None, rtol_retry=None, diag: bool = True):
        import torch
        self.torch = torch
        self.s = solver
        self.conc = conc                          # (nSpc, NZ, NY, NX) float64, device
        self.dev = conc.device
        nspc, NZ, NY, NX = conc.shape
        self.NX, self.NY, self.NZ = NX, NY, NZ
        self.ncells = NX * NY * NZ
        self.kmap = torch.as_tensor(np.asarray(map_kpp_spc, np.int32), device=self.dev)
        if self.kmap.numel() != solver.nspec:
            raise ValueError("MapKppSpc needs one entry per KPP species")
        self.rgrid = rconst_grid                  # (NREACT, NZ, NY, NX) or None
        self.in_chem = None if in_chem is None else \
            torch.as_tensor(np.asarray(in_chem, np.int32), device=self.dev).contiguous()
        self.n = self.ncells if in_chem is None else int(np.count_nonzero(in_chem))
        self.sort = int(bool(sort))
        self.tstart, self.tend = float(tstart), float(tend)
        f64, i32 = torch.float64, torch.int32
        n = self.n
        self.ATOL = torch.as_tensor(np.asarray(atol, np.float64), device=self.dev)
        self.RTOL = torch.as_tensor(np.asarray(rtol, np.float64), device=self.dev)
        self.ATOLr = self.ATOL if atol_retry is None else \
            torch.as_tensor(np.asarray(atol_retry, np.float64), device=self.dev)
        self.RTOLr = self.RTOL if rtol_retry is None else \
            torch.as_tensor(np.asarray(rtol_retry, np.float64), device=self.dev)
        ic = np.zeros(20, np.int32)
        ic[[0, 1, 2, 6, 14]] = (1, 0, 4, 1, -1)   # the model's settings
        if icntrl is not None:
            ic = np.asarray(icntrl, np.int32)
        self.ICNTRL = torch.as_tensor(np.tile(ic, (n, 1)), device=self.dev).contiguous()
        self.RCNTRL = torch.zeros((n, 20), dtype=f64, device=self.dev)
        self.C = torch.zeros((n, solver.nspec), dtype=f64, device=self.dev)
        self.RCONST = torch.zeros((n, solver.nreact), dtype=f64, device=self.dev)
        self.ISTAT = torch.zeros((n, 8), dtype=i32, device=self.dev)
        self.RSTAT = torch.zeros((n, 3), dtype=f64, device=self.dev)
        self.IERR = torch.zeros(n, dtype=i32, device=self.dev)
        self.nfail = torch.zeros(2, dtype=i32, device=self.dev)
        self.order = torch.arange(n, dtype=i32, device=self.dev)
        self.batch_map = torch.zeros((n, 3), dtype=i32, device=self.dev)
        self.kpph = torch.zeros((NZ, NY, NX), dtype=f64, device=self.dev)
        self.prev = torch.zeros((NZ, NY, NX), dtype=i32, device=self.dev)
        self.diag = torch.zeros((9, NZ, NY, NX), dtype=torch.float32, device=self.dev) \
            if diag else None
        self.graph = None
        solver.reserve(n)

    def _call(self, fn, *args):
        rc = fn(*args)
        if rc != 0:
            raise RuntimeError(f"{fn.__name__} failed ({rc})")

    def step(self, stream=None) -> None:
        """Enqueue one chemistry step on `stream` (default: current)."""
        t = self.torch
        st = stream or t.cuda.current_stream()
        sp = ctypes.c_void_p(st.cuda_stream)
        lib = self.s.lib
        vp = ctypes.c_void_p
        mask = vp(self.in_chem.data_ptr()) if self.in_chem is not None else None
        self._call(lib.gcchem_b200_batch_map, self.NX, self.NY, self.NZ,
                   vp(self.prev.data_ptr()), mask, self.sort, self.n,
                   vp(self.batch_map.data_ptr()), sp)
        rg = vp(self.rgrid.data_ptr()) if self.rgrid is not None else None
        rb = vp(self.RCONST.data_ptr()) if self.rgrid is not None else None
        self._call(lib.gcchem_b200_gather, self.n, self.NX, self.NY, self.NZ,
                   vp(self.batch_map.data_ptr()), vp(self.conc.data_ptr()),
                   vp(self.kmap.data_ptr()), vp(self.C.data_ptr()), rg, rb,
                   vp(self.kpph.data_ptr()), vp(self.RCNTRL.data_ptr()), sp)
        self.s.integrate_device_retry(self.C, self.RCONST, self.ATOL, self.RTOL, self.ATOLr,
                                      self.RTOLr, self.ICNTRL, self.RCNTRL, self.order,
                                      self.ISTAT, self.RSTAT, self.IERR, self.nfail,
                                      self.tstart, self.tend, stream=st)
        dg = vp(self.diag.data_ptr()) if self.diag is not None else None
        self._call(lib.gcchem_b200_scatter, self.n, self.NX, self.NY, self.NZ,
                   vp(self.batch_map.data_ptr()), vp(self.conc.data_ptr()),
                   vp(self.kmap.data_ptr()), vp(self.C.data_ptr()), vp(self.ISTAT.data_ptr()),
                   vp(self.RSTAT.data_ptr()), vp(self.kpph.data_ptr()),
                   vp(self.prev.data_ptr()), dg, sp)

    def capture(self, nsteps: int) -> None:
        """Capture `nsteps` consecutive steps into one CUDA graph (after one
        eager step, which sizes every buffer)."""
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

    def replay(self) -> None:
        self.graph.replay()
