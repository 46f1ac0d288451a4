"""ctypes / PyTorch binding of libgcchemgpu.so.

``Solver`` wraps one built library (one mechanism, one arithmetic variant):

* ``integrate_batch`` -- the legacy host-array entry gc_gpu_integrate_batch
  (gpulib/src/gc_gpu_batch_api.F90:115-136) on numpy arrays in the model's
  Fortran layout;
* ``integrate_device`` -- the device-resident, stream-ordered entry
  gcchem_b200_integrate_device on CUDA torch tensors;
* ``selftest`` / ``info`` / ``set_device`` -- gc_gpu_selftest, gc_gpu_info,
  gc_gpu_set_device.

The library is the only compute path: if it is missing, loading fails with
an error that says how to build it.  There is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_DIR = os.path.join(HERE, "lib")

PLAIN = 0
PERSISTENT = 1
PLAIN_FUSED = 2
COOP = 3            # one thread block per cell, cell state in shared memory


def lib_name(mech: str = "fullchem", variant: str = "fma") -> str:
    base = "libgcchemgpu" if mech == "fullchem" else f"libgcchemgpu_{mech}"
    return base + ("_nofma" if variant == "nofma" else "") + ".so"


def lib_path(mech: str = "fullchem", variant: str = "fma") -> str:
    return os.path.join(LIB_DIR, lib_name(mech, variant))


_CACHE: dict = {}
# cpu_tail(first, count, user) of gcchem_b200_hybrid_step
TAIL_FN = ctypes.CFUNCTYPE(None, ctypes.c_int, ctypes.c_int, ctypes.c_void_p)


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


class Solver:
    def __init__(self, mech: str = "fullchem", variant: str = "fma", path: str | None = None):
        path = path or lib_path(mech, variant)
        if not os.path.exists(path):
            raise RuntimeError(
                f"{path} is missing: the CUDA solver library is not built "
                "(run __graft_entry__.build())")
        self.path = path
        self.mech = mech
        self.variant = variant
        lib = ctypes.CDLL(path)
        vp, ci, cd, cl = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_long
        lib.gc_gpu_integrate_batch.argtypes = [ci, cd, cd] + [vp] * 12
        lib.gc_gpu_integrate_batch.restype = None
        lib.gc_gpu_integrate_batch_dev.argtypes = [ci, ci, cd, cd] + [vp] * 12
        lib.gc_gpu_integrate_batch_dev.restype = None
        lib.gc_gpu_selftest.argtypes = [vp, vp, vp]
        lib.gc_gpu_info.argtypes = [vp, ctypes.c_char_p, ci]
        lib.gc_gpu_set_device.argtypes = [ci]
        lib.gc_gpu_set_device.restype = ci
        lib.gcchem_b200_sizes.argtypes = [vp] * 4
        lib.gcchem_b200_set_launch.argtypes = [ci, ci, ci]
        lib.gcchem_b200_set_launch.restype = ci
        lib.gcchem_b200_set_chunk.argtypes = [ci]
        lib.gcchem_b200_set_chunk.restype = ci
        lib.gcchem_b200_set_row_scratch.argtypes = [ci]
        lib.gcchem_b200_set_row_scratch.restype = ci
        lib.gcchem_b200_integrate_device.argtypes = [ci, cd, cd] + [vp] * 11
        lib.gcchem_b200_integrate_device.restype = ci
        lib.gcchem_b200_integrate_device_noalloc.argtypes = [ci, cd, cd] + [vp] * 11
        lib.gcchem_b200_integrate_device_noalloc.restype = ci
        lib.gcchem_b200_integrate_device_retry.argtypes = [ci, cd, cd] + [vp] * 14
        lib.gcchem_b200_integrate_device_retry.restype = ci
        lib.gcchem_b200_integrate_device_ckpt.argtypes = [ci, cd, cd] + [vp] * 11 + [ci, vp]
        lib.gcchem_b200_integrate_device_ckpt.restype = ci
        lib.gcchem_b200_adjoint_device.argtypes = [ci] + [vp] * 4 + [ci] + [vp] * 5
        lib.gcchem_b200_adjoint_device.restype = ci
        lib.gcchem_b200_cost_order.argtypes = [vp, ci, vp, vp]
        lib.gcchem_b200_cost_order.restype = ci
        lib.gcchem_b200_reserve.argtypes = [ci]
        lib.gcchem_b200_reserve.restype = ci
        lib.gcchem_b200_workspace_slots.argtypes = [ci]
        lib.gcchem_b200_workspace_slots.restype = cl
        lib.gcchem_b200_workspace_bytes_per_slot.restype = cl
        lib.gcchem_b200_fp64_peak_tflops.restype = cd
        lib.gcchem_b200_phase_ms.argtypes = [ci, cl, ci]
        lib.gcchem_b200_phase_ms.restype = cd
        lib.gcchem_b200_batch_map.argtypes = [ci, ci, ci, vp, vp, ci, ci, vp, vp]
        lib.gcchem_b200_batch_map.restype = ci
        lib.gcchem_b200_gather.argtypes = [ci, ci, ci, ci] + [vp] * 9
        lib.gcchem_b200_gather.restype = ci
        lib.gcchem_b200_scatter.argtypes = [ci, ci, ci, ci] + [vp] * 10
        lib.gcchem_b200_scatter.restype = ci
        lib.gcchem_b200_hybrid_create.argtypes = [ci, cd, ci]
        lib.gcchem_b200_hybrid_create.restype = vp
        lib.gcchem_b200_hybrid_destroy.argtypes = [vp]
        lib.gcchem_b200_hybrid_plan.argtypes = [vp, ci] + [vp] * 5
        lib.gcchem_b200_hybrid_plan.restype = ci
        lib.gcchem_b200_hybrid_update.argtypes = [vp, vp, cd]
        lib.gcchem_b200_hybrid_update.restype = ci
        lib.gcchem_b200_hybrid_state.argtypes = [vp] * 5
        lib.gcchem_b200_hybrid_state.restype = ci
        # h, nCell, Tstart, Tend, C, RCONST, ATOL, RTOL, ICNTRL, RCNTRL, prevNsteps,
        # ISTAT, RSTAT, IERR, cpu_tail, user, nGpu, tGpu, tCpu
        lib.gcchem_b200_hybrid_step.argtypes = [vp, ci, cd, cd] + [vp] * 10 + [TAIL_FN, vp] + \
            [vp] * 3
        lib.gcchem_b200_hybrid_step.restype = ci
        self.lib = lib
        s = [ctypes.c_int() for _ in range(4)]
        lib.gcchem_b200_sizes(*[ctypes.byref(x) for x in s])
        self.nvar, self.nfix, self.nreact, self.nnz = (x.value for x in s)
        self.nspec = self.nvar + self.nfix

    # -- legacy entry -----------------------------------------------------
    def integrate_batch(self, batch, perm=None, dev: int = -1):
        """Solve a workloads.Batch through gc_gpu_integrate_batch[_dev].

        Returns (C, ISTAT, RSTAT, IERR, tTotal, tKernel) with C (NSPEC, n),
        ISTAT (8, n), RSTAT (3, n) in Fortran order."""
        n = batch.n
        C = np.array(batch.C, dtype=np.float64, order="F", copy=True)
        R = np.asfortranarray(batch.RCONST, dtype=np.float64)
        IC = np.asfortranarray(batch.ICNTRL, dtype=np.int32)
        RC = np.asfortranarray(batch.RCNTRL, dtype=np.float64)
        perm = (np.arange(1, n + 1, dtype=np.int32) if perm is None
                else np.ascontiguousarray(perm, dtype=np.int32))
        atol = np.ascontiguousarray(batch.ATOL, dtype=np.float64)
        rtol = np.ascontiguousarray(batch.RTOL, dtype=np.float64)
        ist = np.zeros((8, n), np.int32, order="F")
        rst = np.zeros((3, n), np.float64, order="F")
        ierr = np.zeros(n, np.int32)
        tt, tk = ctypes.c_double(), ctypes.c_double()
        self.lib.gc_gpu_integrate_batch_dev(
            int(dev), n, float(batch.Tstart), float(batch.Tend), _p(C), _p(R),
            _p(atol), _p(rtol), _p(IC), _p(RC), _p(perm), _p(ist), _p(rst),
            _p(ierr), ctypes.byref(tt), ctypes.byref(tk))
        return C, ist, rst, ierr, tt.value, tk.value

    # -- device entry -----------------------------------------------------
    def integrate_device(self, C, RCONST, ATOL, RTOL, ICNTRL, RCNTRL, order,
                         ISTAT, RSTAT, IERR, Tstart=0.0, Tend=1200.0,
                         stream=None) -> None:
        """Enqueue the solve on CUDA tensors (layouts as the legacy entry,
        order = 0-based int32 columns).  C (NSPEC, n) is a column-major view,
        i.e. a contiguous tensor of shape (n, NSPEC)."""
        import torch
        n = int(order.numel())
        for t in (C, RCONST, ATOL, RTOL, ICNTRL, RCNTRL, order, ISTAT, RSTAT, IERR):
            if not t.is_cuda or not t.is_contiguous():
                raise ValueError("integrate_device needs contiguous CUDA tensors")
        if C.dtype != torch.float64 or RCONST.dtype != torch.float64:
            raise TypeError("C and RCONST must be float64")
        if C.numel() != n * self.nspec or RCONST.numel() != n * self.nreact:
            raise ValueError("array sizes do not match the mechanism")
        if stream is None:
            stream = torch.cuda.current_stream()
        rc = self.lib.gcchem_b200_integrate_device(
            n, float(Tstart), float(Tend), C.data_ptr(), RCONST.data_ptr(),
            ATOL.data_ptr(), RTOL.data_ptr(), ICNTRL.data_ptr(),
            RCNTRL.data_ptr(), order.data_ptr(), ISTAT.data_ptr(),
            RSTAT.data_ptr(), IERR.data_ptr(), ctypes.c_void_p(stream.cuda_stream))
        if rc != 0:
            raise RuntimeError(f"gcchem_b200_integrate_device failed ({rc})")

    def integrate_device_retry(self, C, RCONST, ATOL, RTOL, ATOLr, RTOLr, ICNTRL, RCNTRL,
                               order, ISTAT, RSTAT, IERR, nfail, Tstart=0.0, Tend=1200.0,
                               stream=None) -> None:
        """Solve with the model's retry protocol on the device; nfail is a
        CUDA int32 tensor of 2 entries (first-attempt failures, double
        failures)."""
        import torch
        n = int(order.numel())
        if stream is None:
            stream = torch.cuda.current_stream()
        rc = self.lib.gcchem_b200_integrate_device_retry(
            n, float(Tstart), float(Tend), C.data_ptr(), RCONST.data_ptr(), ATOL.data_ptr(),
            RTOL.data_ptr(), ATOLr.data_ptr(), RTOLr.data_ptr(), ICNTRL.data_ptr(),
            RCNTRL.data_ptr(), order.data_ptr(), ISTAT.data_ptr(), RSTAT.data_ptr(),
            IERR.data_ptr(), nfail.data_ptr(), ctypes.c_void_p(stream.cuda_stream))
        if rc != 0:
            raise RuntimeError(f"gcchem_b200_integrate_device_retry failed ({rc})")

    def integrate_device_ckpt(self, C, RCONST, ATOL, RTOL, ICNTRL, RCNTRL, order, ISTAT,
                              RSTAT, IERR, ckpt, ckpt_max, Tstart=0.0, Tend=1200.0,
                              stream=None) -> None:
        """integrate_device that also records (y_n, h_n) of every accepted
        step in ckpt (n_cells * ckpt_max * (NVAR+1) doubles)."""
        import torch
        n = int(order.numel())
        if stream is None:
            stream = torch.cuda.current_stream()
        rc = self.lib.gcchem_b200_integrate_device_ckpt(
            n, float(Tstart), float(Tend), C.data_ptr(), RCONST.data_ptr(), ATOL.data_ptr(),
            RTOL.data_ptr(), ICNTRL.data_ptr(), RCNTRL.data_ptr(), order.data_ptr(),
            ISTAT.data_ptr(), RSTAT.data_ptr(), IERR.data_ptr(), ckpt.data_ptr(),
            int(ckpt_max), ctypes.c_void_p(stream.cuda_stream))
        if rc != 0:
            raise RuntimeError(f"gcchem_b200_integrate_device_ckpt failed ({rc})")

    def adjoint_device(self, C0, RCONST, ISTAT, ckpt, ckpt_max, lam, gC0, gK, ierr,
                       stream=None) -> None:
        """Discrete adjoint through the recorded steps: gC0 = dL/dC0,
        gK = dL/dln RCONST, given lam = dL/dC at the end."""
        import torch
        n = int(ierr.numel())
        if stream is None:
            stream = torch.cuda.current_stream()
        rc = self.lib.gcchem_b200_adjoint_device(
            n, C0.data_ptr(), RCONST.data_ptr(), ISTAT.data_ptr(), ckpt.data_ptr(),
            int(ckpt_max), lam.data_ptr(), gC0.data_ptr(), gK.data_ptr(), ierr.data_ptr(),
            ctypes.c_void_p(stream.cuda_stream))
        if rc != 0:
            raise RuntimeError(f"gcchem_b200_adjoint_device failed ({rc})")

    def cost_order(self, keys, order=None, stream=None):
        """Columns sorted by descending cost key (CUDA int32 tensors)."""
        import torch
        n = int(keys.numel())
        if order is None:
            order = torch.empty(n, dtype=torch.int32, device=keys.device)
        if stream is None:
            stream = torch.cuda.current_stream()
        rc = self.lib.gcchem_b200_cost_order(keys.data_ptr(), n, order.data_ptr(),
                                             ctypes.c_void_p(stream.cuda_stream))
        if rc != 0:
            raise RuntimeError("gcchem_b200_cost_order failed")
        return order

    def integrate_device_noalloc(self, C, RCONST, ATOL, RTOL, ICNTRL, RCNTRL, order,
                                 ISTAT, RSTAT, IERR, Tstart=0.0, Tend=1200.0,
                                 stream=None) -> int:
        """gcchem_b200_integrate_device_noalloc: the arguments of
        integrate_device, no device allocation, at most 256 cells per call.
        Returns the library's status code (0 = launched, -4 = too many cells)."""
        import torch
        n = int(order.numel())
        if stream is None:
            stream = torch.cuda.current_stream()
        return int(self.lib.gcchem_b200_integrate_device_noalloc(
            n, float(Tstart), float(Tend), C.data_ptr(), RCONST.data_ptr(),
            ATOL.data_ptr(), RTOL.data_ptr(), ICNTRL.data_ptr(),
            RCNTRL.data_ptr(), order.data_ptr(), ISTAT.data_ptr(),
            RSTAT.data_ptr(), IERR.data_ptr(), ctypes.c_void_p(stream.cuda_stream)))

    def set_launch(self, mode: int = PERSISTENT, threads: int = 0,
                   blocks_per_sm: int = 0) -> None:
        if self.lib.gcchem_b200_set_launch(mode, threads, blocks_per_sm) != 0:
            raise ValueError("invalid launch settings")

    def set_chunk(self, cells: int = 0) -> None:
        """Cells per launch of the plain kernels (0: environment / whole batch)."""
        if self.lib.gcchem_b200_set_chunk(int(cells)) != 0:
            raise ValueError("invalid chunk size")

    def set_row_scratch(self, shared: bool = False) -> None:
        """Indexed factorisation's row scratch in shared memory (small
        mechanisms only) or in the workspace."""
        if self.lib.gcchem_b200_set_row_scratch(int(bool(shared))) != 0:
            raise ValueError("shared row scratch not available for this mechanism / block size")

    def reserve(self, n: int) -> None:
        if self.lib.gcchem_b200_reserve(int(n)) != 0:
            raise RuntimeError("could not allocate the solver workspace")

    def release(self) -> None:
        self.lib.gcchem_b200_release()

    def workspace_slots(self, n: int) -> int:
        return int(self.lib.gcchem_b200_workspace_slots(int(n)))

    def fp64_peak_tflops(self) -> float:
        return float(self.lib.gcchem_b200_fp64_peak_tflops())

    def phase_ms(self, phase: int, slots: int, reps: int) -> float:
        return float(self.lib.gcchem_b200_phase_ms(int(phase), int(slots), int(reps)))

    def bytes_per_slot(self) -> int:
        return int(self.lib.gcchem_b200_workspace_bytes_per_slot())

    # -- service entries --------------------------------------------------
    def selftest(self):
        rc, ns, tt = ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
        self.lib.gc_gpu_selftest(ctypes.byref(rc), ctypes.byref(ns), ctypes.byref(tt))
        return rc.value, ns.value, tt.value

    def info(self):
        n = ctypes.c_int()
        buf = ctypes.create_string_buffer(256)
        self.lib.gc_gpu_info(ctypes.byref(n), buf, 256)
        return n.value, buf.value.decode()

    def set_device(self, d: int) -> int:
        return int(self.lib.gc_gpu_set_device(int(d)))


class Hybrid:
    """The hybrid CPU/GPU split of the model's GC_BATCH_CHEM=3 mode
    (gcchem_b200_hybrid_*): a work model over the previous step counts, a
    GPU/CPU share from measured rates, work-balanced device slices.  The
    CPU side is the caller's own integrator, passed as ``cpu_tail``."""

    def __init__(self, solver: Solver, ndev: int = 1, frac: float = 0.5, fixed: bool = False):
        self.s = solver
        self.ndev = int(ndev)
        self.h = solver.lib.gcchem_b200_hybrid_create(self.ndev, float(frac), int(bool(fixed)))
        if not self.h:
            raise ValueError("invalid hybrid settings")

    def __del__(self):
        h, self.h = getattr(self, "h", None), None
        if h:
            self.s.lib.gcchem_b200_hybrid_destroy(h)

    def plan(self, prev_nsteps):
        """(nGpu, [(lo, hi) 1-based inclusive per device]) for cost-ordered keys."""
        prev = np.ascontiguousarray(prev_nsteps, dtype=np.int32)
        ng, nd = ctypes.c_int(), ctypes.c_int()
        lo = np.zeros(self.ndev, np.int32)
        hi = np.zeros(self.ndev, np.int32)
        if self.s.lib.gcchem_b200_hybrid_plan(self.h, prev.size, _p(prev), ctypes.byref(ng),
                                              ctypes.byref(nd), _p(lo), _p(hi)) != 0:
            raise ValueError("hybrid plan failed")
        return ng.value, [(int(lo[d]), int(hi[d])) for d in range(nd.value)]

    def update(self, dev_tw, t_cpu: float) -> None:
        tw = np.ascontiguousarray(dev_tw, dtype=np.float64)
        if self.s.lib.gcchem_b200_hybrid_update(self.h, _p(tw), float(t_cpu)) != 0:
            raise ValueError("hybrid update failed")

    def state(self) -> dict:
        f, rg, rc = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        dr = np.zeros(self.ndev)
        self.s.lib.gcchem_b200_hybrid_state(self.h, ctypes.byref(f), ctypes.byref(rg),
                                            ctypes.byref(rc), _p(dr))
        return {"frac": f.value, "rate_gpu": rg.value, "rate_cpu": rc.value,
                "dev_rate": dr.tolist()}

    def step(self, batch, prev_nsteps, cpu_tail):
        """One hybrid step on a cost-ordered workloads.Batch (host arrays).
        cpu_tail(first, count, C, ISTAT, RSTAT, IERR) must solve columns
        first..first+count-1 in place.  Returns (C, ISTAT, RSTAT, IERR, info)."""
        n = batch.n
        C = np.array(batch.C, dtype=np.float64, order="F", copy=True)
        R = np.asfortranarray(batch.RCONST, dtype=np.float64)
        IC = np.asfortranarray(batch.ICNTRL, dtype=np.int32)
        RC = np.asfortranarray(batch.RCNTRL, dtype=np.float64)
        atol = np.ascontiguousarray(batch.ATOL, dtype=np.float64)
        rtol = np.ascontiguousarray(batch.RTOL, dtype=np.float64)
        prev = np.ascontiguousarray(prev_nsteps, dtype=np.int32)
        ist = np.zeros((8, n), np.int32, order="F")
        rst = np.zeros((3, n), np.float64, order="F")
        ierr = np.zeros(n, np.int32)
        errors = []

        def tail(first, count, _user):
            try:
                cpu_tail(first, count, C, ist, rst, ierr)
            except Exception as exc:   # noqa: BLE001 -- re-raised below
                errors.append(exc)

        fn = TAIL_FN(tail)
        ng, tg, tc = ctypes.c_int(), ctypes.c_double(), ctypes.c_double()
        rc = self.s.lib.gcchem_b200_hybrid_step(
            self.h, n, float(batch.Tstart), float(batch.Tend), _p(C), _p(R), _p(atol),
            _p(rtol), _p(IC), _p(RC), _p(prev), _p(ist), _p(rst), _p(ierr), fn, None,
            ctypes.byref(ng), ctypes.byref(tg), ctypes.byref(tc))
        if errors:
            raise errors[0]
        if rc != 0:
            raise RuntimeError(f"gcchem_b200_hybrid_step failed ({rc})")
        return C, ist, rst, ierr, {"n_gpu": ng.value, "t_gpu": tg.value, "t_cpu": tc.value}


def solver(mech: str = "fullchem", variant: str = "fma") -> Solver:
    key = (mech, variant)
    if key not in _CACHE:
        _CACHE[key] = Solver(mech, variant)
    return _CACHE[key]
