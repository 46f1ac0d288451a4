"""B200 batched Rodas3 gas-phase chemistry solver (GEOS-Chem fullchem KPP).

A drop-in for the batch-solve entry that fullchem_mod.F90 calls through
libgcchemgpu.so (gc_gpu_integrate_batch[_dev], gc_gpu_selftest, gc_gpu_info,
gc_gpu_set_device).  The compute path is the CUDA library in ``lib/``;
this package holds the mechanism generator, the ctypes/PyTorch binding and
the seeded workload generators.  The directory name is not a Python
identifier, so import it with ``importlib.import_module``.
"""
from . import binding, workloads  # noqa: F401
from .binding import Solver, solver, Hybrid, PLAIN, PERSISTENT, PLAIN_FUSED, COOP  # noqa: F401

__all__ = ["binding", "workloads", "Solver", "solver", "Hybrid", "PLAIN", "PERSISTENT", "PLAIN_FUSED", "COOP"]
