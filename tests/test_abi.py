"""The C-ABI library loads without a GPU and exports every symbol that
include/gcchem_gpu.h declares (no compute calls here)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "gcchem_gpu.h")


def declared_symbols():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(gc_gpu_\w+|gcchem_b200_\w+)\s*\(", txt)))


def test_header_declares_reference_entry_points():
    syms = declared_symbols()
    for s in ("gc_gpu_integrate_batch", "gc_gpu_integrate_batch_dev", "gc_gpu_selftest",
              "gc_gpu_info", "gc_gpu_set_device"):
        assert s in syms


@pytest.mark.parametrize("variant", ["fma", "nofma"])
def test_library_exports_header(pkg, variant):
    path = pkg.binding.lib_path("fullchem", variant)
    assert os.path.exists(path), f"{path} not built"
    lib = ctypes.CDLL(path)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_library_sizes_without_gpu(pkg):
    s = pkg.binding.Solver("fullchem", "fma")
    assert (s.nvar, s.nfix, s.nreact, s.nnz) == (353, 3, 1058, 5683)
    assert s.bytes_per_slot() > 0
