"""Every module of the package imports on a machine without a GPU."""
import importlib

import pytest


@pytest.mark.parametrize("mod", ["binding", "workloads", "build", "autotune", "adjoint", "chain",
                                 "mechanism.codegen", "mechanism.fortran_ir",
                                 "mechanism.extract", "mechanism.synthetic"])
def test_import(mod):
    importlib.import_module("geos-chem-gpu-hybrid_b200." + mod)
