"""Build the solver libraries (and, for the tests, the CPU oracle).

For every mechanism: generate the statement lists from the mechanism tables
(``mechanism/codegen.py``) into ``_build/gen/<mech>/``, then compile
``lib/libgcchemgpu[_<mech>][_nofma].so`` for sm_100a with nvcc.  The FMA and
the --fmad=false variants build in parallel.  ``make`` keeps rebuilds
incremental.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
BUILD = os.path.join(ROOT, "_build")

if HERE not in sys.path:
    sys.path.insert(0, HERE)

from mechanism import codegen  # noqa: E402
from binding import lib_path  # noqa: E402

MECHANISMS = ("fullchem", "synth120")


def gen_dir(mech: str) -> str:
    return os.path.join(BUILD, "gen", mech)


def generate(mech: str) -> str:
    m = codegen.load(mech)
    codegen.generate(m, mech, gen_dir(mech))
    return gen_dir(mech)


def build_library(mech: str, variant: str, jobs: int = 8) -> str:
    out = lib_path(mech, variant)
    subprocess.run(["make", "-s", f"-j{jobs}", "-C", os.path.join(HERE, "csrc"),
                    f"MECH={mech}", f"GEN={gen_dir(mech)}", f"VARIANT={variant}",
                    f"OUT={out}"], check=True)
    return out


def build_all(mechanisms=MECHANISMS, variants=("fma", "nofma")) -> list[str]:
    for mech in mechanisms:
        generate(mech)
    jobs = [(m, v) for m in mechanisms for v in variants]
    with ThreadPoolExecutor(max_workers=len(jobs)) as ex:
        outs = list(ex.map(lambda mv: build_library(*mv), jobs))
    return outs


if __name__ == "__main__":
    for p in build_all():
        print(p)
