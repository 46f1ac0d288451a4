"""Launch autotuner for the batched Rodas3 solve.

Picks, for one device / mechanism / arithmetic variant, the fastest of:

* the kernel: ``plain`` (one thread per cell, indexed KppDecomp with its
  dense row scratch, one launch over the batch), ``plain_fused`` (one thread
  per cell with the generated register-blocked LU), ``persistent``
  (resident grid draining the cost-ordered queue, generated register-blocked
  LU) or ``coop`` (one thread block per cell draining the same queue, the
  cell's factors and vectors in shared memory: the thread-per-cell versus
  block-cooperative choice);
* cells (threads) per block: 64, 128 or 256 (threads per cell for coop);
* resident blocks per SM the persistent grid assumes (occupancy maximum, or 1);
* for the plain kernels, the workspace layout: one launch over the whole
  batch, or the reference's low-memory global workspace in chunks of
  32,768 / 65,536 / 131,072 cells per launch (``CHUNKED``, for the large
  grids);
* for mechanisms factorised by the indexed KppDecomp (the synthetic one),
  where its row scratch lives: in the workspace (HBM) or in shared memory.

The persistent kernel's workspace is bounded by the resident threads
(~4.7 GB for fullchem) while a plain launch's grows with the batch, which
the capped sample does not show (it is smaller, and its cells take no warm
steps), so another candidate must beat the best persistent one by
``PREFER_PERSISTENT`` to be chosen.

Every candidate solves the same strided sample of the caller's batch with
the step count capped (ICNTRL(4) = ``cap``), so a candidate costs well under
a few seconds; throughput is measured with CUDA events.  The winner is
applied with gcchem_b200_set_launch / gcchem_b200_set_chunk and cached in a
JSON file (``$GCCHEM_B200_TUNE_CACHE`` or
``~/.cache/gcchem_b200/autotune.json``), keyed by device name, mechanism,
variant and candidate set.
"""
from __future__ import annotations

import json
import os
import time

import numpy as np

# (kernel, threads per block, persistent blocks per SM, plain cells per launch,
#  row scratch of the indexed factorisation)
CANDIDATES = [
    ("coop", 128, 0, 0, "global"), ("coop", 256, 0, 0, "global"),
    ("persistent", 128, 0, 0, "global"), ("persistent", 64, 0, 0, "global"),
    ("persistent", 256, 0, 0, "global"), ("persistent", 128, 1, 0, "global"),
    ("plain", 128, 0, 0, "global"), ("plain", 64, 0, 0, "global"),
    ("plain_fused", 128, 0, 0, "global"),
    # only for mechanisms without the fused LU (others reject these)
    ("persistent", 224, 0, 0, "shared"), ("persistent", 128, 0, 0, "shared"),
    ("plain", 224, 0, 0, "shared"),
]
# the large grids: layout and chunk size of the plain kernels against the
# persistent kernel's resident-thread workspace
CHUNKED = [
    ("coop", 128, 0, 0, "global"),
    ("persistent", 256, 0, 0, "global"), ("persistent", 128, 0, 0, "global"),
    ("plain_fused", 128, 0, 32768, "global"), ("plain_fused", 128, 0, 65536, "global"),
    ("plain_fused", 128, 0, 131072, "global"), ("plain_fused", 128, 0, 0, "global"),
    ("plain", 128, 0, 131072, "global"),
]
PREFER_PERSISTENT = 1.05


def cache_path() -> str:
    return os.environ.get("GCCHEM_B200_TUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "gcchem_b200",
                                       "autotune.json"))


def _key(solver, tag="default") -> str:
    import torch
    return f"{torch.cuda.get_device_name()}|{solver.mech}|{solver.variant}|{tag}"


def load_cached(solver, tag="default"):
    try:
        with open(cache_path()) as fh:
            return json.load(fh).get(_key(solver, tag))
    except (OSError, ValueError):
        return None


def _store(solver, entry, tag="default") -> None:
    path = cache_path()
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        data = {}
        if os.path.exists(path):
            with open(path) as fh:
                data = json.load(fh)
        data[_key(solver, tag)] = entry
        with open(path, "w") as fh:
            json.dump(data, fh, indent=1)
    except (OSError, ValueError):
        pass


def apply(solver, entry) -> None:
    from .binding import PLAIN, PERSISTENT, PLAIN_FUSED, COOP
    mode = {"plain": PLAIN, "plain_fused": PLAIN_FUSED, "coop": COOP}.get(entry["mode"],
                                                                          PERSISTENT)
    shared = entry.get("scratch", "global") == "shared"
    if not shared:
        solver.set_row_scratch(False)
    solver.set_launch(mode, entry["threads"], entry["blocks_per_sm"])
    if shared:
        solver.set_row_scratch(True)
    solver.set_chunk(entry.get("chunk", 0))


def _score(entry) -> float:
    """Throughput, with a bounded workspace (the persistent kernel's) or none
    (the cooperative kernel's) worth PREFER_PERSISTENT."""
    w = PREFER_PERSISTENT if entry["mode"] in ("persistent", "coop") else 1.0
    return entry["cells_per_s"] * w


def tune(solver, batch, sample_cells: int = 37888, cap: int = 24, use_cache: bool = True,
         candidates=CANDIDATES, tag: str = "default") -> dict:
    """Time the candidates on a sample of `batch`; apply and return the best
    ({"mode", "threads", "blocks_per_sm", "chunk", "cells_per_s", "table"})."""
    import torch
    from . import workloads
    if use_cache:
        hit = load_cached(solver, tag)
        if hit:
            apply(solver, hit)
            return dict(hit, cached=True)
    n = min(sample_cells, batch.n)
    idx = np.linspace(0, batch.n - 1, n).astype(np.int64)
    sub = workloads.subset(batch, idx)
    sub.ICNTRL[3, :] = cap
    dev = torch.device("cuda", torch.cuda.current_device())

    def up(a, dt):
        return torch.from_numpy(np.ascontiguousarray(a.T if a.ndim == 2 else a)).to(dev, dt)

    C0 = up(sub.C, torch.float64)
    R = up(sub.RCONST, torch.float64)
    A, T = up(sub.ATOL, torch.float64), up(sub.RTOL, torch.float64)
    IC, RC = up(sub.ICNTRL, torch.int32), up(sub.RCNTRL, torch.float64)
    order = torch.arange(n, dtype=torch.int32, device=dev)
    IST = torch.zeros((n, 8), dtype=torch.int32, device=dev)
    RST = torch.zeros((n, 3), dtype=torch.float64, device=dev)
    IE = torch.zeros(n, dtype=torch.int32, device=dev)
    table = []
    best = None
    for mode, threads, bps, chunk, scratch in candidates:
        entry = {"mode": mode, "threads": threads, "blocks_per_sm": bps, "chunk": chunk,
                 "scratch": scratch}
        try:
            apply(solver, entry)
            solver.reserve(n)
            times = []
            for rep in range(2):
                C = C0.clone()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                torch.cuda.synchronize()
                e0.record()
                solver.integrate_device(C, R, A, T, IC, RC, order, IST, RST, IE,
                                        sub.Tstart, sub.Tend)
                e1.record()
                torch.cuda.synchronize()
                times.append(e0.elapsed_time(e1))
            entry["cells_per_s"] = n / (min(times) * 1e-3)
        except (RuntimeError, ValueError) as exc:   # launch too large etc.
            entry["error"] = str(exc)
            entry["cells_per_s"] = 0.0
        table.append(entry)
        if best is None or _score(entry) > _score(best):
            best = dict(entry)
    result = dict(best, table=table, sample_cells=n, cap=cap, when=time.time(), tag=tag)
    apply(solver, result)
    _store(solver, result, tag)
    return result
