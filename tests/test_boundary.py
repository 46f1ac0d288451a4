"""Boundary behaviour of the C-ABI beyond the parity cases."""
import ctypes
import os
import subprocess
import sys

import numpy as np
import pytest


@pytest.mark.gpu
@pytest.mark.timeout(300)
def test_chunked_global_workspace_matches(pkg, orc):
    """GC_GPU_WORKSPACE=global + GC_GPU_CHUNK (the reference's low-memory mode,
    gc_gpu_batch_api.F90:227-343) gives the same cells, bit for bit; run in a
    child process because the mode is read when a device is first used."""
    code = r'''
import importlib, sys, numpy as np
sys.path[:0] = [".", "oracle", "geos-chem-gpu-hybrid_b200"]
pkg = importlib.import_module("geos-chem-gpu-hybrid_b200")
import oracle
b = pkg.workloads.plain_small(2500, seed=9)
b.ICNTRL[3, :] = 5000
s = pkg.solver("fullchem", "nofma")
assert s.workspace_slots(2500) == 1024, s.workspace_slots(2500)
C, ist, rst, ierr, *_ = s.integrate_batch(b)
rC, rist, rrst, rierr = oracle.integrate_batch(b)
assert np.array_equal(C.view(np.uint64), rC.view(np.uint64)) and np.array_equal(ist, rist)
print("ok")
'''
    env = dict(os.environ, GC_GPU_WORKSPACE="global", GC_GPU_CHUNK="1024",
               GCCHEM_B200_MODE="plain")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, "-c", code], cwd=root, env=env, capture_output=True,
                       text=True, timeout=280)
    assert r.returncode == 0 and "ok" in r.stdout, r.stderr[-2000:]


@pytest.mark.gpu
def test_device_selection_and_info(pkg):
    s = pkg.solver("fullchem", "fma")
    n, name = s.info()
    assert n >= 1 and "B200" in name
    assert s.set_device(0) == 0
    assert s.set_device(n + 7) == -1
    b = pkg.workloads.plain_small(3, seed=1)
    C, ist, rst, ierr, tt, tk = s.integrate_batch(b, dev=n + 7)
    assert (ierr == -99).all()
    C, ist, rst, ierr, tt, tk = s.integrate_batch(b, dev=0)
    assert (ierr == 1).all() and tt >= tk > 0.0


def _rank_main(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world)
    v = bench.max_over_ranks(10.0 * (rank + 1))
    dist.destroy_process_group()
    out.put((rank, v))


def test_replica_timing_is_max_over_ranks():
    """Two gloo ranks on the CPU: every rank sees the slowest rank's time."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29000 + os.getpid() % 1000
    ps = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = dict(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
    assert res == {0: 20.0, 1: 20.0}
