"""Benchmark of the batched Rodas3 chemistry solve on B200.

Workload (default): the full 4x5 grid batch, 72x46x72 = 238,464 fullchem
cells in FP64, one 1200 s chemistry step per bench step, on the persistent
cost-ordered queue kernel.  Seeded synthetic states (workloads.grid_4x5);
the reference's harvested cells are not available.

A step = restore the batch's initial concentrations + one solve of every
cell.  ``value`` is cells/s with all inputs resident in HBM (CUDA events on
the launching stream); ``e2e`` is the same metric through the legacy C-ABI
gc_gpu_integrate_batch with pinned host arrays, host->device and
device->host copies inside the timed region.  Inputs (C 0.68 GB, RCONST
2.0 GB) are larger than the 126 MB L2, so no flush is needed between steps.

Multi-GPU: the solve has no exchange step, so N ranks run N independent
replicas of the workload (``scaling: weak``); rank 0 prints the max-over-ranks
timing.

``--impl reference`` times the reference algorithm's CPU implementation
(the oracle restatement in oracle/, all host threads) on a bounded sample of
the same workload.
"""
from __future__ import annotations

import argparse
import importlib
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = "geos-chem-gpu-hybrid_b200"
sys.path.insert(0, ROOT)


def _pkg():
    return importlib.import_module(PKG)


def _oracle():
    odir = os.path.join(ROOT, "oracle")
    if odir not in sys.path:
        sys.path.insert(0, odir)
    import oracle
    return oracle


WORKLOADS = {
    "grid4x5": ("4x5 grid 72x46x72 = 238,464 fullchem cells, one 1200 s step",
                lambda wl: wl.grid_4x5(seed=0)),
    "grid2x25": ("2x2.5 grid 144x91x72 = 943,488 fullchem cells, one 1200 s step",
                 lambda wl: wl.grid_2x25(seed=0)),
    "plain4096": ("4,096 independent fullchem cells, one 1200 s step",
                  lambda wl: wl.plain_small(4096, seed=0)),
    "synth262k": ("synthetic stiff mechanism (120 species, 360 reactions), 262,144 cells, "
                  "one 1200 s step", lambda wl: wl.synthetic_stiff(262144, seed=0)),
}
MECH_OF = {"synth262k": "synth120"}
# the same grid one 1200 s chemistry step earlier: the sun 5 degrees further
# east (the Earth turns 5 degrees in 1200 s), so the day/night terminator sits
# one 4x5 column over; everything else is the same seeded state
PREVIOUS_STEP = {
    "grid4x5": lambda wl: wl.grid_4x5(seed=0, subsolar_lon=5.0),
    "grid2x25": lambda wl: wl.grid_2x25(seed=0, subsolar_lon=5.0),
}
MODES = {"plain": 0, "persistent": 1, "plain_fused": 2, "coop": 3}   # set_launch modes
METRIC = ("fullchem cells/s per B200 (1200 s step), batched vs plain at 1e-6 rel; "
          "adj/fwd cost")


def max_over_ranks(ms: float, device=None) -> float:
    """The slowest rank's time (all ranks take part; gloo or nccl)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(ms)], dtype=torch.float64,
                     device=device if device is not None else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def flops_per_cell(ist: np.ndarray, fc: dict) -> np.ndarray:
    """Algorithmic FP64 operations of each cell from its ISTAT counters:
    Nfun*F_fun + Njac*F_jac + Ndec*(F_lu+F_prep) + Nsol*F_sol + Nstp*F_vec."""
    ist = ist.astype(np.float64)
    return (ist[:, 0] * fc["fun"] + ist[:, 1] * fc["jac"] + ist[:, 5] * (fc["lu"] + fc["prep"])
            + ist[:, 6] * fc["solve"] + ist[:, 2] * fc["vec"])


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(smax)),
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_sample_size(orc, batch, target_s: float, nthreads: int,
                    mech: str = "fullchem") -> tuple[int, float]:
    """Cells the oracle solves in about target_s seconds on nthreads threads."""
    wl = _pkg().workloads
    n = batch.n
    probe = min(n, max(64, 16 * nthreads))
    idx = np.linspace(0, n - 1, probe).astype(np.int64)
    t0 = time.perf_counter()
    orc.integrate_batch(wl.subset(batch, idx), nthreads=nthreads, mech=mech)
    dt = time.perf_counter() - t0
    rate = probe / max(dt, 1e-6)
    return int(min(n, max(probe, rate * target_s))), rate


def run_cpu(orc, batch, ncells: int, nthreads: int, seed: int = 0,
            mech: str = "fullchem", keep: bool = False):
    """Solve a strided sample of ncells cells; return (cells/s, cells), and
    with keep=True also (sample columns, oracle C, ISTAT, RSTAT, IERR)."""
    wl = _pkg().workloads
    off = seed % max(1, batch.n // max(ncells, 1))
    idx = (np.linspace(0, batch.n - 1 - off, ncells).astype(np.int64) + off)
    sub = wl.subset(batch, idx)
    t0 = time.perf_counter()
    out = orc.integrate_batch(sub, nthreads=nthreads, mech=mech)
    dt = time.perf_counter() - t0
    if keep:
        return ncells / dt, ncells, idx, out
    return ncells / dt, ncells


def cpu_model() -> str:
    """The host CPU's model name (Linux /proc/cpuinfo), or the platform's."""
    try:
        with open("/proc/cpuinfo") as fh:
            for ln in fh:
                if ln.startswith("model name"):
                    return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform
    return platform.processor() or platform.machine()


def cpu_single_thread(orc, batch, seconds: float, mech: str = "fullchem") -> dict:
    """The oracle on one host thread, on a strided sample sized for about
    `seconds`: the figure comparable to a serial CPU build of the reference
    integrator (the reference quotes 1.9-2.8k cells/s for serial gfortran on
    its harvested cells, which take ~6 internal steps against ~78 here)."""
    ncells, _ = cpu_sample_size(orc, batch, seconds, 1, mech)
    rate, nc = run_cpu(orc, batch, ncells, 1, mech=mech)
    return {"value": rate, "unit": "cells/s", "cores": 1,
            "sample": f"{nc} cells strided over the batch, one 1200 s step"}


PARITY_RTOL = 1e-6


def parity_report(nvar: int, idx, ref, gpu_C, gpu_ist, gpu_ierr) -> dict:
    """Per-cell comparison of the GPU solve with the oracle on the sampled
    columns: relative difference of every variable species with the
    denominator floored at ATOL (1e-2 molecule cm^-3, the solver's absolute
    tolerance) and at 1e-20 (the floor of the reference's own comparison,
    standalone/kpp_batch.F90:262-272); solver failures on either side."""
    rC, rist, _, rierr = ref
    g = gpu_C[idx, :nvar].T                 # (NVAR, cells)
    r = rC[:nvar]
    d = np.abs(g - r)
    out = {"cells": int(len(idx)), "tolerance": PARITY_RTOL}
    for name, floor in (("floor_1e-2", 1e-2), ("floor_1e-20", 1e-20)):
        rel = d / np.maximum(np.abs(r), floor)
        per_cell = rel.max(axis=0)
        out[name] = {"max_rel": float(per_cell.max()),
                     "cells_over_tol": int((per_cell > PARITY_RTOL).sum())}
    out["gpu_failures"] = int((gpu_ierr[idx] != 1).sum())
    out["oracle_failures"] = int((rierr != 1).sum())
    out["ierr_equal"] = bool(np.array_equal(gpu_ierr[idx], rierr))
    out["istat_equal_cells"] = int((gpu_ist[idx] == rist.T).all(axis=1).sum())
    return out


def reference_arm(args, rank: int, world: int) -> None:
    """The reference algorithm's CPU implementation on the host cores."""
    if rank != 0:
        return
    pkg = _pkg()
    orc = _oracle()
    desc, make = WORKLOADS[args.workload]
    mech = MECH_OF.get(args.workload, "fullchem")
    batch = make(pkg.workloads)
    nthreads = os.cpu_count() or 1
    ncells, _ = cpu_sample_size(orc, batch, args.cpu_step_seconds, nthreads, mech)
    for w in range(args.warmup):
        run_cpu(orc, batch, max(64, ncells // 8), nthreads, seed=w, mech=mech)
    rates = []
    t0 = time.perf_counter()
    for k in range(args.steps):
        r, _ = run_cpu(orc, batch, ncells, nthreads, seed=100 + k, mech=mech)
        rates.append(r)
    wall = time.perf_counter() - t0
    value = float(args.steps * ncells / wall)
    line = {
        "metric": METRIC, "value": value, "unit": "cells/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": wall / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator)",
        "config": {"workload": desc, "sample_cells_per_step": ncells},
        "impl": "reference",
        "cpu_baseline": {"value": value, "unit": "cells/s", "cores": nthreads, "kind": "port",
                         "sample": f"{ncells} cells per step, strided over the {batch.n}-cell batch"},
        "e2e": {"value": value, "unit": "cells/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def to_dev(a, dtype, dev):
    import torch
    t = torch.from_numpy(np.ascontiguousarray(a.T if a.ndim == 2 else a))
    return t.to(device=dev, dtype=dtype)


def our_arm(args, rank: int, world: int) -> None:
    import torch
    import torch.distributed as dist
    pkg = _pkg()
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    mech = MECH_OF.get(args.workload, "fullchem")
    s = pkg.solver(mech, "fma")
    s.set_device(local)
    mode = MODES.get(args.mode, pkg.PERSISTENT)
    s.set_row_scratch(False)
    s.set_launch(mode, args.threads, args.blocks_per_sm)
    if args.row_scratch == "shared":
        s.set_row_scratch(True)

    desc, make = WORKLOADS[args.workload]
    batch = make(pkg.workloads)
    if args.cells:
        batch = pkg.workloads.subset(batch, np.arange(min(args.cells, batch.n)))
    if args.max_steps:
        batch.ICNTRL[3, :] = args.max_steps
    tuned = None
    if args.mode == "auto" and not args.profile_small:
        at = importlib.import_module(PKG + ".autotune")
        if args.workload == "grid2x25":
            # the large grid: workspace layout and chunk size are candidates too
            tuned = at.tune(s, batch, sample_cells=262144, cap=12, use_cache=False,
                            candidates=at.CHUNKED, tag="chunked")
        else:
            tuned = at.tune(s, batch, use_cache=False)
    n = batch.n
    C0 = to_dev(batch.C, torch.float64, dev)
    R = to_dev(batch.RCONST, torch.float64, dev)
    A = to_dev(batch.ATOL, torch.float64, dev)
    T = to_dev(batch.RTOL, torch.float64, dev)
    IC = to_dev(batch.ICNTRL, torch.int32, dev)
    RC = to_dev(batch.RCNTRL, torch.float64, dev)
    order = torch.arange(n, dtype=torch.int32, device=dev)
    C = torch.empty_like(C0)
    IST = torch.zeros((n, 8), dtype=torch.int32, device=dev)
    RST = torch.zeros((n, 3), dtype=torch.float64, device=dev)
    IE = torch.zeros(n, dtype=torch.int32, device=dev)
    s.reserve(n)
    stream = torch.cuda.current_stream()
    nfail = torch.zeros(2, dtype=torch.int32, device=dev)
    # retry tolerances: Classic/GCHP keep ATOL/RTOL, GEOS inflates both to
    # 1e-2 * KppTolScale (fullchem_mod.F90:736-742; KppTolScale = 1 here)
    if args.retry_tolerances == "geos":
        Ar = torch.full_like(A, 1.0e-2)
        Tr = torch.full_like(T, 1.0e-2)
    else:
        Ar, Tr = A, T

    def step():
        C.copy_(C0)
        if args.retry:
            # the model's retry protocol on the device: failed cells reset and
            # solved again with Hstart = 0 and the retry tolerances (Classic:
            # the same ATOL/RTOL, fullchem_mod.F90:741-742)
            s.integrate_device_retry(C, R, A, T, Ar, Tr, IC, RC, order, IST, RST, IE, nfail,
                                     batch.Tstart, batch.Tend, stream=stream)
        else:
            s.integrate_device(C, R, A, T, IC, RC, order, IST, RST, IE,
                               batch.Tstart, batch.Tend, stream=stream)

    chain = None
    if args.chain:
        # config-3 form: a bench step replays one CUDA graph holding
        # [restore initial state, `chain` consecutive chemistry steps with the
        # state kept on the device]
        chain_mod = importlib.import_module(PKG + ".chain")
        chain = chain_mod.Chain(s, batch, device=dev)
        cC0, cRC0 = chain.C.clone(), chain.RCNTRL.clone()
        cord0 = chain.order.clone()

        def restore(st=None):
            with torch.cuda.stream(st or torch.cuda.current_stream()):
                chain.C.copy_(cC0)
                chain.RCNTRL.copy_(cRC0)
                chain.order.copy_(cord0)

        chain.step()                     # eager setup step
        torch.cuda.synchronize()
        gstream = torch.cuda.Stream()
        gstream.wait_stream(torch.cuda.current_stream())
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.stream(gstream):
            with torch.cuda.graph(graph, stream=gstream):
                restore(gstream)
                for _ in range(args.chain):
                    chain.step(stream=gstream)
        torch.cuda.current_stream().wait_stream(gstream)
        IST, IE = chain.ISTAT, chain.IERR

        def step():  # noqa: F811
            graph.replay()

    def keys_of(b) -> "torch.Tensor":
        """ISTAT(3) of one solve of batch b (same controls), on the device."""
        bC = to_dev(b.C, torch.float64, dev)
        bR = to_dev(b.RCONST, torch.float64, dev)
        s.integrate_device(bC, bR, A, T, IC, RC, order, IST, RST, IE, b.Tstart, b.Tend,
                           stream=stream)
        k = IST[:, 2].contiguous().clone()
        torch.cuda.synchronize()
        del bC, bR
        return k

    order_desc = "stock cell order"
    foresight_order = None
    if not args.chain and args.order != "stock":
        # the model's pre-scan sort: the previous chemistry step's ISTAT(3),
        # most expensive first, stable (fullchem_mod.F90:906-960), on the device
        if args.order == "previous-step" and args.workload in PREVIOUS_STEP:
            prev = PREVIOUS_STEP[args.workload](pkg.workloads)
            if args.cells:
                prev = pkg.workloads.subset(prev, np.arange(n))
            if args.max_steps:
                prev.ICNTRL[3, :] = args.max_steps
            order.copy_(s.cost_order(keys_of(prev)))
            del prev
            order_desc = ("previous-step: descending Nstp of the previous chemistry step "
                          "(same grid with the sun 5 deg east, i.e. 1200 s earlier), "
                          "device stable sort")
        else:
            order.copy_(s.cost_order(keys_of(batch)))
            order_desc = ("foresight: descending Nstp of a solve of the very inputs timed "
                          "(no model has this order), device stable sort")
        torch.cuda.synchronize()
        if order_desc.startswith("previous-step"):
            foresight_order = s.cost_order(keys_of(batch)).clone()
            torch.cuda.synchronize()

    if args.profile_small:
        # one warm-up launch + one launch for ncu (-s 1 -c 1 on the solver kernel)
        step()
        step()
        torch.cuda.synchronize()
        print(json.dumps({"profile_case": desc, "cells": n, "max_steps": args.max_steps}))
        return

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    sampler = ClockSampler(local)
    sampler.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    ms = e0.elapsed_time(e1)
    if world > 1:
        ms = max_over_ranks(ms, dev)
        dist.barrier()
    ms_per_step = ms / args.steps
    value = world * n * max(1, args.chain) / (ms_per_step * 1e-3)

    # per-cell results of the last timed step
    ist = IST.cpu().numpy()
    ierr = IE.cpu().numpy()
    steps_per_cell = float(ist[:, 2].mean())

    from mechanism import codegen  # noqa: E402  (package dir on sys.path below)
    fc = codegen.flop_counts(codegen.load(mech))
    flops = float(flops_per_cell(ist, fc).sum())

    if chain is not None:
        line = {
            "metric": METRIC, "value": value, "unit": "cells/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator)",
            "config": {"workload": desc, "cells": n,
                       "chain": f"{args.chain} consecutive chemistry steps per CUDA-graph replay, "
                                "state on device (clamp, Hnew warm start, cost re-sort)",
                       "mean_internal_steps_per_cell_last_step": steps_per_cell,
                       "failed_cells_last_step": int((ierr != 1).sum())},
            "gpu_launches": args.steps * args.chain * (
                launches_per_step(s, n, MODES[tuned["mode"]] if tuned else mode) +
                cost_order_launches(n)), "clocks": clocks,
        }
        if tuned:
            line["config"]["kernel"] = (f"{tuned['mode']} (autotuned: {tuned['threads']} "
                                        f"threads/block, cells per launch "
                                        f"{tuned.get('chunk') or 'all'})")
            line["config"]["autotune_table"] = [
                {k: e.get(k) for k in ("mode", "threads", "blocks_per_sm", "chunk", "cells_per_s")}
                for e in tuned["table"]]
        if rank == 0 and world == 1 and not args.skip_cpu:
            cpu, par = chain_cpu_baseline(pkg, batch, args, chain.C.cpu().numpy(),
                                          IE.cpu().numpy(), s.nvar)
            line["cpu_baseline"] = cpu
            line["parity"] = par
        if rank == 0:
            print(json.dumps(line), flush=True)
        return

    # kernel-only time of the solve (no C restore) for the roofline
    ek0 = torch.cuda.Event(enable_timing=True)
    ek1 = torch.cuda.Event(enable_timing=True)
    C.copy_(C0)
    torch.cuda.synchronize()
    ek0.record(stream)
    s.integrate_device(C, R, A, T, IC, RC, order, IST, RST, IE, batch.Tstart, batch.Tend,
                       stream=stream)
    ek1.record(stream)
    torch.cuda.synchronize()
    kernel_ms = ek0.elapsed_time(ek1)
    peak = s.fp64_peak_tflops()
    achieved = flops / (kernel_ms * 1e-3) / 1e12
    # DRAM traffic of the persistent kernel measured with ncu
    # (dram__bytes_read.sum + dram__bytes_write.sum, one pass) on the first
    # 151,552 cells of the 4x5 grid solved in full (--profile-small --cells
    # 151552 --mode persistent --threads 128: 10.93 TB over 12,164,043 internal
    # steps), per internal step of a cell, scaled here by this launch's counted
    # steps
    dram_per_cell_step = 0.899e6
    kernel_mode = tuned["mode"] if tuned else args.mode
    traffic = dram_per_cell_step * float(ist[:, 2].sum())
    traffic_ok = kernel_mode == "persistent" and mech == "fullchem"
    hbm_peak = 6547.5
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:  # noqa: SIM115
            hbm_peak = float(json.load(fh)["hbm_gbs"])
    except (OSError, ValueError, KeyError):
        pass

    line = {
        "metric": METRIC, "value": value, "unit": "cells/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator)",
        "config": {"workload": desc, "cells": n,
                   "kernel": (f"{tuned['mode']} (autotuned: {tuned['threads']} threads/block, "
                              f"blocks/SM {tuned['blocks_per_sm'] or 'max'}, "
                              f"cells per launch {tuned.get('chunk') or 'all'})") if tuned
                   else args.mode,
                   "autotune_table": ([{k: e.get(k) for k in ("mode", "threads", "blocks_per_sm",
                                                              "chunk", "cells_per_s")}
                                       for e in tuned["table"]] if tuned else None),
                   "queue_order": order_desc,
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                   "l2": "inputs (C 0.68 GB + RCONST 2.0 GB) larger than L2, no flush",
                   "mean_internal_steps_per_cell": steps_per_cell,
                   "cell_steps_per_s": value * steps_per_cell,
                   "failed_cells": int((ierr != 1).sum()),
                   "retry": ({"protocol": "device retry of failed cells (Hstart 0, retry "
                                          + ("tolerances 1e-2, the GEOS setting)"
                                             if args.retry_tolerances == "geos" else
                                             "tolerances = ATOL/RTOL, the Classic setting)"),
                              "failed_first_attempt": int(nfail[0].item()),
                              "failed_both": int(nfail[1].item())} if args.retry else None)},
        "gpu_launches": args.steps * launches_per_step(
            s, n, MODES[tuned["mode"]] if tuned else mode),
        "clocks": clocks,
        "roofline": {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak if peak > 0 else None,
                     "traffic": traffic if traffic_ok else None,
                     "traffic_note": "bytes per launch, ncu per-cell-step DRAM bytes of the "
                                     "persistent kernel x this launch's internal steps",
                     "hbm_implied": ({"achieved_gbs": traffic / (kernel_ms * 1e-3) / 1e9,
                                      "peak_gbs": hbm_peak,
                                      "frac": traffic / (kernel_ms * 1e-3) / 1e9 / hbm_peak}
                                     if traffic_ok else None),
                     "peak_source": "FP64 FMA probe kernel measured in this run "
                                    "(MEASURED_PEAKS.json has no FP64 figure)",
                     "flops_per_launch": flops, "kernel_ms": kernel_ms},
    }
    # per-cell results of the timed solve, for the parity check below
    gpu_C = C.cpu().numpy()
    gpu_ist = IST.cpu().numpy()
    gpu_ierr = IE.cpu().numpy()
    if rank == 0 and args.extras and not args.profile_small:
        line["batching"] = batching_measure(pkg, s, args, tuned, order, foresight_order,
                                            C, C0, R, A, T, IC, RC, IST, RST, IE, batch,
                                            value, stream)
    if rank == 0 and args.adjoint and mech == "fullchem":
        line["adjoint"] = adjoint_measure(pkg, s, args)
    if rank == 0 and not args.skip_e2e:
        line["e2e"] = e2e_measure(s, batch, args, order.cpu().numpy() + 1)
    if rank == 0 and world == 1 and not args.skip_cpu:
        orc = _oracle()
        nthreads = os.cpu_count() or 1
        ncells, _ = cpu_sample_size(orc, batch, args.cpu_step_seconds, nthreads, mech)
        rate, nc, idx, ref = run_cpu(orc, batch, ncells, nthreads, mech=mech, keep=True)
        line["cpu_baseline"] = {"value": rate, "unit": "cells/s", "cores": nthreads,
                                "kind": "port", "cpu_model": cpu_model(),
                                "sample": f"{nc} cells strided over the batch, one 1200 s step",
                                "single_thread": cpu_single_thread(
                                    orc, batch, min(3.0, args.cpu_step_seconds), mech)}
        # the same sampled cells, solved by the GPU in the last timed step
        line["parity"] = parity_report(s.nvar, idx, ref, gpu_C, gpu_ist, gpu_ierr)
    if rank == 0:
        print(json.dumps(line), flush=True)


def chain_cpu_baseline(pkg, batch, args, gpu_C, gpu_ierr, nvar):
    """The chained workload on the host: the oracle runs the same
    `args.chain` chemistry steps (clamp negatives, warm start Hstart = Hnew)
    on a strided sample of the grid, timed on all host cores; its final
    states are the parity reference for the GPU chain's cells."""
    orc = _oracle()
    wl = pkg.workloads
    nthreads = os.cpu_count() or 1
    ncells, _ = cpu_sample_size(orc, batch, args.cpu_step_seconds / 2, nthreads)
    idx = np.linspace(0, batch.n - 1, ncells).astype(np.int64)
    sub = wl.subset(batch, idx)
    t0 = time.perf_counter()
    for _ in range(args.chain):
        C, ist, rst, ierr = orc.integrate_batch(sub, nthreads=nthreads)
        sub.C = np.asfortranarray(np.maximum(C, 0.0))
        sub.RCNTRL[2, :] = rst[2]
    dt = time.perf_counter() - t0
    cpu = {"value": len(idx) * args.chain / dt, "unit": "cells/s per chemistry step",
           "cores": nthreads, "kind": "port",
           "sample": f"{len(idx)} cells strided over the batch, {args.chain} chained steps"}
    par = parity_report(nvar, idx, (sub.C, ist, rst, ierr), gpu_C,
                        np.zeros((gpu_C.shape[0], 8), np.int32), gpu_ierr)
    par.pop("istat_equal_cells", None)
    par["steps"] = args.chain
    return cpu, par


def batching_measure(pkg, s, args, tuned, order, foresight_order, C, C0, R, A, T, IC, RC,
                     IST, RST, IE, batch, headline, stream) -> dict:
    """What the persistent queue and the cost order gain, like for like: the
    same workload solved once more by (a) the persistent kernel with the
    foresight order and with the stock cell order, and (b) one thread per
    cell with the persistent kernel's own arithmetic (generated fused
    factorisation, pivot reciprocals) in the headline order and in stock
    order.  One timed solve each (CUDA events), after the headline timing."""
    import torch
    n = batch.n
    stock = torch.arange(n, dtype=torch.int32, device=order.device)
    mode_p = MODES[tuned["mode"]] if tuned else MODES[args.mode]
    thr = tuned["threads"] if tuned else args.threads
    bps = tuned["blocks_per_sm"] if tuned else args.blocks_per_sm

    s.set_row_scratch(False)

    def one(mode, threads, ordr) -> float:
        s.set_launch(mode, threads, bps if mode == pkg.PERSISTENT else 0)
        C.copy_(C0)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        s.integrate_device(C, R, A, T, IC, RC, ordr, IST, RST, IE, batch.Tstart, batch.Tend,
                           stream=stream)
        e1.record(stream)
        torch.cuda.synchronize()
        return n / (e0.elapsed_time(e1) * 1e-3)

    pthr = thr if (tuned and tuned["mode"] == "persistent") else 256
    out = {"headline": headline, "headline_kernel": tuned["mode"] if tuned else args.mode}
    out["persistent_headline_order"] = one(pkg.PERSISTENT, pthr, order)
    if foresight_order is not None:
        out["persistent_foresight_order"] = one(pkg.PERSISTENT, pthr, foresight_order)
    out["persistent_stock_order"] = one(pkg.PERSISTENT, pthr, stock)
    # the block-cooperative kernel (one block of 128 threads per cell) on the
    # mechanism it targets; on fullchem it is timed by the autotuner's sample
    if MECH_OF.get(args.workload) == "synth120" or (tuned and tuned["mode"] == "coop"):
        try:
            out["coop_headline_order"] = one(pkg.COOP, 128, order)
            out["coop_stock_order"] = one(pkg.COOP, 128, stock)
        except ValueError:
            pass   # no cooperative tables for this mechanism
    out["plain_same_lu_headline_order"] = one(pkg.PLAIN_FUSED, 128, order)
    out["plain_same_lu_stock_order"] = one(pkg.PLAIN_FUSED, 128, stock)
    if args.extras_reference_mapping:
        out["plain_reference_mapping_stock_order"] = one(pkg.PLAIN, 128, stock)
        out["vs_plain_reference_mapping"] = (out["persistent_headline_order"]
                                             / out["plain_reference_mapping_stock_order"])
    out["vs_plain_same_lu"] = out["persistent_headline_order"] / out["plain_same_lu_stock_order"]
    out["vs_plain_same_lu_same_order"] = (out["persistent_headline_order"]
                                          / out["plain_same_lu_headline_order"])
    if "coop_headline_order" in out:
        out["coop_vs_persistent_headline_order"] = (out["coop_headline_order"]
                                                    / out["persistent_headline_order"])
    out["note"] = ("persistent = the cost-ordered queue kernel; coop = one thread block per "
                   "cell draining the same queue, cell state in shared memory; "
                   "plain_same_lu = one thread per "
                   "cell for the whole solve with the persistent kernel's arithmetic; "
                   "plain_reference_mapping = one thread per cell with the reference's indexed "
                   "KppDecomp; 128 threads per block for the plain kernels; ratios are the "
                   "persistent kernel's cells/s in the headline order over the plain ones")
    if tuned:
        importlib.import_module(PKG + ".autotune").apply(s, tuned)
    else:
        s.set_launch(mode_p, thr, bps)
    return out


def adjoint_measure(pkg, s, args) -> dict:
    """Adjoint workload: 65,536 independent cells, one 1200 s step; cost of
    the discrete adjoint (backward pass through the recorded steps) against
    the checkpointed forward solve, both timed with CUDA events."""
    import torch
    adj = importlib.import_module(PKG + ".adjoint")
    n = args.adjoint_cells
    b = pkg.workloads.plain_small(n, seed=4)
    dev = torch.device("cuda", torch.cuda.current_device())
    ctl = adj.Controls(b, dev)
    C0 = to_dev(b.C, torch.float64, dev)
    R = to_dev(b.RCONST, torch.float64, dev)
    order = torch.arange(n, dtype=torch.int32, device=dev)
    IST = torch.zeros((n, 8), dtype=torch.int32, device=dev)
    RST = torch.zeros((n, 3), dtype=torch.float64, device=dev)
    IE = torch.zeros(n, dtype=torch.int32, device=dev)
    # a plain solve first: the largest accepted-step count sizes the checkpoints
    C = C0.clone()
    s.integrate_device(C, R, ctl.ATOL, ctl.RTOL, ctl.ICNTRL, ctl.RCNTRL, order, IST, RST, IE)
    torch.cuda.synchronize()
    ckmax = int(IST[:, 3].max().item())
    ckpt = torch.empty(n * ckmax * (s.nvar + 1), dtype=torch.float64, device=dev)
    lam = torch.zeros_like(C0)
    lam[:, :s.nvar] = torch.from_numpy(adj.loss_weights(n, s.nvar, seed=4)).to(dev)
    gC0, gK = torch.empty_like(C0), torch.empty_like(R)
    aerr = torch.zeros(n, dtype=torch.int32, device=dev)
    fwd, bwd = [], []
    for rep in range(2):
        C = C0.clone()
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        torch.cuda.synchronize()
        e0.record()
        s.integrate_device_ckpt(C, R, ctl.ATOL, ctl.RTOL, ctl.ICNTRL, ctl.RCNTRL, order, IST,
                                RST, IE, ckpt, ckmax)
        e1.record()
        s.adjoint_device(C0, R, IST, ckpt, ckmax, lam, gC0, gK, aerr)
        e2.record()
        torch.cuda.synchronize()
        fwd.append(e0.elapsed_time(e1))
        bwd.append(e1.elapsed_time(e2))
    f, a = min(fwd), min(bwd)
    ok = int((aerr == 1).sum().item())
    del ckpt
    torch.cuda.empty_cache()
    return {"workload": f"{n} independent fullchem cells, one 1200 s step, gradients w.r.t. C0 "
                        "and ln RCONST of a weighted sum of final concentrations",
            "forward_ms": f, "adjoint_ms": a, "adj_over_fwd": a / f,
            "cells_ok": ok, "checkpoint_steps": ckmax,
            "mean_accepted_steps": float(IST[:, 3].double().mean().item())}


def phase_report(args) -> None:
    """Per-building-block cost (gcchem_b200_phase_ms): `reps` calls of each
    block by one full resident wave of threads on synthetic data."""
    pkg = _pkg()
    mech = MECH_OF.get(args.workload, "fullchem")
    s = pkg.solver(mech, "fma")
    slots = s.workspace_slots(10 ** 7)
    out = {}
    for ph, name in enumerate(["fun", "jac", "prep_lu_fused", "solve", "prep_kppdecomp_indexed"]):
        ms = s.phase_ms(ph, slots, 4)
        if ms == -2.0:
            continue                      # no fused LU generated for this mechanism
        out[name] = {"ms_per_call": ms / 4, "calls_per_s": slots * 4 / (ms * 1e-3)}
    print(json.dumps({"mechanism": mech, "phases": out, "threads": slots}), flush=True)


def cost_order_launches(n: int) -> int:
    """Kernels one device cost sort of n keys launches (fill, tile sort, one
    per global stride plus a tile merge per size above the tile, extract)."""
    n2, k, count = 2048, 4096, 3
    while n2 < n:
        n2 <<= 1
    while k <= n2:
        count += (k.bit_length() - 1) - 11 + 1
        k <<= 1
    return count


def launches_per_step(s, n: int, mode: int) -> int:
    if mode in (0, 2):
        slots = s.workspace_slots(n)
        return (n + slots - 1) // slots
    return 1


def e2e_measure(s, batch, args, perm_host) -> dict:
    """cells/s through gc_gpu_integrate_batch on pinned host arrays."""
    import torch
    import ctypes
    n = batch.n

    def pinned(a, dtype):
        t = torch.empty(a.shape[::-1], dtype=dtype, pin_memory=True)
        t.numpy()[...] = a.T
        return t

    C0 = pinned(batch.C, torch.float64)
    C = pinned(batch.C, torch.float64)
    R = pinned(batch.RCONST, torch.float64)
    IC = pinned(batch.ICNTRL, torch.int32)
    RC = pinned(batch.RCNTRL, torch.float64)
    perm = torch.from_numpy(np.ascontiguousarray(perm_host, dtype=np.int32)).pin_memory()
    ist = torch.zeros((n, 8), dtype=torch.int32).pin_memory()
    rst = torch.zeros((n, 3), dtype=torch.float64).pin_memory()
    ierr = torch.zeros(n, dtype=torch.int32).pin_memory()
    atol = torch.from_numpy(np.ascontiguousarray(batch.ATOL))
    rtol = torch.from_numpy(np.ascontiguousarray(batch.RTOL))
    tt, tk = ctypes.c_double(), ctypes.c_double()

    def call():
        C.copy_(C0)
        s.lib.gc_gpu_integrate_batch(
            n, float(batch.Tstart), float(batch.Tend), C.data_ptr(), R.data_ptr(),
            atol.data_ptr(), rtol.data_ptr(), IC.data_ptr(), RC.data_ptr(), perm.data_ptr(),
            ist.data_ptr(), rst.data_ptr(), ierr.data_ptr(), ctypes.byref(tt), ctypes.byref(tk))

    call()   # warm-up (buffers grow once)
    ksteps = max(1, args.e2e_steps)
    t0 = time.perf_counter()
    for _ in range(ksteps):
        call()
    wall = time.perf_counter() - t0
    # the same call on ordinary (pageable) host arrays, as a Fortran caller
    # passes its batch arrays
    pC0 = np.asfortranarray(batch.C)
    pC = pC0.copy(order="F")
    pR = np.asfortranarray(batch.RCONST)
    pIC = np.asfortranarray(batch.ICNTRL, dtype=np.int32)
    pRC = np.asfortranarray(batch.RCNTRL)
    pperm = np.ascontiguousarray(perm_host, dtype=np.int32)
    pist = np.zeros((8, n), np.int32, order="F")
    prst = np.zeros((3, n), np.float64, order="F")
    pierr = np.zeros(n, np.int32)

    def vp(a):
        return a.ctypes.data_as(ctypes.c_void_p)

    pC[...] = pC0
    t1 = time.perf_counter()
    s.lib.gc_gpu_integrate_batch(
        n, float(batch.Tstart), float(batch.Tend), vp(pC), vp(pR), atol.data_ptr(),
        rtol.data_ptr(), vp(pIC), vp(pRC), vp(pperm), vp(pist), vp(prst), vp(pierr),
        ctypes.byref(tt), ctypes.byref(tk))
    wall_pageable = time.perf_counter() - t1
    h2d = (C.numel() + R.numel() + RC.numel() + atol.numel() + rtol.numel()) * 8 + \
        (IC.numel() + perm.numel()) * 4
    d2h = (C.numel() + rst.numel()) * 8 + (ist.numel() + ierr.numel()) * 4
    return {"value": ksteps * n / wall, "unit": "cells/s", "h2d_bytes_per_step": int(h2d),
            "d2h_bytes_per_step": int(d2h), "steps": ksteps,
            "api": "gc_gpu_integrate_batch (pinned host arrays)",
            "failed_cells": int((ierr.numpy() != 1).sum()),
            "pageable": {"value": n / wall_pageable, "unit": "cells/s", "steps": 1,
                         "api": "gc_gpu_integrate_batch (ordinary pageable numpy arrays)",
                         "failed_cells": int((pierr != 1).sum())}}


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="grid4x5")
    ap.add_argument("--mode", choices=["auto", "persistent", "plain", "plain_fused", "coop"],
                    default="auto",
                    help="auto: the autotuner picks kernel and block size on a capped "
                         "sample of the workload before timing")
    ap.add_argument("--order", choices=["previous-step", "foresight", "stock"],
                    default="previous-step",
                    help="queue order: by the previous chemistry step's step counts (grid "
                         "workloads; others fall back to foresight), by a solve of the very "
                         "inputs timed, or cell order")
    ap.add_argument("--extras-reference-mapping", action=argparse.BooleanOptionalAction,
                    default=True,
                    help="with --extras, also time the reference's own mapping (one thread per "
                         "cell, indexed KppDecomp) in stock order")
    ap.add_argument("--retry", action="store_true",
                    help="solve through the model's retry protocol on the device")
    ap.add_argument("--retry-tolerances", choices=["classic", "geos"], default="classic",
                    help="retry with ATOL/RTOL (Classic, GCHP) or with 1e-2 (GEOS)")
    ap.add_argument("--extras", action=argparse.BooleanOptionalAction, default=True,
                    help="also time the other queue orders and the plain one-thread-per-cell "
                         "kernel with the same arithmetic")
    ap.add_argument("--threads", type=int, default=0)
    ap.add_argument("--row-scratch", choices=["global", "shared"], default="global",
                    help="indexed factorisation's row scratch (mechanisms without the fused "
                         "LU): workspace or shared memory")
    ap.add_argument("--blocks-per-sm", type=int, default=0)
    ap.add_argument("--cells", type=int, default=0, help="use the first N cells only")
    ap.add_argument("--max-steps", type=int, default=0, help="ICNTRL(4) override (profiling)")
    ap.add_argument("--profile-small", action="store_true",
                    help="two solver launches of the workload, for an ncu capture")
    ap.add_argument("--chain", type=int, default=0,
                    help="K > 0: each bench step replays a CUDA graph of K chained "
                         "chemistry steps with the state kept on the device")
    ap.add_argument("--adjoint", action=argparse.BooleanOptionalAction, default=True,
                    help="also time the discrete adjoint against its checkpointed forward")
    ap.add_argument("--adjoint-cells", type=int, default=65536)
    ap.add_argument("--phases", action="store_true",
                    help="time the solver's building blocks separately and exit")
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--skip-e2e", action="store_true")
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--cpu-step-seconds", type=float, default=10.0)
    args = ap.parse_args(argv)
    sys.path.insert(0, os.path.join(ROOT, PKG))

    if args.phases:
        phase_report(args)
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        reference_arm(args, rank, world)
        return
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    try:
        our_arm(args, rank, world)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
