"""Benchmark: J-V curves per second of the batched steady-state solve on B200.

    python bench.py [--gpus N --steps K --warmup W] [--impl ours|reference] [--precision fp64]
                    [--workload curves|uneven|adjoint|impedance|build|transient]
    python -m torch.distributed.run --nproc-per-node N ... bench.py --gpus N ...

Workload: the drawn J-V curves — 16384 devices per GPU drawn from seed 20261203 (grid
NP = 400, 61 voltages from -0.2 to 1.3 V; half pre-biased at 1.0 V with their ions frozen, half
with free ions; interface and bulk traps, doping and ion densities drawn), synthetic SIMsalabim
inputs built by `jaxdd_b200.workloads`. One step = one `solve_batch` of the whole batch (every
device's full J-V curve). Devices are independent: with N GPUs every rank solves its own 16384
(weak scaling, no collective on the data path; the barrier and max-over-ranks timing only).

Reports (one JSON line, rank 0): `value` (curves/s, inputs resident on the GPU, CUDA events),
`e2e` (the same through the C ABI from pinned host buffers, copies in the timed region),
`roofline` (the kernel's algorithmic bytes per launch over its event time, against the measured
HBM copy bandwidth), `cpu_baseline` (the compiled C++ restatement of the FP64 oracle on one
core, a bounded sample of the same workload), `parity` (a fixed-stride sample of the timed
launch's own curves against that restatement), clocks sampled during the timed region.

`--workload uneven`: uneven grids in FP64 — 32768 devices per GPU in one launch,
each with its own grid size NP ~ U{150..900} and voltage count Nv ~ U{21..121} over -0.2..1.3 V
(otherwise the same draws).

`--impl reference`: jaxdd itself needs JAX, which is not installed; its CPU path is stood in for
by the compiled C++ restatement of its FP64 solve_batch (oracle/dd_cpu.cpp, pinned to the NumPy
oracle), one single-threaded process per host core, each solving batch 2 of the same workload
(jaxdd benchmarks/run.py's protocol).
"""

from __future__ import annotations

import argparse
import json
import math
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "J-V curves/s on 1 B200, mixed vs FP64 at 1e-6 of J scale; adjoint grads/s"
DEVICES_PER_GPU = 16384
NP = 400
CHUNK = 512  # devices per build task (a multiple of 32)
#: which kernel build profiles/traffic.json must describe for its traffic to be reported
KERNEL_TAG = "twisted two-thread fused Newton, shared-memory staged record, specialised batch instantiation"
# Kernel launches of one dd_solve / dd_solve_states in batch mode with the exact Bernoulli
# function: the specialised solve kernel, then the generic one for the lanes with the
# differential current (it returns at once for the others).
SOLVE_LAUNCHES = 2


def traffic_entry(precision: str, workload: str, devices: int, npts: int) -> dict | None:
    """The ncu capture of the solve kernel's DRAM traffic per launch (profiles/traffic.json) for
    this kernel build (KERNEL_TAG), precision and workload, or None when none matches."""
    try:
        rec = json.loads((ROOT / "profiles" / "traffic.json").read_text())
    except (OSError, ValueError):
        return None
    entry = rec.get(f"solve_kernel_{precision}_{workload}")
    if (not entry or entry.get("devices") != devices or entry.get("NP") != npts
            or KERNEL_TAG not in entry.get("kernel", "")):
        return None
    return entry


def _peaks() -> tuple[float, str]:
    try:
        data = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
        return float(data["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def _build_chunk(args):
    """Build and pack the drawn workload's devices `indices` (a pool worker); `uneven`: each
    device its own grid size."""
    indices, uneven, npts = args
    os.environ.setdefault("OMP_NUM_THREADS", "1")
    from jaxdd_b200.batch import prepare
    from jaxdd_b200.workloads import RAGGED_NP, drawn_device
    devs = [drawn_device(int(k), NP=RAGGED_NP if uneven else npts) for k in indices]
    return prepare(devs, ragged=uneven)


def build_workload(n: int, start: int, procs: int, uneven: bool = False, npts: int = NP):
    """The packed batch of devices [start, start + n), built in `procs` spawned processes (before
    any CUDA call in this one). `uneven` (the uneven workload): devices ordered by grid size,
    then voltage count, so that a warp's lanes do alike work; returns the batch, each device's
    voltage count (None for the fixed-size workload) and each device's draw index in the
    batch's order."""
    from jaxdd_b200.batch import concat
    indices = np.arange(start, start + n)
    nv = None
    if uneven:
        from jaxdd_b200.workloads import ragged_plan
        NPs, nv = ragged_plan(indices)
        order = np.lexsort((nv, -NPs))
        indices, nv = indices[order], nv[order]
    tasks = [(indices[k:k + CHUNK], uneven, npts) for k in range(0, n, CHUNK)]
    if procs <= 1:
        parts = [_build_chunk(t) for t in tasks]
    else:
        with mp.get_context("spawn").Pool(procs) as pool:
            parts = pool.map(_build_chunk, tasks)
    return concat(parts, ragged=uneven), nv, indices


class Clocks:
    """nvidia-smi sampled every 200 ms while the timed region runs."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.file,
                stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            self.proc.wait(timeout=10)

    def summary(self) -> dict:
        self.file.flush()
        rows = [r.split(", ") for r in Path(self.file.name).read_text().splitlines() if r.strip()]
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        sm, mx, reasons = [], 0.0, set()
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = max(mx, float(r[2]))
            except (ValueError, IndexError):
                continue
            for name, flag in zip(names, r[5:9]):
                if flag.strip() == "Active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def step_bytes(NPk: int, border: bool, frozen: bool, w: int = 8) -> int:
    """Algorithmic HBM bytes of one Newton step of one lane: c' and d' written and read back
    (9 + 3 (1 + K') words per node, K' = 2 with the ions' border, else 0), the state read and
    written (6 words), the static words a node needs (h, and the frozen ions' two)."""
    kp = 2 if border else 0
    n_stat = 1 + (2 if frozen else 0)
    return NPk * (2 * (9 + 3 * (1 + kp)) * w + 48 + 8 * n_stat)


def poisson_bytes(NPk: int, w: int = 8) -> int:
    return NPk * (2 * 2 * w + 16)


def algorithmic_bytes(batch, steps, w: int = 8) -> float:
    """Bytes of one launch from the steps each lane took (`lane_steps`); `w` the sweep's word
    (8 FP64, 4 in the mixed precision)."""
    total = 0.0
    lanes = batch["lane_of"]
    for k, dev in enumerate(batch["devices"]):
        lane = lanes[k]
        NPk = len(dev.x) - 2
        frozen = bool(dev.pre_cond and dev.fix_ions)
        total += steps[0, lane] * step_bytes(NPk, True, False, w)
        total += steps[1, lane] * step_bytes(NPk, False, frozen, w)
        total += steps[2, lane] * poisson_bytes(NPk)
    return total


def cpu_sample(n: int = 256, uneven: bool = False, npts: int = NP):
    """The compiled CPU restatement of the oracle (oracle/dd_cpu.cpp: jaxdd's solve_batch, one
    device at a time, single-threaded) on one core over `n` devices of the workload (a bounded
    sample, devices not in the timed batch); `(curves/s, seconds)` of the solves alone."""
    from jaxdd_b200.workloads import (RAGGED_NP, V_SCAN, drawn_device, ragged_plan,
                                      ragged_voltages)
    from oracle import cpu, dd
    idx = np.arange(10 ** 6, 10 ** 6 + n)
    if uneven:
        _, nv = ragged_plan(idx)
        jobs = [(dd.prepare([drawn_device(int(k), NP=RAGGED_NP)]), ragged_voltages(m))
                for k, m in zip(idx, nv)]
    else:
        jobs = [(dd.prepare([drawn_device(int(k), NP=npts) for k in idx]), V_SCAN)]
    cpu.lib()
    t0 = time.perf_counter()
    for tree, V in jobs:
        cpu.solve_batch(tree, V)
    dt = time.perf_counter() - t0
    return n / dt, dt


def _ref_worker(args):
    """One single-threaded process of the reference arm, pinned to its core: solve its `n`
    devices `reps` times with the compiled CPU restatement of the oracle (the uneven workload's
    one device per batch, as jaxdd needs one grid size and voltage list per batch)."""
    core, start, n, reps, uneven = args
    try:
        os.sched_setaffinity(0, {core})
    except (AttributeError, OSError):
        pass
    os.environ["OMP_NUM_THREADS"] = "1"
    from jaxdd_b200.workloads import (RAGGED_NP, V_SCAN, drawn_device, drawn_devices,
                                      ragged_plan, ragged_voltages)
    from oracle import cpu, dd
    if uneven:
        idx = np.arange(start, start + n)
        _, nv = ragged_plan(idx)
        jobs = [(dd.prepare([drawn_device(int(k), NP=RAGGED_NP)]), ragged_voltages(m))
                for k, m in zip(idx, nv)]
    else:
        jobs = [(dd.prepare(drawn_devices(n, NP=NP, start=start)), V_SCAN)]
    cpu.lib()
    times = []
    for _ in range(reps):
        t0 = time.perf_counter()
        for b, V in jobs:
            cpu.solve_batch(b, V)
        times.append(time.perf_counter() - t0)
    return times


def reference_arm(args, rank: int) -> None:
    if rank != 0:
        return
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    per = 2  # batch 2 per process (jaxdd benchmarks/run.py's CPU protocol)
    reps = args.warmup + args.steps
    uneven = args.workload == "uneven"
    tasks = [(c % (os.cpu_count() or 1), 10 ** 6 + per * c, per, reps, uneven)
             for c in range(cores)]
    t0 = time.perf_counter()
    with mp.get_context("spawn").Pool(cores) as pool:
        res = pool.map(_ref_worker, tasks)
    wall = time.perf_counter() - t0
    timed = [sum(r[args.warmup:]) for r in res]
    # all processes run together: the rate is the curves of the timed steps over their time
    rate = sum(per * args.steps / t for t in timed)
    step_ms = 1e3 * max(timed) / args.steps
    line = {
        "impl": "reference", "metric": METRIC, "value": rate, "unit": "curves/s", "n_gpus": 0,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": ("uneven drawn p-i-n stacks (seed 20261203), NP U{150..900}, "
                                "Nv U{21..121}, 2 devices per process, one per batch")
                   if uneven else "drawn p-i-n stacks (seed 20261203), NP 400, 61 V, "
                                  "batch 2 per process", "processes": cores},
        "cpu_baseline": {"value": rate, "unit": "curves/s", "cores": cores, "kind": "port",
                         "sample": f"{cores} processes x {per} devices x {args.steps} timed "
                                   f"steps (+{args.warmup} warm-up), wall {wall:.0f} s; "
                                   "jaxdd needs JAX (absent): the compiled C++ restatement of "
                                   "its FP64 solve_batch stands in (oracle/dd_cpu.cpp, pinned "
                                   "to the NumPy oracle at 1e-10 of the current scale)",
                         "jaxdd_published_per_core": "~58 curves/s (jaxdd docs/hardware.md)"},
        "e2e": {"value": rate, "unit": "curves/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def _fit_texts(args):
    start, n = args
    from jaxdd_b200.fitting import fit_texts
    return [fit_texts(k, NP=NP) for k in range(start, start + n)]


def adjoint_bench(args, rank: int, world: int, local: int) -> None:
    """The adjoint workload: the gradient of a J-V misfit (against curves of the same devices at
    log-normally perturbed parameters) in 14 log-parameters per device. One step = parameters ->
    packed record (torch) -> checkpointed solve -> misfit -> backward (adjoint kernel, then the
    record's chain to the parameters). Reported as gradients (devices) per second, next to the
    plain forward solve of the same devices."""
    import torch
    from jaxdd_b200 import adjoint as adj
    from jaxdd_b200 import fitting
    from jaxdd_b200.workloads import V_SCAN
    n = args.devices
    procs = args.build_procs or max(1, min(32, (os.cpu_count() or 1) // max(1, world)))
    t0 = time.perf_counter()
    tasks = [(rank * n + k, min(CHUNK, n - k)) for k in range(0, n, CHUNK)]
    with mp.get_context("spawn").Pool(procs) as pool:
        texts = [t for part in pool.map(_fit_texts, tasks) for t in part]
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    st = fitting.Structure(texts)
    build_s = time.perf_counter() - t0
    dev = st.device
    p = adj.plan(st.batch, V_SCAN)
    th0 = torch.tensor(st.theta0, dtype=torch.float64, device=dev)
    with torch.no_grad():
        Jt, okt, _ = adj.curves(*fitting.records(torch.tensor(
            fitting.target_theta(st.theta0, start=rank * n), dtype=torch.float64, device=dev),
            st), p)
    target = (adj.per_device(p, Jt), adj.per_device(p, okt))
    scale = torch.tensor(st.batch["J_scale"], device=dev)
    stream = torch.cuda.current_stream(dev)

    def grad_step():
        th = th0.clone().requires_grad_(True)
        J, ok, _ = adj.curves(*fitting.records(th, st), p)
        both = adj.per_device(p, ok) * target[1]
        loss = fitting.misfit(adj.per_device(p, J), both, target[0], scale)
        loss.backward()
        return loss, th.grad

    rec = [t.contiguous() for t in fitting.records(th0, st)]

    def fwd_step():
        return adj.solve_states(p, *rec)

    def timed(fn, steps):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            out = fn()
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        t = torch.tensor([ms], device=dev, dtype=torch.float64)
        if world > 1:
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        return float(t.item()), out

    with Clocks(local) as clocks:
        ms_grad, (loss, g) = timed(grad_step, args.steps)
    ms_fwd, _ = timed(fwd_step, args.steps)
    value = n * world / (ms_grad / 1e3)
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "gradients/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_grad,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": f"J-V misfit gradients: {n} devices/GPU (drawn p-i-n stacks, "
                                   f"seed 20261203, explicit work functions), NP {NP}, "
                                   f"{len(V_SCAN)} voltages; loss sum of squared J misfits to "
                                   "curves at parameters perturbed log-normally (sigma 0.2, "
                                   "seed 20261204); gradient in 14 log-parameters per device",
                       "build_s": round(build_s, 1), "loss": float(loss),
                       "grad_norm": float(g.norm()), "forward_ms": ms_fwd,
                       "adjoint_over_forward": ms_grad / ms_fwd,
                       "converged_fraction": float(target[1].float().mean())},
            "gpu_launches": args.steps * (4 + SOLVE_LAUNCHES),
            "clocks": clocks.summary(),
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


def impedance_bench(args, rank: int, world: int, local: int) -> None:
    """The small-signal workload: each device's admittance at 41 log-spaced frequencies from
    1 Hz to 1 MHz about 0.8 V, the drawn stacks with free mobile ions (the ions unknowns of
    their own). One step = the steady solve at 0.8 V (`dd_solve_states`) and
    `dd_admittance_ions`, inputs resident on the GPU."""
    import torch
    from jaxdd_b200.batch import concat
    from jaxdd_b200.impedance import Work
    n = args.devices
    procs = args.build_procs or max(1, min(32, (os.cpu_count() or 1) // max(1, world)))
    t0 = time.perf_counter()
    tasks = [(rank * n + k, min(CHUNK, n - k), args.np) for k in range(0, n, CHUNK)]
    with mp.get_context("spawn").Pool(procs) as pool:
        batch = concat(pool.map(_transient_chunk, tasks))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    build_s = time.perf_counter() - t0
    freqs = np.logspace(0, 6, 41)
    work = Work(batch, freqs, 0.8)
    dev = work.eps.device
    stream = torch.cuda.current_stream(dev)
    for _ in range(args.warmup):
        J, ok, Y = work.run()
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(local) as clocks:
        e0.record(stream)
        for _ in range(args.steps):
            J, ok, Y = work.run()
        e1.record(stream)
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    t = torch.tensor([ms], device=dev, dtype=torch.float64)
    if world > 1:
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    ms = float(t.item())
    nonfinite = int((~torch.isfinite(Y[:, :, :batch["n"]]).all(dim=1)).sum())
    if rank == 0:
        line = {
            "metric": METRIC, "value": n * world / (ms / 1e3), "unit": "spectra/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128",
            "data": "synthetic",
            "config": {"workload": f"admittance spectra: {n} devices/GPU "
                                   "(drawn p-i-n stacks with free mobile ions, seed 20261205), "
                                   f"NP {args.np}, 41 frequencies 1 Hz..1 MHz at 0.8 V, the "
                                   "ions unknowns of their own (5x5 blocks + 2 ion slots)",
                       "build_s": round(build_s, 1),
                       "converged_fraction": float(ok[:batch["n"]].float().mean()),
                       "nonfinite_points": nonfinite},
            "gpu_launches": args.steps * (3 + SOLVE_LAUNCHES),
            "clocks": clocks.summary(),
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


def build_bench(args, rank: int, world: int, local: int) -> None:
    """Device building on the GPU (`dd_build`): the packed records of 16384 devices of one
    structure (the drawn stacks pre-biased at 1.0 V, NP 400) from their parameter tables, against
    the host builder and packer of one device on one core."""
    import torch
    from jaxdd_b200.batch import prepare
    from jaxdd_b200.building import SweepStructure, build, parameters
    from jaxdd_b200.device import build_device
    from jaxdd_b200.simss_input import setup_from_texts
    from jaxdd_b200.workloads import SEED_DRAWN, drawn_texts
    n = args.devices
    torch.cuda.set_device(local)
    t0 = time.perf_counter()
    ks = [2 * i for i in range(n)]
    setups = [setup_from_texts(drawn_texts(k, np.random.default_rng([SEED_DRAWN, k]), args.np))
              for k in ks]
    st = SweepStructure(setups[0])
    P, D = parameters(st, setups)
    read_s = time.perf_counter() - t0
    # the host's rate: build and pack a bounded sample on one core
    sample = setups[:64]
    t1 = time.perf_counter()
    for s in sample:
        prepare([build_device(s, layout=st.layout)])
    host_rate = len(sample) / (time.perf_counter() - t1)
    stream = torch.cuda.current_stream()
    for _ in range(args.warmup):
        out = build(st, P, D)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        out = build(st, P, D)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    if rank == 0:
        nbytes = sum(t.numel() * 8 for t in out[:4])
        print(json.dumps({
            "metric": METRIC, "value": n / (ms / 1e3), "unit": "devices built/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": f"{n} drawn p-i-n stacks (seed 20261203) of one structure, "
                                   f"NP {args.np}: packed record and start state from parameter "
                                   "tables (parameter upload, the record's allocation and "
                                   "defaults, dd_build)",
                       "record_bytes": nbytes, "parse_s": round(read_s, 1)},
            "cpu_baseline": {"value": host_rate, "unit": "devices built/s", "cores": 1,
                             "kind": "port",
                             "sample": f"{len(sample)} devices through build_device + prepare"},
        }), flush=True)


def _transient_chunk(args):
    """The mobile-ion stacks `start .. start + n` (a pool worker)."""
    start, n, npts = args
    os.environ.setdefault("OMP_NUM_THREADS", "1")
    from jaxdd_b200.batch import prepare
    from jaxdd_b200.workloads import transient_devices
    return prepare(transient_devices(n, NP=npts, start=start))


def transient_bytes(NPk: int, K: int, w: int = 8) -> int:
    """Algorithmic bytes of one Newton iteration of one device in time: per point the static
    record (26 words) and the transient record (3), the iterate (5) and the state before the
    step (5) read, the new iterate (5) written, and the block sweep's round trip (c' 25 and the
    1 + K right-hand sides' 5 (1 + K) words, written in the elimination and read back)."""
    per_point = 26 + 3 + 5 + 5 + 5 + 2 * (25 + 5 * (1 + K))
    return NPk * per_point * w


def transient_bench(args, rank: int, world: int, local: int) -> None:
    """The transient workload: every device's steady state at 0 V, then 2000 implicit-Euler
    steps at 0.9 V log-spaced from 1 ns to 1 s, mobile ions as unknowns (5x5 blocks). One step =
    the start (`dd_solve_states`) and `dd_transient` of the whole batch, inputs resident on the
    GPU. Devices are independent: with N GPUs every rank solves its own batch (weak scaling)."""
    import torch
    from jaxdd_b200 import _lib
    from jaxdd_b200.batch import concat
    from jaxdd_b200.transient import Work
    from jaxdd_b200.workloads import transient_steps
    n = args.devices
    procs = args.build_procs or max(1, min(32, (os.cpu_count() or 1) // max(1, world)))
    t0 = time.perf_counter()
    tasks = [(rank * n + k, min(CHUNK, n - k), args.np) for k in range(0, n, CHUNK)]
    with mp.get_context("spawn").Pool(procs) as pool:
        batch = concat(pool.map(_transient_chunk, tasks))
    build_s = time.perf_counter() - t0
    cpu = None
    if rank == 0 and world == 1:
        # the oracle on one device of the same workload, a bounded number of its steps
        from jaxdd_b200.workloads import transient_devices
        from oracle import dd, transient
        sample_steps = min(200, args.tsteps)
        tv = transient_steps(args.tsteps)
        d1 = dd.prepare(transient_devices(1, NP=args.np))
        t1 = time.perf_counter()
        transient.solve_transient(d1, tv.t[:sample_steps + 1], tv.Vext[:sample_steps + 1],
                                  tv.G_frac[:sample_steps + 1])
        secs = time.perf_counter() - t1
        cpu = {"value": (sample_steps + 1) / secs / (args.tsteps + 1), "unit": "transients/s",
               "cores": 1, "kind": "port",
               "sample": f"the oracle (NumPy FP64) on 1 device, its start and first "
                         f"{sample_steps} of {args.tsteps} steps, scaled to whole transients"}
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=1800))
    tvg = transient_steps(args.tsteps)
    work = Work(batch, tvg)
    dev = work.X.device
    stream = torch.cuda.current_stream(dev)
    for _ in range(args.warmup):
        out, ok0 = work.run()
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(local) as clocks:
        e0.record(stream)
        for _ in range(args.steps):
            out, ok0 = work.run()
        e1.record(stream)
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    # the transient kernel alone (the start is a steady solve at one voltage)
    k0, k1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    g = work.g
    from jaxdd_b200.adjoint import solve_states as _solve_states
    _, _, _, ckpt = _solve_states(work.plan, g.stat, work.scal0, g.iface)
    import ctypes
    steps_c = _lib.DdSteps(work.S, work.stride, work.tv.data_ptr(), work.vv.data_ptr(),
                           work.gv.data_ptr(), work.trk.data_ptr(), work.fm.data_ptr(), work.zimt)
    o = work.out
    out_c = _lib.DdTransientOut(*(o[k].data_ptr() for k in (
        "J", "J_ext", "converged", "iterations", "accepted", "stop", "state", "logs", "f_bulk",
        "f_iface")))
    opts = _lib.DdOpts(float(work.tol), int(work.max_iter), int(work.max_iter), 0, work.bern,
                       _lib.DD_MODE_BATCH, 0, 0)
    from jaxdd_b200.batch import descriptor
    desc = descriptor(batch, g, work.plan.y0)
    k0.record(stream)
    _lib.check(_lib.lib().dd_transient(
        ctypes.byref(desc), work.X.data_ptr(), ctypes.byref(steps_c),
        ckpt["states"][0].data_ptr(), ckpt["logs"][0].data_ptr(), None, ctypes.byref(opts),
        ctypes.byref(out_c), work.ws.data_ptr(), work.ws.numel(), stream.cuda_stream),
        "dd_transient")
    k1.record(stream)
    torch.cuda.synchronize()
    kernel_ms = k0.elapsed_time(k1)
    # e2e: the packed inputs from pinned host memory, the start and the transient, the per-step
    # results back to pinned host memory, all in the timed region
    dev_in = {"stat": g.stat, "scal": work.scal0, "iface": g.iface, "X": work.X, "y0": work.plan.y0}
    host_in = {k: v.cpu().pin_memory() for k, v in dev_in.items()}
    outs = ("J", "J_ext", "converged", "iterations", "accepted")
    host_out = {k: torch.empty(o[k].shape, dtype=o[k].dtype).pin_memory() for k in outs}
    h2d = sum(v.numel() * v.element_size() for v in host_in.values())
    d2h = sum(v.numel() * v.element_size() for v in host_out.values())
    v0, v1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    v0.record(stream)
    for k, v in dev_in.items():
        v.copy_(host_in[k], non_blocking=True)
    out, ok0 = work.run()
    for k in outs:
        host_out[k].copy_(o[k], non_blocking=True)
    v1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = v0.elapsed_time(v1)
    # the gradients: the integrated current and its derivatives in ln N_ion and ln mu_ion, the
    # tangents carried through every step in the same launch
    gwork = Work(batch, tvg, gradients=True)
    g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    g0.record(stream)
    gout, _ = gwork.run()
    g1.record(stream)
    torch.cuda.synchronize()
    grad_ms = g0.elapsed_time(g1)
    dQ = gout["dQ"][:, :batch["n"]]
    grad_finite = bool(torch.isfinite(dQ).all())
    t = torch.tensor([ms, e2e_ms, kernel_ms, grad_ms], device=dev, dtype=torch.float64)
    if world > 1:
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    ms, e2e_ms, kernel_ms, grad_ms = (float(x) for x in t.tolist())
    m = batch["n"]
    its = o["iterations"][:, :m].to(torch.int64)
    acc = o["accepted"][:, :m]
    total_its = int(its.sum())
    NPs = np.asarray(batch["NP"])
    K = 2 if batch["ka"] + batch["kc"] <= 2 else 4
    per_lane_its = its.sum(dim=0).cpu().numpy()
    alg = float(sum(per_lane_its[j] * transient_bytes(int(NPs[j]), K) for j in range(m)))
    achieved = alg / (kernel_ms / 1e3) / 1e9
    peak, peak_kind = _peaks()
    S = work.S
    if rank == 0:
        line = {
            "metric": METRIC, "value": m * world / (ms / 1e3), "unit": "transients/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": f"transients with mobile ions: {m} devices/GPU (drawn "
                                   "p-i-n stacks with free mobile ions, seed 20261205), NP "
                                   f"{args.np}, steady state at 0 V then {S - 1} implicit-Euler "
                                   "steps at 0.9 V log-spaced 1 ns..1 s, 5x5 blocks + 2 ion "
                                   "slots",
                       "inputs_vs_l2": "the state and sweep buffers (GBs) exceed L2",
                       "build_s": round(build_s, 1),
                       "time_steps_per_s": m * world * S / (ms / 1e3),
                       "newton_steps_per_time_step": total_its / (m * S),
                       "us_per_newton_step_per_device": kernel_ms * 1e3 / total_its,
                       "reference_published_a100": "44,100 time steps/s, 7.22 us per Newton "
                                                   "step per device (ions, 241 steps, 4096 per "
                                                   "batch; docs/hardware.md:62-66)",
                       "transient_kernel_ms": kernel_ms,
                       "start_converged_fraction": float(ok0[:m].float().mean()),
                       "converged_fraction": float(o["converged"][:, :m].float().mean()),
                       "accepted_fraction": float(acc.float().mean()),
                       "gradients": {"value": m * world / (grad_ms / 1e3),
                                     "unit": "gradients/s (Q and dQ/dln N_ion, dQ/dln mu_ion "
                                             "per device, forward mode through 2000 steps)",
                                     "ms": grad_ms, "over_forward": grad_ms / ms,
                                     "finite": grad_finite}},
            "e2e": {"value": m * world / (e2e_ms / 1e3), "unit": "transients/s",
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": None,
                         "peak_source": f"{peak_kind} HBM copy",
                         "kernel": "dd::tr::transient_kernel (two threads per device, the "
                                   "twisted sweep)"},
            "cpu_baseline": cpu,
            "gpu_launches": args.steps * (1 + SOLVE_LAUNCHES),
            "clocks": clocks.summary(),
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


def _parity_worker(args):
    """The oracle's curves of a few devices of the timed workload (one pool task): devices of
    one grid size and voltage list in one batch, as jaxdd's `solve_batch` takes them, solved by
    the compiled restatement of the oracle (pinned to oracle/dd.py at 1e-10 of the scale)."""
    idx, npts, volts = args
    os.environ.setdefault("OMP_NUM_THREADS", "1")
    from jaxdd_b200.workloads import drawn_device
    from oracle import cpu, dd
    b = dd.prepare([drawn_device(int(k), NP=npts) for k in idx])
    J, ok, _ = cpu.solve_batch(b, np.asarray(volts))
    return J, ok, b["J_scale"]


def parity_sample(batch, draw_idx, lists, J, ok, offsets, npts, procs: int,
                  lanes_wanted: int = 1024) -> dict:
    """The timed launch's own curves checked against the oracle (outside the timed region): a
    fixed-stride sample of the batch's devices (the frozen and the free ones alternate in the
    draw order) and every device with a point that did not converge (up to 64 of them); each
    device's J within 1e-6 of its current scale, its converged flags equal to the oracle's."""
    n = batch["n"]
    lanes = batch["lane_of"]
    stride = max(1, n // lanes_wanted)
    pick = list(range(0, n, stride))[:lanes_wanted]
    bad = [k for k in range(n) if not ok[offsets[lanes[k]]:offsets[lanes[k]]
                                          + len(lists[k])].all()]
    pick = sorted(set(pick) | set(bad[:64]))
    groups: dict = {}
    for k in pick:
        NPk = len(batch["devices"][k].x) - 2
        groups.setdefault((NPk, len(lists[k])), []).append(k)
    tasks, owners = [], []
    for (NPk, _), ks in groups.items():
        for c in range(0, len(ks), 8):
            part = ks[c:c + 8]
            tasks.append(([int(draw_idx[k]) for k in part], npts, lists[part[0]]))
            owners.append(part)
    t0 = time.perf_counter()
    with mp.get_context("spawn").Pool(max(1, min(procs, len(tasks)))) as pool:
        res = pool.map(_parity_worker, tasks)
    worst, flags_equal = 0.0, True
    for part, (Jo, oko, scale) in zip(owners, res):
        for j, k in enumerate(part):
            sl = slice(offsets[lanes[k]], offsets[lanes[k]] + len(lists[k]))
            mine = ok[sl].astype(bool)
            flags_equal = flags_equal and bool(np.array_equal(mine, oko[j]))
            both = oko[j] & mine
            if both.any():
                worst = max(worst, float(np.max(np.abs(J[sl][both] - Jo[j][both])) / scale[j]))
    return {"lanes": len(pick), "unconverged_lanes": len(bad),
            "max_err_over_scale": worst, "flags_equal": flags_equal, "tol": 1e-6,
            "oracle": "C++ restatement of the FP64 oracle (oracle/dd_cpu.cpp; pinned to "
                      "oracle/dd.py at 1e-10 of the scale)",
            "seconds": round(time.perf_counter() - t0, 1)}


def workload_name(args, batch, nflat: int) -> str:
    if args.workload == "uneven":
        NPs = batch["NP"]
        return (f"uneven grids in FP64: drawn p-i-n stacks (seed 20261203), {args.devices} "
                f"devices/GPU in one launch, NP U{{150..900}} (mean {NPs.mean():.0f}), voltage "
                f"counts U{{21..121}} (mean {nflat / batch['n']:.1f}) over -0.2..1.3 V, half "
                "frozen after a 1.0 V pre-bias, half free ions")
    return (f"drawn J-V curves: p-i-n stacks (seed 20261203), {args.devices} devices/GPU, "
            f"NP {args.np}, {nflat // batch['n']} voltages -0.2..1.3 V, half frozen after a 1.0 V "
            "pre-bias, half free ions")


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=("ours", "reference"))
    ap.add_argument("--precision", default="fp64", choices=("fp64",))
    ap.add_argument("--workload", default="curves",
                    choices=("curves", "uneven", "adjoint", "impedance", "build", "transient"),
                    help="curves: 16384 devices, NP 400, 61 V (the default); uneven: 32768 "
                         "devices, NP ~ U{150..900}, Nv ~ U{21..121}, one launch; adjoint: "
                         "gradients of a J-V misfit in 14 parameters, 4096 devices; "
                         "impedance: 8192 devices with mobile ions, 41 frequencies; "
                         "transient: 8192 devices with mobile ions, 2000 time steps")
    ap.add_argument("--tsteps", type=int, default=2000,
                    help="time steps of the transient workload (2000; fewer only for "
                         "profiling)")
    ap.add_argument("--devices", type=int, default=0)
    ap.add_argument("--np", type=int, default=NP,
                    help="grid points of the fixed-size workload (400; smaller only for "
                         "profiling the same occupancy on less memory)")
    ap.add_argument("--build-procs", type=int, default=0)
    ap.add_argument("--cpu-sample", type=int, default=256,
                    help="devices the compiled CPU restatement solves on one core for "
                         "cpu_baseline")
    ap.add_argument("--no-tune", dest="tune", action="store_false",
                    help="skip the autotuner (the solve's default launch form)")
    ap.add_argument("--parity-lanes", type=int, default=1024,
                    help="devices of the timed launch checked against the oracle after the "
                         "timed region (0: none)")
    ap.add_argument("--graph", default="auto", choices=("auto", "on", "off"),
                    help="replay the solve from a CUDA graph captured once (auto: the uneven "
                         "workload, whose config asks for it)")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    uneven = args.workload == "uneven"
    if not args.devices:
        args.devices = {"uneven": 2 * DEVICES_PER_GPU, "adjoint": 4096, "impedance": 8192,
                        "transient": 8192}.get(args.workload, DEVICES_PER_GPU)
    if args.impl == "reference":
        reference_arm(args, rank)
        return
    if args.workload == "adjoint":
        adjoint_bench(args, rank, world, local)
        return
    if args.workload == "impedance":
        impedance_bench(args, rank, world, local)
        return
    if args.workload == "build":
        build_bench(args, rank, world, local)
        return
    if args.workload == "transient":
        transient_bench(args, rank, world, local)
        return
    if args.devices % 32:
        raise SystemExit("--devices must be a multiple of 32")
    cores = os.cpu_count() or 1
    procs = args.build_procs or max(1, min(32, cores // max(1, world)))
    t0 = time.perf_counter()
    batch, nv_dev, draw_idx = build_workload(args.devices, rank * args.devices, procs, uneven,
                                             args.np)
    build_s = time.perf_counter() - t0
    cpu = (cpu_sample(args.cpu_sample, uneven, args.np)
           if rank == 0 and world == 1 and args.cpu_sample > 0 else None)

    import ctypes

    import torch
    from jaxdd_b200 import _lib
    from jaxdd_b200.batch import _gpu, descriptor, initial_state
    from jaxdd_b200.workloads import RAGGED_NP, V_SCAN, ragged_voltages

    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    dev = torch.device("cuda", local)
    g = _gpu(batch)
    Bp, npmax = batch["Bp"], batch["np_max"]
    lanes = batch["lane_of"]
    lists = [ragged_voltages(m) for m in nv_dev] if uneven else [V_SCAN] * batch["n"]
    y0 = np.zeros((npmax + 2, 3, Bp))
    counts = np.zeros(Bp, dtype=np.int32)
    for k, d in enumerate(batch["devices"]):
        first = d.V_pre if d.pre_cond else lists[k][0]
        y0[:len(d.x), :, lanes[k]] = initial_state(d, first)
        counts[lanes[k]] = len(lists[k])
    offsets = np.zeros(Bp, dtype=np.int32)
    offsets[1:] = np.cumsum(counts)[:-1]
    nflat = int(counts.sum())
    flat = np.zeros(nflat)
    for k in range(batch["n"]):
        flat[offsets[lanes[k]]:offsets[lanes[k]] + counts[lanes[k]]] = lists[k]
    t_y0 = torch.from_numpy(y0).to(dev)
    t_v = torch.from_numpy(flat).to(dev)
    t_off = torch.from_numpy(offsets).to(dev)
    t_cnt = torch.from_numpy(counts).to(dev)
    J = torch.empty(nflat, dtype=torch.float64, device=dev)
    ok = torch.empty(nflat, dtype=torch.uint8, device=dev)
    its = torch.empty(nflat, dtype=torch.int32, device=dev)
    status = torch.empty(Bp, dtype=torch.int32, device=dev)
    steps = torch.zeros((3, Bp), dtype=torch.int32, device=dev)
    desc = descriptor(batch, g, t_y0)
    volts = _lib.DdVoltages(t_v.data_ptr(), t_off.data_ptr(), t_cnt.data_ptr())
    opts = _lib.DdOpts(1e-10, 60, 60, 0, 0, _lib.DD_MODE_BATCH, _lib.DD_PRECISION[args.precision], 0)
    ws = g.workspace(desc)
    so = _lib.lib()
    stream = torch.cuda.current_stream(dev)

    def launch(d=desc, v=volts, on=None):
        _lib.check(so.dd_solve(ctypes.byref(d), ctypes.byref(v), ctypes.byref(opts),
                               J.data_ptr(), ok.data_ptr(), its.data_ptr(), status.data_ptr(),
                               steps.data_ptr(), ws.data_ptr(), ws.numel(),
                               (on or stream).cuda_stream),
                   "dd_solve")

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    # the autotuner (outside the timed region): every launch form timed once on this batch, the
    # fastest kept for the solves below
    launch_form = None
    if args.tune:
        form = ctypes.c_int32(-1)
        times = (ctypes.c_float * _lib.DD_SOLVE_FORMS)()
        _lib.check(so.dd_tune(ctypes.byref(desc), ctypes.byref(volts), ctypes.byref(opts),
                              J.data_ptr(), ok.data_ptr(), its.data_ptr(), status.data_ptr(),
                              steps.data_ptr(), ws.data_ptr(), ws.numel(), stream.cuda_stream,
                              ctypes.byref(form), times), "dd_tune")
        launch_form = dict(_lib.SOLVE_FORMS[form.value], form=form.value,
                           tune_ms=[round(float(t), 1) for t in times])
    # the solve's launches (the queue's reset, the specialised and the generic kernel) captured
    # once into a CUDA graph and replayed, where asked
    graphed = args.graph == "on" or (args.graph == "auto" and uneven)
    step = launch
    if graphed:
        graph = torch.cuda.CUDAGraph()
        launch()  # the tuned form's attributes set before the capture
        barrier()
        with torch.cuda.graph(graph, capture_error_mode="relaxed"):
            launch(on=torch.cuda.current_stream(dev))
        step = graph.replay
    for _ in range(args.warmup):
        step()
    barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(local) as clocks:
        ev0.record(stream)
        for _ in range(args.steps):
            step()
        ev1.record(stream)
        barrier()
    ms = ev0.elapsed_time(ev1) / args.steps
    t = torch.tensor([ms], device=dev, dtype=torch.float64)
    if world > 1:
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    ms_max = float(t.item())
    curves = args.devices * world
    value = curves / (ms_max / 1e3)
    ok_frac = float(ok.float().mean().item())
    lane_steps = steps.cpu().numpy()
    parity = None
    if rank == 0 and args.parity_lanes > 0:
        parity = parity_sample(batch, draw_idx, lists, J.cpu().numpy(), ok.cpu().numpy(),
                               offsets, RAGGED_NP if uneven else args.np, procs,
                               args.parity_lanes)

    # e2e: the C ABI from pinned host buffers, the copies inside the timed region
    host = {name: torch.from_numpy(arr).pin_memory() for name, arr in
            (("stat", batch["stat"]), ("scal", batch["scal"]), ("iface", batch["iface"]),
             ("y0", y0), ("v", flat), ("off", offsets), ("cnt", counts))}
    dev_in = {k: torch.empty_like(v, device=dev) for k, v in host.items()}
    J_h = torch.empty(nflat, dtype=torch.float64).pin_memory()
    ok_h = torch.empty(nflat, dtype=torch.uint8).pin_memory()
    its_h = torch.empty(nflat, dtype=torch.int32).pin_memory()
    desc2 = _lib.DdBatch(batch["n"], Bp, npmax, batch["ka"], batch["kc"],
                         dev_in["stat"].data_ptr(), dev_in["scal"].data_ptr(),
                         dev_in["iface"].data_ptr(), dev_in["y0"].data_ptr())
    volts2 = _lib.DdVoltages(dev_in["v"].data_ptr(), dev_in["off"].data_ptr(),
                             dev_in["cnt"].data_ptr())
    h2d = sum(v.numel() * v.element_size() for v in host.values())
    d2h = J_h.numel() * 8 + ok_h.numel() + its_h.numel() * 4

    def e2e_step():
        for k in host:
            dev_in[k].copy_(host[k], non_blocking=True)
        launch(desc2, volts2)
        J_h.copy_(J, non_blocking=True)
        ok_h.copy_(ok, non_blocking=True)
        its_h.copy_(its, non_blocking=True)

    e2e_steps = max(1, min(args.steps, 3))
    e2e_step()
    barrier()
    ev2, ev3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev2.record(stream)
    for _ in range(e2e_steps):
        e2e_step()
    ev3.record(stream)
    barrier()
    e2e_ms = ev2.elapsed_time(ev3) / e2e_steps
    t = torch.tensor([e2e_ms], device=dev, dtype=torch.float64)
    if world > 1:
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    e2e_value = curves / (float(t.item()) / 1e3)

    peak, peak_kind = _peaks()
    entry = traffic_entry(args.precision, args.workload, args.devices, args.np)
    traffic = entry["dram_bytes_per_launch"] if entry else None
    alg = algorithmic_bytes(batch, lane_steps, 8 if args.precision == "fp64" else 4)
    achieved = alg / (ms / 1e3) / 1e9
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "curves/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if args.precision == "fp64" else "f32 sweep / f64 residual",
            "data": "synthetic",
            "config": {"workload": workload_name(args, batch, nflat),
                       "precision": args.precision, "devices_per_gpu": args.devices,
                       "l2": f"inputs larger than L2 ({batch['stat'].nbytes / 1e9:.2f} GB of "
                             "statics per launch)",
                       "converged_fraction": ok_frac, "build_s": round(build_s, 1),
                       "launch": launch_form, "cuda_graph": graphed},
            "parity": parity,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "peak_kind": ("measured (MEASURED_PEAKS.json hbm_gbs)"
                                       if peak_kind == "measured" else
                                       "fallback (an earlier B200 copy-bandwidth measurement; "
                                       "MEASURED_PEAKS.json absent)"),
                         "algorithmic_bytes_per_launch": alg},
            "cpu_baseline": None if cpu is None else {
                "value": cpu[0], "unit": "curves/s", "cores": 1, "kind": "port",
                "sample": f"{args.cpu_sample} devices of the same workload (outside the timed "
                          f"batch), {cpu[1]:.1f} s on one core: the compiled C++ restatement "
                          "of jaxdd's FP64 solve_batch (oracle/dd_cpu.cpp; jaxdd needs JAX)"},
            "e2e": {"value": e2e_value, "unit": "curves/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h)},
            "gpu_launches": args.steps * SOLVE_LAUNCHES,
            "clocks": clocks.summary(),
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
