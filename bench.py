#!/usr/bin/env python
"""Benchmark of the B200 geodesic FDTD time step (prints one JSON line).

Workload (default ``config4``): icosahedral subdivision 9 (2,621,442 dual
cells) x 80 radial cells over 0-100 km (209.7 M cells), FP32 fields,
exponential conductive integrator, surface-impedance lower boundary over a
seeded smooth log-normal ground-conductivity map, Drude electron plasma ADE,
one 20 Hz Gaussian source and 256 barycentric receivers; seeded synthetic
inputs, random 1e-6 initial fields.  One bench "step" is ``--time-steps``
leapfrog steps (default 100) of that simulation, launched as CUDA-graph chunks
on one GPU, each leapfrog step sampling the 256 receivers into a
device-resident float64 trace buffer (``ifdtd_step_sampled``).  ``value`` is
whole-job Gcell-updates/s (cells = vertices x radial cells) with the state and
the step currents resident in HBM; ``e2e`` is the same metric through the
public API (``GeodesicFDTD.record_er_observations``) with host-computed source
currents copied in and receiver traces copied out every bench step.
``--workload config2`` runs the s7 / 40-cell plasma workload (64 receivers,
1000 leapfrog steps per bench step) the same way.  After the s9 state is
freed, the default run also measures the batched ensemble below on the same
GPU and attaches its record as the line's ``ensemble`` object
(``--no-ensemble`` skips it).

``--workload config3`` measures ensemble runs/s instead: 64 seeded members
of uneven size (s5-s7, 24-60 radial cells, exponential ionospheres, 16
receivers each), each run being 5000 leapfrog steps; ``value`` is the batched
``Ensemble`` step (all members per launch) and ``sequential`` the same members
stepped one after another, both with the receivers sampled on the device.

``--impl reference`` times the CPU oracle (a NumPy restatement of the
reference's own solver, the reference being pure Python, run on PyTorch CPU
tensors over every host thread) on a bounded sample of the same workload,
built with the oracle's own mesh builder and inputs (nothing of the CUDA
product is loaded).  Under torchrun every rank runs an independent replica
(the plain solver does not shard), timing is the max over ranks.
"""

from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

FALLBACK_HBM_GBS = 6650.0
METRIC = "Gcell-updates/s"
UNIT = "Gcell/s"


def parse() -> argparse.Namespace:
    p = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=("engine", "reference"), default="engine")
    p.add_argument("--workload", choices=("config2", "config3", "config4", "config5"), default="config4")
    p.add_argument("--runs", type=int, default=4096, help="config5: training runs generated by the engine")
    p.add_argument("--eval-runs", type=int, default=512, help="config5: held-out runs (16 receivers each)")
    p.add_argument("--iterations", type=int, default=30000, help="config5: training iterations per network")
    p.add_argument("--lr", type=float, default=2e-3, help="config5: initial Adam learning rate")
    p.add_argument("--lr-final", type=float, default=2e-5, help="config5: final learning rate (geometric schedule)")
    p.add_argument("--batch", type=int, default=512, help="config5: traces per training iteration")
    p.add_argument("--gemm", choices=("tcgen05", "mma"), default="tcgen05", help="config5: the surrogate's GEMM kernel")
    p.add_argument("--decoder", default="16x64:4:32,16,1",
                   help="config5: decoder shape t0 x c0 : stride : channels (t0 * stride ** len(channels) = 1024)")
    p.add_argument("--members", type=int, default=64, help="config3: ensemble members")
    p.add_argument("--no-autotune", action="store_true", help="keep the automatic launch geometry (no tuning run)")
    p.add_argument("--time-steps", type=int, default=None, help="leapfrog steps per bench step")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-drift", action="store_true", help="skip the float32-vs-float64 drift run")
    p.add_argument("--no-ensemble", action="store_true",
                   help="config4: skip the 64-member ensemble measurement attached to the line")
    p.add_argument("--subdivision", type=int, default=None, help="override the workload's subdivision (small profiling cases)")
    p.add_argument("--plasma-frame", type=int, choices=(0, 1, 2), default=0,
                   help="config2/config4: frame of the plasma current in the kernels (0 auto, 1 Cartesian, 2 face frames)")
    return p.parse_args()


def measured_peak() -> tuple[float, str]:
    path = ROOT / "MEASURED_PEAKS.json"
    try:
        return float(json.loads(path.read_text())["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM_GBS, "fallback"


def traffic_from_profile(workload: str) -> dict[str, float]:
    """DRAM bytes per launch of each step kernel from the committed ncu summary
    (lines ``dram_bytes_per_launch <kernel>: <bytes>``), if any."""

    out = {}
    path = ROOT / "profiles" / f"fdtd_step_{workload}_traffic.txt"
    try:
        for line in path.read_text().splitlines():
            if line.startswith("dram_bytes_per_launch "):
                name, value = line[len("dram_bytes_per_launch ") :].split(":", 1)
                out[name.strip()] = float(value)
    except OSError:
        pass
    return out


def kernel_bytes(sim) -> dict[str, int]:
    """Algorithmic bytes of one launch of each phase kernel: every array it
    needs read once and every array it updates written once.  H phase: reads
    Er, Et; reads and writes Hr, Ht, the plasma currents and the surface-
    impedance memory.  E phase: reads Hr, Ht and the plasma currents; reads and
    writes Er, Et."""

    item = sim.backend.itemsize
    e = sum(int(getattr(sim, f).numel()) for f in ("er", "et"))
    h = sum(int(getattr(sim, f).numel()) for f in ("hr", "ht"))
    j = sum(int(x.numel()) for x in sim._plasma_coupler.ade.current_density) if sim._plasma_coupler is not None else 0
    si = int(sim._surface_impedance_ade.memory.numel()) if sim._surface_impedance_ade is not None else 0
    return {"h_phase": item * (e + 2 * (h + j + si)), "e_phase": item * (h + j + 2 * e)}


def phase_times_ms(sim, reps: int) -> dict[str, float]:
    """Median device time of each phase kernel: CUDA events around every launch on the
    launching stream (``ifdtd_time_phases``, the plasma current turned into the plan's
    frame once around all launches)."""

    h, e = sim._engine.phase_times_ms(sim._state(), reps)
    return {"h_phase": h, "e_phase": e}


class ClockSampler:
    """nvidia-smi samples of one GPU while the timed region runs."""

    QUERY = (
        "clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
        "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"
    )

    def __init__(self, uuid: str | None):
        self.proc = None
        self.path = Path(os.environ.get("TMPDIR", "/tmp")) / f"bench_clocks_{os.getpid()}.csv"
        if uuid is None:
            return
        try:
            self.handle = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", uuid, f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.handle,
                stderr=subprocess.DEVNULL,
            )
        except OSError:
            self.proc = None

    def stop(self) -> dict | None:
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.handle.close()
        sm, smax, reasons = [], None, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in self.path.read_text().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                smax = float(parts[1])
            except ValueError:
                continue
            for name, flag in zip(names, parts[3:7]):
                if flag.lower() == "active":
                    reasons.add(name)
        self.path.unlink(missing_ok=True)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons), "samples": len(sm)}


def max_over_ranks(value: float, dist, device) -> float:
    """The largest value over all ranks (every rank gets it); ``dist`` None = one rank."""

    if dist is None:
        return value
    import torch

    t = torch.tensor([value], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def build(workload: str, device: str, dtype: str = "float32", subdivision: int | None = None, plasma_frame: int = 0):
    from ionosphere_fdtd_b200 import workloads as W
    from ionosphere_fdtd_b200.engine import Tuning

    extra = {} if subdivision is None else {"subdivision": subdivision}
    if plasma_frame:
        extra["tuning"] = Tuning(plasma_frame=plasma_frame)
    if workload == "config4":
        wl = W.config4(device=device, dtype=dtype, **extra)
    else:
        wl = W.config2(device=device, dtype=dtype, **extra)
    W.seed_fields(wl.simulation)
    return wl


def fp32_drift(workload: str, device: str, steps: int, subdivision: int | None = None, plasma_frame: int = 0) -> dict:
    """Relative L2 per (E, H) group between float32 and float64 runs of the
    engine from the same seeded state (the float64 run stands in for the
    float64 NumPy path, far too slow at these sizes) after ``steps`` steps."""

    import torch

    out = {}
    sims = {}
    for dtype in ("float64", "float32"):
        sim = build(workload, device, dtype, subdivision, plasma_frame).simulation
        sim.step(steps)
        sims[dtype] = {f: getattr(sim, f).to(torch.float64) for f in ("er", "et", "hr", "ht")}
        del sim
        torch.cuda.empty_cache()
    for name, group in (("E", ("er", "et")), ("H", ("hr", "ht"))):
        a = torch.cat([sims["float32"][f].flatten() for f in group])
        b = torch.cat([sims["float64"][f].flatten() for f in group])
        out[f"rel_l2_{name}"] = float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))
    return {"steps": steps, **out, "against": "float64 engine from the same seeded state"}


# Subdivision of the CPU oracle's sample per workload. A full s9 / 80-cell step takes the
# oracle tens of seconds even on every host thread, so the s9 workload is sampled on the same
# 80-cell column with the same plasma and surface impedance at s7 (163,842 vertices): the
# oracle's rate per cell hardly depends on the mesh level (on 8 threads 0.0039 Gcell/s at s6
# against 0.0037 at s7).
ORACLE_SAMPLE_SUB = {"config2": 7, "config4": 7}


def host_threads() -> int:
    """Host threads this process may run on: its CPU affinity set, capped by a cgroup CPU
    quota when one is set (a container may see more cores than it may use)."""

    try:
        n = len(os.sched_getaffinity(0))
    except AttributeError:
        n = os.cpu_count() or 1
    quota = None
    try:  # cgroup v2: "<quota> <period>" or "max <period>"
        q, period = Path("/sys/fs/cgroup/cpu.max").read_text().split()[:2]
        if q != "max":
            quota = int(q) / int(period)
    except (OSError, ValueError):
        try:  # cgroup v1
            q = int(Path("/sys/fs/cgroup/cpu/cpu.cfs_quota_us").read_text())
            period = int(Path("/sys/fs/cgroup/cpu/cpu.cfs_period_us").read_text())
            if q > 0 and period > 0:
                quota = q / period
        except (OSError, ValueError):
            pass
    if quota is not None:
        n = min(n, max(1, int(quota)))
    return max(1, n)


# The plain-solver workloads: mesh level, radial cells, receivers, leapfrog steps per bench step.
PLAIN = {
    "config2": {"subdivision": 7, "radial_cells": 40, "receivers": 64, "time_steps": 1000, "surface_impedance": False},
    "config4": {"subdivision": 9, "radial_cells": 80, "receivers": 256, "time_steps": 100, "surface_impedance": True},
}


def workload_config(workload: str, subdivision: int | None, world: int) -> dict:
    """The ``config`` object of the JSON line, the same in both arms: the workload's
    static description (no timings or tuning results)."""

    spec = PLAIN[workload]
    sub = spec["subdivision"] if subdivision is None else subdivision
    L = spec["radial_cells"]
    V, E, F = 10 * 4**sub + 2, 30 * 4**sub, 20 * 4**sub
    state = 4 * (V * (L + 1) + E * (L + 1) + E * L + F * L + 3 * F * L + (16 * E if spec["surface_impedance"] else 0))
    return {
        "workload": workload,
        "subdivision": sub,
        "radial_cells": L,
        "cells": V * L,
        "plasma": "drude (1 species)",
        "surface_impedance": spec["surface_impedance"],
        "receivers": spec["receivers"],
        "precision": "float32 fields, float64 receiver accumulation",
        "l2": f"state {state / 1e6:.0f} MB > 126 MB L2, no flush needed",
        "parallelism": f"replicas x{world}",
    }


def oracle_build(workload: str, sub: int | None = None):
    """The CPU oracle on the workload's radial column, plasma and surface (float32), built
    from the oracle's own mesh builder and inputs, fields seeded; ``sub`` overrides the mesh
    level (the sample level by default)."""

    import oracle.workloads as OW

    spec = PLAIN[workload]
    L = spec["radial_cells"]
    sub = ORACLE_SAMPLE_SUB[workload] if sub is None else sub
    builder = OW.config4 if workload == "config4" else OW.config2
    sim = builder(subdivision=sub, radial_cells=L, dtype=np.float32)
    OW.seed_fields(sim)
    full = spec["subdivision"]
    note = "" if sub == full else f" (the s{full} workload's column, plasma and surface on an s{sub} mesh)"
    return sim, {"cells": sim.mesh.n_vertices * L, "sub": sub, "L": L, "note": note}


def oracle_stepper(sim):
    """The oracle's step on PyTorch CPU tensors over every host thread: the reference's
    multi-threaded CPU path (its Torch backend on the CPU with ``torch_threads``)."""

    from oracle.threaded import ThreadedOracleStep

    return ThreadedOracleStep(sim, host_threads())


def oracle_time(stepper, info: dict, steps: int) -> dict:
    t0 = time.perf_counter()
    stepper.step(steps)
    dt = time.perf_counter() - t0
    return {"gcells": info["cells"] * steps / dt / 1e9, "seconds": dt, "steps": steps, "cores": stepper.threads, **info}


def oracle_sample(workload: str, steps: int, warm: int = 1) -> dict:
    """Time the CPU oracle on ``steps`` leapfrog steps of the same workload (float32)."""

    sim, info = oracle_build(workload)
    stepper = oracle_stepper(sim)
    stepper.step(warm)
    return oracle_time(stepper, info, steps)


ENSEMBLE_METRIC = "ensemble runs/s"
RUN_STEPS = 5000  # leapfrog steps per ensemble run


ENSEMBLE_SAMPLE = 4  # the first four members of the draws: s7/51, s6/41, s6/39 and s7/26 (15.9 M cells)


def oracle_ensemble_sampler(members: int = ENSEMBLE_SAMPLE) -> tuple[list, int]:
    """The oracle on the first ``members`` members of the ensemble workload
    (float32, each member with its own threaded stepper) and their cells."""

    import oracle.workloads as OW
    from oracle.fdtd import build_mesh

    meshes, steppers, cells = {}, [], 0
    for d in OW.config3_draws(members=members):
        sub = d["subdivision"]
        if sub not in meshes:
            meshes[sub] = build_mesh(sub)
        steppers.append(oracle_stepper(OW.config3_member(d, mesh=meshes[sub])))
        cells += meshes[sub].n_vertices * d["radial_cells"]
    return steppers, cells


def oracle_ensemble_time(steppers: list, cells: int, steps: int = 1) -> dict:
    """Time ``steps`` leapfrog steps of every sampled member, one member after another."""

    t0 = time.perf_counter()
    for stepper in steppers:
        stepper.step(steps)
    dt = time.perf_counter() - t0
    return {"gcells": cells * steps / dt / 1e9, "seconds": dt, "steps": steps, "cores": steppers[0].threads, "cells": cells}


def ensemble_sample_text(r: dict, mean_cells: float, per: str) -> str:
    return (f"{per} of the ensemble's first {ENSEMBLE_SAMPLE} members (s7/51, s6/41, s6/39, s7/26; {r['cells']} cells; "
            f"{r['seconds']:.1f} s), oracle on PyTorch CPU tensors over {r['cores']} threads; runs/s = rate / "
            f"({RUN_STEPS} steps x mean member cells {mean_cells:.0f})")


def ensemble_reference_arm(args) -> None:
    cells = ensemble_cells(args.members)
    mean_cells = statistics.mean(cells)
    steppers, sample_cells = oracle_ensemble_sampler()
    rates, secs = [], 0.0
    for _ in range(args.warmup):
        oracle_ensemble_time(steppers, sample_cells)
    for _ in range(args.steps):
        r = oracle_ensemble_time(steppers, sample_cells)
        rates.append(r["gcells"])
        secs += r["seconds"]
    gcells = statistics.median(rates)
    value = gcells * 1e9 / (RUN_STEPS * mean_cells)
    sample = ensemble_sample_text(r, mean_cells, "1 leapfrog step per bench step")
    line = {
        "impl": "reference", "metric": ENSEMBLE_METRIC, "value": value, "unit": "runs/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * secs / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "config3", "members": args.members, "run_steps": RUN_STEPS, "device": "cpu"},
        "cpu_baseline": {"value": value, "unit": "runs/s", "cores": r["cores"], "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": "runs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def ensemble_cells(members: int) -> list[int]:
    """Cells (vertices x radial cells) of the config3 members (the oracle's restatement
    of the seeded draws, so the reference arm loads nothing of the product)."""

    import oracle.workloads as OW

    return [(10 * 4 ** d["subdivision"] + 2) * d["radial_cells"] for d in OW.config3_draws(members=members)]


def ensemble_main(args, world: int, rank: int, local: int) -> None:
    import torch

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=torch.device("cuda", local))
    line = ensemble_measure(args, world, rank, local, dist, cpu_baseline=not args.no_cpu_baseline)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def ensemble_measure(args, world: int, rank: int, local: int, dist, cpu_baseline: bool) -> dict | None:
    """Batched and sequential runs/s of the 64-member ensemble on this rank's GPU (max over
    ranks); returns the config-3 JSON line on rank 0, None elsewhere."""

    import torch

    from ionosphere_fdtd_b200 import Ensemble
    from ionosphere_fdtd_b200 import workloads as W

    device = f"cuda:{local}"
    t_setup = time.perf_counter()
    wls = W.config3_members(device=device, members=args.members)
    setup_s = time.perf_counter() - t_setup
    sims = [w.simulation for w in wls]
    for sim in sims:
        W.seed_fields(sim)
    tuning = None
    if not args.no_autotune:
        from ionosphere_fdtd_b200.autotune import SHAPE_FREE_CANDIDATES, autotune_ensemble

        t_tune = time.perf_counter()
        tuned = autotune_ensemble(sims, SHAPE_FREE_CANDIDATES, steps=32, repeats=3,
                                  key=lambda m: (m.config.subdivision, m.backend.itemsize))
        tuning = {
            "seconds": time.perf_counter() - t_tune,
            "candidates": len(SHAPE_FREE_CANDIDATES),
            "classes": {f"s{k[0]}": {**tuning_fields(r.best), "ms_per_step": r.best_ms}
                        for k, r in tuned.items()},
        }
    T = args.time_steps or 100
    stream = torch.cuda.current_stream()
    probes = [sim._engine.probe("er", w.receivers[0], np.broadcast_to(w.receivers[1][:, None], w.receivers[0].shape), w.receivers[2])
              for sim, w in zip(sims, wls)]
    outs = [torch.zeros((T, w.receivers[0].shape[0]), dtype=torch.float64, device=device) for w in wls]
    ens = Ensemble(sims)
    layout = ens.launch_layout()

    def batched():
        ens._run(T, probes, outs)
        ens._advance_clocks(T)

    def sequential():
        for sim, probe, out in zip(sims, probes, outs):
            sim._engine.step_sampled(sim._state(), sim._source_currents(T), T, probe, out)
            sim.steps += T
            sim.time_s = sim.steps * sim.time_step_s

    def timed(fn, reps):
        marks = [torch.cuda.Event(enable_timing=True) for _ in range(reps + 1)]
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        marks[0].record(stream)
        for i in range(reps):
            fn()
            marks[i + 1].record(stream)
        torch.cuda.synchronize()
        return [marks[i].elapsed_time(marks[i + 1]) for i in range(reps)]

    for _ in range(max(args.warmup, 3)):
        batched()
        sequential()
    uuid = getattr(torch.cuda.get_device_properties(local), "uuid", None)
    sampler = ClockSampler(f"GPU-{uuid}" if uuid is not None and not str(uuid).startswith("GPU-") else (str(uuid) if uuid else None))
    b_ms = timed(batched, args.steps)
    clocks = sampler.stop()
    s_ms = timed(sequential, args.steps)
    b_total, s_total = sum(b_ms), sum(s_ms)
    if dist:
        b_total = max_over_ranks(b_total, dist, device)
        s_total = max_over_ranks(s_total, dist, device)
    n = len(sims)
    b_step = b_total / args.steps / T  # ms per leapfrog step of the whole ensemble
    s_step = s_total / args.steps / T
    value = world * n / (RUN_STEPS * b_step / 1e3)
    seq_value = world * n / (RUN_STEPS * s_step / 1e3)

    e2e = None
    if not args.no_e2e:
        obs = [w.receivers for w in wls]
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            traces = ens.record_er_observations(obs, T)
        wall = time.perf_counter() - t0
        if dist:
            wall = max_over_ranks(wall, dist, device)
        e2e = {
            "value": world * n / (RUN_STEPS * wall / args.steps / T),
            "unit": "runs/s",
            "h2d_bytes_per_step": 8 * T * n,
            "d2h_bytes_per_step": int(sum(t.nbytes for t in traces)),
            "api": "Ensemble.record_er_observations",
        }
    peak, peak_kind = measured_peak()
    step_bytes = sum(w.bytes_per_step for w in wls)
    achieved = step_bytes / (b_step / 1e3) / 1e9
    seq_achieved = step_bytes / (s_step / 1e3) / 1e9
    roofline = {
        "bound": "hbm",
        "kernel": "kh_tma_batch + ke_tma_batch + sample_batch_kernel (one batched leapfrog step of all members)",
        "achieved": achieved,
        "peak": peak,
        "peak_source": f"{peak_kind} hbm_gbs (burst copy)",
        "unit": "GB/s",
        "frac": achieved / peak,
        "traffic": None,
        "algorithmic_bytes_per_step": step_bytes,
    }
    cells = [w.cells for w in wls]
    cpu = None
    if rank == 0 and world == 1 and cpu_baseline:
        steppers, sample_cells = oracle_ensemble_sampler()
        oracle_ensemble_time(steppers, sample_cells)
        r = oracle_ensemble_time(steppers, sample_cells, steps=60)
        cpu = {
            "value": r["gcells"] * 1e9 / (RUN_STEPS * statistics.mean(cells)),
            "unit": "runs/s",
            "cores": r["cores"],
            "kind": "port",
            "sample": ensemble_sample_text(r, statistics.mean(cells), "60 leapfrog steps, after 1 warm-up step,"),
        }
        del steppers
    for p in probes:
        p.close()
    if rank == 0:
        line = {
            "metric": ENSEMBLE_METRIC,
            "value": value,
            "unit": "runs/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": b_total / args.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32",
            "data": "synthetic",
            "config": {
                "workload": "config3",
                "members": n,
                "subdivisions": sorted({s.config.subdivision for s in sims}),
                "radial_cells": [min(s.config.radial_cells for s in sims), max(s.config.radial_cells for s in sims)],
                "cells_total": int(sum(cells)),
                "receivers_per_member": int(wls[0].receivers[0].shape[0]),
                "run_steps": RUN_STEPS,
                "time_steps_per_step": T,
                "setup_s": setup_s,
                "launch_layout": layout,
                "autotune": tuning,
                "l2": f"ensemble state {step_bytes // 2 / 1e6:.0f} MB > 126 MB L2, no flush needed",
                "parallelism": f"replicas x{world}",
            },
            "sequential": {"value": seq_value, "unit": "runs/s", "ms_per_step": s_total / args.steps, "achieved_gbs": seq_achieved,
                           "api": "each member's own ifdtd_step_sampled, one member after another"},
            "speedup_vs_sequential": value / seq_value,
            "gcell_updates_per_s": sum(cells) / (b_step / 1e3) / 1e9,
            "roofline": roofline,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": args.steps * T * (2 * layout["groups"] + 2 * layout["solo"] + 1),
            "clocks": clocks,
        }
    ens.close()
    return line if rank == 0 else None


def ensemble_summary(line: dict | None) -> dict | None:
    """The config-3 line abridged for the config-4 line's ``ensemble`` object: batched and
    sequential runs/s of the 64 members, their step times, roofline, e2e, launches and clocks."""

    if line is None:
        return None
    keep = ("metric", "value", "unit", "ms_per_step", "sequential", "speedup_vs_sequential", "gcell_updates_per_s",
            "e2e", "gpu_launches", "clocks")
    out = {k: line[k] for k in keep}
    cfg = line["config"]
    out["config"] = {k: cfg[k] for k in ("workload", "members", "subdivisions", "radial_cells", "cells_total",
                                         "receivers_per_member", "run_steps", "time_steps_per_step", "launch_layout",
                                         "autotune")}
    out["roofline"] = {k: line["roofline"][k] for k in ("bound", "kernel", "achieved", "peak", "unit", "frac")}
    return out


SURROGATE_METRIC = "surrogate traces/s"


def surrogate_main(args, world: int, rank: int, local: int) -> None:
    """Config 5: train the trace surrogate on engine-generated runs (s6 / 40
    cells, 1024 samples, 16 receivers per run), score it on held-out runs
    against the engine, and compare traces/s of the surrogate with the batched engine
    that generated them.  One replica per rank; rank 0 prints the line."""

    import torch

    from ionosphere_fdtd_b200.surrogate import SurrogateEnsemble, architecture, encode_features, generate_traces, relative_l2

    torch.cuda.set_device(local)
    device = f"cuda:{local}"
    steps, receivers = 1024, 16
    n_runs = args.runs + args.eval_runs
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    # receivers 1-6 degrees from the source: the pulse (centred at 35 % of the
    # 1024-step window) reaches all of them inside the window
    params, traces = generate_traces(n_runs, subdivision=6, radial_cells=40, steps=steps, receivers=receivers, seed=20260805 + rank,
                                     distance_deg=(1.0, 6.0), batch_members=32, device=device)
    torch.cuda.synchronize()
    gen_s = time.perf_counter() - t0
    scale = float(np.sqrt(np.mean(traces**2)))
    x = torch.tensor(encode_features(params), dtype=torch.bfloat16, device=device)
    y = torch.tensor(traces / scale, dtype=torch.float32, device=device)
    n_train = args.runs * receivers
    shape, stride, chans = args.decoder.split(":")
    seq0, c0 = (int(v) for v in shape.split("x"))
    layers = architecture(samples=steps, t0=seq0, c0=c0, channels=tuple(int(c) for c in chans.split(",")), stride=int(stride))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    # each trace weighted by the inverse of its mean square: the loss is the
    # mean squared relative error, the metric the held-out traces are scored by
    ens, hist = SurrogateEnsemble.train(layers, x[:n_train], y[:n_train], k=4, iterations=args.iterations, batch=args.batch,
                                        lr=args.lr, lr_final=args.lr_final, device=device, seed=11, relative=True, gemm=args.gemm)
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t0
    xe, ye = x[n_train:], y[n_train:]
    # inference rate: the 4-member ensemble over the held-out cases, CUDA events
    for _ in range(3):
        ens.predict(xe)
    reps = max(args.steps, 3)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(reps):
        mean, spread = ens.predict(xe)
    b.record()
    torch.cuda.synchronize()
    infer_ms = a.elapsed_time(b) / reps
    # per-trace relative L2 over traces above 1 % of the median trace norm (a
    # near-empty trace makes the per-trace ratio meaningless), and the global
    # relative L2 over all held-out traces
    norms = ye.norm(dim=1)
    live = norms > 0.01 * norms.median()
    err_all = relative_l2(mean, ye)
    err = err_all[live]
    mean_trace = y[:n_train].mean(dim=0, keepdim=True).expand_as(ye)
    baseline = relative_l2(mean_trace, ye)[live]
    glob = lambda p: float((p - ye).norm() / ye.norm())  # noqa: E731
    n_eval = int(ye.shape[0])
    value = world * n_eval / (infer_ms / 1e3)
    engine_traces_s = world * n_runs * receivers / gen_s
    # solver fallback: the cases whose ensemble spread is above a quantile go back
    # to the engine; the hybrid's rate counts the engine time of those traces
    fallback = {}
    for frac in (0.1, 0.2, 0.3):
        tau = float(torch.quantile(spread, 1.0 - frac))
        back = spread > tau
        hybrid_pred = torch.where(back[:, None], ye, mean)
        hybrid = relative_l2(hybrid_pred, ye)[live]
        n_back = int(back.sum())
        rate = world * n_eval / (infer_ms / 1e3 + n_back / (engine_traces_s / world))
        fallback[f"{int(frac * 100)}%"] = {
            "spread_threshold": tau, "fraction": n_back / n_eval, "global": glob(hybrid_pred),
            "median": float(hybrid.median()), "p90": float(torch.quantile(hybrid, 0.9)), "traces_per_s": rate,
            "accepted_median": float(err_all[~back & live].median()), "accepted_p90": float(torch.quantile(err_all[~back & live], 0.9)),
        }
    # error against source-receiver distance (degrees)
    from ionosphere_fdtd_b200.surrogate import encode_features as _enc

    dist = torch.tensor(_enc(params[n_train:])[:, 4] * 10.0, device=device)
    by_distance = {}
    for lo, hi in ((1.0, 2.0), (2.0, 3.0), (3.0, 4.0), (4.0, 6.0)):
        sel = (dist >= lo) & (dist < hi) & live
        if int(sel.sum()):
            by_distance[f"{lo:g}-{hi:g} deg"] = {"traces": int(sel.sum()), "median": float(err_all[sel].median()),
                                                 "p90": float(torch.quantile(err_all[sel], 0.9))}
    line = {
        "metric": SURROGATE_METRIC,
        "value": value,
        "unit": "traces/s",
        "n_gpus": world,
        "steps": reps,
        "warmup": 3,
        "ms_per_step": infer_ms,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "bf16",
        "data": "synthetic (engine-generated traces)",
        "config": {
            "workload": "config5", "subdivision": 6, "radial_cells": 40, "samples": steps, "receivers_per_run": receivers,
            "train_runs": args.runs, "eval_runs": args.eval_runs, "network": f"MLP 8-512x4 + transposed-conv decoder ({seq0}x{c0}, stride {stride}, channels {chans} -> 1024)",
            "ensemble": 4, "iterations": args.iterations, "batch": args.batch, "lr": [args.lr, args.lr_final],
            "loss": "per-trace relative squared error",
            "gemm": args.gemm, "parallelism": f"replicas x{world}",
        },
        "engine": {"traces_per_s": engine_traces_s, "generation_s": gen_s, "api": "Ensemble.record_er_observations (setup included)"},
        "speedup_vs_engine": value / engine_traces_s,
        "train_s": train_s,
        "final_loss": [float(np.mean(h[-50:])) for h in hist],
        "rel_l2": {"global": glob(mean), "median": float(err.median()), "p90": float(torch.quantile(err, 0.9)),
                   "traces_scored": int(live.sum()), "traces": n_eval, "by_distance": by_distance,
                   "mean_trace_baseline": {"global": glob(mean_trace), "median": float(baseline.median())}},
        "fallback": fallback,
        "e2e": None,
        "gpu_launches": None,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)


def reference_arm(args, world: int, rank: int) -> None:
    if rank != 0:
        return
    if args.workload == "config5":
        print(json.dumps({"impl": "reference", "metric": SURROGATE_METRIC,
                          "unavailable": "the reference has no learned surrogate"}), flush=True)
        return
    if args.workload == "config3":
        ensemble_reference_arm(args)
        return
    per_step = 1
    sim, info = oracle_build(args.workload, None if args.subdivision is None else min(args.subdivision, ORACLE_SAMPLE_SUB[args.workload]))
    stepper = oracle_stepper(sim)
    for _ in range(args.warmup):
        oracle_time(stepper, info, per_step)
    rates, secs = [], 0.0
    for _ in range(args.steps):
        r = oracle_time(stepper, info, per_step)
        rates.append(r["gcells"])
        secs += r["seconds"]
    value = statistics.median(rates)
    sample = (f"{per_step} leapfrog step(s) of s{r['sub']}/L{r['L']} float32 per bench step{r['note']}, the oracle's "
              f"step on PyTorch CPU tensors over {r['cores']} threads (the reference's Torch-on-CPU path); "
              f"Gcell/s = sample cells / step time")
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": UNIT,
        "n_gpus": args.gpus,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": 1e3 * secs / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic",
        "config": workload_config(args.workload, args.subdivision, world),
        "time_steps_per_step": per_step,
        "device": "cpu",
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": r["cores"], "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def tuning_fields(t) -> dict:
    """The launch-geometry fields of a tuning that differ from the automatic plan's
    (patch sizes, staging, producer warps, lane layout, E-phase threads and stages)."""

    from dataclasses import asdict

    from ionosphere_fdtd_b200.engine import Tuning

    default = asdict(Tuning())
    return {k: v for k, v in asdict(t).items() if k != "graph_chunk" and v != default[k]}


def tune_launch_geometry(sim) -> dict:
    """Time the launch geometries that fix no patch size on the simulation's own state
    (restored afterwards) and keep the fastest; every candidate computes the same bits.
    Returns the record for the JSON line; on a failure the automatic geometry stays."""

    from ionosphere_fdtd_b200.autotune import SHAPE_FREE_CANDIDATES, autotune

    t_tune = time.perf_counter()
    try:
        res = autotune(sim, SHAPE_FREE_CANDIDATES, steps=32, repeats=3)
    except (RuntimeError, ValueError) as err:
        return {"seconds": time.perf_counter() - t_tune, "error": str(err)}
    return {
        "seconds": time.perf_counter() - t_tune,
        "candidates": len(SHAPE_FREE_CANDIDATES),
        "best": {**tuning_fields(res.best), "ms_per_step": res.best_ms},
        "timings": [{**tuning_fields(t), "ms_per_step": ms, "error": err} for t, ms, err in res.timings],
    }


def main() -> None:
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        reference_arm(args, world, rank)
        return
    if args.workload == "config3":
        ensemble_main(args, world, rank, local)
        return
    if args.workload == "config5":
        surrogate_main(args, world, rank, local)
        return
    import torch

    from ionosphere_fdtd_b200 import _native as N

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=180), device_id=torch.device("cuda", local))
    device = f"cuda:{local}"
    t_setup = time.perf_counter()
    wl = build(args.workload, device, subdivision=args.subdivision, plasma_frame=args.plasma_frame)
    setup_s = time.perf_counter() - t_setup
    sim = wl.simulation
    tuning = None if args.no_autotune else tune_launch_geometry(sim)
    T = args.time_steps or PLAIN[args.workload]["time_steps"]
    K = args.steps
    stream = torch.cuda.current_stream()
    eng = sim._engine
    lib = N.load()

    # receivers sampled every leapfrog step into device-resident float64 traces
    v, k, w = wl.receivers
    probe = eng.probe("er", v, np.broadcast_to(k[:, None], v.shape), w)
    traces = torch.zeros((T, v.shape[0]), dtype=torch.float64, device=device)

    def device_currents(first_step: int):
        """The source currents I((n + 1/2) dt) of T steps from ``first_step``, on the device."""
        dt = sim.time_step_s
        times = (first_step + np.arange(T, dtype=np.float64) + 0.5) * dt
        series = getattr(sim.source, "current_series", None)
        host = (np.asarray(series(times, dt), dtype=np.float64) if series is not None
                else np.fromiter((sim.source.current_a(float(t), dt) for t in times), dtype=np.float64, count=T))
        return torch.tensor(host, dtype=torch.float64, device=device)

    def bench_step(cur) -> None:
        N.check(lib.ifdtd_step_sampled(eng.plan, ctypes.byref(sim._state()), cur.data_ptr(), T, probe.handle,
                                       traces.data_ptr(), eng.backend.stream_handle()), "ifdtd_step_sampled")
        sim.steps += T
        sim.time_s = sim.steps * sim.time_step_s

    W_ = max(args.warmup, 3)
    warm = [device_currents(sim.steps + i * T) for i in range(W_)]
    for cur in warm:
        bench_step(cur)
    # every timed bench step's currents are uploaded before the timed region
    timed_cur = [device_currents(sim.steps + i * T) for i in range(K)]
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    uuid = getattr(torch.cuda.get_device_properties(local), "uuid", None)
    sampler = ClockSampler(f"GPU-{uuid}" if uuid is not None and not str(uuid).startswith("GPU-") else (str(uuid) if uuid else None))
    marks = [torch.cuda.Event(enable_timing=True) for _ in range(K + 1)]
    torch.cuda.synchronize()
    marks[0].record(stream)
    for i in range(K):
        bench_step(timed_cur[i])
        marks[i + 1].record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    elapsed_ms = marks[0].elapsed_time(marks[K])
    per_step_ms = [marks[i].elapsed_time(marks[i + 1]) for i in range(K)]
    if dist:
        elapsed_ms = max_over_ranks(elapsed_ms, dist, device)
        dist.barrier()
    total_cells = wl.cells * T * K * world
    value = total_cells / (elapsed_ms / 1e3) / 1e9
    trace_finite = bool(torch.isfinite(traces).all())
    probe.close()

    # end to end through the public API: host currents in, receiver traces out
    e2e = None
    if not args.no_e2e:
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(K):
            out = sim.record_er_observations(v, k, w, T)
        wall = time.perf_counter() - t0
        if dist:
            wall = max_over_ranks(wall, dist, device)
        e2e = {
            "value": wl.cells * T * K * world / wall / 1e9,
            "unit": UNIT,
            "h2d_bytes_per_step": 8 * T,
            "d2h_bytes_per_step": int(out.nbytes),
            "api": "GeodesicFDTD.record_er_observations",
        }

    peak, peak_kind = measured_peak()
    step_ms = statistics.median(per_step_ms) / T
    achieved = wl.bytes_per_step / (step_ms / 1e3) / 1e9
    # per-kernel roofline: each phase kernel timed alone after the timed region
    phase_ms = phase_times_ms(sim, 50)
    nbytes = kernel_bytes(sim)
    modes = eng.kernel_modes
    names = {"h_phase": "kh_tma" if modes[0] == "pipeline" else "kh_kernel", "e_phase": "ke_tma" if modes[1] == "pipeline" else "ke_kernel"}
    traffic = traffic_from_profile(args.workload) if args.subdivision is None else {}
    kernels = {
        phase: {
            "kernel": names[phase],
            "launch_ms": phase_ms[phase],
            "algorithmic_bytes_per_launch": nbytes[phase],
            "achieved": nbytes[phase] / (phase_ms[phase] / 1e3) / 1e9,
            "frac": nbytes[phase] / (phase_ms[phase] / 1e3) / 1e9 / peak,
            "traffic": traffic.get(names[phase]),
        }
        for phase in ("h_phase", "e_phase")
    }
    top = max(kernels, key=lambda q: kernels[q]["launch_ms"])
    roofline = {
        "bound": "hbm",
        "kernel": f"{kernels[top]['kernel']} ({top.replace('_', ' ')}, dominant)",
        "achieved": kernels[top]["achieved"],
        "peak": peak,
        "peak_source": f"{peak_kind} hbm_gbs (burst copy; kernels timed alone)",
        "unit": "GB/s",
        "frac": kernels[top]["frac"],
        "traffic": kernels[top]["traffic"],
        "algorithmic_bytes_per_launch": kernels[top]["algorithmic_bytes_per_launch"],
        "kernels": kernels,
        "step": {"achieved": achieved, "frac": achieved / peak, "algorithmic_bytes_per_step": wl.bytes_per_step, "ms": step_ms,
                 "note": "timed region: both phase kernels and the receiver sampling of every leapfrog step"},
    }
    config = workload_config(args.workload, args.subdivision, world)
    n_species, face_frames = eng.species, eng.face_frames
    del wl, sim, eng
    torch.cuda.empty_cache()
    drift = None
    if rank == 0 and world == 1 and not args.no_drift:
        drift = fp32_drift(args.workload, device, T, args.subdivision, args.plasma_frame)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        r = oracle_sample(args.workload, 3)
        cpu = {
            "value": r["gcells"],
            "unit": UNIT,
            "cores": r["cores"],
            "kind": "port",
            "sample": (f"{r['steps']} leapfrog steps of s{r['sub']}/L{r['L']} float32{r['note']} after 1 warm-up step "
                       f"({r['seconds']:.1f} s), the oracle's step on PyTorch CPU tensors over {r['cores']} threads"),
        }
    ensemble = None
    if args.workload == "config4" and args.subdivision is None and not args.no_ensemble:
        # the batched-ensemble form (config 3) on the same GPU, after the s9 state is freed
        torch.cuda.empty_cache()
        ensemble = ensemble_summary(ensemble_measure(args, world, rank, local, dist, cpu_baseline=False))
    if rank == 0:
        line = {
            "metric": METRIC,
            "value": value,
            "unit": UNIT,
            "n_gpus": world,
            "steps": K,
            "warmup": args.warmup,
            "ms_per_step": elapsed_ms / K,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32",
            "data": "synthetic",
            "config": config,
            "time_steps_per_step": T,
            "setup_s": setup_s,
            "autotune": tuning,
            "hbm_gbs": achieved,
            "kernel_modes": list(modes),
            "plasma_frame": {0: "auto: face frames (unmagnetised plasma)", 1: "cartesian", 2: "face frames"}[args.plasma_frame],
            "roofline": roofline,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "fp32_drift": drift,
            "traces_finite": trace_finite,
            # per bench step: H phase, E phase and sampling per leapfrog step, and with the plasma
            # current in face frames one conversion per species each way around the call
            "gpu_launches": (3 * T + (2 * n_species if face_frames else 0)) * K,
            "clocks": clocks,
            "ensemble": ensemble,
        }
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
