"""Multi-rank plumbing of bench.py on CPU (gloo, world size 2): the timing
reduction gives every rank the maximum over ranks, and the reference arm does
its work on rank 0 only."""

import os
import socket
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out) -> None:
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, str(ROOT))
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        out[rank] = bench.max_over_ranks(10.0 * (rank + 1), dist, "cpu")
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_timing_is_the_maximum_over_ranks():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as manager:
        out = manager.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        assert dict(out) == {0: 20.0, 1: 20.0}


def test_single_rank_reduction_is_the_value():
    sys.path.insert(0, str(ROOT))
    import bench

    assert bench.max_over_ranks(3.5, None, "cpu") == 3.5


def test_reference_arm_works_on_rank_zero_only(capsys):
    sys.path.insert(0, str(ROOT))
    import bench

    class Args:
        workload, steps, warmup, gpus = "config2", 1, 0, 2

    bench.reference_arm(Args, world=2, rank=1)  # returns at once: no oracle run, no output
    assert capsys.readouterr().out == ""


def test_surrogate_reference_arm_reports_unavailable(capsys):
    import json

    sys.path.insert(0, str(ROOT))
    import bench

    class Args:
        workload, steps, warmup, gpus = "config5", 1, 0, 1

    bench.reference_arm(Args, world=1, rank=0)
    line = json.loads(capsys.readouterr().out)
    assert line["impl"] == "reference" and "unavailable" in line


def test_ensemble_cells_follow_the_member_generator():
    sys.path.insert(0, str(ROOT))
    import bench

    from ionosphere_fdtd_b200 import workloads as W

    draws = W.config3_draws(members=64)
    cells = bench.ensemble_cells(64)
    assert len(cells) == 64
    assert cells == [(10 * 4 ** d["subdivision"] + 2) * d["radial_cells"] for d in draws]
    assert {d["subdivision"] for d in draws} == {5, 6, 7}
    assert all(24 <= d["radial_cells"] <= 60 for d in draws)
    assert all(1e-8 <= d["sigma0"] <= 1e-6 and 1e-3 <= d["ground"] <= 1e-1 for d in draws)
    assert all(55e3 <= d["h0"] <= 70e3 and 3e3 <= d["zeta"] <= 6e3 and 10.0 <= d["carrier"] <= 60.0 for d in draws)


def test_ensemble_summary_keeps_the_runs_per_second_record():
    sys.path.insert(0, str(ROOT))
    import bench

    assert bench.ensemble_summary(None) is None
    config = {k: k for k in ("workload", "members", "subdivisions", "radial_cells", "cells_total",
                             "receivers_per_member", "run_steps", "time_steps_per_step", "launch_layout",
                             "autotune", "setup_s", "l2", "parallelism")}
    roofline = {"bound": "hbm", "kernel": "k", "achieved": 1.0, "peak": 2.0, "unit": "GB/s", "frac": 0.5,
                "traffic": None, "peak_source": "p", "algorithmic_bytes_per_step": 3}
    line = {"metric": bench.ENSEMBLE_METRIC, "value": 2.8, "unit": "runs/s", "ms_per_step": 450.0,
            "sequential": {"value": 2.4}, "speedup_vs_sequential": 2.8 / 2.4, "gcell_updates_per_s": 46.0,
            "e2e": None, "gpu_launches": 10, "clocks": None, "config": config, "roofline": roofline,
            "cpu_baseline": None, "n_gpus": 1}
    out = bench.ensemble_summary(line)
    assert out["metric"] == bench.ENSEMBLE_METRIC and out["value"] == 2.8 and out["sequential"] == {"value": 2.4}
    assert "setup_s" not in out["config"] and out["config"]["members"] == "members"
    assert out["roofline"] == {k: roofline[k] for k in ("bound", "kernel", "achieved", "peak", "unit", "frac")}
    assert "cpu_baseline" not in out and "n_gpus" not in out


def test_launch_geometry_record_lists_every_candidate(monkeypatch):
    """The bench's tuning record from an autotune result (the timing itself needs a GPU)."""

    sys.path.insert(0, str(ROOT))
    import bench
    import ionosphere_fdtd_b200.autotune as A

    def fake(sim, candidates, *, steps, repeats):
        assert candidates == A.SHAPE_FREE_CANDIDATES and steps == 32 and repeats == 3
        timings = [(c, 1.0 + i, None) for i, c in enumerate(candidates)]
        timings[-1] = (candidates[-1], None, "stage does not fit")
        return A.AutotuneResult(best=candidates[0], best_ms=1.0, timings=timings)

    monkeypatch.setattr(A, "autotune", fake)
    rec = bench.tune_launch_geometry(object())
    assert rec["candidates"] == len(A.SHAPE_FREE_CANDIDATES) == len(rec["timings"])
    assert rec["best"] == {**bench.tuning_fields(A.SHAPE_FREE_CANDIDATES[0]), "ms_per_step": 1.0}
    assert rec["timings"][1] == {"producer_warps": A.SHAPE_FREE_CANDIDATES[1].producer_warps, "ms_per_step": 2.0, "error": None}
    assert rec["timings"][-1]["error"] == "stage does not fit"

    def failing(sim, candidates, *, steps, repeats):
        raise RuntimeError("plan build failed")

    monkeypatch.setattr(A, "autotune", failing)
    assert bench.tune_launch_geometry(object())["error"] == "plan build failed"


def test_profile_traffic_and_clock_records_parse():
    sys.path.insert(0, str(ROOT))
    import bench

    for workload in ("config2", "config4"):
        traffic = bench.traffic_from_profile(workload)
        assert set(traffic) == {"kh_tma", "ke_tma"} and all(v > 1e8 for v in traffic.values())
    assert bench.traffic_from_profile("no-such-workload") == {}

    sampler = bench.ClockSampler(None)  # no nvidia-smi process: parse a recorded file instead
    sampler.path.write_text(
        "1965, 1965, 700.1, Not Active, Not Active, Not Active, Not Active\n"
        "1800, 1965, 990.0, Not Active, Not Active, Not Active, Active\n"
        "[N/A], 1965, 10.0, Not Active, Not Active, Not Active, Not Active\n"
        "1815, 1965, 995.5, Not Active, Not Active, Not Active, Active\n"
    )

    class Done:
        def terminate(self):
            pass

        def wait(self, timeout):
            return 0

    sampler.proc, sampler.handle = Done(), open(os.devnull, "w")
    rec = sampler.stop()
    assert rec == {"sm_mhz": 1815.0, "sm_max_mhz": 1965.0, "reasons": ["sw_power_cap"], "samples": 3}
    assert not sampler.path.exists()


def test_reference_arm_loads_nothing_of_the_product():
    """The reference arm times the oracle on its own mesh and inputs: the product
    package is never imported and its CUDA library never mapped, and its config
    object is the engine arm's."""

    import json
    import subprocess

    code = r"""
import json, sys
sys.path.insert(0, sys.argv[1])
import bench

class Args:
    workload, steps, warmup, gpus, subdivision = "config4", 1, 0, 1, 2

bench.reference_arm(Args, world=1, rank=0)
maps = open("/proc/self/maps").read()
print(json.dumps({"imported": any(m.startswith("ionosphere_fdtd_b200") for m in sys.modules),
                  "mapped": "libifdtd" in maps,
                  "config": bench.workload_config("config4", 2, 1)}))
"""
    out = subprocess.run([sys.executable, "-c", code, str(ROOT)], capture_output=True, text=True, timeout=600, check=True)
    lines = [json.loads(x) for x in out.stdout.splitlines() if x.startswith("{")]
    line, probe = lines[0], lines[1]
    assert line["impl"] == "reference" and line["value"] > 0.0
    assert line["config"] == probe["config"]
    assert not probe["imported"] and not probe["mapped"]
