"""Autotuner for the launch geometry of a simulation's plan.

The tile shapes of the step kernels are the patch sizes of the two phases
(faces per H-phase patch; faces per E-phase patch or the balanced E
partition), the warps that issue the stage copies and the copy engine (TMA
bulk copies, cp.async, or direct global gathers).  ``autotune`` builds a plan
for every candidate from the simulation's own mesh and physics, times
graph-captured steps of each on the simulation's own state with CUDA events,
restores that state, and installs the fastest plan.  Every candidate computes
the same bits (patch size, lane layout, kernel family and the fused
one-launch step do not change any result; every candidate keeps the
simulation's plasma frame, which does), so tuning changes speed only.  ``autotune_ensemble`` tunes the largest member
of each class (by default: mesh level, radial cells, precision and physics)
and gives the winner to the whole class.
"""

from __future__ import annotations

import statistics
from dataclasses import dataclass, field, replace
from typing import Sequence

from .engine import Engine, Tuning
from .errors import BackendUnavailableError

DEFAULT_CANDIDATES: tuple[Tuning, ...] = (
    Tuning(),  # largest H patch whose stage fits twice; balanced E patches; 2 H-phase and 4 E-phase producer warps
    Tuning(producer_warps=1),
    Tuning(producer_warps=3),
    Tuning(faces_per_patch=32),
    Tuning(faces_per_patch=16),
    Tuning(e_faces_per_patch=32),
    Tuning(e_faces_per_patch=16),
    Tuning(staging=3),
    Tuning(staging=1),
    Tuning(lane_layout=2),
    Tuning(e_producer_warps=2),
    Tuning(e_producer_warps=3),
    Tuning(e_threads=576),
    Tuning(e_stages=3),
    # one launch per step with halo recomputation (plans without plasma or
    # surface impedance; the others reject it)
    Tuning(fused_step=1),
    Tuning(fused_step=1, e_faces_per_patch=32),
    Tuning(fused_step=1, e_faces_per_patch=16),
)


@dataclass
class AutotuneResult:
    best: Tuning
    best_ms: float
    # (candidate, median ms per leapfrog step or None, error message or None)
    timings: list[tuple[Tuning, float | None, str | None]] = field(default_factory=list)


def _snapshot(sim) -> dict:
    out = {f: getattr(sim, f).clone() for f in ("er", "et", "hr", "ht")}
    if sim._plasma_coupler is not None:
        out["J"] = [j.clone() for j in sim._plasma_coupler.ade.buffers]
    if sim._surface_impedance_ade is not None:
        out["si"] = sim._surface_impedance_ade.memory.clone()
    return out


def _restore(sim, saved: dict) -> None:
    for f in ("er", "et", "hr", "ht"):
        getattr(sim, f).copy_(saved[f])
    if "J" in saved:
        for j, s in zip(sim._plasma_coupler.ade.buffers, saved["J"]):
            j.copy_(s)
    if "si" in saved:
        sim._surface_impedance_ade.memory.copy_(saved["si"])


def _engine_for(sim, tuning: Tuning) -> Engine:
    return Engine(sim.mesh, sim.radii_m, sim.config.geometry_mode == "full-spherical", sim.time_step_s, sim._physics(),
                  sim.backend, tuning)


def _time_engine(sim, engine: Engine, steps: int, repeats: int) -> float:
    torch = sim.backend.torch
    stream = torch.cuda.current_stream(sim.backend.torch_device)
    state = sim._state()
    engine.step(state, None, steps)  # warm-up: captures the step graphs
    times = []
    for _ in range(repeats):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        engine.step(state, None, steps)
        b.record(stream)
        b.synchronize()
        times.append(a.elapsed_time(b) / steps)
    return statistics.median(times)


def autotune(sim, candidates: Sequence[Tuning] = DEFAULT_CANDIDATES, *, steps: int = 32, repeats: int = 3) -> AutotuneResult:
    """Time every candidate on ``sim`` and install the fastest plan.

    ``steps`` leapfrog steps (one captured graph when it equals the graph
    chunk) are timed ``repeats`` times per candidate; the median counts.  The
    simulation's fields, plasma currents and surface-impedance memory are
    restored afterwards, and its step count and time do not move.  A
    candidate the plan builder rejects (for example a pipelined staging whose
    stage does not fit twice in shared memory), or whose launches the device
    refuses, is recorded with its error."""

    if steps < 1 or repeats < 1:
        raise ValueError("steps and repeats must be positive")
    if not candidates:
        raise ValueError("at least one candidate tuning is required")
    chunk = sim._engine.tuning.graph_chunk
    # the plasma frame changes rounding, not only speed: every candidate keeps the simulation's
    frame = sim._engine.tuning.plasma_frame
    saved = _snapshot(sim)
    result = AutotuneResult(best=sim._engine.tuning, best_ms=float("inf"))
    best_engine = None
    try:
        for cand in candidates:
            tuning = replace(cand, graph_chunk=chunk, plasma_frame=frame)
            try:
                engine = _engine_for(sim, tuning)
            except (ValueError, RuntimeError, BackendUnavailableError) as err:
                result.timings.append((tuning, None, str(err)))
                continue
            try:
                ms = _time_engine(sim, engine, steps, repeats)
            except RuntimeError as err:
                # a launch the device refuses (for example a launch shape with no
                # resident CTA) is recorded like a plan the builder rejects
                engine.close()
                _restore(sim, saved)
                result.timings.append((tuning, None, str(err)))
                continue
            except BaseException:
                engine.close()
                raise
            _restore(sim, saved)
            result.timings.append((tuning, ms, None))
            if ms < result.best_ms:
                if best_engine is not None:
                    best_engine.close()
                best_engine, result.best, result.best_ms = engine, tuning, ms
            else:
                engine.close()
    except BaseException:
        if best_engine is not None:
            best_engine.close()
        raise
    finally:
        _restore(sim, saved)
        sim.backend.synchronize()
    if best_engine is not None:
        old = sim._engine
        sim._engine = best_engine
        sim.backend._engine = best_engine
        old.close()
    return result


def _tuning_class(sim) -> tuple:
    return (
        sim.config.subdivision,
        sim.config.radial_cells,
        sim.backend.itemsize,
        sim._plasma_coupler is not None,
        sim._surface_impedance_ade is not None,
    )


# Candidates that fix no patch size (the plan sizes patches for each member's
# own radial grid), so one winner suits members of different radial cells.
SHAPE_FREE_CANDIDATES: tuple[Tuning, ...] = (
    Tuning(),
    Tuning(producer_warps=1),
    Tuning(producer_warps=3),
    Tuning(e_producer_warps=2),
    Tuning(e_producer_warps=3),
    Tuning(fused_step=1),
    Tuning(fused_step=1, lane_layout=2),
)


def autotune_ensemble(members: Sequence, candidates: Sequence[Tuning] = DEFAULT_CANDIDATES, *, steps: int = 32,
                      repeats: int = 3, key=None) -> dict[tuple, AutotuneResult]:
    """Tune the largest member of every class and install the winner on the
    rest of the class.  Classes default to (subdivision, radial cells,
    precision, plasma, surface impedance); ``key`` may map a member to a
    coarser class (then use candidates that fix no patch size, such as
    ``SHAPE_FREE_CANDIDATES``).  Call it before building the ``Ensemble``: the
    batch reads the members' plans when it is created."""

    classes: dict[tuple, list] = {}
    for m in members:
        classes.setdefault((key or _tuning_class)(m), []).append(m)
    for group in classes.values():
        group.sort(key=lambda m: -m.mesh.n_vertices * m.config.radial_cells)
    out = {}
    for cls, group in classes.items():
        res = autotune(group[0], candidates, steps=steps, repeats=repeats)
        out[cls] = res
        for m in group[1:]:
            if m._engine.tuning != res.best:
                engine = _engine_for(m, res.best)
                old = m._engine
                m._engine = engine
                m.backend._engine = engine
                old.close()
    return out


def main(argv: Sequence[str] | None = None) -> None:
    """Time the candidates on one benchmark workload and print one JSON line
    per candidate (median milliseconds per leapfrog step, or the plan
    builder's refusal): ``python -m ionosphere_fdtd_b200.autotune config1
    --subdivision 9 --radial-cells 80``."""

    import argparse
    import json
    from dataclasses import asdict

    from . import workloads as W

    p = argparse.ArgumentParser(description=main.__doc__)
    p.add_argument("workload", choices=("config1", "config2", "config4"))
    p.add_argument("--subdivision", type=int, default=None)
    p.add_argument("--radial-cells", type=int, default=None)
    p.add_argument("--dtype", choices=("float32", "float64"), default="float32")
    p.add_argument("--steps", type=int, default=32)
    p.add_argument("--repeats", type=int, default=5)
    p.add_argument("--fused-only", action="store_true", help="the default plan, the direct kernels and the fused step only")
    a = p.parse_args(argv)
    kw = {k: v for k, v in (("subdivision", a.subdivision), ("radial_cells", a.radial_cells)) if v is not None}
    wl = getattr(W, a.workload)(device="cuda", dtype=a.dtype, **kw)
    W.seed_fields(wl.simulation)
    cands = DEFAULT_CANDIDATES
    if a.fused_only:
        cands = [Tuning(), Tuning(staging=1)] + [c for c in DEFAULT_CANDIDATES if c.fused_step] + [
            Tuning(fused_step=1, e_faces_per_patch=48), Tuning(fused_step=1, e_faces_per_patch=24),
            Tuning(fused_step=1, e_producer_warps=2), Tuning(fused_step=1, e_producer_warps=3),
            Tuning(fused_step=1, lane_layout=2), Tuning(fused_step=1, staging=1, e_faces_per_patch=32)]
    res = autotune(wl.simulation, cands, steps=a.steps, repeats=a.repeats)
    for t, ms, err in res.timings:
        line = {"workload": a.workload, "cells": wl.cells, "dtype": a.dtype, "tuning": asdict(t), "ms_per_step": ms}
        if ms is not None:
            line["gcell_per_s"] = wl.cells / (ms / 1e3) / 1e9
            line["algorithmic_gbs"] = wl.bytes_per_step / (ms / 1e3) / 1e9
        if err:
            line["error"] = err
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
