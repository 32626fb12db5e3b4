"""Control flow of the autotuner on the host (no device): every candidate is
timed on the simulation's state, restored afterwards, and the fastest plan is
installed; a candidate whose plan the builder rejects or whose launches the
device refuses is recorded with its error and the tuning goes on.  The engine
builder, the timer and the state snapshot are replaced by fakes."""

from types import SimpleNamespace

import pytest

from ionosphere_fdtd_b200 import autotune as A
from ionosphere_fdtd_b200.engine import Tuning


class FakeEngine:
    def __init__(self, tuning):
        self.tuning = tuning
        self.closed = False

    def close(self):
        self.closed = True


def _fake_sim():
    backend = SimpleNamespace(synchronize=lambda: None, _engine=None)
    sim = SimpleNamespace(backend=backend, restores=0)
    sim._engine = FakeEngine(Tuning(graph_chunk=16, plasma_frame=1))
    backend._engine = sim._engine
    return sim


def test_refused_launches_and_rejected_plans_are_recorded_and_tuning_goes_on(monkeypatch):
    times = {1: 3.0, 2: 2.0, 3: 1.0}
    built = []

    def engine_for(sim, tuning):
        if tuning.producer_warps == 4:
            raise ValueError("plan rejected")
        built.append(FakeEngine(tuning))
        return built[-1]

    def time_engine(sim, engine, steps, repeats):
        if engine.tuning.producer_warps == 3:
            raise RuntimeError("ifdtd_step: graph capture: invalid configuration argument")
        return times[engine.tuning.producer_warps]

    def restore(sim, saved):
        sim.restores += 1

    monkeypatch.setattr(A, "_engine_for", engine_for)
    monkeypatch.setattr(A, "_time_engine", time_engine)
    monkeypatch.setattr(A, "_snapshot", lambda sim: {})
    monkeypatch.setattr(A, "_restore", restore)
    sim = _fake_sim()
    old = sim._engine
    cands = [Tuning(producer_warps=1), Tuning(producer_warps=3), Tuning(producer_warps=4), Tuning(producer_warps=2)]
    res = A.autotune(sim, cands)
    errors = {t.producer_warps: err for t, ms, err in res.timings}
    assert errors[3].endswith("invalid configuration argument") and errors[4] == "plan rejected"
    assert errors[1] is None and errors[2] is None
    # the fastest timed candidate is installed; every candidate kept the graph chunk and plasma frame
    assert res.best.producer_warps == 2 and res.best_ms == 2.0
    assert sim._engine.tuning.producer_warps == 2 and sim.backend._engine is sim._engine
    assert all(t.graph_chunk == 16 and t.plasma_frame == 1 for t, _, _ in res.timings)
    # engines that lost or failed are closed, the old plan too; the state was restored after each timing
    assert old.closed and all(e.closed for e in built if e is not sim._engine)
    assert not sim._engine.closed
    assert sim.restores >= 3


def test_an_interrupt_while_timing_closes_the_candidate_and_propagates(monkeypatch):
    built = []

    def engine_for(sim, tuning):
        built.append(FakeEngine(tuning))
        return built[-1]

    def time_engine(sim, engine, steps, repeats):
        raise KeyboardInterrupt

    monkeypatch.setattr(A, "_engine_for", engine_for)
    monkeypatch.setattr(A, "_time_engine", time_engine)
    monkeypatch.setattr(A, "_snapshot", lambda sim: {})
    monkeypatch.setattr(A, "_restore", lambda sim, saved: None)
    sim = _fake_sim()
    old = sim._engine
    with pytest.raises(KeyboardInterrupt):
        A.autotune(sim, [Tuning(producer_warps=1)])
    assert built[0].closed and sim._engine is old and not old.closed
