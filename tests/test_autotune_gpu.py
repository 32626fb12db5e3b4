"""Autotuner: every candidate plan is timed on the simulation's own state, the
state is restored, and the fastest plan is installed.  Plans of different
patch sizes and kernel families compute the same bits, so a tuned simulation
must continue bitwise like an untuned twin."""

import numpy as np
import pytest

import cases as CS
from casebuild import build_product

pytestmark = pytest.mark.gpu


def _arrays(sim) -> dict[str, np.ndarray]:
    out = {f: sim.to_numpy(getattr(sim, f)) for f in ("er", "et", "hr", "ht")}
    if sim._plasma_coupler is not None:
        for i, j in enumerate(sim._plasma_coupler.ade.current_density):
            out[f"plasma_current_{i}"] = sim.to_numpy(j)
    if sim._surface_impedance_ade is not None:
        out["si_memory"] = sim.to_numpy(sim._surface_impedance_ade.memory)
    return out


def _same(a: dict, b: dict) -> bool:
    return a.keys() == b.keys() and all(np.array_equal(a[k], b[k]) for k in a)


@pytest.mark.parametrize("name", ["plasma_drude_s2", "config4_mini_s2", "source_s1"])
def test_autotune_installs_the_fastest_plan_and_keeps_the_state(name):
    from ionosphere_fdtd_b200.autotune import DEFAULT_CANDIDATES, autotune

    case = CS.CASES[name]
    sim, twin = build_product(case, "float32"), build_product(case, "float32")
    sim.step(5)
    twin.step(5)
    before = _arrays(sim)
    res = autotune(sim, steps=8, repeats=2)
    assert _same(_arrays(sim), before) and sim.steps == 5
    assert len(res.timings) == len(DEFAULT_CANDIDATES)
    timed = [(t, ms) for t, ms, err in res.timings if ms is not None]
    assert timed
    assert res.best == min(timed, key=lambda x: x[1])[0] and res.best_ms == min(ms for _, ms in timed)
    assert sim._engine.tuning == res.best
    # the fused candidates are timed on plans without plasma or surface impedance only
    fused_timed = [t for t, ms, err in res.timings if t.fused_step and ms is not None]
    assert bool(fused_timed) == (name == "source_s1")
    sim.step(40)
    twin.step(40)
    assert _same(_arrays(sim), _arrays(twin))


def test_tuned_ensemble_members_match_untuned_twins():
    from ionosphere_fdtd_b200 import Ensemble
    from ionosphere_fdtd_b200.autotune import autotune_ensemble

    names = ["plasma_drude_s2", "plasma_drude_s2", "source_s1"]
    together = [build_product(CS.CASES[n], "float32") for n in names]
    alone = [build_product(CS.CASES[n], "float32") for n in names]
    tuned = autotune_ensemble(together, steps=8, repeats=2)
    assert len(tuned) == 2
    assert together[1]._engine.tuning == together[0]._engine.tuning
    with Ensemble(together) as ens:
        ens.step(36)
    for sim in alone:
        sim.step(36)
    for a, b in zip(together, alone):
        assert _same(_arrays(a), _arrays(b))
