"""Batched ensembles (``Ensemble``, C ABI ``ifdtd_batch_*``).

Members of different mesh levels, radial grids, materials, sources and physics
advance together; every member must come out bitwise equal to the same member
advanced on its own, because the batched kernels run the same per-patch
arithmetic.  The step counts cross a captured-graph chunk (32 steps) so both
the graph and the direct-launch paths of the batched step are covered.
"""

import numpy as np
import pytest

import cases as CS
from casebuild import build_product

pytestmark = pytest.mark.gpu

MIXED = [
    "source_s1",
    "tangential_s1",
    "surface_s1",
    "plasma_magnetized_s1",
    "plasma_drude_s2",
    "config4_mini_s2",
    "config1_s2",
    "thin_shell_s1",
    "trapezoidal_s1",
    "adaptive_s1",  # vertex degree 7-8: the 12-slot kernels, a group of their own
    "adaptive_plasma_si_s1",
]


def _arrays(sim) -> dict[str, np.ndarray]:
    out = {f: sim.to_numpy(getattr(sim, f)) for f in ("er", "et", "hr", "ht")}
    if sim._plasma_coupler is not None:
        for i, j in enumerate(sim._plasma_coupler.ade.current_density):
            out[f"plasma_current_{i}"] = sim.to_numpy(j)
    if sim._surface_impedance_ade is not None:
        out["si_memory"] = sim.to_numpy(sim._surface_impedance_ade.memory)
    return out


def _assert_same(a, b, label):
    x, y = _arrays(a), _arrays(b)
    assert x.keys() == y.keys()
    for k in x:
        assert np.array_equal(x[k], y[k]), (label, k, float(np.max(np.abs(x[k] - y[k]))))
    assert a.steps == b.steps and a.time_s == b.time_s


@pytest.mark.parametrize("dtype", ["float32", "float64"])
def test_batched_members_match_their_own_runs_bitwise(dtype):
    from ionosphere_fdtd_b200 import Ensemble

    together = [build_product(CS.CASES[n], dtype) for n in MIXED]
    alone = [build_product(CS.CASES[n], dtype) for n in MIXED]
    with Ensemble(together) as ens:
        layout = ens.launch_layout()
        assert layout["groups"] >= 2 and layout["solo"] == 0, layout
        ens.step(37)
        ens.step(3)
    for sim in alone:
        sim.step(37)
        sim.step(3)
    for name, a, b in zip(MIXED, together, alone):
        _assert_same(a, b, name)
        assert a._engine.status_word() == 0


def test_member_on_direct_kernels_runs_on_its_own_inside_the_batch():
    from ionosphere_fdtd_b200 import Ensemble
    from ionosphere_fdtd_b200.engine import Tuning

    names = ["plasma_drude_s2", "source_s1"]
    direct = Tuning(staging=1, graph_chunk=32)
    together = [build_product(CS.CASES[names[0]], "float32", tuning=direct), build_product(CS.CASES[names[1]], "float32")]
    alone = [build_product(CS.CASES[names[0]], "float32", tuning=direct), build_product(CS.CASES[names[1]], "float32")]
    with Ensemble(together) as ens:
        assert ens.launch_layout()["solo"] == 1
        ens.step(35)
    for sim in alone:
        sim.step(35)
    for name, a, b in zip(names, together, alone):
        _assert_same(a, b, name)


def test_batched_receiver_traces_match_each_members_own_recording():
    from ionosphere_fdtd_b200 import Ensemble

    names = ["config1_s2", "plasma_drude_s2", "source_s1"]
    together = [build_product(CS.CASES[n], "float32") for n in names]
    alone = [build_product(CS.CASES[n], "float32") for n in names]
    rng = np.random.default_rng(7)
    obs = []
    for sim in alone:
        rows = 5
        v = rng.integers(0, sim.mesh.n_vertices, size=(rows, 3))
        w = rng.random((rows, 3))
        w /= w.sum(axis=1, keepdims=True)
        layers = rng.integers(0, len(sim.radii_m), size=rows)
        obs.append((v, layers, w))
    obs[1] = None  # a member without receivers
    with Ensemble(together) as ens:
        traces = ens.record_er_observations(obs, 40)
    for i, sim in enumerate(alone):
        if obs[i] is None:
            sim.step(40)
            assert traces[i] is None
        else:
            expected = sim.record_er_observations(*obs[i], 40)
            assert traces[i].shape == expected.shape
            assert np.array_equal(traces[i], expected), names[i]
        _assert_same(together[i], sim, names[i])


def test_members_with_different_launch_tunings_form_groups_and_match_their_own_runs():
    from ionosphere_fdtd_b200 import Ensemble
    from ionosphere_fdtd_b200.engine import Tuning

    # producer warps 1 / 2 / 3 and the cp.async copy engine: four groups, two of
    # which share a kernel instantiation with different shared-memory sizes
    # (and rows on 8-lane boundaries: a fifth group)
    spec = [
        ("config1_s2", Tuning(producer_warps=1)),
        ("plasma_drude_s2", Tuning()),
        ("source_s1", Tuning(producer_warps=3)),
        ("config4_mini_s2", Tuning(staging=3)),
        ("surface_s1", Tuning(producer_warps=1)),
        ("plasma_magnetized_s1", Tuning(lane_layout=2)),
    ]
    together = [build_product(CS.CASES[n], "float32", tuning=t) for n, t in spec]
    alone = [build_product(CS.CASES[n], "float32", tuning=t) for n, t in spec]
    with Ensemble(together) as ens:
        assert ens.launch_layout()["groups"] == 5
        ens.step(34)
    for sim in alone:
        sim.step(34)
    for (name, _), a, b in zip(spec, together, alone):
        _assert_same(a, b, name)


def test_ensemble_refuses_members_whose_plan_changed():
    from ionosphere_fdtd_b200 import Ensemble
    from ionosphere_fdtd_b200.autotune import SHAPE_FREE_CANDIDATES, autotune

    sims = [build_product(CS.CASES["source_s1"], "float32"), build_product(CS.CASES["plasma_drude_s2"], "float32")]
    with Ensemble(sims) as ens:
        ens.step(2)
        autotune(sims[1], SHAPE_FREE_CANDIDATES[1:2], steps=4, repeats=1)  # installs a new plan
        with pytest.raises(ValueError, match="plan changed"):
            ens.step(1)
