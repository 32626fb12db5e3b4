"""The fused one-launch step (``Tuning(fused_step=1)``).

Each CTA of the fused kernel computes the new H of its E patch's halo from the
old state into shared memory, then the new E of the vertices and edges it
owns; halo H values are recomputed with the owner's arithmetic, so the fused
plan must reproduce the two-launch plan bit for bit.  The step reads one copy
of the fields and writes the other, so the tests cover even and odd step
counts (an odd count ends with a copy back into the caller's arrays), steps
inside and across a captured graph chunk, direct launches (graph_chunk 0),
the sampled step's receiver traces, several patch sizes, both kernels (the
pipelined ring, whose stage holds the old rows and takes the new H in place,
and direct gathers) and the 12-slot vertex tables of adaptive meshes.  Plans
with plasma or surface impedance and odd graph chunks are refused; fused
members of an ensemble run the batched fused kernel and must match their own
runs bit for bit.
"""

import numpy as np
import pytest

import cases as CS
from casebuild import build_product, run_product

pytestmark = pytest.mark.gpu

NO_PLASMA = ["source_s1", "tangential_s1", "config1_s2", "thin_shell_s1", "trapezoidal_s1", "adaptive_s1"]


def _fields(sim) -> dict[str, np.ndarray]:
    return {f: sim.to_numpy(getattr(sim, f)) for f in ("er", "et", "hr", "ht")}


# the ring (TMA bulk copies, cp.async, rows on 8-lane boundaries, fixed patch
# sizes, more compute threads) and the direct-gather kernel
KERNELS = [
    (dict(), "pipeline"),
    (dict(staging=3), "pipeline"),
    (dict(lane_layout=2), "pipeline"),
    (dict(e_faces_per_patch=16, e_producer_warps=2), "pipeline"),
    (dict(staging=1), "direct"),
    (dict(staging=1, e_faces_per_patch=32), "direct"),
]


@pytest.mark.parametrize("kernel", KERNELS, ids=lambda k: str(k[0]))
@pytest.mark.parametrize("dtype", ["float32", "float64"])
@pytest.mark.parametrize("name", NO_PLASMA)
def test_fused_step_equals_two_launch_step_bitwise(name, dtype, kernel):
    from ionosphere_fdtd_b200.engine import Tuning

    ref = run_product(CS.CASES[name], dtype)
    fused = run_product(CS.CASES[name], dtype, tuning=Tuning(fused_step=1, **kernel[0]))
    assert fused["_sim"]._engine.kernel_modes == ("fused", kernel[1])
    for key in ("er", "et", "hr", "ht", "traces"):
        if key in ref:
            np.testing.assert_array_equal(fused[key], ref[key], err_msg=key)
    assert fused["_sim"]._engine.status_word() == 0


@pytest.mark.parametrize("tuning", [dict(graph_chunk=32), dict(graph_chunk=0), dict(graph_chunk=4, e_faces_per_patch=16),
                                    dict(graph_chunk=32, e_faces_per_patch=64, staging=1), dict(graph_chunk=0, staging=1)])
@pytest.mark.parametrize("counts", [(1,), (2, 3), (33,), (31, 1, 32)])
def test_fused_step_counts_and_graph_chunks(counts, tuning):
    """Step counts that end in either copy, inside and across graph chunks:
    after every call the caller's arrays hold the same bits as the two-launch
    plan after the same calls."""

    from ionosphere_fdtd_b200.engine import Tuning

    case = CS.CASES["source_s1"]
    ref = build_product(case, "float32")
    fused = build_product(case, "float32", tuning=Tuning(fused_step=1, **tuning))
    for n in counts:
        ref.step(n)
        fused.step(n)
        a, b = _fields(ref), _fields(fused)
        for key in a:
            np.testing.assert_array_equal(b[key], a[key], err_msg=f"{key} after {n} steps")
    assert np.abs(_fields(fused)["er"]).max() > 0.0


def test_fused_step_sampled_traces_across_a_chunk():
    from ionosphere_fdtd_b200.engine import Tuning

    case = CS.CASES["config1_s2"]
    ref = build_product(case, "float32")
    fused = build_product(case, "float32", tuning=Tuning(fused_step=1))
    v, k, w = CS.receiver_rows(ref.mesh.n_vertices, ref.altitudes_m, 5, 8)
    for n in (37, 5):
        np.testing.assert_array_equal(fused.record_er_observations(v, k, w, n), ref.record_er_observations(v, k, w, n))


def test_fused_step_refusals():
    from ionosphere_fdtd_b200 import Ensemble
    from ionosphere_fdtd_b200.engine import Tuning
    from ionosphere_fdtd_b200.errors import BackendUnavailableError

    for name in ("plasma_drude_s2", "surface_s1"):
        with pytest.raises(BackendUnavailableError, match="fused_step supports plans without plasma"):
            build_product(CS.CASES[name], "float32", tuning=Tuning(fused_step=1))
    with pytest.raises(ValueError, match="even graph_chunk"):
        build_product(CS.CASES["source_s1"], "float32", tuning=Tuning(fused_step=1, graph_chunk=3))
    with pytest.raises(ValueError, match="fused_step must be 0 or 1"):
        build_product(CS.CASES["source_s1"], "float32", tuning=Tuning(fused_step=2))
    direct = build_product(CS.CASES["source_s1"], "float32", tuning=Tuning(fused_step=1, staging=1))
    other = build_product(CS.CASES["source_s1"], "float32")
    with pytest.raises(BackendUnavailableError, match="fused-step plan on direct gathers cannot join a batch"):
        Ensemble([other, direct])


def _state(sim) -> dict[str, np.ndarray]:
    out = _fields(sim)
    if sim._plasma_coupler is not None:
        for i, j in enumerate(sim._plasma_coupler.ade.current_density):
            out[f"plasma_current_{i}"] = sim.to_numpy(j)
    if sim._surface_impedance_ade is not None:
        out["si_memory"] = sim.to_numpy(sim._surface_impedance_ade.memory)
    return out


@pytest.mark.parametrize("dtype", ["float32", "float64"])
def test_fused_members_in_an_ensemble_match_their_own_runs(dtype):
    """Fused-step members (two tunings, so two fused groups, and the 12-slot
    adaptive mesh) batched with two-launch members: after odd and even step
    counts and a sampled run across a graph chunk, every member holds the same
    bits as the same member advanced on its own."""

    from ionosphere_fdtd_b200 import Ensemble
    from ionosphere_fdtd_b200.engine import Tuning

    spec = [("source_s1", Tuning(fused_step=1)), ("config1_s2", Tuning(fused_step=1, lane_layout=2)),
            ("adaptive_s1", Tuning(fused_step=1)), ("plasma_drude_s2", Tuning()), ("config1_s2", Tuning())]
    together = [build_product(CS.CASES[n], dtype, tuning=t) for n, t in spec]
    alone = [build_product(CS.CASES[n], dtype, tuning=t) for n, t in spec]
    assert together[0]._engine.kernel_modes == ("fused", "pipeline")
    rows = [CS.receiver_rows(m.mesh.n_vertices, m.altitudes_m, 3 + i, 4) for i, m in enumerate(together)]
    with Ensemble(together) as ens:
        assert ens.launch_layout()["groups"] >= 4 and ens.launch_layout()["solo"] == 0
        for n in (3, 2):
            ens.step(n)
            for sim in alone:
                sim.step(n)
            for a, b in zip(together, alone):
                ea, eb = _state(a), _state(b)
                for key in ea:
                    np.testing.assert_array_equal(ea[key], eb[key], err_msg=f"{key} after {n} steps")
        traces = ens.record_er_observations(rows, 37)
    for sim, (v, k, w), tr in zip(alone, rows, traces):
        np.testing.assert_array_equal(tr, sim.record_er_observations(v, k, w, 37))
    for a, b in zip(together, alone):
        ea, eb = _state(a), _state(b)
        for key in ea:
            np.testing.assert_array_equal(ea[key], eb[key], err_msg=key)
        assert a._engine.status_word() == 0
