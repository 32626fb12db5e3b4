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
with plasma or surface impedance, odd graph chunks and batches of fused plans
are refused.
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
    fused = build_product(CS.CASES["source_s1"], "float32", tuning=Tuning(fused_step=1))
    other = build_product(CS.CASES["source_s1"], "float32")
    with pytest.raises(BackendUnavailableError, match="fused-step plan cannot join a batch"):
        Ensemble([other, fused])
