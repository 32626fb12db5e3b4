"""Parity of the CUDA engine with the reference (golden fixtures) and the oracle.

Tolerances:
* float64 engine vs reference float64: per (E, H) group relative L2 < 1e-11
  and elementwise rtol 1e-8 against the group scale (operation order differs
  from NumPy's, so results agree to accumulated rounding, not bitwise);
* float32 engine vs reference float64: per-group relative L2 <= 1e-5 (the
  north-star bound) for every case, the 1000-step config-1 run included
  (measured 2.0e-7 / 3.5e-7 for E / H there); receiver traces likewise; the
  reference's own FP32 pin (tests/test_backends.py:262-293) keeps its 2e-5.
"""

import numpy as np
import pytest

import cases as C
from casebuild import build_product, golden, grouped_rel_l2, rel_l2, run_product

pytestmark = pytest.mark.gpu

STATE = ("er", "et", "hr", "ht")


def _scale(ref, key):
    groups = {"er": ("er", "et"), "et": ("er", "et"), "hr": ("hr", "ht"), "ht": ("hr", "ht")}
    return max(float(np.max(np.abs(ref[n]))) for n in groups.get(key, (key,)) if n in ref) or 1.0


@pytest.mark.parametrize("name", sorted(C.CASES))
def test_float64_engine_matches_reference(name):
    ref = golden(f"case_{name}")
    out = run_product(C.CASES[name], "float64")
    assert float(out["time_step_s"]) == pytest.approx(float(ref["time_step_s"]), rel=1e-14)
    errs = grouped_rel_l2(out, ref)
    assert max(errs.values()) < 1e-11, errs
    for key in ref:
        if key in ("time_step_s", "cfl_limit_s", "max_abs"):
            continue
        np.testing.assert_allclose(out[key], ref[key], rtol=1e-8, atol=1e-10 * _scale(ref, key), err_msg=key)


@pytest.mark.parametrize("name", sorted(C.CASES))
def test_float32_engine_tracks_reference_float64(name):
    ref = golden(f"case_{name}")
    out = run_product(C.CASES[name], "float32")
    limit = 1e-5
    errs = grouped_rel_l2(out, ref)
    assert max(errs.values()) < limit, errs
    if "traces" in ref:
        assert rel_l2(out["traces"], ref["traces"]) < limit
    for key in ("si_memory", "plasma_current_0"):
        if key in ref:
            assert rel_l2(out[key], ref[key]) < 10 * limit, key


def test_float32_pin_of_the_reference():
    """80 steps of the default source case: FP32 engine vs reference FP64 < 2e-5,
    and Hr round-off below 1e-6 max|Ht| (tests/test_backends.py:262-293)."""

    case = dict(C.CASES["source_s1"], steps=80)
    ref = golden("case_source_s1_f64x80")
    out = run_product(case, "float32")
    errs = grouped_rel_l2(out, ref)
    assert max(errs.values()) < 2.0e-5, errs
    assert np.max(np.abs(out["hr"] - ref["hr"])) < 1.0e-6 * np.max(np.abs(ref["ht"]))
    sim = out["_sim"]
    assert sim.er.dtype.itemsize == 4 and sim.memory_bytes * 2 == sum(ref[f].nbytes for f in STATE)


def test_receiver_traces_start_with_initial_state():
    case = C.CASES["config4_mini_s2"]
    ref = golden("case_config4_mini_s2")
    out = run_product(case, "float64")
    assert out["traces"].shape == ref["traces"].shape
    np.testing.assert_allclose(out["traces"], ref["traces"], rtol=1e-8, atol=1e-10 * np.max(np.abs(ref["traces"])))


def test_h_observations_with_decimation_match_reference():
    ref = golden("obs_h_source_s1")
    sim = build_product(C.CASES["source_s1"], "float64")
    hr, ht = sim.record_h_observations(
        np.asarray(((0,), (5,))),
        np.asarray(((2,), (4,))),
        np.asarray(((1.0,), (1.0,))),
        np.asarray(((0, 1, 2), (7, 8, 9))),
        np.asarray(((2, 2, 2), (0, 3, 6))),
        np.asarray(((0.2, -0.3, 0.5), (1.0, 0.5, -0.5))),
        11,
        sample_every=3,
    )
    assert sim.steps == 11
    np.testing.assert_allclose(hr, ref["hr"], rtol=1e-8, atol=1e-10 * np.max(np.abs(ref["ht"])))
    np.testing.assert_allclose(ht, ref["ht"], rtol=1e-8, atol=1e-10 * np.max(np.abs(ref["ht"])))


def test_receiver_helper_matches_the_reference_helper():
    """record_receiver_traces (visualization.py:212-252) through the engine's sampled
    steps: the reference's receiver placement, sample rows, clock and labels."""

    from ionosphere_fdtd_b200 import Receiver, record_receiver_traces

    spec = C.RECEIVER_TRACES
    ref = golden(f"receiver_traces_{spec['case']}")
    sim = build_product(C.CASES[spec["case"]], "float64")
    out = record_receiver_traces(sim, [Receiver(*r) for r in spec["receivers"]], spec["steps"],
                                 sample_every=spec["sample_every"])
    assert out.labels == tuple(str(x) for x in ref["labels"])
    np.testing.assert_allclose(out.time_s, ref["time_s"], rtol=1e-14, atol=0)
    scale = float(np.max(np.abs(ref["er_v_m"])))
    np.testing.assert_allclose(out.er_v_m, ref["er_v_m"], rtol=1e-8, atol=1e-10 * scale)
    assert sim.steps == int(ref["steps_after"])


@pytest.mark.parametrize("name", ["config4_mini_s2", "plasma_magnetized_s1", "surface_map_s2"])
def test_engine_is_bitwise_repeatable(name):
    first = run_product(C.CASES[name], "float32")
    second = run_product(C.CASES[name], "float32")
    for f in STATE:
        np.testing.assert_array_equal(first[f], second[f])


def test_graph_chunks_and_direct_launches_agree_bitwise():
    from ionosphere_fdtd_b200.engine import Tuning

    case = dict(C.CASES["config4_mini_s2"], steps=19)
    direct = run_product(case, "float64", tuning=Tuning(graph_chunk=0))
    graphed = run_product(case, "float64", tuning=Tuning(graph_chunk=8))
    for key in ("er", "et", "hr", "ht", "si_memory", "plasma_current_0", "traces"):
        np.testing.assert_array_equal(direct[key], graphed[key], err_msg=key)


@pytest.mark.parametrize("fpp", [4, 16, 64])
def test_patch_size_does_not_change_results(fpp):
    from ionosphere_fdtd_b200.engine import Tuning

    case = C.CASES["config4_mini_s2"]
    ref = run_product(case, "float64", tuning=Tuning(faces_per_patch=32))
    other = run_product(case, "float64", tuning=Tuning(faces_per_patch=fpp, threads=128))
    for f in STATE:
        np.testing.assert_array_equal(ref[f], other[f])


@pytest.mark.parametrize("staging", [2, 3])
@pytest.mark.parametrize("fpp", [(16, 8), (32, 16), (4, 4)])
@pytest.mark.parametrize(
    "name", ["config4_mini_s2", "plasma_magnetized_s1", "tangential_s1", "thin_shell_s1", "adaptive_s1", "adaptive_plasma_si_s1"]
)
def test_pipeline_and_direct_kernels_agree_bitwise(name, fpp, staging):
    """The pipeline (TMA bulk copies or cp.async) stages every row in shared
    memory and runs the same per-run arithmetic as the direct global gathers:
    results match bit for bit (adaptive meshes: vertex degree 7-8, the
    12-slot vertex tables)."""

    from ionosphere_fdtd_b200.engine import Tuning

    direct = run_product(C.CASES[name], "float32", tuning=Tuning(staging=1))
    staged = run_product(C.CASES[name], "float32", tuning=Tuning(staging=staging, faces_per_patch=fpp[0], e_faces_per_patch=fpp[1]))
    assert direct["_sim"]._engine.kernel_modes == ("direct", "direct")
    assert staged["_sim"]._engine.kernel_modes == ("pipeline", "pipeline")
    for key in ("er", "et", "hr", "ht", "si_memory", "plasma_current_0", "traces"):
        if key in direct:
            np.testing.assert_array_equal(direct[key], staged[key], err_msg=key)
    assert staged["_sim"]._engine.status_word() == 0


@pytest.mark.parametrize("dtype", ["float32", "float64"])
@pytest.mark.parametrize("name", ["config4_mini_s2", "plasma_magnetized_s1", "config1_s2", "adaptive_plasma_si_s1", "tangential_s1"])
def test_lane_layouts_agree_bitwise(name, dtype):
    """Rows packed across lanes and rows started on 8-lane boundaries run the
    same per-run arithmetic on the same quads: bit-for-bit equal results, with
    and without plasma, float32 (4 reals per quad) and float64 (2)."""

    from ionosphere_fdtd_b200.engine import Tuning

    packed = run_product(C.CASES[name], dtype, tuning=Tuning(staging=2, lane_layout=1))
    aligned = run_product(C.CASES[name], dtype, tuning=Tuning(staging=2, lane_layout=2))
    assert aligned["_sim"]._engine.kernel_modes == ("pipeline", "pipeline")
    for key in ("er", "et", "hr", "ht", "si_memory", "plasma_current_0", "plasma_current_1", "traces"):
        if key in packed:
            np.testing.assert_array_equal(packed[key], aligned[key], err_msg=key)
    assert aligned["_sim"]._engine.status_word() == 0


@pytest.mark.parametrize("tuning", [dict(e_threads=576), dict(e_threads=608, producer_warps=1, lane_layout=2),
                                    dict(e_stages=3), dict(e_stages=3, e_threads=544, producer_warps=3),
                                    dict(e_producer_warps=3), dict(e_producer_warps=4, producer_warps=1),
                                    dict(e_producer_warps=1, e_threads=576), dict(e_copy_gap=2, e_producer_warps=4),
                                    dict(e_copy_gap=8)])
@pytest.mark.parametrize("dtype", ["float32", "float64"])
@pytest.mark.parametrize("name", ["config4_mini_s2", "plasma_magnetized_s1", "adaptive_plasma_si_s1", "tangential_s1"])
def test_wide_e_ctas_and_deeper_e_rings_agree_bitwise(name, dtype, tuning):
    """E-phase CTAs of up to 20 warps at 96 registers, E patches sized for three
    ring stages, and E-phase producer warp counts other than the H phase's
    compute the same bits as the default plan."""

    from ionosphere_fdtd_b200.engine import Tuning

    ref = run_product(C.CASES[name], dtype, tuning=Tuning(staging=2))
    other = run_product(C.CASES[name], dtype, tuning=Tuning(staging=2, **tuning))
    assert other["_sim"]._engine.kernel_modes == ("pipeline", "pipeline")
    for key in ("er", "et", "hr", "ht", "si_memory", "plasma_current_0", "plasma_current_1", "traces"):
        if key in ref:
            np.testing.assert_array_equal(ref[key], other[key], err_msg=key)
    assert other["_sim"]._engine.status_word() == 0


@pytest.mark.parametrize("threads,producers,lanes", [(32, 1, 0), (128, 4, 0), (352, 1, 0), (256, 2, 0), (64, 3, 0),
                                                     (32, 1, 2), (96, 2, 2), (352, 1, 2)])
def test_pipeline_warp_counts_do_not_change_results(threads, producers, lanes):
    from ionosphere_fdtd_b200.engine import Tuning

    case = C.CASES["plasma_magnetized_s1"]
    ref = run_product(case, "float64", tuning=Tuning(staging=2))
    other = run_product(case, "float64", tuning=Tuning(staging=2, threads=threads, producer_warps=producers, lane_layout=lanes))
    for f in STATE:
        np.testing.assert_array_equal(ref[f], other[f])
