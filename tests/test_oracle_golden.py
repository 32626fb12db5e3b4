"""Pin the CPU oracle to the reference's own outputs (golden fixtures)."""

import json

import numpy as np
import pytest

import cases as C
from casebuild import GOLDEN, golden, grouped_rel_l2, run_oracle

import oracle.fdtd as O

STATE = ("er", "et", "hr", "ht")


def group_scale(ref, key):
    """Absolute scale for a compared array: the largest magnitude in its
    (E or H) field group, so pure round-off fields such as Hr under a
    vertical source are compared against the physical scale."""

    groups = {"er": ("er", "et"), "et": ("er", "et"), "hr": ("hr", "ht"), "ht": ("hr", "ht")}
    names = groups.get(key, (key,))
    return max(float(np.max(np.abs(ref[n]))) for n in names if n in ref) or 1.0


@pytest.mark.parametrize("level", [0, 1, 2, 3])
def test_oracle_mesh_tables_match_reference_bitwise(level):
    ref = golden(f"mesh_s{level}")
    mesh = O.build_mesh(level)
    for name in ("edges", "faces", "face_edges", "face_edge_signs", "edge_left_faces", "edge_right_faces", "vertex_degree"):
        np.testing.assert_array_equal(getattr(mesh, name), ref[name], err_msg=name)
    table, signs = O.vertex_incidence(mesh)
    np.testing.assert_array_equal(table, ref["vertex_edges"])
    np.testing.assert_array_equal(signs, ref["vertex_edge_signs"])
    for name in ("vertices", "face_centers", "primal_edge_angles", "dual_edge_angles", "face_solid_angles", "dual_cell_solid_angles"):
        np.testing.assert_array_equal(getattr(mesh, name), ref[name], err_msg=name)


def test_oracle_mesh_digests_match_reference_to_level_5():
    digests = json.loads((GOLDEN / "mesh_digests.json").read_text())
    import hashlib

    for level in (4, 5):
        mesh = O.build_mesh(level)
        for name in ("edges", "faces", "face_edges", "edge_left_faces", "edge_right_faces"):
            got = hashlib.sha256(np.ascontiguousarray(getattr(mesh, name), dtype=np.int64).tobytes()).hexdigest()
            assert got == digests[str(level)][name], (level, name)


@pytest.mark.parametrize("name", sorted(C.CASES))
def test_oracle_float64_matches_reference(name):
    case = C.CASES[name]
    ref = golden(f"case_{name}")
    out = run_oracle(case)
    assert float(out["time_step_s"]) == pytest.approx(float(ref["time_step_s"]), rel=1e-15)
    for key in ref:
        if key in ("time_step_s", "cfl_limit_s", "max_abs"):
            continue
        np.testing.assert_allclose(out[key], ref[key], rtol=1e-11, atol=1e-12 * group_scale(ref, key), err_msg=key)


def test_oracle_float32_tracks_reference_float32_pin():
    """The reference's FP32 pin: 80 steps of the default source case."""

    case = dict(C.CASES["source_s1"], steps=80)
    ref64 = golden("case_source_s1_f64x80")
    ref32 = golden("case_source_s1_f32x80")
    out32 = run_oracle(case, dtype=np.float32)
    errs = grouped_rel_l2(out32, ref64)
    assert max(errs.values()) < 2.0e-5, errs
    errs_ref = grouped_rel_l2(ref32, ref64)
    assert max(errs_ref.values()) < 2.0e-5, errs_ref


def test_oracle_h_observations_match_reference():
    ref = golden("obs_h_source_s1")
    from casebuild import build_oracle

    sim = build_oracle(C.CASES["source_s1"])
    hr, ht = sim.record_h(
        np.asarray(((0,), (5,))),
        np.asarray(((2,), (4,))),
        np.asarray(((1.0,), (1.0,))),
        np.asarray(((0, 1, 2), (7, 8, 9))),
        np.asarray(((2, 2, 2), (0, 3, 6))),
        np.asarray(((0.2, -0.3, 0.5), (1.0, 0.5, -0.5))),
        11,
        sample_every=3,
    )
    np.testing.assert_allclose(hr, ref["hr"], rtol=1e-11, atol=1e-30)
    np.testing.assert_allclose(ht, ref["ht"], rtol=1e-11, atol=1e-30)


@pytest.mark.parametrize("name", sorted(C.CASES))
def test_threaded_oracle_float64_matches_reference(name):
    """The all-threads CPU baseline (PyTorch CPU tensors, ``oracle.threaded``)
    advances every golden case to the reference's own state."""

    import torch

    from casebuild import build_oracle
    from oracle.threaded import ThreadedOracleStep

    case = C.CASES[name]
    ref = golden(f"case_{name}")
    sim = build_oracle(case)
    threads = torch.get_num_threads()
    try:
        ThreadedOracleStep(sim, 2).step(case["steps"])
    finally:
        torch.set_num_threads(threads)
    assert sim.steps == case["steps"]
    out = {f: getattr(sim, f) for f in STATE}
    if sim.surface is not None:
        out["si_memory"] = sim.si_memory
    if sim.plasma is not None:
        out.update({f"plasma_current_{i}": j for i, j in enumerate(sim.p_current)})
    for key, value in out.items():
        np.testing.assert_allclose(value, ref[key], rtol=1e-11, atol=1e-12 * group_scale(ref, key), err_msg=key)
