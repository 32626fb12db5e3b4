"""The plasma current in face frames (``Tuning.plasma_frame``).

With an unmagnetised plasma the step kernels hold each face's current in a
frame of its own while they run: component 0 along the face centre, 1 and 2 in
the face's tangent plane.  The Drude update treats every component alike, so
it is the same update in that frame; the E phase then reads one current row
per face for a vertex's radial current and two per face for an edge's
tangential current, instead of three.  Every call turns the caller's Cartesian
currents into face frames first and back at the end, so the state between
calls is the reference's (plasma.py:413-442, 489-527).

These tests check, on the reference's own fixtures and on the oracle, that
both frames give the reference's results within the parity bounds (float64
< 1e-11, float32 <= 1e-5 relative L2 per (E, H) group), that the two frames
agree with each other to float64 round-off across several calls (so nothing
stays rotated between calls), that the automatic choice is the face frame for
an unmagnetised plasma, that the pipelined and direct kernels agree bit for
bit in either frame, and that a magnetised plasma refuses face frames.
"""

import numpy as np
import pytest

import cases as C
from casebuild import build_product, golden, grouped_rel_l2, rel_l2, run_oracle, run_product

pytestmark = pytest.mark.gpu

DRUDE = ["plasma_drude_s2", "config4_mini_s2"]

# two unmagnetised species with a vertical source: the summed current runs in face frames too
TWO_SPECIES_DRUDE = dict(
    C.CASES["plasma_magnetized_s1"],
    plasma=dict(kind="uniform", magnetic_t=0.0, density_m3=1.0e6, collision_hz=1.0e4, two_species=True),
    source=dict(kind="vertical", peak_current_a=1.0e6, seed_vertex=5),
)

STATE = ("er", "et", "hr", "ht")


def _tuning(**kw):
    from ionosphere_fdtd_b200.engine import Tuning

    return Tuning(**kw)


@pytest.mark.parametrize("frame", [1, 2])
@pytest.mark.parametrize("name", DRUDE)
def test_either_frame_matches_the_reference(name, frame):
    ref = golden(f"case_{name}")
    out64 = run_product(C.CASES[name], "float64", tuning=_tuning(plasma_frame=frame))
    errs = grouped_rel_l2(out64, ref)
    assert max(errs.values()) < 1e-11, errs
    assert rel_l2(out64["plasma_current_0"], ref["plasma_current_0"]) < 1e-11
    out32 = run_product(C.CASES[name], "float32", tuning=_tuning(plasma_frame=frame))
    errs = grouped_rel_l2(out32, ref)
    assert max(errs.values()) <= 1e-5, errs
    assert rel_l2(out32["plasma_current_0"], ref["plasma_current_0"]) <= 1e-4
    if "traces" in ref:
        assert rel_l2(out32["traces"], ref["traces"]) <= 1e-5


def test_automatic_frame_is_the_face_frame_for_an_unmagnetised_plasma():
    case = C.CASES["config4_mini_s2"]
    auto = run_product(case, "float32")
    local = run_product(case, "float32", tuning=_tuning(plasma_frame=2))
    cart = run_product(case, "float32", tuning=_tuning(plasma_frame=1))
    for key in STATE + ("plasma_current_0", "si_memory", "traces"):
        np.testing.assert_array_equal(auto[key], local[key], err_msg=key)
    # the frames round differently: the face-frame run really ran
    assert not np.array_equal(local["plasma_current_0"], cart["plasma_current_0"])


def test_frames_agree_across_calls_and_two_species_match_the_oracle():
    case = TWO_SPECIES_DRUDE
    expected = run_oracle(case, np.float64)
    out = {}
    for frame in (1, 2):
        sim = build_product(case, "float64", tuning=_tuning(plasma_frame=frame))
        # several calls of uneven length: each converts on entry and back on exit
        for n in (1, 2, case["steps"] - 3):
            sim.step(n)
        out[frame] = {f: sim.to_numpy(getattr(sim, f)) for f in STATE}
        for i, j in enumerate(sim._plasma_coupler.ade.current_density):
            out[frame][f"plasma_current_{i}"] = sim.to_numpy(j)
    for key in out[1]:
        assert rel_l2(out[2][key], out[1][key]) < 1e-13, key
    errs = grouped_rel_l2(out[2], expected)
    assert max(errs.values()) < 1e-11, errs
    for key in ("plasma_current_0", "plasma_current_1"):
        assert rel_l2(out[2][key], expected[key]) < 1e-11, key


@pytest.mark.parametrize("frame", [1, 2])
@pytest.mark.parametrize("name", ["config4_mini_s2", "two_species_drude"])
def test_pipeline_and_direct_kernels_agree_bitwise_in_either_frame(name, frame):
    case = TWO_SPECIES_DRUDE if name == "two_species_drude" else C.CASES[name]
    direct = run_product(case, "float32", tuning=_tuning(staging=1, plasma_frame=frame))
    staged = run_product(case, "float32", tuning=_tuning(staging=2, faces_per_patch=16, e_faces_per_patch=8,
                                                         plasma_frame=frame))
    assert direct["_sim"]._engine.kernel_modes == ("direct", "direct")
    assert staged["_sim"]._engine.kernel_modes == ("pipeline", "pipeline")
    for key in STATE + ("si_memory", "plasma_current_0", "plasma_current_1", "traces"):
        if key in direct:
            np.testing.assert_array_equal(direct[key], staged[key], err_msg=key)
    assert staged["_sim"]._engine.status_word() == 0


def test_face_frames_need_an_unmagnetised_plasma():
    from ionosphere_fdtd_b200 import BackendUnavailableError

    with pytest.raises(BackendUnavailableError, match="unmagnetised"):
        build_product(C.CASES["plasma_magnetized_s1"], "float32", tuning=_tuning(plasma_frame=2))
    # the automatic choice keeps the magnetised plasma Cartesian
    ref = golden("case_plasma_magnetized_s1")
    out = run_product(C.CASES["plasma_magnetized_s1"], "float64")
    assert max(grouped_rel_l2(out, ref).values()) < 1e-11
