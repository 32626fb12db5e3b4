"""Host logic of ``record_receiver_traces`` (visualization.py:212-252) on the CPU:
receiver placement, sample rows, clock and labels, driven through the NumPy
oracle in place of the engine and pinned to the reference's own fixture."""

import numpy as np
import pytest

import cases as C
from casebuild import build_oracle, golden

from ionosphere_fdtd_b200 import receivers as R
from ionosphere_fdtd_b200.solver import GeodesicFDTD


class OracleSim:
    """The part of ``GeodesicFDTD`` that the receiver helper calls, over the oracle."""

    _validated_count = staticmethod(GeodesicFDTD._validated_count)

    def __init__(self, oracle):
        self.oracle = oracle
        self.mesh = oracle.mesh
        self.altitudes_m = oracle.altitudes_m
        self.time_step_s = oracle.dt
        self.calls = []

    @property
    def steps(self):
        return self.oracle.steps

    @property
    def time_s(self):
        return self.oracle.time_s

    def record_er_observations(self, vertex_indices, radial_layers, weights, steps):
        self.calls.append(steps)
        return self.oracle.record_er(vertex_indices, radial_layers, weights, steps)


def _receivers():
    return [R.Receiver(lat, lon, alt, label) for lat, lon, alt, label in C.RECEIVER_TRACES["receivers"]]


def test_receiver_traces_match_the_reference_helper():
    spec = C.RECEIVER_TRACES
    ref = golden(f"receiver_traces_{spec['case']}")
    sim = OracleSim(build_oracle(C.CASES[spec["case"]]))
    out = R.record_receiver_traces(sim, _receivers(), spec["steps"], sample_every=spec["sample_every"])
    assert out.labels == tuple(str(x) for x in ref["labels"])
    np.testing.assert_allclose(out.time_s, ref["time_s"], rtol=1e-14, atol=0)
    scale = float(np.max(np.abs(ref["er_v_m"])))
    np.testing.assert_allclose(out.er_v_m, ref["er_v_m"], rtol=1e-9, atol=1e-10 * scale)
    assert sim.steps == int(ref["steps_after"])
    assert sim.time_s == pytest.approx(float(ref["time_after"]), rel=1e-14)


@pytest.mark.parametrize("steps, every, block", [(11, 4, 3), (11, 4, 8), (12, 4, 4), (0, 3, 4096), (7, 1, 2), (5, 9, 4096)])
def test_sample_rows_do_not_depend_on_the_recording_blocks(monkeypatch, steps, every, block):
    case = C.CASES[C.RECEIVER_TRACES["case"]]
    whole = R.record_receiver_traces(OracleSim(build_oracle(case)), _receivers(), steps, sample_every=every)
    monkeypatch.setattr(R, "_BLOCK_STEPS", block)
    sim = OracleSim(build_oracle(case))
    split = R.record_receiver_traces(sim, _receivers(), steps, sample_every=every)
    expected_rows = sorted(set(range(0, steps + 1, every)) | {steps})
    assert len(split.time_s) == len(expected_rows)
    np.testing.assert_array_equal(split.er_v_m, whole.er_v_m)
    np.testing.assert_array_equal(split.time_s, whole.time_s)
    assert sum(sim.calls) == steps and sim.steps == steps


def test_receiver_arguments_are_checked_with_the_reference_messages():
    sim = OracleSim(build_oracle(C.CASES["source_s1"]))
    with pytest.raises(ValueError, match="at least one receiver"):
        R.record_receiver_traces(sim, [], 3)
    with pytest.raises(ValueError, match="steps must be non-negative"):
        R.record_receiver_traces(sim, _receivers(), -1)
    with pytest.raises(ValueError, match="sample_every must be positive"):
        R.record_receiver_traces(sim, _receivers(), 3, sample_every=0)
    assert sim.calls == []
