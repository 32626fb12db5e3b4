"""The allocation-free step, ``ifdtd_step_static_scratch``.

Some callers of this library may not allocate device memory while they run: a
process that gives all free device memory to its own pool at start-up (so
``cudaMalloc`` would fail), or a latency-bound loop that cannot afford the
device-wide synchronisation ``cudaMalloc`` and ``cudaFree`` may perform.  For
them the C ABI offers a step that keeps its scratch (the summed current of a
plasma with more than one species) in a static device array of 16 MiB instead
of plan memory.  It launches the same kernels on the same inputs as
``ifdtd_step``, so these tests call both through the C ABI on two calls in a
row and require every state array (fields, plasma currents, surface-impedance
memory) to be bitwise equal after each call.  They cover a source current
vector and a null one (the static zero current), and one and two plasma
species.  A mesh whose summed current does not fit is refused with a clear
error.  The file is named so that pytest collects it last.
"""

import ctypes as C

import numpy as np
import pytest

import cases as CS
from casebuild import build_product

pytestmark = pytest.mark.gpu

STEPS = 5

# two plasma species (summed current in the static scratch) with a vertical
# source driven by the per-step current vector
TWO_SPECIES_SOURCE = dict(
    CS.CASES["plasma_magnetized_s1"],
    source=dict(kind="vertical", peak_current_a=1.0e6, seed_vertex=5),
)


def _case(name: str) -> dict:
    return TWO_SPECIES_SOURCE if name == "two_species_source_s1" else CS.CASES[name]


def _state_arrays(sim) -> dict[str, np.ndarray]:
    out = {f: sim.to_numpy(getattr(sim, f)) for f in ("er", "et", "hr", "ht")}
    if sim._plasma_coupler is not None:
        for i, j in enumerate(sim._plasma_coupler.ade.current_density):
            out[f"plasma_current_{i}"] = sim.to_numpy(j)
    if sim._surface_impedance_ade is not None:
        out["si_memory"] = sim.to_numpy(sim._surface_impedance_ade.memory)
    return out


def _call(entry: str, sim, currents) -> None:
    from ionosphere_fdtd_b200 import _native as N

    eng = sim._engine
    state = sim._state()
    ptr = 0 if currents is None else currents.data_ptr()
    status = getattr(N.load(), entry)(eng.plan, C.byref(state), ptr, STEPS, eng.backend.stream_handle())
    N.check(status, entry)


@pytest.mark.parametrize("source_currents", ["vector", "null"])
@pytest.mark.parametrize("name", ["plasma_magnetized_s1", "two_species_source_s1", "config4_mini_s2"])
def test_static_scratch_step_equals_ifdtd_step_bitwise_on_two_calls(name, source_currents):
    import torch

    case = _case(name)
    ref = build_product(case, "float32")
    alt = build_product(case, "float32")
    currents = None
    if source_currents == "vector":
        currents = torch.linspace(-1.0, 1.0, STEPS, dtype=torch.float64, device=ref.backend.torch_device)
    for call in range(2):
        _call("ifdtd_step", ref, currents)
        _call("ifdtd_step_static_scratch", alt, currents)
        expected, actual = _state_arrays(ref), _state_arrays(alt)
        assert expected.keys() == actual.keys()
        for key in expected:
            np.testing.assert_array_equal(actual[key], expected[key], err_msg=f"call {call}: {key}")
        if source_currents == "vector" and "source" in case:
            # the source drove the fields: the comparison is not of two idle runs
            assert np.abs(expected["er"]).max() > 0.0
    assert alt._engine.status_word() == 0


def test_static_scratch_step_refuses_a_summed_current_above_its_limit():
    import torch

    from ionosphere_fdtd_b200.errors import BackendUnavailableError

    base = CS.CASES["plasma_magnetized_s1"]
    # s5, 40 cells, float64, two species: 20,480 x 3 x 40 x 8 B = 19.7 MB > 16 MiB
    case = dict(base, config=dict(base["config"], subdivision=5, radial_cells=40))
    sim = build_product(case, "float64")
    currents = torch.zeros(STEPS, dtype=torch.float64, device=sim.backend.torch_device)
    before = sim.to_numpy(sim.er).copy()
    with pytest.raises(BackendUnavailableError, match="static scratch"):
        _call("ifdtd_step_static_scratch", sim, currents)
    np.testing.assert_array_equal(sim.to_numpy(sim.er), before)
