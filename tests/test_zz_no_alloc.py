"""The allocation-free step, ``ifdtd_step_static_scratch``.

Some callers of this library may not allocate device memory while they run:
code that sits between the reservations of a custom memory pool, host
callbacks, or processes whose device memory budget is fixed after start-up.
For them the C ABI offers a step that keeps its scratch (the summed current of
a plasma with more than one species) in a static device array of 16 MiB
instead of plan memory.  These tests call it through the C ABI and compare it
with ``ifdtd_step`` on two calls in a row, within the float32 tolerance of the
parity tests (per (E, H) group relative L2 < 2e-5), and check that a mesh whose
summed current does not fit is refused with a clear error.  The file is named
so that pytest collects it last.
"""

import ctypes as C

import numpy as np
import pytest

import cases as CS
from casebuild import build_product, grouped_rel_l2, rel_l2

pytestmark = pytest.mark.gpu

STEPS = 5
LIMIT = 2.0e-5


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
    status = getattr(N.load(), entry)(eng.plan, C.byref(state), currents.data_ptr(), int(currents.numel()), eng.backend.stream_handle())
    N.check(status, entry)


@pytest.mark.parametrize("name", ["plasma_magnetized_s1", "config4_mini_s2"])
def test_static_scratch_step_matches_ifdtd_step_on_two_calls(name):
    import torch

    case = CS.CASES[name]
    ref = build_product(case, "float32")
    alt = build_product(case, "float32")
    currents = torch.linspace(-1.0, 1.0, STEPS, dtype=torch.float64, device=ref.backend.torch_device)
    for call in range(2):
        _call("ifdtd_step", ref, currents)
        _call("ifdtd_step_static_scratch", alt, currents)
        expected, actual = _state_arrays(ref), _state_arrays(alt)
        errs = grouped_rel_l2(actual, expected)
        assert max(errs.values()) < LIMIT, (call, errs)
        for key in expected:
            if key.startswith("plasma_current") or key == "si_memory":
                assert rel_l2(actual[key], expected[key]) < LIMIT, (call, key)
    assert alt._engine.status_word() == 0


def test_static_scratch_step_refuses_a_summed_current_above_its_limit():
    import torch

    from ionosphere_fdtd_b200.errors import BackendUnavailableError

    base = CS.CASES["plasma_magnetized_s1"]
    # s5, 40 cells, float64, two species: 20,480 x 3 x 40 x 8 B = 19.7 MB > 16 MiB
    case = dict(base, config=dict(base["config"], subdivision=5, radial_cells=40))
    sim = build_product(case, "float64")
    currents = torch.zeros(1, dtype=torch.float64, device=sim.backend.torch_device)
    before = sim.to_numpy(sim.er).copy()
    with pytest.raises(BackendUnavailableError, match="static scratch"):
        _call("ifdtd_step_static_scratch", sim, currents)
    np.testing.assert_array_equal(sim.to_numpy(sim.er), before)
