"""The reference's host-side surface-impedance tests (tests/test_surface_impedance.py
there) on the package's model and ADE, with NumPy arrays standing in for device
arrays, and the lower-boundary update against the oracle's."""

import numpy as np
import pytest

from ionosphere_fdtd_b200 import ConductiveHalfSpaceSurface, SurfaceImpedanceADE


class HostArrays:
    def asarray(self, values):
        return np.asarray(values, dtype=np.float64)

    def zeros(self, shape):
        return np.zeros(shape, dtype=np.float64)

    def nbytes(self, values):
        return values.nbytes


def test_diffusive_fit_matches_the_passive_half_space_and_scales_with_conductivity():
    model = ConductiveHalfSpaceSurface(1.0 / 50.0)
    f = np.geomspace(5.0, 45.0, 301)
    fitted, exact = model.impedance_ohm(f)[0], model.exact_impedance_ohm(f)[0]
    assert np.max(np.abs(fitted / exact - 1.0)) < 6.0e-3
    assert np.all(fitted.real > 0.0) and np.all(fitted.imag > 0.0)
    assert np.all(model.pole_rates_s_inv > 0.0) and np.all(model.diffusive_weights_sqrt_s_inv > 0.0)
    z = ConductiveHalfSpaceSurface(np.asarray((4.0, 1.0))).impedance_ohm(20.0)[:, 0]
    assert z[1] / z[0] == pytest.approx(2.0)


def test_ade_harmonic_response_is_causal_passive_and_accurate():
    model = ConductiveHalfSpaceSurface(1.0 / 50.0)
    dt, freq, n = 1.0e-4, 20.0, 50_000
    ade = SurfaceImpedanceADE(model, edge_count=1, time_step_s=dt, backend=HostArrays())
    electric, magnetic = np.empty(n), np.empty(n)
    for k in range(n):
        t = k * dt
        h_old = np.asarray((np.cos(2.0 * np.pi * freq * (t - 0.5 * dt)),))
        h_new = np.asarray((np.cos(2.0 * np.pi * freq * (t + 0.5 * dt)),))
        magnetic[k] = 0.5 * (h_old[0] + h_new[0])
        electric[k] = ade.advance_prescribed_magnetic(h_old, h_new)[0]
    tail = slice(n - 10_000, None)
    basis = np.exp(-2j * np.pi * freq * np.arange(n)[tail] * dt)
    measured = -np.sum(electric[tail] * basis) / np.sum(magnetic[tail] * basis)
    assert measured == pytest.approx(model.impedance_ohm(freq)[0, 0], rel=3.0e-4)
    assert np.mean(-electric[tail] * magnetic[tail]) > 0.0


def test_lower_boundary_update_equals_the_oracle():
    """advance_lower_boundary on host arrays against the oracle's boundary step
    (surface_impedance.py:225-270), rows subset included."""

    import oracle.fdtd as O

    rng = np.random.default_rng(3)
    n = 30  # edges of the level-0 mesh
    sigma = 10.0 ** rng.uniform(-3, -1, n)
    model = ConductiveHalfSpaceSurface(sigma)
    ora = O.OracleFDTD(subdivision=0, radial_cells=3, minimum_altitude_m=0.0, maximum_altitude_m=90_000.0,
                       courant_factor=0.3, surface=O.OracleSurface(sigma), dtype=np.float64)
    ade = SurfaceImpedanceADE(model, edge_count=n, time_step_s=ora.dt, backend=HostArrays())
    memory = rng.standard_normal(ade.memory.shape)
    ade.memory[:] = memory
    ora.si_memory[:] = memory
    h_old, e1, g0 = (rng.standard_normal(n) for _ in range(3))
    got = ade.advance_lower_boundary(h_old, e1, g0, ora.dr[0], ora.dt)
    want = ora._surface_advance(h_old, e1, g0)
    np.testing.assert_allclose(got, want, rtol=1e-13, atol=0)
    np.testing.assert_allclose(ade.memory, ora.si_memory, rtol=1e-13, atol=1e-300)
    rows = np.asarray((3, 17, 26))
    before = ade.memory.copy()
    ade.advance_lower_boundary(h_old[rows], e1[rows], g0[rows], ora.dr[0], ora.dt, rows=rows)
    untouched = np.setdiff1d(np.arange(n), rows)
    np.testing.assert_array_equal(ade.memory[untouched], before[untouched])
    assert not np.array_equal(ade.memory[rows], before[rows])
