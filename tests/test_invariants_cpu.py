"""Discrete invariants of the reference's test strategy
(tests/test_maxwell_invariants.py:76-163 in the reference), on the CPU: the
adjoint pairs of the mesh's incidence operators, and the exact leapfrog
dispersion of surface TM-r and TE-r eigenmodes run through the oracle's half
steps.  ``tests/test_solver_gpu.py`` runs the same eigenmodes through the
engine."""

import numpy as np
import pytest

import ionosphere_fdtd_b200 as P
import oracle.fdtd as O
from invariants import SURFACE_MODE, Vacuum, expected_amplitudes, surface_mode, tangential_case, tangential_moment_error


def test_incidence_operators_are_adjoint_pairs():
    mesh = P.build_geodesic_mesh(2)
    rng = np.random.default_rng(20260805)
    e = rng.standard_normal(mesh.n_edges)
    f = rng.standard_normal(mesh.n_faces)
    v = rng.standard_normal(mesh.n_vertices)
    assert f @ mesh.face_circulation(e) == pytest.approx(mesh.dual_edge_difference(f) @ e, abs=2.0e-13)
    assert v @ mesh.dual_cell_circulation(e) == pytest.approx(-mesh.edge_difference(v) @ e, abs=2.0e-13)


def _oracle():
    return O.OracleFDTD(material=Vacuum(), dtype=np.float64, **SURFACE_MODE)


def test_oracle_tm_surface_mode_follows_the_leapfrog_dispersion():
    sim = _oracle()
    eigen, mode = surface_mode(P.build_geodesic_mesh(1), "tm")
    sim.er[:, 1] = mode
    amplitudes = [1.0]
    for _ in range(100):
        sim.update_magnetic()
        sim.update_electric(0.0)
        sim.et[:] = 0.0
        sim.hr[:] = 0.0
        amplitudes.append(float(sim.er[:, 1] @ mode / (mode @ mode)))
    expected = expected_amplitudes(eigen, sim.dt, sim.radii_m[1], 100, 0.5)
    np.testing.assert_allclose(amplitudes, expected, rtol=0.0, atol=8.0e-14)
    assert not np.any(sim.hr)


def test_oracle_te_surface_mode_follows_the_leapfrog_dispersion():
    sim = _oracle()
    eigen, mode = surface_mode(P.build_geodesic_mesh(1), "te")
    sim.hr[:, 1] = mode
    amplitudes = [1.0]
    for _ in range(100):
        sim.update_magnetic()
        sim.ht[:] = 0.0
        sim.update_electric(0.0)
        sim.er[:] = 0.0
        amplitudes.append(float(sim.hr[:, 1] @ mode / (mode @ mode)))
    expected = expected_amplitudes(eigen, sim.dt, sim.midpoints_m[1], 100, -0.5)
    np.testing.assert_allclose(amplitudes, expected, rtol=0.0, atol=8.0e-14)
    assert not np.any(sim.er)


def test_surface_laplacian_spectrum_is_rotation_invariant():
    from invariants import tm_operator

    spectra = []
    for orientation in ("native", "polar"):
        mesh = P.build_geodesic_mesh(1, orientation=orientation)
        matrix = np.column_stack([tm_operator(mesh, e) for e in np.eye(mesh.n_vertices)])
        spectra.append(np.sort(np.linalg.eigvals(matrix).real))
    np.testing.assert_allclose(spectra[0], spectra[1], rtol=0.0, atol=2.0e-13)


@pytest.mark.parametrize("orientation", ("native", "polar"))
def test_oracle_time_step_keeps_surface_spectra_inside_the_cfl_limit(orientation):
    from invariants import courant_numbers

    ora = O.OracleFDTD(material=Vacuum(), dtype=np.float64, orientation=orientation,
                       **dict(SURFACE_MODE, courant_factor=1.0))
    mesh = P.build_geodesic_mesh(1, orientation=orientation)  # the oracle's mesh, bit for bit
    np.testing.assert_array_equal(mesh.vertices, ora.mesh.vertices)
    tm_q, te_q = courant_numbers(mesh, ora.dt, ora.radii_m.min(), ora.midpoints_m.min())
    assert 0.0 < tm_q < 4.0 and 0.0 < te_q < 4.0


@pytest.mark.parametrize("orientation", ("polar", "native"))
@pytest.mark.parametrize("subdivision", (1, 3))
def test_tangential_source_samples_reconstruct_the_requested_moment(subdivision, orientation):
    """On the package's mesh and source code, with the radial midpoints of a
    -5 km .. 5 km two-cell grid (the GPU tests repeat it on a simulation)."""

    from types import SimpleNamespace

    source, line = tangential_case()
    config = P.SimulationConfig(subdivision=subdivision, radial_cells=2, minimum_altitude_m=-5_000.0,
                                maximum_altitude_m=5_000.0, mesh_orientation=orientation)
    radii = config.earth_radius_m + np.linspace(-5_000.0, 5_000.0, 3)
    host = SimpleNamespace(mesh=P.build_geodesic_mesh(subdivision, orientation=orientation), config=config,
                           radial_midpoint_altitudes_m=0.5 * (radii[:-1] + radii[1:]) - config.earth_radius_m)
    assert tangential_moment_error(host, source, line) < 2.0e-11


def _graded_oracle(geometry_mode):
    from invariants import GRADED_ALTITUDES

    a = GRADED_ALTITUDES
    return O.OracleFDTD(subdivision=0, radial_cells=len(a) - 1, minimum_altitude_m=a[0], maximum_altitude_m=a[-1],
                        radial_altitudes_m=a, geometry_mode=geometry_mode, material=Vacuum(), dtype=np.float64)


def test_oracle_radial_stencils_are_weighted_adjoints():
    """tests/test_maxwell_invariants.py:344-430 of the reference on the oracle's radial
    stencils (the engine's fused rows are pinned to them by the parity tests)."""

    rng = np.random.default_rng(20260805)
    thin = _graded_oracle("thin-shell")
    thin.et[:] = rng.standard_normal(thin.et.shape)
    thin.ht[:] = rng.standard_normal(thin.ht.shape)
    left = np.sum(thin.ht * thin._d_et() * thin.control_m[None, :])
    right = np.sum(thin.et * thin._d_ht() * thin.steps_m[None, :])
    assert left + right == pytest.approx(0.0, abs=2.0e-11)
    thin.ht[:] = 1.0
    np.testing.assert_array_equal(thin._d_ht(), 0.0)

    full = _graded_oracle("full-spherical")
    full.et[:] = rng.standard_normal(full.et.shape)
    full.ht[:] = rng.standard_normal(full.ht.shape)
    left = np.sum(full.ht * full._d_et() * (full.control_m * full.radii_m**2)[None, :])
    right = np.sum(full.et * full._d_ht() * (full.steps_m * full.midpoints_m**2)[None, :])
    assert abs(left + right) <= 2.0e-15 * max(abs(left), abs(right))


def test_oracle_full_spherical_metric_annihilates_inverse_radius_profiles():
    base = dict(subdivision=0, radial_cells=8, minimum_altitude_m=-100_000.0, maximum_altitude_m=100_000.0,
                material=Vacuum(), dtype=np.float64)
    full = O.OracleFDTD(geometry_mode="full-spherical", **base)
    full.et[:] = 1.0 / full.midpoints_m[None, :]
    full.ht[:] = 1.0 / full.radii_m[None, :]
    np.testing.assert_allclose(full._d_et()[:, 1:-1], 0.0, atol=1.0e-27)
    np.testing.assert_allclose(full._d_ht(), 0.0, atol=1.0e-27)
    thin = O.OracleFDTD(geometry_mode="thin-shell", **base)
    thin.et[:] = 1.0 / thin.midpoints_m[None, :]
    assert np.max(np.abs(thin._d_et()[:, 1:-1])) > 2.0e-14
