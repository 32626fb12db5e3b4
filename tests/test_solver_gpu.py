"""Reference-style behaviour tests of the CUDA engine (mirrors of the reference's
tests/test_backends.py, test_solver.py, test_surface_impedance.py,
test_checkpoint.py on the public API)."""

import numpy as np
import pytest

import ionosphere_fdtd_b200 as P
from ionosphere_fdtd_b200 import GeodesicFDTD, SimulationConfig
from ionosphere_fdtd_b200.constants import MU_0

pytestmark = pytest.mark.gpu


def small_config(**changes):
    values = dict(subdivision=1, radial_cells=6, courant_factor=0.25)
    values.update(changes)
    return SimulationConfig(**values)


def sim(config=None, **kw):
    kw.setdefault("device", "cuda")
    kw.setdefault("dtype", "float64")
    return GeodesicFDTD(config or small_config(), **kw)


@pytest.mark.parametrize("trailing", [(), (7,), (3, 4)])
def test_primitives_match_mesh_operators(trailing):
    s = sim()
    mesh = s.mesh
    rng = np.random.default_rng(42)
    b = s.backend
    ev = rng.standard_normal((mesh.n_edges,) + trailing)
    vv = rng.standard_normal((mesh.n_vertices,) + trailing)
    fv = rng.standard_normal((mesh.n_faces,) + trailing)
    np.testing.assert_allclose(b.to_numpy(b.face_circulation(b.asarray(ev))), mesh.face_circulation(ev), rtol=1e-13, atol=1e-13)
    np.testing.assert_allclose(b.to_numpy(b.dual_cell_circulation(b.asarray(ev))), mesh.dual_cell_circulation(ev), rtol=1e-13, atol=1e-13)
    np.testing.assert_allclose(b.to_numpy(b.edge_difference(b.asarray(vv))), mesh.edge_difference(vv), rtol=0, atol=0)
    np.testing.assert_allclose(b.to_numpy(b.dual_edge_difference(b.asarray(fv))), mesh.dual_edge_difference(fv), rtol=0, atol=0)


def test_dual_cell_circulation_is_bitwise_repeatable():
    s = sim(SimulationConfig(subdivision=3, radial_cells=6, courant_factor=0.2))
    values = s.backend.asarray(np.random.default_rng(20260805).standard_normal((s.mesh.n_edges, 7)))
    first = s.backend.dual_cell_circulation(values)
    for _ in range(10):
        assert s.backend.torch.equal(first, s.backend.dual_cell_circulation(values))


def test_float32_face_circulation_keeps_precision_semantics():
    s = sim(dtype="float32")
    mesh = s.mesh
    values = np.zeros(mesh.n_edges, dtype=np.float32)
    values[mesh.face_edges[0]] = np.asarray((1.0e8, 1.0, -1.0e8), dtype=np.float32) * mesh.face_edge_signs[0]
    out = s.backend.to_numpy(s.backend.face_circulation(s.backend.asarray(values)))
    assert out.dtype == np.float32
    np.testing.assert_array_equal(out, mesh.face_circulation(values))


def test_zero_fields_are_stationary():
    s = sim()
    s.step(3)
    for f in ("er", "et", "hr", "ht"):
        assert not np.any(s.to_numpy(getattr(s, f)))


def test_loss_coefficient_damps_uncoupled_radial_field():
    s = sim(material=P.EarthIonosphereMaterial(lithosphere_conductivity_s_m=1.0e-2))
    s.er[:, 0] = 1.0
    expected = s.to_numpy(s._ca_er)[:, 0].copy()
    s.step()
    assert np.allclose(s.to_numpy(s.er)[:, 0], expected)


def test_radial_pec_ghosts_give_the_one_sided_curl():
    s = sim(small_config(geometry_mode="thin-shell"))
    profile = np.arange(1, s.et.shape[1] + 1, dtype=np.float64)
    s.et[0] = s.backend.asarray(profile)
    expected = np.empty(s.ht.shape[1])
    expected[0] = 2.0 * profile[0] / s.radial_steps_m[0]
    expected[-1] = -2.0 * profile[-1] / s.radial_steps_m[-1]
    expected[1:-1] = np.diff(profile) / np.diff(s.radial_midpoints_m)
    s._update_magnetic_fields()
    np.testing.assert_allclose(s.to_numpy(s.ht)[0], -s.time_step_s / MU_0 * expected, rtol=1e-14, atol=0.0)


def test_high_conductivity_surface_converges_to_lower_pec_curl():
    base = dict(subdivision=0, radial_cells=4, minimum_altitude_m=0.0, maximum_altitude_m=100_000.0, courant_factor=0.2)
    pec = sim(SimulationConfig(**base))
    imp = sim(SimulationConfig(radial_boundary_condition="surface-impedance", **base), surface_impedance=P.ConductiveHalfSpaceSurface(1.0e30))
    rng = np.random.default_rng(20260820)
    er = rng.standard_normal(tuple(pec.er.shape))
    et = rng.standard_normal(tuple(pec.et.shape))
    ht = rng.standard_normal(tuple(pec.ht.shape))
    for s in (pec, imp):
        s.er.copy_(s.backend.asarray(er))
        s.et.copy_(s.backend.asarray(et))
        s.ht.copy_(s.backend.asarray(ht))
        s._update_magnetic_fields()
    np.testing.assert_allclose(imp.to_numpy(imp.ht), pec.to_numpy(pec.ht), rtol=2e-13, atol=2e-14)


def test_plasma_current_changes_et_and_limits_time_step():
    from casebuild import product_provenance

    mesh = P.build_geodesic_mesh(0)
    shape = (mesh.n_faces, 2)
    magnetic = np.zeros((*shape, 3))
    magnetic[..., 2] = 50e-6
    species = P.ColdPlasmaSpecies("electron", -P.ELEMENTARY_CHARGE_C, P.ELECTRON_MASS_KG, np.full(shape, 1e8), np.full(shape, 200.0))
    model = P.MeshPlasmaModel.from_mesh(mesh, np.asarray((25_000.0, 75_000.0)), magnetic, (species,), provenance=(product_provenance(),), interpolation="synthetic")
    cfg = SimulationConfig(subdivision=0, radial_cells=2, minimum_altitude_m=0.0, maximum_altitude_m=100_000.0, courant_factor=0.2)
    plasma = sim(cfg, mesh=mesh, plasma=model)
    vacuum = sim(cfg, mesh=mesh)
    values = np.random.default_rng(20260820).standard_normal(tuple(plasma.et.shape)) * 1e-6
    plasma.et.copy_(plasma.backend.asarray(values))
    vacuum.et.copy_(vacuum.backend.asarray(values))
    plasma._update_electric_fields()
    vacuum._update_electric_fields()
    assert np.max(np.abs(plasma.to_numpy(plasma.et) - vacuum.to_numpy(vacuum.et))) > 0.0
    assert plasma.cfl_time_step_limit_s < vacuum.cfl_time_step_limit_s
    assert plasma.diagnostics()["plasma_species"] == 1


def test_observation_recording_includes_initial_state():
    s = sim(source=P.GaussianCurrent(peak_current_a=1.0e6))
    traces = s.record_er_observations(np.asarray(((0, 1, 2),)), np.asarray((3,)), np.asarray(((0.2, 0.3, 0.5),)), 5, synchronize_every=2)
    assert traces.shape == (6, 1)
    assert traces[0, 0] == 0.0
    assert s.steps == 5
    assert np.isfinite(traces).all()


def test_observation_validation_matches_reference_messages():
    s = sim()
    with pytest.raises(ValueError, match="sum to one"):
        s.record_er_observations(np.asarray(((0, 1),)), np.asarray((0,)), np.asarray(((0.2, 0.3),)), 1)
    with pytest.raises(ValueError, match="finite"):
        s.record_er_observations(np.asarray(((0,),)), np.asarray((0,)), np.asarray(((np.nan,),)), 1)
    with pytest.raises(ValueError, match="integer"):
        s.step(1.5)


def test_leapfrog_clocks_and_diagnostics():
    s = sim()
    assert s.magnetic_time_s == pytest.approx(-0.5 * s.time_step_s)
    s.er.copy_(s.backend.asarray(np.random.default_rng(1).standard_normal(tuple(s.er.shape))))
    s.step(3)
    d = s.diagnostics()
    assert d["electric_time_s"] == pytest.approx(3 * s.time_step_s)
    assert d["magnetic_time_s"] == pytest.approx(2.5 * s.time_step_s)
    for f, key in (("er", "max_abs_er_v_m"), ("et", "max_abs_et_v_m"), ("hr", "max_abs_hr_a_m"), ("ht", "max_abs_ht_a_m")):
        assert d[key] == float(np.max(np.abs(s.to_numpy(getattr(s, f)))))
    assert d["backend"] == "torch" and d["device"].startswith("cuda")


def test_diagnostics_report_nonfinite_fields():
    s = sim(dtype="float32")
    s.hr[3, 2] = float("nan")
    assert np.isnan(s.diagnostics()["max_abs_hr_a_m"])


def test_checkpoint_round_trip_and_continuation(tmp_path):
    material = P.EarthIonosphereMaterial(anomalies=(P.SphericalAnomaly(35.0, 126.0, 500_000.0, -20_000.0, -1_000.0, 0.5),))
    source = P.GaussianCurrent(peak_current_a=2.0e6, center_time_s=0.01, one_over_e_half_width_s=0.02, carrier_frequency_hz=5.0)
    whole = sim(material=material, source=source)
    part = sim(material=material, source=source)
    whole.step(12)
    part.step(5)
    resumed = GeodesicFDTD.load_checkpoint(part.save_checkpoint(tmp_path / "state.npz"), device="cuda")
    assert resumed.steps == 5
    resumed.step(7)
    for f in ("er", "et", "hr", "ht"):
        np.testing.assert_array_equal(resumed.to_numpy(getattr(resumed, f)), whole.to_numpy(getattr(whole, f)))


def test_reference_checkpoint_loads_and_continues():
    """A checkpoint written by the reference (NumPy, float64) restores on CUDA and
    continues to the reference's own continuation."""

    from casebuild import GOLDEN, golden

    resumed = GeodesicFDTD.load_checkpoint(GOLDEN / "reference_checkpoint_v4.npz", device="cuda", dtype="float64")
    cont = golden("reference_checkpoint_continuation")
    assert resumed.steps == int(cont["steps_before"])
    resumed.step(int(cont["steps_after"]))
    for f in ("er", "et", "hr", "ht", "si_memory"):
        got = resumed.to_numpy(resumed._surface_impedance_ade.memory) if f == "si_memory" else resumed.to_numpy(getattr(resumed, f))
        scale = max(np.max(np.abs(cont[g])) for g in (("er", "et") if f in ("er", "et") else ("hr", "ht")))
        np.testing.assert_allclose(got, cont[f], rtol=1e-9, atol=1e-11 * scale, err_msg=f)


def test_surface_impedance_solver_remains_bounded():
    cfg = SimulationConfig(subdivision=0, radial_cells=4, minimum_altitude_m=0.0, maximum_altitude_m=100_000.0, courant_factor=0.35, radial_boundary_condition="surface-impedance")
    s = sim(cfg, surface_impedance=P.ConductiveHalfSpaceSurface(1.0 / 50.0))
    rng = np.random.default_rng(20260820)
    for name in ("er", "et"):
        getattr(s, name).copy_(s.backend.asarray(377.0e-9 * rng.standard_normal(tuple(getattr(s, name).shape))))
    for name in ("hr", "ht"):
        getattr(s, name).copy_(s.backend.asarray(1.0e-9 * rng.standard_normal(tuple(getattr(s, name).shape))))
    e0 = max(float(s.er.abs().max()), float(s.et.abs().max()))
    h0 = max(float(s.hr.abs().max()), float(s.ht.abs().max()))
    s.step(500)
    e1 = max(float(s.er.abs().max()), float(s.et.abs().max()))
    h1 = max(float(s.hr.abs().max()), float(s.ht.abs().max()))
    assert np.isfinite(e1) and np.isfinite(h1) and e1 < 2 * e0 and h1 < 2 * h0


def test_bounded_wait_gives_up_reports_and_keeps_the_context():
    """Failure detection without a fault: a wait of the pipelined kernels on a
    barrier that nothing completes gives up after its bound (0.5 s), sets bit 0
    of the status word, and the same context then steps and matches the
    reference fixture."""

    import ctypes

    import cases as CS
    from casebuild import golden, grouped_rel_l2, run_product

    from ionosphere_fdtd_b200 import _native as N

    s = sim(small_config(), dtype="float32")
    eng = s._engine
    assert eng.kernel_modes == ("pipeline", "pipeline")
    assert eng.status_word(reset=True) == 0
    waited = ctypes.c_double()
    N.check(N.load().ifdtd_wait_selftest(eng.plan, ctypes.byref(waited), eng.backend.stream_handle()), "ifdtd_wait_selftest")
    assert 0.45 < waited.value < 5.0
    assert eng.status_word(reset=True) & 1
    assert eng.status_word() == 0
    s.step(3)
    assert eng.status_word() == 0
    out = run_product(CS.CASES["config4_mini_s2"], "float32")
    assert max(grouped_rel_l2(out, golden("case_config4_mini_s2")).values()) < 2.0e-5
    assert out["_sim"]._engine.status_word() == 0


def test_uncompressed_checkpoint_has_the_same_arrays_and_resumes(tmp_path):
    """save_checkpoint(compress=False): same keys, shapes, dtypes and values as
    the compressed file (plasma and surface-impedance state included), a stored
    zip, and a bitwise continuation after loading."""

    import zipfile

    import cases as CS
    from casebuild import build_product

    case = dict(CS.CASES["config4_mini_s2"], steps=4, material="default")  # checkpoints need the stock material
    whole = build_product(case, "float32")
    part = build_product(case, "float32")
    whole.step(9)
    part.step(4)
    packed = part.save_checkpoint(tmp_path / "packed.npz")
    stored = part.save_checkpoint(tmp_path / "stored.npz", compress=False)
    with zipfile.ZipFile(stored) as z:
        assert all(i.compress_type == zipfile.ZIP_STORED for i in z.infolist())
    with np.load(packed) as a, np.load(stored) as b:
        assert sorted(a.files) == sorted(b.files)
        assert any(k.startswith("plasma_current_") for k in a.files) and "surface_impedance_memory" in a.files
        for k in a.files:
            assert a[k].dtype == b[k].dtype and a[k].shape == b[k].shape, k
            np.testing.assert_array_equal(a[k], b[k], err_msg=k)
    resumed = GeodesicFDTD.load_checkpoint(stored, device="cuda")
    resumed.step(5)
    for f in ("er", "et", "hr", "ht"):
        np.testing.assert_array_equal(resumed.to_numpy(getattr(resumed, f)), whole.to_numpy(getattr(whole, f)))


@pytest.mark.parametrize("kind", ["tm", "te"])
def test_surface_eigenmodes_follow_the_leapfrog_dispersion(kind):
    """The reference's eigenmode invariants (tests/test_maxwell_invariants.py:91-163)
    through the engine's half steps: an l = 1 surface mode keeps its shape and its
    amplitude follows the exact leapfrog dispersion (the oracle meets it to 8e-14,
    tests/test_invariants_cpu.py)."""

    from invariants import SURFACE_MODE, Vacuum, expected_amplitudes, surface_mode

    s = sim(SimulationConfig(**SURFACE_MODE), material=Vacuum())
    eigen, mode = surface_mode(s.mesh, kind)
    (s.er if kind == "tm" else s.hr)[:, 1] = s.backend.asarray(mode)
    amplitudes = [1.0]
    for _ in range(100):
        s._update_magnetic_fields()
        if kind == "te":
            s.ht.zero_()
        s._update_electric_fields()
        if kind == "tm":
            s.et.zero_()
            s.hr.zero_()
        else:
            s.er.zero_()
        values = s.to_numpy(s.er if kind == "tm" else s.hr)[:, 1]
        amplitudes.append(float(values @ mode / (mode @ mode)))
    radius = s.radii_m[1] if kind == "tm" else s.radial_midpoints_m[1]
    expected = expected_amplitudes(eigen, s.time_step_s, radius, 100, 0.5 if kind == "tm" else -0.5)
    np.testing.assert_allclose(amplitudes, expected, rtol=0.0, atol=1.0e-11)
    assert not np.any(s.to_numpy(s.hr if kind == "tm" else s.er))


def _peak(s) -> float:
    return max(float(np.max(np.abs(s.to_numpy(s.er)))), float(np.max(np.abs(s.to_numpy(s.et)))))


def test_conductive_update_is_passive_and_exact_in_the_stiff_limit():
    """The reference's loss invariants (tests/test_maxwell_invariants.py:219-291): a
    stiff conductor decays monotonically, to the exact exp(-sigma dt / eps0), with
    no sign flip."""

    from invariants import UniformConductive

    from ionosphere_fdtd_b200.constants import EPSILON_0

    s = sim(SimulationConfig(subdivision=0, radial_cells=2, courant_factor=0.2), material=UniformConductive(1.0))
    s.er.fill_(1.0)
    norms = [float(np.linalg.norm(s.to_numpy(s.er)))]
    s.step()
    np.testing.assert_allclose(s.to_numpy(s.er), np.exp(-1.0 * s.time_step_s / EPSILON_0), rtol=0.0, atol=1.0e-300)
    assert np.all(s.to_numpy(s.er) >= 0.0)
    norms.append(float(np.linalg.norm(s.to_numpy(s.er))))
    for _ in range(19):
        s.step()
        norms.append(float(np.linalg.norm(s.to_numpy(s.er))))
    assert np.all(np.diff(norms) <= 0.0)
    ca = s.to_numpy(s._ca_er)
    assert np.max(ca) < 1.0 and np.min(ca) >= 0.0


def test_exponential_conductive_forcing_converges_at_second_order():
    from invariants import UniformConductive, Vacuum

    from ionosphere_fdtd_b200.constants import EPSILON_0

    base = sim(SimulationConfig(subdivision=0, radial_cells=2, courant_factor=1.0), material=Vacuum())
    coarse_dt = 0.4 * base.cfl_time_step_limit_s
    coarse_steps = 20
    duration = coarse_steps * coarse_dt
    conductivity = 0.5 * EPSILON_0 / duration
    errors = []
    for refinement in (1, 2):
        dt = coarse_dt / refinement
        s = sim(SimulationConfig(subdivision=0, radial_cells=2, courant_factor=1.0, time_step_s=dt),
                material=UniformConductive(conductivity))
        a, b = float(s.to_numpy(s._ca_er)[0, 0]), float(s.to_numpy(s._cb_er)[0, 0])
        field = 0.0
        for step in range(coarse_steps * refinement):
            field = a * field + b * (step + 0.5) * dt
        exact = duration / conductivity - EPSILON_0 / conductivity**2 * (1.0 - np.exp(-conductivity * duration / EPSILON_0))
        errors.append(abs(field - exact))
    assert errors[0] / errors[1] == pytest.approx(4.0, rel=3.0e-3)


def test_trapezoidal_loss_keeps_its_coefficients():
    from invariants import UniformConductive

    from ionosphere_fdtd_b200.constants import EPSILON_0

    s = sim(SimulationConfig(subdivision=0, radial_cells=2, courant_factor=0.2, loss_integration="trapezoidal"),
            material=UniformConductive(1.0))
    loss = 1.0 * s.time_step_s / (2.0 * EPSILON_0)
    ca = s.to_numpy(s._ca_er)
    np.testing.assert_allclose(ca, (1.0 - loss) / (1.0 + loss), rtol=0.0, atol=0.0)
    assert np.all(ca < 0.0)


@pytest.mark.parametrize("case", ["subvacuum", "graded", "balanced"])
def test_runs_at_the_material_aware_cfl_limit_stay_bounded(case):
    """tests/test_maxwell_invariants.py:317-342 and 463-497 and tests/test_radial_grid.py
    of the reference: random fields at the CFL limit stay below twice their initial
    peak (sub-vacuum permittivity, an abruptly graded grid, a refined 2:1 grid)."""

    from invariants import GRADED_ALTITUDES, UniformPermittivity, Vacuum

    if case == "subvacuum":
        s = sim(SimulationConfig(subdivision=0, radial_cells=2, courant_factor=1.0), material=UniformPermittivity(0.01))
        steps = 400
    elif case == "balanced":
        a = P.build_refined_radial_grid(0.0, 100_000.0, 10_000.0, (P.RadialRefinementRegion(60_000.0, 90_000.0, 2_000.0),))
        s = sim(SimulationConfig(subdivision=0, radial_cells=len(a) - 1, minimum_altitude_m=a[0], maximum_altitude_m=a[-1],
                                 radial_altitudes_m=a, radial_grid_policy="balanced-2to1", courant_factor=1.0))
        steps = 1000
    else:
        a = GRADED_ALTITUDES
        s = sim(SimulationConfig(subdivision=0, radial_cells=len(a) - 1, minimum_altitude_m=a[0], maximum_altitude_m=a[-1],
                                 radial_altitudes_m=a, radial_grid_policy="allow-abrupt", courant_factor=1.0),
                material=Vacuum())
        steps = 1000
    rng = np.random.default_rng(20260805)
    s.er.copy_(s.backend.asarray(rng.standard_normal(tuple(s.er.shape))))
    s.et.copy_(s.backend.asarray(rng.standard_normal(tuple(s.et.shape))))
    initial = peak = _peak(s)
    for _ in range(steps):
        s.step()
        peak = max(peak, _peak(s))
    assert np.isfinite(peak) and peak < 2.0 * initial


def test_source_supports_keep_the_direction_and_staggered_altitude():
    """tests/test_solver.py of the reference: barycentric source weights reproduce the
    source direction, and the two radial nodes reproduce its altitude."""

    source = P.GaussianCurrent(altitude_m=2_500.0)
    s = sim(small_config(), source=source)
    vertices, _, weights = source.distribution(s)
    represented = weights @ s.mesh.vertices[vertices]
    represented /= np.linalg.norm(represented)
    assert weights.sum() == pytest.approx(1.0) and np.all(weights >= 0.0)
    assert represented @ source.direction() == pytest.approx(1.0)
    vertices, layers, weights = source.staggered_distribution(s)
    assert weights @ s.altitudes_m[layers] == pytest.approx(source.altitude_m)
    assert weights.sum() == pytest.approx(1.0) and len(np.unique(layers)) == 2
    s3 = sim(small_config(subdivision=3))
    assert P.geographic_face_index(s3, 0.0, 43.0) != P.geographic_face_index(s3, 0.0, -137.0)
    for lat, lon in ((0.0, 43.0), (0.0, -137.0), (89.9, 12.0), (-45.0, 180.0)):
        v, _, w = P.geographic_distribution(s3, lat, lon, 0.0)
        d = w @ s3.mesh.vertices[v]
        np.testing.assert_allclose(d / np.linalg.norm(d), P.geographic_direction(lat, lon), atol=1.0e-12)


def _represented_moments(s, source, current):
    vertices, layers, weights = source.staggered_distribution(s)
    s._update_electric_fields(current)
    er = s.to_numpy(s.er)
    cb = np.broadcast_to(s.to_numpy(s._cb_er), er.shape)
    density = -er[vertices, layers] / cb[vertices, layers]
    area = s.mesh.dual_cell_solid_angles[vertices] * s.radii_m[layers] ** 2
    return density * area * s.radial_node_control_lengths_m[layers], weights


@pytest.mark.parametrize("grid", ["uniform-24", "uniform-40", "uniform-80", "graded"])
def test_vertical_source_deposits_its_current_moment(grid):
    """The E update with current I deposits exactly I x element length, split by the
    support weights, on any radial grid (tests/test_solver.py of the reference)."""

    from invariants import GRADED_ALTITUDES

    if grid == "graded":
        a = GRADED_ALTITUDES
        cfg = SimulationConfig(subdivision=0, radial_cells=len(a) - 1, minimum_altitude_m=a[0], maximum_altitude_m=a[-1],
                               radial_altitudes_m=a, radial_grid_policy="allow-abrupt", courant_factor=0.2)
        source = P.GaussianCurrent(altitude_m=-500.0, peak_current_a=3.0, vertical_element_length_m=7_500.0)
    else:
        cfg = SimulationConfig(subdivision=0, radial_cells=int(grid.split("-")[1]), courant_factor=0.2)
        source = P.GaussianCurrent(altitude_m=2_500.0, peak_current_a=3.0, vertical_element_length_m=7_500.0)
    s = sim(cfg, source=source)
    moments, weights = _represented_moments(s, source, source.peak_current_a)
    np.testing.assert_allclose(moments, source.peak_current_a * source.vertical_element_length_m * weights, rtol=1e-12)
    assert moments.sum() == pytest.approx(source.peak_current_a * source.vertical_element_length_m)


@pytest.mark.parametrize("version", [1, 2])
def test_legacy_checkpoints_load_to_the_same_state(tmp_path, version):
    """Version-1 files (no face table) and version-2 files (no surface-impedance
    entry) restore the state of the current format (tests/test_checkpoint.py:163-202
    of the reference)."""

    import json

    s = sim(small_config(radial_cells=4), source=P.GaussianCurrent(peak_current_a=1.0e6))
    s.step(7)
    path = s.save_checkpoint(tmp_path / "current.npz")
    drop = {"mesh_faces", "mesh_face_levels"} if version == 1 else {"surface_impedance_memory"}
    with np.load(path, allow_pickle=False) as archive:
        arrays = {n: np.array(archive[n], copy=True) for n in archive.files if n not in drop}
    meta = json.loads(str(arrays["metadata"].item()))
    meta["version"] = version
    meta.pop("mesh" if version == 1 else "surface_impedance")
    arrays["metadata"] = np.asarray(json.dumps(meta))
    legacy = tmp_path / f"legacy-v{version}.npz"
    np.savez_compressed(legacy, **arrays)
    restored = GeodesicFDTD.load_checkpoint(legacy, device="cuda")
    assert restored.steps == s.steps and restored.time_s == s.time_s
    for f in ("er", "et", "hr", "ht"):
        np.testing.assert_array_equal(restored.to_numpy(getattr(restored, f)), s.to_numpy(getattr(s, f)))
    np.testing.assert_array_equal(restored.mesh.faces, s.mesh.faces)
    s.step(3)
    restored.step(3)
    for f in ("er", "et", "hr", "ht"):
        np.testing.assert_array_equal(restored.to_numpy(getattr(restored, f)), s.to_numpy(getattr(s, f)))


def test_compiled_steps_match_eager_and_the_gpu_alias_resolves_to_cuda():
    """tests/test_backends.py of the reference: compiled chunks of 8 plus a remainder
    give the eager result; ``device="gpu"`` is the CUDA device."""

    source = P.GaussianCurrent(peak_current_a=1.0e6)
    eager = sim(small_config(), source=source)
    compiled = sim(small_config(), source=source, compile_step=True, compile_chunk_size=8)
    eager.step(19)
    compiled.step(19)
    assert compiled.diagnostics()["compile_chunk_size"] == 8 and compiled.steps == 19
    for f in ("er", "et", "hr", "ht"):
        np.testing.assert_allclose(compiled.to_numpy(getattr(compiled, f)), eager.to_numpy(getattr(eager, f)),
                                   rtol=5.0e-13, atol=5.0e-29)
    alias = sim(small_config(), device="gpu")
    assert alias.er.device.type == "cuda" and alias.backend.device.startswith("cuda")


def _same_state(a, b):
    assert a.steps == b.steps and a.time_s == b.time_s
    for f in ("er", "et", "hr", "ht"):
        np.testing.assert_array_equal(a.to_numpy(getattr(a, f)), b.to_numpy(getattr(b, f)))


def test_checkpoint_keeps_tangential_source_optimised_mesh_and_precision(tmp_path):
    """tests/test_checkpoint.py:103-128 of the reference: a float32 run with a
    tangential source on an optimised mesh restores bitwise, and loads as float64."""

    source = P.TangentialGaussianCurrent(azimuths_deg=(15.0, 90.0), line_lengths_m=(10_000.0, 20_000.0),
                                         edge_assignment="nearest")
    s = sim(small_config(radial_cells=4, mesh_optimization_steps=1), source=source, dtype="float32")
    s.step(3)
    path = s.save_checkpoint(tmp_path / "tangential.npz")
    restored = GeodesicFDTD.load_checkpoint(path, device="cuda")
    assert restored.backend.dtype_name == "float32"
    _same_state(s, restored)
    np.testing.assert_array_equal(restored.mesh.vertices, s.mesh.vertices)
    converted = GeodesicFDTD.load_checkpoint(path, device="cuda", dtype="float64")
    assert converted.backend.dtype_name == "float64"
    for f in ("er", "et", "hr", "ht"):
        np.testing.assert_array_equal(converted.to_numpy(getattr(converted, f)),
                                      s.to_numpy(getattr(s, f)).astype(np.float64))


def test_checkpoint_keeps_custom_topology_and_refinement_metadata(tmp_path):
    """tests/test_checkpoint.py:131-162 of the reference."""

    import json

    uniform = P.build_geodesic_mesh(1)
    faces = np.roll(uniform.faces, 7, axis=0)
    levels = np.where(np.arange(len(faces)) % 2, 2, 1)
    mesh = P.build_geodesic_mesh_from_topology(uniform.vertices, faces, subdivision=1, face_levels=levels,
                                               refinement_spec={"balance": "2:1", "regions": [{"level": 2}]})
    s = sim(small_config(radial_cells=4), mesh=mesh, source=P.GaussianCurrent(peak_current_a=1.0e6))
    s.step(3)
    path = s.save_checkpoint(tmp_path / "adaptive.npz")
    with np.load(path, allow_pickle=False) as archive:
        assert json.loads(str(archive["metadata"].item()))["version"] == 4
        np.testing.assert_array_equal(archive["mesh_faces"], faces)
        np.testing.assert_array_equal(archive["mesh_face_levels"], levels)
    restored = GeodesicFDTD.load_checkpoint(path, device="cuda")
    assert restored.mesh.topology_kind == mesh.topology_kind and restored.mesh.refinement_spec == mesh.refinement_spec
    _same_state(s, restored)
    s.step(2)
    restored.step(2)
    _same_state(s, restored)


@pytest.mark.parametrize("orientation", ("native", "polar"))
def test_time_step_keeps_surface_spectra_inside_the_cfl_limit(orientation):
    """tests/test_maxwell_invariants.py:499-536 of the reference, on the engine's CFL step."""

    from invariants import SURFACE_MODE, Vacuum, courant_numbers

    s = sim(SimulationConfig(**dict(SURFACE_MODE, courant_factor=1.0, mesh_orientation=orientation)), material=Vacuum())
    tm_q, te_q = courant_numbers(s.mesh, s.time_step_s, float(s.radii_m.min()), float(s.radial_midpoints_m.min()))
    assert 0.0 < tm_q < 4.0 and 0.0 < te_q < 4.0


@pytest.mark.parametrize("orientation", ("polar", "native"))
@pytest.mark.parametrize("subdivision", (1, 3))
def test_tangential_source_samples_reconstruct_the_requested_moment(subdivision, orientation):
    """tests/test_maxwell_invariants.py:165-217 of the reference, on a simulation."""

    from invariants import tangential_case, tangential_moment_error

    source, line = tangential_case()
    s = sim(SimulationConfig(subdivision=subdivision, radial_cells=2, minimum_altitude_m=-5_000.0, maximum_altitude_m=5_000.0,
                             mesh_orientation=orientation), source=source)
    assert tangential_moment_error(s, source, line) < 2.0e-11
