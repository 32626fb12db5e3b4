"""Host-side parts of the engine that need no GPU: mesh tables (bit-exact with
the reference), setup coefficients (against the oracle), validation, and the
C ABI library's exports."""

import hashlib
import json
import re
from pathlib import Path

import numpy as np
import pytest

import cases as C
from casebuild import GOLDEN, golden

import ionosphere_fdtd_b200 as P
from ionosphere_fdtd_b200 import plasma as PL

ROOT = Path(__file__).resolve().parent.parent
INT_TABLES = ("edges", "faces", "face_edges", "face_edge_signs", "edge_left_faces", "edge_right_faces", "vertex_degree")
FLOAT_TABLES = ("vertices", "face_centers", "primal_edge_angles", "dual_edge_angles", "face_solid_angles", "dual_cell_solid_angles")


@pytest.mark.parametrize("level", [0, 1, 2, 3])
def test_mesh_tables_are_bit_exact_with_reference(level):
    ref = golden(f"mesh_s{level}")
    mesh = P.build_geodesic_mesh(level)
    for name in INT_TABLES + FLOAT_TABLES:
        np.testing.assert_array_equal(getattr(mesh, name), ref[name], err_msg=name)


# levels 7-9 are the benchmark meshes (s7: 163,842 vertices; s9: 2,621,442),
# whose digests the reference's own builder produced
@pytest.mark.parametrize("level", [4, 5, 6, 7, 8, 9])
def test_mesh_digests_match_reference(level):
    digests = json.loads((GOLDEN / "mesh_digests.json").read_text())[str(level)]
    mesh = P.build_geodesic_mesh(level)
    for name in INT_TABLES:
        got = hashlib.sha256(np.ascontiguousarray(getattr(mesh, name), dtype=np.int64).tobytes()).hexdigest()
        assert got == digests[name], name
    for name in FLOAT_TABLES:
        got = hashlib.sha256(np.ascontiguousarray(getattr(mesh, name), dtype=np.float64).tobytes()).hexdigest()
        assert got == digests[name], name


def test_mesh_counts_and_topology():
    for level in range(5):
        m = P.build_geodesic_mesh(level)
        assert (m.n_vertices, m.n_edges, m.n_faces) == (10 * 4**level + 2, 30 * 4**level, 20 * 4**level)
        assert np.count_nonzero(m.vertex_degree == 5) == 12
        assert not m.vertices.flags.writeable
        # boundary of boundary: grad then curl vanishes
        x = np.random.default_rng(level).standard_normal(m.n_vertices)
        np.testing.assert_allclose(m.face_circulation(m.edge_difference(x)), 0.0, atol=1e-12)


def test_custom_topology_renumbering_is_accepted():
    uniform = P.build_geodesic_mesh(1)
    custom = P.build_geodesic_mesh_from_topology(uniform.vertices, np.roll(uniform.faces, 1, axis=0))
    assert custom.topology_kind == "custom" and custom.n_edges == uniform.n_edges


def test_plasma_tables_match_oracle():
    import oracle.fdtd as O
    from casebuild import build_oracle

    case = C.CASES["plasma_magnetized_s1"]
    ora = build_oracle(case)
    mesh = P.build_geodesic_mesh(1)
    recon, _ = PL.face_reconstruction(mesh)
    np.testing.assert_array_equal(recon, ora.p_recon)
    faces, weights = PL.vertex_face_average(mesh)
    np.testing.assert_array_equal(faces, ora.p_vfaces)
    np.testing.assert_array_equal(weights, ora.p_vweights)
    assert O.OracleFDTD is type(ora)


def test_plasma_coefficients_compress_exactly_for_altitude_profiles():
    from casebuild import plasma_arrays, product_provenance

    case = C.CASES["plasma_drude_s2"]
    mesh = P.build_geodesic_mesh(2)
    mids, magnetic, species = plasma_arrays(case["plasma"], mesh.n_faces, case["config"])
    model = P.MeshPlasmaModel.from_mesh(
        mesh, mids, magnetic, tuple(P.ColdPlasmaSpecies(f"s{i}", *s) for i, s in enumerate(species)),
        provenance=(product_provenance(),), interpolation="synthetic",
    )
    coef, bdir, magnetized, rows = PL.ade_coefficients(model, 1.0e-6)
    assert rows == 1 and not magnetized
    # the same coefficients computed on the full grid, row by row
    full = []
    nu = species[0][3]
    full_decay = np.exp(-nu * 1.0e-6)
    np.testing.assert_array_equal(np.broadcast_to(coef[0, 0], full_decay.shape), full_decay)
    assert coef.shape == (1, 6, 1, len(mids)) and not full


def test_simulation_config_validation_messages():
    with pytest.raises(ValueError, match="mesh_relaxations"):
        P.SimulationConfig(mesh_relaxations=-1)
    with pytest.raises(ValueError, match="finite"):
        P.SimulationConfig(time_step_s=np.nan)
    with pytest.raises(ValueError, match="radial_cells"):
        P.SimulationConfig(subdivision=1, radial_cells=6, radial_altitudes_m=(-100_000.0, 0.0, 100_000.0))
    with pytest.raises(ValueError, match="minimum_altitude_m=0"):
        P.SimulationConfig(radial_boundary_condition="surface-impedance")
    with pytest.raises(ValueError, match="geometry_mode"):
        P.SimulationConfig(geometry_mode="flat")
    with pytest.raises(ValueError, match="smoothly graded"):
        P.SimulationConfig(subdivision=0, radial_cells=5, minimum_altitude_m=-10_000.0, maximum_altitude_m=4_000.0,
                           radial_altitudes_m=(-10_000.0, -6_000.0, -2_000.0, -1_000.0, 0.0, 4_000.0))


def test_sources_match_oracle_supports_and_waveform():
    import oracle.fdtd as O

    src = P.GaussianCurrent(peak_current_a=2.0, carrier_frequency_hz=20.0)
    osrc = O.OracleSource(peak_current_a=2.0, carrier_frequency_hz=20.0)
    times = np.linspace(0.0, 0.2, 101)
    np.testing.assert_array_equal(src.current_series(times, 1e-5), [src.current_a(t, 1e-5) for t in times])
    np.testing.assert_allclose([src.current_a(t, 1e-5) for t in times], [osrc.current_a(t, 1e-5) for t in times], rtol=0, atol=0)


def test_surface_impedance_fit_and_coefficients():
    model = P.ConductiveHalfSpaceSurface(1.0e-2)
    import oracle.fdtd as O

    ref = O.OracleSurface(1.0e-2)
    np.testing.assert_array_equal(model.pole_rates_s_inv, ref.poles())
    np.testing.assert_array_equal(model.diffusive_weights_sqrt_s_inv, ref.weights())
    f = np.linspace(5.0, 45.0, 9)
    rel = np.abs(model.impedance_ohm(f) - model.exact_impedance_ohm(f)) / np.abs(model.exact_impedance_ohm(f))
    assert np.max(rel) < 0.05


def test_geodesic_fdtd_refuses_cpu_backends():
    with pytest.raises(P.BackendUnavailableError):
        P.GeodesicFDTD(P.SimulationConfig(subdivision=0, radial_cells=2), backend="numpy")
    try:
        import torch

        cuda = torch.cuda.is_available()
    except ImportError:  # pragma: no cover
        cuda = False
    if not cuda:
        with pytest.raises(P.BackendUnavailableError):
            P.GeodesicFDTD(P.SimulationConfig(subdivision=0, radial_cells=2), backend="torch", device="cuda")
    with pytest.raises(P.BackendUnavailableError):
        P.GeodesicFDTD(P.SimulationConfig(subdivision=0, radial_cells=2), backend="torch", device="cpu")


def test_checkpoint_metadata_rejects_foreign_files(tmp_path):
    path = tmp_path / "bad.npz"
    np.savez_compressed(path, metadata=np.asarray(json.dumps({"format": "other", "version": 4})))
    with pytest.raises(P.CheckpointError, match="not an ionosphere-fdtd checkpoint"):
        P.load_checkpoint(path)
    np.savez_compressed(path, metadata=np.asarray(json.dumps({"format": "ionosphere-fdtd-checkpoint", "version": 9})))
    with pytest.raises(P.CheckpointError, match="unsupported checkpoint version"):
        P.load_checkpoint(path)
    (tmp_path / "trunc.npz").write_bytes(b"PK\x03\x04 truncated")
    with pytest.raises(P.CheckpointError):
        P.load_checkpoint(tmp_path / "trunc.npz")


def test_checkpoint_table_gives_the_keys_of_every_version():
    """The archive keys each format version must hold (checkpoint.py:23-477 of the
    reference: v2 adds the mesh topology, v3 the surface memory, v4 the plasma)."""

    from ionosphere_fdtd_b200 import checkpoint as CK

    base = {"metadata", "mesh_vertices", "er", "et", "hr", "ht"}
    assert CK.required_keys(1, None) == base
    assert CK.required_keys(2, None) == base | {"mesh_faces", "mesh_face_levels"}
    assert CK.required_keys(3, None) == base | {"mesh_faces", "mesh_face_levels", "surface_impedance_memory"}
    plasma = {"arrays": ["number_density", "magnetic_field"], "species": [{}, {}]}
    assert CK.required_keys(4, plasma) == CK.required_keys(3, None) | {
        "plasma_model_number_density", "plasma_model_magnetic_field", "plasma_current_0", "plasma_current_1"}
    assert [e.key for e in CK.ARCHIVE][:8] == ["metadata", "mesh_vertices", "mesh_faces", "mesh_face_levels", "er", "et", "hr", "ht"]


def test_checkpoint_reports_missing_arrays_and_metadata_sections(tmp_path):
    meta = {"format": "ionosphere-fdtd-checkpoint", "version": 1, "simulation_config": {}, "material": {}, "source": None,
            "state": {}, "runtime": {}}
    path = tmp_path / "v1.npz"
    np.savez(path, metadata=np.asarray(json.dumps(meta)), mesh_vertices=np.zeros((12, 3)), er=np.zeros(1))
    with pytest.raises(P.CheckpointError, match="checkpoint is missing arrays: et, hr, ht"):
        P.load_checkpoint(path)
    np.savez(path, metadata=np.asarray(json.dumps(dict(meta, version=3))))
    with pytest.raises(P.CheckpointError, match="checkpoint metadata is missing: mesh, surface_impedance"):
        P.load_checkpoint(path)
    np.savez(path, er=np.zeros(1))
    with pytest.raises(P.CheckpointError, match="checkpoint is missing arrays: metadata"):
        P.load_checkpoint(path)


def test_plasma_artifact_round_trip_and_corruption(tmp_path):
    from casebuild import product_provenance

    mesh = P.build_geodesic_mesh(0)
    shape = (mesh.n_faces, 2)
    magnetic = np.zeros((*shape, 3))
    magnetic[..., 2] = 5e-5
    sp = P.ColdPlasmaSpecies("electron", -P.ELEMENTARY_CHARGE_C, P.ELECTRON_MASS_KG, np.full(shape, 1e3), np.full(shape, 200.0))
    model = P.MeshPlasmaModel.from_mesh(mesh, np.asarray((25e3, 75e3)), magnetic, (sp,), provenance=(product_provenance(),), interpolation="x")
    restored = P.MeshPlasmaModel.load(model.save(tmp_path / "p.npz"))
    assert restored.content_sha256 == model.content_sha256
    with np.load(tmp_path / "p.npz") as a:
        arrays = {n: np.array(a[n]) for n in a.files}
    arrays["magnetic_field_t"][0, 0, 0] += 1e-9
    np.savez_compressed(tmp_path / "c.npz", **arrays)
    with pytest.raises(ValueError, match="checksum mismatch"):
        P.MeshPlasmaModel.load(tmp_path / "c.npz")


def _declared_symbols() -> set[str]:
    """Every entry point declared in the public headers (include/*.h)."""

    names: set[str] = set()
    for header in sorted((ROOT / "include").glob("*.h")):
        names |= set(re.findall(r"^\s*int32_t\s+(ifdtd_\w+)\s*\(", header.read_text(), flags=re.M))
    return names


def test_c_abi_library_exports_every_declared_symbol():
    import ctypes

    from ionosphere_fdtd_b200 import _native as N
    from ionosphere_fdtd_b200.build import build

    build()
    lib = ctypes.CDLL(str(N.LIBRARY))
    declared = _declared_symbols()
    assert len(declared) >= 15
    for name in declared:
        assert hasattr(lib, name), name
    assert declared == set(N.exported_symbols())
    assert N.load().ifdtd_version() >= 10000


def test_c_abi_reports_missing_device_or_bad_arguments():
    import ctypes

    from ionosphere_fdtd_b200 import _native as N

    lib = N.load()
    plan = ctypes.c_void_p()
    status = lib.ifdtd_plan_create(None, None, None, None, 4, 0, ctypes.byref(plan))
    assert status == N.ERR_ARGUMENT and "null" in N.last_error()
    count = ctypes.c_int32(-1)
    lib.ifdtd_device_count(ctypes.byref(count))
    assert count.value >= 0


def test_kernel_division_by_magic_multiply_is_exact():
    """The step kernels split flat work indices with q = umulhi(n, ceil(2^32/d))
    (d = 1 encoded as the identity); exact for every divisor they use."""

    for d in range(1, 1025):
        m = 0 if d == 1 else (0xFFFFFFFF // d + 1)
        n = np.arange(0, 1 << 16, dtype=np.uint64)
        q = n if m == 0 else (n * np.uint64(m)) >> np.uint64(32)
        assert np.array_equal(q, n // d), d


def test_geographic_face_search_equals_the_full_scan():
    """The cone-filtered face search picks the face the test over all faces
    picks (sources.py:53-85), random directions, vertices and edge midpoints."""

    from ionosphere_fdtd_b200 import sources as S
    from ionosphere_fdtd_b200.mesh import build_geodesic_mesh

    class Sim:
        pass

    def full_scan(sim, lat, lon):
        d = S.geographic_direction(lat, lon)
        tri = sim.mesh.vertices[sim.mesh.faces]
        sides = np.column_stack([np.einsum("ij,j->i", np.cross(tri[:, k], tri[:, (k + 1) % 3]), d) for k in range(3)])
        inside = np.all(sides >= -1.0e-12, axis=1) | np.all(sides <= 1.0e-12, axis=1)
        cand = np.flatnonzero(inside)
        c = sim.mesh.face_centers
        return int(cand[np.argmax(c[cand] @ d)]) if len(cand) else int(np.argmax(c @ d))

    rng = np.random.default_rng(7)
    for sub in (0, 1, 3, 5):
        sim = Sim()
        sim.mesh = build_geodesic_mesh(sub)
        v, e = sim.mesh.vertices, sim.mesh.edges
        step = max(1, len(v) // 150)
        dirs = [v[i] for i in range(0, len(v), step)]
        dirs += [(v[a] + v[b]) / np.linalg.norm(v[a] + v[b]) for a, b in e[:: 3 * step + 8]]
        points = [(float(np.degrees(np.arcsin(np.clip(u[2], -1, 1)))), float(np.degrees(np.arctan2(u[1], u[0])))) for u in dirs]
        points += [(90.0, 0.0), (-90.0, 0.0), (89.9999, 17.0), (-89.9999, -163.0), (0.0, 180.0), (0.0, -180.0)]
        points += [(float(rng.uniform(-90, 90)), float(rng.uniform(-180, 180))) for _ in range(100)]
        for lat, lon in points:
            assert S.geographic_face_index(sim, lat, lon) == full_scan(sim, lat, lon), (sub, lat, lon)


def test_ensemble_rejects_empty_member_lists_and_bad_chunks():
    from ionosphere_fdtd_b200 import Ensemble

    with pytest.raises(ValueError, match="at least one member"):
        Ensemble([])
    with pytest.raises(ValueError, match="graph_chunk"):
        Ensemble([object()], graph_chunk=0)
    with pytest.raises(TypeError, match="GeodesicFDTD"):
        Ensemble([object()])


def test_ensemble_refuses_a_replaced_engine_even_at_the_same_plan_address():
    """A freed plan's address can be handed to the next plan; the batch must still
    refuse a member whose engine was replaced (host logic only, no device)."""

    import ctypes

    from ionosphere_fdtd_b200 import Ensemble

    class FakeEngine:
        def __init__(self, address):
            self.plan = ctypes.c_void_p(address)

    class FakeMember:
        def __init__(self, engine):
            self._engine = engine

    members = [FakeMember(FakeEngine(0x1000)), FakeMember(FakeEngine(0x2000))]
    ens = Ensemble.__new__(Ensemble)
    ens._members = members
    ens._engines = [m._engine for m in members]
    ens._handle = ctypes.c_void_p(0x3000)
    assert ens._live().value == 0x3000
    members[1]._engine = FakeEngine(0x2000)  # a new engine whose plan reuses the freed address
    with pytest.raises(ValueError, match="plan changed"):
        ens._live()
    members[1]._engine = ens._engines[1]
    ens._engines[1].plan = ctypes.c_void_p()  # the original engine closed in place
    with pytest.raises(ValueError, match="plan changed"):
        ens._live()
    ens._handle = ctypes.c_void_p()  # nothing to destroy on the fake handle
    with pytest.raises(ValueError, match="closed"):
        ens._live()


def test_autotune_rejects_bad_arguments_before_touching_the_device():
    from ionosphere_fdtd_b200.autotune import autotune

    with pytest.raises(ValueError, match="positive"):
        autotune(object(), steps=0)
    with pytest.raises(ValueError, match="candidate"):
        autotune(object(), candidates=())


def test_threaded_row_chunks_give_the_same_mesh_bits(monkeypatch):
    import ionosphere_fdtd_b200.mesh as M

    serial = M.build_geodesic_mesh(3)
    serial_midpoints = serial.edge_midpoints()
    monkeypatch.setattr(M, "_ROWS_PER_CHUNK", 97)  # many uneven chunks on several threads
    chunked = M.build_geodesic_mesh(3)
    for name in ("faces", "edges", "face_centers", "primal_edge_angles", "dual_edge_angles", "face_solid_angles",
                 "dual_cell_solid_angles", "vertex_degree"):
        np.testing.assert_array_equal(getattr(chunked, name), getattr(serial, name), err_msg=name)
    np.testing.assert_array_equal(chunked.edge_midpoints(), serial_midpoints)
    np.testing.assert_array_equal(serial_midpoints, M._unit(serial.vertices[serial.edges].sum(axis=1)))


def test_first_use_numbering_matches_a_sequential_dict():
    import ionosphere_fdtd_b200.mesh as M

    rng = np.random.default_rng(5)
    for n, nv in ((0, 5), (1, 3), (1000, 40), (20000, 3000)):
        lo = rng.integers(0, nv, n)
        hi = rng.integers(0, nv, n)
        seen: dict = {}
        rank_ref, first_ref = [], []
        for i, key in enumerate(zip(lo.tolist(), hi.tolist())):
            if key not in seen:
                seen[key] = len(seen)
                first_ref.append(i)
            rank_ref.append(seen[key])
        rank, first = M._first_use_numbering(lo, hi, nv)
        np.testing.assert_array_equal(rank, np.asarray(rank_ref, dtype=np.int64).reshape(rank.shape))
        np.testing.assert_array_equal(first, np.asarray(first_ref, dtype=np.int64).reshape(first.shape))


def test_new_entry_points_reject_bad_arguments_before_any_device_work():
    import ctypes

    from ionosphere_fdtd_b200 import _native as N

    lib = N.load()
    out = ctypes.c_void_p()
    assert lib.ifdtd_batch_create(None, 0, 32, ctypes.byref(out)) == 1  # IFDTD_ERR_ARGUMENT
    plans = (ctypes.c_void_p * 1)(None)
    assert lib.ifdtd_batch_create(plans, 1, 32, ctypes.byref(out)) == 1
    assert lib.ifdtd_batch_create(plans, 1, 0, ctypes.byref(out)) == 1
    assert lib.ifdtd_batch_step(None, None, None, 1, None, None, None) == 1
    # surrogate kernels: shapes and leading dimensions are checked on the host
    assert lib.ifdtd_nn_gemm(0, 4, 4, 1, 4, 0, 1, 4, 0, 1.0, 0.0, 1, 4, None) == 1
    assert lib.ifdtd_nn_gemm(4, 4, 8, 1, 4, 0, 1, 4, 0, 1.0, 0.0, 1, 4, None) == 1  # lda < k
    assert lib.ifdtd_nn_gemm(4, 4, 4, 1, 4, 0, 1, 4, 0, 1.0, 0.0, 1, 2, None) == 1  # ldc < n
    assert lib.ifdtd_nn_adam(4, 1, 1, 1, 1, 1e-3, 0.9, 0.999, 1e-8, 0, None, None) == 1  # step must be >= 1
    assert lib.ifdtd_nn_bias_act(4, 4, 1, 1, 2, None, None) == 1  # act must be 0 or 1
    buf = ctypes.create_string_buffer(64)
    lib.ifdtd_last_error(buf, 64)
    assert b"bias_act" in buf.value
    # host numbering: indices outside [0, n_vertices) are refused
    lo = np.asarray([0, 5], dtype=np.int64)
    hi = np.asarray([1, 2], dtype=np.int64)
    rank = np.empty(2, dtype=np.int64)
    first = np.empty(2, dtype=np.int64)
    count = ctypes.c_int64()
    assert lib.ifdtd_first_use_numbering(N.ptr_i64(lo), N.ptr_i64(hi), 2, 4, N.ptr_i64(rank), N.ptr_i64(first), ctypes.byref(count)) == 1


def test_material_validation_checks_broadcast_samples_once_with_the_same_messages():
    from ionosphere_fdtd_b200.solver import _validated_material_sample as validate

    ones = np.ones((5, 2))
    with pytest.raises(ValueError, match="must be finite"):
        validate((np.broadcast_to(np.array([1.0, np.nan]), (5, 2)), ones), (5, 2), "node")
    with pytest.raises(ValueError, match="conductivity cannot be negative"):
        validate((np.broadcast_to(np.array([[1.0], [-1.0]]), (2, 5)), np.ones((2, 5))), (2, 5), "node")
    with pytest.raises(ValueError, match="permittivity must be positive"):
        validate((ones, np.broadcast_to(0.0, (5, 2))), (5, 2), "edge")
    with pytest.raises(ValueError, match="must have shape"):
        validate((np.broadcast_to(1.0, (5, 3)), ones), (5, 2), "node")
    sigma, eps = validate((np.broadcast_to(np.array([0.0, 1e-3]), (5, 2)), ones), (5, 2), "node")
    assert sigma.shape == (5, 2) and sigma.strides[0] == 0


def test_array_digest_is_the_digest_of_the_canonical_bytes():
    """Chunked hashing gives the SHA-256 of the whole array's little-endian C-order
    bytes (floats as <f8, integers as <i8), for any layout."""

    from ionosphere_fdtd_b200.provenance import array_sha256

    def whole(a):
        a = np.asarray(a)
        dtype = "<f8" if np.issubdtype(a.dtype, np.floating) else "<i8"
        return hashlib.sha256(np.asarray(a, dtype=dtype, order="C").tobytes()).hexdigest()

    rng = np.random.default_rng(3)
    cases = [
        rng.standard_normal((3000, 80, 3)),
        np.broadcast_to(rng.standard_normal((1, 40, 3)), (70_000, 40, 3)),
        rng.standard_normal((500, 7)).T,
        rng.integers(0, 1 << 30, (9000, 3)).astype(np.int32),
        rng.standard_normal(100).astype(">f8"),
        rng.standard_normal((4, 5)).astype(np.float32),
        np.float64(2.5),
        np.zeros((0, 3)),
        np.arange(17),
    ]
    for a in cases:
        assert array_sha256(a) == whole(a)


def test_plasma_validation_sees_bad_values_in_broadcast_profiles():
    from casebuild import product_provenance

    mesh = P.build_geodesic_mesh(0)
    h = np.array([60_000.0, 80_000.0])
    shape = (mesh.n_faces, 2)
    good = np.broadcast_to(np.array([1e6, 1e8]), shape)
    with pytest.raises(ValueError, match="density/collision"):
        P.ColdPlasmaSpecies("e", -P.ELEMENTARY_CHARGE_C, P.ELECTRON_MASS_KG, np.broadcast_to(np.array([1e6, -1.0]), shape), good)
    with pytest.raises(ValueError, match="density/collision"):
        P.ColdPlasmaSpecies("e", -P.ELEMENTARY_CHARGE_C, P.ELECTRON_MASS_KG, good, np.broadcast_to(np.array([0.0, 1e3]), shape))
    sp = P.ColdPlasmaSpecies("e", -P.ELEMENTARY_CHARGE_C, P.ELECTRON_MASS_KG, good, good)
    bad_b = np.broadcast_to(np.array([[[0.0, 0.0, 5e-5], [0.0, np.inf, 0.0]]]), (*shape, 3))
    with pytest.raises(ValueError, match="magnetic field must be finite"):
        P.MeshPlasmaModel.from_mesh(mesh, h, bad_b, (sp,), provenance=(product_provenance(),), interpolation="profile")
    ok_b = np.broadcast_to(np.zeros((1, 2, 3)), (*shape, 3))
    model = P.MeshPlasmaModel.from_mesh(mesh, h, ok_b, (sp,), provenance=(product_provenance(),), interpolation="profile")
    assert model.magnetic_field_t.shape == (*shape, 3)


def test_stable_grouping_is_the_stable_argsort():
    from ionosphere_fdtd_b200 import _native as N

    rng = np.random.default_rng(11)
    for n, n_keys in ((0, 3), (1, 1), (1000, 7), (200_000, 5000), (50_000, 100_000)):
        keys = rng.integers(0, n_keys, n).astype(np.int64)
        order = np.empty(n, dtype=np.int64)
        counts = np.empty(n_keys, dtype=np.int64)
        assert N.load().ifdtd_stable_group(N.ptr_i64(keys), n, n_keys, N.ptr_i64(order), N.ptr_i64(counts)) == 0
        np.testing.assert_array_equal(order, np.argsort(keys, kind="stable"))
        np.testing.assert_array_equal(counts, np.bincount(keys, minlength=n_keys))
    bad = np.array([0, 3, 1], dtype=np.int64)
    order = np.empty(3, dtype=np.int64)
    counts = np.empty(3, dtype=np.int64)
    assert N.load().ifdtd_stable_group(N.ptr_i64(bad), 3, 3, N.ptr_i64(order), N.ptr_i64(counts)) != 0
    assert N.load().ifdtd_stable_group(N.ptr_i64(bad), 3, 0, N.ptr_i64(order), N.ptr_i64(counts)) != 0


def test_vertex_face_tables_equal_the_incidence_scan():
    """The incident faces of every vertex in face order with area weights, as a
    sequential scan over the faces builds them (plasma.py:572-588)."""

    for level in (0, 2, 4):
        mesh = P.build_geodesic_mesh(level)
        faces, weights = PL.vertex_face_average(mesh)
        inc = [[] for _ in range(mesh.n_vertices)]
        for f, tri in enumerate(mesh.faces.tolist()):
            for v in tri:
                inc[v].append(f)
        width = max(len(x) for x in inc)
        assert faces.shape == (mesh.n_vertices, width)
        for v, fl in enumerate(inc):
            np.testing.assert_array_equal(faces[v, : len(fl)], fl)
            assert not faces[v, len(fl) :].any() and not weights[v, len(fl) :].any()
            w = mesh.face_solid_angles[fl] / np.sum(mesh.face_solid_angles[fl])
            np.testing.assert_allclose(weights[v, : len(fl)], w, rtol=1e-15, atol=0)


def test_backend_contract_names_of_the_reference_are_available():
    """The reference's seam (backends/base.py:19-89): CudaBackend implements every
    abstract method of ArrayBackend and answers to the Torch backend's name."""

    import inspect

    assert issubclass(P.CudaBackend, P.ArrayBackend) and not inspect.isabstract(P.CudaBackend)
    assert P.TorchBackend is P.CudaBackend and P.CudaBackend.name == "torch"
    assert issubclass(P.DataArtifactError, ValueError)
    with pytest.raises(P.BackendUnavailableError):
        P.create_backend("numpy", P.build_geodesic_mesh(0))
    with pytest.raises(ValueError, match="backend must be"):
        P.create_backend("jax", P.build_geodesic_mesh(0))
