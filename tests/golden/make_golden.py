"""Generate golden fixtures by running the reference solver itself.

Run it where the reference source tree is available, giving the reference's
``src`` directory as the first argument (required):

    python tests/golden/make_golden.py <reference>/src [--mesh-levels=7,8,9]

It imports the reference package from the given source directory, runs every
case of ``cases.py`` on the reference NumPy float64 backend (plus the float32
pin of the reference's own FP32 test), and writes compressed ``.npz``
fixtures next to this script.  The fixtures travel with the repository; no
test reads the reference at run time.
"""

from __future__ import annotations

import hashlib
import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))

import cases as C  # noqa: E402


def _import_reference(src: str):
    sys.path.insert(0, src)
    import ionosphere_fdtd  # noqa: F401
    from ionosphere_fdtd import mesh as rmesh
    from ionosphere_fdtd import solver as rsolver
    from ionosphere_fdtd import sources as rsources
    from ionosphere_fdtd import surface_impedance as rsi
    from ionosphere_fdtd import plasma as rplasma
    from ionosphere_fdtd import materials as rmat
    from ionosphere_fdtd import data_artifacts as rdata
    from ionosphere_fdtd.backends import numpy_backend as rnb

    return rmesh, rsolver, rsources, rsi, rplasma, rmat, rdata, rnb


def _sha(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def _provenance(rdata):
    return rdata.DatasetProvenance(
        dataset_id="golden.synthetic-plasma.v1",
        title="Synthetic plasma for parity fixtures",
        version="1",
        source_url="https://example.invalid/golden-plasma",
        citation="Synthetic fixture.",
        license="CC0-1.0",
        retrieved_at="2026-12-01T00:00:00Z",
        source_sha256="0" * 64,
        coordinate_reference_system="geocentric Cartesian",
        variables=(
            rdata.VariableProvenance("B", "T", "T", "identity"),
            rdata.VariableProvenance("number_density", "m^-3", "m^-3", "identity"),
            rdata.VariableProvenance("collision_frequency", "Hz", "Hz", "identity"),
        ),
    )


def build_reference(case: dict, mods, dtype: str = "float64"):
    rmesh, rsolver, rsources, rsi, rplasma, rmat, rdata, _ = mods
    cfg = rsolver.SimulationConfig(**case["config"])
    if "adaptive" in case:
        from ionosphere_fdtd import adaptive_mesh as ram

        base, regions = case["adaptive"]
        mesh = ram.build_adaptive_geodesic_mesh(base, tuple(ram.SphericalRefinementRegion(*r) for r in regions))
    else:
        mesh = rmesh.build_geodesic_mesh(cfg.subdivision)
    mat = case.get("material", "default")
    if mat == "default":
        material = None
    elif mat == "profile":
        material = C.ProfileMaterial()
    elif mat == "patchy":
        material = C.PatchyMaterial()
    else:
        material = rmat.EarthIonosphereMaterial(**mat[1])
    source = None
    spec = case.get("source")
    if spec is not None:
        spec = dict(spec)
        kind = spec.pop("kind")
        if "seed_vertex" in spec:
            lat, lon = C.vertex_lat_lon(mesh.vertices, C.source_vertex(mesh.n_vertices, spec.pop("seed_vertex")))
            spec.update(latitude_deg=lat, longitude_deg=lon)
        source = (rsources.TangentialGaussianCurrent if kind == "tangential" else rsources.GaussianCurrent)(**spec)
    surface = None
    sspec = case.get("surface")
    if sspec is not None:
        if sspec["conductivity"] == "scalar":
            surface = rsi.ConductiveHalfSpaceSurface(sspec["value"])
        else:
            surface = rsi.ConductiveHalfSpaceSurface(C.smooth_log_normal(mesh.edge_midpoints(), sspec["seed"]))
    plasma = None
    pspec = case.get("plasma")
    if pspec is not None:
        alt = np.linspace(cfg.minimum_altitude_m, cfg.maximum_altitude_m, cfg.radial_cells + 1)
        mids = 0.5 * (alt[:-1] + alt[1:])
        shape = (mesh.n_faces, len(mids))
        if pspec["kind"] == "profile":
            magnetic, density, collision = C.profile_plasma_arrays(mesh.n_faces, mids, pspec["magnetic_t"])
        else:
            magnetic = np.zeros((*shape, 3))
            magnetic[..., 2] = pspec["magnetic_t"]
            density = np.full(shape, pspec["density_m3"])
            collision = np.full(shape, pspec["collision_hz"])
        species = [rplasma.ColdPlasmaSpecies("electron", -rplasma.ELEMENTARY_CHARGE_C, rplasma.ELECTRON_MASS_KG, density, collision)]
        if pspec.get("two_species"):
            species.append(rplasma.ColdPlasmaSpecies("O+", rplasma.ELEMENTARY_CHARGE_C, 16 * 1.672_621_925_95e-27, 0.5 * density, 0.1 * collision))
        plasma = rplasma.MeshPlasmaModel.from_mesh(
            mesh, mids, magnetic, tuple(species), provenance=(_provenance(rdata),), interpolation="synthetic"
        )
    sim = rsolver.GeodesicFDTD(
        cfg, material=material, source=source, surface_impedance=surface, plasma=plasma, mesh=mesh, backend="numpy", dtype=dtype
    )
    init = case.get("init")
    if init is not None:
        shapes = {name: getattr(sim, name).shape for name in ("er", "et", "hr", "ht")}
        for name, values in C.initial_fields(shapes, *init).items():
            getattr(sim, name)[:] = values
    return sim


def run_case(name: str, case: dict, mods, dtype: str = "float64") -> dict:
    sim = build_reference(case, mods, dtype)
    out: dict[str, np.ndarray] = {"time_step_s": np.asarray(sim.time_step_s), "cfl_limit_s": np.asarray(sim.cfl_time_step_limit_s)}
    rspec = case.get("receivers")
    if rspec is not None:
        v, k, w = C.receiver_rows(sim.mesh.n_vertices, sim.altitudes_m, rspec["seed"], rspec["count"])
        out["traces"] = sim.record_er_observations(v, k, w, case["steps"])
    else:
        sim.step(case["steps"])
    for field in ("er", "et", "hr", "ht"):
        out[field] = np.asarray(getattr(sim, field))
    if sim._surface_impedance_ade is not None:
        out["si_memory"] = np.asarray(sim._surface_impedance_ade.memory)
    if sim._plasma_coupler is not None:
        for i, j in enumerate(sim._plasma_coupler.ade.current_density):
            out[f"plasma_current_{i}"] = np.asarray(j)
    out["max_abs"] = np.asarray([float(np.max(np.abs(out[f]))) for f in ("er", "et", "hr", "ht")])
    return out


def mesh_fixtures(mods, levels=range(0, 7)) -> None:
    """SHA-256 digests of the reference's mesh tables per subdivision level
    (merged into ``mesh_digests.json``), and full tables up to level 3."""

    rmesh = mods[0]
    rnb = mods[7]
    path = HERE / "mesh_digests.json"
    digests = json.loads(path.read_text()) if path.exists() else {}
    tables = ("edges", "faces", "face_edges", "face_edge_signs", "edge_left_faces", "edge_right_faces", "vertex_degree")
    floats = ("vertices", "face_centers", "primal_edge_angles", "dual_edge_angles", "face_solid_angles", "dual_cell_solid_angles")
    for level in levels:
        mesh = rmesh.build_geodesic_mesh(level)
        backend = rnb.NumPyBackend(mesh)
        entry = {t: _sha(np.asarray(getattr(mesh, t), dtype=np.int64)) for t in tables}
        entry["vertex_edges"] = _sha(np.asarray(backend.vertex_edges, dtype=np.int64))
        entry["vertex_edge_signs"] = _sha(np.asarray(backend.vertex_edge_signs, dtype=np.float64))
        entry.update({f: _sha(np.asarray(getattr(mesh, f), dtype=np.float64)) for f in floats})
        digests[str(level)] = entry
        print("mesh digests", level, flush=True)
        if level <= 3:
            arrays = {t: np.asarray(getattr(mesh, t)) for t in tables + floats}
            arrays["vertex_edges"] = backend.vertex_edges
            arrays["vertex_edge_signs"] = backend.vertex_edge_signs
            np.savez_compressed(HERE / f"mesh_s{level}.npz", **arrays)
        path.write_text(json.dumps(digests, indent=1, sort_keys=True) + "\n")


def checkpoint_fixture(mods) -> None:
    """A reference-written v4 checkpoint (surface impedance + source, float64)
    and the reference's continuation after 7 more steps."""

    _, rsolver, rsources, rsi, _, rmat, _, _ = mods
    cfg = rsolver.SimulationConfig(
        subdivision=1, radial_cells=4, minimum_altitude_m=0.0, maximum_altitude_m=100_000.0,
        courant_factor=0.25, radial_boundary_condition="surface-impedance",
    )
    source = rsources.GaussianCurrent(peak_current_a=2.0e6, center_time_s=1.0e-4, one_over_e_half_width_s=5.0e-5, carrier_frequency_hz=5.0)
    sim = rsolver.GeodesicFDTD(cfg, material=rmat.EarthIonosphereMaterial(), source=source,
                               surface_impedance=rsi.ConductiveHalfSpaceSurface(1.0 / 30.0), backend="numpy", dtype="float64")
    shapes = {n: getattr(sim, n).shape for n in ("er", "et", "hr", "ht")}
    for n, v in C.initial_fields(shapes, 99, 1.0e-9).items():
        getattr(sim, n)[:] = v
    sim.step(5)
    sim.save_checkpoint(HERE / "reference_checkpoint_v4.npz")
    sim.step(7)
    np.savez_compressed(
        HERE / "reference_checkpoint_continuation.npz",
        steps_before=np.asarray(5), steps_after=np.asarray(7),
        er=sim.er, et=sim.et, hr=sim.hr, ht=sim.ht, si_memory=sim._surface_impedance_ade.memory,
    )


def receiver_traces_fixture(mods) -> None:
    """The reference's ``record_receiver_traces`` (visualization.py:212-252) on the
    receiver-trace case of ``cases.py``."""

    from ionosphere_fdtd import visualization as rvis

    spec = C.RECEIVER_TRACES
    sim = build_reference(C.CASES[spec["case"]], mods)
    receivers = [rvis.Receiver(lat, lon, alt, label) for lat, lon, alt, label in spec["receivers"]]
    traces = rvis.record_receiver_traces(sim, receivers, spec["steps"], sample_every=spec["sample_every"])
    np.savez_compressed(
        HERE / "receiver_traces_source_s1.npz",
        time_s=traces.time_s, er_v_m=traces.er_v_m, labels=np.asarray(traces.labels),
        steps_after=np.asarray(sim.steps), time_after=np.asarray(sim.time_s),
    )


def radial_grid_fixture() -> None:
    """The reference's refined radial grids and their validation records."""

    from ionosphere_fdtd.radial_grid import RadialRefinementRegion, build_refined_radial_grid, validate_radial_grid

    out = {}
    for i, (lo, hi, step, regions) in enumerate(C.RADIAL_GRIDS):
        nodes = build_refined_radial_grid(lo, hi, step, tuple(RadialRefinementRegion(*r) for r in regions))
        v = validate_radial_grid(nodes)
        out[f"nodes_{i}"] = np.asarray(nodes)
        out[f"validation_{i}"] = np.asarray((v.cells, v.minimum_step_m, v.maximum_step_m, v.maximum_adjacent_step_ratio))
    np.savez_compressed(HERE / "radial_grids.npz", **out)


def main(src: str) -> None:
    mods = _import_reference(src)
    if "--radial-grids-only" in sys.argv:
        radial_grid_fixture()
        return
    if "--checkpoint-only" in sys.argv:
        checkpoint_fixture(mods)
        return
    if "--receivers-only" in sys.argv:
        receiver_traces_fixture(mods)
        return
    levels = [a.split("=", 1)[1] for a in sys.argv if a.startswith("--mesh-levels=")]
    if levels:
        # the large levels only (s9 takes the reference's builder minutes): --mesh-levels=7,8,9
        mesh_fixtures(mods, [int(v) for v in levels[0].split(",")])
        return
    only = [a.split("=", 1)[1] for a in sys.argv if a.startswith("--cases=")]
    if only:
        # regenerate the named cases only: --cases=name1,name2
        for name in only[0].split(","):
            np.savez_compressed(HERE / f"case_{name}.npz", **run_case(name, C.CASES[name], mods))
            print("wrote", name)
        return
    checkpoint_fixture(mods)
    mesh_fixtures(mods)
    for name, case in C.CASES.items():
        np.savez_compressed(HERE / f"case_{name}.npz", **run_case(name, case, mods))
        print("wrote", name)
    # the reference's float32 pin: 80 steps of source_s1 in float32
    pin = dict(C.CASES["source_s1"], steps=80)
    np.savez_compressed(HERE / "case_source_s1_f32x80.npz", **run_case("source_s1_f32", pin, mods, dtype="float32"))
    np.savez_compressed(HERE / "case_source_s1_f64x80.npz", **run_case("source_s1_f64", pin, mods, dtype="float64"))
    # H observations with decimation (solver.py:1138-1229)
    sim = build_reference(C.CASES["source_s1"], mods)
    hr, ht = sim.record_h_observations(
        np.asarray(((0,), (5,)), dtype=np.int64),
        np.asarray(((2,), (4,)), dtype=np.int64),
        np.asarray(((1.0,), (1.0,))),
        np.asarray(((0, 1, 2), (7, 8, 9)), dtype=np.int64),
        np.asarray(((2, 2, 2), (0, 3, 6)), dtype=np.int64),
        np.asarray(((0.2, -0.3, 0.5), (1.0, 0.5, -0.5))),
        11,
        sample_every=3,
    )
    np.savez_compressed(HERE / "obs_h_source_s1.npz", hr=hr, ht=ht)
    receiver_traces_fixture(mods)
    radial_grid_fixture()
    print("done")


if __name__ == "__main__":
    args = [a for a in sys.argv[1:] if not a.startswith("--")]
    if not args:
        sys.exit("usage: make_golden.py <reference src directory> [--cases=a,b | --mesh-levels=7,8,9 | ...]")
    main(args[0])
