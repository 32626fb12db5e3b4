"""Build the oracle and the CUDA engine from one parity case (see golden/cases.py)."""

from __future__ import annotations

from pathlib import Path

import numpy as np

import cases as C

GOLDEN = Path(__file__).resolve().parent / "golden"


def golden(name: str) -> dict[str, np.ndarray]:
    with np.load(GOLDEN / f"{name}.npz", allow_pickle=False) as archive:
        return {key: np.array(archive[key]) for key in archive.files}


def _material_for_oracle(spec):
    import oracle.fdtd as O

    if spec == "default":
        return O.EarthIonosphereParams()
    if spec == "profile":
        return C.ProfileMaterial()
    if spec == "patchy":
        return C.PatchyMaterial()
    return O.EarthIonosphereParams(**spec[1])


def _midpoint_altitudes(cfg: dict) -> np.ndarray:
    alt = np.asarray(
        cfg.get("radial_altitudes_m")
        or np.linspace(cfg.get("minimum_altitude_m", -100_000.0), cfg.get("maximum_altitude_m", 100_000.0), cfg["radial_cells"] + 1)
    )
    return 0.5 * (alt[:-1] + alt[1:])


def plasma_arrays(spec: dict, n_faces: int, cfg: dict):
    mids = _midpoint_altitudes(cfg)
    shape = (n_faces, len(mids))
    if spec["kind"] == "profile":
        magnetic, density, collision = C.profile_plasma_arrays(n_faces, mids, spec["magnetic_t"])
    else:
        magnetic = np.zeros((*shape, 3))
        magnetic[..., 2] = spec["magnetic_t"]
        density = np.full(shape, spec["density_m3"])
        collision = np.full(shape, spec["collision_hz"])
    qe = 1.602_176_634e-19
    me = 9.109_383_713_9e-31
    species = [(-qe, me, density, collision)]
    if spec.get("two_species"):
        species.append((qe, 16 * 1.672_621_925_95e-27, 0.5 * density, 0.1 * collision))
    return mids, magnetic, species


def adaptive_mesh(case: dict):
    """The package's locally refined mesh of an adaptive case."""

    import ionosphere_fdtd_b200 as P
    from ionosphere_fdtd_b200.adaptive_mesh import SphericalRefinementRegion, build_adaptive_geodesic_mesh

    base, regions = case["adaptive"]
    return build_adaptive_geodesic_mesh(base, tuple(SphericalRefinementRegion(*r) for r in regions))


def build_oracle(case: dict, dtype=np.float64):
    import oracle.fdtd as O

    cfg = dict(case["config"])
    if "adaptive" in case:
        # the refined vertices and faces come from the package's builder, pinned
        # bit for bit to the reference's by tests/test_adaptive_cpu.py
        m = adaptive_mesh(case)
        mesh = O.assemble_mesh(np.array(m.vertices), np.array(m.faces), m.subdivision)
    else:
        mesh = O.build_mesh(cfg["subdivision"])
    kwargs = dict(
        subdivision=cfg["subdivision"],
        radial_cells=cfg["radial_cells"],
        minimum_altitude_m=cfg.get("minimum_altitude_m", -100_000.0),
        maximum_altitude_m=cfg.get("maximum_altitude_m", 100_000.0),
        earth_radius_m=cfg.get("earth_radius_m", O.EARTH_RADIUS_M),
        courant_factor=cfg.get("courant_factor", 0.35),
        radial_altitudes_m=cfg.get("radial_altitudes_m"),
        geometry_mode=cfg.get("geometry_mode", "full-spherical"),
        loss_integration=cfg.get("loss_integration", "exponential"),
        material=_material_for_oracle(case.get("material", "default")),
        mesh=mesh,
        dtype=dtype,
    )
    spec = case.get("source")
    if spec is not None:
        spec = dict(spec)
        kind = spec.pop("kind")
        if "seed_vertex" in spec:
            lat, lon = C.vertex_lat_lon(mesh.vertices, C.source_vertex(mesh.n_vertices, spec.pop("seed_vertex")))
            spec.update(latitude_deg=lat, longitude_deg=lon)
        if kind == "tangential":
            spec.setdefault("altitude_m", 0.0)
        kwargs["source"] = O.OracleSource(tangential=(kind == "tangential"), **spec)
    sspec = case.get("surface")
    if sspec is not None:
        sigma = sspec["value"] if sspec["conductivity"] == "scalar" else C.smooth_log_normal(mesh.edge_midpoints(), sspec["seed"])
        kwargs["surface"] = O.OracleSurface(sigma)
    pspec = case.get("plasma")
    if pspec is not None:
        _, magnetic, species = plasma_arrays(pspec, mesh.n_faces, cfg)
        kwargs["plasma"] = O.OraclePlasma(magnetic, [O.OracleSpecies(*s) for s in species])
    sim = O.OracleFDTD(**kwargs)
    init = case.get("init")
    if init is not None:
        shapes = {n: getattr(sim, n).shape for n in ("er", "et", "hr", "ht")}
        for n, v in C.initial_fields(shapes, *init).items():
            getattr(sim, n)[:] = v
    return sim


def run_oracle(case: dict, dtype=np.float64) -> dict[str, np.ndarray]:
    sim = build_oracle(case, dtype)
    out = {"time_step_s": np.asarray(sim.dt), "cfl_limit_s": np.asarray(sim.cfl_limit_s)}
    rspec = case.get("receivers")
    if rspec is not None:
        v, k, w = C.receiver_rows(sim.mesh.n_vertices, sim.altitudes_m, rspec["seed"], rspec["count"])
        out["traces"] = sim.record_er(v, k, w, case["steps"])
    else:
        sim.step(case["steps"])
    for f in ("er", "et", "hr", "ht"):
        out[f] = getattr(sim, f)
    if sim.surface is not None:
        out["si_memory"] = sim.si_memory
    if sim.plasma is not None:
        for i, j in enumerate(sim.p_current):
            out[f"plasma_current_{i}"] = j
    return out


def rel_l2(actual, expected) -> float:
    a = np.asarray(actual, dtype=np.float64).ravel()
    e = np.asarray(expected, dtype=np.float64).ravel()
    n = np.linalg.norm(e)
    return float(np.linalg.norm(a - e) / n) if n > 0 else float(np.linalg.norm(a - e))


def grouped_rel_l2(actual: dict, expected: dict) -> dict[str, float]:
    """Relative L2 per (E, H) group, as the reference's FP32 pin groups them."""

    out = {}
    for group in (("er", "et"), ("hr", "ht")):
        a = np.concatenate([np.asarray(actual[f], dtype=np.float64).ravel() for f in group])
        e = np.concatenate([np.asarray(expected[f], dtype=np.float64).ravel() for f in group])
        out["".join(group)] = rel_l2(a, e)
    return out


def product_provenance():
    from ionosphere_fdtd_b200 import DatasetProvenance, VariableProvenance

    return DatasetProvenance(
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
            VariableProvenance("B", "T", "T", "identity"),
            VariableProvenance("number_density", "m^-3", "m^-3", "identity"),
            VariableProvenance("collision_frequency", "Hz", "Hz", "identity"),
        ),
    )


def build_product(case: dict, dtype: str = "float64", **kwargs):
    """The CUDA engine (GeodesicFDTD of ionosphere_fdtd_b200) for a parity case."""

    import ionosphere_fdtd_b200 as P

    cfg = P.SimulationConfig(**case["config"])
    mesh = adaptive_mesh(case) if "adaptive" in case else P.build_geodesic_mesh(cfg.subdivision)
    mat = case.get("material", "default")
    if mat == "default":
        material = None
    elif mat == "profile":
        material = C.ProfileMaterial()
    elif mat == "patchy":
        material = C.PatchyMaterial()
    else:
        material = P.EarthIonosphereMaterial(**mat[1])
    source = None
    spec = case.get("source")
    if spec is not None:
        spec = dict(spec)
        kind = spec.pop("kind")
        if "seed_vertex" in spec:
            lat, lon = C.vertex_lat_lon(mesh.vertices, C.source_vertex(mesh.n_vertices, spec.pop("seed_vertex")))
            spec.update(latitude_deg=lat, longitude_deg=lon)
        source = (P.TangentialGaussianCurrent if kind == "tangential" else P.GaussianCurrent)(**spec)
    surface = None
    sspec = case.get("surface")
    if sspec is not None:
        sigma = sspec["value"] if sspec["conductivity"] == "scalar" else C.smooth_log_normal(mesh.edge_midpoints(), sspec["seed"])
        surface = P.ConductiveHalfSpaceSurface(sigma)
    plasma = None
    pspec = case.get("plasma")
    if pspec is not None:
        mids, magnetic, species = plasma_arrays(pspec, mesh.n_faces, case["config"])
        names = ["electron", "O+"]
        plasma = P.MeshPlasmaModel.from_mesh(
            mesh,
            mids,
            magnetic,
            tuple(P.ColdPlasmaSpecies(names[i], q, m, n, nu) for i, (q, m, n, nu) in enumerate(species)),
            provenance=(product_provenance(),),
            interpolation="synthetic",
        )
    sim = P.GeodesicFDTD(
        cfg, material=material, source=source, surface_impedance=surface, plasma=plasma, mesh=mesh,
        backend="torch", device="cuda", dtype=dtype, **kwargs,
    )
    init = case.get("init")
    if init is not None:
        shapes = {n: tuple(getattr(sim, n).shape) for n in ("er", "et", "hr", "ht")}
        for n, v in C.initial_fields(shapes, *init).items():
            getattr(sim, n).copy_(sim.backend.asarray(v))
    return sim


def run_product(case: dict, dtype: str = "float64", **kwargs) -> dict[str, np.ndarray]:
    sim = build_product(case, dtype, **kwargs)
    out = {"time_step_s": np.asarray(sim.time_step_s), "cfl_limit_s": np.asarray(sim.cfl_time_step_limit_s)}
    rspec = case.get("receivers")
    if rspec is not None:
        v, k, w = C.receiver_rows(sim.mesh.n_vertices, sim.altitudes_m, rspec["seed"], rspec["count"])
        out["traces"] = sim.record_er_observations(v, k, w, case["steps"])
    else:
        sim.step(case["steps"])
    for f in ("er", "et", "hr", "ht"):
        out[f] = sim.to_numpy(getattr(sim, f))
    if sim._surface_impedance_ade is not None:
        out["si_memory"] = sim.to_numpy(sim._surface_impedance_ade.memory)
    if sim._plasma_coupler is not None:
        for i, j in enumerate(sim._plasma_coupler.ade.current_density):
            out[f"plasma_current_{i}"] = sim.to_numpy(j)
    out["_sim"] = sim
    return out
