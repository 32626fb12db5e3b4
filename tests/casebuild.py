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


def build_oracle(case: dict, dtype=np.float64):
    import oracle.fdtd as O

    cfg = dict(case["config"])
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
