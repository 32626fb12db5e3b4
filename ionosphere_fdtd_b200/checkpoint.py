"""Portable, versioned NPZ checkpoints in the reference's layout.

Same keys, dtypes, JSON metadata and validation as the reference
(checkpoint.py:23-477): format ``ionosphere-fdtd-checkpoint`` version 4,
readable back to version 1.  Files written here load in the reference and
vice versa.  Field arrays are copied device-to-host once per field.
"""

from __future__ import annotations

import json
import os
import tempfile
import zipfile
from dataclasses import asdict, replace
from pathlib import Path
from typing import Any

import numpy as np

from .errors import CheckpointError
from .materials import EarthIonosphereMaterial, SphericalAnomaly
from .mesh import build_geodesic_mesh_from_topology, build_geodesic_mesh_from_vertices
from .plasma import MeshPlasmaModel
from .sources import GaussianCurrent, TangentialGaussianCurrent
from .surface_impedance import ConductiveHalfSpaceSurface

CHECKPOINT_FORMAT = "ionosphere-fdtd-checkpoint"
CHECKPOINT_VERSION = 4
SUPPORTED_CHECKPOINT_VERSIONS = (1, 2, 3, CHECKPOINT_VERSION)


def _device_arrays_to_host(tensors: dict[str, Any]) -> dict[str, np.ndarray]:
    """Copy device tensors into pinned host buffers with asynchronous copies on
    the current stream and one synchronisation (instead of a blocking copy per
    array)."""

    import torch

    hosts = {}
    for name, t in tensors.items():
        host = torch.empty(tuple(t.shape), dtype=t.dtype, pin_memory=True)
        host.copy_(t, non_blocking=True)
        hosts[name] = host
    torch.cuda.current_stream().synchronize()
    return {name: h.numpy() for name, h in hosts.items()}


def save_checkpoint(simulation: Any, path: str | Path, *, compress: bool = True) -> Path:
    """Atomically write the NPZ (checkpoint.py:32-93).

    ``compress=False`` writes the same keys, shapes and dtypes without zlib
    compression (a stored zip that ``np.load`` reads like the compressed one),
    for large meshes where compression dominates the save time.  Device arrays
    come to the host through pinned buffers with one synchronisation."""

    destination = Path(path)
    metadata = _metadata(simulation)
    destination.parent.mkdir(parents=True, exist_ok=True)
    ade = simulation._surface_impedance_ade
    device = {f: getattr(simulation, f) for f in ("er", "et", "hr", "ht")}
    if ade is not None:
        device["surface_impedance_memory"] = ade.memory
    if simulation.plasma is not None:
        for i, v in enumerate(simulation._plasma_coupler.ade.current_density):
            device[f"plasma_current_{i}"] = v
    host = _device_arrays_to_host(device)
    arrays = {
        "metadata": np.asarray(json.dumps(metadata, default=_json_default, sort_keys=True)),
        "mesh_vertices": np.asarray(simulation.mesh.vertices, dtype=np.float64),
        "mesh_faces": np.asarray(simulation.mesh.faces, dtype=np.int64),
        "mesh_face_levels": (
            np.asarray(simulation.mesh.face_levels, dtype=np.int64) if simulation.mesh.face_levels is not None else np.empty(0, dtype=np.int64)
        ),
        "er": host["er"],
        "et": host["et"],
        "hr": host["hr"],
        "ht": host["ht"],
        "surface_impedance_memory": host["surface_impedance_memory"] if ade is not None else np.empty((0, 0), dtype=np.float64),
    }
    if simulation.plasma is not None:
        _, plasma_arrays = simulation.plasma.archive_payload()
        arrays.update({f"plasma_model_{n}": v for n, v in plasma_arrays.items()})
        arrays.update({k: v for k, v in host.items() if k.startswith("plasma_current_")})
    temporary = None
    try:
        with tempfile.NamedTemporaryFile(mode="wb", dir=destination.parent, prefix=f".{destination.name}.", delete=False) as handle:
            temporary = handle.name
            (np.savez_compressed if compress else np.savez)(handle, **arrays)
            handle.flush()
            os.fsync(handle.fileno())
        os.replace(temporary, destination)
    finally:
        if temporary is not None and os.path.exists(temporary):
            os.unlink(temporary)
    return destination


def load_checkpoint(
    path: str | Path,
    *,
    backend: str = "torch",
    device: str = "auto",
    dtype: str | None = None,
    compile_step: bool = False,
    compile_chunk_size: int = 8,
    torch_threads: int | None = None,
) -> Any:
    """Restore a checkpoint onto the CUDA engine (checkpoint.py:96-332)."""

    from .solver import GeodesicFDTD, SimulationConfig

    source_path = Path(path)
    try:
        with np.load(source_path, allow_pickle=False) as archive:
            if "metadata" not in archive.files:
                raise CheckpointError("checkpoint is missing arrays: metadata")
            metadata = _read_metadata(archive["metadata"])
            version = metadata["version"]
            required = {"metadata", "mesh_vertices", "er", "et", "hr", "ht"}
            if version >= 2:
                required.update(("mesh_faces", "mesh_face_levels"))
            if version >= 3:
                required.add("surface_impedance_memory")
            plasma_meta = metadata.get("plasma") if version >= 4 else None
            if plasma_meta is not None:
                required.update(f"plasma_model_{n}" for n in plasma_meta["arrays"])
                required.update(f"plasma_current_{i}" for i in range(len(plasma_meta["species"])))
            missing = required.difference(archive.files)
            if missing:
                raise CheckpointError(f"checkpoint is missing arrays: {', '.join(sorted(missing))}")
            vertices = np.array(archive["mesh_vertices"], dtype=np.float64, copy=True)
            faces = np.array(archive["mesh_faces"], copy=True) if version >= 2 else None
            face_levels = np.array(archive["mesh_face_levels"], copy=True) if version >= 2 else None
            fields = {n: np.array(archive[n], copy=True) for n in ("er", "et", "hr", "ht")}
            si_memory = np.array(archive["surface_impedance_memory"], copy=True) if version >= 3 else np.empty((0, 0), dtype=np.float64)
            plasma_arrays = {n: np.array(archive[f"plasma_model_{n}"], copy=True) for n in plasma_meta["arrays"]} if plasma_meta else {}
            plasma_currents = (
                tuple(np.array(archive[f"plasma_current_{i}"], copy=True) for i in range(len(plasma_meta["species"]))) if plasma_meta else ()
            )
    except CheckpointError:
        raise
    except (OSError, ValueError, KeyError, EOFError, zipfile.BadZipFile, json.JSONDecodeError) as error:
        raise CheckpointError(f"cannot read checkpoint {source_path}: {error}") from error

    try:
        config_values = dict(metadata["simulation_config"])
        if config_values["radial_altitudes_m"] is not None:
            config_values["radial_altitudes_m"] = tuple(config_values["radial_altitudes_m"])
        config = SimulationConfig(**config_values)
        if version == 1:
            mesh = build_geodesic_mesh_from_vertices(config.subdivision, vertices, orientation=config.mesh_orientation, normalize_vertices=False)
        else:
            mesh_meta = metadata["mesh"]
            if not isinstance(mesh_meta, dict):
                raise CheckpointError("checkpoint mesh metadata must be an object")
            has_levels = mesh_meta["has_face_levels"]
            if not isinstance(has_levels, bool):
                raise CheckpointError("checkpoint has_face_levels must be boolean")
            if has_levels:
                restored_levels = face_levels
            else:
                if face_levels.shape != (0,):
                    raise CheckpointError("checkpoint has unexpected face-level values")
                restored_levels = None
            mesh = build_geodesic_mesh_from_topology(
                vertices,
                faces,
                subdivision=mesh_meta["subdivision"],
                face_levels=restored_levels,
                refinement_spec=mesh_meta["refinement_spec"],
                topology_kind=mesh_meta["topology_kind"],
                normalize_vertices=False,
                require_well_centered=False,
            )
        material = _deserialize_material(metadata["material"])
        source = _deserialize_source(metadata["source"])
        surface = _deserialize_surface_impedance(metadata["surface_impedance"]) if version >= 3 else None
        plasma = MeshPlasmaModel.from_archive_payload(plasma_meta, plasma_arrays) if plasma_meta is not None else None
    except CheckpointError:
        raise
    except (KeyError, TypeError, ValueError, RuntimeError) as error:
        raise CheckpointError(f"invalid checkpoint model metadata: {error}") from error

    selected_dtype = dtype or str(metadata["runtime"]["dtype"])
    simulation = GeodesicFDTD(
        replace(config, mesh_relaxations=0, mesh_optimization_steps=0),
        material=material,
        source=source,
        surface_impedance=surface,
        plasma=plasma,
        mesh=mesh,
        backend=backend,
        device=device,
        dtype=selected_dtype,
        compile_step=compile_step,
        compile_chunk_size=compile_chunk_size,
        torch_threads=torch_threads,
    )
    simulation.config = config
    for name, values in fields.items():
        expected = tuple(getattr(simulation, name).shape)
        if values.shape != expected:
            raise CheckpointError(f"checkpoint field {name} has shape {values.shape}, expected {expected}")
        if not np.issubdtype(values.dtype, np.floating):
            raise CheckpointError(f"checkpoint field {name} must be floating point")
        if not np.all(np.isfinite(values)):
            raise CheckpointError(f"checkpoint field {name} contains non-finite values")
        setattr(simulation, name, simulation.backend.asarray(values))
    ade = simulation._surface_impedance_ade
    if ade is None:
        if si_memory.shape != (0, 0):
            raise CheckpointError("checkpoint has ADE state without a surface impedance model")
    else:
        if si_memory.shape != tuple(ade.memory.shape):
            raise CheckpointError(f"checkpoint surface impedance state has shape {si_memory.shape}, expected {tuple(ade.memory.shape)}")
        if not np.issubdtype(si_memory.dtype, np.floating) or not np.all(np.isfinite(si_memory)):
            raise CheckpointError("checkpoint surface impedance state is invalid")
        ade.memory = simulation.backend.asarray(si_memory)
    if simulation._plasma_coupler is not None:
        expected_currents = simulation._plasma_coupler.ade.current_density
        if len(plasma_currents) != len(expected_currents):
            raise CheckpointError("checkpoint plasma species state count is invalid")
        for i, (saved, current) in enumerate(zip(plasma_currents, expected_currents, strict=True)):
            if saved.shape != tuple(current.shape):
                raise CheckpointError(f"checkpoint plasma current {i} has shape {saved.shape}, expected {tuple(current.shape)}")
            if not np.issubdtype(saved.dtype, np.floating) or not np.all(np.isfinite(saved)):
                raise CheckpointError(f"checkpoint plasma current {i} is invalid")
            current.copy_(simulation.backend.asarray(saved))
    steps = metadata["state"]["steps"]
    if isinstance(steps, bool) or not isinstance(steps, int) or steps < 0:
        raise CheckpointError("checkpoint step count must be a non-negative integer")
    saved_dt = float(metadata["state"]["time_step_s"])
    if not np.isclose(saved_dt, simulation.time_step_s, rtol=0.0, atol=1.0e-15):
        raise CheckpointError("checkpoint time step is inconsistent with the reconstructed model")
    saved_time = float(metadata["state"]["time_s"])
    expected_time = steps * saved_dt
    if not np.isfinite(saved_time) or not np.isclose(saved_time, expected_time, rtol=1.0e-12, atol=1.0e-15):
        raise CheckpointError("checkpoint time is inconsistent with its step count")
    simulation.steps = steps
    simulation.time_s = expected_time
    return simulation


def _metadata(simulation: Any) -> dict[str, Any]:
    if not isinstance(simulation.material, EarthIonosphereMaterial):
        raise CheckpointError("checkpoints currently support EarthIonosphereMaterial only")
    if simulation.source is not None and not isinstance(simulation.source, (GaussianCurrent, TangentialGaussianCurrent)):
        raise CheckpointError("checkpoints currently support GaussianCurrent and TangentialGaussianCurrent sources only")
    return {
        "format": CHECKPOINT_FORMAT,
        "version": CHECKPOINT_VERSION,
        "simulation_config": asdict(simulation.config),
        "mesh": {
            "topology_kind": simulation.mesh.topology_kind,
            "subdivision": simulation.mesh.subdivision,
            "has_face_levels": simulation.mesh.face_levels is not None,
            "refinement_spec": simulation.mesh.refinement_spec,
        },
        "material": _serialize_material(simulation.material),
        "source": None if simulation.source is None else {"type": type(simulation.source).__name__, "parameters": asdict(simulation.source)},
        "surface_impedance": simulation.surface_impedance.to_metadata() if simulation.surface_impedance is not None else None,
        "plasma": simulation.plasma.archive_payload()[0] if simulation.plasma is not None else None,
        "state": {"steps": simulation.steps, "time_s": simulation.time_s, "time_step_s": simulation.time_step_s},
        "runtime": {
            "backend": simulation.backend.name,
            "device": simulation.backend.device,
            "dtype": simulation.backend.dtype_name,
            "compiled": simulation.compiled,
            "compile_chunk_size": simulation.compile_chunk_size,
        },
    }


def _read_metadata(value: np.ndarray) -> dict[str, Any]:
    if value.shape != () or value.dtype.kind not in {"U", "S"}:
        raise CheckpointError("checkpoint metadata must be a scalar string")
    metadata = json.loads(str(value.item()))
    if not isinstance(metadata, dict):
        raise CheckpointError("checkpoint metadata must be a JSON object")
    if metadata.get("format") != CHECKPOINT_FORMAT:
        raise CheckpointError("file is not an ionosphere-fdtd checkpoint")
    if metadata.get("version") not in SUPPORTED_CHECKPOINT_VERSIONS:
        raise CheckpointError(
            f"unsupported checkpoint version {metadata.get('version')!r}; supported versions are {SUPPORTED_CHECKPOINT_VERSIONS}"
        )
    required = {"simulation_config", "material", "source", "state", "runtime"}
    if metadata["version"] >= 2:
        required.add("mesh")
    if metadata["version"] >= 3:
        required.add("surface_impedance")
    if metadata["version"] >= 4:
        required.add("plasma")
    missing = required.difference(metadata)
    if missing:
        raise CheckpointError(f"checkpoint metadata is missing: {', '.join(sorted(missing))}")
    return metadata


def _serialize_material(material: EarthIonosphereMaterial) -> dict[str, Any]:
    values = asdict(material)
    values["anomalies"] = [asdict(a) for a in material.anomalies]
    return {"type": "EarthIonosphereMaterial", "parameters": values}


def _deserialize_material(data: Any) -> EarthIonosphereMaterial:
    if not isinstance(data, dict) or data.get("type") != "EarthIonosphereMaterial":
        raise CheckpointError("checkpoint material type is unsupported")
    values = dict(data.get("parameters", {}))
    try:
        values["anomalies"] = tuple(SphericalAnomaly(**item) for item in values.get("anomalies", ()))
        return EarthIonosphereMaterial(**values)
    except (TypeError, ValueError) as error:
        raise CheckpointError(f"invalid checkpoint material: {error}") from error


def _deserialize_source(data: Any):
    if data is None:
        return None
    if not isinstance(data, dict):
        raise CheckpointError("checkpoint source metadata must be an object")
    kinds = {"GaussianCurrent": GaussianCurrent, "TangentialGaussianCurrent": TangentialGaussianCurrent}
    try:
        kind = kinds[data["type"]]
        values = dict(data.get("parameters", {}))
        for name in ("azimuths_deg", "line_lengths_m"):
            if name in values and values[name] is not None:
                values[name] = tuple(values[name])
        return kind(**values)
    except (KeyError, TypeError, ValueError) as error:
        raise CheckpointError(f"invalid checkpoint source: {error}") from error


def _deserialize_surface_impedance(data: Any):
    if data is None:
        return None
    if not isinstance(data, dict):
        raise CheckpointError("checkpoint surface impedance metadata must be an object")
    try:
        return ConductiveHalfSpaceSurface.from_metadata(data)
    except (KeyError, TypeError, ValueError) as error:
        raise CheckpointError(f"invalid checkpoint surface impedance: {error}") from error


def _json_default(value: Any) -> Any:
    if isinstance(value, np.generic):
        return value.item()
    raise TypeError(f"cannot encode {type(value).__name__} in checkpoint metadata")
