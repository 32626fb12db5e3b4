"""Portable, versioned NPZ checkpoints in the reference's file layout.

The file is the reference's (``checkpoint.py:23-477``): format
``ionosphere-fdtd-checkpoint`` version 4, readable back to version 1, the same
archive keys, dtypes, JSON metadata schema and error messages, so files
written here load in the reference and vice versa.

The code is organised around one declarative table, ``ARCHIVE``: every array
of the archive is an ``Entry`` naming its key, the first format version that
carries it, where its value comes from when writing, and, for the state
arrays, how it is checked and restored when reading.  ``save_checkpoint``
walks the table once to gather arrays (device arrays reach the host through
pinned buffers with a single synchronisation); ``load_checkpoint`` walks it
to find the keys a file of its version must hold, to read them, and, after
the model is rebuilt from the metadata, to validate and restore the state.
"""

from __future__ import annotations

import contextlib
import json
import os
import tempfile
import zipfile
from dataclasses import asdict, dataclass, replace
from pathlib import Path
from typing import Any, Iterator

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

# Metadata sections and the first format version that requires each.
METADATA_SECTIONS = {
    "simulation_config": 1, "material": 1, "source": 1, "state": 1, "runtime": 1,
    "mesh": 2, "surface_impedance": 3, "plasma": 4,
}

SOURCE_TYPES = {"GaussianCurrent": GaussianCurrent, "TangentialGaussianCurrent": TangentialGaussianCurrent}


# ---------------------------------------------------------------------------
# The archive table
# ---------------------------------------------------------------------------


@dataclass(frozen=True)
class Entry:
    """One array of the archive.

    ``key``: archive key; entries of one per plasma species or model array
    carry ``{}`` and are expanded by ``keys_for``.  ``since``: first format
    version that carries it.  ``group``: how it is produced and consumed
    (``mesh``, ``field``, ``surface``, ``plasma_model``, ``plasma_current``).
    ``what``: its name in validation messages."""

    key: str
    since: int
    group: str
    what: str = ""


ARCHIVE: tuple[Entry, ...] = (
    Entry("metadata", 1, "metadata"),
    Entry("mesh_vertices", 1, "mesh"),
    Entry("mesh_faces", 2, "mesh"),
    Entry("mesh_face_levels", 2, "mesh"),
    Entry("er", 1, "field", "er"),
    Entry("et", 1, "field", "et"),
    Entry("hr", 1, "field", "hr"),
    Entry("ht", 1, "field", "ht"),
    Entry("surface_impedance_memory", 3, "surface", "surface impedance state"),
    Entry("plasma_model_{}", 4, "plasma_model"),
    Entry("plasma_current_{}", 4, "plasma_current", "plasma current {}"),
)


def keys_for(entry: Entry, plasma_meta: dict | None) -> list[str]:
    """The archive keys of one table entry for a file with this plasma metadata."""

    if entry.group == "plasma_model":
        return [entry.key.format(n) for n in plasma_meta["arrays"]] if plasma_meta else []
    if entry.group == "plasma_current":
        return [entry.key.format(i) for i in range(len(plasma_meta["species"]))] if plasma_meta else []
    return [entry.key]


def required_keys(version: int, plasma_meta: dict | None) -> set[str]:
    """Every archive key a file of ``version`` must hold."""

    return {k for e in ARCHIVE if version >= e.since for k in keys_for(e, plasma_meta)}


# ---------------------------------------------------------------------------
# Writing
# ---------------------------------------------------------------------------


def _to_host(tensors: dict[str, Any]) -> dict[str, np.ndarray]:
    """Device tensors to pinned host arrays: asynchronous copies on the current
    stream, then one synchronisation."""

    import torch

    pinned = {}
    for key, t in tensors.items():
        pinned[key] = torch.empty(tuple(t.shape), dtype=t.dtype, pin_memory=True)
        pinned[key].copy_(t, non_blocking=True)
    torch.cuda.current_stream().synchronize()
    return {key: p.numpy() for key, p in pinned.items()}


def _entry_values(entry: Entry, sim: Any, payload: tuple | None) -> tuple[dict[str, Any], dict[str, Any]]:
    """(host arrays, device tensors) that ``entry`` stores for ``sim``; ``payload``
    is the plasma model's (metadata, arrays) archive payload or None."""

    mesh = sim.mesh
    if entry.group == "metadata":
        meta = _metadata(sim, payload[0] if payload else None)
        return {entry.key: np.asarray(json.dumps(meta, default=_json_default, sort_keys=True))}, {}
    if entry.group == "mesh":
        value = {
            "mesh_vertices": lambda: np.asarray(mesh.vertices, dtype=np.float64),
            "mesh_faces": lambda: np.asarray(mesh.faces, dtype=np.int64),
            "mesh_face_levels": lambda: np.asarray(mesh.face_levels if mesh.face_levels is not None else (), dtype=np.int64),
        }[entry.key]()
        return {entry.key: value}, {}
    if entry.group == "field":
        return {}, {entry.key: getattr(sim, entry.key)}
    if entry.group == "surface":
        ade = sim._surface_impedance_ade
        return ({}, {entry.key: ade.memory}) if ade is not None else ({entry.key: np.empty((0, 0), dtype=np.float64)}, {})
    if payload is None:
        return {}, {}
    if entry.group == "plasma_model":
        return {entry.key.format(n): v for n, v in payload[1].items()}, {}
    currents = sim._plasma_coupler.ade.current_density
    return {}, {entry.key.format(i): c for i, c in enumerate(currents)}


@contextlib.contextmanager
def _replacing(destination: Path) -> Iterator[Any]:
    """A temporary file beside ``destination`` that replaces it atomically once
    written and flushed to disk; removed if writing fails."""

    fd, name = tempfile.mkstemp(dir=destination.parent, prefix=f".{destination.name}.")
    try:
        with os.fdopen(fd, "wb") as handle:
            yield handle
            handle.flush()
            os.fsync(handle.fileno())
        os.replace(name, destination)
    finally:
        if os.path.exists(name):
            os.unlink(name)


def save_checkpoint(simulation: Any, path: str | Path, *, compress: bool = True) -> Path:
    """Atomically write the simulation's checkpoint (the reference's
    ``save_checkpoint``, checkpoint.py:32-93).

    ``compress=False`` writes the same keys, shapes and dtypes without zlib
    compression (a stored zip that ``np.load`` reads like the compressed one),
    for large meshes where compression dominates the save time."""

    destination = Path(path)
    payload = simulation.plasma.archive_payload() if simulation.plasma is not None else None
    host: dict[str, Any] = {}
    device: dict[str, Any] = {}
    for entry in ARCHIVE:
        h, d = _entry_values(entry, simulation, payload)
        host.update(h)
        device.update(d)
    host.update(_to_host(device))
    arrays = {k: host[k] for e in ARCHIVE for k in keys_for(e, payload[0] if payload else None)}
    destination.parent.mkdir(parents=True, exist_ok=True)
    with _replacing(destination) as handle:
        (np.savez_compressed if compress else np.savez)(handle, **arrays)
    return destination


# ---------------------------------------------------------------------------
# Reading
# ---------------------------------------------------------------------------


def _read_archive(path: Path) -> tuple[dict[str, Any], dict[str, np.ndarray]]:
    """The metadata and every array the file's version requires (copied out)."""

    try:
        with np.load(path, allow_pickle=False) as archive:
            if "metadata" not in archive.files:
                raise CheckpointError("checkpoint is missing arrays: metadata")
            metadata = _read_metadata(archive["metadata"])
            plasma_meta = metadata.get("plasma") if metadata["version"] >= 4 else None
            wanted = required_keys(metadata["version"], plasma_meta) - {"metadata"}
            missing = wanted.difference(archive.files)
            if missing:
                raise CheckpointError(f"checkpoint is missing arrays: {', '.join(sorted(missing))}")
            return metadata, {k: np.array(archive[k], copy=True) for k in wanted}
    except CheckpointError:
        raise
    except (OSError, ValueError, KeyError, EOFError, zipfile.BadZipFile, json.JSONDecodeError) as error:
        raise CheckpointError(f"cannot read checkpoint {path}: {error}") from error


def _read_metadata(value: np.ndarray) -> dict[str, Any]:
    if value.shape != () or value.dtype.kind not in {"U", "S"}:
        raise CheckpointError("checkpoint metadata must be a scalar string")
    metadata = json.loads(str(value.item()))
    if not isinstance(metadata, dict):
        raise CheckpointError("checkpoint metadata must be a JSON object")
    if metadata.get("format") != CHECKPOINT_FORMAT:
        raise CheckpointError("file is not an ionosphere-fdtd checkpoint")
    version = metadata.get("version")
    if version not in SUPPORTED_CHECKPOINT_VERSIONS:
        raise CheckpointError(f"unsupported checkpoint version {version!r}; supported versions are {SUPPORTED_CHECKPOINT_VERSIONS}")
    missing = {name for name, since in METADATA_SECTIONS.items() if version >= since}.difference(metadata)
    if missing:
        raise CheckpointError(f"checkpoint metadata is missing: {', '.join(sorted(missing))}")
    return metadata


def _mesh_from(metadata: dict, arrays: dict, config: Any):
    """The mesh: rebuilt from the vertices alone (version 1) or from the stored
    topology and refinement metadata (version 2 on)."""

    vertices = np.asarray(arrays["mesh_vertices"], dtype=np.float64)
    if metadata["version"] == 1:
        return build_geodesic_mesh_from_vertices(config.subdivision, vertices, orientation=config.mesh_orientation, normalize_vertices=False)
    about = metadata["mesh"]
    if not isinstance(about, dict):
        raise CheckpointError("checkpoint mesh metadata must be an object")
    if not isinstance(about["has_face_levels"], bool):
        raise CheckpointError("checkpoint has_face_levels must be boolean")
    levels = arrays["mesh_face_levels"]
    if not about["has_face_levels"]:
        if levels.shape != (0,):
            raise CheckpointError("checkpoint has unexpected face-level values")
        levels = None
    return build_geodesic_mesh_from_topology(
        vertices, arrays["mesh_faces"], subdivision=about["subdivision"], face_levels=levels,
        refinement_spec=about["refinement_spec"], topology_kind=about["topology_kind"],
        normalize_vertices=False, require_well_centered=False,
    )


def _config_from(metadata: dict):
    from .solver import SimulationConfig

    values = dict(metadata["simulation_config"])
    if values["radial_altitudes_m"] is not None:
        values["radial_altitudes_m"] = tuple(values["radial_altitudes_m"])
    return SimulationConfig(**values)


def _model_from(metadata: dict, arrays: dict) -> dict[str, Any]:
    """Configuration, mesh and physics models described by the metadata."""

    version = metadata["version"]
    try:
        config = _config_from(metadata)
        plasma_meta = metadata["plasma"] if version >= 4 else None
        plasma_arrays = {n: arrays[f"plasma_model_{n}"] for n in plasma_meta["arrays"]} if plasma_meta else {}
        return {
            "config": config,
            "mesh": _mesh_from(metadata, arrays, config),
            "material": _material_from(metadata["material"]),
            "source": _source_from(metadata["source"]),
            "surface_impedance": _surface_from(metadata["surface_impedance"]) if version >= 3 else None,
            "plasma": MeshPlasmaModel.from_archive_payload(plasma_meta, plasma_arrays) if plasma_meta is not None else None,
        }
    except CheckpointError:
        raise
    except (KeyError, TypeError, ValueError, RuntimeError) as error:
        raise CheckpointError(f"invalid checkpoint model metadata: {error}") from error


def _checked_state(what: str, saved: np.ndarray, expected: tuple, *, check_dtype_first: bool) -> None:
    """The shape, dtype and finiteness checks of one restored state array."""

    if saved.shape != expected:
        raise CheckpointError(f"checkpoint {what} has shape {saved.shape}, expected {expected}")
    if check_dtype_first:
        if not np.issubdtype(saved.dtype, np.floating):
            raise CheckpointError(f"checkpoint {what} must be floating point")
        if not np.all(np.isfinite(saved)):
            raise CheckpointError(f"checkpoint {what} contains non-finite values")
    elif not np.issubdtype(saved.dtype, np.floating) or not np.all(np.isfinite(saved)):
        raise CheckpointError(f"checkpoint {what} is invalid")


def _restore(entry: Entry, sim: Any, arrays: dict[str, np.ndarray], version: int) -> None:
    """Validate and restore the state arrays of one table entry."""

    b = sim.backend
    if entry.group == "field":
        saved = arrays[entry.key]
        _checked_state(f"field {entry.what}", saved, tuple(getattr(sim, entry.key).shape), check_dtype_first=True)
        setattr(sim, entry.key, b.asarray(saved))
    elif entry.group == "surface":
        saved = arrays[entry.key] if version >= entry.since else np.empty((0, 0), dtype=np.float64)
        ade = sim._surface_impedance_ade
        if ade is None:
            if saved.shape != (0, 0):
                raise CheckpointError("checkpoint has ADE state without a surface impedance model")
            return
        _checked_state(entry.what, saved, tuple(ade.memory.shape), check_dtype_first=False)
        ade.memory = b.asarray(saved)
    elif entry.group == "plasma_current" and sim._plasma_coupler is not None:
        targets = sim._plasma_coupler.ade.current_density
        saved = [arrays[k] for k in sorted((k for k in arrays if k.startswith("plasma_current_")), key=lambda k: int(k.rsplit("_", 1)[1]))]
        if len(saved) != len(targets):
            raise CheckpointError("checkpoint plasma species state count is invalid")
        for i, (values, target) in enumerate(zip(saved, targets, strict=True)):
            _checked_state(entry.what.format(i), values, tuple(target.shape), check_dtype_first=False)
            target.copy_(b.asarray(values))


def _restore_clock(sim: Any, state: dict) -> None:
    """Step count, time step and time of the saved state (checked against the
    rebuilt model's time step)."""

    steps = state["steps"]
    if isinstance(steps, bool) or not isinstance(steps, int) or steps < 0:
        raise CheckpointError("checkpoint step count must be a non-negative integer")
    dt = float(state["time_step_s"])
    if not np.isclose(dt, sim.time_step_s, rtol=0.0, atol=1.0e-15):
        raise CheckpointError("checkpoint time step is inconsistent with the reconstructed model")
    t = float(state["time_s"])
    if not np.isfinite(t) or not np.isclose(t, steps * dt, rtol=1.0e-12, atol=1.0e-15):
        raise CheckpointError("checkpoint time is inconsistent with its step count")
    sim.steps = steps
    sim.time_s = steps * dt


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
    """Restore a checkpoint onto the CUDA engine (the reference's
    ``load_checkpoint``, checkpoint.py:96-332)."""

    from .solver import GeodesicFDTD

    metadata, arrays = _read_archive(Path(path))
    model = _model_from(metadata, arrays)
    config = model.pop("config")
    sim = GeodesicFDTD(
        replace(config, mesh_relaxations=0, mesh_optimization_steps=0),
        **model,
        backend=backend,
        device=device,
        dtype=dtype or str(metadata["runtime"]["dtype"]),
        compile_step=compile_step,
        compile_chunk_size=compile_chunk_size,
        torch_threads=torch_threads,
    )
    sim.config = config
    for entry in ARCHIVE:
        _restore(entry, sim, arrays, metadata["version"])
    _restore_clock(sim, metadata["state"])
    return sim


# ---------------------------------------------------------------------------
# Metadata (the reference's JSON schema)
# ---------------------------------------------------------------------------


def _metadata(sim: Any, plasma_meta: dict | None) -> dict[str, Any]:
    if not isinstance(sim.material, EarthIonosphereMaterial):
        raise CheckpointError("checkpoints currently support EarthIonosphereMaterial only")
    if sim.source is not None and not isinstance(sim.source, tuple(SOURCE_TYPES.values())):
        raise CheckpointError("checkpoints currently support GaussianCurrent and TangentialGaussianCurrent sources only")
    mesh = sim.mesh
    material = asdict(sim.material)
    material["anomalies"] = [asdict(a) for a in sim.material.anomalies]
    return {
        "format": CHECKPOINT_FORMAT,
        "version": CHECKPOINT_VERSION,
        "simulation_config": asdict(sim.config),
        "mesh": {
            "topology_kind": mesh.topology_kind,
            "subdivision": mesh.subdivision,
            "has_face_levels": mesh.face_levels is not None,
            "refinement_spec": mesh.refinement_spec,
        },
        "material": {"type": "EarthIonosphereMaterial", "parameters": material},
        "source": None if sim.source is None else {"type": type(sim.source).__name__, "parameters": asdict(sim.source)},
        "surface_impedance": sim.surface_impedance.to_metadata() if sim.surface_impedance is not None else None,
        "plasma": plasma_meta,
        "state": {"steps": sim.steps, "time_s": sim.time_s, "time_step_s": sim.time_step_s},
        "runtime": {
            "backend": sim.backend.name,
            "device": sim.backend.device,
            "dtype": sim.backend.dtype_name,
            "compiled": sim.compiled,
            "compile_chunk_size": sim.compile_chunk_size,
        },
    }


def _material_from(data: Any) -> EarthIonosphereMaterial:
    if not isinstance(data, dict) or data.get("type") != "EarthIonosphereMaterial":
        raise CheckpointError("checkpoint material type is unsupported")
    values = dict(data.get("parameters", {}))
    try:
        values["anomalies"] = tuple(SphericalAnomaly(**item) for item in values.get("anomalies", ()))
        return EarthIonosphereMaterial(**values)
    except (TypeError, ValueError) as error:
        raise CheckpointError(f"invalid checkpoint material: {error}") from error


def _source_from(data: Any):
    if data is None:
        return None
    if not isinstance(data, dict):
        raise CheckpointError("checkpoint source metadata must be an object")
    try:
        kind = SOURCE_TYPES[data["type"]]
        values = {k: tuple(v) if k in ("azimuths_deg", "line_lengths_m") and v is not None else v
                  for k, v in dict(data.get("parameters", {})).items()}
        return kind(**values)
    except (KeyError, TypeError, ValueError) as error:
        raise CheckpointError(f"invalid checkpoint source: {error}") from error


def _surface_from(data: Any):
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


__all__ = ["ARCHIVE", "CHECKPOINT_FORMAT", "CHECKPOINT_VERSION", "Entry", "SUPPORTED_CHECKPOINT_VERSIONS",
           "load_checkpoint", "required_keys", "save_checkpoint"]
