"""Magnetised cold-plasma model, ADE coefficients and mesh coupling tables.

Same model, artifact format, coefficients and coupling geometry as the
reference (plasma.py:32-602).  The ADE update and the face-vector
reconstruction / scatter run inside the CUDA step kernels; this module
builds their inputs:

* per-species ADE coefficients (decay, cos, sin, d_par, d_re, d_im) on
  faces x radial midpoints, stored as one altitude row when the inputs are
  horizontally uniform (the reduction is exact: identical rows give
  identical coefficients);
* the per-face reconstruction ``pinv(tangents).T``, edge tangents within
  the left/right faces and the area-weighted vertex-face table, computed
  with array operations instead of the reference's per-face loops.
"""

from __future__ import annotations

import hashlib
import json
import os
import tempfile
from concurrent.futures import ThreadPoolExecutor
from dataclasses import asdict, dataclass
from pathlib import Path
from typing import Any

import numpy as np
from numpy.typing import NDArray

from .provenance import (
    DatasetProvenance,
    VariableProvenance,
    array_sha256,
    distinct_elements,
    mesh_faces_sha256,
    mesh_vertices_sha256,
)

ELEMENTARY_CHARGE_C = 1.602_176_634e-19
ELECTRON_MASS_KG = 9.109_383_713_9e-31
MESH_PLASMA_FORMAT = "ionosphere-fdtd-mesh-plasma"
MESH_PLASMA_VERSION = 1


def _readonly(values) -> NDArray[np.float64]:
    """Read-only float64 copy; horizontally broadcast inputs stay views."""

    array = np.asarray(values, dtype=np.float64)
    if array.ndim >= 1 and array.shape[0] > 1 and array.strides[0] == 0:
        view = array.view()
        view.setflags(write=False)
        return view
    out = np.array(array, dtype=np.float64, order="C", copy=True)
    out.setflags(write=False)
    return out


def horizontally_uniform(values: NDArray[np.float64]) -> bool:
    """True when every face row equals the first (exact comparison)."""

    a = np.asarray(values)
    if a.shape[0] <= 1 or a.strides[0] == 0:
        return True
    return bool(np.array_equal(a, np.broadcast_to(a[:1], a.shape)))


@dataclass(frozen=True, slots=True)
class ColdPlasmaSpecies:
    """One charged fluid sampled at face / radial-cell centres."""

    name: str
    charge_c: float
    mass_kg: float
    number_density_m3: NDArray[np.float64]
    collision_frequency_hz: NDArray[np.float64]

    def __post_init__(self) -> None:
        if not isinstance(self.name, str) or not self.name.strip():
            raise ValueError("plasma species name must be nonempty")
        if not np.isfinite(self.charge_c) or self.charge_c == 0.0:
            raise ValueError("plasma species charge must be finite and nonzero")
        if not np.isfinite(self.mass_kg) or self.mass_kg <= 0.0:
            raise ValueError("plasma species mass must be finite and positive")
        density = np.asarray(self.number_density_m3, dtype=np.float64)
        collision = np.asarray(self.collision_frequency_hz, dtype=np.float64)
        if density.ndim != 2 or collision.shape != density.shape:
            raise ValueError("plasma density and collision grids must have one shape")
        d_core, c_core = distinct_elements(density), distinct_elements(collision)
        if not np.all(np.isfinite(d_core)) or np.any(d_core < 0.0) or not np.all(np.isfinite(c_core)) or np.any(c_core <= 0.0):
            raise ValueError("plasma density/collision values are invalid")
        object.__setattr__(self, "number_density_m3", _readonly(density))
        object.__setattr__(self, "collision_frequency_hz", _readonly(collision))


@dataclass(frozen=True, slots=True)
class MeshPlasmaModel:
    """Magnetic field and charged fluids bound to one mesh and radial grid."""

    mesh_vertices_sha256: str
    mesh_faces_sha256: str
    radial_midpoint_altitudes_m: NDArray[np.float64]
    magnetic_field_t: NDArray[np.float64]
    species: tuple[ColdPlasmaSpecies, ...]
    provenance: tuple[DatasetProvenance, ...]
    interpolation: str

    def __post_init__(self) -> None:
        alt = np.asarray(self.radial_midpoint_altitudes_m, dtype=np.float64)
        magnetic = np.asarray(self.magnetic_field_t, dtype=np.float64)
        species = tuple(self.species)
        if alt.ndim != 1 or len(alt) < 1 or not np.all(np.isfinite(alt)) or not np.all(np.diff(alt) > 0.0):
            raise ValueError("plasma radial midpoints must be finite and increasing")
        if magnetic.ndim != 3 or magnetic.shape[1:] != (len(alt), 3):
            raise ValueError("magnetic field must have shape (face, radial, 3)")
        if not np.all(np.isfinite(distinct_elements(magnetic))):
            raise ValueError("magnetic field must be finite")
        if not species or not all(isinstance(s, ColdPlasmaSpecies) for s in species):
            raise ValueError("plasma model requires charged species")
        if any(s.number_density_m3.shape != magnetic.shape[:2] for s in species):
            raise ValueError("plasma species grids must match the magnetic grid")
        names = [s.name for s in species]
        if len(set(names)) != len(names):
            raise ValueError("plasma species names must be unique")
        provenance = tuple(self.provenance)
        if not provenance or not all(isinstance(p, DatasetProvenance) for p in provenance):
            raise ValueError("plasma model requires dataset provenance")
        if not isinstance(self.interpolation, str) or not self.interpolation.strip():
            raise ValueError("plasma interpolation policy must be nonempty")
        object.__setattr__(self, "radial_midpoint_altitudes_m", _readonly(alt))
        object.__setattr__(self, "magnetic_field_t", _readonly(magnetic))
        object.__setattr__(self, "species", species)
        object.__setattr__(self, "provenance", provenance)

    @classmethod
    def from_mesh(cls, mesh, radial_midpoint_altitudes_m, magnetic_field_t, species, *, provenance, interpolation) -> "MeshPlasmaModel":
        return cls(
            mesh_vertices_sha256=mesh_vertices_sha256(mesh),
            mesh_faces_sha256=mesh_faces_sha256(mesh),
            radial_midpoint_altitudes_m=radial_midpoint_altitudes_m,
            magnetic_field_t=magnetic_field_t,
            species=tuple(species),
            provenance=tuple(provenance),
            interpolation=interpolation,
        )

    def validate_grid(self, mesh, radial_midpoint_altitudes_m) -> None:
        if mesh_vertices_sha256(mesh) != self.mesh_vertices_sha256:
            raise ValueError("plasma model mesh vertices do not match")
        if mesh_faces_sha256(mesh) != self.mesh_faces_sha256:
            raise ValueError("plasma model mesh faces do not match")
        if not np.array_equal(radial_midpoint_altitudes_m, self.radial_midpoint_altitudes_m):
            raise ValueError("plasma model radial grid does not match")
        if self.magnetic_field_t.shape[0] != mesh.n_faces:
            raise ValueError("plasma model face count does not match")

    def conductivity_components(self, frequency_hz: float):
        """Summed parallel, Pedersen and Hall conductivities (exp(+i w t))."""

        if not np.isfinite(frequency_hz) or frequency_hz < 0.0:
            raise ValueError("plasma response frequency must be nonnegative")
        shape = self.magnetic_field_t.shape[:2]
        parallel = np.zeros(shape, dtype=np.complex128)
        pedersen = np.zeros_like(parallel)
        hall = np.zeros_like(parallel)
        bmag = np.linalg.norm(self.magnetic_field_t, axis=2)
        w = 2.0 * np.pi * frequency_hz
        for s in self.species:
            a = s.collision_frequency_hz + 1j * w
            gyro = s.charge_c * bmag / s.mass_kg
            drive = s.number_density_m3 * s.charge_c**2 / s.mass_kg
            den = a**2 + gyro**2
            parallel += drive / a
            pedersen += drive * a / den
            hall += drive * gyro / den
        return parallel, pedersen, hall

    @property
    def content_sha256(self) -> str:
        payload = {
            "mesh_vertices_sha256": self.mesh_vertices_sha256,
            "mesh_faces_sha256": self.mesh_faces_sha256,
            "radial_midpoints_sha256": array_sha256(self.radial_midpoint_altitudes_m),
            "magnetic_field_sha256": array_sha256(self.magnetic_field_t),
            "species": [
                {
                    "name": s.name,
                    "charge_c": s.charge_c,
                    "mass_kg": s.mass_kg,
                    "density_sha256": array_sha256(s.number_density_m3),
                    "collision_sha256": array_sha256(s.collision_frequency_hz),
                }
                for s in self.species
            ],
            "provenance": [(p.dataset_id, p.source_sha256) for p in self.provenance],
            "interpolation": self.interpolation,
        }
        return hashlib.sha256(json.dumps(payload, sort_keys=True, separators=(",", ":")).encode()).hexdigest()

    def save(self, path: str | Path) -> Path:
        destination = Path(path)
        destination.parent.mkdir(parents=True, exist_ok=True)
        metadata, arrays = self.archive_payload()
        arrays["metadata"] = np.asarray(json.dumps(metadata, sort_keys=True))
        temporary = None
        try:
            with tempfile.NamedTemporaryFile(mode="wb", dir=destination.parent, prefix=f".{destination.name}.", delete=False) as handle:
                temporary = handle.name
                np.savez_compressed(handle, **arrays)
                handle.flush()
                os.fsync(handle.fileno())
            os.replace(temporary, destination)
        finally:
            if temporary is not None and os.path.exists(temporary):
                os.unlink(temporary)
        return destination

    @classmethod
    def load(cls, path: str | Path) -> "MeshPlasmaModel":
        try:
            with np.load(path, allow_pickle=False) as archive:
                if "metadata" not in archive.files:
                    raise ValueError("plasma artifact is missing metadata")
                metadata = json.loads(str(archive["metadata"].item()))
                arrays = {n: np.array(archive[n], copy=True) for n in archive.files if n != "metadata"}
        except (OSError, KeyError, json.JSONDecodeError) as error:
            raise ValueError(f"cannot read plasma artifact {path}: {error}") from error
        return cls.from_archive_payload(metadata, arrays)

    def archive_payload(self) -> tuple[dict[str, Any], dict[str, Any]]:
        arrays: dict[str, Any] = {
            "radial_midpoint_altitudes_m": np.ascontiguousarray(self.radial_midpoint_altitudes_m),
            "magnetic_field_t": np.ascontiguousarray(self.magnetic_field_t),
        }
        for i, s in enumerate(self.species):
            arrays[f"species_{i}_number_density_m3"] = np.ascontiguousarray(s.number_density_m3)
            arrays[f"species_{i}_collision_frequency_hz"] = np.ascontiguousarray(s.collision_frequency_hz)
        return self._metadata(arrays), arrays

    @classmethod
    def from_archive_payload(cls, metadata: dict[str, Any], arrays: dict[str, Any]) -> "MeshPlasmaModel":
        if metadata.get("format") != MESH_PLASMA_FORMAT:
            raise ValueError("unsupported plasma artifact format")
        if metadata.get("version") != MESH_PLASMA_VERSION:
            raise ValueError("unsupported plasma artifact version")
        records = metadata.get("arrays")
        if not isinstance(records, dict):
            raise ValueError("plasma artifact array metadata is invalid")
        for name, record in records.items():
            if name not in arrays:
                raise ValueError(f"plasma artifact is missing {name}")
            if record.get("shape") != list(arrays[name].shape):
                raise ValueError(f"plasma artifact {name} shape mismatch")
            if record.get("sha256") != array_sha256(arrays[name]):
                raise ValueError(f"plasma artifact {name} checksum mismatch")
        try:
            species = tuple(
                ColdPlasmaSpecies(
                    name=r["name"],
                    charge_c=r["charge_c"],
                    mass_kg=r["mass_kg"],
                    number_density_m3=arrays[f"species_{i}_number_density_m3"],
                    collision_frequency_hz=arrays[f"species_{i}_collision_frequency_hz"],
                )
                for i, r in enumerate(metadata["species"])
            )
            provenance = tuple(
                DatasetProvenance(**{**r, "variables": tuple(VariableProvenance(**v) for v in r["variables"])})
                for r in metadata["provenance"]
            )
            return cls(
                mesh_vertices_sha256=metadata["mesh"]["vertices_sha256"],
                mesh_faces_sha256=metadata["mesh"]["faces_sha256"],
                radial_midpoint_altitudes_m=arrays["radial_midpoint_altitudes_m"],
                magnetic_field_t=arrays["magnetic_field_t"],
                species=species,
                provenance=provenance,
                interpolation=metadata["interpolation"],
            )
        except (KeyError, TypeError, ValueError) as error:
            raise ValueError(f"invalid plasma artifact metadata: {error}") from error

    def _metadata(self, arrays: dict[str, Any]) -> dict[str, Any]:
        return {
            "format": MESH_PLASMA_FORMAT,
            "version": MESH_PLASMA_VERSION,
            "mesh": {"vertices_sha256": self.mesh_vertices_sha256, "faces_sha256": self.mesh_faces_sha256},
            "species": [{"name": s.name, "charge_c": s.charge_c, "mass_kg": s.mass_kg} for s in self.species],
            "provenance": [asdict(p) for p in self.provenance],
            "interpolation": self.interpolation,
            "arrays": {n: {"shape": list(np.asarray(v).shape), "sha256": array_sha256(v)} for n, v in arrays.items()},
        }


def ade_coefficients(model: MeshPlasmaModel, time_step_s: float):
    """Exact constant-E species update coefficients (plasma.py:374-411).

    Returns ``(coef (S, 6, rows, L), bdir (rows, L, 3), magnetized, rows)``
    with ``rows == 1`` when every input is horizontally uniform.
    """

    magnetic = model.magnetic_field_t
    inputs = [magnetic] + [a for s in model.species for a in (s.number_density_m3, s.collision_frequency_hz)]
    uniform = all(horizontally_uniform(a) for a in inputs)
    pick = (lambda a: np.asarray(a[:1])) if uniform else (lambda a: np.asarray(a))
    b = pick(magnetic)
    bmag = np.linalg.norm(b, axis=2)
    bdir = np.zeros_like(b)
    nz = bmag > 0.0
    bdir[nz] = b[nz] / bmag[nz, None]
    coef = []
    for s in model.species:
        nu = pick(s.collision_frequency_hz)
        gyro = s.charge_c * bmag / s.mass_kg
        decay = np.exp(-nu * time_step_s)
        angle = gyro * time_step_s
        eig = -nu + 1j * gyro
        integral = np.expm1(eig * time_step_s) / eig
        parallel = -np.expm1(-nu * time_step_s) / nu
        drive = pick(s.number_density_m3) * s.charge_c**2 / s.mass_kg
        coef.append(np.stack((decay, np.cos(angle), np.sin(angle), drive * parallel, drive * integral.real, drive * integral.imag)))
    return np.ascontiguousarray(np.stack(coef)), np.ascontiguousarray(bdir), bool(np.any(bmag > 0.0)), b.shape[0]


def face_reconstruction(mesh) -> tuple[NDArray[np.float64], NDArray[np.float64]]:
    """Per-face ``pinv(tangents).T`` and the unit edge tangents (plasma.py:548-559)."""

    edges, face_edges, centres = mesh.edges, mesh.face_edges, mesh.face_centers
    tangents = np.empty((mesh.n_faces, 3, 3))
    recon = np.empty_like(tangents)
    normals = np.empty((mesh.n_edges, 3))
    step = 1 << 15

    # every step is row-wise (an edge's normal, a face's tangents and its 3 x 3
    # pseudo-inverse), so the chunks may run on threads (NumPy and LAPACK
    # release the GIL in them) and the bits do not change
    def edge_chunk(start: int) -> None:
        e = edges[start : start + step]
        n = np.cross(mesh.vertices[e[:, 0]], mesh.vertices[e[:, 1]])
        normals[start : start + step] = n / np.linalg.norm(n, axis=1, keepdims=True)

    def face_chunk(start: int) -> None:
        t = np.cross(normals[face_edges[start : start + step]], centres[start : start + step, None, :])
        t /= np.linalg.norm(t, axis=2, keepdims=True)
        tangents[start : start + step] = t
        recon[start : start + step] = np.swapaxes(np.linalg.pinv(t), 1, 2)

    for job, n in ((edge_chunk, mesh.n_edges), (face_chunk, mesh.n_faces)):
        starts = range(0, n, step)
        workers = min(len(starts), os.cpu_count() or 1)
        if workers > 1:
            with ThreadPoolExecutor(workers) as pool:
                list(pool.map(job, starts))
        else:
            for start in starts:
                job(start)
    return recon, tangents


def edge_face_slots(mesh, faces) -> NDArray[np.int64]:
    """Position of each edge inside its left (or right) face (plasma.py:562-569)."""

    slots = mesh.face_edges[faces]
    edge = np.arange(mesh.n_edges)
    m0, m1, m2 = (slots[:, k] == edge for k in range(3))
    if not np.all(m0.astype(np.int8) + m1 + m2 == 1):
        raise RuntimeError("edge is absent from an adjacent face")
    return np.where(m0, 0, np.where(m1, 1, 2))


def vertex_face_average(mesh) -> tuple[NDArray[np.int64], NDArray[np.float64]]:
    """Incident faces per vertex in face order with area weights (plasma.py:572-588)."""

    import ctypes

    from . import _native as N

    owners = np.ascontiguousarray(mesh.faces, dtype=np.int64).ravel()
    # face corners grouped by vertex, each group in face order (a stable counting sort
    # in the library's host code)
    order = np.empty(len(owners), dtype=np.int64)
    counts = np.empty(mesh.n_vertices, dtype=np.int64)
    N.check(
        N.load().ifdtd_stable_group(N.ptr_i64(owners), len(owners), mesh.n_vertices, N.ptr_i64(order), N.ptr_i64(counts)),
        "ifdtd_stable_group",
    )
    owners, face_of = owners[order], order // 3
    width = int(counts.max())
    starts = np.concatenate(([0], np.cumsum(counts)[:-1]))
    slot = np.arange(len(owners)) - np.repeat(starts, counts)
    faces = np.zeros((mesh.n_vertices, width), dtype=np.int64)
    areas = np.zeros((mesh.n_vertices, width), dtype=np.float64)
    faces[owners, slot] = face_of
    areas[owners, slot] = mesh.face_solid_angles[face_of]
    total = np.zeros(mesh.n_vertices)
    for k in range(width):  # sequential, in face order
        total = total + areas[:, k]
    return faces, areas / total[:, None]


def _face_layer_component_view(component_major):
    """(F, 3, L) storage seen as the reference's (F, L, 3) array, without a copy."""

    if hasattr(component_major, "permute"):
        return component_major.permute(0, 2, 1)
    return np.swapaxes(component_major, 1, 2)


def _cross_with(v, b, backend):
    """v x b over the last axis (plasma.py:591-596)."""

    out = backend.empty_like(v)
    out[..., 0] = v[..., 1] * b[..., 2] - v[..., 2] * b[..., 1]
    out[..., 1] = v[..., 2] * b[..., 0] - v[..., 0] * b[..., 2]
    out[..., 2] = v[..., 0] * b[..., 1] - v[..., 1] * b[..., 0]
    return out


class MagnetizedPlasmaADE:
    """Species coefficients and device current densities.

    Each species' current lives in a component-major buffer (F, 3, mid_pitch)
    (16-byte aligned rows for the step kernels); ``current_density[s]`` is the
    reference-shaped (F, L, 3) view of it, so reads, in-place writes and
    checkpoints see the reference layout (plasma.py:411)."""

    def __init__(self, model: MeshPlasmaModel, time_step_s: float, backend: Any, mid_pitch: int | None = None):
        self.model = model
        self.backend = backend
        self.coef, self.bdir, self.magnetized, self.rows = ade_coefficients(model, time_step_s)
        n_faces, layers = model.magnetic_field_t.shape[:2]
        pitch = mid_pitch or (layers + 3) // 4 * 4
        self.buffers = [backend.zeros((n_faces, 3, pitch)) for _ in model.species]
        self.current_density = [_face_layer_component_view(buf[:, :, :layers]) for buf in self.buffers]
        self._arrays = None  # backend copies of coef / bdir for ``advance``, made on first use

    def advance(self, electric_v_m: Any) -> Any:
        """Advance every species' current by one step under the face-centred field
        ``electric_v_m`` (F, L, 3) and return their sum (plasma.py:413-442).  The
        engine's H kernel runs this update inside the step; this is the same
        arithmetic on the backend's arrays, for callers that drive the ADE directly."""

        if self._arrays is None:
            asarray = self.backend.asarray
            self._arrays = ([[asarray(c[k])[..., None] for k in range(6)] for c in self.coef], asarray(self.bdir))
        coefs, b = self._arrays
        e_par = (electric_v_m * b).sum(-1)[..., None] * b
        e_perp = electric_v_m - e_par
        e_cross = _cross_with(e_perp, b, self.backend)
        total = None
        for current, (decay, cosine, sine, d_par, d_re, d_im) in zip(self.current_density, coefs):
            j_par = (current * b).sum(-1)[..., None] * b
            j_perp = current - j_par
            j_cross = _cross_with(j_perp, b, self.backend)
            updated = (decay * j_par + d_par * e_par + decay * (cosine * j_perp + sine * j_cross)
                       + d_re * e_perp + d_im * e_cross)
            current[...] = updated
            total = updated if total is None else total + updated
        return total

    @property
    def state_bytes(self) -> int:
        return sum(self.backend.nbytes(j) for j in self.current_density)

    @property
    def persistent_bytes(self) -> int:
        itemsize = 4 if self.backend.dtype_name == "float32" else 8
        return self.state_bytes + itemsize * (self.coef.size + (self.bdir.size if self.magnetized else 0))


class GeodesicPlasmaCoupler:
    """Reconstruction and scatter tables of the plasma coupling (plasma.py:455-545)."""

    def __init__(self, model: MeshPlasmaModel, mesh, radial_midpoint_altitudes_m, time_step_s: float, backend: Any, mid_pitch: int | None = None) -> None:
        model.validate_grid(mesh, radial_midpoint_altitudes_m)
        self.mesh = mesh
        self.backend = backend
        recon, tangents = face_reconstruction(mesh)
        self.reconstruction = np.ascontiguousarray(recon)
        left_slots = edge_face_slots(mesh, mesh.edge_left_faces)
        right_slots = edge_face_slots(mesh, mesh.edge_right_faces)
        self.left_tangents = np.ascontiguousarray(tangents[mesh.edge_left_faces, left_slots])
        self.right_tangents = np.ascontiguousarray(tangents[mesh.edge_right_faces, right_slots])
        self.vertex_faces, self.vertex_face_weights = vertex_face_average(mesh)
        self.ade = MagnetizedPlasmaADE(model, time_step_s, backend, mid_pitch)

    @property
    def persistent_bytes(self) -> int:
        itemsize = 4 if self.backend.dtype_name == "float32" else 8
        n = self.reconstruction.size + 3 * self.mesh.n_faces + self.left_tangents.size + self.right_tangents.size
        return self.ade.persistent_bytes + itemsize * n + 4 * self.vertex_faces.size + itemsize * self.vertex_face_weights.size
