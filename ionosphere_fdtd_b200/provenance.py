"""Dataset provenance records and canonical array checksums.

Same record fields, validation and hashing convention as the reference
(data_artifacts.py:26-109, 447-480) so that a plasma model's identity
(``MeshPlasmaModel.content_sha256``) and its checkpoint payload are
interchangeable between the two implementations.
"""

from __future__ import annotations

import hashlib
import re
from dataclasses import dataclass
from datetime import datetime
from pathlib import Path
from typing import Any

import numpy as np
from numpy.typing import NDArray

_SHA256 = re.compile(r"[0-9a-f]{64}")


class DataArtifactError(ValueError):
    """Raised when material data provenance or content is invalid."""


@dataclass(frozen=True, slots=True)
class VariableProvenance:
    name: str
    source_units: str
    canonical_units: str
    conversion: str

    def __post_init__(self) -> None:
        if not all(isinstance(v, str) and v.strip() for v in (self.name, self.source_units, self.canonical_units, self.conversion)):
            raise DataArtifactError("variable provenance fields must be nonempty")


@dataclass(frozen=True, slots=True)
class DatasetProvenance:
    dataset_id: str
    title: str
    version: str
    source_url: str
    citation: str
    license: str
    retrieved_at: str
    source_sha256: str
    coordinate_reference_system: str
    variables: tuple[VariableProvenance, ...]

    def __post_init__(self) -> None:
        text = (
            self.dataset_id,
            self.title,
            self.version,
            self.source_url,
            self.citation,
            self.license,
            self.retrieved_at,
            self.coordinate_reference_system,
        )
        if not all(isinstance(v, str) and v.strip() for v in text):
            raise DataArtifactError("dataset provenance fields must be nonempty")
        if _SHA256.fullmatch(self.source_sha256) is None:
            raise DataArtifactError("source_sha256 must be a lowercase SHA-256")
        try:
            when = datetime.fromisoformat(self.retrieved_at.replace("Z", "+00:00"))
        except ValueError as error:
            raise DataArtifactError("retrieved_at must be ISO 8601") from error
        if when.tzinfo is None:
            raise DataArtifactError("retrieved_at must include a timezone")
        variables = tuple(self.variables)
        if not variables or not all(isinstance(v, VariableProvenance) for v in variables):
            raise DataArtifactError("dataset provenance requires variable records")
        names = [v.name for v in variables]
        if len(set(names)) != len(names):
            raise DataArtifactError("dataset variable names must be unique")
        object.__setattr__(self, "variables", variables)

    @classmethod
    def from_file(cls, path: str | Path, **metadata: Any) -> "DatasetProvenance":
        return cls(source_sha256=file_sha256(path), **metadata)


def file_sha256(path: str | Path) -> str:
    try:
        with Path(path).open("rb") as stream:
            return hashlib.file_digest(stream, "sha256").hexdigest()
    except OSError as error:
        raise DataArtifactError(f"cannot hash source file {path}: {error}") from error


def distinct_elements(a: Any) -> NDArray:
    """``a`` restricted to index 0 along its zero-stride (broadcast) axes: the
    same set of values, each stored element once, for validity checks."""

    a = np.asarray(a)
    return a[tuple(slice(0, 1) if st == 0 else slice(None) for st in a.strides)]


def array_sha256(values: Any) -> str:
    """SHA-256 of the array in little-endian C order, floats as <f8 and integers as <i8."""

    array = np.asarray(values)
    if np.issubdtype(array.dtype, np.floating):
        dtype = "<f8"
    elif np.issubdtype(array.dtype, np.integer):
        dtype = "<i8"
    else:
        raise DataArtifactError("only numeric arrays can be checksummed")
    digest = hashlib.sha256()
    if array.ndim == 0:
        digest.update(np.asarray(array, dtype=dtype).tobytes())
        return digest.hexdigest()
    # leading-axis chunks of about 16 MiB, hashed in order: the same bytes as the whole
    # array in C order, without materialising broadcast or converted arrays in full
    rows = max(1, (1 << 24) // max(1, 8 * int(np.prod(array.shape[1:]))))
    for lo in range(0, array.shape[0], rows):
        digest.update(np.ascontiguousarray(array[lo : lo + rows], dtype=dtype).data)
    return digest.hexdigest()


def mesh_vertices_sha256(mesh: Any) -> str:
    return array_sha256(mesh.vertices)


def mesh_faces_sha256(mesh: Any) -> str:
    return array_sha256(mesh.faces)
