"""Icosahedral geodesic mesh with the reference's exact numbering.

Same topology, index tables and float64 geometry as the reference builder
(src/ionosphere_fdtd/mesh.py), computed with array operations instead of
per-face Python loops, so a subdivision-9 mesh (2.6 M cells) builds in
seconds.  Midpoint vertices and edges are numbered in order of first use
during the face scan, which is exactly the reference's dictionary-insertion
order (mesh.py:569-593, 674-708); the golden tests check the tables bitwise.
"""

from __future__ import annotations

import json
import os
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass
from typing import Any, Mapping

import numpy as np
from numpy.typing import NDArray

FloatArray = NDArray[np.float64]
IntArray = NDArray[np.int64]


@dataclass(frozen=True, slots=True)
class GeodesicMesh:
    """Topology and unit-sphere metric terms (mesh.py:21-188)."""

    vertices: FloatArray
    faces: IntArray
    edges: IntArray
    face_edges: IntArray
    face_edge_signs: IntArray
    edge_left_faces: IntArray
    edge_right_faces: IntArray
    face_centers: FloatArray
    primal_edge_angles: FloatArray
    dual_edge_angles: FloatArray
    face_solid_angles: FloatArray
    dual_cell_solid_angles: FloatArray
    vertex_degree: IntArray
    subdivision: int | None
    topology_kind: str
    face_levels: IntArray | None
    refinement_spec_json: str | None

    def __post_init__(self) -> None:
        for values in (
            self.vertices,
            self.faces,
            self.edges,
            self.face_edges,
            self.face_edge_signs,
            self.edge_left_faces,
            self.edge_right_faces,
            self.face_centers,
            self.primal_edge_angles,
            self.dual_edge_angles,
            self.face_solid_angles,
            self.dual_cell_solid_angles,
            self.vertex_degree,
        ):
            values.setflags(write=False)
        if self.face_levels is not None:
            self.face_levels.setflags(write=False)

    @property
    def n_vertices(self) -> int:
        return int(self.vertices.shape[0])

    @property
    def n_edges(self) -> int:
        return int(self.edges.shape[0])

    @property
    def n_faces(self) -> int:
        return int(self.faces.shape[0])

    @property
    def refinement_spec(self) -> dict[str, Any] | None:
        if self.refinement_spec_json is None:
            return None
        value = json.loads(self.refinement_spec_json)
        if not isinstance(value, dict):
            raise RuntimeError("mesh refinement specification is not a JSON object")
        return value

    def edge_midpoints(self) -> FloatArray:
        return _rowwise(lambda e: _unit(self.vertices[e].sum(axis=1)), self.edges)

    def edge_diamond_solid_angles(self) -> FloatArray:
        tail = self.vertices[self.edges[:, 0]]
        head = self.vertices[self.edges[:, 1]]
        left = self.face_centers[self.edge_left_faces]
        right = self.face_centers[self.edge_right_faces]
        return _signed_triangle(tail, head, left) - _signed_triangle(tail, head, right)

    def edge_diamond_quadrant_solid_angles(self) -> FloatArray:
        tail = self.vertices[self.edges[:, 0]]
        head = self.vertices[self.edges[:, 1]]
        mid = self.edge_midpoints()
        left = self.face_centers[self.edge_left_faces]
        right = self.face_centers[self.edge_right_faces]
        return -np.column_stack(
            (
                _signed_triangle(mid, tail, left),
                _signed_triangle(mid, left, head),
                _signed_triangle(mid, head, right),
                _signed_triangle(mid, right, tail),
            )
        )

    def dual_cell_wedge_quadrature(self, vertex_indices: IntArray, edge_indices: IntArray) -> tuple[FloatArray, FloatArray]:
        vertices = np.asarray(vertex_indices, dtype=np.int64)
        edges = np.asarray(edge_indices, dtype=np.int64)
        if vertices.ndim != 1 or edges.shape != vertices.shape:
            raise ValueError("dual-cell wedge indices must be matching 1-D arrays")
        if np.any(vertices < 0) or np.any(vertices >= self.n_vertices):
            raise ValueError("dual-cell wedge vertex index is out of bounds")
        if np.any(edges < 0) or np.any(edges >= self.n_edges):
            raise ValueError("dual-cell wedge edge index is out of bounds")
        if np.any(~np.any(self.edges[edges] == vertices[:, None], axis=1)):
            raise ValueError("dual-cell wedge vertex must be incident to its edge")
        points = self.vertices[vertices]
        left = self.face_centers[self.edge_left_faces[edges]]
        right = self.face_centers[self.edge_right_faces[edges]]
        areas = _signed_triangle(points, left, right)
        return _unit(points + left + right), np.where(self.edges[edges, 1] == vertices, areas, -areas)

    # host-side reference operators (used by setup and tests, not the step)
    def face_circulation(self, edge_values: FloatArray) -> FloatArray:
        picked = edge_values[self.face_edges]
        signs = self.face_edge_signs.astype(edge_values.dtype, copy=False)
        while signs.ndim < picked.ndim:
            signs = signs[..., None]
        return np.sum(picked * signs, axis=1)

    def dual_cell_circulation(self, dual_edge_values: FloatArray) -> FloatArray:
        out = np.zeros((self.n_vertices,) + dual_edge_values.shape[1:], dtype=dual_edge_values.dtype)
        np.add.at(out, self.edges[:, 0], dual_edge_values)
        np.add.at(out, self.edges[:, 1], -dual_edge_values)
        return out

    def edge_difference(self, vertex_values: FloatArray) -> FloatArray:
        return vertex_values[self.edges[:, 1]] - vertex_values[self.edges[:, 0]]

    def dual_edge_difference(self, face_values: FloatArray) -> FloatArray:
        return face_values[self.edge_left_faces] - face_values[self.edge_right_faces]


def _unit(values: FloatArray) -> FloatArray:
    return values / np.linalg.norm(values, axis=-1, keepdims=True)


_ROWS_PER_CHUNK = 1 << 16


def _rowwise(fn, *arrays):
    """fn(*arrays) for functions that treat every row on its own: large inputs
    are cut into row chunks run on threads (NumPy releases the GIL in them),
    which gives the same bits as one call."""

    n = len(arrays[0])
    workers = min(os.cpu_count() or 1, n // _ROWS_PER_CHUNK)
    if workers < 2:
        return fn(*arrays)
    starts = range(0, n, _ROWS_PER_CHUNK)
    with ThreadPoolExecutor(workers) as pool:
        parts = list(pool.map(lambda a: fn(*(x[a : a + _ROWS_PER_CHUNK] for x in arrays)), starts))
    return np.concatenate(parts)


# The 12-vertex / 20-face seed of every level (the reference's table,
# mesh.py:475-519): all downstream numbering descends from this order.
_G = (1.0 + np.sqrt(5.0)) / 2.0
_SEED_VERTICES = np.asarray(
    [
        (-1, _G, 0), (1, _G, 0), (-1, -_G, 0), (1, -_G, 0),
        (0, -1, _G), (0, 1, _G), (0, -1, -_G), (0, 1, -_G),
        (_G, 0, -1), (_G, 0, 1), (-_G, 0, -1), (-_G, 0, 1),
    ],
    dtype=np.float64,
)
_SEED_FACES = np.asarray(
    [
        (0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11),
        (1, 5, 9), (5, 11, 4), (11, 10, 2), (10, 7, 6), (7, 1, 8),
        (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9),
        (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1),
    ],
    dtype=np.int64,
)


def _orient_outward(vertices: FloatArray, faces: IntArray) -> IntArray:
    out = faces.copy()
    a, b, c = (vertices[out[:, i]] for i in range(3))
    inward = np.einsum("ij,ij->i", np.cross(b - a, c - a), a + b + c) < 0.0
    out[inward, 1], out[inward, 2] = out[inward, 2].copy(), out[inward, 1].copy()
    return out


def _seed() -> tuple[FloatArray, IntArray]:
    v = _unit(_SEED_VERTICES)
    return v, _orient_outward(v, _SEED_FACES)


def _to_poles(vertices: FloatArray) -> FloatArray:
    """Rodrigues rotation of seed vertex 5 to +z, then a twist putting seed
    vertex 9 at longitude 0 (mesh.py:522-555)."""

    src = vertices[5]
    dst = np.asarray((0.0, 0.0, 1.0))
    axis = np.cross(src, dst)
    sine = np.linalg.norm(axis)
    cosine = float(src @ dst)
    k = np.asarray(((0.0, -axis[2], axis[1]), (axis[2], 0.0, -axis[0]), (-axis[1], axis[0], 0.0)))
    rotation = np.eye(3) + k + k @ k * ((1.0 - cosine) / sine**2)
    turned = vertices @ rotation.T
    lon = np.arctan2(turned[9, 1], turned[9, 0])
    c, s = np.cos(-lon), np.sin(-lon)
    return turned @ np.asarray(((c, -s, 0.0), (s, c, 0.0), (0.0, 0.0, 1.0))).T


def _first_use_numbering(lo: IntArray, hi: IntArray, n_vertices: int) -> tuple[IntArray, IntArray]:
    """Number the distinct (lo, hi) pairs in order of first appearance.

    Returns ``(rank_of_each_pair, first_position_of_each_number)``; identical
    to assigning ``len(dict)`` on first insertion during a sequential scan.
    """

    import ctypes

    from . import _native as N

    lo = np.ascontiguousarray(lo, dtype=np.int64).ravel()
    hi = np.ascontiguousarray(hi, dtype=np.int64).ravel()
    rank = np.empty(len(lo), dtype=np.int64)
    first = np.empty(len(lo), dtype=np.int64)
    count = ctypes.c_int64()
    # one pass with a hash table in the library (host code, no device needed)
    N.check(
        N.load().ifdtd_first_use_numbering(N.ptr_i64(lo), N.ptr_i64(hi), len(lo), int(n_vertices), N.ptr_i64(rank),
                                           N.ptr_i64(first), ctypes.byref(count)),
        "ifdtd_first_use_numbering",
    )
    return rank, first[: count.value].copy()


def _quarter(vertices: FloatArray, faces: IntArray) -> tuple[FloatArray, IntArray]:
    """One 4:1 refinement, midpoints numbered in face-scan order (mesh.py:569-593)."""

    n = len(vertices)
    p = faces
    q = np.roll(faces, -1, axis=1)  # (a,b), (b,c), (c,a) per face
    lo = np.minimum(p, q).ravel()
    hi = np.maximum(p, q).ravel()
    rank, first = _first_use_numbering(lo, hi, n)
    new_points = _unit(vertices[lo[first]] + vertices[hi[first]])
    mid = (n + rank).reshape(-1, 3)
    a, b, c = faces[:, 0], faces[:, 1], faces[:, 2]
    ab, bc, ca = mid[:, 0], mid[:, 1], mid[:, 2]
    children = np.stack(
        (
            np.stack((a, ab, ca), axis=1),
            np.stack((b, bc, ab), axis=1),
            np.stack((c, ca, bc), axis=1),
            np.stack((ab, bc, ca), axis=1),
        ),
        axis=1,
    ).reshape(-1, 3)
    return np.concatenate((vertices, new_points)), children


def _edge_tables(faces: IntArray, n_vertices: int):
    """Edges numbered in face-scan order; left face carries sign +1 (mesh.py:674-708)."""

    p = faces
    q = np.roll(faces, -1, axis=1)
    lo = np.minimum(p, q).ravel()
    hi = np.maximum(p, q).ravel()
    rank, first = _first_use_numbering(lo, hi, n_vertices)
    edges = np.stack((lo[first], hi[first]), axis=1)
    face_edges = rank.reshape(-1, 3)
    signs = np.where(p < q, 1, -1).astype(np.int64)
    counts = np.bincount(rank, minlength=len(edges))
    plus = np.bincount(rank, weights=(signs.ravel() > 0), minlength=len(edges))
    if np.any(counts != 2) or np.any(plus != 1):
        raise RuntimeError("geodesic mesh is not a closed two-manifold")
    face_of = np.repeat(np.arange(len(faces), dtype=np.int64), 3)
    left = np.empty(len(edges), dtype=np.int64)
    right = np.empty(len(edges), dtype=np.int64)
    positive = signs.ravel() > 0
    left[rank[positive]] = face_of[positive]
    right[rank[~positive]] = face_of[~positive]
    return edges, face_edges, signs, left, right


def _arc(a: FloatArray, b: FloatArray) -> FloatArray:
    return np.arctan2(np.linalg.norm(np.cross(a, b), axis=1), np.einsum("ij,ij->i", a, b))


def _signed_triangle(a: FloatArray, b: FloatArray, c: FloatArray) -> FloatArray:
    num = np.einsum("ij,ij->i", a, np.cross(b, c))
    den = 1.0 + np.einsum("ij,ij->i", a, b) + np.einsum("ij,ij->i", b, c) + np.einsum("ij,ij->i", c, a)
    return 2.0 * np.arctan2(num, den)


def _circumcentres(vertices: FloatArray, faces: IntArray) -> FloatArray:
    a, b, c = (vertices[faces[:, i]] for i in range(3))
    n = _unit(np.cross(b - a, c - a))
    flip = np.einsum("ij,ij->i", n, a + b + c) < 0.0
    n[flip] *= -1.0
    return n


def _assemble(
    vertices: FloatArray,
    faces: IntArray,
    subdivision: int | None,
    *,
    topology_kind: str,
    face_levels: IntArray | None = None,
    refinement_spec_json: str | None = None,
    require_well_centered: bool = False,
) -> GeodesicMesh:
    """Orient, number and measure a closed triangulation (mesh.py:397-468)."""

    # every measure below is row-wise, so large meshes compute it in threaded
    # row chunks with the same bits (_rowwise)
    faces = _rowwise(lambda f: _orient_outward(vertices, f), faces)
    centres = _rowwise(lambda f: _circumcentres(vertices, f), faces)
    edges, face_edges, signs, left, right = _edge_tables(faces, len(vertices))
    primal = _rowwise(lambda e: _arc(vertices[e[:, 0]], vertices[e[:, 1]]), edges)
    cl, cr = centres[left], centres[right]
    dual = _rowwise(_arc, cl, cr)
    face_area = np.abs(_rowwise(lambda f: _signed_triangle(vertices[f[:, 0]], vertices[f[:, 1]], vertices[f[:, 2]]), faces))
    # dual areas: the tail wedges (negated) of every edge in edge order, then the
    # head wedges, accumulated per vertex in that order (mesh.py:768-789)
    tail_w = -_rowwise(lambda e, a, b: _signed_triangle(vertices[e], a, b), edges[:, 0], cl, cr)
    head_w = _rowwise(lambda e, a, b: _signed_triangle(vertices[e], a, b), edges[:, 1], cl, cr)
    dual_area = np.bincount(
        np.concatenate((edges[:, 0], edges[:, 1])), weights=np.concatenate((tail_w, head_w)), minlength=len(vertices)
    )
    degree = np.bincount(edges.ravel(), minlength=len(vertices))
    if not np.all(degree >= 3):
        raise RuntimeError("invalid closed geodesic topology")
    if len(vertices) - len(edges) + len(faces) != 2:
        raise RuntimeError("geodesic mesh topology is not a sphere")
    for values, label in ((primal, "primal edges"), (dual, "dual edges"), (face_area, "primal faces"), (dual_area, "dual cells")):
        if not np.all(np.isfinite(values)) or not np.all(values > 0.0):
            raise ValueError(f"geodesic mesh contains degenerate {label}")
    if require_well_centered:
        _check_well_centered(vertices, faces, centres)
    if not np.isclose(face_area.sum(), 4.0 * np.pi, rtol=1e-11):
        raise RuntimeError("primal face areas do not cover the unit sphere")
    if not np.isclose(dual_area.sum(), 4.0 * np.pi, rtol=1e-10):
        raise RuntimeError("dual cell areas do not cover the unit sphere")
    return GeodesicMesh(
        vertices=vertices,
        faces=faces,
        edges=edges,
        face_edges=face_edges,
        face_edge_signs=signs,
        edge_left_faces=left,
        edge_right_faces=right,
        face_centers=centres,
        primal_edge_angles=primal,
        dual_edge_angles=dual,
        face_solid_angles=face_area,
        dual_cell_solid_angles=dual_area,
        vertex_degree=degree,
        subdivision=subdivision,
        topology_kind=topology_kind,
        face_levels=face_levels,
        refinement_spec_json=refinement_spec_json,
    )


def _check_well_centered(vertices: FloatArray, faces: IntArray, centres: FloatArray) -> None:
    tri = vertices[faces]
    side = np.column_stack(
        [np.einsum("ij,ij->i", np.cross(tri[:, k], tri[:, (k + 1) % 3]), centres) for k in range(3)]
    )
    bad = np.flatnonzero(np.any(side <= 64.0 * np.finfo(np.float64).eps, axis=1))
    if len(bad):
        raise ValueError(
            "optimized vertices must form a well-centered spherical mesh; "
            f"{len(bad)} circumcenter(s) lie outside or on a primal face"
        )


def _relax(vertices: FloatArray, faces: IntArray) -> FloatArray:
    """Centroid relaxation (mesh.py:596-603)."""

    centres = _unit(vertices[faces].sum(axis=1))
    acc = np.zeros_like(vertices)
    counts = np.zeros(len(vertices), dtype=np.int64)
    for corner in range(3):
        np.add.at(acc, faces[:, corner], centres)
        np.add.at(counts, faces[:, corner], 1)
    return _unit(acc / counts[:, None])


def _optimize_edge_lengths(vertices: FloatArray, faces: IntArray, steps: int) -> FloatArray:
    """Projected edge-length equalisation with the 12 pentagons fixed (mesh.py:606-663)."""

    edges = _edge_tables(faces, len(vertices))[0]
    degree = np.bincount(edges.ravel(), minlength=len(vertices))
    fixed = degree == 5
    out = vertices.copy()
    tails, heads = edges[:, 0], edges[:, 1]
    for _ in range(steps):
        tv, hv = out[tails], out[heads]
        dot = np.clip(np.einsum("ij,ij->i", tv, hv), -1.0, 1.0)
        sine = np.linalg.norm(np.cross(tv, hv), axis=1)
        residual = np.arctan2(sine, dot)
        residual = residual - float(np.mean(residual))
        tg = residual[:, None] * (dot[:, None] * tv - hv) / sine[:, None]
        hg = residual[:, None] * (dot[:, None] * hv - tv) / sine[:, None]
        grad = np.zeros_like(out)
        np.add.at(grad, tails, tg)
        np.add.at(grad, heads, hg)
        grad /= degree[:, None]
        grad -= np.einsum("ij,ij->i", grad, out)[:, None] * out
        grad[fixed] = 0.0
        out = _unit(out - grad)
        out[fixed] = vertices[fixed]
    return out


def subdivided_icosahedron(subdivision: int, orientation: str) -> tuple[FloatArray, IntArray]:
    vertices, faces = _seed()
    if orientation == "polar":
        vertices = _to_poles(vertices)
    for _ in range(subdivision):
        vertices, faces = _quarter(vertices, faces)
    return vertices, faces


def build_geodesic_mesh(
    subdivision: int = 2, relaxations: int = 0, orientation: str = "polar", optimization_steps: int = 0
) -> GeodesicMesh:
    """Recursively quartered icosahedron on the unit sphere (mesh.py:191-227)."""

    if subdivision < 0:
        raise ValueError("subdivision must be non-negative")
    if relaxations < 0:
        raise ValueError("relaxations must be non-negative")
    if optimization_steps < 0:
        raise ValueError("optimization_steps must be non-negative")
    if orientation not in {"native", "polar"}:
        raise ValueError("orientation must be 'native' or 'polar'")
    vertices, faces = subdivided_icosahedron(subdivision, orientation)
    for _ in range(relaxations):
        vertices = _relax(vertices, faces)
    if optimization_steps:
        vertices = _optimize_edge_lengths(vertices, faces, optimization_steps)
    return _assemble(
        vertices, faces, subdivision, topology_kind="uniform", face_levels=np.full(len(faces), subdivision, dtype=np.int64)
    )


def build_geodesic_mesh_from_vertices(
    subdivision: int, vertices: FloatArray, *, orientation: str = "polar", normalize_vertices: bool = True
) -> GeodesicMesh:
    """Standard topology with externally optimised coordinates (mesh.py:230-273)."""

    if subdivision < 0:
        raise ValueError("subdivision must be non-negative")
    if orientation not in {"native", "polar"}:
        raise ValueError("orientation must be 'native' or 'polar'")
    _, faces = subdivided_icosahedron(subdivision, orientation)
    coords = np.asarray(vertices, dtype=np.float64)
    shape = (10 * 4**subdivision + 2, 3)
    if coords.shape != shape:
        raise ValueError(f"optimized vertices must have shape {shape}, got {coords.shape}")
    if not np.all(np.isfinite(coords)):
        raise ValueError("optimized vertices must be finite")
    radii = np.linalg.norm(coords, axis=1)
    if not np.allclose(radii, 1.0, rtol=0.0, atol=1.0e-7):
        raise ValueError("optimized vertices must lie on the unit sphere")
    coords = coords / radii[:, None] if normalize_vertices else coords.copy()
    return _assemble(
        coords,
        faces,
        subdivision,
        topology_kind="uniform",
        face_levels=np.full(len(faces), subdivision, dtype=np.int64),
        require_well_centered=True,
    )


def build_geodesic_mesh_from_topology(
    vertices: FloatArray,
    faces: IntArray,
    *,
    subdivision: int | None = None,
    face_levels: IntArray | None = None,
    refinement_spec: Mapping[str, Any] | None = None,
    topology_kind: str | None = None,
    normalize_vertices: bool = True,
    require_well_centered: bool = True,
) -> GeodesicMesh:
    """Mesh from any closed spherical triangulation (mesh.py:276-383)."""

    if subdivision is not None and (
        isinstance(subdivision, bool) or not isinstance(subdivision, (int, np.integer)) or subdivision < 0
    ):
        raise ValueError("subdivision must be a non-negative integer or None")
    coords = np.asarray(vertices, dtype=np.float64)
    if coords.ndim != 2 or coords.shape[1:] != (3,):
        raise ValueError("vertices must have shape (n_vertices, 3)")
    if len(coords) < 4:
        raise ValueError("a closed spherical triangulation needs at least 4 vertices")
    if not np.all(np.isfinite(coords)):
        raise ValueError("vertices must be finite")
    radii = np.linalg.norm(coords, axis=1)
    if np.any(~np.isfinite(radii)) or np.any(radii == 0.0):
        raise ValueError("vertices must have finite non-zero radii")
    if not np.allclose(radii, 1.0, rtol=0.0, atol=1.0e-7):
        raise ValueError("vertices must lie on the unit sphere")
    coords = coords / radii[:, None] if normalize_vertices else coords.copy()
    raw = np.asarray(faces)
    if raw.ndim != 2 or raw.shape[1:] != (3,):
        raise ValueError("faces must have shape (n_faces, 3)")
    if not np.issubdtype(raw.dtype, np.integer):
        raise ValueError("faces must contain integer vertex indices")
    tri = np.asarray(raw, dtype=np.int64)
    if len(tri) < 4:
        raise ValueError("a closed spherical triangulation needs at least 4 faces")
    if np.any(tri < 0) or np.any(tri >= len(coords)):
        raise ValueError("face vertex index is out of bounds")
    if np.any((tri[:, 0] == tri[:, 1]) | (tri[:, 1] == tri[:, 2]) | (tri[:, 2] == tri[:, 0])):
        raise ValueError("faces must reference three distinct vertices")
    levels = None
    if face_levels is not None:
        raw_levels = np.asarray(face_levels)
        if raw_levels.shape != (len(tri),):
            raise ValueError(f"face_levels must have shape ({len(tri)},)")
        if not np.issubdtype(raw_levels.dtype, np.integer):
            raise ValueError("face_levels must contain integers")
        levels = np.array(raw_levels, dtype=np.int64, copy=True)
        if np.any(levels < 0):
            raise ValueError("face_levels must be non-negative")
    spec_json = None
    if refinement_spec is not None:
        if not isinstance(refinement_spec, Mapping):
            raise ValueError("refinement_spec must be a mapping or None")
        try:
            spec_json = json.dumps(dict(refinement_spec), allow_nan=False, separators=(",", ":"), sort_keys=True)
        except (TypeError, ValueError) as error:
            raise ValueError("refinement_spec must contain JSON-compatible finite values") from error
    kind = topology_kind or ("adaptive" if levels is not None else "custom")
    if kind not in {"uniform", "custom", "adaptive"}:
        raise ValueError("topology_kind must be 'uniform', 'custom', or 'adaptive'")
    if kind == "uniform" and subdivision is None:
        raise ValueError("uniform topology requires subdivision metadata")
    return _assemble(
        coords,
        tri,
        int(subdivision) if subdivision is not None else None,
        topology_kind=kind,
        face_levels=levels,
        refinement_spec_json=spec_json,
        require_well_centered=require_well_centered,
    )
