"""Conforming local refinement of geodesic meshes (adaptive_mesh.py:1-553).

A refined mesh is built from a uniform base level by repeated rounds:
faces whose desired level (from circular refinement regions with optional
transition rings) exceeds their own are split into four; their neighbours get
a two- or three-child transition triangulation so no hanging midpoint
remains; the vertices of the touched faces are relaxed towards the centroid
of their incident face centres; and Lawson edge flips restore a positive
circumcentric dual edge everywhere.  The vertex coordinates, face list and
face levels are bit-exact with the reference builder: each floating-point
step is the reference's, in the same order, and midpoints, children and flips
are numbered and ordered as the reference numbers them.  The resulting mesh
feeds the same step kernels as a uniform one (transition vertices reach
degree 7 or 8, served by the kernels' 12-slot vertex tables).
"""

from __future__ import annotations

from collections import deque
from dataclasses import asdict, dataclass

import numpy as np
from numpy.typing import NDArray

from .mesh import (
    GeodesicMesh,
    _arc,
    _circumcentres,
    _edge_tables,
    _first_use_numbering,
    _relax,
    _unit,
    build_geodesic_mesh,
    build_geodesic_mesh_from_topology,
)

FloatArray = NDArray[np.float64]
IntArray = NDArray[np.int64]


def _is_int(value) -> bool:
    return not isinstance(value, bool) and isinstance(value, (int, np.integer))


@dataclass(frozen=True, slots=True)
class SphericalRefinementRegion:
    """A circular fine core with optional equal-width transition rings
    (adaptive_mesh.py:24-75)."""

    latitude_deg: float
    longitude_deg: float
    radius_deg: float
    target_subdivision: int
    transition_width_deg: float = 0.0
    label: str = ""

    def __post_init__(self) -> None:
        values = np.asarray((self.latitude_deg, self.longitude_deg, self.radius_deg, self.transition_width_deg), dtype=np.float64)
        if not np.all(np.isfinite(values)):
            raise ValueError("refinement-region coordinates and widths must be finite")
        if not -90.0 <= self.latitude_deg <= 90.0:
            raise ValueError("refinement-region latitude must be in [-90, 90]")
        if not 0.0 < self.radius_deg <= 180.0:
            raise ValueError("refinement-region radius must be in (0, 180]")
        if not 0.0 <= self.transition_width_deg <= 180.0:
            raise ValueError("transition width must be in [0, 180]")
        if not _is_int(self.target_subdivision) or self.target_subdivision < 0:
            raise ValueError("target subdivision must be a non-negative integer")
        if not isinstance(self.label, str):
            raise ValueError("refinement-region label must be a string")

    def direction(self) -> FloatArray:
        """Unit Cartesian direction of the region centre."""

        lat = np.deg2rad(self.latitude_deg)
        lon = np.deg2rad(self.longitude_deg)
        return np.asarray((np.cos(lat) * np.cos(lon), np.cos(lat) * np.sin(lon), np.sin(lat)))


@dataclass(frozen=True, slots=True)
class AdaptiveMeshValidation:
    """Invariant measurements of a conforming adaptive mesh (adaptive_mesh.py:77-85)."""

    maximum_adjacent_level_jump: int
    minimum_dual_edge_angle: float
    minimum_dual_to_primal_ratio: float
    primal_area_error: float
    dual_area_error: float


def build_adaptive_geodesic_mesh(
    base_subdivision: int,
    regions: tuple[SphericalRefinementRegion, ...],
    *,
    orientation: str = "polar",
    relaxations_per_level: int = 4,
    optimization_steps_per_level: int = 0,
) -> GeodesicMesh:
    """One closed mesh with conforming local refinement (adaptive_mesh.py:88-186).

    Without a region finer than the base level the uniform base mesh is
    returned unchanged."""

    if not _is_int(base_subdivision) or base_subdivision < 0:
        raise ValueError("base subdivision must be a non-negative integer")
    if not _is_int(relaxations_per_level) or relaxations_per_level < 1:
        raise ValueError("relaxations_per_level must be a positive integer")
    if not _is_int(optimization_steps_per_level) or optimization_steps_per_level < 0:
        raise ValueError("optimization_steps_per_level must be a non-negative integer")
    if not isinstance(regions, tuple) or not all(isinstance(r, SphericalRefinementRegion) for r in regions):
        raise ValueError("regions must be a tuple of SphericalRefinementRegion")

    base = build_geodesic_mesh(int(base_subdivision), orientation=orientation)
    active = tuple(r for r in regions if r.target_subdivision > base_subdivision)
    if not active:
        return base
    vertices = np.array(base.vertices, copy=True)
    faces = np.array(base.faces, copy=True)
    levels = np.full(len(faces), base_subdivision, dtype=np.int64)
    for _ in range(base_subdivision, max(r.target_subdivision for r in active)):
        marked = _desired_face_levels(vertices, faces, active) > levels
        if not np.any(marked):
            break
        first_new = len(vertices)
        vertices, faces, levels = _refine_marked_faces(vertices, faces, levels, marked)
        touched = np.any(faces >= first_new, axis=1)
        movable = np.zeros(len(vertices), dtype=np.bool_)
        movable[np.unique(faces[touched])] = True
        for _ in range(int(relaxations_per_level)):
            vertices = _relax_selected(vertices, faces, movable)
        if optimization_steps_per_level:
            vertices = _optimize_selected_edge_lengths(vertices, faces, movable, int(optimization_steps_per_level))
        faces, levels = _enforce_local_delaunay(vertices, faces, levels)

    spec = {
        "algorithm": "conforming-red-transition-v3",
        "base_subdivision": int(base_subdivision),
        "orientation": orientation,
        "relaxations_per_level": int(relaxations_per_level),
        "optimization_steps_per_level": int(optimization_steps_per_level),
        "regions": [asdict(r) for r in regions],
    }
    mesh = build_geodesic_mesh_from_topology(
        vertices,
        faces,
        subdivision=int(base_subdivision),
        face_levels=levels,
        refinement_spec=spec,
        topology_kind="adaptive",
        normalize_vertices=False,
        require_well_centered=False,
    )
    validate_adaptive_mesh(mesh)
    return mesh


def _signed_dual_angles(vertices: FloatArray, edges: IntArray, left_centres: FloatArray, right_centres: FloatArray) -> FloatArray:
    """Dual-edge angle from the left to the right circumcentre, measured in
    the edge's midpoint frame (adaptive_mesh.py:198-210, 396-408)."""

    tail = vertices[edges[:, 0]]
    head = vertices[edges[:, 1]]
    mid = _unit(tail + head)
    normal = _unit(np.cross(tail, head))
    left = np.arctan2(np.einsum("ij,ij->i", left_centres, normal), np.einsum("ij,ij->i", left_centres, mid))
    right = np.arctan2(np.einsum("ij,ij->i", right_centres, normal), np.einsum("ij,ij->i", right_centres, mid))
    return left - right


def validate_adaptive_mesh(mesh: GeodesicMesh) -> AdaptiveMeshValidation:
    """2:1 level balance, area closure and a positive Hodge star
    (adaptive_mesh.py:189-248), with the reference's messages."""

    if mesh.face_levels is None:
        raise ValueError("adaptive mesh validation requires face_levels")
    jump = np.abs(mesh.face_levels[mesh.edge_left_faces] - mesh.face_levels[mesh.edge_right_faces])
    max_jump = int(np.max(jump, initial=0))
    if max_jump > 1:
        raise ValueError("adaptive mesh violates 2:1 face-level balance")
    signed = _signed_dual_angles(
        mesh.vertices, mesh.edges, mesh.face_centers[mesh.edge_left_faces], mesh.face_centers[mesh.edge_right_faces]
    )
    min_dual = float(np.min(signed))
    min_ratio = float(np.min(signed / mesh.primal_edge_angles))
    tol = 64.0 * np.finfo(np.float64).eps
    if min_dual <= tol:
        raise ValueError("adaptive mesh has a non-positive circumcentric Hodge star")
    if not np.allclose(signed, mesh.dual_edge_angles, rtol=1.0e-12, atol=tol):
        raise ValueError("adaptive mesh dual-edge orientation is inconsistent")
    primal_error = float(abs(np.sum(mesh.face_solid_angles) - 4.0 * np.pi))
    dual_error = float(abs(np.sum(mesh.dual_cell_solid_angles) - 4.0 * np.pi))
    if primal_error > 1.0e-11 or dual_error > 1.0e-10:
        raise ValueError("adaptive mesh areas do not close on the sphere")
    supports = mesh.edge_diamond_solid_angles()
    if np.any(supports <= 0.0) or not np.isclose(np.sum(supports), 4.0 * np.pi, rtol=0.0, atol=1.0e-10):
        raise ValueError("adaptive edge supports are not positive and disjoint")
    return AdaptiveMeshValidation(max_jump, min_dual, min_ratio, primal_error, dual_error)


def _desired_face_levels(vertices: FloatArray, faces: IntArray, regions) -> IntArray:
    """Requested level per face: the region target inside a core (distance
    from the region centre to the face's nearest possible point), one level
    less per transition ring outside it (adaptive_mesh.py:251-283)."""

    centres = _circumcentres(vertices, faces)
    radius = np.max(_arc(np.repeat(centres, 3, axis=0), vertices[faces].reshape(-1, 3)).reshape(-1, 3), axis=1)
    desired = np.zeros(len(faces), dtype=np.int64)
    for region in regions:
        distance = np.arccos(np.clip(centres @ region.direction(), -1.0, 1.0))
        effective = np.rad2deg(np.maximum(distance - radius, 0.0))
        requested = np.full(len(faces), -1, dtype=np.int64)
        core = effective <= region.radius_deg
        requested[core] = region.target_subdivision
        if region.transition_width_deg > 0.0:
            outside = ~core
            rings = np.ceil((effective[outside] - region.radius_deg) / region.transition_width_deg).astype(np.int64)
            requested[outside] = region.target_subdivision - rings
        desired = np.maximum(desired, requested)
    return desired


def _refine_marked_faces(vertices: FloatArray, faces: IntArray, levels: IntArray, marked) -> tuple[FloatArray, IntArray, IntArray]:
    """Red refinement of the marked faces and transition children for their
    neighbours (adaptive_mesh.py:286-334, children 337-365).  Midpoints are
    numbered in face-scan order of first use, as the reference's dict does."""

    n = len(vertices)
    p = faces
    q = np.roll(faces, -1, axis=1)  # edges (a, b), (b, c), (c, a)
    lo = np.minimum(p, q)
    hi = np.maximum(p, q)
    key = lo * np.int64(n) + hi
    split = np.isin(key, np.unique(key[marked]))
    rank, first = _first_use_numbering(lo[split], hi[split], n)
    mids = np.full(faces.shape, -1, dtype=np.int64)
    mids[split] = n + rank
    s_lo, s_hi = lo[split][first], hi[split][first]
    points = _unit(vertices[s_lo] + vertices[s_hi])
    a, b, c = faces[:, 0], faces[:, 1], faces[:, 2]
    ab, bc, ca = mids[:, 0], mids[:, 1], mids[:, 2]
    s0, s1, s2 = split[:, 0], split[:, 1], split[:, 2]
    count = split.sum(axis=1)
    n_children = np.asarray((1, 2, 3, 4))[count]
    start = np.concatenate(([0], np.cumsum(n_children)[:-1]))
    out = np.empty((int(n_children.sum()), 3), dtype=np.int64)

    def put(mask, k, x, y, z):
        rows = start[mask] + k
        out[rows, 0], out[rows, 1], out[rows, 2] = x[mask], y[mask], z[mask]

    m = count == 0
    put(m, 0, a, b, c)
    m = count == 3
    put(m, 0, a, ab, ca)
    put(m, 1, b, bc, ab)
    put(m, 2, c, ca, bc)
    put(m, 3, ab, bc, ca)
    one = count == 1
    m = one & s0
    put(m, 0, a, ab, c)
    put(m, 1, ab, b, c)
    m = one & s1
    put(m, 0, b, bc, a)
    put(m, 1, bc, c, a)
    m = one & s2
    put(m, 0, c, ca, b)
    put(m, 1, ca, a, b)
    two = count == 2
    # the unsplit edge decides the corner roles (x, y, z, xy, yz)
    for mask, (x, y, z, xy, yz) in (
        (two & ~s0, (b, c, a, bc, ca)),
        (two & s0 & ~s1, (c, a, b, ca, ab)),
        (two & s0 & s1, (a, b, c, ab, bc)),
    ):
        put(mask, 0, y, yz, xy)
        put(mask, 1, x, xy, z)
        put(mask, 2, xy, yz, z)
    new_levels = np.repeat(levels + (count > 0), n_children)
    return np.concatenate((vertices, points)), out, new_levels.astype(np.int64)


def _relax_selected(vertices: FloatArray, faces: IntArray, movable) -> FloatArray:
    """One centroid relaxation of the movable vertices only (adaptive_mesh.py:368-382)."""

    proposed = _relax(vertices, faces)
    result = np.array(vertices, copy=True)
    result[movable] = proposed[movable]
    return result


def _optimize_selected_edge_lengths(vertices: FloatArray, faces: IntArray, movable, steps: int) -> FloatArray:
    """Projected edge-length equalisation of the movable, non-pentagon
    vertices (adaptive_mesh.py:385-426)."""

    edges = _edge_tables(faces, len(vertices))[0]
    degree = np.bincount(edges.ravel(), minlength=len(vertices))
    selected = movable & (degree != 5)
    result = np.array(vertices, copy=True)
    tails, heads = edges[:, 0], edges[:, 1]
    for _ in range(steps):
        t = result[tails]
        h = result[heads]
        dot = np.clip(np.einsum("ij,ij->i", t, h), -1.0, 1.0)
        sine = np.linalg.norm(np.cross(t, h), axis=1)
        lengths = np.arctan2(sine, dot)
        residual = lengths - float(np.mean(lengths))
        g_tail = residual[:, None] * (dot[:, None] * t - h) / sine[:, None]
        g_head = residual[:, None] * (dot[:, None] * h - t) / sine[:, None]
        gradient = np.zeros_like(result)
        np.add.at(gradient, tails, g_tail)
        np.add.at(gradient, heads, g_head)
        gradient /= degree[:, None]
        gradient -= np.einsum("ij,ij->i", gradient, result)[:, None] * result
        updated = _unit(result - gradient)
        result[selected] = updated[selected]
    return result


def _sorted_edges(face) -> tuple[tuple[int, int], tuple[int, int], tuple[int, int]]:
    a, b, c = (int(v) for v in face)
    return (tuple(sorted((a, b))), tuple(sorted((b, c))), tuple(sorted((c, a))))


def _enforce_local_delaunay(vertices: FloatArray, faces: IntArray, levels: IntArray) -> tuple[IntArray, IntArray]:
    """Lawson flips until every circumcentric dual edge is positive
    (adaptive_mesh.py:429-553).  The work queue starts with the failing edges
    in edge order; a flip re-queues the edges of both new faces in the
    reference's set order, so the flips, and the faces they produce, are the
    reference's."""

    result = np.array(faces, dtype=np.int64, copy=True)
    result_levels = np.array(levels, dtype=np.int64, copy=True)
    edges, _, _, left_faces, right_faces = _edge_tables(result, len(vertices))
    adjacency: dict[tuple[int, int], list[int]] = {}
    for edge, lf, rf in zip(edges, left_faces, right_faces):
        adjacency[(int(edge[0]), int(edge[1]))] = [int(lf), int(rf)]
    centres = _circumcentres(vertices, result)
    signed = _signed_dual_angles(vertices, edges, centres[left_faces], centres[right_faces])
    tol = 256.0 * np.finfo(np.float64).eps
    work = deque((int(e[0]), int(e[1])) for e in edges[signed <= tol])
    queued = set(work)
    max_flips = max(1, 10 * len(adjacency))
    flips = 0

    def follows(face, tail: int, head: int) -> bool:
        return any(int(face[k]) == tail and int(face[(k + 1) % 3]) == head for k in range(3))

    while work:
        edge = work.popleft()
        queued.remove(edge)
        adjacent = adjacency.get(edge)
        if adjacent is None or len(adjacent) != 2:
            continue
        i1, i2 = adjacent
        a, b = edge
        f1, f2 = result[i1], result[i2]
        if follows(f1, b, a):
            i1, i2 = i2, i1
            f1, f2 = f2, f1
        if not follows(f1, a, b) or not follows(f2, b, a):
            raise RuntimeError("adaptive face orientations are inconsistent")
        c = next(int(v) for v in f1 if v not in edge)
        d = next(int(v) for v in f2 if v not in edge)
        pair = _circumcentres(vertices, np.asarray((f1, f2), dtype=np.int64))
        mid = _unit((vertices[a] + vertices[b])[None, :])[0]
        normal = _unit(np.cross(vertices[a], vertices[b])[None, :])[0]
        coords = np.arctan2(pair @ normal, pair @ mid)
        if coords[0] - coords[1] > tol:
            continue
        replacement = tuple(sorted((c, d)))
        if replacement in adjacency:
            continue
        for old in set(_sorted_edges(f1)) | set(_sorted_edges(f2)):
            nb = adjacency[old]
            nb[:] = [i for i in nb if i not in {i1, i2}]
            if not nb:
                del adjacency[old]
        result[i1] = (c, d, b)
        result[i2] = (d, c, a)
        lvl = max(int(result_levels[i1]), int(result_levels[i2]))
        result_levels[i1] = lvl
        result_levels[i2] = lvl
        changed = set(_sorted_edges(result[i1])) | set(_sorted_edges(result[i2]))
        for ce in changed:
            nb = adjacency.setdefault(ce, [])
            for i in (i1, i2):
                if ce in _sorted_edges(result[i]) and i not in nb:
                    nb.append(i)
            if ce not in queued:
                queued.add(ce)
                work.append(ce)
        if any(len(adjacency[ce]) != 2 for ce in changed):
            raise RuntimeError("Delaunay flip broke the closed mesh topology")
        flips += 1
        if flips > max_flips:
            raise RuntimeError("adaptive Delaunay edge flips did not converge")
    return result, result_levels
