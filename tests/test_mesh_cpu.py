"""The reference's mesh tests (tests/test_mesh.py there) on the package's mesh
builder: counts and dual topology, read-only tables, operator identities, edge
diamonds, dual areas as explicit polygon fans, orientations, the edge optimiser,
external vertices and custom topologies with their error messages."""

import numpy as np
import pytest

from ionosphere_fdtd_b200.mesh import (
    build_geodesic_mesh,
    build_geodesic_mesh_from_topology,
    build_geodesic_mesh_from_vertices,
)


@pytest.mark.parametrize("level", range(4))
def test_counts_and_dual_topology(level):
    mesh = build_geodesic_mesh(level)
    assert (mesh.n_vertices, mesh.n_edges, mesh.n_faces) == (10 * 4**level + 2, 30 * 4**level, 20 * 4**level)
    assert np.count_nonzero(mesh.vertex_degree == 5) == 12
    if level > 0:
        assert np.count_nonzero(mesh.vertex_degree == 6) == mesh.n_vertices - 12
    assert np.isclose(mesh.face_solid_angles.sum(), 4 * np.pi)
    assert np.isclose(mesh.dual_cell_solid_angles.sum(), 4 * np.pi)


def test_tables_are_read_only_and_operators_keep_identities():
    mesh = build_geodesic_mesh(1)
    for name in ("vertices", "faces", "edges", "face_edges", "face_edge_signs", "edge_left_faces", "edge_right_faces",
                 "face_centers", "primal_edge_angles", "dual_edge_angles", "face_solid_angles", "dual_cell_solid_angles",
                 "vertex_degree", "face_levels"):
        values = getattr(mesh, name)
        if values is None:
            continue
        with pytest.raises(ValueError, match="read-only"):
            values.flat[0] = values.flat[0]
    assert mesh.face_circulation(np.ones(mesh.n_edges, dtype=np.float32)).dtype == np.float32
    assert np.isclose(mesh.dual_cell_circulation(np.linspace(-1.0, 1.0, mesh.n_edges)).sum(), 0.0)
    mesh2 = build_geodesic_mesh(2)
    assert np.allclose(mesh2.face_circulation(mesh2.edge_difference(np.arange(mesh2.n_vertices, dtype=float))), 0.0)


def test_edge_diamonds_partition_the_sphere_and_their_quadrants_each_diamond():
    mesh = build_geodesic_mesh(3)
    areas = mesh.edge_diamond_solid_angles()
    assert np.all(areas > 0.0) and np.sum(areas) == pytest.approx(4.0 * np.pi, rel=1.0e-12)
    quadrants = mesh.edge_diamond_quadrant_solid_angles()
    assert quadrants.shape == (mesh.n_edges, 4) and np.all(quadrants > 0.0)
    np.testing.assert_allclose(quadrants.sum(axis=1), areas, rtol=2.0e-14, atol=2.0e-16)


def test_dual_areas_equal_ordered_polygon_fans():
    """Each dual cell's solid angle is the fan of spherical triangles (vertex, two
    consecutive circumcentres around it), by the half-angle tangent formula."""

    mesh = build_geodesic_mesh(3)
    expected = np.empty(mesh.n_vertices)
    for v in range(mesh.n_vertices):
        p = mesh.vertices[v]
        centres = mesh.face_centers[np.flatnonzero(np.any(mesh.faces == v, axis=1))]
        axis = np.array((0.0, 1.0, 0.0)) if abs(p[0]) > 0.9 else np.array((1.0, 0.0, 0.0))
        ex = axis - (axis @ p) * p
        ex /= np.linalg.norm(ex)
        ey = np.cross(p, ex)
        flat = centres - (centres @ p)[:, None] * p
        ring = centres[np.argsort(np.arctan2(flat @ ey, flat @ ex))]
        nxt = np.roll(ring, -1, axis=0)
        num = np.abs(np.cross(ring, nxt) @ p)
        den = 1.0 + ring @ p + np.einsum("ij,ij->i", ring, nxt) + nxt @ p
        expected[v] = np.sum(2.0 * np.arctan2(num, den))
    np.testing.assert_allclose(mesh.dual_cell_solid_angles, expected, rtol=0.0, atol=8.0 * np.finfo(np.float64).eps)


def test_polar_orientation_puts_pentagons_at_the_poles():
    native = build_geodesic_mesh(2, orientation="native")
    polar = build_geodesic_mesh(2)
    pentagons = polar.vertices[polar.vertex_degree == 5]
    assert np.max(pentagons[:, 2]) == pytest.approx(1.0) and np.min(pentagons[:, 2]) == pytest.approx(-1.0)
    assert native.vertex_degree[int(np.argmax(native.vertices[:, 2]))] == 6
    assert native.vertex_degree[int(np.argmin(native.vertices[:, 2]))] == 6
    np.testing.assert_allclose(np.sort(native.primal_edge_angles), np.sort(polar.primal_edge_angles))
    np.testing.assert_allclose(np.sort(native.dual_cell_solid_angles), np.sort(polar.dual_cell_solid_angles))
    with pytest.raises(ValueError, match="orientation"):
        build_geodesic_mesh(0, orientation="sideways")
    with pytest.raises(ValueError, match="optimization_steps"):
        build_geodesic_mesh(0, optimization_steps=-1)


def test_edge_optimiser_evens_the_mesh_and_keeps_the_pentagons():
    base = build_geodesic_mesh(3)
    opt = build_geodesic_mesh(3, optimization_steps=1)
    np.testing.assert_array_equal(opt.vertices[base.vertex_degree == 5], base.vertices[base.vertex_degree == 5])
    for name in ("primal_edge_angles", "face_solid_angles", "dual_cell_solid_angles"):
        assert np.std(getattr(opt, name)) < np.std(getattr(base, name)), name

    def jumps(m):
        return np.abs(m.dual_cell_solid_angles[m.edges[:, 0]] - m.dual_cell_solid_angles[m.edges[:, 1]])

    assert np.sqrt(np.mean(jumps(opt) ** 2)) < np.sqrt(np.mean(jumps(base) ** 2))
    assert np.max(jumps(opt)) < np.max(jumps(base))


def test_external_vertices_are_accepted_or_rejected_as_in_the_reference():
    base = build_geodesic_mesh(2)
    rebuilt = build_geodesic_mesh_from_vertices(2, np.round(base.vertices, decimals=10))
    np.testing.assert_array_equal(rebuilt.faces, base.faces)
    np.testing.assert_array_equal(rebuilt.edges, base.edges)
    np.testing.assert_allclose(np.linalg.norm(rebuilt.vertices, axis=1), 1.0)
    assert np.isclose(rebuilt.face_solid_angles.sum(), 4.0 * np.pi)
    with pytest.raises(ValueError, match="shape"):
        build_geodesic_mesh_from_vertices(1, np.ones((4, 3)))
    with pytest.raises(ValueError, match="unit sphere"):
        build_geodesic_mesh_from_vertices(0, np.ones((12, 3)))
    s1 = build_geodesic_mesh(1)
    distorted = s1.vertices.copy()
    distorted[12] = distorted[12] + 0.6 * (distorted[0] - distorted[12])
    distorted[12] /= np.linalg.norm(distorted[12])
    with pytest.raises(ValueError, match="well-centered"):
        build_geodesic_mesh_from_vertices(1, distorted)


def test_custom_closed_topologies_and_their_errors():
    vertices = np.asarray(((1.0, 0, 0), (-1.0, 0, 0), (0, 1.0, 0), (0, -1.0, 0), (0, 0, 1.0), (0, 0, -1.0)))
    faces = np.asarray(((0, 2, 4), (2, 1, 4), (1, 3, 4), (3, 0, 4), (2, 0, 5), (1, 2, 5), (3, 1, 5), (0, 3, 5)))
    spec = {"regions": [{"level": 3, "radius_deg": 10.0}]}
    mesh = build_geodesic_mesh_from_topology(vertices, faces[:, ::-1], subdivision=3, face_levels=np.full(8, 3),
                                             refinement_spec=spec)
    assert mesh.topology_kind == "adaptive" and mesh.subdivision == 3
    assert (mesh.n_vertices, mesh.n_edges, mesh.n_faces) == (6, 12, 8)
    assert np.all(mesh.vertex_degree == 4) and np.all(mesh.face_levels == 3)
    assert mesh.refinement_spec == spec
    assert np.isclose(mesh.face_solid_angles.sum(), 4.0 * np.pi)
    assert np.isclose(mesh.dual_cell_solid_angles.sum(), 4.0 * np.pi)
    assert not mesh.faces.flags.writeable and not mesh.face_levels.flags.writeable
    base = build_geodesic_mesh(0)
    with pytest.raises(RuntimeError, match="closed two-manifold"):
        build_geodesic_mesh_from_topology(base.vertices, base.faces[:-1])
    bad = base.faces.copy()
    bad[0, 0] = len(base.vertices)
    with pytest.raises(ValueError, match="out of bounds"):
        build_geodesic_mesh_from_topology(base.vertices, bad)
    with pytest.raises(ValueError, match="face_levels"):
        build_geodesic_mesh_from_topology(base.vertices, base.faces, face_levels=np.zeros(len(base.faces) - 1))
    with pytest.raises(ValueError, match="refinement_spec"):
        build_geodesic_mesh_from_topology(base.vertices, base.faces, refinement_spec={"radius": np.nan})
