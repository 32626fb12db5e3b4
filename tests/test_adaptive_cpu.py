"""Adaptive (locally refined) meshes: the builder against meshes the
reference's own builder produced (``tests/golden/adaptive_meshes.npz``, made by
``tests/golden/make_adaptive_golden.py``), bit for bit, and the invariants and
input checks of the reference's tests (tests/test_adaptive_mesh.py)."""

import numpy as np
import pytest

from make_adaptive_golden import ADAPTIVE_CASES, FLIP_POSITION, FLIP_VERTEX, MESH_ARRAYS

import ionosphere_fdtd_b200 as P
from ionosphere_fdtd_b200.adaptive_mesh import SphericalRefinementRegion, _enforce_local_delaunay, build_adaptive_geodesic_mesh, validate_adaptive_mesh

GOLDEN = np.load(__import__("pathlib").Path(__file__).parent / "golden" / "adaptive_meshes.npz")


@pytest.mark.parametrize("name", sorted(ADAPTIVE_CASES))
def test_adaptive_mesh_is_bit_exact_with_the_reference_builder(name):
    base, regions, options = ADAPTIVE_CASES[name]
    mesh = build_adaptive_geodesic_mesh(base, tuple(SphericalRefinementRegion(*r) for r in regions), **options)
    assert mesh.topology_kind == "adaptive"
    for key in MESH_ARRAYS:
        np.testing.assert_array_equal(np.asarray(getattr(mesh, key)), GOLDEN[f"{name}/{key}"], err_msg=key)
    assert int(np.bincount(mesh.edges.ravel()).max()) == int(GOLDEN[f"{name}/max_degree"])


def test_lawson_flips_are_the_reference_flips_and_repair_the_mesh():
    base = P.build_geodesic_mesh(1)
    vertices = base.vertices.copy()
    vertices[FLIP_VERTEX] = FLIP_POSITION
    levels = np.ones(base.n_faces, dtype=np.int64)
    invalid = P.build_geodesic_mesh_from_topology(vertices, base.faces, face_levels=levels, require_well_centered=False)
    with pytest.raises(ValueError, match="non-positive"):
        validate_adaptive_mesh(invalid)
    faces, repaired = _enforce_local_delaunay(vertices, base.faces, levels)
    np.testing.assert_array_equal(faces, GOLDEN["flip/faces"])
    np.testing.assert_array_equal(repaired, GOLDEN["flip/levels"])
    mesh = P.build_geodesic_mesh_from_topology(vertices, faces, face_levels=repaired, require_well_centered=False)
    assert validate_adaptive_mesh(mesh).minimum_dual_edge_angle > 0.0


def test_disabled_adaptation_is_the_uniform_mesh():
    expected = P.build_geodesic_mesh(2)
    actual = build_adaptive_geodesic_mesh(2, ())
    assert actual.topology_kind == "uniform"
    np.testing.assert_array_equal(actual.vertices, expected.vertices)
    np.testing.assert_array_equal(actual.faces, expected.faces)
    np.testing.assert_array_equal(actual.dual_edge_angles, expected.dual_edge_angles)


def test_refinement_is_conforming_balanced_and_closes_on_the_sphere():
    mesh = build_adaptive_geodesic_mesh(1, (SphericalRefinementRegion(35.0, 126.0, 8.0, 3, 8.0, "source"),))
    v = validate_adaptive_mesh(mesh)
    assert set(np.unique(mesh.face_levels)) == {1, 2, 3}
    assert v.maximum_adjacent_level_jump <= 1 and v.minimum_dual_edge_angle > 0.0
    assert v.primal_area_error < 1e-12 and v.dual_area_error < 1e-12
    assert mesh.refinement_spec["regions"][0]["label"] == "source"
    values = np.arange(mesh.n_vertices, dtype=np.float64)
    assert not np.any(mesh.face_circulation(mesh.edge_difference(values)))


def test_refinement_inputs_are_checked_with_the_reference_messages():
    with pytest.raises(ValueError, match="latitude"):
        SphericalRefinementRegion(91.0, 0.0, 5.0, 2)
    with pytest.raises(ValueError, match="radius"):
        SphericalRefinementRegion(0.0, 0.0, 0.0, 2)
    with pytest.raises(ValueError, match="target subdivision"):
        SphericalRefinementRegion(0.0, 0.0, 5.0, -1)
    with pytest.raises(ValueError, match="regions"):
        build_adaptive_geodesic_mesh(1, [])
    with pytest.raises(ValueError, match="relaxations_per_level"):
        build_adaptive_geodesic_mesh(1, (), relaxations_per_level=0)
    with pytest.raises(ValueError, match="optimization_steps_per_level"):
        build_adaptive_geodesic_mesh(1, (), optimization_steps_per_level=-1)


def test_two_labelled_regions_reach_their_levels_with_positive_supports():
    """tests/test_adaptive_mesh.py:67-96 of the reference."""


    regions = (SphericalRefinementRegion(46.5, -90.9, 6.0, 2, 6.0, "source"), SphericalRefinementRegion(69.0, -156.0, 6.0, 2, 6.0, "oil"))
    mesh = build_adaptive_geodesic_mesh(1, regions)
    for region in regions:
        assert mesh.face_levels[int(np.argmax(mesh.face_centers @ region.direction()))] == region.target_subdivision
    assert [r["label"] for r in mesh.refinement_spec["regions"]] == ["source", "oil"]
    deep = build_adaptive_geodesic_mesh(1, (SphericalRefinementRegion(46.5, -90.9, 8.0, 3, 8.0, "source"),
                                            SphericalRefinementRegion(69.0, -156.0, 8.0, 3, 8.0, "oil")))
    assert validate_adaptive_mesh(deep).minimum_dual_edge_angle > 0.0
    assert np.all(deep.dual_cell_solid_angles > 0.0) and np.all(deep.edge_diamond_solid_angles() > 0.0)
    assert np.sum(deep.edge_diamond_solid_angles()) == pytest.approx(4.0 * np.pi)


def test_default_relaxation_keeps_transition_dual_edges_open():
    """tests/test_adaptive_mesh.py:98-113 of the reference."""


    mesh = build_adaptive_geodesic_mesh(3, (SphericalRefinementRegion(46.5, -90.9, 3.0, 5, 3.0, "source"),
                                            SphericalRefinementRegion(69.0, -156.0, 3.0, 5, 3.0, "oil")))
    assert validate_adaptive_mesh(mesh).minimum_dual_to_primal_ratio > 0.05
    spec = mesh.refinement_spec
    assert spec["algorithm"] == "conforming-red-transition-v3"
    assert spec["relaxations_per_level"] == 4 and spec["optimization_steps_per_level"] == 0
