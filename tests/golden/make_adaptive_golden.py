"""Golden adaptive meshes from the reference's own builder.

Run it where the reference source tree is available, giving the reference's
``src`` directory as the only argument (required):

    python tests/golden/make_adaptive_golden.py <reference>/src

It imports the reference package from the given source directory, builds the
adaptive meshes of ``ADAPTIVE_CASES`` (and one Lawson-flip repair) with the
reference's ``build_adaptive_geodesic_mesh`` / ``_enforce_local_delaunay``, and
writes their vertex coordinates, topology tables, face levels and geometry to
``adaptive_meshes.npz`` next to this script.  No test reads the reference.
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent

# (base subdivision, regions as (lat, lon, radius, target, width, label), builder options)
ADAPTIVE_CASES = {
    "one_region_s1": (1, ((35.0, 126.0, 8.0, 3, 8.0, "source"),), {}),
    "two_regions_s1": (1, ((46.5, -90.9, 8.0, 3, 8.0, "source"), (69.0, -156.0, 8.0, 3, 8.0, "oil")), {}),
    "deep_s2": (2, ((10.0, 20.0, 12.0, 4, 6.0, "core"),), {}),
    "optimized_s1": (1, ((35.0, 126.0, 8.0, 2, 8.0, "opt"),), {"optimization_steps_per_level": 2}),
    "native_s1": (1, ((-20.0, 40.0, 10.0, 3, 10.0, ""),), {"orientation": "native", "relaxations_per_level": 2}),
}

MESH_ARRAYS = (
    "vertices", "faces", "edges", "face_edges", "face_edge_signs", "edge_left_faces", "edge_right_faces",
    "face_levels", "face_centers", "primal_edge_angles", "dual_edge_angles", "face_solid_angles",
    "dual_cell_solid_angles",
)

# The reference's Lawson-flip test: base s1 with vertex 15 moved off its place
FLIP_VERTEX = 15
FLIP_POSITION = (0.3779688486851255, 0.0824166650239095, 0.9221426368789035)


def main(src: str) -> None:
    sys.path.insert(0, src)
    from ionosphere_fdtd import adaptive_mesh as ram
    from ionosphere_fdtd import mesh as rmesh

    out = {}
    for name, (base, regions, options) in ADAPTIVE_CASES.items():
        mesh = ram.build_adaptive_geodesic_mesh(base, tuple(ram.SphericalRefinementRegion(*r) for r in regions), **options)
        for key in MESH_ARRAYS:
            out[f"{name}/{key}"] = np.asarray(getattr(mesh, key))
        out[f"{name}/max_degree"] = np.asarray(np.bincount(mesh.edges.ravel()).max())
    base = rmesh.build_geodesic_mesh(1)
    vertices = base.vertices.copy()
    vertices[FLIP_VERTEX] = FLIP_POSITION
    faces, levels = ram._enforce_local_delaunay(vertices, base.faces, np.ones(base.n_faces, dtype=np.int64))
    out["flip/faces"] = faces
    out["flip/levels"] = levels
    np.savez_compressed(HERE / "adaptive_meshes.npz", **out)
    for name in ADAPTIVE_CASES:
        print(name, out[f"{name}/vertices"].shape[0], "vertices, max degree", int(out[f"{name}/max_degree"]))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_adaptive_golden.py <reference src directory>")
    main(sys.argv[1])
