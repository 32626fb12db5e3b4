"""Surface-eigenmode helpers shared by the CPU and GPU invariant tests: the TM-r
and TE-r surface operators of the mesh, one of their l = 1 eigenvectors, and
the exact leapfrog dispersion of its amplitude (the reference's
tests/test_maxwell_invariants.py:60-163)."""

import numpy as np

from ionosphere_fdtd_b200.constants import C_0

# a shell thin against a huge radius, so the radial metric leaves the surface modes alone
SURFACE_MODE = dict(subdivision=1, radial_cells=2, minimum_altitude_m=-1.0e9, maximum_altitude_m=1.0e9,
                    earth_radius_m=1.0e10, courant_factor=0.8)


class Vacuum:
    """sigma = 0, relative permittivity 1 everywhere."""

    def sample(self, directions, altitudes_m, earth_radius_m):
        shape = (len(directions), len(altitudes_m))
        return np.zeros(shape), np.ones(shape)


def tm_operator(mesh, values):
    """Circumcentric finite-volume Laplacian on the unit sphere: dual/primal weighted
    edge differences summed around each dual cell, over its solid angle."""

    flux = mesh.dual_edge_angles / mesh.primal_edge_angles * mesh.edge_difference(values)
    return mesh.dual_cell_circulation(flux) / mesh.dual_cell_solid_angles


def te_operator(mesh, values):
    """The face counterpart: primal/dual weighted dual differences around each face."""

    grad = mesh.primal_edge_angles / mesh.dual_edge_angles * mesh.dual_edge_difference(values)
    return mesh.face_circulation(grad) / mesh.face_solid_angles


def surface_mode(mesh, kind: str):
    """A real eigenvector of the TM (vertex) or TE (face) operator with eigenvalue
    near the l = 1 value (-2 for TM, +2 for TE), and minus that eigenvalue's sign."""

    n = mesh.n_vertices if kind == "tm" else mesh.n_faces
    apply = (lambda v: tm_operator(mesh, v)) if kind == "tm" else (lambda v: te_operator(mesh, v))
    eye = np.eye(n)
    matrix = np.column_stack([apply(eye[:, i]) for i in range(n)])
    values, vectors = np.linalg.eig(matrix)
    target = -2.0 if kind == "tm" else 2.0
    pick = int(np.argmin(np.abs(values.real - target)))
    eigen = -float(values[pick].real) if kind == "tm" else float(values[pick].real)
    return eigen, vectors[:, pick].real


def expected_amplitudes(eigen, dt, radius, steps, offset):
    q = (C_0 * dt) ** 2 * eigen / radius**2
    phase = np.arccos(1.0 - 0.5 * q)
    n = np.arange(steps + 1)
    return np.cos((n + offset) * phase) / np.cos(0.5 * phase)


class UniformConductive(Vacuum):
    """One conductivity everywhere, vacuum permittivity."""

    def __init__(self, conductivity_s_m: float) -> None:
        self.conductivity_s_m = conductivity_s_m

    def sample(self, directions, altitudes_m, earth_radius_m):
        sigma, eps = super().sample(directions, altitudes_m, earth_radius_m)
        sigma.fill(self.conductivity_s_m)
        return sigma, eps


class UniformPermittivity(Vacuum):
    """One relative permittivity everywhere, no conductivity."""

    def __init__(self, relative_permittivity: float) -> None:
        self.relative_permittivity = relative_permittivity

    def sample(self, directions, altitudes_m, earth_radius_m):
        sigma, eps = super().sample(directions, altitudes_m, earth_radius_m)
        eps.fill(self.relative_permittivity)
        return sigma, eps


# an abruptly graded radial grid (the reference's nonuniform-stencil cases)
GRADED_ALTITUDES = (-10_000.0, -6_000.0, -2_000.0, -1_000.0, 0.0, 4_000.0)


def extreme_surface_eigenvalues(mesh) -> tuple[float, float]:
    """The largest |eigenvalue| of the TM (vertex) and TE (face) surface operators."""

    tm = np.column_stack([tm_operator(mesh, e) for e in np.eye(mesh.n_vertices)])
    te = np.column_stack([te_operator(mesh, e) for e in np.eye(mesh.n_faces)])
    return -float(np.linalg.eigvals(tm).real.min()), float(np.linalg.eigvals(te).real.max())


def courant_numbers(mesh, dt, node_radius_min, mid_radius_min) -> tuple[float, float]:
    """(c dt / r)^2 x the extreme surface eigenvalues: leapfrog is stable below 4."""

    tm, te = extreme_surface_eigenvalues(mesh)
    return (C_0 * dt / node_radius_min) ** 2 * tm, (C_0 * dt / mid_radius_min) ** 2 * te


def tangential_moment_error(simulation, source, line_length):
    """Reconstruct the (east, north) line moments from the covariant edge samples
    of a tangential source and return their error (tests/test_maxwell_invariants.py:165-217)."""

    from ionosphere_fdtd_b200.sources import geographic_tangent_basis

    edges, _, weights = source.edge_distribution(simulation)
    unique = np.unique(edges)
    ends = simulation.mesh.vertices[simulation.mesh.edges[unique]]
    dirs = ends[:, 1] - ends[:, 0]
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    lengths = simulation.mesh.primal_edge_angles[unique] * simulation.config.earth_radius_m
    samples = np.asarray([weights[edges == e].sum() * ln for e, ln in zip(unique, lengths, strict=True)])
    east, north = geographic_tangent_basis(source.latitude_deg, source.longitude_deg)
    moments = np.linalg.pinv(np.column_stack((dirs @ east, dirs @ north))) @ samples
    return np.abs(moments - line_length).max()


def tangential_case():
    line = 22_500.0
    from ionosphere_fdtd_b200 import TangentialGaussianCurrent

    source = TangentialGaussianCurrent(latitude_deg=46.5, longitude_deg=-90.9, altitude_m=0.0, azimuths_deg=(0.0, 90.0),
                                         line_lengths_m=(line, line))
    return source, line
