"""The reference's host-side plasma tests (tests/test_plasma.py there) on the
package's model, reconstruction tables and ADE, with NumPy arrays standing in for
device arrays; and the array-level ADE update against the oracle's."""

import numpy as np
import pytest

from casebuild import product_provenance

import ionosphere_fdtd_b200 as P
from ionosphere_fdtd_b200 import plasma as PL


class HostArrays:
    dtype_name = "float64"

    def asarray(self, values):
        return np.asarray(values, dtype=np.float64)

    def zeros(self, shape):
        return np.zeros(shape, dtype=np.float64)

    def empty_like(self, values):
        return np.empty_like(values)

    def nbytes(self, values):
        return values.nbytes


def model(magnetic_t=50.0e-6, density_m3=1.0e3, collision_hz=200.0, mesh=None, altitudes=(25_000.0, 75_000.0)):
    mesh = P.build_geodesic_mesh(0) if mesh is None else mesh
    h = np.asarray(altitudes)
    shape = (mesh.n_faces, len(h))
    magnetic = np.zeros((*shape, 3))
    magnetic[..., 2] = magnetic_t
    species = P.ColdPlasmaSpecies("electron", -P.ELEMENTARY_CHARGE_C, P.ELECTRON_MASS_KG, np.full(shape, density_m3),
                                  np.full(shape, collision_hz))
    return P.MeshPlasmaModel.from_mesh(mesh, h, magnetic, (species,), provenance=(product_provenance(),),
                                       interpolation="synthetic constants")


def test_conductivity_tensor_isotropic_without_field_and_passive_with_it():
    parallel, pedersen, hall = model(magnetic_t=0.0).conductivity_components(20.0)
    np.testing.assert_allclose(pedersen, parallel, rtol=3.0e-16, atol=0.0)
    np.testing.assert_array_equal(hall, 0.0)
    assert np.all(parallel.real > 0.0)
    parallel, pedersen, hall = model().conductivity_components(20.0)
    assert np.all(parallel.real > 0.0) and np.all(pedersen.real > 0.0) and np.all(hall.real < 0.0)
    assert np.max(np.abs(hall)) > np.max(np.abs(pedersen))


def test_face_reconstruction_recovers_tangent_vectors():
    mesh = P.build_geodesic_mesh(1)
    recon, tangents = PL.face_reconstruction(mesh)
    vector = np.asarray((0.3, -0.4, 0.5))
    tangent = vector - (mesh.face_centers @ vector)[:, None] * mesh.face_centers
    samples = np.sum(tangents * tangent[:, None, :], axis=2)
    np.testing.assert_allclose(np.sum(samples[:, :, None] * recon, axis=1), tangent, rtol=0.0, atol=8.0e-16)


def test_vector_ade_matches_the_complex_tensor_response():
    full = model(magnetic_t=1.0e-8, density_m3=1.0e6)
    sp = full.species[0]
    one = P.MeshPlasmaModel(
        mesh_vertices_sha256=full.mesh_vertices_sha256, mesh_faces_sha256=full.mesh_faces_sha256,
        radial_midpoint_altitudes_m=np.asarray((25_000.0,)), magnetic_field_t=full.magnetic_field_t[:1, :1],
        species=(P.ColdPlasmaSpecies("electron", sp.charge_c, sp.mass_kg, sp.number_density_m3[:1, :1],
                                     sp.collision_frequency_hz[:1, :1]),),
        provenance=full.provenance, interpolation=full.interpolation)
    dt, freq, n = 1.0e-5, 20.0, 100_000
    ade = PL.MagnetizedPlasmaADE(one, dt, HostArrays())
    electric = np.zeros((1, 1, 3))
    current = np.empty((n, 2))
    drive = np.cos(2.0 * np.pi * freq * np.arange(n) * dt)
    for k in range(n):
        electric[..., 0] = drive[k]
        current[k] = ade.advance(electric)[0, 0, :2]
    tail = slice(n - 20_000, None)
    basis = np.exp(-2j * np.pi * freq * (np.arange(n)[tail] * dt + dt))
    den = np.sum(drive[tail] * basis)
    _, pedersen, hall = one.conductivity_components(freq)
    assert np.sum(current[tail, 0] * basis) / den == pytest.approx(pedersen[0, 0], rel=2.0e-3)
    assert np.sum(current[tail, 1] * basis) / den == pytest.approx(-hall[0, 0], rel=2.0e-3)


def test_array_level_ade_update_equals_the_oracle():
    """Two magnetised species on a level-1 mesh: ``advance`` against the oracle's
    species update (plasma.py:413-442), state and summed current."""

    import cases as C
    from casebuild import build_oracle, plasma_arrays

    case = C.CASES["plasma_magnetized_s1"]
    ora = build_oracle(case)
    mesh = P.build_geodesic_mesh(case["config"]["subdivision"])
    mids, magnetic, species = plasma_arrays(case["plasma"], mesh.n_faces, case["config"])
    assert len(species) == len(ora.p_coef) == 2
    m = P.MeshPlasmaModel.from_mesh(mesh, mids, magnetic, tuple(P.ColdPlasmaSpecies(f"s{i}", *s) for i, s in enumerate(species)),
                                    provenance=(product_provenance(),), interpolation="synthetic")
    ade = PL.MagnetizedPlasmaADE(m, ora.dt, HostArrays())
    rng = np.random.default_rng(8)
    e = rng.standard_normal((mesh.n_faces, len(mids), 3))
    start = [rng.standard_normal(tuple(j.shape)) for j in ade.current_density]
    for j, s0 in zip(ade.current_density, start):
        j[...] = s0
    total = ade.advance(e)
    # the oracle's own coefficients and field direction, its update formulas
    b = ora.p_b
    e_par = (e * b).sum(axis=2)[..., None] * b
    e_perp = e - e_par
    e_x = ora._cross(e_perp, b)
    want_total = np.zeros_like(e)
    for j, s0, (decay, cs, sn, dpar, dre, dim) in zip(ade.current_density, start, ora.p_coef):
        j_par = (s0 * b).sum(axis=2)[..., None] * b
        j_perp = s0 - j_par
        want = (decay[..., None] * j_par + dpar[..., None] * e_par
                + decay[..., None] * (cs[..., None] * j_perp + sn[..., None] * ora._cross(j_perp, b))
                + dre[..., None] * e_perp + dim[..., None] * e_x)
        np.testing.assert_allclose(j, want, rtol=1e-13, atol=1e-15)
        want_total += want
    np.testing.assert_allclose(total, want_total, rtol=1e-13, atol=1e-15)


@pytest.mark.parametrize("level", [0, 2, 4])
def test_edge_tangents_and_reconstruction_lie_in_the_face_tangent_planes(level):
    """The face frames of the step kernels (component 0 along the face centre, 1 and 2
    in the face's tangent plane) drop the centre component of every edge tangent and
    carry the face centre as (|c|, 0, 0): both rest on the reference's tangents being
    normal to their face's centre (plasma.py:548-559, cross(normal, centre)) and on
    |centre| = 1.  Here the dropped parts are round-off, and the reconstruction rows
    (the pseudo-inverse of the tangents) lie in the tangent planes too."""

    mesh = P.build_geodesic_mesh(level)
    recon, tangents = PL.face_reconstruction(mesh)
    centres = np.asarray(mesh.face_centers)
    np.testing.assert_allclose(np.linalg.norm(centres, axis=1), 1.0, rtol=0, atol=1e-15)
    left = PL.edge_face_slots(mesh, mesh.edge_left_faces)
    right = PL.edge_face_slots(mesh, mesh.edge_right_faces)
    for faces, slots in ((mesh.edge_left_faces, left), (mesh.edge_right_faces, right)):
        t = tangents[faces, slots]
        np.testing.assert_allclose(np.linalg.norm(t, axis=1), 1.0, rtol=0, atol=1e-15)
        assert np.max(np.abs(np.einsum("ec,ec->e", t, centres[faces]))) < 1e-15
    # reconstruction rows: no component along the centre beyond round-off of their own size
    along = np.einsum("fic,fc->fi", recon, centres)
    assert np.max(np.abs(along)) < 1e-14 * np.max(np.abs(recon))
