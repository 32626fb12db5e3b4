"""The reference's configuration and source-waveform validation tests
(tests/test_solver.py there) on the package's SimulationConfig,
GaussianCurrent and TangentialGaussianCurrent: the same rejections with the
same message keys, and the default source."""

import numpy as np
import pytest

from ionosphere_fdtd_b200 import GaussianCurrent, SimulationConfig, TangentialGaussianCurrent


def config(**changes):
    values = dict(subdivision=1, radial_cells=6, courant_factor=0.25)
    values.update(changes)
    return SimulationConfig(**values)


@pytest.mark.parametrize(
    "changes, message",
    [
        (dict(mesh_relaxations=-1), "mesh_relaxations"),
        (dict(mesh_optimization_steps=-1), "mesh_optimization_steps"),
        (dict(time_step_s=np.nan), "finite"),
        (dict(earth_radius_m=np.nan), "finite"),
        (dict(radial_altitudes_m=(-100_000.0, 0.0, 100_000.0)), "radial_cells"),
        (dict(mesh_orientation="sideways"), "mesh_orientation"),
        (dict(tangential_material_support="unknown"), "tangential_material_support"),
        (dict(radial_material_support="unknown"), "radial_material_support"),
        (dict(radial_boundary_condition="absorbing"), "radial_boundary_condition"),
        (dict(loss_integration="forward-euler"), "loss_integration"),
        (dict(radial_grid_policy="unchecked"), "radial_grid_policy"),
        (dict(geometry_mode="cylindrical"), "geometry_mode"),
        (dict(radial_cells=4, radial_altitudes_m=(-100_000.0, -5_000.0, -1_250.0, 0.0, 100_000.0)), "smoothly graded"),
    ],
)
def test_config_rejections_match_the_reference(changes, message):
    with pytest.raises(ValueError, match=message):
        config(**changes)


def test_source_waveform_rejections_match_the_reference():
    with pytest.raises(ValueError, match="finite"):
        GaussianCurrent(one_over_e_half_width_s=np.nan)
    with pytest.raises(ValueError, match="positive"):
        GaussianCurrent(one_over_e_half_width_s=0.0)
    with pytest.raises(ValueError, match="latitude"):
        TangentialGaussianCurrent(latitude_deg=91.0)
    with pytest.raises(ValueError, match="finite"):
        TangentialGaussianCurrent(line_lengths_m=(np.inf,))
    with pytest.raises(ValueError, match="finite"):
        GaussianCurrent(vertical_element_length_m=np.inf)
    with pytest.raises(ValueError, match="positive"):
        GaussianCurrent(vertical_element_length_m=0.0)


def test_default_source_and_modulated_envelope():
    source = GaussianCurrent()
    assert source.latitude_deg == pytest.approx(35.1595) and source.longitude_deg == pytest.approx(126.8526)
    assert GaussianCurrent(carrier_frequency_hz=20.0, peak_current_a=1.0).current_a(0.1, 1.0e-6) == pytest.approx(1.0)


@pytest.mark.parametrize("chunk_size", (0, True, 1.5))
def test_compile_chunk_size_must_be_a_positive_integer(chunk_size):
    from ionosphere_fdtd_b200 import GeodesicFDTD

    with pytest.raises(ValueError, match="compile_chunk_size"):
        GeodesicFDTD(config=config(), compile_chunk_size=chunk_size)


def test_gpu_alias_reports_a_missing_cuda_device():
    import torch

    from ionosphere_fdtd_b200 import BackendUnavailableError, GeodesicFDTD

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present; the GPU tests cover the alias")
    with pytest.raises(BackendUnavailableError, match="CUDA"):
        GeodesicFDTD(config=config(), backend="torch", device="gpu")


def _host(config):
    """Mesh and radial midpoints of a configuration: what the source supports read."""

    from types import SimpleNamespace

    from ionosphere_fdtd_b200 import build_geodesic_mesh

    alt = (np.asarray(config.radial_altitudes_m) if config.radial_altitudes_m is not None
           else np.linspace(config.minimum_altitude_m, config.maximum_altitude_m, config.radial_cells + 1))
    radii = config.earth_radius_m + alt
    mids = 0.5 * (radii[:-1] + radii[1:])
    return SimpleNamespace(mesh=build_geodesic_mesh(config.subdivision), config=config, altitudes_m=alt,
                           radial_midpoint_altitudes_m=mids - config.earth_radius_m)


def test_tangential_source_lines_and_edge_assignment():
    """tests/test_solver.py of the reference: ground lines must match the azimuths,
    nearest-edge assignment uses at most one edge per line."""

    with pytest.raises(ValueError, match="line_lengths_m must match"):
        TangentialGaussianCurrent(azimuths_deg=(0.0, 90.0), line_lengths_m=(22_500.0,))
    source = TangentialGaussianCurrent(azimuths_deg=(0.0, 90.0), line_lengths_m=(22_500.0, 22_500.0), edge_assignment="nearest")
    edges, _, weights = source.edge_distribution(_host(config()))
    assert len(np.unique(edges[weights != 0.0])) <= 2


def test_tangential_surface_source_keeps_its_staggered_altitude():
    source = TangentialGaussianCurrent(altitude_m=0.0, azimuths_deg=(0.0,), line_lengths_m=(22_500.0,))
    host = _host(config(radial_altitudes_m=(-5_000.0, -3_750.0, -2_500.0, -1_250.0, 0.0, 5_000.0, 10_000.0), radial_cells=6,
                        minimum_altitude_m=-5_000.0, maximum_altitude_m=10_000.0, radial_grid_policy="allow-abrupt"))
    edges, layers, weights = source.edge_distribution(host)
    assert set(host.radial_midpoint_altitudes_m[layers]) == {-625.0, 2_500.0}
    for edge in np.unique(edges):
        w = weights[edges == edge]
        if np.any(w):
            assert w.sum() != pytest.approx(0.0)
            assert w @ host.radial_midpoint_altitudes_m[layers[edges == edge]] / w.sum() == pytest.approx(source.altitude_m)


def test_provided_meshes_must_match_the_configuration():
    """tests/test_solver.py of the reference; the checks run before any device work."""

    from ionosphere_fdtd_b200 import GeodesicFDTD, build_geodesic_mesh

    with pytest.raises(ValueError, match="orientation"):
        GeodesicFDTD(config=config(), mesh=build_geodesic_mesh(1, orientation="native"))
    with pytest.raises(ValueError, match="cannot accompany"):
        GeodesicFDTD(config=config(mesh_optimization_steps=1), mesh=build_geodesic_mesh(1, orientation="polar"))
    with pytest.raises(ValueError, match="subdivision"):
        GeodesicFDTD(config=config(subdivision=2), mesh=build_geodesic_mesh(1))
