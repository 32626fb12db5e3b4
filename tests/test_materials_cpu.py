"""The reference's tests of the default Earth-ionosphere material
(tests/test_materials.py there) on the package's EarthIonosphereMaterial."""

import numpy as np
import pytest

from ionosphere_fdtd_b200 import EarthIonosphereMaterial, SphericalAnomaly


def test_profile_is_lithosphere_below_and_exponential_above():
    material = EarthIonosphereMaterial()
    sigma, eps = material.sample(np.asarray(((1.0, 0.0, 0.0),)), np.asarray((-1_000.0, 0.0, 80_000.0)), 6_371_000.0)
    assert sigma[0, 0] == material.lithosphere_conductivity_s_m
    assert sigma[0, 2] > sigma[0, 1]
    assert eps[0, 0] == material.lithosphere_relative_permittivity
    assert eps[0, 1] == material.atmosphere_relative_permittivity


def test_anomaly_changes_only_its_volume():
    material = EarthIonosphereMaterial(anomalies=(SphericalAnomaly(0.0, 0.0, 100_000.0, -2_000.0, -500.0, 0.1),))
    sigma, _ = material.sample(np.asarray(((1.0, 0.0, 0.0), (-1.0, 0.0, 0.0))), np.asarray((-1_000.0,)), 6_371_000.0)
    assert np.isclose(sigma[0, 0], 1.0e-4) and np.isclose(sigma[1, 0], 1.0e-3)


@pytest.mark.parametrize(
    "parameter, value",
    [("lithosphere_conductivity_s_m", np.inf), ("ionosphere_reference_height_m", -np.inf),
     ("ionosphere_scale_height_m", np.inf), ("ionosphere_prefactor_hz", np.nan)],
)
def test_default_material_rejects_nonfinite_parameters(parameter, value):
    with pytest.raises(ValueError, match="finite"):
        EarthIonosphereMaterial(**{parameter: value})
