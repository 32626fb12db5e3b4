"""Refined radial grids: bit-exact with grids the reference built
(tests/golden/radial_grids.npz), and the reference's own radial-grid tests
(tests/test_radial_grid.py there) on the package."""

import numpy as np
import pytest

import cases as C
from casebuild import golden

import ionosphere_fdtd_b200 as P


@pytest.mark.parametrize("index", range(len(C.RADIAL_GRIDS)))
def test_refined_grids_are_the_reference_grids(index):
    lo, hi, step, regions = C.RADIAL_GRIDS[index]
    ref = golden("radial_grids")
    nodes = P.build_refined_radial_grid(lo, hi, step, tuple(P.RadialRefinementRegion(*r) for r in regions))
    np.testing.assert_array_equal(np.asarray(nodes), ref[f"nodes_{index}"])
    v = P.validate_radial_grid(nodes)
    np.testing.assert_array_equal((v.cells, v.minimum_step_m, v.maximum_step_m, v.maximum_adjacent_step_ratio),
                                  ref[f"validation_{index}"])


def test_refinement_resolves_each_region_with_2to1_balance():
    single = P.RadialRefinementRegion(60_000.0, 90_000.0, 1_000.0)
    overlapping = (P.RadialRefinementRegion(40_000.0, 80_000.0, 2_000.0), P.RadialRefinementRegion(60_000.0, 70_000.0, 500.0))
    for regions in ((single,), overlapping):
        nodes = np.asarray(P.build_refined_radial_grid(0.0, 100_000.0, 10_000.0, regions))
        steps, lower, upper = np.diff(nodes), nodes[:-1], nodes[1:]
        assert nodes[0] == 0.0 and nodes[-1] == 100_000.0
        assert P.validate_radial_grid(nodes).maximum_adjacent_step_ratio <= 2.0
        for r in regions:
            meets = (upper > r.minimum_altitude_m) & (lower < r.maximum_altitude_m)
            assert np.max(steps[meets]) <= r.maximum_step_m
    assert P.validate_radial_grid(P.build_refined_radial_grid(0.0, 100_000.0, 10_000.0, (single,))).cells == 61


def test_radial_grid_errors_match_the_reference():
    with pytest.raises(ValueError, match="adjacent-step ratio"):
        P.SimulationConfig(subdivision=0, radial_cells=3, minimum_altitude_m=0.0, maximum_altitude_m=7_000.0,
                           radial_altitudes_m=(0.0, 1_000.0, 2_000.0, 7_000.0), radial_grid_policy="balanced-2to1")
    with pytest.raises(ValueError, match="outside"):
        P.build_refined_radial_grid(0.0, 100_000.0, 10_000.0, (P.RadialRefinementRegion(-1.0, 1_000.0, 100.0),))
    with pytest.raises(ValueError, match="finite increasing nodes"):
        P.build_refined_radial_grid(-5_000.0, 5_000.0, 10_000.0, ())  # a single cell
    with pytest.raises(ValueError, match="reversed"):
        P.RadialRefinementRegion(2.0, 1.0, 0.5)
    with pytest.raises(TypeError, match="RadialRefinementRegion"):
        P.build_refined_radial_grid(0.0, 1.0, 0.1, ((0.0, 1.0, 0.1),))
    with pytest.raises(ValueError, match="at least one"):
        P.validate_radial_grid((0.0, 1.0, 2.0), maximum_adjacent_step_ratio=0.5)
