"""Static dyadic radial refinement with 2:1 balance, and radial-grid validation
(the reference's radial_grid.py:13-165).

A refined grid starts from equal background cells and halves every cell that
meets a refinement region until the cell is no wider than the region's step
(the finest step wins where regions overlap).  Neighbouring cells are then kept
within one halving of each other: wherever two neighbours differ by more, the
coarser one must be halved in any balanced refinement, so halving every such
cell until none is left gives the unique coarsest balanced grid.  Midpoints are
always halves of their parent cell, so the nodes are the reference's bit for
bit.  The grid feeds ``SimulationConfig(radial_altitudes_m=...)`` with
``radial_grid_policy="balanced-2to1"``.
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np
from numpy.typing import NDArray


@dataclass(frozen=True, slots=True)
class RadialRefinementRegion:
    """Altitude interval with a requested maximum radial cell size (radial_grid.py:13-32)."""

    minimum_altitude_m: float
    maximum_altitude_m: float
    maximum_step_m: float

    def __post_init__(self) -> None:
        if not all(np.isfinite(v) for v in (self.minimum_altitude_m, self.maximum_altitude_m, self.maximum_step_m)):
            raise ValueError("radial refinement values must be finite")
        if self.minimum_altitude_m >= self.maximum_altitude_m:
            raise ValueError("radial refinement bounds are reversed")
        if self.maximum_step_m <= 0.0:
            raise ValueError("radial refinement step must be positive")


@dataclass(frozen=True, slots=True)
class RadialGridValidation:
    """Cell count, step extremes and the largest adjacent-step ratio (radial_grid.py:35-41)."""

    cells: int
    minimum_step_m: float
    maximum_step_m: float
    maximum_adjacent_step_ratio: float


def _target_step(lower: float, upper: float, regions) -> float:
    """The finest step requested by a region that the open cell (lower, upper) meets."""

    return min((r.maximum_step_m for r in regions if upper > r.minimum_altitude_m and lower < r.maximum_altitude_m),
               default=math.inf)


def _refine(lower: float, upper: float, level: int, regions, out: list) -> None:
    if upper - lower > _target_step(lower, upper, regions) * (1.0 + 1.0e-12):
        middle = 0.5 * (lower + upper)
        _refine(lower, middle, level + 1, regions, out)
        _refine(middle, upper, level + 1, regions, out)
    else:
        out.append((lower, upper, level))


def build_refined_radial_grid(minimum_altitude_m: float, maximum_altitude_m: float, background_step_m: float,
                              regions: tuple[RadialRefinementRegion, ...]) -> tuple[float, ...]:
    """Node altitudes of the refined, 2:1-balanced grid (radial_grid.py:44-132)."""

    if not all(np.isfinite(v) for v in (minimum_altitude_m, maximum_altitude_m, background_step_m)):
        raise ValueError("radial grid bounds and spacing must be finite")
    if minimum_altitude_m >= maximum_altitude_m:
        raise ValueError("radial grid bounds are reversed")
    if background_step_m <= 0.0:
        raise ValueError("background radial step must be positive")
    regions = tuple(regions)
    if not all(isinstance(r, RadialRefinementRegion) for r in regions):
        raise TypeError("regions must contain RadialRefinementRegion values")
    if any(r.minimum_altitude_m < minimum_altitude_m or r.maximum_altitude_m > maximum_altitude_m for r in regions):
        raise ValueError("radial refinement region lies outside the grid")

    count = int(math.ceil((maximum_altitude_m - minimum_altitude_m) / background_step_m))
    base = np.linspace(minimum_altitude_m, maximum_altitude_m, count + 1)
    cells: list[tuple[float, float, int]] = []
    for k in range(count):
        _refine(float(base[k]), float(base[k + 1]), 0, regions, cells)

    # 2:1 balance: halve every cell more than one level coarser than a neighbour
    while True:
        levels = [c[2] for c in cells]
        split = {i for i in range(len(cells) - 1) if levels[i + 1] - levels[i] > 1}
        split |= {i + 1 for i in range(len(cells) - 1) if levels[i] - levels[i + 1] > 1}
        if not split:
            break
        balanced = []
        for i, (lower, upper, level) in enumerate(cells):
            if i in split:
                middle = 0.5 * (lower + upper)
                balanced += [(lower, middle, level + 1), (middle, upper, level + 1)]
            else:
                balanced.append((lower, upper, level))
        cells = balanced

    nodes = (cells[0][0], *(c[1] for c in cells))
    validate_radial_grid(nodes, maximum_adjacent_step_ratio=2.0)
    return tuple(float(v) for v in nodes)


def validate_radial_grid(altitudes_m: tuple[float, ...] | NDArray[np.float64], *,
                         maximum_adjacent_step_ratio: float = 2.0) -> RadialGridValidation:
    """Finite increasing nodes whose adjacent steps differ by at most the given ratio
    (radial_grid.py:135-165)."""

    altitudes = np.asarray(altitudes_m, dtype=np.float64)
    if altitudes.ndim != 1 or len(altitudes) < 3 or not np.all(np.isfinite(altitudes)) or not np.all(np.diff(altitudes) > 0.0):
        raise ValueError("radial grid must contain finite increasing nodes")
    if not np.isfinite(maximum_adjacent_step_ratio) or maximum_adjacent_step_ratio < 1.0:
        raise ValueError("maximum adjacent step ratio must be at least one")
    steps = np.diff(altitudes)
    ratio = float(np.max(np.maximum(steps[:-1] / steps[1:], steps[1:] / steps[:-1])))
    if ratio > maximum_adjacent_step_ratio * (1.0 + 1.0e-12):
        raise ValueError("radial grid violates the adjacent-step ratio")
    return RadialGridValidation(cells=len(steps), minimum_step_m=float(np.min(steps)), maximum_step_m=float(np.max(steps)),
                                maximum_adjacent_step_ratio=ratio)
