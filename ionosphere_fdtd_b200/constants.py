"""SI constants of the reference solver (constants.py:3-6)."""

EPSILON_0 = 8.854_187_812_8e-12
MU_0 = 1.256_637_062_12e-6
C_0 = 1.0 / (EPSILON_0 * MU_0) ** 0.5
EARTH_RADIUS_M = 6_371_000.0
