"""CPU oracle for the geodesic FDTD time step.

TEST INFRASTRUCTURE ONLY. This package restates, in NumPy, the algorithm of
the reference solver (ruddyscent/ionosphere-fdtd v0.2.0, ``src/ionosphere_fdtd``)
for the time-step loop behind ``GeodesicFDTD.step``.  It is the checker for
the CUDA path, never the thing measured or shipped: only ``tests/``,
``__graft_entry__.smoke()`` and the ``cpu_baseline`` / ``--impl reference``
legs of ``bench.py`` may import it.  The product package
(``ionosphere_fdtd_b200``) never imports it and has no CPU fallback.

Parity is pinned: ``tests/golden/make_golden.py`` runs the reference itself
(imported from its source tree in the build container) and commits its mesh
tables, fields, ADE states and receiver traces as fixtures;
``tests/test_oracle_golden.py`` checks this oracle against them.

``oracle.threaded`` runs the same step on PyTorch CPU tensors over every host
thread (the reference's Torch-on-CPU path); it is the timed CPU baseline and is
checked against the same fixtures.
"""

from .fdtd import (  # noqa: F401
    OracleFDTD,
    OracleMesh,
    build_mesh,
    earth_ionosphere_sample,
    vertex_incidence,
)
