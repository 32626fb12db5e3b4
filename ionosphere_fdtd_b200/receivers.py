"""Receivers at geographic locations and their recorded Er traces.

The reference's ``Receiver``, ``ReceiverTraces`` and ``record_receiver_traces``
(visualization.py:38-54, 212-252; receiver placement ``_receiver_location``
751-757) advance the simulation ``sample_every`` steps at a time and read each
receiver's value with one scalar device read per receiver and sample.  Here the
receivers become one weight-1 probe on the engine: the step kernels' sampling
launch records every receiver at every step on the device (inside the captured
step graphs), in blocks of at most a few thousand steps, and the host keeps the
rows of the sample times.  A weight of exactly 1 makes each recorded value the
field value itself, so the traces, times and labels are those of the reference.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import TYPE_CHECKING, Sequence

import numpy as np
from numpy.typing import NDArray

from .sources import geographic_direction

if TYPE_CHECKING:
    from .solver import GeodesicFDTD

FloatArray = NDArray[np.float64]

# Steps recorded per device trace buffer (rounded down to a multiple of
# sample_every): bounds the device memory to about 4096 x receivers x 8 bytes.
_BLOCK_STEPS = 4096


@dataclass(frozen=True, slots=True)
class Receiver:
    """A radial electric-field observation location (visualization.py:38-45)."""

    latitude_deg: float
    longitude_deg: float
    altitude_m: float = 0.0
    label: str | None = None


@dataclass(frozen=True, slots=True)
class ReceiverTraces:
    """Time samples recorded at one or more receivers (visualization.py:48-54)."""

    time_s: FloatArray
    er_v_m: FloatArray
    labels: tuple[str, ...]


def receiver_location(simulation: GeodesicFDTD, receiver: Receiver) -> tuple[int, int]:
    """The nearest mesh vertex and radial node of a receiver (visualization.py:751-757)."""

    direction = geographic_direction(receiver.latitude_deg, receiver.longitude_deg)
    vertex = int(np.argmax(simulation.mesh.vertices @ direction))
    layer = int(np.argmin(np.abs(simulation.altitudes_m - receiver.altitude_m)))
    return vertex, layer


def record_receiver_traces(
    simulation: GeodesicFDTD,
    receivers: Sequence[Receiver],
    steps: int,
    *,
    sample_every: int = 1,
) -> ReceiverTraces:
    """Advance a simulation while recording ``Er`` at fixed receivers
    (visualization.py:212-252).

    Row 0 is the current state; then one row after every ``sample_every``
    steps, and one after the last step when ``steps`` is not a multiple of it."""

    if not receivers:
        raise ValueError("at least one receiver is required")
    if steps < 0:
        raise ValueError("steps must be non-negative")
    if sample_every <= 0:
        raise ValueError("sample_every must be positive")
    steps = simulation._validated_count(steps, "step count", minimum=0)
    sample_every = simulation._validated_count(sample_every, "sample_every", minimum=1)

    locations = [receiver_location(simulation, r) for r in receivers]
    labels = tuple(r.label or f"{r.latitude_deg:g}°, {r.longitude_deg:g}°" for r in receivers)
    vertices = np.asarray([[v] for v, _ in locations], dtype=np.int64)
    layers = np.asarray([k for _, k in locations], dtype=np.int64)
    weights = np.ones((len(locations), 1), dtype=np.float64)

    # completed steps at each sample, counted from the current state
    rows = np.unique(np.concatenate((np.arange(0, steps + 1, sample_every, dtype=np.int64),
                                     np.asarray((steps,), dtype=np.int64))))
    start_step, start_time = simulation.steps, simulation.time_s
    er = np.empty((len(rows), len(locations)), dtype=np.float64)
    block = sample_every * max(1, _BLOCK_STEPS // sample_every)
    done = filled = 0
    while True:
        n = min(block, steps - done)
        traces = simulation.record_er_observations(vertices, layers, weights, n)  # rows done .. done + n
        lo = done + 1 if filled else done
        picked = rows[(rows >= lo) & (rows <= done + n)]
        er[filled : filled + len(picked)] = traces[picked - done]
        filled += len(picked)
        done += n
        if done >= steps:
            break
    # the reference reads the clock after every advance: steps x time step
    time_s = (start_step + rows) * simulation.time_step_s
    time_s[0] = start_time
    return ReceiverTraces(time_s=time_s, er_v_m=er, labels=labels)
