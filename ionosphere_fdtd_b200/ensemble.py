"""Ensembles of independent simulations advanced together on one GPU.

The reference runs an ensemble as a Python loop over ``GeodesicFDTD``
objects, each calling ``step`` or ``record_er_observations``
(solver.py:789-816, 1080-1136).  ``Ensemble`` keeps those per-member calls
and their results, but advances every member through the C ABI's batched step
(``ifdtd_batch_step``): one launch per phase covers all members whose plans
run on the pipelined kernels (members of any mesh level, radial grid,
material, source and physics), and one launch per step samples every
member's receivers.  A member's fields, step counter and time come out as
from the same calls on the member alone.
"""

from __future__ import annotations

import ctypes as C
from typing import Any, Sequence

import numpy as np

from . import _native as N
from .solver import GeodesicFDTD


class Ensemble:
    """Advance several ``GeodesicFDTD`` members together.

    All members must live on one CUDA device with one field precision.  The
    members stay usable on their own (``member.step``, ``diagnostics``,
    checkpoints); the ensemble only adds the batched step.  ``graph_chunk``
    is the number of steps per captured CUDA graph."""

    def __init__(self, members: Sequence[GeodesicFDTD], *, graph_chunk: int = 32):
        members = list(members)
        if not members:
            raise ValueError("an ensemble needs at least one member")
        if len({id(m) for m in members}) != len(members):
            raise ValueError("a simulation appears twice in the ensemble")
        if isinstance(graph_chunk, bool) or not isinstance(graph_chunk, (int, np.integer)) or graph_chunk < 1:
            raise ValueError("graph_chunk must be a positive integer")
        for m in members:
            if not isinstance(m, GeodesicFDTD):
                raise TypeError("ensemble members must be GeodesicFDTD simulations")
        first = members[0].backend
        for m in members:
            if m.backend.torch_device != first.torch_device or m.backend.dtype != first.dtype:
                raise ValueError("ensemble members must share one CUDA device and one dtype")
        self._members = members
        self._backend = first
        # the engines themselves, not their plan addresses: a replaced engine's plan is freed,
        # and a new plan may be allocated at the same address
        self._engines = [m._engine for m in members]
        plans = (C.c_void_p * len(members))(*[e.plan.value for e in self._engines])
        handle = C.c_void_p()
        N.check(N.load().ifdtd_batch_create(plans, len(members), int(graph_chunk), C.byref(handle)), "ifdtd_batch_create")
        self._handle = handle
        self._currents_dev = None  # kept alive until the next call (the step is asynchronous)

    # -- properties ------------------------------------------------------------------

    @property
    def members(self) -> list[GeodesicFDTD]:
        return list(self._members)

    def __len__(self) -> int:
        return len(self._members)

    def launch_layout(self) -> dict[str, int]:
        """Batched launch groups, members launched on their own, and the CTAs of
        the first group's H and E launches."""

        vals = [C.c_int32() for _ in range(4)]
        N.check(N.load().ifdtd_batch_info(self._live(), *[C.byref(v) for v in vals]), "ifdtd_batch_info")
        return dict(zip(("groups", "solo", "kh_grid", "ke_grid"), (int(v.value) for v in vals)))

    # -- stepping --------------------------------------------------------------------

    def step(self, count: int = 1) -> None:
        """Advance every member by ``count`` leapfrog steps."""

        count = self._members[0]._validated_count(count, "step count", minimum=0)
        if not count:
            return
        self._run(count, None, None)
        self._advance_clocks(count)

    def record_er_observations(self, observations: Sequence[Any], steps: int) -> list[np.ndarray | None]:
        """Advance every member by ``steps`` steps while recording weighted Er
        samples.  ``observations[i]`` is member i's ``(vertex_indices,
        radial_layers, weights)`` as for ``GeodesicFDTD.record_er_observations``,
        or None for a member without receivers; the result holds member i's
        float64 (steps + 1, rows) traces with the initial state in row 0."""

        if len(observations) != len(self._members):
            raise ValueError("one observation set (or None) per member is required")
        steps = self._members[0]._validated_count(steps, "step count", minimum=0)
        torch = self._backend.torch
        probes, traces = [], []
        try:
            for m, obs in zip(self._members, observations):
                if obs is None:
                    probes.append(None)
                    traces.append(None)
                    continue
                vertex_indices, radial_layers, weights = obs
                vertices = m._validated_index_array(vertex_indices, "vertex_indices")
                layers = m._validated_index_array(radial_layers, "radial_layers")
                w = np.asarray(weights, dtype=np.float64)
                m._check_er_observation(vertices, layers, w)
                probe = m._engine.probe("er", vertices, np.broadcast_to(layers[:, None], vertices.shape), w)
                probes.append(probe)
                t = torch.zeros((steps + 1, vertices.shape[0]), dtype=torch.float64, device=m.backend.torch_device)
                m._engine.sample(m._state(), probe, t[0])
                traces.append(t)
            if steps:
                self._run(steps, probes, [None if t is None else t[1:] for t in traces])
            self._advance_clocks(steps)
            self._backend.synchronize()
        finally:
            for p in probes:
                if p is not None:
                    p.close()
        return [None if t is None else t.cpu().numpy() for t in traces]

    def close(self) -> None:
        if self._handle:
            N.load().ifdtd_batch_destroy(self._handle)
            self._handle = C.c_void_p()

    def __enter__(self) -> "Ensemble":
        return self

    def __exit__(self, *exc) -> None:
        self.close()

    def __del__(self) -> None:
        try:
            self.close()
        except Exception:
            pass

    # -- internals -------------------------------------------------------------------

    def _live(self) -> C.c_void_p:
        if not self._handle:
            raise ValueError("the ensemble is closed")
        # the batch holds the members' plans: a member whose engine was replaced
        # (autotuning, for instance) must not be stepped through a stale plan
        if any(m._engine is not e or not e.plan for m, e in zip(self._members, self._engines)):
            raise ValueError("a member's plan changed after the ensemble was built; build a new Ensemble")
        return self._handle

    def _advance_clocks(self, count: int) -> None:
        for m in self._members:
            m.steps += count
            m.time_s = m.steps * m.time_step_s

    def _run(self, count: int, probes, out_rows) -> None:
        handle = self._live()
        n = len(self._members)
        states = (N.State * n)(*[m._state() for m in self._members])
        series = [m._source_currents(count) for m in self._members]
        cur_ptr = None
        if any(s is not None for s in series):
            host = np.zeros((n, count), dtype=np.float64)
            for i, s in enumerate(series):
                if s is not None:
                    host[i] = s
            torch = self._backend.torch
            self._currents_dev = torch.from_numpy(host).to(self._backend.torch_device)
            cur_ptr = self._currents_dev.data_ptr()
        probe_arr = out_arr = None
        if probes is not None:
            probe_arr = (C.c_void_p * n)(*[None if p is None else p.handle.value for p in probes])
            out_arr = (C.c_void_p * n)(*[None if t is None else t.data_ptr() for t in out_rows])
        N.check(
            N.load().ifdtd_batch_step(handle, states, cur_ptr, count, probe_arr, out_arr, self._backend.stream_handle()),
            "ifdtd_batch_step",
        )
