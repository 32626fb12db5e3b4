"""Owner of one native plan: descriptors in, CUDA launches out.

``Engine`` turns a solver's host setup (mesh tables, radial grid, loss
coefficients, source supports, surface-impedance and plasma coefficients)
into the plain-pointer descriptors of ``include/ifdtd.h``, creates the plan
and drives it on torch's current CUDA stream.  It keeps every host array
referenced by a descriptor alive for the plan's lifetime.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Any

import numpy as np

from . import _native as N
from .constants import MU_0


@dataclass
class Physics:
    """Host-side physics inputs of one plan (float64)."""

    ca_er: np.ndarray
    cb_er: np.ndarray
    ca_et: np.ndarray
    cb_et: np.ndarray
    src_er: tuple[np.ndarray, np.ndarray, np.ndarray] | None = None  # vertex, layer, coef
    src_et: tuple[np.ndarray, np.ndarray, np.ndarray] | None = None  # edge, layer, coef
    si: dict[str, Any] | None = None
    plasma: dict[str, Any] | None = None


@dataclass
class Tuning:
    """Launch geometry of a plan: faces per H-phase and E-phase patch (0: the
    largest patch whose pipeline stage fits twice in shared memory), threads
    per CTA (direct kernels, at most 256) or compute threads per CTA besides
    the producer warps (pipelined kernels; 0: 256 direct, 384 - 32 x producer
    warps pipelined), steps per captured
    CUDA graph, and the kernel family (0 auto: the pipeline wherever two patch
    stages fit in shared memory, 1 direct global gathers, 2 the warp-specialised
    pipeline fed by TMA bulk copies, 3 the same pipeline fed by 16-byte cp.async
    copies), the copy-issuing warps per pipelined CTA (1 to 4), and the lane
    layout of the pipelined consumers (0 auto = 1, rows packed back to back
    across lanes; 2, every row starting on an 8-lane boundary), the compute
    threads of an E-phase CTA (0: as ``threads``; above 384 minus the producer
    warps the E phase runs wide CTAs of at most 640 threads at 96 registers)
    the ring stages the balanced E patches are sized for (0: 2), the
    copy-issuing warps of an E-phase CTA (0: 4 when both thread counts are
    automatic, else as ``producer_warps``), the
    row gaps every E-phase copy bridges (0-8: fewer, longer bulk copies), and
    ``fused_step`` (1: one launch per leapfrog step in which every E patch
    recomputes the new H on its halo, for plans without plasma or surface
    impedance; the plan then holds a second copy of the field arrays, and in
    an ``Ensemble`` it runs the batched fused kernel).
    Every choice above computes the same bits.  ``plasma_frame`` (0 auto:
    face frames for an unmagnetised plasma, 1 Cartesian, 2 face frames) picks
    the frame the plasma current is held in while the kernels run; the state
    is Cartesian between calls, and the two frames round differently."""

    faces_per_patch: int = 0
    threads: int = 0
    graph_chunk: int = 32
    e_faces_per_patch: int = 0
    staging: int = 0
    producer_warps: int = 2
    lane_layout: int = 0
    e_threads: int = 0
    e_stages: int = 0
    e_producer_warps: int = 0
    e_copy_gap: int = 0
    fused_step: int = 0
    plasma_frame: int = 0


def _dedupe_last(index_a, index_b, coef):
    """Keep the last of repeated (a, b) supports, as NumPy fancy assignment does."""

    keys = list(zip(index_a.tolist(), index_b.tolist()))
    last = {k: i for i, k in enumerate(keys)}
    keep = np.asarray(sorted(last.values()), dtype=np.int64)
    return index_a[keep], index_b[keep], coef[keep]


class Probe:
    def __init__(self, engine: "Engine", kind: int, index, layer, weight):
        self.engine = engine
        self.rows, self.width = index.shape
        self._index = N.i64(index)
        self._layer = N.i64(layer)
        self._weight = N.f64(weight)
        handle = C.c_void_p()
        N.check(
            N.load().ifdtd_probe_create(
                engine.plan, kind, self.rows, self.width, N.ptr_i64(self._index), N.ptr_i64(self._layer), N.ptr_f64(self._weight), C.byref(handle)
            ),
            "ifdtd_probe_create",
        )
        self.handle = handle

    def close(self) -> None:
        if self.handle:
            N.load().ifdtd_probe_destroy(self.handle)
            self.handle = C.c_void_p()


class Engine:
    def __init__(self, mesh, radii_m: np.ndarray, full_spherical: bool, time_step_s: float, physics: Physics, backend, tuning: Tuning | None = None):
        lib = N.load()
        self.backend = backend
        self.mesh = mesh
        self.L = len(radii_m) - 1
        self.tuning = tuning or Tuning()
        keep: list[Any] = []

        def i64(a):
            arr = N.i64(a)
            keep.append(arr)
            return N.ptr_i64(arr)

        def f64(a):
            arr = N.f64(a)
            keep.append(arr)
            return N.ptr_f64(arr)

        md = N.MeshDesc(
            mesh.n_vertices,
            mesh.n_edges,
            mesh.n_faces,
            i64(mesh.edges),
            i64(mesh.faces),
            i64(mesh.face_edges),
            i64(mesh.face_edge_signs),
            i64(mesh.edge_left_faces),
            i64(mesh.edge_right_faces),
            f64(mesh.primal_edge_angles),
            f64(mesh.dual_edge_angles),
            f64(mesh.face_solid_angles),
            f64(mesh.dual_cell_solid_angles),
        )
        gd = N.GridDesc(self.L, 1 if full_spherical else 0, f64(radii_m), float(time_step_s))
        pd = N.PhysicsDesc()
        pd.coef_rows_er = int(physics.ca_er.shape[0])
        pd.coef_rows_et = int(physics.ca_et.shape[0])
        pd.ca_er, pd.cb_er = f64(physics.ca_er), f64(physics.cb_er)
        pd.ca_et, pd.cb_et = f64(physics.ca_et), f64(physics.cb_et)
        if physics.src_er is not None and len(physics.src_er[0]):
            v, k, c = _dedupe_last(*physics.src_er)
            if len(v) > N.MAX_SOURCES:
                raise ValueError("too many vertical source supports")
            pd.n_src_er, pd.src_er_vertex, pd.src_er_layer, pd.src_er_coef = len(v), i64(v), i64(k), f64(c)
        if physics.src_et is not None and len(physics.src_et[0]):
            e, j, c = _dedupe_last(*physics.src_et)
            if len(e) > N.MAX_SOURCES:
                raise ValueError("too many tangential source supports")
            pd.n_src_et, pd.src_et_edge, pd.src_et_layer, pd.src_et_coef = len(e), i64(e), i64(j), f64(c)
        self.si_terms = 0
        if physics.si is not None:
            si = physics.si
            self.si_terms = int(len(si["decay"]))
            pd.si_terms = self.si_terms
            pd.si_scale, pd.si_decay, pd.si_drive, pd.si_history = f64(si["scale"]), f64(si["decay"]), f64(si["drive"]), f64(si["history"])
            pd.si_metric = float(si["metric"])
        self.species = 0
        # the plan holds the plasma current in face frames while its kernels run
        # (automatic for an unmagnetised plasma unless the Cartesian frame is asked for)
        self.face_frames = False
        if physics.plasma is not None:
            p = physics.plasma
            self.species = int(p["coef"].shape[0])
            self.face_frames = not p["magnetized"] and self.tuning.plasma_frame != 1
            if self.species > N.MAX_SPECIES:
                raise ValueError(f"at most {N.MAX_SPECIES} plasma species are supported")
            pd.plasma_species = self.species
            pd.plasma_rows = int(p["rows"])
            pd.plasma_magnetized = 1 if p["magnetized"] else 0
            pd.plasma_coef = f64(p["coef"])
            pd.plasma_bdir = f64(p["bdir"])
            pd.plasma_reconstruction = f64(p["reconstruction"])
            pd.face_centers = f64(mesh.face_centers)
            pd.plasma_tangent_left = f64(p["left_tangents"])
            pd.plasma_tangent_right = f64(p["right_tangents"])
            pd.vertex_face_width = int(p["vertex_faces"].shape[1])
            pd.vertex_faces = i64(p["vertex_faces"])
            pd.vertex_face_weights = f64(p["vertex_face_weights"])
        t = self.tuning
        td = N.Tuning(t.faces_per_patch, t.threads, t.graph_chunk, t.e_faces_per_patch, t.staging, t.producer_warps, t.lane_layout,
                      t.e_threads, t.e_stages, t.e_producer_warps, t.e_copy_gap,
                      t.fused_step, t.plasma_frame)
        handle = C.c_void_p()
        with backend.torch.cuda.device(backend.torch_device):
            N.check(
                lib.ifdtd_plan_create(C.byref(md), C.byref(gd), C.byref(pd), C.byref(td), backend.itemsize, backend.torch_device.index, C.byref(handle)),
                "ifdtd_plan_create",
            )
        self.plan = handle
        node_pitch, mid_pitch = C.c_int32(), C.c_int32()
        N.check(lib.ifdtd_plan_layout(handle, C.byref(node_pitch), C.byref(mid_pitch)), "ifdtd_plan_layout")
        self.node_pitch, self.mid_pitch = int(node_pitch.value), int(mid_pitch.value)
        self._keep = keep  # descriptors are copied by the plan; arrays kept for clarity of ownership
        self._state_key = None
        self._state = N.State()
        self._cur = None
        self._cur_host = None
        self._cur_event = None
        self._max_out = None

    def close(self) -> None:
        if getattr(self, "plan", None):
            N.load().ifdtd_plan_destroy(self.plan)
            self.plan = C.c_void_p()

    def __del__(self):  # pragma: no cover - interpreter shutdown ordering
        try:
            self.close()
        except Exception:
            pass

    @property
    def kernel_modes(self) -> tuple[str, str]:
        """Kernel family of the H and E phases: "direct" (global gathers) or
        "pipeline" (warp-specialised shared-memory pipeline); a fused plan
        reports ("fused", family of its one-launch kernel)."""

        h, e = C.c_int32(), C.c_int32()
        N.check(N.load().ifdtd_plan_kernels(self.plan, C.byref(h), C.byref(e)), "ifdtd_plan_kernels")
        name = {1: "direct", 2: "pipeline", 3: "fused"}
        return name[h.value], name[e.value]

    def status_word(self, reset: bool = False) -> int:
        out = C.c_int32()
        N.check(N.load().ifdtd_status_word(self.plan, 1 if reset else 0, C.byref(out)), "ifdtd_status_word")
        return int(out.value)

    @property
    def plan_bytes(self) -> int:
        out = C.c_int64()
        N.check(N.load().ifdtd_plan_bytes(self.plan, C.byref(out)), "ifdtd_plan_bytes")
        return int(out.value)

    # -- state ------------------------------------------------------------------

    def state(self, er, et, hr, ht, si_memory=None, plasma_currents=()) -> N.State:
        """Bind the padded state buffers: er/ht (V|E, node_pitch), et/hr
        (E|F, mid_pitch), plasma currents (F, 3, mid_pitch), SI memory (E, T)."""

        tensors = (er, et, hr, ht, si_memory, *plasma_currents)
        key = tuple(0 if t is None else t.data_ptr() for t in tensors)
        if key == self._state_key:
            return self._state
        b = self.backend
        mesh = self.mesh
        pn, pm = self.node_pitch, self.mid_pitch
        expect = {
            "er": (er, (mesh.n_vertices, pn)),
            "et": (et, (mesh.n_edges, pm)),
            "hr": (hr, (mesh.n_faces, pm)),
            "ht": (ht, (mesh.n_edges, pn)),
        }
        if self.si_terms:
            expect["surface_impedance_memory"] = (si_memory, (mesh.n_edges, self.si_terms))
        for i in range(self.species):
            expect[f"plasma_current_{i}"] = (plasma_currents[i], (mesh.n_faces, 3, pm))
        for name, (t, shape) in expect.items():
            if t is None or not b.torch.is_tensor(t):
                raise ValueError(f"{name} must be a device tensor")
            if tuple(t.shape) != shape:
                raise ValueError(f"{name} buffer has shape {tuple(t.shape)}, expected {shape}")
            if t.dtype != b.dtype or t.device != b.torch_device:
                raise ValueError(f"{name} must be a {b.dtype_name} tensor on {b.device}")
            if not t.is_contiguous() or t.data_ptr() % 16:
                raise ValueError(f"{name} must be contiguous and 16-byte aligned")
        st = N.State()
        st.er, st.et, st.hr, st.ht = er.data_ptr(), et.data_ptr(), hr.data_ptr(), ht.data_ptr()
        st.si_memory = si_memory.data_ptr() if self.si_terms else None
        for i in range(self.species):
            st.plasma_current[i] = plasma_currents[i].data_ptr()
        self._state, self._state_key = st, key
        return st

    # -- launches -----------------------------------------------------------------

    def _currents(self, values: np.ndarray | None, count: int):
        """Upload the step currents through a pinned buffer without blocking the host.

        The pinned buffer is rewritten only after the previous upload from it
        has completed (an event recorded after the copy guards it)."""

        if values is None:
            return None
        torch = self.backend.torch
        if self._cur is None or self._cur.numel() < count:
            size = max(count, 64)
            if self._cur_event is not None:
                self._cur_event.synchronize()
            self._cur = torch.empty(size, dtype=torch.float64, device=self.backend.torch_device)
            self._cur_host = torch.empty(size, dtype=torch.float64, pin_memory=True)
        if self._cur_event is not None:
            self._cur_event.synchronize()
        self._cur_host.numpy()[:count] = values
        self._cur[:count].copy_(self._cur_host[:count], non_blocking=True)
        if self._cur_event is None:
            self._cur_event = torch.cuda.Event()
        self._cur_event.record(torch.cuda.current_stream(self.backend.torch_device))
        return self._cur

    def step(self, state: N.State, currents: np.ndarray | None, count: int) -> None:
        if count <= 0:
            return
        cur = self._currents(currents, count)
        N.check(
            N.load().ifdtd_step(self.plan, C.byref(state), None if cur is None else cur.data_ptr(), count, self.backend.stream_handle()),
            "ifdtd_step",
        )

    def step_sampled(self, state: N.State, currents: np.ndarray | None, count: int, probe: Probe, out_rows) -> None:
        if count <= 0:
            return
        cur = self._currents(currents, count)
        N.check(
            N.load().ifdtd_step_sampled(
                self.plan, C.byref(state), None if cur is None else cur.data_ptr(), count, probe.handle, out_rows.data_ptr(), self.backend.stream_handle()
            ),
            "ifdtd_step_sampled",
        )

    def update_magnetic(self, state: N.State) -> None:
        N.check(N.load().ifdtd_update_magnetic(self.plan, C.byref(state), self.backend.stream_handle()), "ifdtd_update_magnetic")

    def update_electric(self, state: N.State, current: float) -> None:
        N.check(
            N.load().ifdtd_update_electric(self.plan, C.byref(state), float(current), self.backend.stream_handle()),
            "ifdtd_update_electric",
        )

    def phase_times_ms(self, state: N.State, reps: int) -> tuple[float, float]:
        """Median device time (ms) of the H and E phase kernels over ``reps`` launches
        each (``ifdtd_time_phases``; advances the state by 3 + reps steps)."""

        h, e = C.c_float(), C.c_float()
        N.check(N.load().ifdtd_time_phases(self.plan, C.byref(state), int(reps), C.byref(h), C.byref(e),
                                           self.backend.stream_handle()), "ifdtd_time_phases")
        return float(h.value), float(e.value)

    def probe(self, kind: str, index, layer, weight) -> Probe:
        return Probe(self, {"er": 0, "et": 1, "hr": 2, "ht": 3}[kind], index, layer, weight)

    def sample(self, state: N.State, probe: Probe, out_row) -> None:
        N.check(N.load().ifdtd_sample(self.plan, C.byref(state), probe.handle, out_row.data_ptr(), self.backend.stream_handle()), "ifdtd_sample")

    def max_abs(self, state: N.State) -> np.ndarray:
        torch = self.backend.torch
        if self._max_out is None:
            self._max_out = torch.empty(4, dtype=torch.float64, device=self.backend.torch_device)
        N.check(N.load().ifdtd_max_abs(self.plan, C.byref(state), self._max_out.data_ptr(), self.backend.stream_handle()), "ifdtd_max_abs")
        return self._max_out.cpu().numpy()


def topology_engine(mesh, backend) -> Engine:
    """A plan carrying only the mesh tables (for the backend primitives)."""

    radii = np.asarray((1.0, 2.0, 3.0))
    ones = np.ones((1, 3))
    physics = Physics(ca_er=ones, cb_er=ones, ca_et=ones[:, :2], cb_et=ones[:, :2])
    return Engine(mesh, radii, True, 1.0, physics, backend, Tuning(graph_chunk=0))


def surface_inputs(ade, radii_m, midpoints_m, full_spherical: bool) -> dict[str, Any]:
    """Surface-impedance descriptor inputs (surface_impedance.py:194-203, solver.py:900-912)."""

    return {
        "scale": ade.scale_host,
        "decay": ade.decay_host,
        "drive": ade.drive_host,
        "history": ade.history_host,
        "metric": (midpoints_m[0] / radii_m[0]) if full_spherical else 1.0,
    }


def plasma_inputs(coupler) -> dict[str, Any]:
    ade = coupler.ade
    return {
        "coef": ade.coef,
        "bdir": ade.bdir,
        "rows": ade.rows,
        "magnetized": ade.magnetized,
        "reconstruction": coupler.reconstruction,
        "left_tangents": coupler.left_tangents,
        "right_tangents": coupler.right_tangents,
        "vertex_faces": coupler.vertex_faces,
        "vertex_face_weights": coupler.vertex_face_weights,
    }


__all__ = ["Engine", "Physics", "Tuning", "Probe", "topology_engine", "surface_inputs", "plasma_inputs", "MU_0"]
