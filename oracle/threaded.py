"""The oracle's leapfrog step on PyTorch CPU tensors, using every host thread
(test and CPU-baseline infrastructure only).

This restates the reference's own multi-threaded CPU path:
``GeodesicFDTD(..., backend="torch", device="cpu", torch_threads=n)``
(``backends/torch_backend.py:18-60``). The solver code is the one
``oracle/fdtd.py`` restates (``solver.py:877-989``), and the array primitives are
those of the Torch backend (``backends/torch_backend.py:160-198``). Every array
of an ``OracleFDTD`` is wrapped zero-copy (``torch.from_numpy``) and updated in
place, so the NumPy object sees each step: its receivers, ``max_abs`` and
parity checks keep working unchanged.

Imported only by ``tests/`` and ``bench.py``'s CPU legs.
"""

from __future__ import annotations

import os

import numpy as np
import torch

from .fdtd import MU_0, OracleFDTD


def _t(values) -> torch.Tensor:
    """Zero-copy tensor view of a NumPy array (indices stay int64)."""

    a = np.asarray(values)
    if not a.flags.writeable or not a.flags.c_contiguous:
        a = np.ascontiguousarray(a).copy()
    return torch.from_numpy(a)


class ThreadedOracleStep:
    """Advance an ``OracleFDTD`` with PyTorch CPU kernels on ``threads`` threads."""

    def __init__(self, sim: OracleFDTD, threads: int | None = None) -> None:
        self.sim = sim
        self.threads = int(threads or os.cpu_count() or 1)
        if self.threads < 1:
            raise ValueError("threads must be a positive integer")
        torch.set_num_threads(self.threads)
        m = sim.mesh
        # fields and ADE state: views of the oracle's own arrays
        self.er, self.et, self.hr, self.ht = (_t(getattr(sim, f)) for f in ("er", "et", "hr", "ht"))
        for name in ("er", "et", "hr", "ht"):
            if not np.shares_memory(getattr(sim, name), getattr(self, name).numpy()):
                raise RuntimeError(f"field {name} is not contiguous and writeable")
        # backend tables (torch_backend.py:56-63, 66-89)
        self.edges = _t(m.edges)
        self.face_edges = _t(m.face_edges)
        self.left = _t(m.edge_left_faces)
        self.right = _t(m.edge_right_faces)
        self.faces = _t(m.faces)
        self.face_signs = _t(sim.face_signs)
        self.v_edges = _t(sim.v_edges)
        self.v_signs = _t(sim.v_signs)
        for name in ("g_primal", "g_inv_primal", "g_dual", "g_inv_dual", "g_inv_dual_area", "g_inv_face_area",
                     "r", "inv_r", "mid", "inv_mid", "dr", "ctrl", "cd", "ca_er", "cb_er", "ca_et", "cb_et"):
            setattr(self, name, _t(getattr(sim, name)))
        self.full = sim.full
        self.compress = sim.compress
        self.dt = float(sim.dt)
        self.src_v = tuple(_t(a) for a in sim.src_v) if sim.src_v is not None else None
        self.src_t = tuple(_t(a) for a in sim.src_t) if sim.src_t is not None else None
        self.surface = sim.surface is not None
        if self.surface:
            self.si_memory = _t(sim.si_memory)
            if not np.shares_memory(sim.si_memory, self.si_memory.numpy()):
                raise RuntimeError("surface memory is not contiguous and writeable")
            self.si_decay, self.si_drive, self.si_hist, self.si_scale = (
                _t(getattr(sim, n)) for n in ("si_decay", "si_drive", "si_hist", "si_scale"))
        self.plasma = sim.plasma is not None
        if self.plasma:
            self.p_recon, self.p_centres, self.p_ltan, self.p_rtan, self.p_b = (
                _t(getattr(sim, n)) for n in ("p_recon", "p_centres", "p_ltan", "p_rtan", "p_b"))
            self.p_vfaces = _t(sim.p_vfaces)
            self.p_vweights = _t(sim.p_vweights)
            self.p_coef = [tuple(_t(c) for c in coef) for coef in sim.p_coef]
            self.p_current = [_t(j) for j in sim.p_current]
            for j_np, j_t in zip(sim.p_current, self.p_current):
                if not np.shares_memory(j_np, j_t.numpy()):
                    raise RuntimeError("plasma current is not contiguous and writeable")

    # -- primitives (torch_backend.py:172-198) ------------------------------

    def _edge_difference(self, values):
        return values[self.edges[:, 1]] - values[self.edges[:, 0]]

    def _dual_edge_difference(self, values):
        return values[self.left] - values[self.right]

    def _face_circulation(self, values):
        shape = (self.face_edges.shape[0],) + (1,) * (values.ndim - 1)
        out = values[self.face_edges[:, 0]]
        out.mul_(self.face_signs[:, 0].reshape(shape))
        for corner in (1, 2):
            term = values[self.face_edges[:, corner]]
            term.mul_(self.face_signs[:, corner].reshape(shape))
            out.add_(term)
        return out

    def _dual_cell_circulation(self, values):
        shape = (self.v_edges.shape[0],) + (1,) * (values.ndim - 1)
        out = values[self.v_edges[:, 0]]
        out.mul_(self.v_signs[:, 0].reshape(shape))
        for slot in range(1, self.v_edges.shape[1]):
            term = values[self.v_edges[:, slot]]
            term.mul_(self.v_signs[:, slot].reshape(shape))
            out.add_(term)
        return out

    # -- radial stencils (solver.py:443-465) --------------------------------

    def _d_et(self):
        vals = self.et * self.mid[None, :] if self.full else self.et
        out = torch.empty_like(self.ht)
        out[:, 0] = 2.0 * vals[:, 0] / self.dr[0]
        out[:, -1] = -2.0 * vals[:, -1] / self.dr[-1]
        if self.ht.shape[1] > 2:
            out[:, 1:-1] = torch.diff(vals, dim=1) / self.cd
        if self.full:
            out *= self.inv_r
        return out

    def _d_ht(self):
        vals = self.ht * self.r[None, :] if self.full else self.ht
        out = torch.diff(vals, dim=1) / self.dr[None, :]
        if self.full:
            out *= self.inv_mid
        return out

    # -- ADEs (surface_impedance.py:225-270, plasma.py:413-442, 489-527) -----

    def _surface_advance(self, h_old, e1, g0):
        hist = self.si_scale * (self.si_memory * self.si_hist[None, :]).sum(dim=1)
        gain = self.si_scale * self.si_hist.sum()
        k = 2.0 * self.dt / (MU_0 * self.dr[0])
        force = self.dt / MU_0 * g0
        c = k * gain
        h_new = ((1.0 - 0.5 * c) * h_old + force - k * e1 + k * hist) / (1.0 + 0.5 * c)
        self.si_memory.copy_(self.si_memory * self.si_decay[None, :] + (h_new + h_old)[:, None] * self.si_drive[None, :])
        return h_new

    @staticmethod
    def _cross(v, b):
        out = torch.empty_like(v)
        out[..., 0] = v[..., 1] * b[..., 2] - v[..., 2] * b[..., 1]
        out[..., 1] = v[..., 2] * b[..., 0] - v[..., 0] * b[..., 2]
        out[..., 2] = v[..., 0] * b[..., 1] - v[..., 1] * b[..., 0]
        return out

    def _plasma_advance(self):
        nodes = self.er[self.faces].sum(dim=1) / 3.0
        radial = 0.5 * (nodes[:, :-1] + nodes[:, 1:])
        ev = self.et[self.face_edges]
        tang = (ev[..., None] * self.p_recon[:, :, None, :]).sum(dim=1)
        efield = tang + radial[..., None] * self.p_centres[:, None, :]
        b = self.p_b
        total = torch.zeros_like(efield)
        e_par = (efield * b).sum(dim=2)[..., None] * b
        e_perp = efield - e_par
        e_x = self._cross(e_perp, b)
        for i, (decay, cs, sn, dpar, dre, dim) in enumerate(self.p_coef):
            j = self.p_current[i]
            j_par = (j * b).sum(dim=2)[..., None] * b
            j_perp = j - j_par
            j_x = self._cross(j_perp, b)
            new = (
                decay[..., None] * j_par
                + dpar[..., None] * e_par
                + decay[..., None] * (cs[..., None] * j_perp + sn[..., None] * j_x)
                + dre[..., None] * e_perp
                + dim[..., None] * e_x
            )
            j.copy_(new)
            total += new
        left = (total[self.left] * self.p_ltan[:, None, :]).sum(dim=2)
        right = (total[self.right] * self.p_rtan[:, None, :]).sum(dim=2)
        jt = 0.5 * (left + right)
        at_faces = (total * self.p_centres[:, None, :]).sum(dim=2)
        at_vertices = (at_faces[self.p_vfaces] * self.p_vweights[:, :, None]).sum(dim=1)
        jr = torch.zeros((at_vertices.shape[0], at_vertices.shape[1] + 1), dtype=at_vertices.dtype)
        jr[:, 0] = at_vertices[:, 0]
        jr[:, -1] = at_vertices[:, -1]
        if at_vertices.shape[1] > 1:
            jr[:, 1:-1] = 0.5 * (at_vertices[:, :-1] + at_vertices[:, 1:])
        return jr, jt

    # -- the step (solver.py:867-989) ----------------------------------------

    def update_magnetic(self) -> None:
        """solver.py:877-921."""

        g = self._edge_difference(self.er)
        g *= self.g_inv_primal
        g *= self.inv_r
        if self.surface:
            g0 = g[:, 0] + 0.0
            h_old = self.ht[:, 0] + 0.0
        g -= self._d_et()
        g *= self.dt / MU_0
        self.ht += g
        if self.surface:
            s = self.sim
            metric = s.midpoints_m[0] / s.radii_m[0] if self.full else 1.0
            self.ht[:, 0] = self._surface_advance(h_old, metric * self.et[:, 0], g0)
        circ = self._face_circulation(self.et * self.g_primal)
        circ *= self.g_inv_face_area
        circ *= self.inv_mid
        circ *= self.dt / MU_0
        self.hr -= circ

    def update_electric(self, current_a: float = 0.0) -> None:
        """solver.py:923-989."""

        pc = self._plasma_advance() if self.plasma else None
        mc = self._dual_cell_circulation(self.ht * self.g_dual)
        mc *= self.g_inv_dual_area
        mc *= self.inv_r
        dens = None
        if self.src_v is not None:
            v, k, w = self.src_v
            length = self.sim.source.vertical_element_length_m
            dens = w * current_a * length * self.g_inv_dual_area[v, 0] / self.r[k] ** 2 / self.ctrl[k]
        self.er *= self.ca_er
        mc *= self.cb_er
        self.er += mc
        if dens is not None:
            v, k, _ = self.src_v
            cv = torch.zeros_like(v) if self.compress else v
            self.er[v, k] -= self.cb_er[cv, k] * dens
        if pc is not None:
            self.er -= self.cb_er * pc[0]
        g = self._dual_edge_difference(self.hr)
        g *= self.g_inv_dual
        g *= self.inv_mid
        g -= self._d_ht()
        self.et *= self.ca_et
        g *= self.cb_et
        self.et += g
        if self.src_t is not None:
            e, k, w = self.src_t
            dens_t = w * current_a * self.g_inv_dual[e, 0] / self.mid[k] / self.dr[k]
            ce = torch.zeros_like(e) if self.compress else e
            self.et[e, k] -= self.cb_et[ce, k] * dens_t
        if pc is not None:
            self.et -= self.cb_et * pc[1]

    def step(self, count: int = 1) -> None:
        """solver.py:789-816 (eager path); the step counter and time live on the oracle."""

        s = self.sim
        for _ in range(count):
            current = s.current_at(s.steps)
            self.update_magnetic()
            self.update_electric(current)
            s.steps += 1
            s.time_s = s.steps * s.dt
