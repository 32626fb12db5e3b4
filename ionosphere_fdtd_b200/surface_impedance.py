"""Diffusive conductive half-space impedance and its ADE state.

Same fit and coefficients as the reference (surface_impedance.py:14-289).
The ADE update itself runs inside the CUDA H-phase kernel; this module owns
the model, the per-edge/per-pole coefficients and the ``memory`` state array
(a device tensor of shape (E, terms)).
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Any

import numpy as np
from numpy.typing import NDArray

from .constants import MU_0


@dataclass(frozen=True, slots=True)
class ConductiveHalfSpaceSurface:
    """Positive-real log-pole fit of Z(s) = sqrt(mu s / sigma)."""

    conductivity_s_m: float | NDArray[np.float64]
    minimum_frequency_hz: float = 5.0
    maximum_frequency_hz: float = 45.0
    terms: int = 16
    pole_span_decades: float = 5.0
    permeability_h_m: float = MU_0

    def __post_init__(self) -> None:
        sigma = np.asarray(self.conductivity_s_m, dtype=np.float64)
        if sigma.ndim > 1 or sigma.size == 0:
            raise ValueError("surface conductivity must be scalar or one-dimensional")
        sigma = sigma.reshape(-1)
        if not np.all(np.isfinite(sigma)) or np.any(sigma <= 0.0):
            raise ValueError("surface conductivity must be finite and positive")
        if not all(np.isfinite(v) for v in (self.minimum_frequency_hz, self.maximum_frequency_hz, self.pole_span_decades, self.permeability_h_m)):
            raise ValueError("surface impedance controls must be finite")
        if not 0.0 < self.minimum_frequency_hz < self.maximum_frequency_hz:
            raise ValueError("surface impedance frequency band is invalid")
        if isinstance(self.terms, bool) or not isinstance(self.terms, (int, np.integer)) or self.terms < 1:
            raise ValueError("surface impedance terms must be a positive integer")
        if self.pole_span_decades <= 0.0 or self.permeability_h_m <= 0.0:
            raise ValueError("surface impedance span and permeability must be positive")
        sigma = np.array(sigma, copy=True)
        sigma.setflags(write=False)
        object.__setattr__(self, "conductivity_s_m", sigma)

    @property
    def pole_rates_s_inv(self) -> NDArray[np.float64]:
        widen = self.pole_span_decades * np.log(10.0)
        lower = np.log(2.0 * np.pi * self.minimum_frequency_hz) - widen
        upper = np.log(2.0 * np.pi * self.maximum_frequency_hz) + widen
        step = (upper - lower) / self.terms
        return np.exp(lower + (np.arange(self.terms) + 0.5) * step)

    @property
    def diffusive_weights_sqrt_s_inv(self) -> NDArray[np.float64]:
        poles = self.pole_rates_s_inv
        if self.terms > 1:
            spacing = np.log(poles[-1] / poles[0]) / (self.terms - 1)
        else:
            spacing = np.log(self.maximum_frequency_hz / self.minimum_frequency_hz) + 2.0 * self.pole_span_decades * np.log(10.0)
        return spacing * np.sqrt(poles) / np.pi

    def conductivity_for_edges(self, edge_count: int, edge_indices=None) -> NDArray[np.float64]:
        sigma = np.asarray(self.conductivity_s_m)
        if edge_indices is not None:
            idx = np.asarray(edge_indices, dtype=np.int64)
            if sigma.size == 1:
                return np.full(len(idx), sigma[0])
            if sigma.size != edge_count:
                raise ValueError("surface conductivity does not match mesh edges")
            return sigma[idx]
        if sigma.size == 1:
            return np.full(edge_count, sigma[0])
        if sigma.size != edge_count:
            raise ValueError("surface conductivity does not match mesh edges")
        return np.array(sigma, copy=True)

    def impedance_ohm(self, frequency_hz) -> NDArray[np.complex128]:
        f = np.asarray(frequency_hz, dtype=np.float64)
        if not np.all(np.isfinite(f)) or np.any(f <= 0.0):
            raise ValueError("surface impedance frequencies must be positive")
        s = 2j * np.pi * f.reshape(-1)
        root = np.sum(self.diffusive_weights_sqrt_s_inv[:, None] * s[None, :] / (s[None, :] + self.pole_rates_s_inv[:, None]), axis=0)
        scale = np.sqrt(self.permeability_h_m / np.asarray(self.conductivity_s_m))
        return scale[:, None] * root[None, :]

    def exact_impedance_ohm(self, frequency_hz) -> NDArray[np.complex128]:
        f = np.asarray(frequency_hz, dtype=np.float64)
        if not np.all(np.isfinite(f)) or np.any(f <= 0.0):
            raise ValueError("surface impedance frequencies must be positive")
        s = 2j * np.pi * f.reshape(-1)
        scale = np.sqrt(self.permeability_h_m / np.asarray(self.conductivity_s_m))
        return scale[:, None] * np.sqrt(s)[None, :]

    def to_metadata(self) -> dict[str, Any]:
        return {
            "type": "conductive-half-space-diffusive",
            "conductivity_s_m": np.asarray(self.conductivity_s_m).tolist(),
            "minimum_frequency_hz": self.minimum_frequency_hz,
            "maximum_frequency_hz": self.maximum_frequency_hz,
            "terms": int(self.terms),
            "pole_span_decades": self.pole_span_decades,
            "permeability_h_m": self.permeability_h_m,
        }

    @classmethod
    def from_metadata(cls, metadata: dict[str, Any]) -> "ConductiveHalfSpaceSurface":
        if metadata.get("type") != "conductive-half-space-diffusive":
            raise ValueError("unsupported surface impedance model")
        return cls(
            conductivity_s_m=np.asarray(metadata["conductivity_s_m"]),
            minimum_frequency_hz=metadata["minimum_frequency_hz"],
            maximum_frequency_hz=metadata["maximum_frequency_hz"],
            terms=metadata["terms"],
            pole_span_decades=metadata["pole_span_decades"],
            permeability_h_m=metadata["permeability_h_m"],
        )


class SurfaceImpedanceADE:
    """Trapezoidal ADE coefficients and device memory for the lower boundary."""

    def __init__(self, model: ConductiveHalfSpaceSurface, *, edge_count: int, time_step_s: float, backend: Any) -> None:
        self.model = model
        self.backend = backend
        sigma = model.conductivity_for_edges(edge_count)
        poles = model.pole_rates_s_inv
        weights = model.diffusive_weights_sqrt_s_inv
        alpha = 0.5 * time_step_s * poles
        self.decay_host = (1.0 - alpha) / (1.0 + alpha)
        self.drive_host = alpha / (1.0 + alpha)
        self.history_host = weights / (1.0 + alpha)
        self.scale_host = np.sqrt(model.permeability_h_m / sigma)
        self._decay = backend.asarray(self.decay_host)
        self._drive = backend.asarray(self.drive_host)
        self._history_weights = backend.asarray(self.history_host)
        self._scale = backend.asarray(self.scale_host)
        self.memory = backend.zeros((edge_count, model.terms))

    # -- array-level updates (surface_impedance.py:205-270) -------------------------
    # The engine's H kernel applies the lower-boundary update inside the step; these
    # are the same formulas on the backend's arrays for callers that drive the ADE
    # directly (harmonic-response checks, custom boundary experiments).

    def _history(self, rows):
        memory = self.memory if rows is None else self.memory[rows]
        scale = self._scale if rows is None else self._scale[rows]
        history = scale * (memory * self._history_weights[None, :]).sum(axis=1)
        return memory, history, scale * self._history_weights.sum()

    def _store_memory(self, memory, h_old, h_new, rows) -> None:
        """Trapezoidal pole memories: m <- m (1 - a) / (1 + a) + (h_old + h_new) a / (1 + a)."""

        updated = memory * self._decay[None, :] + (h_new + h_old)[:, None] * self._drive[None, :]
        if rows is None:
            self.memory[:] = updated
        else:
            self.memory[rows] = updated

    def advance_prescribed_magnetic(self, h_old, h_new, *, rows=None):
        """Boundary E for a prescribed H history, advancing the memories
        (surface_impedance.py:205-223): E = history - gain x (H_old + H_new) / 2."""

        memory, history, gain = self._history(rows)
        electric = history - gain * (0.5 * (h_new + h_old))
        self._store_memory(memory, h_old, h_new, rows)
        return electric

    def advance_lower_boundary(self, h_old, electric_first_cell, surface_gradient_er, radial_step_m, time_step_s, *, rows=None):
        """Implicit lower-boundary Ht coupled to the impedance memories
        (surface_impedance.py:225-254); the engine's H kernel runs the same update."""

        memory, history, gain = self._history(rows)
        kappa = 2.0 * time_step_s / (MU_0 * radial_step_m)
        coupling = kappa * gain
        h_new = ((1.0 - 0.5 * coupling) * h_old + time_step_s / MU_0 * surface_gradient_er
                 - kappa * electric_first_cell + kappa * history) / (1.0 + 0.5 * coupling)
        self._store_memory(memory, h_old, h_new, rows)
        return h_new

    @property
    def state_bytes(self) -> int:
        return self.backend.nbytes(self.memory)

    @property
    def persistent_bytes(self) -> int:
        return sum(self.backend.nbytes(a) for a in (self.memory, self._decay, self._drive, self._history_weights, self._scale))
