"""CUDA array backend: the reference's ``ArrayBackend`` seam on B200.

``CudaBackend`` has the same name ("torch"), attributes and methods as the
reference's ``TorchBackend`` (backends/torch_backend.py:15-222) restricted to
CUDA devices.  Arrays are torch tensors (PyTorch is the device-memory and
stream plumbing); the four topology primitives run as CUDA kernels of
``libifdtd.so``.  The time step itself does not go through these primitives:
it is one fused H launch and one fused E launch per step (see ``engine``).
"""

from __future__ import annotations

from abc import ABC, abstractmethod
from collections.abc import Callable
from typing import Any

import numpy as np

from . import _native as N
from .errors import BackendUnavailableError


def _torch():
    try:
        import torch
    except ImportError as error:  # pragma: no cover - torch is part of the image
        raise BackendUnavailableError("PyTorch is required for device memory and streams") from error
    return torch


class ArrayBackend(ABC):
    """The array operations the time integrator needs (the reference's backend
    contract, backends/base.py:19-89): allocation and transfer, adjacent
    differences, the four oriented topology sums, and host reads.  ``CudaBackend``
    is the only implementation here; the contract is kept so that code written
    against the reference's seam (type checks, duck-typed callers) keeps working."""

    name: str
    device: str
    dtype_name: str
    threads: int | None = None

    def compile_step(self, step: Callable[[Any], None]) -> Callable[[Any], None]:
        raise BackendUnavailableError(f"the {self.name} backend does not support compiled field steps")

    def synchronize(self) -> None:
        """Wait for queued device work (no-op for synchronous backends)."""

    @abstractmethod
    def asarray(self, values: Any) -> Any: ...

    @abstractmethod
    def index_array(self, values: Any) -> Any: ...

    @abstractmethod
    def zeros(self, shape: tuple[int, ...]) -> Any: ...

    @abstractmethod
    def empty_like(self, values: Any) -> Any: ...

    @abstractmethod
    def diff(self, values: Any, axis: int) -> Any: ...

    @abstractmethod
    def edge_difference(self, vertex_values: Any) -> Any: ...

    @abstractmethod
    def dual_edge_difference(self, face_values: Any) -> Any: ...

    @abstractmethod
    def face_circulation(self, edge_values: Any) -> Any: ...

    @abstractmethod
    def dual_cell_circulation(self, edge_values: Any) -> Any: ...

    @abstractmethod
    def to_numpy(self, values: Any) -> np.ndarray: ...

    @abstractmethod
    def scalar(self, value: Any) -> float: ...

    @abstractmethod
    def max_abs(self, values: Any) -> float: ...

    @abstractmethod
    def nbytes(self, values: Any) -> int: ...


class CudaBackend(ArrayBackend):
    """Tensor plumbing on one CUDA device plus the CUDA topology primitives."""

    name = "torch"
    threads = None

    def __init__(self, mesh: Any, *, device: str = "auto", dtype: str = "auto", threads: int | None = None):
        torch = _torch()
        self.torch = torch
        if threads is not None:
            if isinstance(threads, bool) or not isinstance(threads, (int, np.integer)) or threads < 1:
                raise ValueError("torch_threads must be a positive integer")
            raise BackendUnavailableError("torch_threads is only valid for the PyTorch CPU backend")
        self.torch_device = self._resolve_device(device)
        self.device = str(self.torch_device)
        if dtype == "auto":
            dtype = "float32"
        if dtype not in {"float32", "float64"}:
            raise ValueError("dtype must be 'auto', 'float32', or 'float64'")
        self.dtype = torch.float32 if dtype == "float32" else torch.float64
        self.dtype_name = dtype
        self.itemsize = 4 if dtype == "float32" else 8
        self.mesh = mesh
        self.n_vertices = mesh.n_vertices
        self.edges = self.index_array(mesh.edges)
        self.face_edges = self.index_array(mesh.face_edges)
        self.face_edge_signs = self.asarray(mesh.face_edge_signs)
        self.edge_left_faces = self.index_array(mesh.edge_left_faces)
        self.edge_right_faces = self.index_array(mesh.edge_right_faces)
        self._engine = None  # set by the solver; primitives then share its tables

    # -- device resolution (torch_backend.py:104-149, CUDA only) -------------

    def _resolve_device(self, requested: str):
        torch = self.torch
        requested = str(requested).lower()
        if requested in {"auto", "gpu"}:
            requested = "cuda"
        if not requested.startswith("cuda"):
            raise BackendUnavailableError(
                "this engine runs the time step on CUDA (B200) only; device must be cuda, cuda:N, gpu or auto"
            )
        if not torch.cuda.is_available():
            raise BackendUnavailableError("CUDA is unavailable in this PyTorch runtime")
        try:
            device = torch.device(requested)
        except (RuntimeError, ValueError) as error:
            raise BackendUnavailableError(f"unsupported PyTorch device: {requested}") from error
        if device.index is not None and device.index >= torch.cuda.device_count():
            raise BackendUnavailableError(
                f"CUDA device index {device.index} is unavailable; found {torch.cuda.device_count()} device(s)"
            )
        if device.index is None:
            device = torch.device("cuda", torch.cuda.current_device())
        return device

    def compile_step(self, step: Callable[[Any], None]) -> Callable[[Any], None]:
        """Steps are always native CUDA launches; chunks are replayed as CUDA graphs."""

        return step

    def synchronize(self) -> None:
        self.torch.cuda.synchronize(self.torch_device)

    def stream_handle(self) -> int:
        return int(self.torch.cuda.current_stream(self.torch_device).cuda_stream)

    # -- array plumbing -------------------------------------------------------

    def asarray(self, values: Any):
        if self.torch.is_tensor(values):
            return values.detach().to(device=self.torch_device, dtype=self.dtype).clone()
        return self.torch.tensor(np.asarray(values), dtype=self.dtype, device=self.torch_device)

    def index_array(self, values: Any):
        return self.torch.tensor(np.asarray(values), dtype=self.torch.long, device=self.torch_device)

    def zeros(self, shape: tuple[int, ...]):
        return self.torch.zeros(shape, dtype=self.dtype, device=self.torch_device)

    def empty_like(self, values: Any):
        return self.torch.empty_like(values)

    def diff(self, values: Any, axis: int):
        return self.torch.diff(values, dim=axis)

    def to_numpy(self, values: Any) -> np.ndarray:
        if not self.torch.is_tensor(values):
            return np.asarray(values)
        return values.detach().cpu().numpy()

    def scalar(self, value: Any) -> float:
        return float(value.detach().item())

    def max_abs(self, values: Any) -> float:
        return float(self.torch.max(self.torch.abs(values)).detach().item())

    def nbytes(self, values: Any) -> int:
        return int(values.numel() * values.element_size())

    # -- topology primitives (CUDA kernels) ------------------------------------

    def _primitive_engine(self):
        if self._engine is None:
            from .engine import topology_engine

            self._engine = topology_engine(self.mesh, self)
        return self._engine

    def _primitive(self, fn_name: str, values: Any, rows_out: int):
        torch = self.torch
        x = values if torch.is_tensor(values) else self.asarray(values)
        x = x.to(device=self.torch_device, dtype=self.dtype).contiguous()
        trailing = tuple(x.shape[1:])
        cols = int(np.prod(trailing)) if trailing else 1
        out = torch.empty((rows_out,) + trailing, dtype=self.dtype, device=self.torch_device)
        engine = self._primitive_engine()
        fn = getattr(N.load(), fn_name)
        N.check(fn(engine.plan, x.data_ptr(), cols, out.data_ptr(), self.stream_handle()), fn_name)
        return out

    def edge_difference(self, vertex_values: Any):
        return self._primitive("ifdtd_edge_difference", vertex_values, self.mesh.n_edges)

    def dual_edge_difference(self, face_values: Any):
        return self._primitive("ifdtd_dual_edge_difference", face_values, self.mesh.n_edges)

    def face_circulation(self, edge_values: Any):
        return self._primitive("ifdtd_face_circulation", edge_values, self.mesh.n_faces)

    def dual_cell_circulation(self, edge_values: Any):
        return self._primitive("ifdtd_dual_cell_circulation", edge_values, self.mesh.n_vertices)


def create_backend(name: str, mesh: Any, *, device: str = "auto", dtype: str = "auto", torch_threads: int | None = None) -> CudaBackend:
    """Backend factory with the reference's signature (backends/__init__.py:12-33)."""

    normalized = str(name).lower()
    if normalized in {"torch", "pytorch", "cuda"}:
        return CudaBackend(mesh, device=device, dtype=dtype, threads=torch_threads)
    if normalized == "numpy":
        raise BackendUnavailableError(
            "this engine runs the time step on CUDA only; use backend='torch' with a CUDA device"
        )
    raise ValueError("backend must be 'numpy' or 'torch'")


# The reference's name for its PyTorch backend (backends/torch_backend.py:13); here
# it is the CUDA-only engine backend.
TorchBackend = CudaBackend
