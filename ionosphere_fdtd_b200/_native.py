"""ctypes binding of ``libifdtd.so`` (the C ABI in ``include/ifdtd.h``).

The library is built in-tree by ``ionosphere_fdtd_b200.build``.  Loading
fails loudly when it is missing: there is no CPU fallback for the time step.
"""

from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from .errors import BackendUnavailableError

LIBRARY = Path(__file__).resolve().parent / "libifdtd.so"
MAX_SPECIES = 4
MAX_SOURCES = 16

OK, ERR_ARGUMENT, ERR_CUDA, ERR_NONFINITE, ERR_UNSUPPORTED = range(5)

_i32 = C.c_int32
_i64p = C.POINTER(C.c_int64)
_f64p = C.POINTER(C.c_double)
_vp = C.c_void_p


class MeshDesc(C.Structure):
    _fields_ = [
        ("n_vertices", _i32),
        ("n_edges", _i32),
        ("n_faces", _i32),
        ("edges", _i64p),
        ("faces", _i64p),
        ("face_edges", _i64p),
        ("face_edge_signs", _i64p),
        ("edge_left_faces", _i64p),
        ("edge_right_faces", _i64p),
        ("primal_edge_angles", _f64p),
        ("dual_edge_angles", _f64p),
        ("face_solid_angles", _f64p),
        ("dual_cell_solid_angles", _f64p),
    ]


class GridDesc(C.Structure):
    _fields_ = [
        ("radial_cells", _i32),
        ("full_spherical", _i32),
        ("radii_m", _f64p),
        ("time_step_s", C.c_double),
    ]


class PhysicsDesc(C.Structure):
    _fields_ = [
        ("coef_rows_er", _i32),
        ("coef_rows_et", _i32),
        ("ca_er", _f64p),
        ("cb_er", _f64p),
        ("ca_et", _f64p),
        ("cb_et", _f64p),
        ("n_src_er", _i32),
        ("src_er_vertex", _i64p),
        ("src_er_layer", _i64p),
        ("src_er_coef", _f64p),
        ("n_src_et", _i32),
        ("src_et_edge", _i64p),
        ("src_et_layer", _i64p),
        ("src_et_coef", _f64p),
        ("si_terms", _i32),
        ("si_scale", _f64p),
        ("si_decay", _f64p),
        ("si_drive", _f64p),
        ("si_history", _f64p),
        ("si_metric", C.c_double),
        ("plasma_species", _i32),
        ("plasma_rows", _i32),
        ("plasma_magnetized", _i32),
        ("plasma_coef", _f64p),
        ("plasma_bdir", _f64p),
        ("plasma_reconstruction", _f64p),
        ("face_centers", _f64p),
        ("plasma_tangent_left", _f64p),
        ("plasma_tangent_right", _f64p),
        ("vertex_face_width", _i32),
        ("vertex_faces", _i64p),
        ("vertex_face_weights", _f64p),
    ]


class Tuning(C.Structure):
    _fields_ = [("faces_per_patch", _i32), ("threads", _i32), ("graph_chunk", _i32), ("e_faces_per_patch", _i32), ("staging", _i32),
                ("producer_warps", _i32), ("lane_layout", _i32), ("e_threads", _i32), ("e_stages", _i32),
                ("e_producer_warps", _i32), ("e_copy_gap", _i32),
                ("fused_step", _i32), ("plasma_frame", _i32)]


class State(C.Structure):
    _fields_ = [
        ("er", _vp),
        ("et", _vp),
        ("hr", _vp),
        ("ht", _vp),
        ("si_memory", _vp),
        ("plasma_current", _vp * MAX_SPECIES),
    ]


_SIGNATURES = {
    "ifdtd_version": ([], _i32),
    "ifdtd_last_error": ([C.c_char_p, C.c_size_t], _i32),
    "ifdtd_device_count": ([C.POINTER(_i32)], _i32),
    "ifdtd_plan_create": (
        [C.POINTER(MeshDesc), C.POINTER(GridDesc), C.POINTER(PhysicsDesc), C.POINTER(Tuning), _i32, _i32, C.POINTER(_vp)],
        _i32,
    ),
    "ifdtd_plan_destroy": ([_vp], _i32),
    "ifdtd_plan_bytes": ([_vp, C.POINTER(C.c_int64)], _i32),
    "ifdtd_plan_layout": ([_vp, C.POINTER(_i32), C.POINTER(_i32)], _i32),
    "ifdtd_status_word": ([_vp, _i32, C.POINTER(_i32)], _i32),
    "ifdtd_plan_kernels": ([_vp, C.POINTER(_i32), C.POINTER(_i32)], _i32),
    "ifdtd_wait_selftest": ([_vp, C.POINTER(C.c_double), _vp], _i32),
    "ifdtd_step": ([_vp, C.POINTER(State), _vp, _i32, _vp], _i32),
    "ifdtd_step_static_scratch": ([_vp, C.POINTER(State), _vp, _i32, _vp], _i32),
    "ifdtd_update_magnetic": ([_vp, C.POINTER(State), _vp], _i32),
    "ifdtd_update_electric": ([_vp, C.POINTER(State), C.c_double, _vp], _i32),
    "ifdtd_time_phases": ([_vp, C.POINTER(State), _i32, C.POINTER(C.c_float), C.POINTER(C.c_float), _vp], _i32),
    "ifdtd_probe_create": ([_vp, _i32, _i32, _i32, _i64p, _i64p, _f64p, C.POINTER(_vp)], _i32),
    "ifdtd_probe_destroy": ([_vp], _i32),
    "ifdtd_sample": ([_vp, C.POINTER(State), _vp, _vp, _vp], _i32),
    "ifdtd_step_sampled": ([_vp, C.POINTER(State), _vp, _i32, _vp, _vp, _vp], _i32),
    "ifdtd_first_use_numbering": ([_i64p, _i64p, C.c_int64, C.c_int64, _i64p, _i64p, C.POINTER(C.c_int64)], _i32),
    "ifdtd_stable_group": ([_i64p, C.c_int64, C.c_int64, _i64p, _i64p], _i32),
    "ifdtd_batch_create": ([C.POINTER(_vp), _i32, _i32, C.POINTER(_vp)], _i32),
    "ifdtd_batch_destroy": ([_vp], _i32),
    "ifdtd_batch_step": ([_vp, C.POINTER(State), _vp, _i32, C.POINTER(_vp), C.POINTER(_vp), _vp], _i32),
    "ifdtd_batch_info": ([_vp, C.POINTER(_i32), C.POINTER(_i32), C.POINTER(_i32), C.POINTER(_i32)], _i32),
    "ifdtd_max_abs": ([_vp, C.POINTER(State), _vp, _vp], _i32),
    "ifdtd_nn_gemm": ([_i32, _i32, _i32, _vp, _i32, _i32, _vp, _i32, _i32, C.c_float, C.c_float, _vp, _i32, _vp], _i32),
    "ifdtd_nn_gemm_tc": ([_i32, _i32, _i32, _vp, _i32, _i32, _vp, _i32, _i32, C.c_float, C.c_float, _vp, _i32, _vp], _i32),
    "ifdtd_nn_gemm_tc_ws": ([_i32, _i32, _i32, _vp, _i32, _i32, _vp, _i32, _i32, C.c_float, C.c_float, _vp, _i32, _vp, C.c_int64, _vp],
                            _i32),
    "ifdtd_nn_gemm_tc_status": ([_i32, C.POINTER(_i32)], _i32),
    "ifdtd_nn_bias_act": ([_i32, _i32, _vp, _vp, _i32, _vp, _vp], _i32),
    "ifdtd_nn_act_grad": ([_i32, _i32, _vp, _vp, _i32, _vp, _vp, _vp], _i32),
    "ifdtd_nn_col_sum": ([_i32, _i32, _vp, _vp, _vp], _i32),
    "ifdtd_nn_mse": ([_i32, _vp, _vp, _vp, _vp, _vp], _i32),
    "ifdtd_nn_wmse": ([_i32, _i32, _vp, _vp, _vp, _vp, _vp, _vp], _i32),
    "ifdtd_nn_adam": ([_i32, _vp, _vp, _vp, _vp, C.c_float, C.c_float, C.c_float, C.c_float, _i32, _vp, _vp], _i32),
    "ifdtd_nn_to_bf16": ([C.c_int64, _vp, _vp, _vp], _i32),
    "ifdtd_edge_difference": ([_vp, _vp, _i32, _vp, _vp], _i32),
    "ifdtd_dual_edge_difference": ([_vp, _vp, _i32, _vp, _vp], _i32),
    "ifdtd_face_circulation": ([_vp, _vp, _i32, _vp, _vp], _i32),
    "ifdtd_dual_cell_circulation": ([_vp, _vp, _i32, _vp, _vp], _i32),
}

_lib: C.CDLL | None = None


def exported_symbols() -> tuple[str, ...]:
    return tuple(_SIGNATURES)


def load() -> C.CDLL:
    """Load (and bind) the CUDA library; raise if it was not built."""

    global _lib
    if _lib is not None:
        return _lib
    if not LIBRARY.exists():
        raise BackendUnavailableError(
            f"{LIBRARY.name} is not built; run `python -m ionosphere_fdtd_b200.build` (needs nvcc)"
        )
    lib = C.CDLL(str(LIBRARY))
    for name, (args, res) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _lib = lib
    return lib


def last_error() -> str:
    buf = C.create_string_buffer(1024)
    load().ifdtd_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(status: int, what: str) -> None:
    """Map an ifdtd_status to the reference's exception types."""

    if status == OK:
        return
    message = f"{what}: {last_error()}"
    if status == ERR_ARGUMENT:
        raise ValueError(message)
    if status == ERR_UNSUPPORTED:
        raise BackendUnavailableError(message)
    raise RuntimeError(message)


def row_pitch(n: int) -> int:
    """Row pitch (elements) the plan uses for a radial extent of n samples:
    n rounded up to a multiple of 4, so rows are 16-byte aligned."""

    return (int(n) + 3) // 4 * 4


def i64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.int64)


def f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def ptr_i64(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(_i64p)


def ptr_f64(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(_f64p)
