"""ctypes binding of the C ABI in ``include/pd_b200.h`` (``_build/libpdb200.so``).

The library is required: there is no CPU or PyTorch fallback of the solver
path, and a missing library raises :class:`LibraryMissing` on first use.
"""

from __future__ import annotations

import ctypes
import os
import threading
from pathlib import Path

import numpy as np

LIBRARY = Path(os.environ.get("PD_B200_LIBRARY", Path(__file__).resolve().parent / "_build" / "libpdb200.so"))

PD_OK = 0
PD_ERR_INVALID = 1
PD_ERR_CUDA = 2
PD_ERR_NOT_SPD = 3
PD_ERR_STATE = 4
PD_ERR_UNSUPPORTED = 5

STATUS_NOT_CONVERGED = 1
STATUS_SINGULAR = 2
STATUS_ACTIVATION = 4
STATUS_ADJOINT_NOT_CONVERGED = 8
STATUS_ADJOINT_SAFEGUARD = 16
STATUS_BARRIER_TIMEOUT = 1024

PRECISION_FP64 = 0
PRECISION_FP32_REFINE = 1
PRECISION_FP32 = 2
BATCH_TEAMS = 0
BATCH_PHASES = 1
ADJOINT_REFERENCE = 0
ADJOINT_EXACT = 1


class LibraryMissing(RuntimeError):
    """The compiled sm_100a library is absent; build it with ``python -m newton_solver_diff_phd_b200.build``."""


class PdMeshDesc(ctypes.Structure):
    _fields_ = [
        ("n_vertices", ctypes.c_int32),
        ("n_elements", ctypes.c_int32),
        ("corners", ctypes.c_int32),
        ("indices", ctypes.POINTER(ctypes.c_int32)),
        ("gradients", ctypes.POINTER(ctypes.c_double)),
        ("mean_volume", ctypes.c_double),
        ("free", ctypes.POINTER(ctypes.c_uint8)),
    ]


class PdOptions(ctypes.Structure):
    _fields_ = [
        ("material", ctypes.c_int32),
        ("max_iterations", ctypes.c_int32),
        ("abs_tol", ctypes.c_double),
        ("rel_tol", ctypes.c_double),
        ("anderson_window", ctypes.c_int32),
        ("density", ctypes.c_double),
        ("integrate_pinned_velocities", ctypes.c_int32),
        ("precision", ctypes.c_int32),
        ("adjoint_mode", ctypes.c_int32),
        ("blocks", ctypes.c_int32),
        ("resident", ctypes.c_int32),
        ("svd_warm_start", ctypes.c_int32),
        ("adjoint_solver", ctypes.c_int32),
        ("state_precision", ctypes.c_int32),
    ]


class PdDiffPdOptions(ctypes.Structure):
    _fields_ = [
        ("max_pd_iter", ctypes.c_int32),
        ("max_ls_iter", ctypes.c_int32),
        ("history", ctypes.c_int32),
        ("use_corotated", ctypes.c_int32),
        ("use_volume", ctypes.c_int32),
        ("corotated_weight", ctypes.c_double),
        ("volume_weight", ctypes.c_double),
        ("abs_tol", ctypes.c_double),
        ("rel_tol", ctypes.c_double),
        ("recursion", ctypes.c_int32),
    ]


DIFFPD_TWO_LOOP, DIFFPD_GRAM = 0, 1


class PdBatchOptions(ctypes.Structure):
    _fields_ = [
        ("svd_warm_start", ctypes.c_int32),
        ("task_nnz", ctypes.c_int32),
        ("run_gap", ctypes.c_int32),
        ("local_cells", ctypes.c_int32),
        ("schedule", ctypes.c_int32),
        ("team_nnz", ctypes.c_int32),
        ("team_samples", ctypes.c_int32),
        ("measured_us", ctypes.c_void_p),
        ("measured_iterations", ctypes.c_void_p),
        ("measured_team", ctypes.c_void_p),
        ("measured_adjoint_us", ctypes.c_void_p),
    ]


_P = ctypes.c_void_p
_I32 = ctypes.c_int32
_I64 = ctypes.c_int64
_D = ctypes.c_double

SIGNATURES = {
    "pd_version": ([], ctypes.c_char_p),
    "pd_last_error": ([], ctypes.c_char_p),
    "pd_create": ([ctypes.POINTER(PdMeshDesc), ctypes.POINTER(PdOptions), ctypes.c_int, ctypes.POINTER(_P)], ctypes.c_int),
    "pd_destroy": ([_P], ctypes.c_int),
    "pd_set_tolerances": ([_P, _I32, _D, _D], ctypes.c_int),
    "pd_set_anderson_window": ([_P, _I32], ctypes.c_int),
    "pd_set_materials": ([_P, _P], ctypes.c_int),
    "pd_set_muscles": ([_P, _P, _P], ctypes.c_int),
    "pd_set_muscle_targets": ([_P, _P], ctypes.c_int),
    "pd_set_activations": ([_P, _P], ctypes.c_int),
    "pd_set_planar_energies": ([_P, _I32, _P, _P, _P], ctypes.c_int),
    "pd_set_mesh_contact": ([_P, _D, _D, _D, _D, _D, _I32, _P, _I32, _P], ctypes.c_int),
    "pd_mesh_contact_force": ([_P, _P, _P, _P, _P, _P], ctypes.c_int),
    "pd_mesh_contact_pairs": ([_P, _P, _P], ctypes.c_int),
    "pd_set_frictional_boundary": ([_P, _I32, _P, _I32, _P, _D, _D, _I32, _I32, _P, _I32, _P], ctypes.c_int),
    "pd_frictional_buffers": ([_P, ctypes.POINTER(_P), ctypes.POINTER(_P), ctypes.POINTER(_I32)], ctypes.c_int),
    "pd_frictional_state": ([_P, _P, _P, _P, _P, _P], ctypes.c_int),
    "pd_set_woodbury_lanes": ([_P, _I32], ctypes.c_int),
    "pd_set_woodbury_team": ([_P, _I32], ctypes.c_int),
    "pd_build": ([_P, _D], ctypes.c_int),
    "pd_factor_stats": ([_P, ctypes.POINTER(_I64), ctypes.POINTER(_I64), ctypes.POINTER(_I64)], ctypes.c_int),
    "pd_step": ([_P, _P, _P, _P, _P, _P, _D, _P, _P, _P, _P], ctypes.c_int),
    "pd_backward": ([_P, _P, _P, _D, _P, _P, _P, _P, _P, _P, _P, _P, _P], ctypes.c_int),
    "pd_backward_contact": ([_P, _P, _P, _D] + [_P] * 12, ctypes.c_int),
    "pd_set_phase_timers": ([_P, _P], ctypes.c_int),
    "pd_set_spin_limit": ([_P, ctypes.c_uint32], ctypes.c_int),
    "pd_diffpd_set_state_forces": ([_P, _I32, _P, _P], ctypes.c_int),
    "pd_diffpd_step": ([_P, ctypes.POINTER(PdDiffPdOptions), _P, _P, _P, _P, _D, _P, _P, _P], ctypes.c_int),
    "pd_diffpd_results": ([_P, ctypes.POINTER(_P), ctypes.POINTER(_P), ctypes.POINTER(_I32), _P], ctypes.c_int),
    "pd_barrier_probe": ([ctypes.c_int, _I32, _I32, _I32, ctypes.c_uint32, _P, _P], ctypes.c_int),
    "pd_read_status": ([_P, ctypes.POINTER(_I32), _P], ctypes.c_int),
    "pd_iterations": ([_P, ctypes.POINTER(_I32), ctypes.POINTER(_I32), _P], ctypes.c_int),
    "pd_deformation_determinants": ([_P, _P, _P, _P], ctypes.c_int),
    "pd_apply_inverse": ([_P, _P, _P, _P], ctypes.c_int),
    "pd_apply_inverse_static": ([_P, _P, _P, _P], ctypes.c_int),
    "pd_batch_create": ([_P, _I32, ctypes.POINTER(PdBatchOptions), ctypes.POINTER(_P)], ctypes.c_int),
    "pd_batch_destroy": ([_P], ctypes.c_int),
    "pd_batch_layout": ([_P, _P, _P], ctypes.c_int),
    "pd_batch_factor_stats": ([_P, ctypes.POINTER(_I64), ctypes.POINTER(_I64), _P], ctypes.c_int),
    "pd_batch_forward": ([_P, _I32, _D, _P, _P, _P, _P, _I64, _P, _P, _P, _P], ctypes.c_int),
    "pd_batch_forward_stepwise": ([_P, _I32, _D, _P, _P, _P, _P, _I64, _P, _P, _P, _P], ctypes.c_int),
    "pd_batch_read": ([_P, _P, _P, _P], ctypes.c_int),
    "pd_batch_backward": ([_P, _I32, _D, _P, _P, _P, _P, _P, _P, _P, _P, _P], ctypes.c_int),
    "pd_batch_team_sizes": ([_P, _P, _P], ctypes.c_int),
    "pd_batch_timeline": ([_P, _P, _P, _P], ctypes.c_int),
    "pd_batch_set_phase_timers": ([_P, _I32, _P], ctypes.c_int),
    "pd_inverse_parallel_work": ([_I64], ctypes.c_int),
    "pd_inverse_parallel_levels": ([_I64], ctypes.c_int),
    "pd_factor_device_rows": ([_I32], ctypes.c_int),
    "pd_inverse_build": ([_I32, _P, _P, _P, ctypes.POINTER(_P)], ctypes.c_int),
    "pd_inverse_build_on": ([_I32, _I32, _P, _P, _P, ctypes.POINTER(_P)], ctypes.c_int),
    "pd_set_factor_device": ([_P, _I32], ctypes.c_int),
    "pd_inverse_sizes": ([_P, ctypes.POINTER(_I32), ctypes.POINTER(_I64), ctypes.POINTER(_I64)], ctypes.c_int),
    "pd_inverse_export": ([_P, _P, _P, _P, _P, _P, _P, _P], ctypes.c_int),
    "pd_inverse_free": ([_P], ctypes.c_int),
    "pd_inverse_run_sizes": ([_P, _I32, ctypes.POINTER(_I64), ctypes.POINTER(_I64), ctypes.POINTER(_I64),
                              ctypes.POINTER(_I64)], ctypes.c_int),
    "pd_inverse_run_export": ([_P, _I32] + [_P] * 9, ctypes.c_int),
}

_lock = threading.Lock()
_library = None


def library() -> ctypes.CDLL:
    """Load the compiled library once; raise :class:`LibraryMissing` when absent."""
    global _library
    with _lock:
        if _library is None:
            if not LIBRARY.exists():
                raise LibraryMissing(f"{LIBRARY} is missing; run `python -m newton_solver_diff_phd_b200.build`")
            lib = ctypes.CDLL(str(LIBRARY))
            for name, (arguments, result) in SIGNATURES.items():
                function = getattr(lib, name)
                function.argtypes = arguments
                function.restype = result
            _library = lib
        return _library


class PdError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(message)
        self.code = code


def check(code: int) -> None:
    """Raise the reference's exception type for a failed C call."""
    if code == PD_OK:
        return
    message = library().pd_last_error().decode()
    if code in (PD_ERR_INVALID, PD_ERR_NOT_SPD):
        raise ValueError(message)
    if code == PD_ERR_UNSUPPORTED:
        raise NotImplementedError(message)
    if code == PD_ERR_STATE:
        raise RuntimeError(message)
    raise PdError(code, message)


def ptr(array) -> int | None:
    """Address of a NumPy array (host) or a torch tensor (host or device); None passes NULL."""
    if array is None:
        return None
    if isinstance(array, np.ndarray):
        return array.ctypes.data
    return array.data_ptr()


def inverse_factor(matrix_csr, run_gap=None, device=None):
    """Build the exact inverse factor of an SPD CSR matrix with the C++ builder.

    ``matrix_csr`` is ``(offsets, columns, values)`` of the full symmetric matrix.
    Returns a dict with ``permutation`` and the CSR arrays of S and S^T; with
    ``run_gap`` also ``runs``, the postorder run format of both. ``device``: a
    CUDA device index computes the rows of L^{-1} there (bit-identical).
    """
    offsets, columns, values = (
        np.ascontiguousarray(matrix_csr[0], dtype=np.int32),
        np.ascontiguousarray(matrix_csr[1], dtype=np.int32),
        np.ascontiguousarray(matrix_csr[2], dtype=np.float64),
    )
    lib = library()
    handle = _P()
    if device is None:
        check(lib.pd_inverse_build(len(offsets) - 1, ptr(offsets), ptr(columns), ptr(values), ctypes.byref(handle)))
    else:
        check(lib.pd_inverse_build_on(int(device), len(offsets) - 1, ptr(offsets), ptr(columns), ptr(values),
                                      ctypes.byref(handle)))
    try:
        size, nnz, factorization = _I32(), _I64(), _I64()
        check(lib.pd_inverse_sizes(handle, ctypes.byref(size), ctypes.byref(nnz), ctypes.byref(factorization)))
        n, m = size.value, nnz.value
        out = {
            "permutation": np.empty(n, np.int32),
            "s_offsets": np.empty(n + 1, np.int32),
            "s_columns": np.empty(m, np.int32),
            "s_values": np.empty(m, np.float64),
            "st_offsets": np.empty(n + 1, np.int32),
            "st_columns": np.empty(m, np.int32),
            "st_values": np.empty(m, np.float64),
        }
        check(
            lib.pd_inverse_export(
                handle,
                *(ptr(out[k]) for k in ("permutation", "s_offsets", "s_columns", "s_values", "st_offsets", "st_columns", "st_values")),
            )
        )
        out["factorization_nnz"] = factorization.value
        if run_gap is not None:
            counts = [_I64() for _ in range(4)]
            check(lib.pd_inverse_run_sizes(handle, int(run_gap), *(ctypes.byref(c) for c in counts)))
            s_runs, s_values, st_runs, st_values = (c.value for c in counts)
            runs = {
                "label_of": np.empty(n, np.int32),
                "s_row_runs": np.empty(n + 1, np.int32),
                "s_run_col": np.empty(s_runs, np.int32),
                "s_run_off": np.empty(s_runs + 1, np.int32),
                "s_values": np.empty(s_values, np.float64),
                "st_row_runs": np.empty(n + 1, np.int32),
                "st_run_col": np.empty(st_runs, np.int32),
                "st_run_off": np.empty(st_runs + 1, np.int32),
                "st_values": np.empty(st_values, np.float64),
            }
            check(lib.pd_inverse_run_export(handle, int(run_gap), *(ptr(runs[k]) for k in runs)))
            out["runs"] = runs
        return out
    finally:
        lib.pd_inverse_free(handle)


def dense_to_csr(matrix):
    matrix = np.asarray(matrix, dtype=np.float64)
    offsets, columns, values = [0], [], []
    for row in matrix:
        nz = np.flatnonzero(row)
        columns.extend(nz.tolist())
        values.extend(row[nz].tolist())
        offsets.append(len(columns))
    return np.asarray(offsets), np.asarray(columns), np.asarray(values)


class DeviceView:
    """A library-owned device array as a ``__cuda_array_interface__`` object, so that
    ``torch.as_tensor(view, device=...)`` aliases it without a copy."""

    def __init__(self, pointer: int, shape: tuple, typestr: str, owner):
        self._owner = owner  # keeps the solver (and its allocation) alive
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": typestr, "data": (int(pointer), False),
                                         "version": 3, "strides": None}

