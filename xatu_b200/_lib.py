"""ctypes binding of the engine's C ABI (include/xatu_bse.h).

Loads ``xatu_b200/_lib/libxatu_bse.so`` built in-tree by ``xatu_b200.build``.
There is no fallback: if the library is missing or a CUDA device is not
available, the calls raise.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libxatu_bse.so")

XATU_OK = 0
XATU_ERR_INVALID = 1
STATUS_NAMES = {0: "XATU_OK", 1: "XATU_ERR_INVALID", 2: "XATU_ERR_CUDA", 3: "XATU_ERR_NOT_CONVERGED",
                4: "XATU_ERR_STATE", 5: "XATU_ERR_ALLOC", 6: "XATU_ERR_UNSUPPORTED", 7: "XATU_ERR_NUMERIC"}

MODE_REALSPACE, MODE_RECIPROCAL = 0, 1
POT_KELDYSH, POT_COULOMB = 0, 1
GAUGE_LATTICE, GAUGE_ATOMIC = 0, 1
PREC_FP64, PREC_MIXED = 0, 1
SOLVER_DENSE_FP64, SOLVER_DAVIDSON = 0, 1
BROAD_OTHER, BROAD_LORENTZIAN, BROAD_GAUSSIAN, BROAD_EXPONENTIAL = 0, 1, 2, 3

EXPORTED_SYMBOLS = [
    "xatu_ctx_create", "xatu_ctx_destroy", "xatu_last_error", "xatu_ctx_set_stream", "xatu_abi_version",
    "xatu_system_upload", "xatu_exciton_set", "xatu_bands_compute", "xatu_bands_upload", "xatu_bands_download",
    "xatu_interaction_build", "xatu_motif_ft_download", "xatu_bse_build", "xatu_bse_dim", "xatu_bse_copy_to_host",
    "xatu_bse_device_buffers", "xatu_bse_solve", "xatu_davidson_config", "xatu_davidson_stats", "xatu_stage_times",
    "xatu_hx_backend", "xatu_bands_backend", "xatu_kernel_matvec", "xatu_kernel_stats", "xatu_hx_noalloc", "xatu_oscillator_strength",
    "xatu_state_observables", "xatu_realspace_amplitude", "xatu_envelope_ft", "xatu_absorption",
    "xatu_bse_build_basis", "xatu_adjoint", "xatu_oscillator_window_gradient", "xatu_batch_create", "xatu_batch_destroy", "xatu_batch_last_error",
    "xatu_batch_set_stream", "xatu_batch_add", "xatu_batch_run", "xatu_batch_dim", "xatu_batch_result",
    "xatu_batch_stats",
    "xatu_kernel_launches", "xatu_selftest_small_eigh", "xatu_reciprocal_lattice", "xatu_mesh_mp", "xatu_mesh_reduced",
    "xatu_equivalent_points", "xatu_truncate_supercell",
]


class XatuError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class SystemDesc(ctypes.Structure):
    _fields_ = [("ndim", ctypes.c_int), ("bravais", ctypes.c_void_p), ("natoms", ctypes.c_int),
                ("motif", ctypes.c_void_p), ("nspecies", ctypes.c_int), ("norbitals", ctypes.c_void_p),
                ("ncells", ctypes.c_int), ("cells", ctypes.c_void_p), ("hamiltonian", ctypes.c_void_p),
                ("overlap", ctypes.c_void_p), ("filling", ctypes.c_int), ("is_triangular", ctypes.c_int),
                ("is_au", ctypes.c_int)]


class ExcitonDesc(ctypes.Structure):
    _fields_ = [("ncell", ctypes.c_int), ("factor", ctypes.c_int), ("nk", ctypes.c_int),
                ("kpoints", ctypes.c_void_p), ("nmesh", ctypes.c_int), ("mesh", ctypes.c_void_p),
                ("nvalence", ctypes.c_int), ("nconduction", ctypes.c_int), ("valence_bands", ctypes.c_void_p),
                ("conduction_bands", ctypes.c_void_p), ("eps_m", ctypes.c_double), ("eps_s", ctypes.c_double),
                ("r0", ctypes.c_double), ("regularization", ctypes.c_double), ("cutoff", ctypes.c_double),
                ("Q", ctypes.c_double * 3), ("scissor", ctypes.c_double), ("exchange", ctypes.c_int),
                ("mode", ctypes.c_int), ("n_reciprocal", ctypes.c_int), ("potential", ctypes.c_int),
                ("exchange_potential", ctypes.c_int), ("gauge", ctypes.c_int)]


_lib = None


def lib() -> ctypes.CDLL:
    """The loaded engine library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"engine library not built: {LIB_PATH} (run `python -m xatu_b200.build`)")
    L = ctypes.CDLL(LIB_PATH)
    vp, ci, cd_, i64p = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.POINTER(ctypes.c_int64)
    sig = {
        "xatu_ctx_create": ([ctypes.POINTER(vp), ci], ci),
        "xatu_ctx_destroy": ([vp], ci),
        "xatu_last_error": ([vp], ctypes.c_char_p),
        "xatu_ctx_set_stream": ([vp, vp], ci),
        "xatu_abi_version": ([], ci),
        "xatu_system_upload": ([vp, ctypes.POINTER(SystemDesc)], ci),
        "xatu_exciton_set": ([vp, ctypes.POINTER(ExcitonDesc)], ci),
        "xatu_bands_compute": ([vp], ci),
        "xatu_bands_upload": ([vp, vp, vp, vp, vp], ci),
        "xatu_bands_download": ([vp, vp, vp, vp, vp], ci),
        "xatu_interaction_build": ([vp], ci),
        "xatu_motif_ft_download": ([vp, vp, vp], ci),
        "xatu_bse_build": ([vp, ci], ci),
        "xatu_bse_dim": ([vp, i64p], ci),
        "xatu_bse_copy_to_host": ([vp, vp], ci),
        "xatu_bse_device_buffers": ([vp, ctypes.POINTER(vp), ctypes.POINTER(vp), ctypes.POINTER(vp)], ci),
        "xatu_bse_solve": ([vp, ci, ci, vp, vp], ci),
        "xatu_davidson_config": ([vp, cd_, ci, ci], ci),
        "xatu_davidson_stats": ([vp, ctypes.POINTER(ci), ctypes.POINTER(cd_)], ci),
        "xatu_stage_times": ([vp, ctypes.POINTER(ctypes.c_float)], ci),
        "xatu_hx_backend": ([vp, ci], ci),
        "xatu_bands_backend": ([vp, ci], ci),
        "xatu_kernel_matvec": ([vp, ci, vp, vp], ci),
        "xatu_kernel_stats": ([vp, ci, i64p, ctypes.POINTER(cd_), ctypes.POINTER(ci)], ci),
        "xatu_hx_noalloc": ([vp, vp, vp, ctypes.c_int64, ctypes.c_int64, ci, vp, vp, vp], ci),
        "xatu_oscillator_strength": ([vp, ci, vp, vp], ci),
        "xatu_state_observables": ([vp, ci, vp, vp, vp, vp, vp], ci),
        "xatu_realspace_amplitude": ([vp, ci, vp, ci, vp, ci, vp, vp], ci),
        "xatu_envelope_ft": ([vp, ci, vp, ci, vp, vp], ci),
        "xatu_absorption": ([vp, ci, vp, vp, cd_, cd_, ci, cd_, ci, vp, vp, vp], ci),
        "xatu_bse_build_basis": ([vp, ci, ctypes.c_int64, vp], ci),
        "xatu_adjoint": ([vp, ci, vp, vp, vp], ci),
        "xatu_oscillator_window_gradient": ([vp, ctypes.c_double, ctypes.c_double, vp, vp, vp, vp], ci),
        "xatu_batch_create": ([vp, ci], ci),
        "xatu_batch_destroy": ([vp], ci),
        "xatu_batch_last_error": ([vp], ctypes.c_char_p),
        "xatu_batch_set_stream": ([vp, vp], ci),
        "xatu_batch_add": ([vp, vp, vp, vp], ci),
        "xatu_batch_run": ([vp, ci, ctypes.c_double, ci], ci),
        "xatu_batch_dim": ([vp, ci, i64p], ci),
        "xatu_batch_result": ([vp, ci, vp, vp], ci),
        "xatu_batch_stats": ([vp, vp, vp, vp, vp, vp, ctypes.c_size_t], ci),
        "xatu_kernel_launches": ([vp, i64p], ci),
        "xatu_selftest_small_eigh": ([ci, ci, ci, vp, vp, vp, vp], ci),
        "xatu_reciprocal_lattice": ([ci, vp, vp], ci),
        "xatu_mesh_mp": ([ci, vp, ci, vp], ci),
        "xatu_mesh_reduced": ([ci, vp, ci, ci, vp], ci),
        "xatu_equivalent_points": ([ci, vp, ci, ci, vp, vp], ci),
        "xatu_truncate_supercell": ([ci, vp, ci, cd_, ctypes.POINTER(ci), vp], ci),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return L


def ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data


def check(status: int, ctx=None):
    if status != XATU_OK:
        msg = lib().xatu_last_error(ctx).decode() if ctx else "(no context)"
        raise XatuError(status, msg)


# ------------------------------------------------------------------ geometry helpers (host)
def reciprocal_lattice(ndim: int, bravais: np.ndarray) -> np.ndarray:
    b = np.ascontiguousarray(bravais, dtype=np.float64).reshape(-1, 3)
    out = np.zeros((ndim, 3))
    check(lib().xatu_reciprocal_lattice(ndim, ptr(b), ptr(out)))
    return out


def mesh_mp(ndim: int, recip: np.ndarray, n: int) -> np.ndarray:
    r = np.ascontiguousarray(recip, dtype=np.float64)
    out = np.zeros((n ** ndim, 3))
    check(lib().xatu_mesh_mp(ndim, ptr(r), n, ptr(out)))
    return out


def mesh_reduced(ndim: int, recip: np.ndarray, n: int, factor: int) -> np.ndarray:
    r = np.ascontiguousarray(recip, dtype=np.float64)
    out = np.zeros((n ** ndim, 3))
    check(lib().xatu_mesh_reduced(ndim, ptr(r), n, factor, ptr(out)))
    return out


def equivalent_points(ndim: int, recip: np.ndarray, n_eff: int, k: np.ndarray) -> np.ndarray:
    r = np.ascontiguousarray(recip, dtype=np.float64)
    kk = np.ascontiguousarray(k, dtype=np.float64).reshape(-1, 3)
    out = np.zeros(kk.shape[0], dtype=np.int32)
    check(lib().xatu_equivalent_points(ndim, ptr(r), n_eff, kk.shape[0], ptr(kk), ptr(out)))
    return out


def truncate_supercell(ndim: int, bravais: np.ndarray, ncell: int, radius: float) -> np.ndarray:
    b = np.ascontiguousarray(bravais, dtype=np.float64)
    cnt = ctypes.c_int(0)
    check(lib().xatu_truncate_supercell(ndim, ptr(b), ncell, radius, ctypes.byref(cnt), None))
    out = np.zeros((cnt.value, 3))
    check(lib().xatu_truncate_supercell(ndim, ptr(b), ncell, radius, ctypes.byref(cnt), ptr(out)))
    return out
