"""ctypes binding of libfcfd_b200.so (the C ABI declared in include/fcfd.h).

The shared library is built in-tree by ``freecfd_b200/Makefile`` (nvcc,
sm_100a).  There is no Python or CPU fallback: if the library is missing,
importing this module raises.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_build", "libfcfd_b200.so")

FCFD_OK = 0
FCFD_DEVICE_PTRS = 1
FCFD_NO_SYNC = 8
STATUS = {0: "OK", 1: "ERR_INPUT", 2: "ERR_MESH", 3: "ERR_DIVERGED", 4: "ERR_NOT_CONVERGED", 5: "ERR_CUDA",
          6: "ERR_TIMEOUT", 7: "ERR_UNSUPPORTED", 8: "ERR_BC"}

EXPORTED = [
    "fcfd_last_error", "fcfd_version", "fcfd_case_from_deck", "fcfd_case_destroy", "fcfd_case_summary",
    "fcfd_mesh_create", "fcfd_mesh_destroy", "fcfd_mesh_sizes", "fcfd_mesh_connectivity", "fcfd_mesh_geometry",
    "fcfd_mesh_lsq", "fcfd_mesh_rcm", "fcfd_mesh_grad_weights",
    "fcfd_ctx_create", "fcfd_ctx_destroy", "fcfd_ctx_set_exact_gradients", "fcfd_residual", "fcfd_last_stages", "fcfd_local_dt",
    "fcfd_time_residual", "fcfd_point_flux", "fcfd_jvp", "fcfd_vjp", "fcfd_drag", "fcfd_rans_residual", "fcfd_rans_bcs", "fcfd_time_rans", "fcfd_newton_solve", "fcfd_local_dt_cflmax_noalloc",
    "fcfd_run", "fcfd_restart_write", "fcfd_restart_read", "fcfd_mesh_from_tecplot", "fcfd_rans_jvp", "fcfd_rans_vjp", "fcfd_ctx_set_launch_overlap",
    "fcfd_partition_sets", "fcfd_ctx_set_partition", "fcfd_partition_extrema", "fcfd_partition_residual", "fcfd_ctx_check",
    "fcfd_ctx_stream", "fcfd_diag_blocks", "fcfd_rans_newton_solve", "fcfd_residual_mixed",
    "fcfd_time_residual_mixed", "fcfd_ctx_set_gradient_kernel", "fcfd_time_terms", "fcfd_ctx_gradient_info",
]


class FcfdError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


def build(force: bool = False) -> str:
    """Compile the CUDA library in-tree (nvcc, -gencode arch=compute_100a,code=sm_100a)."""
    cmd = ["make", "-C", _HERE, "-s"]
    if force:
        subprocess.run(["make", "-C", _HERE, "-s", "clean"], check=True)
    subprocess.run(cmd, check=True)
    return LIB_PATH


class _RawMesh(ctypes.Structure):
    _fields_ = [("n_nodes", ctypes.c_int32), ("xyz", ctypes.POINTER(ctypes.c_double)),
                ("n_cells", ctypes.c_int32), ("conn_index", ctypes.POINTER(ctypes.c_int32)),
                ("conn", ctypes.POINTER(ctypes.c_int32)), ("n_bc", ctypes.c_int32),
                ("bc_index", ctypes.POINTER(ctypes.c_int32)), ("bc_nodes", ctypes.POINTER(ctypes.c_int32))]


class RunOpts(ctypes.Structure):
    _fields_ = [("work_dir", ctypes.c_char_p), ("restart_step", ctypes.c_int32), ("max_steps", ctypes.c_int32),
                ("jvp_mode", ctypes.c_int32), ("fp32_krylov", ctypes.c_int32), ("precond_sweeps", ctypes.c_int32),
                ("echo", ctypes.c_int32), ("K", ctypes.POINTER(ctypes.c_double))]


class RunReport(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int32), ("steps", ctypes.c_int32), ("krylov_iterations", ctypes.c_int32),
                ("pad", ctypes.c_int32), ("time", ctypes.c_double), ("res", ctypes.c_double),
                ("wall_seconds", ctypes.c_double)]


class NewtonOpts(ctypes.Structure):
    _fields_ = [("max_newton", ctypes.c_int32), ("tol", ctypes.c_double), ("krylov_dim", ctypes.c_int32),
                ("krylov_rtol", ctypes.c_double), ("cfl0", ctypes.c_double), ("cfl_growth", ctypes.c_double),
                ("cfl_max", ctypes.c_double), ("cfl_mode", ctypes.c_int32), ("ser_exponent", ctypes.c_double),
                ("jvp_mode", ctypes.c_int32), ("fp32_krylov", ctypes.c_int32), ("max_seconds", ctypes.c_double),
                ("precond_sweeps", ctypes.c_int32), ("krylov_cycles", ctypes.c_int32),
                ("stop_all_rows", ctypes.c_int32), ("gs_launch", ctypes.c_int32), ("precond_ilu0", ctypes.c_int32),
                ("local_relax", ctypes.c_int32), ("startup_steps", ctypes.c_int32), ("startup_drop", ctypes.c_double)]


class NewtonReport(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int32), ("newton_iterations", ctypes.c_int32),
                ("krylov_iterations", ctypes.c_int32), ("pad", ctypes.c_int32), ("res0", ctypes.c_double),
                ("res_final", ctypes.c_double), ("wall_seconds", ctypes.c_double), ("last_cfl", ctypes.c_double),
                ("history", ctypes.c_double * 512), ("rows_final", ctypes.c_double * 3),
                ("seconds_to_tol", ctypes.c_double), ("seconds_history", ctypes.c_double * 512),
                ("kw_final", ctypes.c_double * 2), ("startup_steps", ctypes.c_int32), ("pad2", ctypes.c_int32)]


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"libfcfd_b200.so not found at {LIB_PATH}; build it with `make -C {_HERE}`")
    L = ctypes.CDLL(LIB_PATH)
    vp, dp, ip, i64p = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int32), \
        ctypes.POINTER(ctypes.c_int64)
    L.fcfd_last_error.restype = ctypes.c_char_p
    L.fcfd_version.restype = ctypes.c_char_p
    L.fcfd_case_from_deck.argtypes = [ctypes.c_char_p, ctypes.POINTER(vp)]
    L.fcfd_case_destroy.argtypes = [vp]
    L.fcfd_case_destroy.restype = None
    L.fcfd_case_summary.argtypes = [vp, dp, ip, ctypes.c_int32]
    L.fcfd_mesh_create.argtypes = [ctypes.POINTER(_RawMesh), vp, ctypes.POINTER(vp)]
    L.fcfd_mesh_destroy.argtypes = [vp]
    L.fcfd_mesh_destroy.restype = None
    L.fcfd_mesh_sizes.argtypes = [vp, i64p]
    L.fcfd_mesh_connectivity.argtypes = [vp] + [ip] * 10
    L.fcfd_mesh_geometry.argtypes = [vp] + [dp] * 9
    L.fcfd_mesh_lsq.argtypes = [vp, dp, dp]
    L.fcfd_mesh_rcm.argtypes = [vp, ip]
    L.fcfd_mesh_grad_weights.argtypes = [vp, dp]
    L.fcfd_residual_mixed.argtypes = [vp, vp, vp, ctypes.c_double, ctypes.c_int32, i64p]
    L.fcfd_time_residual_mixed.argtypes = [vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_double, dp]
    L.fcfd_ctx_create.argtypes = [vp, vp, ctypes.c_int, ctypes.POINTER(vp)]
    L.fcfd_ctx_destroy.argtypes = [vp]
    L.fcfd_ctx_destroy.restype = None
    L.fcfd_ctx_set_exact_gradients.argtypes = [vp, ctypes.c_int]
    L.fcfd_ctx_set_gradient_kernel.argtypes = [vp, ctypes.c_int]
    L.fcfd_time_terms.argtypes = [vp, dp, dp, dp]
    L.fcfd_ctx_gradient_info.argtypes = [vp, i64p]
    L.fcfd_residual.argtypes = [vp, vp, vp, ctypes.c_int]
    L.fcfd_last_stages.argtypes = [vp, dp, dp, dp, dp, dp]
    L.fcfd_local_dt.argtypes = [vp, vp, ctypes.c_double, ctypes.c_int, vp, ctypes.c_int]
    L.fcfd_jvp.argtypes = [vp, vp, vp, vp, vp, ctypes.c_int]
    L.fcfd_vjp.argtypes = [vp, vp, vp, vp, ctypes.c_int]
    L.fcfd_rans_residual.argtypes = [vp, vp, vp, vp, vp, ctypes.c_int]
    L.fcfd_rans_jvp.argtypes = [vp, dp, dp, dp, dp, dp, dp, dp, dp, ctypes.c_int]
    L.fcfd_rans_vjp.argtypes = [vp, dp, dp, dp, dp, dp, dp, ctypes.c_int]
    L.fcfd_ctx_set_launch_overlap.argtypes = [vp, ctypes.c_int32]
    L.fcfd_rans_bcs.argtypes = [vp, vp, ctypes.c_int32]
    L.fcfd_time_rans.argtypes = [vp, ctypes.c_int, ctypes.c_int, vp, ctypes.c_int]
    L.fcfd_drag.argtypes = [vp, vp, ctypes.c_uint32, vp, vp, vp, ctypes.c_int]
    L.fcfd_newton_solve.argtypes = [vp, dp, ctypes.POINTER(NewtonOpts), ctypes.POINTER(NewtonReport)]
    L.fcfd_local_dt_cflmax_noalloc.argtypes = [vp, vp, ctypes.c_int32, ctypes.c_double, ctypes.c_double,
                                                ctypes.c_double, ctypes.c_double, ctypes.c_double, vp, vp]
    L.fcfd_time_residual.argtypes = [vp, ctypes.c_int, ctypes.c_int, dp, ctypes.c_int]
    L.fcfd_run.argtypes = [vp, dp, ctypes.POINTER(RunOpts), ctypes.POINTER(RunReport)]
    L.fcfd_mesh_from_tecplot.argtypes = [ctypes.c_char_p, vp, ctypes.POINTER(ctypes.c_void_p), ctypes.c_char_p,
                                         ctypes.c_int32]
    L.fcfd_restart_write.argtypes = [ctypes.c_char_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_double, dp, dp,
                                     ctypes.c_int32, ctypes.c_int32, dp, dp, dp, dp]
    L.fcfd_restart_read.argtypes = [ctypes.c_char_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, dp, dp, dp,
                                    dp, dp, dp]
    L.fcfd_point_flux.argtypes = [ctypes.c_int, dp, dp, dp, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                  ctypes.c_double, ctypes.c_double, dp, dp]
    L.fcfd_partition_sets.argtypes = [vp, vp, ctypes.c_int, ctypes.c_int, ip, ip, ip, ip]
    L.fcfd_ctx_set_partition.argtypes = [vp, ctypes.c_int, ctypes.c_int]
    L.fcfd_partition_extrema.argtypes = [vp, vp, vp, ctypes.c_int]
    L.fcfd_partition_residual.argtypes = [vp, vp, vp, ctypes.c_int]
    L.fcfd_ctx_check.argtypes = [vp]
    L.fcfd_ctx_stream.argtypes = [vp, ctypes.POINTER(vp)]
    L.fcfd_diag_blocks.argtypes = [vp, dp, dp, dp]
    L.fcfd_rans_newton_solve.argtypes = [vp, dp, dp, ctypes.POINTER(NewtonOpts), ctypes.POINTER(NewtonReport)]
    for name in EXPORTED:
        getattr(L, name)
    return L


lib = _load()


def check(rc: int):
    if rc != FCFD_OK:
        raise FcfdError(rc, lib.fcfd_last_error().decode())


def _d(a):
    return None if a is None else a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _i(a):
    return None if a is None else a.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))


def _ptr(a):
    """Host numpy array or CUDA torch tensor -> (void*, flags)."""
    if isinstance(a, np.ndarray):
        return ctypes.c_void_p(a.ctypes.data), 0
    return ctypes.c_void_p(a.data_ptr()), FCFD_DEVICE_PTRS
