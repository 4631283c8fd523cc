"""ctypes binding of ``libqsim_b200.so`` (the C ABI declared in include/qsim_b200.h).

There is no CPU fallback: if the library is missing, importing anything that needs it
raises ``ImportError`` naming the build command.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_double, c_int, c_ulonglong, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libqsim_b200.so")

QS_C64 = 0
QS_C128 = 1
MODES = {"cooperative": 0, "graphed": 1, "sequential": 2}
QS_OP_1Q = 1
QS_OP_2Q = 2
QS_ERR_INVALID = -1
QS_ERR_CUDA = -2
QS_ERR_DEVICE = -3

# gate ids of qs_prepare_ops / qs_gate_matrix (include/qsim_b200.h)
GATE_IDS = {"id": 1, "h": 2, "x": 3, "y": 4, "z": 5, "s": 6, "sdg": 7, "t": 8, "tdg": 9, "sx": 10, "rx": 11,
            "ry": 12, "rz": 13, "p": 14, "u": 15, "cx": 32, "cy": 33, "cz": 34, "cp": 35, "crz": 36, "swap": 37,
            "rzz": 38}
QS_GATE_MATRIX = 0

# qs_op {int kind, q0, q1, u_on_device; const void* U}
OP_DTYPE = np.dtype({"names": ["kind", "q0", "q1", "dev", "U"],
                     "formats": ["<i4", "<i4", "<i4", "<i4", "<u8"],
                     "offsets": [0, 4, 8, 12, 16], "itemsize": 24})


class QsConfig(ctypes.Structure):
    _fields_ = [("m", c_int), ("k", c_int), ("hill_iters", c_int), ("grid_mult", c_int), ("jit", c_int),
                ("jit_lr", c_int), ("jit_blocks", c_int), ("jit_packed", c_int), ("wait_limit_ns", c_ulonglong),
                ("jit_async", c_int), ("pad", c_int)]


class QsStats(ctypes.Structure):
    _fields_ = [(name, c_ulonglong) for name in
                ("gates", "sweeps", "perm_sweeps", "gate_sweeps", "launches", "graph_replays",
                 "graph_builds", "flushes", "permutes", "plans", "jit_compile_ms", "jit_modules",
                 "jit_disk_hits", "jit_pending_flushes")]

    def as_dict(self) -> dict:
        return {name: int(getattr(self, name)) for name, _ in self._fields_}


# name -> (argtypes); every function returns int status
_SIGS = {
    "qs_version": [],
    "qs_debug_fail_alloc": [c_int],
    "qs_jit_wait": [],
    "qs_device_count": [POINTER(c_int)],
    "qs_create": [c_int, c_int, POINTER(c_void_p)],
    "qs_destroy": [c_void_p],
    "qs_num_qubits": [c_void_p, POINTER(c_int)],
    "qs_dim": [c_void_p, POINTER(c_ulonglong)],
    "qs_dtype": [c_void_p, POINTER(c_int)],
    "qs_reset": [c_void_p],
    "qs_synchronize": [c_void_p],
    "qs_copy_to_host": [c_void_p, c_void_p, c_ulonglong],
    "qs_copy_from_host": [c_void_p, c_void_p, c_ulonglong],
    "qs_permute": [c_void_p, c_void_p, c_void_p, c_int],
    "qs_apply_tile": [c_void_p, c_void_p, c_int, c_int],
    "qs_apply_1q": [c_void_p, c_int, c_void_p, c_int],
    "qs_apply_2q": [c_void_p, c_int, c_int, c_void_p, c_int],
    "qs_apply_diagonal_1q": [c_void_p, c_int, c_void_p, c_void_p],
    "qs_flush": [c_void_p],
    "qs_materialize": [c_void_p],
    "qs_device_ptr": [c_void_p, POINTER(c_void_p)],
    "qs_set_stream": [c_void_p, c_void_p],
    "qs_get_stream": [c_void_p, POINTER(c_void_p)],
    "qs_set_config": [c_void_p, POINTER(QsConfig)],
    "qs_get_config": [c_void_p, POINTER(QsConfig)],
    "qs_get_stats": [c_void_p, POINTER(QsStats)],
    "qs_reset_stats": [c_void_p],
    "qs_get_pos2bit": [c_void_p, c_void_p, c_int],
    "qs_norm_squared": [c_void_p, POINTER(c_double)],
    "qs_inner_product": [c_void_p, c_void_p, POINTER(c_double), POINTER(c_double)],
    "qs_expect_zz_x": [c_void_p, c_void_p, c_void_p, c_void_p, POINTER(c_double)],
    "qs_adjoint_sweep": [c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_int],
    "qs_grad_create": [c_int, c_void_p, c_int, c_int, c_void_p, POINTER(c_void_p)],
    "qs_grad_run": [c_void_p, c_void_p, c_int, c_void_p, c_void_p, c_void_p, c_void_p],
    "qs_grad_info": [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p],
    "qs_grad_stats": [c_void_p, c_void_p],
    "qs_grad_destroy": [c_void_p],
    "qs_grad_emulate": [c_int, c_void_p, c_int, c_int, c_void_p, c_void_p, c_void_p, c_void_p],
    "qs_grad_jit_check": [c_int, c_void_p, c_int, c_int, c_void_p, c_void_p, c_void_p, c_int],
    "qs_apply_1q_gate": [c_void_p, c_int, c_void_p, c_int, c_int, c_void_p],
    "qs_apply_2q_gate": [c_void_p, c_int, c_void_p, c_int, c_int, c_int, c_void_p],
    "qs_permute_scatter": [c_void_p, c_void_p, c_int, c_int, c_void_p, c_void_p],
    "qs_plan_info": [c_int, c_int, c_void_p, c_int, POINTER(QsConfig), POINTER(c_int), POINTER(c_int)],
    "qs_lqr_flat_tiling": [c_int, c_int, c_void_p, c_int, c_void_p, c_void_p, c_void_p, c_void_p],
    "qs_fuse_ops": [c_int, c_void_p, c_int, c_void_p, c_void_p, c_void_p],
    "qs_gate_matrix": [c_int, c_void_p, c_void_p, POINTER(c_int)],
    "qs_prepare_ops": [c_int, c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_void_p,
                       c_void_p],
    "qs_plan_emulate": [c_int, c_int, c_void_p, c_int, POINTER(QsConfig), c_void_p],
    "qs_perm_emulate": [c_int, c_int, c_void_p, POINTER(QsConfig), c_void_p, POINTER(c_int)],
    "qs_jit_check": [c_int, c_void_p, c_int, POINTER(QsConfig), POINTER(c_int), c_void_p, c_int],
    "qs_apply_ops_noalloc": [c_void_p, c_int, c_int, c_void_p, c_int, c_void_p],
    "qs_apply_dense6": [c_void_p, c_void_p],
    "qs_apply_dense": [c_void_p, c_int, c_void_p, c_void_p],
    "qs_dense6_weights": [c_void_p, c_void_p],
    "qs_sample": [c_void_p, c_ulonglong, c_ulonglong, c_void_p],
    "qs_batch_create": [c_void_p, c_int, c_void_p, POINTER(c_void_p)],
    "qs_batch_set_params": [c_void_p, c_void_p, c_int],
    "qs_batch_run": [c_void_p, c_void_p, c_void_p],
    "qs_batch_results": [c_void_p, c_void_p, c_void_p],
    "qs_batch_info": [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p],
    "qs_batch_destroy": [c_void_p],
    "qs_batch_emulate": [c_void_p, c_int, c_void_p, c_void_p, c_void_p],
    "qs_batch_describe": [c_void_p, c_int, c_void_p, c_void_p],
}

_lib = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is not built; run: python -m frontierlabproject_b200.build")
        L = ctypes.CDLL(LIB_PATH)
        for name, args in _SIGS.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = c_int
        L.qs_last_error.argtypes = []
        L.qs_last_error.restype = ctypes.c_char_p
        _lib = L
    return _lib


def check(rc: int) -> None:
    if rc != 0:
        msg = lib().qs_last_error().decode("utf-8", "replace")
        raise RuntimeError(msg)


def call(name: str, *args) -> None:
    check(getattr(lib(), name)(*args))


def device_count() -> int:
    n = c_int(0)
    call("qs_device_count", ctypes.byref(n))
    return n.value


def exported_symbols() -> list:
    return sorted(list(_SIGS) + ["qs_last_error"])
