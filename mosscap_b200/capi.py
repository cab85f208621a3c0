"""ctypes binding of the C ABI in ``include/mosscap_b200.h``.

The shared library is ``mosscap_b200/libmosscap_b200.so`` (built by
``mosscap_b200.build``). Loading fails loudly when it is missing: there is no
fallback implementation.
"""
from __future__ import annotations

import ctypes
import os
import re
from typing import List

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libmosscap_b200.so")
HEADER = os.path.join(os.path.dirname(PKG), "include", "mosscap_b200.h")

MC_OK = 0
STATUS_NAMES = {0: "MC_OK", 1: "MC_ERR_INVALID_ARGUMENT", 2: "MC_ERR_UNSUPPORTED", 3: "MC_ERR_CUDA",
                4: "MC_ERR_OUT_OF_MEMORY", 5: "MC_ERR_STATE"}
FLAG_NONFINITE, FLAG_NEG_DENSITY, FLAG_NEG_PRESSURE, FLAG_BAD_DT = 0x1, 0x2, 0x4, 0x8
FLAG_EOS = 0x10
EOS = {"ideal": 0, "analyticlteh": 1, "tabulatedlteh": 2}

RECON = {"fog": 0, "muscl": 1, "ppm": 2, "weno5z": 3}
LIMITER = {"vanleer": 0, "monotonizedcentral": 1, "minmod": 2}
RIEMANN = {"rusanov": 0, "hll": 1, "hllc": 2}
STEPPER = {"rk2": 0, "ssprk3": 1, "ssprk4": 2}
BOUNDARY = {"wall": 0, "periodic": 1, "symmetric": 2, "symmetricoutflowdiode": 3,
            "zerograd": 4, "constant": 5, "userfn": 6}
PRECISION = {"fp64": 0, "fp32": 1}


class McGrid(ctypes.Structure):
    _fields_ = [
        ("num_dim", ctypes.c_int32),
        ("xc", ctypes.c_int32), ("yc", ctypes.c_int32), ("zc", ctypes.c_int32),
        ("ng", ctypes.c_int32),
        ("num_tracers", ctypes.c_int32),
        ("dx", ctypes.c_double),
        ("loc", ctypes.c_double * 3),
        ("bc", ctypes.c_int32 * 6),
        ("bc_const", (ctypes.c_double * 5) * 6),
    ]


class McScheme(ctypes.Structure):
    _fields_ = [
        ("reconstruction", ctypes.c_int32),
        ("slope_limiter", ctypes.c_int32),
        ("riemann_solver", ctypes.c_int32),
        ("time_stepper", ctypes.c_int32),
        ("precision", ctypes.c_int32),
        ("gamma", ctypes.c_double),
        ("max_cfl", ctypes.c_double),
    ]


class McClock(ctypes.Structure):
    _fields_ = [
        ("time", ctypes.c_double),
        ("max_time", ctypes.c_double),
        ("prev_output_time", ctypes.c_double),
        ("output_delta", ctypes.c_double),
    ]


class McBatchProblem(ctypes.Structure):
    _fields_ = [
        ("grid", McGrid),
        ("offset", ctypes.c_int64),
        ("max_cfl", ctypes.c_double),
        ("clock", McClock),
    ]


USER_BC_FN = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p)
# void (*)(void* user, uint64_t* cfl_min_bits, void* stream)
CFL_REDUCE_FN = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p)
# int32_t (*)(void* user, int32_t op, void* const* bufs, int64_t count, void* stream)
COMM_FN = ctypes.CFUNCTYPE(ctypes.c_int32, ctypes.c_void_p, ctypes.c_int32, ctypes.POINTER(ctypes.c_void_p),
                           ctypes.c_int64, ctypes.c_void_p)
COMM_HALO, COMM_MIN_U64, COMM_SUM_F64, COMM_MIN_I64 = 0, 1, 2, 3


class McEosTable(ctypes.Structure):
    _fields_ = [
        ("log_eint_rho_start", ctypes.c_double), ("log_eint_rho_step", ctypes.c_double),
        ("n_eint_rho", ctypes.c_int32),
        ("log_rho_start", ctypes.c_double), ("log_rho_step", ctypes.c_double),
        ("n_rho", ctypes.c_int32),
        ("y_table", ctypes.POINTER(ctypes.c_double)),
        ("log_T_table", ctypes.POINTER(ctypes.c_double)),
    ]


class McError(RuntimeError):
    def __init__(self, status: int, where: str, msg: str):
        super().__init__(f"{where}: {STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


_LIB = None


def load() -> ctypes.CDLL:
    """Load the C-ABI library (raises if it was not built)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise FileNotFoundError(f"{LIB_PATH} is missing; build it with python -m mosscap_b200.build")
    lib = ctypes.CDLL(LIB_PATH)
    vp, i32, i64, d = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_double
    P = ctypes.POINTER
    lib.mc_abi_version.restype = i32
    lib.mc_last_error.restype = ctypes.c_char_p
    lib.mc_create.argtypes = [P(McGrid), P(McScheme), P(vp)]
    lib.mc_create.restype = i32
    lib.mc_destroy.argtypes = [vp]
    lib.mc_destroy.restype = i32
    lib.mc_set_user_bc.argtypes = [vp, USER_BC_FN, vp]
    lib.mc_set_user_bc.restype = i32
    lib.mc_fill_bcs.argtypes = [vp, vp, vp]
    lib.mc_fill_bcs.restype = i32
    lib.mc_compute_dt.argtypes = [vp, vp, P(McClock), P(d), vp]
    lib.mc_compute_dt.restype = i32
    lib.mc_time_step.argtypes = [vp, vp, d, vp]
    lib.mc_time_step.restype = i32
    lib.mc_step_host.argtypes = [vp, vp, vp, P(McClock), P(d), vp]
    lib.mc_step_host.restype = i32
    lib.mc_advance.argtypes = [vp, vp, P(McClock), i64, P(i64), P(d), vp]
    lib.mc_advance.restype = i32
    lib.mc_last_cfl_min.argtypes = [vp, P(d), vp]
    lib.mc_last_cfl_min.restype = i32
    lib.mc_slab_unique_id.argtypes = [ctypes.c_char_p]
    lib.mc_slab_unique_id.restype = i32
    lib.mc_set_slab_decomposition.argtypes = [vp, ctypes.c_char_p, i32, i32]
    lib.mc_set_slab_decomposition.restype = i32
    lib.mc_set_slab_overlap.argtypes = [vp, i32]
    lib.mc_set_slab_overlap.restype = i32
    lib.mc_tangent_linear.argtypes = [P(McGrid), P(McScheme), vp, vp, P(d), i32, P(McClock), i64, vp]
    lib.mc_tangent_linear.restype = i32
    lib.mc_get_status.argtypes = [vp, P(ctypes.c_uint32), vp]
    lib.mc_get_status.restype = i32
    lib.mc_profile_stages.argtypes = [vp, i32]
    lib.mc_profile_stages.restype = i32
    lib.mc_stage_time.argtypes = [vp, i32, P(d), P(i64)]
    lib.mc_stage_time.restype = i32
    lib.mc_batch_create.argtypes = [P(McBatchProblem), i32, P(McScheme), i64, P(vp)]
    lib.mc_batch_create.restype = i32
    lib.mc_batch_destroy.argtypes = [vp]
    lib.mc_batch_destroy.restype = i32
    lib.mc_batch_fill_bcs.argtypes = [vp, vp, vp]
    lib.mc_batch_fill_bcs.restype = i32
    lib.mc_batch_tune.argtypes = [vp, vp, vp]
    lib.mc_batch_tune.restype = i32
    lib.mc_batch_advance.argtypes = [vp, vp, i64, vp]
    lib.mc_batch_advance.restype = i32
    lib.mc_batch_clocks.argtypes = [vp, P(McClock), P(i64), P(ctypes.c_uint32), vp]
    lib.mc_batch_clocks.restype = i32
    lib.mc_batch_schedule.argtypes = [vp, P(i32), P(i32), P(i32)]
    lib.mc_batch_schedule.restype = i32
    lib.mc_batch_set_stage_launches.argtypes = [vp, i32]
    lib.mc_batch_set_stage_launches.restype = i32
    lib.mc_batch_stage_launches.argtypes = [vp, P(i32)]
    lib.mc_batch_stage_launches.restype = i32
    lib.mc_time_step_noalloc.argtypes = [P(McGrid), P(McScheme), vp, d, vp]
    lib.mc_time_step_noalloc.restype = i32
    lib.mc_set_cfl_reduce_hook.argtypes = [vp, CFL_REDUCE_FN, vp]
    lib.mc_set_cfl_reduce_hook.restype = i32
    lib.mc_set_gravity.argtypes = [vp, i32, d, d, d]
    lib.mc_set_gravity.restype = i32
    lib.mc_set_eos.argtypes = [vp, i32, d, i32, P(McEosTable)]
    lib.mc_set_eos.restype = i32
    lib.mc_update_eos.argtypes = [vp, vp, vp]
    lib.mc_update_eos.restype = i32
    lib.mc_get_eos_fields.argtypes = [vp, vp, vp, vp]
    lib.mc_get_eos_fields.restype = i32
    lib.mc_get_prim.argtypes = [vp, vp, vp, vp]
    lib.mc_get_prim.restype = i32
    lib.mc_launch_count.argtypes = [vp]
    lib.mc_launch_count.restype = i64
    lib.mc_adjoint_create.argtypes = [P(McGrid), P(McScheme), i32, P(vp)]
    lib.mc_adjoint_create.restype = i32
    lib.mc_adjoint_destroy.argtypes = [vp]
    lib.mc_adjoint_destroy.restype = i32
    lib.mc_adjoint_forward.argtypes = [vp, vp, P(McClock), i64, vp]
    lib.mc_adjoint_forward.restype = i32
    lib.mc_adjoint_backward.argtypes = [vp, vp, P(d), vp]
    lib.mc_adjoint_backward.restype = i32
    lib.mc_adjoint_set_slab_decomposition.argtypes = [vp, ctypes.c_char_p, i32, i32]
    lib.mc_adjoint_set_slab_decomposition.restype = i32
    lib.mc_adjoint_set_slab_hook.argtypes = [vp, COMM_FN, vp, i32, i32]
    lib.mc_adjoint_set_slab_hook.restype = i32
    lib.mc_debug_reverse_reciprocal.argtypes = [vp, vp, i64, vp]
    lib.mc_debug_reverse_reciprocal.restype = i32
    if lib.mc_abi_version() != 1:
        raise RuntimeError("unexpected ABI version")
    _LIB = lib
    return lib


def check(status: int, where: str) -> None:
    if status != MC_OK:
        raise McError(status, where, load().mc_last_error().decode())


def declared_functions(header: str = HEADER) -> List[str]:
    """Names of the functions ``include/mosscap_b200.h`` declares."""
    text = open(header).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(mc_[a-z_0-9]+)\s*\(", text)))
