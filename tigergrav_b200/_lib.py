"""ctypes binding of libtigergrav_b200.so (the C ABI in include/tigergrav_b200.h).

The shared library is the product: every compute call goes to its sm_100a
kernels.  There is no CPU fallback -- if the library is missing this module
raises at import time, and if no GPU is present the calls return TG_ERR_CUDA.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libtigergrav_b200.so")

TG_OK, TG_ERR_ARG, TG_ERR_CUDA, TG_ERR_CAPACITY, TG_ERR_DEPTH, TG_ERR_TIMEOUT, TG_ERR_STATE, TG_ERR_NOMEM, \
    TG_ERR_SIZE = range(9)
TG_NOALLOC_MAX_N = 1 << 26
TG_PREC_F32, TG_PREC_F64 = 0, 1
TG_HOST, TG_DEVICE = 0, 1
LIST_KINDS = {"CC_D": 0, "CP_D": 1, "CC_E": 2, "CP_E": 3, "PC_D": 4, "PP_D": 5, "PC_E": 6, "PP_E": 7}


class tg_params(C.Structure):
    _fields_ = [("theta", C.c_double), ("soft_len", C.c_double), ("m", C.c_double), ("G", C.c_double),
                ("ewald", C.c_int32), ("leaf_max", C.c_int32), ("precision", C.c_int32), ("device", C.c_int32)]


class tg_cosmo_params(C.Structure):
    _fields_ = [("H0", C.c_double), ("omega_m", C.c_double), ("omega_lambda", C.c_double)]


class tg_rung_params(C.Structure):
    _fields_ = [("t_max", C.c_double), ("dt_max", C.c_double), ("eta", C.c_double)]


class tg_rung_state(C.Structure):
    _fields_ = [("itime", C.c_uint32), ("max_rung", C.c_int32), ("min_rung", C.c_int32), ("reserved", C.c_int32),
                ("num_active", C.c_int64), ("t", C.c_double)]


class tg_cosmo_rung_state(C.Structure):
    _fields_ = [("a", C.c_double), ("adot", C.c_double), ("tau", C.c_double), ("a_last", C.c_double),
                ("time", C.c_float), ("reserved", C.c_int32), ("kick1", C.c_double * 31)]


class tg_stats(C.Structure):
    _fields_ = [("n", C.c_int64), ("nodes", C.c_int64), ("leaves", C.c_int64), ("depth", C.c_int32),
                ("walk_retries", C.c_int32), ("ref_stats", C.c_uint64 * 6), ("counts", C.c_uint64 * 8),
                ("flops", C.c_double), ("ms_build", C.c_double), ("ms_multipoles", C.c_double),
                ("ms_walk", C.c_double), ("ms_nodes", C.c_double), ("ms_leaves", C.c_double),
                ("ms_kick_drift", C.c_double), ("launches", C.c_int64), ("ms_pp", C.c_double),
                ("device_bytes", C.c_int64)]


# every symbol the header declares (checked by the CPU test suite)
EXPORTS = [
    "tg_error_string", "tg_version", "tg_create", "tg_destroy", "tg_set_particles", "tg_get_particles",
    "tg_build", "tg_multipoles", "tg_walk", "tg_set_walk_capacity", "tg_forces", "tg_solve_gravity", "tg_get_forces",
    "tg_get_forces_f64", "tg_kick", "tg_drift", "tg_kick_drift", "tg_energy", "tg_leapfrog", "tg_get_stats", "tg_memory_report",
    "tg_num_nodes",
    "tg_get_nodes", "tg_get_perm", "tg_list_size", "tg_get_list", "tg_gravity_PP_direct",
    "tg_gravity_PP_ewald", "tg_gravity_PC_direct", "tg_gravity_PC_ewald", "tg_gravity_CC_direct",
    "tg_gravity_CC_ewald", "tg_gravity_CP_direct", "tg_gravity_CP_ewald", "tg_truth", "tg_device_fp32_peak",
    "tg_energy_noalloc", "tg_forward", "tg_backward", "tg_tidal", "tg_batch_create", "tg_batch_destroy",
    "tg_batch_size", "tg_batch_set_particles", "tg_batch_autotune", "tg_batch_solve", "tg_batch_leapfrog",
    "tg_batch_get_forces", "tg_cosmo_kdk", "tg_leapfrog_cosmo", "tg_load_gadget1",
    "tg_find_groups", "tg_set_fof_retry_limit", "tg_group_catalog", "tg_rung_step", "tg_rung_step_cosmo", "tg_cosmo_rung_init", "tg_get_rungs",
]


class TGError(RuntimeError):
    def __init__(self, fn: str, status: int, msg: str):
        super().__init__(f"{fn} failed: {msg} (status {status})")
        self.status = status


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            "tigergrav_b200: CUDA library %s is missing; build it with `make -C tigergrav_b200/csrc` "
            "or __graft_entry__.build()" % LIB_PATH)
    L = C.CDLL(LIB_PATH)
    vp, i64, i32, d = C.c_void_p, C.c_int64, C.c_int, C.c_double
    P = C.POINTER
    L.tg_error_string.restype = C.c_char_p
    L.tg_error_string.argtypes = [i32]
    L.tg_version.restype = C.c_char_p
    L.tg_create.argtypes = [P(tg_params), P(vp)]
    L.tg_destroy.argtypes = [vp]
    L.tg_set_particles.argtypes = [vp, vp, vp, i64, i32, vp]
    L.tg_get_particles.argtypes = [vp, vp, vp, i32, vp]
    for f in ("tg_build", "tg_multipoles", "tg_walk", "tg_forces", "tg_solve_gravity"):
        getattr(L, f).argtypes = [vp, vp]
    L.tg_set_walk_capacity.argtypes = [vp, i64]
    L.tg_get_forces.argtypes = [vp, vp, vp, i32, vp]
    L.tg_get_forces_f64.argtypes = [vp, vp, vp, i32, vp]
    L.tg_kick.argtypes = [vp, d, vp]
    L.tg_drift.argtypes = [vp, d, vp]
    L.tg_kick_drift.argtypes = [vp, d, d, d, vp]
    L.tg_energy.argtypes = [vp, vp, vp]
    L.tg_leapfrog.argtypes = [vp, d, i32, vp]
    L.tg_get_stats.argtypes = [vp, P(tg_stats)]
    L.tg_memory_report.argtypes = [vp, vp, i64]
    L.tg_num_nodes.restype = i64
    L.tg_num_nodes.argtypes = [vp]
    L.tg_get_nodes.argtypes = [vp] + [vp] * 10
    L.tg_get_perm.argtypes = [vp, vp]
    L.tg_list_size.restype = i64
    L.tg_list_size.argtypes = [vp, i32]
    L.tg_get_list.argtypes = [vp, i32, vp, vp]
    L.tg_gravity_PP_direct.argtypes = [P(tg_params), i64, vp, vp, vp, vp, vp, i32, vp, vp]
    L.tg_gravity_PP_ewald.argtypes = [P(tg_params), i64, vp, vp, vp, vp, vp, vp, vp]
    L.tg_gravity_PC_direct.argtypes = [P(tg_params), i64, vp, vp, vp, vp, vp, vp, vp, vp]
    L.tg_gravity_PC_ewald.argtypes = [P(tg_params), i64, vp, vp, vp, vp, vp, vp, vp, vp]
    L.tg_gravity_CC_direct.argtypes = [P(tg_params), i64, vp, vp, vp, vp, vp, vp, vp]
    L.tg_gravity_CC_ewald.argtypes = [P(tg_params), i64, vp, vp, vp, vp, vp, vp, vp]
    L.tg_gravity_CP_direct.argtypes = [P(tg_params), i64, vp, vp, vp, vp, vp, vp]
    L.tg_gravity_CP_ewald.argtypes = [P(tg_params), i64, vp, vp, vp, vp, vp, vp]
    L.tg_truth.argtypes = [vp, vp, i64, d, vp, vp, vp]
    L.tg_device_fp32_peak.argtypes = [i32, P(d), vp]
    L.tg_energy_noalloc.argtypes = [vp, vp, i64, d, d, vp, i32, vp]
    L.tg_forward.argtypes = [vp, d, i32, vp]
    L.tg_backward.argtypes = [vp, vp, vp, vp, vp, i32, vp]
    L.tg_tidal.argtypes = [vp, vp, vp, i32, vp]
    L.tg_batch_create.argtypes = [P(tg_params), i32, vp, i32, P(vp)]
    L.tg_batch_destroy.argtypes = [vp]
    L.tg_batch_size.restype = i64
    L.tg_batch_size.argtypes = [vp]
    L.tg_batch_set_particles.argtypes = [vp, vp, vp, i32]
    L.tg_batch_autotune.argtypes = [vp, vp, i32, vp]
    L.tg_batch_solve.argtypes = [vp]
    L.tg_batch_leapfrog.argtypes = [vp, d, i32]
    L.tg_batch_get_forces.argtypes = [vp, vp, vp, i32]
    L.tg_cosmo_kdk.argtypes = [P(tg_cosmo_params), vp, d, vp]
    L.tg_leapfrog_cosmo.argtypes = [vp, P(tg_cosmo_params), vp, d, i32, vp]
    L.tg_load_gadget1.argtypes = [C.c_char_p, vp, vp, vp, i64, P(i64)]
    L.tg_find_groups.argtypes = [vp, d, vp, P(i64), i32, vp]
    L.tg_set_fof_retry_limit.argtypes = [vp, i32]
    L.tg_group_catalog.argtypes = [vp, d, vp, i64, P(i64), vp]
    L.tg_rung_step.argtypes = [vp, P(tg_rung_params), P(tg_rung_state), i32, vp]
    L.tg_get_rungs.argtypes = [vp, vp, i32, vp]
    L.tg_rung_step_cosmo.argtypes = [vp, P(tg_rung_params), P(tg_rung_state), P(tg_cosmo_params),
                                     P(tg_cosmo_rung_state), i32, vp]
    L.tg_cosmo_rung_init.argtypes = [P(tg_cosmo_rung_state), d, d]
    return L


lib = _load()


def check(fn: str, status: int) -> None:
    if status != TG_OK:
        raise TGError(fn, status, lib.tg_error_string(status).decode())
