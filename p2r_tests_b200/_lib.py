"""ctypes binding of libp2r_b200.so (the C ABI declared in include/p2r.h).

The library is built in-tree by p2r_tests_b200/build.py. There is no fallback: if the
library is missing or does not load, every call raises.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / "libp2r_b200.so"
ABI_VERSION = 1  # P2R_ABI_VERSION of include/p2r.h, which these signatures follow

P2R_OK = 0
P2R_ERR_INVALID = 1
P2R_ERR_CUDA = 2
P2R_ERR_TIMEOUT = 3
P2R_ERR_UNSUPPORTED = 4
P2R_ERR_WORKSPACE = 5
P2R_ERR_QUEUE = 6

MODE_RESTART = 0
MODE_CHAINED = 1
FLAG_FP32_DET = 0x1
FLAG_NO_STAGING = 0x2
FLAG_ADJ_FP32 = 0x4
FLAG_SQUASH_PHI = 0x8
FLAG_ORDER_BY_LAYERS = 0x10
MATH_REFINED, MATH_IEEE, MATH_FAST = 0, 1, 2


class P2RError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"p2r error {code}: {msg}")
        self.code = code


class CConfig(ctypes.Structure):
    _fields_ = [
        ("bsize", ctypes.c_int32),
        ("nlayer", ctypes.c_int32),
        ("nevts", ctypes.c_int64),
        ("nb", ctypes.c_int64),
        ("bz", ctypes.c_double),
        ("mode", ctypes.c_int32),
        ("flags", ctypes.c_uint32),
        ("block_threads", ctypes.c_int32),
        ("stages", ctypes.c_int32),
    ]


class CGenParams(ctypes.Structure):
    _fields_ = [
        ("seed", ctypes.c_uint64),
        ("bz", ctypes.c_double),
        ("r_seed", ctypes.c_double),
        ("r_first", ctypes.c_double),
        ("r_last", ctypes.c_double),
        ("pt", ctypes.c_double),
        ("pop_smear", ctypes.c_double),
        ("theta_min", ctypes.c_double),
        ("theta_max", ctypes.c_double),
        ("cov_pos", ctypes.c_double),
        ("cov_ang", ctypes.c_double),
        ("est_smear", ctypes.c_double),
        ("hit_sigma", ctypes.c_double),
    ]


class CQueueItem(ctypes.Structure):
    _fields_ = [("event", ctypes.c_int32), ("nblk", ctypes.c_int32), ("block0", ctypes.c_int64)]


class CQueue(ctypes.Structure):
    _fields_ = [
        ("bsize", ctypes.c_int32), ("nlayer", ctypes.c_int32), ("nevts", ctypes.c_int64),
        ("nblocks", ctypes.c_int64), ("bz", ctypes.c_double), ("flags", ctypes.c_uint32),
        ("block_threads", ctypes.c_int32), ("stages", ctypes.c_int32), ("ctas_per_sm", ctypes.c_int32),
        ("event_block_offset", ctypes.c_void_p), ("items", ctypes.c_void_p), ("n_items", ctypes.c_int64),
        ("nlay_lane", ctypes.c_void_p),
    ]


class CTuneResult(ctypes.Structure):
    _fields_ = [("best_ms", ctypes.c_float), ("block_threads", ctypes.c_int32), ("stages", ctypes.c_int32),
                ("n_tried", ctypes.c_int32), ("tried_threads", ctypes.c_int32 * 64),
                ("tried_stages", ctypes.c_int32 * 64), ("tried_ms", ctypes.c_float * 64)]


class CSummary(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in (
        "avg_x", "avg_y", "avg_z", "avg_r", "avg_pt", "avg_phi", "avg_theta",
        "avg_dx", "avg_dy", "avg_dz", "avg_dr",
        "std_x", "std_y", "std_z", "std_r", "std_dx", "std_dy", "std_dz", "std_dr")] + [
        ("nnans", ctypes.c_int64), ("nfail", ctypes.c_int64)]


_vp = ctypes.c_void_p
_i32 = ctypes.c_int32
_i64 = ctypes.c_int64
_cfgp = ctypes.POINTER(CConfig)

# name -> (restype, argtypes); every function in include/p2r.h
SIGNATURES = {
    "p2r_abi_version": (ctypes.c_int, []),
    "p2r_last_error_string": (ctypes.c_char_p, []),
    "p2r_kfact": (ctypes.c_float, [ctypes.c_double]),
    "p2r_propagate_to_r": (ctypes.c_int, [_cfgp, _vp, _vp, _i32, _vp, _vp, _vp]),
    "p2r_kalman_update": (ctypes.c_int, [_cfgp, _vp, _vp, _i32, _vp, _vp]),
    "p2r_kalman_gain_inv": (ctypes.c_int, [_cfgp, _vp, _vp, _i32, _vp, _vp]),
    "p2r_kalman_gain": (ctypes.c_int, [_cfgp, _vp, _vp, _vp, _vp]),
    "p2r_forward": (ctypes.c_int, [_cfgp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "p2r_forward_masked": (ctypes.c_int, [_cfgp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "p2r_count_nonfinite": (ctypes.c_int, [_vp, _i64, _i32, _vp, _vp]),
    "p2r_forward_host": (ctypes.c_int, [_cfgp, _vp, _vp, _vp, _vp, _vp, _vp, _i32, _vp]),
    "p2r_fp32_fma_probe": (ctypes.c_int, [_i64, _i32, _i32, _vp, _vp]),
    "p2r_fp32x2_fma_probe": (ctypes.c_int, [_i64, _i32, _i32, _vp, _vp]),
    "p2r_fp64_fma_probe": (ctypes.c_int, [_i64, _i32, _i32, _vp, _vp]),
    "p2r_math_variant": (ctypes.c_int32, []),
    "p2r_math_check": (ctypes.c_int, [_i64, _vp, _vp, _vp, _vp, _vp]),
    "p2r_forward_backward_workspace_size": (ctypes.c_size_t, [_cfgp]),
    "p2r_forward_backward_workspace_size_tape": (ctypes.c_size_t, [_cfgp, _i32]),
    "p2r_forward_backward_noalloc": (ctypes.c_int, [_cfgp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                                                    _vp, _vp, _vp, _i32, _vp]),
    "p2r_queue_plan": (ctypes.c_int64, [_vp, _i64, _i32, _vp, _i64]),
    "p2r_autotune_forward": (ctypes.c_int, [_cfgp, _vp, _vp, _vp, _vp, _i32, _vp, _i32, _i32, _vp, _vp]),
    "p2r_queue_workspace_size": (ctypes.c_size_t, [_vp]),
    "p2r_queue_error": (ctypes.c_int, [_vp, _vp, _vp]),
    "p2r_queue_adjoint_workspace_size": (ctypes.c_size_t, [_vp]),
    "p2r_run_queue_adjoint": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                                             _vp, ctypes.c_size_t, _vp]),
    "p2r_queue_adjoint_graph_create": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                                                      _vp, _vp, ctypes.c_size_t, _vp]),
    "p2r_run_queue": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, ctypes.c_size_t, _vp]),
    "p2r_queue_graph_create": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, ctypes.c_size_t, _vp]),
    "p2r_graph_launch": (ctypes.c_int, [_vp, _vp]),
    "p2r_graph_destroy": (ctypes.c_int, [_vp]),
    "p2r_forward_backward": (ctypes.c_int, [_cfgp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                                            _vp, _vp, _i32, _vp, ctypes.c_size_t, _vp]),
    "p2r_gen_params_default": (None, [ctypes.POINTER(CGenParams)]),
    "p2r_gen_helix": (ctypes.c_int, [ctypes.POINTER(CGenParams), _i32, _i64, _i64, _i32, _vp, _vp, _vp, _i32]),
    "p2r_gen_helix_device": (ctypes.c_int, [ctypes.POINTER(CGenParams), _i32, _i64, _i64, _i32, _vp, _vp, _vp, _vp]),
    "p2r_gen_fixture": (ctypes.c_int, [_vp, _vp, _i32, _vp, _i32, _i32, _i64, _i64, _i32, ctypes.c_double, _vp, _vp]),
    "p2r_summary": (ctypes.c_int, [_vp, _i32, _i64, _i64, _vp, ctypes.POINTER(CSummary)]),
}

_lib = None


def lib() -> ctypes.CDLL:
    """Loads libp2r_b200.so once; raises if it is missing (no fallback path exists)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: run `python -m p2r_tests_b200.build` "
                               "(or __graft_entry__.build()) first")
        l = ctypes.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(l, name)
            fn.restype = res
            fn.argtypes = args
        if l.p2r_abi_version() != ABI_VERSION:
            raise RuntimeError(f"{LIB_PATH} reports ABI version {l.p2r_abi_version()}, these bindings follow "
                               f"{ABI_VERSION}: rebuild with `python -m p2r_tests_b200.build`")
        _lib = l
    return _lib


def check(rc: int) -> None:
    if rc != P2R_OK:
        raise P2RError(rc, lib().p2r_last_error_string().decode(errors="replace"))


def exported_symbols() -> list[str]:
    return list(SIGNATURES)
