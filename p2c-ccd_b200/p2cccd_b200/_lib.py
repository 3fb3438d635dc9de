"""ctypes binding of libp2c_b200.so (the C ABI in include/p2c_b200.h).

The library is the only compute path: if it is missing or fails to load, every
entry point raises.  There is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os
import threading
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libp2c_b200.so"

P2C_OK = 0
P2C_ERR_INVALID = 1
P2C_ERR_CUDA = 2
P2C_ERR_CAPACITY = 3
P2C_ERR_TIMEOUT = 4

_c_void_p = ctypes.c_void_p
_i64 = ctypes.c_int64
_f64 = ctypes.c_double
_int = ctypes.c_int
_size = ctypes.c_size_t


class CertConfig(ctypes.Structure):
    _fields_ = [("eps_time", ctypes.c_double), ("eps_space", ctypes.c_double),
                ("max_subdivision_depth", ctypes.c_uint16), ("pad", ctypes.c_uint16 * 3)]


class P2CError(RuntimeError):
    """Raised when the library reports a failure that is not a ValueError."""


# Signatures of every exported entry point: name -> (restype, argtypes).
SIGNATURES: dict[str, tuple] = {
    "p2c_last_error": (ctypes.c_char_p, []),
    "p2c_abi_version": (_int, []),
    "p2c_is_cuda_exact_built": (_int, []),
    "p2c_device_info": (_int, [_c_void_p, _c_void_p, _c_void_p, _c_void_p]),
    "p2c_certify_workspace_bytes": (_size, [_i64]),
    "p2c_certify_pt_batch": (_int, [_c_void_p, _i64, _f64, _f64, ctypes.POINTER(CertConfig), _c_void_p,
                                    _c_void_p, _size, _c_void_p, _c_void_p]),
    "p2c_certify_ee_batch": (_int, [_c_void_p, _i64, _f64, _f64, ctypes.POINTER(CertConfig), _c_void_p,
                                    _c_void_p, _size, _c_void_p, _c_void_p]),
    "p2c_certify_pt_batch_host": (_int, [_c_void_p, _i64, _f64, _f64, ctypes.POINTER(CertConfig), _c_void_p]),
    "p2c_certify_ee_batch_host": (_int, [_c_void_p, _i64, _f64, _f64, ctypes.POINTER(CertConfig), _c_void_p]),
    "p2c_certify_pt_batch_cpu": (_int, [_c_void_p, _i64, _f64, _f64, ctypes.POINTER(CertConfig), _c_void_p]),
    "p2c_certify_ee_batch_cpu": (_int, [_c_void_p, _i64, _f64, _f64, ctypes.POINTER(CertConfig), _c_void_p]),
    "p2c_certify_batch2": (_int, [_c_void_p, _i64, _c_void_p, _i64, _f64, _f64, ctypes.POINTER(CertConfig),
                                  _c_void_p, _c_void_p, _c_void_p, _size, _c_void_p, _c_void_p]),
    "p2c_certify_queries_workspace_bytes": (_size, [_i64]),
    "p2c_certify_queries": (_int, [_c_void_p, _i64, _c_void_p, _c_void_p, _i64, _c_void_p, _i64, _c_void_p,
                                   _c_void_p, _c_void_p, _c_void_p, _c_void_p, ctypes.POINTER(CertConfig),
                                   _c_void_p, _c_void_p, _c_void_p, _c_void_p, _size, _c_void_p, _c_void_p]),
    "p2c_certify_queries_static": (_int, [_c_void_p, _i64, _c_void_p, _c_void_p, _i64, _c_void_p, _i64,
                                          _c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_void_p,
                                          ctypes.POINTER(CertConfig), _c_void_p, _c_void_p, _c_void_p, _c_void_p,
                                          _c_void_p]),
    "p2c_scene_candidates_workspace_bytes": (_size, [_i64, _i64, _i64, _i64, _i64]),
    "p2c_scene_candidates": (_int, [_c_void_p, _c_void_p, _i64, _c_void_p, _i64, _c_void_p, _int, _c_void_p,
                                    _size, _c_void_p]),
    "p2c_scene_certify_workspace_bytes": (_size, []),
    "p2c_scene_certify": (_int, [_c_void_p, _c_void_p, _i64, _c_void_p, _i64, _c_void_p, _f64, _f64,
                                 ctypes.POINTER(CertConfig), ctypes.c_uint32, _c_void_p, _c_void_p, _c_void_p, _i64,
                                 _c_void_p, _c_void_p, _size, _c_void_p]),
    "p2c_scene_materialize": (_int, [_c_void_p, _c_void_p, _i64, _c_void_p, _i64, _c_void_p, _c_void_p,
                                     _c_void_p]),
    "p2c_batch_certify_workspace_bytes": (_size, [ctypes.c_int32]),
    "p2c_batch_candidates_workspace_bytes": (_size, [_c_void_p, ctypes.c_int32]),
    "p2c_batch_candidates": (_int, [_c_void_p, _c_void_p, ctypes.c_int32, _c_void_p, _size, _c_void_p]),
    "p2c_batch_certify": (_int, [_c_void_p, ctypes.c_int32, _f64, _f64, ctypes.POINTER(CertConfig), ctypes.c_uint32,
                                 _c_void_p, _c_void_p, _i64, _c_void_p, _c_void_p, _size, _c_void_p]),
    "p2c_group_anyhit_workspace_bytes": (_size, [_i64, ctypes.c_int32]),
    "p2c_group_anyhit": (_int, [_c_void_p, _int, _c_void_p, _i64, _c_void_p, _c_void_p, _i64, _f64, _f64,
                                ctypes.POINTER(CertConfig), _c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_void_p,
                                _c_void_p, _c_void_p, _size, _c_void_p]),
    "p2c_stub_scores": (_int, [_c_void_p, _c_void_p, _i64, _int, ctypes.c_uint64, _c_void_p, _c_void_p]),
    "p2c_batch_anyhit_workspace_bytes": (_size, [_c_void_p, ctypes.c_int32, ctypes.c_uint32]),
    "p2c_batch_anyhit": (_int, [_c_void_p, _c_void_p, ctypes.c_int32, ctypes.c_uint32, _c_void_p, _c_void_p, _i64,
                                _f64, _f64, ctypes.POINTER(CertConfig), _c_void_p, _c_void_p, _c_void_p, _c_void_p,
                                _c_void_p, _size, _c_void_p]),
    "p2c_serve_create": (_int, [_c_void_p, _c_void_p]),
    "p2c_serve_destroy": (_int, [_c_void_p]),
    "p2c_serve_register_mesh": (_int, [_c_void_p, _c_void_p, _c_void_p]),
    "p2c_serve_admit": (_int, [_c_void_p, _c_void_p, _c_void_p]),
    "p2c_serve_poll": (_int, [_c_void_p, _c_void_p, ctypes.c_int32, _c_void_p]),
    "p2c_serve_read_stats": (_int, [_c_void_p, _c_void_p]),
    "p2c_refinement_children_workspace_bytes": (_size, [_i64]),
    "p2c_refinement_children": (_int, [_i64, _c_void_p, _c_void_p, _c_void_p, _c_void_p, ctypes.c_uint16, _f64,
                                       ctypes.c_uint64, _c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_void_p,
                                       _c_void_p, _c_void_p, _c_void_p, _size, _c_void_p]),
    "p2c_proxy_candidates_workspace_bytes": (_size, [_i64, _i64, ctypes.c_uint32]),
    "p2c_proxy_candidates": (_int, [_c_void_p, _c_void_p, _i64, _c_void_p, _c_void_p, _c_void_p, _size, _c_void_p]),
    "p2c_compact_raw_candidates_workspace_bytes": (_size, [_i64, _i64, ctypes.c_uint32]),
    "p2c_compact_raw_candidates": (_int, [_c_void_p, _c_void_p, _i64, _c_void_p, _c_void_p, _c_void_p, _size,
                                          _c_void_p]),
    "p2c_proxy_scene_count": (_i64, [_c_void_p, _i64]),
    "p2c_proxy_scene_build_workspace_bytes": (_size, [_c_void_p, _i64]),
    "p2c_proxy_scene_build": (_int, [ctypes.c_uint64, _c_void_p, _i64, _c_void_p, _c_void_p, _c_void_p, _i64, _i64,
                                     _c_void_p, _c_void_p, _c_void_p, _size, _c_void_p]),
    "p2c_proposal_feature_rows_workspace_bytes": (_size, [_i64]),
    "p2c_proposal_feature_rows": (_int, [_c_void_p, _c_void_p, _i64, _c_void_p, _c_void_p, _c_void_p, _c_void_p,
                                         _c_void_p, _size, _c_void_p]),
    "p2c_runtime_feature_rows": (_int, [_c_void_p, _i64, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64, _c_void_p,
                                        _c_void_p, _i64, _c_void_p, _c_void_p, _c_void_p]),
    "p2c_audit_rows": (_int, [_c_void_p, _c_void_p, _i64, ctypes.c_uint64, ctypes.c_uint64, _int, _c_void_p,
                              _c_void_p, _c_void_p]),
    "p2c_schedule_work_items_workspace_bytes": (_size, [_i64, _i64, _i64]),
    "p2c_schedule_work_items": (_int, [_int, _c_void_p, _i64, _c_void_p, _i64, _c_void_p, _i64, _c_void_p, _c_void_p,
                                       _i64, _c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_void_p, _size, _c_void_p]),
    "p2c_dummy_schedule": (_int, [_int, _c_void_p, _i64, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64,
                                  _c_void_p, _c_void_p, _i64, _c_void_p, _c_void_p, _c_void_p, _c_void_p, _c_void_p,
                                  _c_void_p, _c_void_p, _size, _c_void_p]),
    "p2c_ordered_sum": (_int, [_c_void_p, _i64, _c_void_p, _c_void_p]),
    "p2c_dense_group_early_stop_workspace_bytes": (_size, [_i64]),
    "p2c_dense_group_early_stop": (_int, [_i64] + [_c_void_p] * 8 + [_c_void_p, _c_void_p, _c_void_p, _size,
                                                                     _c_void_p]),
    "p2c_probe_fp64": (_int, [_c_void_p, _int, ctypes.POINTER(ctypes.c_longlong), _c_void_p]),
    "p2c_certify_census": (_int, [_c_void_p, _i64, _c_void_p, _i64, _f64, _f64, ctypes.POINTER(CertConfig),
                                  _c_void_p, _c_void_p, _c_void_p, _size, _c_void_p, _c_void_p]),
}

_lock = threading.Lock()
_lib = None


def load() -> ctypes.CDLL:
    """Load the library once; raise if it is absent (no fallback path exists)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        path = Path(os.environ.get("P2C_B200_LIB", LIB_PATH))
        if not path.exists():
            raise P2CError(f"libp2c_b200.so not found at {path}; build it with p2cccd_b200.build.build()")
        lib = ctypes.CDLL(str(path))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib


def last_error() -> str:
    msg = load().p2c_last_error()
    return msg.decode("utf-8", "replace") if msg else ""


def check(rc: int) -> None:
    """Map a status code to the reference's error convention (ValueError)."""
    if rc == P2C_OK:
        return
    msg = last_error()
    if rc == P2C_ERR_INVALID:
        raise ValueError(msg)
    raise P2CError(f"p2c error {rc}: {msg}")


def make_config(eps_time: float, eps_space: float, max_subdivision_depth: int) -> CertConfig:
    cfg = CertConfig()
    cfg.eps_time = float(eps_time)
    cfg.eps_space = float(eps_space)
    cfg.max_subdivision_depth = int(max_subdivision_depth) & 0xFFFF
    return cfg
