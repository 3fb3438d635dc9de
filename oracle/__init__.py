"""Python access to the CPU oracle — TEST INFRASTRUCTURE ONLY.

Two checkers, both loaded with ctypes:
  * ``_build/libccd_oracle.so``: ccd_oracle.c, a plain-C restatement of the
    reference algorithms (certifier, aggregation, swept boxes, sort-and-sweep
    pairs, group any-hit with fallback replay, refinement children);
  * ``_ref/libp2c_ref.so``: the reference's own sources compiled unchanged with
    ref_abi.cpp (present when the reference checkout was available at build
    time; the built file travels with the tree).
  * ``_ref/libp2c_ref_tool.so``: the reference's scene any-hit tool compiled
    unchanged (ref_tool.cpp), its Tight-Inclusion calls answered by the
    reference certifier through shim/tight_inclusion/ccd.hpp.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this package.  The product library never does.
"""
from __future__ import annotations

import ctypes
import math
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "_build" / "libccd_oracle.so"
REF_SO = HERE / "_ref" / "libp2c_ref.so"
REF_TOOL_SO = HERE / "_ref" / "libp2c_ref_tool.so"
REF_CUDA_SO = HERE / "_ref" / "libp2c_ref_cuda.so"

TRAJ = np.dtype([("feature_id", "<i8"), ("position_t0", "<f8", (3,)), ("position_t1", "<f8", (3,))])
PT = np.dtype([("point_id", "<i8"), ("triangle_id", "<i8"), ("point", TRAJ), ("triangle_v0", TRAJ),
               ("triangle_v1", TRAJ), ("triangle_v2", TRAJ)])
EE = np.dtype([("edge_a_id", "<i8"), ("edge_b_id", "<i8"), ("edge_a0", TRAJ), ("edge_a1", TRAJ),
               ("edge_b0", TRAJ), ("edge_b1", TRAJ)])
RESULT = np.dtype({
    "names": ["status", "covered_feature_mask", "interval_t0", "interval_t1", "toi_upper", "safe_margin_lb",
              "witness_family", "witness_id_a", "witness_id_b", "reason_code", "next_refinement_mode"],
    "formats": ["u1", "<u4", "<f8", "<f8", "<f8", "<f8", "u1", "<i8", "<i8", "<u2", "u1"],
    "offsets": [0, 4, 8, 16, 24, 32, 40, 48, 56, 64, 66],
    "itemsize": 72,
})
QUERY_CERT = np.dtype({
    "names": ["status", "witness_family", "reason_code", "covered_feature_mask", "toi_upper", "safe_margin_lb",
              "witness_id_a", "witness_id_b", "witness_index", "next_refinement_mode"],
    "formats": ["u1", "u1", "<u2", "<u4", "<f8", "<f8", "<i8", "<i8", "<i8", "u1"],
    "offsets": [0, 1, 2, 4, 8, 16, 24, 32, 40, 48],
    "itemsize": 56,
})


class _Cfg(ctypes.Structure):
    _fields_ = [("eps_time", ctypes.c_double), ("eps_space", ctypes.c_double),
                ("max_subdivision_depth", ctypes.c_uint16), ("pad", ctypes.c_uint16 * 3)]


def build() -> None:
    """Compile the oracle (always) and the reference library (when its sources exist)."""
    subprocess.run(["make", "-s", "-C", str(HERE), "all"], check=True)


_oracle = None
_ref = None


def _p(a):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


def lib() -> ctypes.CDLL:
    global _oracle
    if _oracle is None:
        if not ORACLE_SO.exists():
            build()
        _oracle = ctypes.CDLL(str(ORACLE_SO))
        L = _oracle
        vp, i64, f64 = ctypes.c_void_p, ctypes.c_int64, ctypes.c_double
        L.oracle_eval_pt_batch.argtypes = [vp, i64, f64, f64, ctypes.POINTER(_Cfg), vp, vp, vp]
        L.oracle_eval_ee_batch.argtypes = [vp, i64, f64, f64, ctypes.POINTER(_Cfg), vp, vp, vp]
        L.oracle_eval_pt_batch.restype = i64
        L.oracle_eval_ee_batch.restype = i64
        L.oracle_aggregate.argtypes = [ctypes.c_uint32, f64, vp, i64, vp, i64, vp]
        L.oracle_swept_boxes.argtypes = [vp, vp, vp, ctypes.c_int, i64, f64, vp]
        for name in ("oracle_vf_pairs_brute", "oracle_vf_pairs_sweep"):
            getattr(L, name).argtypes = [vp, vp, vp, i64, vp, vp, vp, i64, vp, ctypes.c_int32, vp, i64]
            getattr(L, name).restype = i64
        for name in ("oracle_ee_pairs_brute", "oracle_ee_pairs_sweep"):
            getattr(L, name).argtypes = [vp, vp, vp, i64, vp, ctypes.c_int32, vp, i64]
            getattr(L, name).restype = i64
        L.oracle_object_allowed.argtypes = [vp, vp, vp, i64, ctypes.c_int32, f64, ctypes.c_int, vp]
        L.oracle_group_anyhit.argtypes = [i64, vp, vp, ctypes.c_int32, vp, vp, vp, vp, vp, vp]
        L.oracle_refinement_children.argtypes = [f64, f64, ctypes.c_uint16, ctypes.c_uint8, ctypes.c_uint8, f64,
                                                 ctypes.c_uint16, f64, vp, vp]
        L.oracle_refinement_children.restype = ctypes.c_int
    return _oracle


def ref_available() -> bool:
    return REF_SO.exists()


_ref_cuda = None


def ref_cuda_available() -> bool:
    return REF_CUDA_SO.exists()


def ref_cuda() -> ctypes.CDLL:
    """The reference's CUDA batch certifier compiled unchanged
    (certificate_cuda.cu, oracle/ref_cuda.cpp): needs a GPU to run."""
    global _ref_cuda
    if _ref_cuda is None:
        if not REF_CUDA_SO.exists():
            raise FileNotFoundError(f"{REF_CUDA_SO} is not built (reference CUDA sources or nvcc absent)")
        _ref_cuda = ctypes.CDLL(str(REF_CUDA_SO))
        C = _ref_cuda
        vp, i64, f64, ci = ctypes.c_void_p, ctypes.c_int64, ctypes.c_double, ctypes.c_int
        C.ref_cuda_last_error.restype = ctypes.c_char_p
        C.ref_cuda_eval_batch.argtypes = [ci, vp, i64, f64, f64, f64, f64, ci, vp]
        C.ref_cuda_cross_check.argtypes = [vp, i64, vp, i64, f64, f64, f64, f64, ci, f64]
    return _ref_cuda


def ref_cuda_eval_batch(records: np.ndarray, t0: float, t1: float, eps_time: float, eps_space: float,
                        max_depth: int) -> np.ndarray:
    """EvaluatePointTriangleBatchCuda / EvaluateEdgeEdgeBatchCuda of the
    reference (host records in, results out; the family from the dtype)."""
    C = ref_cuda()
    fam = 1 if records.dtype.names[0] == "point_id" else 2
    out = np.zeros(len(records), dtype=RESULT)
    if C.ref_cuda_eval_batch(fam, _p(records), len(records), t0, t1, eps_time, eps_space, max_depth, _p(out)):
        raise RuntimeError(C.ref_cuda_last_error().decode())
    return out


def ref_cuda_cross_check(pt: np.ndarray, ee: np.ndarray, t0: float, t1: float, eps_time: float, eps_space: float,
                         max_depth: int, eps_cert: float) -> tuple[bool, str]:
    """The reference's CrossCheckCpuCudaExact: (agree, message)."""
    C = ref_cuda()
    rc = C.ref_cuda_cross_check(_p(pt), len(pt), _p(ee), len(ee), t0, t1, eps_time, eps_space, max_depth, eps_cert)
    return rc == 0, C.ref_cuda_last_error().decode()


def ref() -> ctypes.CDLL:
    global _ref
    if _ref is None:
        if not REF_SO.exists():
            raise FileNotFoundError(f"{REF_SO} is not built (the reference sources were not available)")
        _ref = ctypes.CDLL(str(REF_SO))
        R = _ref
        vp, i64, f64, ci = ctypes.c_void_p, ctypes.c_int64, ctypes.c_double, ctypes.c_int
        R.ref_last_error.restype = ctypes.c_char_p
        for name in ("ref_eval_pt_batch", "ref_eval_ee_batch"):
            getattr(R, name).argtypes = [vp, i64, f64, f64, f64, f64, ci, vp, vp, ci]
            getattr(R, name).restype = i64
        for name in ("ref_eval_pt_one", "ref_eval_ee_one"):
            getattr(R, name).argtypes = [vp, f64, f64, f64, f64, ci, vp]
            getattr(R, name).restype = ci
        R.ref_evaluate_query.argtypes = [ctypes.c_uint32, f64, f64, f64, f64, ci, vp, i64, vp, i64, vp]
        R.ref_build_mesh_query.argtypes = [vp, i64, vp, i64, vp, vp, vp, i64, vp, i64, vp, vp, ctypes.c_uint32,
                                           ci, ctypes.c_uint64, ctypes.c_uint64, vp, vp, vp, vp]
        R.ref_refinement_children.argtypes = [f64, f64, ctypes.c_uint16, ctypes.c_uint8, ctypes.c_uint8, f64,
                                              ctypes.c_uint16, f64, vp, vp]
        R.ref_refinement_children.restype = ci
    return _ref


def _family(records: np.ndarray) -> int:
    if records.dtype.itemsize != 240:
        raise ValueError("records must be 240-byte primitives")
    return 1 if records.dtype.names[0] == "point_id" else 2


def eval_batch(records: np.ndarray, t0: float = 0.0, t1: float = 1.0, eps_time: float = 1e-4,
               eps_space: float = 1e-6, max_depth: int = 32):
    """Oracle certificates: returns (results RESULT array, status uint8 (0 ok / 1 invalid), nodes uint64)."""
    rec = np.ascontiguousarray(records)
    n = len(rec)
    out = np.zeros(n, dtype=RESULT)
    status = np.zeros(n, dtype=np.uint8)
    nodes = np.zeros(n, dtype=np.uint64)
    cfg = _Cfg(eps_time, eps_space, max_depth)
    fn = lib().oracle_eval_pt_batch if _family(rec) == 1 else lib().oracle_eval_ee_batch
    fn(_p(rec), n, t0, t1, ctypes.byref(cfg), _p(out), _p(status), _p(nodes))
    return out, status, nodes


def ref_eval_batch(records: np.ndarray, t0: float = 0.0, t1: float = 1.0, eps_time: float = 1e-4,
                   eps_space: float = 1e-6, max_depth: int = 32, threads: int = 1):
    """Reference certificates (unchanged reference code): (results, status)."""
    rec = np.ascontiguousarray(records)
    n = len(rec)
    out = np.zeros(n, dtype=RESULT)
    status = np.zeros(n, dtype=np.uint8)
    fn = ref().ref_eval_pt_batch if _family(rec) == 1 else ref().ref_eval_ee_batch
    fn(_p(rec), n, t0, t1, eps_time, eps_space, max_depth, _p(out), _p(status), threads)
    return out, status


def ref_eval_error(record: np.ndarray, t0: float, t1: float, eps_time: float, eps_space: float,
                   max_depth: int) -> str | None:
    """Error message the reference raises for one primitive (None if it succeeds)."""
    rec = np.ascontiguousarray(record.reshape(1))
    out = np.zeros(1, dtype=RESULT)
    fn = ref().ref_eval_pt_one if _family(rec) == 1 else ref().ref_eval_ee_one
    rc = fn(_p(rec), t0, t1, eps_time, eps_space, max_depth, _p(out))
    return ref().ref_last_error().decode() if rc else None


def aggregate(family_mask: int, pt_results: np.ndarray, ee_results: np.ndarray,
              interval_t1: float = 1.0) -> np.ndarray:
    out = np.zeros(1, dtype=QUERY_CERT)
    pt_r = np.ascontiguousarray(pt_results)
    ee_r = np.ascontiguousarray(ee_results)
    lib().oracle_aggregate(family_mask, interval_t1, _p(pt_r), len(pt_r), _p(ee_r), len(ee_r), _p(out))
    return out[0]


def ref_evaluate_query(family_mask: int, pts: np.ndarray, ees: np.ndarray, t0: float = 0.0, t1: float = 1.0,
                       eps_time: float = 1e-4, eps_space: float = 1e-6, max_depth: int = 32):
    out = np.zeros(1, dtype=QUERY_CERT)
    a = np.ascontiguousarray(pts)
    b = np.ascontiguousarray(ees)
    rc = ref().ref_evaluate_query(family_mask, t0, t1, eps_time, eps_space, max_depth, _p(a), len(a), _p(b),
                                  len(b), _p(out))
    if rc:
        raise ValueError(ref().ref_last_error().decode())
    return out[0]


def swept_boxes(v_t0: np.ndarray, v_t1: np.ndarray, prim_vertices: np.ndarray | None, k: int,
                thickness: float = 0.0) -> np.ndarray:
    v_t0 = np.ascontiguousarray(v_t0, dtype=np.float64)
    v_t1 = np.ascontiguousarray(v_t1, dtype=np.float64)
    if prim_vertices is None:
        n = len(v_t0)
        pv = None
    else:
        pv = np.ascontiguousarray(prim_vertices, dtype=np.int32)
        n = pv.shape[0]
    out = np.zeros((n, 6), dtype=np.float64)
    lib().oracle_swept_boxes(_p(v_t0), _p(v_t1), _p(pv), k, n, thickness, _p(out))
    return out


def _pairs(fn, *args, cap: int | None = None) -> np.ndarray:
    n = fn(*args, None, 0)
    out = np.zeros(max(n, 1), dtype=np.uint64)
    fn(*args, _p(out), n)
    return out[:n]


def vf_pairs(vbox, v_obj, v_valid, fbox, f_obj, faces, allowed, method: str = "sweep") -> np.ndarray:
    vbox = np.ascontiguousarray(vbox, dtype=np.float64)
    fbox = np.ascontiguousarray(fbox, dtype=np.float64)
    v_obj = np.ascontiguousarray(v_obj, dtype=np.int32)
    f_obj = np.ascontiguousarray(f_obj, dtype=np.int32)
    faces = np.ascontiguousarray(faces, dtype=np.int32)
    allowed = np.ascontiguousarray(allowed, dtype=np.uint8)
    v_valid = None if v_valid is None else np.ascontiguousarray(v_valid, dtype=np.uint8)
    fn = lib().oracle_vf_pairs_sweep if method == "sweep" else lib().oracle_vf_pairs_brute
    return _pairs(fn, _p(vbox), _p(v_obj), _p(v_valid), len(vbox), _p(fbox), _p(f_obj), _p(faces), len(fbox),
                  _p(allowed), allowed.shape[0])


def ee_pairs(ebox, e_obj, edges, allowed, method: str = "sweep") -> np.ndarray:
    ebox = np.ascontiguousarray(ebox, dtype=np.float64)
    e_obj = np.ascontiguousarray(e_obj, dtype=np.int32)
    edges = np.ascontiguousarray(edges, dtype=np.int32)
    allowed = np.ascontiguousarray(allowed, dtype=np.uint8)
    fn = lib().oracle_ee_pairs_sweep if method == "sweep" else lib().oracle_ee_pairs_brute
    return _pairs(fn, _p(ebox), _p(e_obj), _p(edges), len(ebox), _p(allowed), allowed.shape[0])


def object_allowed(v_t0, v_t1, v_obj, n_obj: int, thickness: float = 0.0, exclude_self: bool = False):
    v_t0 = np.ascontiguousarray(v_t0, dtype=np.float64)
    v_t1 = np.ascontiguousarray(v_t1, dtype=np.float64)
    v_obj = np.ascontiguousarray(v_obj, dtype=np.int32)
    out = np.zeros((n_obj, n_obj), dtype=np.uint8)
    lib().oracle_object_allowed(_p(v_t0), _p(v_t1), _p(v_obj), len(v_obj), n_obj, thickness, int(exclude_self),
                                _p(out))
    return out


def group_anyhit(cand_group, cand_hit, n_groups: int, top_offsets, top_index):
    cand_group = np.ascontiguousarray(cand_group, dtype=np.int32)
    cand_hit = np.ascontiguousarray(cand_hit, dtype=np.uint8)
    top_offsets = np.ascontiguousarray(top_offsets, dtype=np.int64)
    top_index = np.ascontiguousarray(top_index, dtype=np.int64)
    det = np.zeros(n_groups, dtype=np.uint8)
    pc = np.zeros(n_groups, dtype=np.int64)
    fc = np.zeros(n_groups, dtype=np.int64)
    ev = np.zeros(len(cand_group), dtype=np.uint8)
    lib().oracle_group_anyhit(len(cand_group), _p(cand_group), _p(cand_hit), n_groups, _p(top_offsets),
                              _p(top_index), _p(det), _p(pc), _p(fc), _p(ev))
    return det, pc, fc, ev


def refinement_children(t0, t1, depth, status, mode, toi, max_child_depth=64, min_width=1e-4, use_ref=False):
    c0 = np.zeros(2)
    c1 = np.zeros(2)
    L = ref() if use_ref else lib()
    fn = L.ref_refinement_children if use_ref else L.oracle_refinement_children
    n = fn(t0, t1, depth, status, mode, toi, max_child_depth, min_width, _p(c0), _p(c1))
    return [(float(c0[i]), float(c1[i])) for i in range(max(n, 0))]


def ref_build_mesh_query(va, fa, ta0, ta1, vb, fb, tb0, tb1, family_mask=3, prune=True, max_pt=0, max_ee=0):
    """BuildMeshExactCertificateQuery via the reference: (pt records, ee records)."""
    va = np.ascontiguousarray(va, dtype=np.float64)
    vb = np.ascontiguousarray(vb, dtype=np.float64)
    fa = np.ascontiguousarray(fa, dtype=np.uint32)
    fb = np.ascontiguousarray(fb, dtype=np.uint32)
    t = [np.ascontiguousarray(x, dtype=np.float64) for x in (ta0, ta1, tb0, tb1)]
    npt = ctypes.c_int64(0)
    nee = ctypes.c_int64(0)
    R = ref()
    args = [_p(va), len(va), _p(fa), len(fa), _p(t[0]), _p(t[1]), _p(vb), len(vb), _p(fb), len(fb), _p(t[2]),
            _p(t[3]), family_mask, int(prune), max_pt, max_ee]
    rc = R.ref_build_mesh_query(*args, None, ctypes.byref(npt), None, ctypes.byref(nee))
    if rc:
        raise ValueError(R.ref_last_error().decode())
    pts = np.zeros(npt.value, dtype=PT)
    ees = np.zeros(nee.value, dtype=EE)
    R.ref_build_mesh_query(*args, _p(pts), ctypes.byref(npt), _p(ees), ctypes.byref(nee))
    return pts, ees


# ---- the reference scene tool (tools/scene_object_envelope_native_ti_walltime.cpp) ----

_ref_tool = None

TOOL_ROW_FIELDS = ("all_exact_calls", "all_hit_count", "all_group_count", "all_positive_groups",
                   "exact_calls", "proposal_exact_calls", "fallback_exact_calls", "hit_count", "group_count",
                   "positive_groups", "fallback_groups", "tp", "fp", "fn", "tn", "positive_first_hit_rank_sum")


def ref_tool() -> ctypes.CDLL:
    global _ref_tool
    if _ref_tool is None:
        if not REF_TOOL_SO.exists():
            raise FileNotFoundError(f"{REF_TOOL_SO} is not built (the reference sources were not available)")
        T = ctypes.CDLL(str(REF_TOOL_SO))
        vp, i64, f64, ci, u64 = ctypes.c_void_p, ctypes.c_int64, ctypes.c_double, ctypes.c_int, ctypes.c_uint64
        T.ref_tool_last_error.restype = ctypes.c_char_p
        T.ref_tool_prepare.argtypes = [vp, vp, i64, vp, i64, f64, ci]
        T.ref_tool_objects.argtypes = [vp, vp]
        T.ref_tool_edges.argtypes = [vp, vp]
        T.ref_tool_edges.restype = i64
        T.ref_tool_candidates.argtypes = [ci, u64, vp, vp, i64, vp]
        T.ref_tool_candidates.restype = i64
        T.ref_tool_random_scores.argtypes = [ci, vp]
        T.ref_tool_anyhit.argtypes = [ci, u64, f64, f64, ci, vp]
        T.ref_tool_time_step.argtypes = [u64, f64, f64, ci, vp, vp, vp]
        T.ref_tool_time_all_exact.argtypes = [f64, f64, ci, vp, vp]
        _ref_tool = T
    return _ref_tool


class RefToolScene:
    """The reference tool's PrepareScene over one step of a triangle soup,
    then its candidate lists, random-policy scores and any-hit rows."""

    def __init__(self, v_t0, v_t1, faces, thickness: float = 0.0, exclude_self: bool = False):
        T = ref_tool()
        self.v_t0 = np.ascontiguousarray(v_t0, dtype=np.float64)
        self.v_t1 = np.ascontiguousarray(v_t1, dtype=np.float64)
        self.faces = np.ascontiguousarray(faces, dtype=np.int32)
        if T.ref_tool_prepare(_p(self.v_t0), _p(self.v_t1), len(self.v_t0), _p(self.faces), len(self.faces),
                              float(thickness), int(exclude_self)):
            raise ValueError(T.ref_tool_last_error().decode())
        self.v_obj = np.zeros(len(self.v_t0), dtype=np.int32)
        self.f_obj = np.zeros(len(self.faces), dtype=np.int32)
        self.n_obj = T.ref_tool_objects(_p(self.v_obj), _p(self.f_obj))
        ne = T.ref_tool_edges(None, None)
        self.edges = np.zeros((ne, 2), dtype=np.int32)
        self.e_obj = np.zeros(ne, dtype=np.int32)
        T.ref_tool_edges(_p(self.edges), _p(self.e_obj))

    def candidates(self, kind: str, max_candidates: int = 0) -> np.ndarray:
        """(n, 2) int32 pairs in the tool's emission order: (vertex, face) or (edge, edge)."""
        T = ref_tool()
        k = 0 if kind == "vf" else 1
        capped = ctypes.c_int(0)
        n = T.ref_tool_candidates(k, max_candidates, None, None, 0, ctypes.byref(capped))
        a = np.zeros(max(n, 1), dtype=np.int32)
        b = np.zeros(max(n, 1), dtype=np.int32)
        T.ref_tool_candidates(k, max_candidates, _p(a), _p(b), n, ctypes.byref(capped))
        self.capped = bool(capped.value)
        return np.stack([a[:n], b[:n]], axis=1)

    def random_scores(self, kind: str, n: int) -> np.ndarray:
        out = np.zeros(max(n, 1), dtype=np.float64)
        ref_tool().ref_tool_random_scores(0 if kind == "vf" else 1, _p(out))
        return out[:n]

    def anyhit(self, kind: str, top_k: int, eps_time: float, eps_space: float, max_depth: int) -> dict:
        out = np.zeros(16, dtype=np.uint64)
        T = ref_tool()
        if T.ref_tool_anyhit(0 if kind == "vf" else 1, top_k, eps_time, eps_space, max_depth, _p(out)):
            raise ValueError(T.ref_tool_last_error().decode())
        return {k: int(v) for k, v in zip(TOOL_ROW_FIELDS, out)}

    def time_step(self, top_k: int, eps_time: float, eps_space: float, max_depth: int) -> dict:
        """The tool's candidates + scheduled any-hit of both families, timed inside the library."""
        secs = np.zeros(3)
        calls = np.zeros(2, dtype=np.uint64)
        cands = np.zeros(2, dtype=np.uint64)
        T = ref_tool()
        if T.ref_tool_time_step(top_k, eps_time, eps_space, max_depth, _p(secs), _p(calls), _p(cands)):
            raise ValueError(T.ref_tool_last_error().decode())
        return {"candidates_s": float(secs[0]), "anyhit_vf_s": float(secs[1]), "anyhit_ee_s": float(secs[2]),
                "calls": int(calls.sum()), "candidates": int(cands.sum())}

    def time_all_exact(self, eps_time: float, eps_space: float, max_depth: int) -> dict:
        """The tool's candidates + every-candidate certificates of both families, timed inside the library."""
        secs = np.zeros(2)
        calls = np.zeros(1, dtype=np.uint64)
        T = ref_tool()
        if T.ref_tool_time_all_exact(eps_time, eps_space, max_depth, _p(secs), _p(calls)):
            raise ValueError(T.ref_tool_last_error().decode())
        return {"candidates_s": float(secs[0]), "certify_s": float(secs[1]), "calls": int(calls[0])}


# ---- proxy-scene candidates (rt_candidate/candidate_buffer.cpp) ----

def _proxy_args(sc):
    a = {k: np.ascontiguousarray(sc[k]) for k in ("object_id", "patch_id", "slab_id", "proxy_type", "t0", "t1",
                                                   "bounds", "motion_bound")}
    return a


def ref_proxy_candidates(sc: dict):
    """The reference's GenerateRawCandidatesCpu + CompactRawCandidates on a
    proxy scene: (raw hits as 64-byte records, candidates as 80-byte records)."""
    from p2cccd_b200.records import CANDIDATE_RECORD_DTYPE, RAW_HIT_DTYPE

    R = ref()
    if not hasattr(R, "_proxy_ready"):
        vp, i64 = ctypes.c_void_p, ctypes.c_int64
        R.ref_proxy_candidates.argtypes = [ctypes.c_uint64, i64] + [vp] * 8 + [vp, i64, vp, i64, vp, vp]
        R.ref_proxy_last_error.restype = ctypes.c_char_p
        R._proxy_ready = True
    a = _proxy_args(sc)
    n_raw, n_cand = ctypes.c_int64(0), ctypes.c_int64(0)
    args = [int(sc["query_id"]), int(sc["n"])] + [_p(a[k]) for k in ("object_id", "patch_id", "slab_id",
                                                                      "proxy_type", "t0", "t1", "bounds",
                                                                      "motion_bound")]
    if R.ref_proxy_candidates(*args, None, 0, None, 0, ctypes.byref(n_raw), ctypes.byref(n_cand)):
        raise ValueError(R.ref_proxy_last_error().decode())
    raw = np.zeros(max(1, n_raw.value), dtype=RAW_HIT_DTYPE)
    cand = np.zeros(max(1, n_cand.value), dtype=CANDIDATE_RECORD_DTYPE)
    R.ref_proxy_candidates(*args, _p(raw), n_raw.value, _p(cand), n_cand.value, ctypes.byref(n_raw),
                           ctypes.byref(n_cand))
    return raw[:n_raw.value], cand[:n_cand.value]


def proxy_candidates(sc: dict):
    """Restatement of GenerateRawCandidatesCpu (candidate_buffer.cpp:144-179)
    and CompactRawCandidates (:181-227) in numpy: every pair i < j of
    different objects in one slab whose time intervals and inclusive AABBs
    overlap, in (i, j) order; then hits grouped by MakeCandidateKey (:104-124)
    in key order with counts, float-max motion bounds and or-ed flags."""
    from p2cccd_b200.records import CANDIDATE_RECORD_DTYPE, RAW_HIT_DTYPE

    a = _proxy_args(sc)
    n = int(sc["n"])
    obj, pat, slab, typ = a["object_id"], a["patch_id"], a["slab_id"], a["proxy_type"]
    t0, t1, b, mb = a["t0"], a["t1"], a["bounds"], a["motion_bound"]
    hits = []
    for i in range(n):
        j = np.arange(i + 1, n)
        ok = (obj[j] != obj[i]) & (slab[j] == slab[i]) & (t0[i] < t1[j]) & (t0[j] < t1[i])
        for ax in range(3):
            ok &= ~((b[i, 3 + ax] < b[j, ax]) | (b[j, 3 + ax] < b[i, ax]))
        hits.extend((i, int(x)) for x in j[ok])
    raw = np.zeros(len(hits), dtype=RAW_HIT_DTYPE)
    for k, (i, j) in enumerate(hits):
        raw[k]["query_id"] = sc["query_id"]
        raw[k]["pair_key"] = (i << 32) | j
        raw[k]["proxy_a_index"], raw[k]["proxy_b_index"] = i, j
        raw[k]["slab_id"] = slab[i]
        raw[k]["rt_hit_count"] = 1
        raw[k]["flags"] = 3
        raw[k]["motion_bound"] = np.maximum(mb[i], mb[j]).astype(np.float32)
    groups = {}
    for k, (i, j) in enumerate(hits):
        f, s2 = (i, j) if (obj[i], pat[i], i) <= (obj[j], pat[j], j) else (j, i)
        key = (int(slab[i]), int(obj[f]), int(pat[f]), int(obj[s2]), int(pat[s2]), int(typ[f]), int(typ[s2]))
        if key not in groups:
            groups[key] = [0, raw[k]["motion_bound"].copy(), 0]
        g = groups[key]
        g[0] += 1
        g[1] = np.maximum(g[1], raw[k]["motion_bound"])
        g[2] |= int(raw[k]["flags"])
    cand = np.zeros(len(groups), dtype=CANDIDATE_RECORD_DTYPE)
    for cid, key in enumerate(sorted(groups)):
        c = cand[cid]
        c["schema_version"], c["candidate_id"], c["query_id"] = 1, cid + 1, sc["query_id"]
        (c["slab_id"], c["object_a_id"], c["patch_a_id"], c["object_b_id"], c["patch_b_id"], c["proxy_type_a"],
         c["proxy_type_b"]) = key
        c["rt_hit_count"], c["motion_bound"], c["flags"] = groups[key]
    return raw, cand


# ---- proxy-scene build (rt_candidate/proxy_scene.cpp, geometry/) ----

def _build_flat(inp: dict):
    objs = inp["objects"]
    n_p = np.array([len(o["patch_id"]) for o in objs], np.int64)
    n_s = np.array([len(o["segments"]) for o in objs], np.int64)
    flat = {
        "object_id": np.array([o["object_id"] for o in objs], np.uint32),
        "proxy_type": np.array([o["proxy_type"] for o in objs], np.uint32),
        "slabs": np.array([o["slabs_per_motion_segment"] for o in objs], np.uint32),
        "eps": np.array([o["eps_proxy"] for o in objs], np.float64),
        "patch_offset": np.concatenate([[0], np.cumsum(n_p)[:-1]]).astype(np.int64), "n_patches": n_p,
        "segment_offset": np.concatenate([[0], np.cumsum(n_s)[:-1]]).astype(np.int64), "n_segments": n_s,
        "patch_id": np.ascontiguousarray(np.concatenate([np.asarray(o["patch_id"], np.uint32) for o in objs])),
        "patch_center": np.ascontiguousarray(np.concatenate([np.asarray(o["local_center"], np.float64).reshape(-1, 3)
                                                             for o in objs])),
        "patch_radius": np.ascontiguousarray(np.concatenate([np.asarray(o["radius"], np.float64) for o in objs])),
        "segments": np.ascontiguousarray(np.concatenate([np.asarray(o["segments"], np.float64).reshape(-1, 16)
                                                         for o in objs])),
    }
    return flat


BUILT_FIELDS = (("object_id", np.uint32, ()), ("patch_id", np.uint32, ()), ("slab_id", np.uint32, ()),
                ("motion_segment_id", np.uint32, ()), ("proxy_type", np.uint8, ()), ("t0", np.float64, ()),
                ("t1", np.float64, ()), ("bounds", np.float64, (6,)), ("motion_bound", np.float64, (4,)),
                ("motion_detail", np.float64, (8,)), ("capsule_radius", np.float64, ()))


def ref_build_proxy_scene(inp: dict) -> dict:
    """The reference's BuildProxyScene on a build input (the dict of
    ``scenes.proxy_build_input``): the primitive arrays, or ValueError with
    the reference's message."""
    R = ref()
    if not hasattr(R, "_build_ready"):
        vp, i64 = ctypes.c_void_p, ctypes.c_int64
        R.ref_build_proxy_scene.argtypes = [ctypes.c_uint64, i64] + [vp] * 12 + [i64] + [vp] * 12
        R.ref_proxy_last_error.restype = ctypes.c_char_p
        R._build_ready = True
    f = _build_flat(inp)
    n = ctypes.c_int64(0)
    ins = [int(inp["query_id"]), len(inp["objects"])] + [_p(f[k]) for k in (
        "object_id", "proxy_type", "slabs", "eps", "patch_offset", "n_patches", "segment_offset", "n_segments",
        "patch_id", "patch_center", "patch_radius", "segments")]
    if R.ref_build_proxy_scene(*ins, 0, *([None] * 11), ctypes.byref(n)):
        raise ValueError(R.ref_proxy_last_error().decode())
    out = {k: np.zeros((max(n.value, 1),) + sh, dt) for k, dt, sh in BUILT_FIELDS}
    R.ref_build_proxy_scene(*ins, n.value, *[_p(out[k]) for k, _, _ in BUILT_FIELDS], ctypes.byref(n))
    out = {k: v[:n.value] for k, v in out.items()}
    out["query_id"], out["n"] = int(inp["query_id"]), n.value
    return out


def _norm4(q):
    """NormalizeQuaternion (geometry/motion_utils.cpp:64-77)."""
    if not all(math.isfinite(x) for x in q):
        raise ValueError("quaternion contains a non-finite value")
    nrm = math.sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3])
    if not math.isfinite(nrm) or nrm <= 0.0:
        raise ValueError("quaternion norm must be positive and finite")
    return [q[0] / nrm, q[1] / nrm, q[2] / nrm, q[3] / nrm]


def _clamp(v, lo, hi):
    return lo if v < lo else (hi if hi < v else v)


def _slerp(a, b, alpha):
    """Slerp (:99-126), LerpAndNormalize (:87-97) past dot 0.9995."""
    d = a[0] * b[0] + a[1] * b[1] + a[2] * b[2] + a[3] * b[3]
    if d < 0.0:
        b = [-x for x in b]
        d = -d
    d = _clamp(d, -1.0, 1.0)
    if d > 0.9995:
        q = [(1.0 - alpha) * a[k] + alpha * b[k] for k in range(4)]
        nrm = math.sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3])
        return [x / nrm for x in q]
    th0 = math.acos(d)
    th = th0 * alpha
    st, st0 = math.sin(th), math.sin(th0)
    s0 = math.cos(th) - d * st / st0
    s1 = st / st0
    return [s0 * a[k] + s1 * b[k] for k in range(4)]


def _rotate(q, v):
    """RotateVector (:128-135)."""
    u0, u1, u2, s = q
    k0 = 2.0 * (u0 * v[0] + u1 * v[1] + u2 * v[2])
    k1 = s * s - (u0 * u0 + u1 * u1 + u2 * u2)
    k2 = 2.0 * s
    c = (u1 * v[2] - u2 * v[1], u2 * v[0] - u0 * v[2], u0 * v[1] - u1 * v[0])
    return [(q[a] * k0 + v[a] * k1) + c[a] * k2 for a in range(3)]


def _check_aabb(mn, mx, msg_finite, msg_order):
    """ValidateAabb (geometry/proxy.cpp:21-31) / ValidateAabbBounds
    (proxy_scene.cpp:25-35): axis by axis, finiteness then order."""
    for a in range(3):
        if not (math.isfinite(mn[a]) and math.isfinite(mx[a])):
            raise ValueError(msg_finite)
        if mn[a] > mx[a]:
            raise ValueError(msg_order)


def build_proxy_scene(inp: dict) -> dict:
    """Restatement of BuildProxyScene (proxy_scene.cpp:156-213): per object,
    motion segment, uniform slab (GenerateUniformTimeSlabs,
    motion_utils.cpp:175-185) and patch one proxy; ComputePatchMotionBound
    (:269-325) with the interpolated poses (InterpolateRigidMotion, :196-229)
    and the swept-AABB / capsule bounds (geometry/proxy.cpp:70-131), then
    ValidateProxyScene's slab partition (proxy_scene.cpp:58-85).  Python
    floats and the math module (the C library's acos/sin/cos)."""
    if int(inp["query_id"]) == 0:
        raise ValueError("ProxySceneBuildInput.query_id is required")
    if not inp["objects"]:
        raise ValueError("ProxySceneBuildInput.objects is empty")
    rows = []
    for o in inp["objects"]:
        if o["proxy_type"] not in (1, 2):
            raise ValueError("ProxyObjectBuildInput.proxy_type must be concrete")
        if len(o["patch_id"]) == 0:
            raise ValueError("ProxyObjectBuildInput.patches is empty")
        if len(o["segments"]) == 0:
            raise ValueError("ProxyObjectBuildInput.motion_segments is empty")
        S = int(o["slabs_per_motion_segment"])
        if S == 0:
            raise ValueError("slabs_per_motion_segment must be positive")
        eps = float(o["eps_proxy"])
        if not math.isfinite(eps) or eps < 0.0:
            raise ValueError("eps_proxy must be finite and non-negative")
        for si, seg in enumerate(np.asarray(o["segments"], np.float64).reshape(-1, 16).tolist()):
            st0, st1 = seg[0], seg[1]
            if not (math.isfinite(st0) and math.isfinite(st1)) or st0 >= st1:
                raise ValueError("motion segment must satisfy finite t0 < t1")
            for name, tr, rot in (("pose_t0", seg[2:5], seg[5:9]), ("pose_t1", seg[9:12], seg[12:16])):
                if not all(math.isfinite(x) for x in tr):
                    raise ValueError(f"{name}.translation contains a non-finite value")
                _norm4(rot)
            dt = (st1 - st0) / float(S)
            for k in range(S):
                t0 = st0 if k == 0 else st0 + dt * k
                t1 = st1 if k + 1 == S else st0 + dt * (k + 1)
                if not (math.isfinite(t0) and math.isfinite(t1)) or t0 >= t1:
                    raise ValueError("time slab must satisfy finite t0 < t1")
                tol = 1.0e-12 * max(1.0, st1 - st0)
                if t0 < st0 - tol or t1 > st1 + tol:
                    raise ValueError("time slab must lie inside the motion segment")
                poses = []
                for t in (t0, t1):
                    alpha = (_clamp(t, st0, st1) - st0) / (st1 - st0)
                    tr = [(1.0 - alpha) * seg[2 + a] + alpha * seg[9 + a] for a in range(3)]
                    rot = _slerp(_norm4(seg[5:9]), _norm4(seg[12:16]), alpha)
                    if not all(math.isfinite(x) for x in tr):
                        raise ValueError("pose.translation contains a non-finite value")
                    poses.append((tr, _norm4(rot)))
                (tr0, q0), (tr1, q1) = poses
                d = _clamp(abs(q0[0] * q1[0] + q0[1] * q1[1] + q0[2] * q1[2] + q0[3] * q1[3]), 0.0, 1.0)
                angle = 2.0 * math.acos(d)
                dx, dy, dz = tr0[0] - tr1[0], tr0[1] - tr1[1], tr0[2] - tr1[2]
                tb = math.sqrt(dx * dx + dy * dy + dz * dz)
                hs = math.sin(0.5 * angle)
                for p_id, lc, rad in zip(np.asarray(o["patch_id"]).tolist(),
                                         np.asarray(o["local_center"], np.float64).reshape(-1, 3).tolist(),
                                         np.asarray(o["radius"], np.float64).tolist()):
                    if not all(math.isfinite(x) for x in lc):
                        raise ValueError("patch.local_center contains a non-finite value")
                    if not math.isfinite(rad) or rad < 0.0:
                        raise ValueError("patch.radius must be finite and non-negative")
                    c0 = [x + y for x, y in zip(_rotate(q0, lc), tr0)]
                    c1 = [x + y for x, y in zip(_rotate(q1, lc), tr1)]
                    crb = 2.0 * math.sqrt(lc[0] * lc[0] + lc[1] * lc[1] + lc[2] * lc[2]) * hs
                    srb = 2.0 * rad * hs
                    cons = rad + crb
                    lo = [c1[a] if c1[a] < c0[a] else c0[a] for a in range(3)]  # std::min(c0, c1)
                    hi = [c1[a] if c0[a] < c1[a] else c0[a] for a in range(3)]  # std::max(c0, c1)
                    if o["proxy_type"] == 1:
                        mn = [lo[a] - cons for a in range(3)]
                        mx = [hi[a] + cons for a in range(3)]
                        _check_aabb(mn, mx, "AABB contains a non-finite bound", "AABB min cannot exceed max")
                        mn = [x - eps for x in mn]
                        mx = [x + eps for x in mx]
                        cap_r = 0.0
                    else:
                        if not math.isfinite(cons) or cons < 0.0:
                            raise ValueError("capsule radius must be finite and non-negative")
                        cap_r = cons + eps
                        mn = [lo[a] - cap_r for a in range(3)]
                        mx = [hi[a] + cap_r for a in range(3)]
                    _check_aabb(mn, mx, "proxy bounds contain a non-finite value",
                                "proxy bounds min cannot exceed max")
                    rows.append((o["object_id"], p_id, si * S + k, si, o["proxy_type"], t0, t1, mn + mx,
                                 [tb, angle, tb + crb + srb, cons], c0 + c1 + [crb, srb], cap_r))
    # ValidateGlobalSlabPartition (proxy_scene.cpp:58-85)
    first = {}
    for r in rows:
        a, b = first.setdefault(r[2], (r[5], r[6]))
        tol = 1.0e-12 * max(1.0, abs(a), abs(b), abs(b - a))
        if not abs(a - r[5]) <= tol or not abs(b - r[6]) <= tol:
            raise ValueError("proxy scene slab_id must map to one global time interval")
    ordered = sorted(first.items(), key=lambda kv: (kv[1][0], kv[0]))
    for (_, (a0, a1)), (_, (b0, b1)) in zip(ordered, ordered[1:]):
        tol = max(1.0e-12 * max(1.0, abs(a0), abs(a1), abs(a1 - a0)),
                  1.0e-12 * max(1.0, abs(b0), abs(b1), abs(b1 - b0)))
        if a0 < b1 - tol and b0 < a1 - tol:
            raise ValueError("proxy scene global slab intervals must not overlap")
    n = len(rows)
    out = {"query_id": int(inp["query_id"]), "n": n}
    for j, (k, dt_, sh) in enumerate(BUILT_FIELDS):
        out[k] = np.array([r[j] for r in rows], dt_).reshape((n,) + sh)
    return out



# ---- proposal feature rows (proposal/proposal_features.cpp) ----

def ref_proposal_feature_rows(sc: dict):
    """The reference's ComputeCandidateDensityStats and ExtractProposalFeatureRows
    for the candidates of a proxy scene: (density record, feature rows)."""
    from p2cccd_b200.records import DENSITY_DTYPE, FEATURE_ROW_DTYPE

    R = ref()
    if not hasattr(R, "_rows_ready"):
        vp, i64 = ctypes.c_void_p, ctypes.c_int64
        R.ref_proposal_feature_rows.argtypes = [ctypes.c_uint64, i64] + [vp] * 8 + [vp, vp, i64, vp]
        R.ref_proxy_last_error.restype = ctypes.c_char_p
        R._rows_ready = True
    a = _proxy_args(sc)
    args = [int(sc["query_id"]), int(sc["n"])] + [_p(a[k]) for k in ("object_id", "patch_id", "slab_id",
                                                                      "proxy_type", "t0", "t1", "bounds",
                                                                      "motion_bound")]
    dens = np.zeros(1, DENSITY_DTYPE)
    n_rows = ctypes.c_int64(0)
    if R.ref_proposal_feature_rows(*args, _p(dens), None, 0, ctypes.byref(n_rows)):
        raise ValueError(R.ref_proxy_last_error().decode())
    rows = np.zeros(max(1, n_rows.value), FEATURE_ROW_DTYPE)
    R.ref_proposal_feature_rows(*args, _p(dens), _p(rows), n_rows.value, ctypes.byref(n_rows))
    return dens[0], rows[:n_rows.value]


def candidate_density(sc: dict, raw, cand):
    """Restatement of ComputeCandidateDensityStats (candidate_stats.cpp:128-170,
    pair count :31-43 by its definition) without timing / backend name."""
    from p2cccd_b200.records import DENSITY_DTYPE

    n = int(sc["n"])
    obj, slab = np.asarray(sc["object_id"]), np.asarray(sc["slab_id"])
    pairs = 0
    for s_id in np.unique(slab):
        o = obj[slab == s_id]
        _, per = np.unique(o, return_counts=True)
        m = len(o)
        pairs += m * (m - 1) // 2 - int((per * (per - 1) // 2).sum())
    def ratio(x, y):
        return float(x) / float(y) if y else 0.0
    d = np.zeros(1, DENSITY_DTYPE)[0]
    d["query_id"], d["proxy_count"] = int(sc["query_id"]), n
    d["object_count"], d["slab_count"] = len(np.unique(obj)), len(np.unique(slab))
    d["cross_object_same_slab_pair_count"] = pairs
    d["raw_hit_count"], d["compact_candidate_count"] = len(raw), len(cand)
    d["raw_hits_per_proxy"] = ratio(len(raw), n)
    d["candidates_per_proxy"] = ratio(len(cand), n)
    d["candidates_per_slab"] = ratio(len(cand), d["slab_count"])
    d["aabb_overlap_ratio"] = ratio(len(raw), pairs)
    d["avg_rt_hits_per_candidate"] = ratio(int(cand["rt_hit_count"].astype(np.uint64).sum()) if len(cand) else 0,
                                           len(cand))
    return d


def _clamp_feature(v: float) -> np.float32:
    """ClampFeature (proposal_features.cpp:82-88)."""
    if not math.isfinite(v):
        return np.float32(0.0)
    return np.float32(-1.0e6 if v < -1.0e6 else (1.0e6 if 1.0e6 < v else v))


def proposal_feature_rows(sc: dict, cand, density):
    """Restatement of ExtractProposalFeatureRows / FillFeatureRow
    (proposal_features.cpp:122-205, 236-259): per candidate, the first proxy
    (in scene order) matching each side's (slab, object, patch, type), then
    the 32 features and the targets."""
    from p2cccd_b200.records import FEATURE_ROW_DTYPE

    a = _proxy_args(sc)
    first = {}
    for i in range(int(sc["n"])):
        key = (int(a["slab_id"][i]), int(a["object_id"][i]), int(a["patch_id"][i]), int(a["proxy_type"][i]))
        first.setdefault(key, i)
    rows = np.zeros(len(cand), FEATURE_ROW_DTYPE)
    ext = lambda b, k: max(0.0, b[3 + k] - b[k])
    vol = lambda b: ext(b, 0) * ext(b, 1) * ext(b, 2)
    def area(b):
        x, y, z = ext(b, 0), ext(b, 1), ext(b, 2)
        return 2.0 * (x * y + y * z + z * x)
    def ov(l, r, k):
        return max(0.0, min(l[3 + k], r[3 + k]) - max(l[k], r[k]))
    for r, c in zip(rows, cand):
        if not (c["schema_version"] == 1 and c["candidate_id"] and c["query_id"] and c["proxy_type_a"] in (1, 2)
                and c["proxy_type_b"] in (1, 2) and c["rt_hit_count"]):
            raise ValueError("invalid CandidateRecord")
        ia = first.get((int(c["slab_id"]), int(c["object_a_id"]), int(c["patch_a_id"]), int(c["proxy_type_a"])))
        ib = first.get((int(c["slab_id"]), int(c["object_b_id"]), int(c["patch_b_id"]), int(c["proxy_type_b"])))
        if ia is None or ib is None:
            raise ValueError("candidate does not map to proxy primitives")
        A, B = a["bounds"][ia].tolist(), a["bounds"][ib].tolist()
        ma, mb = a["motion_bound"][ia].tolist(), a["motion_bound"][ib].tolist()
        t0, t1 = float(a["t0"][ia]), float(a["t1"][ia])
        va, vb = vol(A), vol(B)
        ovol = ov(A, B, 0) * ov(A, B, 1) * ov(A, B, 2)
        uvol = max(0.0, va + vb - ovol)
        ca = [0.5 * (A[k] + A[3 + k]) for k in range(3)]
        cb = [0.5 * (B[k] + B[3 + k]) for k in range(3)]
        dx, dy, dz = ca[0] - cb[0], ca[1] - cb[1], ca[2] - cb[2]
        mbc = [float(x) for x in c["motion_bound"]]
        f = [t0, t1, max(0.0, t1 - t0), float(c["rt_hit_count"]), float(c["proxy_type_a"]),
             float(c["proxy_type_b"]), *mbc, ext(A, 0), ext(A, 1), ext(A, 2), ext(B, 0), ext(B, 1), ext(B, 2),
             va, vb, ovol, ovol / uvol if uvol > 0.0 else 0.0, math.sqrt(dx * dx + dy * dy + dz * dz), area(A),
             area(B), ma[3], mb[3], ma[0], mb[0], ma[1], mb[1], float(density["candidates_per_proxy"]),
             float(density["aabb_overlap_ratio"]), float(density["avg_rt_hits_per_candidate"])]
        feats = np.array([_clamp_feature(v) for v in f], np.float32)
        r["schema_version"], r["query_id"], r["candidate_id"] = 1, c["query_id"], c["candidate_id"]
        for k in ("slab_id", "object_a_id", "patch_a_id", "object_b_id", "patch_b_id"):
            r[k] = c[k]
        r["features"] = feats
        center = 0.5 * (t0 + t1)
        center = 0.0 if center < 0.0 else (math.nextafter(1.0, 0.0) if math.nextafter(1.0, 0.0) < center else center)
        r["interval_targets"][int(center * 8)] = 1.0
        r["family_targets"][0] = r["family_targets"][1] = 1.0
        r["priority_target"] = _clamp_feature(0.5 * float(c["rt_hit_count"]) +
                                              0.5 * float(density["candidates_per_proxy"]))
        r["cost_target"] = _clamp_feature(1.0 + mbc[3])
        r["uncertainty_target"] = _clamp_feature(1.0 - min(1.0, float(feats[19])))
        r["target_mask"] = 31
    return rows



def ref_runtime_feature_rows(cand, primitive_count: int, raw_hit_count: int, compact_candidate_count: int,
                             masks: dict | None = None):
    """The reference's BuildProposalFeatureRowsFromRuntimeCandidates (with the
    binding's MakeRuntimeDensityStats) on CANDIDATE_RECORD_DTYPE records."""
    from p2cccd_b200.records import FEATURE_ROW_DTYPE

    R = ref()
    if not hasattr(R, "_rt_rows_ready"):
        vp, i64, u64 = ctypes.c_void_p, ctypes.c_int64, ctypes.c_uint64
        R.ref_runtime_feature_rows.argtypes = [vp, i64, u64, u64, u64, vp, vp, i64, vp]
        R.ref_proxy_last_error.restype = ctypes.c_char_p
        R._rt_rows_ready = True
    cand = np.ascontiguousarray(cand)
    keys = np.array(sorted((masks or {}).keys()), np.uint64)
    vals = np.array([masks[int(k)] for k in keys], np.uint32)
    rows = np.zeros(max(1, len(cand)), FEATURE_ROW_DTYPE)
    if R.ref_runtime_feature_rows(_p(cand), len(cand), primitive_count, raw_hit_count, compact_candidate_count,
                                  _p(keys) if len(keys) else None, _p(vals) if len(vals) else None, len(keys),
                                  _p(rows)):
        raise ValueError(R.ref_proxy_last_error().decode())
    return rows[:len(cand)]


def runtime_feature_rows(cand, primitive_count: int, raw_hit_count: int, compact_candidate_count: int,
                         masks: dict | None = None):
    """Restatement of BuildRuntimeFeatureRowFromDerived (proposal_policy.cpp:
    184-226) with MakeRuntimeDensityDerivedStats (:44-58)."""
    from p2cccd_b200.records import FEATURE_ROW_DTYPE

    if primitive_count == 0:
        raise ValueError("CandidateDensityStats.proxy_count must be non-zero")
    def ratio(x, y):
        return float(x) / float(y) if y else 0.0
    cpp = ratio(compact_candidate_count, primitive_count)
    aor = ratio(raw_hit_count, primitive_count // 2 if primitive_count >= 2 else 1)
    avg = ratio(raw_hit_count, compact_candidate_count)
    rows = np.zeros(len(cand), FEATURE_ROW_DTYPE)
    for r, c in zip(rows, cand):
        if not (c["schema_version"] == 1 and c["candidate_id"] and c["query_id"] and c["proxy_type_a"] in (1, 2)
                and c["proxy_type_b"] in (1, 2) and c["rt_hit_count"]
                and all(math.isfinite(float(x)) and x >= 0 for x in c["motion_bound"])):
            raise ValueError("invalid CandidateRecord")
        mask = (masks or {}).get(int(c["query_id"]), 0) or 3
        for k in ("query_id", "candidate_id", "slab_id", "object_a_id", "patch_a_id", "object_b_id", "patch_b_id"):
            r[k] = c[k]
        r["schema_version"] = 1
        rt = float(c["rt_hit_count"])
        f = np.zeros(32, np.float32)
        f[1] = f[2] = 1.0
        f[3], f[4], f[5] = _clamp_feature(rt), _clamp_feature(float(c["proxy_type_a"])), \
            _clamp_feature(float(c["proxy_type_b"]))
        for k in range(4):
            f[6 + k] = _clamp_feature(float(c["motion_bound"][k]))
        f[19] = _clamp_feature(min(1.0, aor))
        f[29], f[30], f[31] = _clamp_feature(cpp), _clamp_feature(aor), _clamp_feature(avg)
        r["features"] = f
        r["interval_targets"][0] = 1.0
        r["family_targets"][0] = 1.0 if mask & 1 else 0.0
        r["family_targets"][1] = 1.0 if mask & 2 else 0.0
        r["priority_target"] = _clamp_feature(min(1.0, 0.5 * rt + 0.5 * cpp))
        r["cost_target"] = _clamp_feature(max(1.0, 1.0 + rt))
        r["uncertainty_target"] = 0.25 if mask == 3 else 0.0
        r["target_mask"] = 31
    return rows



# ---- exact work queue audit rows (certificate_engine.cpp:593-661) ----

def ref_process_queue(items, pts, pt_off, ees, ee_off, eps_time=1e-6, eps_space=1e-6, max_depth=32,
                      first_event_id=1, first_timestamp_us=1, emit_dequeue=True):
    """The reference's ProcessExactWorkQueueCpu: (certificates as QUERY_CERT
    records, audit rows as AUDIT_ROW_DTYPE records)."""
    from p2cccd_b200.records import AUDIT_ROW_DTYPE

    R = ref()
    if not hasattr(R, "_queue_ready"):
        vp, i64 = ctypes.c_void_p, ctypes.c_int64
        R.ref_process_queue.argtypes = [vp, i64, vp, vp, vp, vp, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                        ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int, vp, vp, vp]
        R._queue_ready = True
    items = np.ascontiguousarray(items)
    n = len(items)
    certs = np.zeros(max(n, 1), QUERY_CERT)
    rows = np.zeros(max(2 * n, 1), AUDIT_ROW_DTYPE)
    n_rows = ctypes.c_int64(0)
    a, b = np.ascontiguousarray(pts), np.ascontiguousarray(ees)
    po, eo = np.ascontiguousarray(pt_off, np.int64), np.ascontiguousarray(ee_off, np.int64)
    if R.ref_process_queue(_p(items), n, _p(a), _p(po), _p(b), _p(eo), eps_time, eps_space, max_depth,
                           first_event_id, first_timestamp_us, 1 if emit_dequeue else 0, _p(certs), _p(rows),
                           ctypes.byref(n_rows)):
        raise ValueError(ref().ref_last_error().decode())
    return certs[:n], rows[:n_rows.value]


def audit_rows(items, certs, first_event_id=1, first_timestamp_us=1, emit_dequeue=True):
    """Restatement of the audit rows of ProcessExactWorkQueueCpu (:593-661,
    MakeAuditRow :456-477, AuditActionForCertificate :443-454)."""
    from p2cccd_b200.records import AUDIT_ROW_DTYPE

    rows = []
    ev, ts = int(first_event_id), int(first_timestamp_us)
    for it, c in zip(items, certs):
        def row(stage, action, aux0, aux1):
            return (ev, it["query_id"], it["candidate_id"], it["work_item_id"], stage, action, it["depth"],
                    it["interval_t0"], it["interval_t1"], ts, aux0, aux1)
        if emit_dequeue:
            rows.append(row(2, 1, float(it["priority_score"]), float(it["feature_family_mask"])))
            ev, ts = ev + 1, ts + 1
        st = int(c["status"])
        action = 2 if st == 0 else (3 if st == 1 else (5 if int(c["reason_code"]) == 3 else 4))
        rows.append(row(4, action, float(c["safe_margin_lb"] if st == 1 else c["toi_upper"]),
                        float(c["next_refinement_mode"])))
        ev, ts = ev + 1, ts + 1
    out = np.zeros(len(rows), AUDIT_ROW_DTYPE)
    for o, r in zip(out, rows):
        for k, v in zip(AUDIT_ROW_DTYPE.names, r):
            o[k] = v
    return out



# ---- runtime exact work queue from proposals (proposal_policy.cpp:595-742) ----

SCHED_DEFAULTS = dict(first_work_item_id=1, conservative_feature_family_mask=3, fallback_interval_t0=0.0,
                      fallback_interval_t1=1.0, family_score_threshold=0.5, uncertainty_fallback_threshold=0.95,
                      ood_abs_feature_threshold=1.0e5, preserve_candidate_order=False)


def ref_schedule_runtime(cand, rows, outs, masks=None, **cfg):
    """The reference's ScheduleRuntimeExactWorkItemsFromProposals: (work items
    as EXACT_WORK_ITEM_DTYPE records, stats as SCHEDULE_STATS_DTYPE)."""
    from p2cccd_b200.records import EXACT_WORK_ITEM_DTYPE, SCHEDULE_STATS_DTYPE

    c = dict(SCHED_DEFAULTS, **cfg)
    R = ref()
    if not hasattr(R, "_sched_ready"):
        vp, i64, f32, f64 = ctypes.c_void_p, ctypes.c_int64, ctypes.c_float, ctypes.c_double
        R.ref_schedule_runtime.argtypes = [vp, i64, vp, i64, vp, i64, vp, vp, i64, ctypes.c_uint64, ctypes.c_uint32,
                                           f64, f64, f32, f32, f32, ctypes.c_int, vp, vp]
        R.ref_proxy_last_error.restype = ctypes.c_char_p
        R._sched_ready = True
    cand, rows, outs = (np.ascontiguousarray(x) for x in (cand, rows, outs))
    keys = np.array(sorted((masks or {}).keys()), np.uint64)
    vals = np.array([masks[int(k)] for k in keys], np.uint32)
    items = np.zeros(max(1, len(cand)), EXACT_WORK_ITEM_DTYPE)
    stats = np.zeros(1, SCHEDULE_STATS_DTYPE)
    if R.ref_schedule_runtime(_p(cand), len(cand), _p(rows), len(rows), _p(outs), len(outs),
                              _p(keys) if len(keys) else None, _p(vals) if len(vals) else None, len(keys),
                              c["first_work_item_id"], c["conservative_feature_family_mask"],
                              c["fallback_interval_t0"], c["fallback_interval_t1"], c["family_score_threshold"],
                              c["uncertainty_fallback_threshold"], c["ood_abs_feature_threshold"],
                              1 if c["preserve_candidate_order"] else 0, _p(items), _p(stats)):
        raise ValueError(R.ref_proxy_last_error().decode())
    return items[:len(cand)], stats[0]


def schedule_runtime(cand, rows, outs, masks=None, mode=0, **cfg):
    """Restatement of ScheduleRuntimeExactWorkItemsFromProposals
    (proposal_policy.cpp:595-742; mode 0) and of the binding's aligned-array
    form (py_module.cpp:1088-1174; mode 1: rows / outputs paired by position,
    candidate fields from the row, fallback priority features[3]).  Returns
    (work items, stats) or raises ValueError."""
    from p2cccd_b200.records import EXACT_WORK_ITEM_DTYPE, SCHEDULE_STATS_DTYPE

    c = dict(SCHED_DEFAULTS, **cfg)
    f32 = np.float32
    def fin(x):
        return bool(np.isfinite(x))
    def invalid(o):
        vals = list(o["interval_scores"]) + list(o["family_scores"]) + [o["priority_score"], o["cost_score"],
                                                                       o["uncertainty_score"]]
        return int(o["candidate_id"]) == 0 or not all(fin(v) for v in vals) or o["cost_score"] < 0 or \
            o["uncertainty_score"] < 0
    def ood(r):
        return r is None or any((not fin(v)) or abs(f32(v)) > f32(c["ood_abs_feature_threshold"]) for v in r["features"])
    n = len(cand) if mode == 0 else len(rows)
    if mode == 0:
        rows_by = {}
        for r in rows:
            if int(r["candidate_id"]) == 0 or int(r["candidate_id"]) in rows_by:
                raise ValueError("proposal feature row candidate_id zero or repeated")
            rows_by[int(r["candidate_id"])] = r
        outs_by = {}
        for o in outs:
            if int(o["candidate_id"]) == 0 or int(o["candidate_id"]) in outs_by:
                raise ValueError("proposal output candidate_id zero or repeated")
            outs_by[int(o["candidate_id"])] = o
    stats = np.zeros(1, SCHEDULE_STATS_DTYPE)[0]
    items = np.zeros(n, EXACT_WORK_ITEM_DTYPE)
    for i in range(n):
        if mode == 0:
            cd = cand[i]
            ok = cd["schema_version"] == 1 and cd["candidate_id"] and cd["query_id"] and \
                cd["proxy_type_a"] in (1, 2) and cd["proxy_type_b"] in (1, 2) and cd["rt_hit_count"] and \
                all(fin(v) and v >= 0 for v in cd["motion_bound"])
            if not ok:
                raise ValueError("invalid CandidateRecord")
            src = cd
            r, o = rows_by.get(int(cd["candidate_id"])), outs_by.get(int(cd["candidate_id"]))
            fb_prio = f32(int(cd["rt_hit_count"]))
        else:
            r, o = rows[i], outs[i]
            if int(r["candidate_id"]) == 0 or int(o["candidate_id"]) != int(r["candidate_id"]):
                raise ValueError("proposal arrays must preserve candidate_id order")
            src = r
            fb_prio = f32(r["features"][3])
        miss = o is None
        inv = not miss and invalid(o)
        od = ood(r)
        unc = not miss and fin(o["uncertainty_score"]) and f32(o["uncertainty_score"]) >= f32(c["uncertainty_fallback_threshold"])
        fb = miss or inv or od or unc
        stats["fallback_count"] += fb
        stats["missing_proposal_fallback_count"] += miss
        stats["invalid_proposal_fallback_count"] += inv
        stats["ood_fallback_count"] += od
        stats["high_uncertainty_fallback_count"] += unc
        base = (masks or {}).get(int(src["query_id"]), 0) or c["conservative_feature_family_mask"]
        it = items[i]
        it["parent_candidate_id"], it["query_id"] = src["candidate_id"], src["query_id"]
        it["slab_id"], it["patch_a_id"], it["patch_b_id"] = src["slab_id"], src["patch_a_id"], src["patch_b_id"]
        it["interval_t0"], it["interval_t1"] = c["fallback_interval_t0"], c["fallback_interval_t1"]
        it["feature_family_mask"], it["priority_score"], it["source"] = base, fb_prio, 2
        if not fb:
            pred = (1 if f32(o["family_scores"][0]) >= f32(c["family_score_threshold"]) else 0) | \
                (2 if f32(o["family_scores"][1]) >= f32(c["family_score_threshold"]) else 0)
            it["feature_family_mask"], it["priority_score"], it["source"] = base | pred, o["priority_score"], 1
    if not c["preserve_candidate_order"]:
        order = sorted(range(n), key=lambda k: -float(items[k]["priority_score"]))  # stable
        items = items[order]
    originals = (cand if mode == 0 else rows)["candidate_id"]
    for i in range(n):
        items[i]["work_item_id"] = c["first_work_item_id"] + i
        stats["reordered_count"] += int(items[i]["parent_candidate_id"] != originals[i])
        if not (items[i]["parent_candidate_id"] and items[i]["query_id"] and items[i]["feature_family_mask"]
                and fin(items[i]["priority_score"])):
            raise ValueError("invalid ExactWorkItem")
    if mode == 0:
        if len(set(int(x) for x in cand["candidate_id"])) != n:
            raise ValueError("runtime candidates contain duplicate candidate_id")
        for it in items:
            if not int(it["feature_family_mask"]) & 3 or int(it["feature_family_mask"]) & 0xFFFFFFFC:
                raise ValueError("runtime scheduled work item family bits")
    stats["raw_candidate_count"], stats["proposal_output_count"], stats["work_item_count"] = n, len(outs), n
    stats["monotonic_safe"] = 1
    clean = np.zeros(n, EXACT_WORK_ITEM_DTYPE)  # zero padding between the fields
    for k in EXACT_WORK_ITEM_DTYPE.names:
        clean[k] = items[k]
    return clean, stats



# ---- external batch candidates (rt_candidate/external_batch_candidate.cpp) ----

def _external_args(batch: dict):
    n = len(batch["query_id"])
    return (n, np.ascontiguousarray(batch["query_id"], np.uint64),
            np.ascontiguousarray(batch["source_query_index"], np.uint32),
            np.ascontiguousarray(batch["family"], np.uint8),
            np.ascontiguousarray(batch["vertices_t0"], np.float64).reshape(n, 12),
            np.ascontiguousarray(batch["vertices_t1"], np.float64).reshape(n, 12),
            np.ascontiguousarray(batch["ground_truth"], np.int8), np.ascontiguousarray(batch["has_box"], np.uint8),
            np.ascontiguousarray(batch["box_pair"], np.uint32).reshape(n, 2))


def ref_external_batch(batch: dict):
    """The reference's GenerateCandidatesForExternalBatch: (candidates,
    runtime query ids, counts {primitives, raw hits, candidates}, recall)."""
    from p2cccd_b200.records import CANDIDATE_RECORD_DTYPE

    R = ref()
    if not hasattr(R, "_ext_ready"):
        vp = ctypes.c_void_p
        R.ref_external_batch.argtypes = [ctypes.c_int64] + [vp] * 12
        R.ref_proxy_last_error.restype = ctypes.c_char_p
        R._ext_ready = True
    a = _external_args(batch)
    n = a[0]
    cand = np.zeros(max(1, n), CANDIDATE_RECORD_DTYPE)
    rid = np.zeros(max(1, n), np.uint64)
    counts = np.zeros(3, np.uint64)
    recall = np.zeros(1, np.float64)
    if R.ref_external_batch(n, *[_p(x) for x in a[1:]], _p(cand), _p(rid), _p(counts), _p(recall)):
        raise ValueError(R.ref_proxy_last_error().decode())
    cand = cand[:int(counts[2])]
    clean = np.zeros(len(cand), cand.dtype)  # the reference struct's padding bytes are indeterminate
    for f in cand.dtype.names:
        clean[f] = cand[f]
    return clean, rid[:n], counts, float(recall[0])


# ---- candidate-group early-stop replay (common/group_scheduler.cpp) ----

DENSE_KEYS = ("query_id", "candidate_id", "cost_target", "oracle_trace", "interval_scores", "priority_score",
              "cost_score", "uncertainty_score")


def _dense_arrays(rows: dict):
    return (np.ascontiguousarray(rows["query_id"], np.uint64), np.ascontiguousarray(rows["candidate_id"], np.uint64),
            np.ascontiguousarray(rows["cost_target"], np.float32),
            np.ascontiguousarray(rows["oracle_trace"], np.float64).reshape(-1, 8),
            np.ascontiguousarray(rows["interval_scores"], np.float32).reshape(-1, 8),
            np.ascontiguousarray(rows["priority_score"], np.float32),
            np.ascontiguousarray(rows["cost_score"], np.float32),
            np.ascontiguousarray(rows["uncertainty_score"], np.float32))


def ref_dense_group(rows: dict, threshold=0.75, limit=3, penalty=0.22, preserve=False) -> np.ndarray:
    """The reference's RunDenseGroupExactEarlyStop on rows parsed as its
    binding parses them: one DENSE_GROUP_STATS_DTYPE record."""
    from p2cccd_b200.records import DENSE_GROUP_STATS_DTYPE

    R = ref()
    if not hasattr(R, "_dense_ready"):
        vp = ctypes.c_void_p
        R.ref_dense_group.argtypes = [ctypes.c_int64] + [vp] * 8 + [ctypes.c_float, ctypes.c_uint32, ctypes.c_double,
                                                                    ctypes.c_int, vp]
        R.ref_proxy_last_error.restype = ctypes.c_char_p
        R._dense_ready = True
    a = _dense_arrays(rows)
    out = np.zeros(1, DENSE_GROUP_STATS_DTYPE)
    if R.ref_dense_group(len(a[0]), *[_p(x) for x in a], float(np.float32(threshold)), int(limit), float(penalty),
                         int(bool(preserve)), _p(out)):
        raise ValueError(R.ref_proxy_last_error().decode())
    return out[0]


def dense_group(rows: dict, threshold=0.75, limit=3, penalty=0.22, preserve=False) -> dict:
    """Restatement of RunDenseGroupExactEarlyStop (group_scheduler.cpp:60-239)
    after the binding's parse (py_module.cpp:1212-1244), in plain Python over
    the rows: the same order (stable by query id, then priority desc, cost
    asc, index) and the same additions in the same order."""
    qid, cid, ct, tr, isc, pr, cs, unc = _dense_arrays(rows)
    n = len(qid)
    thr = np.float32(threshold)
    if limit == 0:
        raise ValueError("representative_attempt_limit must be positive")
    if not np.isfinite(thr) or thr < 0:
        raise ValueError("uncertainty_fallback_threshold must be finite and non-negative")
    if not math.isfinite(penalty) or penalty < 0:
        raise ValueError("interval_miss_penalty_scale must be finite and non-negative")
    cand = []
    for i in range(n):
        best, bs = 0, isc[i, 0]
        for k in range(1, 8):
            if isc[i, k] > bs:
                best, bs = k, isc[i, k]
        full = float(tr[i, 5])
        ratio = float(ct[i])
        narrow = max(1e-12, full * ratio) if (math.isfinite(ratio) and ratio > 0.0) else full
        t0 = 0.125 * best
        t1 = min(1.0, t0 + 0.125)
        cand.append(dict(q=int(qid[i]), c=int(cid[i]), full=full, narrow=narrow, t0=t0, t1=t1, c0=float(tr[i, 6]),
                         c1=float(tr[i, 7]), pr=np.float32(pr[i]), cs=np.float32(cs[i]), unc=np.float32(unc[i]),
                         coll=bool(tr[i, 0] > 0.5)))
    for c in cand:
        if c["q"] == 0 or c["c"] == 0:
            raise ValueError("dense group candidate ids must be non-zero")
        if not all(math.isfinite(float(c[k])) for k in ("full", "narrow", "t0", "t1", "c0", "c1", "pr", "cs", "unc")):
            raise ValueError("dense group candidate contains a non-finite field")

    def pos_cost(v, fb):
        return fb if (not math.isfinite(v) or v <= 0.0) else v

    if preserve:
        order = sorted(range(n), key=lambda i: (cand[i]["q"], i))
    else:  # -0 == +0 in float comparisons; Python's sort is stable
        order = sorted(range(n), key=lambda i: (cand[i]["q"], -float(cand[i]["pr"]), float(cand[i]["cs"]), i))
    out = dict(candidate_count=n, group_count=0, positive_group_count=0, no_proposal_exact_calls=0,
               no_proposal_exact_work=0.0, learned_exact_calls=0, learned_fallback_calls=0,
               learned_interval_hit_count=0, learned_interval_miss_count=0, learned_exact_work=0.0,
               first_positive_rank_sum=0.0, cost_before_first_positive_sum=0.0, tp=0, tn=0, fp=0, fn=0,
               reordered_count=sum(1 for i, o in enumerate(order) if o != i), high_uncertainty_group_count=0)
    b = 0
    while b < n:
        e = b + 1
        while e < n and cand[order[e]]["q"] == cand[order[b]]["q"]:
            e += 1
        out["group_count"] += 1
        truth, gwork = False, 0.0
        for p in range(b, e):
            c = cand[order[p]]
            truth = truth or c["coll"]
            gwork += pos_cost(c["full"], 1.0)
        out["positive_group_count"] += truth
        out["no_proposal_exact_calls"] += e - b
        out["no_proposal_exact_work"] += gwork
        predicted, resolved, high, wb = False, False, False, 0.0
        for p in range(b, e):
            c = cand[order[p]]
            full = pos_cost(c["full"], 1.0)
            nar = pos_cost(c["narrow"], full)
            if c["unc"] >= thr:
                high = True
                for fp in range(p, e):  # run_full_fallback
                    f = cand[order[fp]]
                    fc = pos_cost(f["full"], 1.0)
                    out["learned_exact_calls"] += 1
                    out["learned_fallback_calls"] += 1
                    out["learned_exact_work"] += fc
                    if f["coll"]:
                        predicted = True
                        out["first_positive_rank_sum"] += fp - b + 1
                        out["cost_before_first_positive_sum"] += wb + fc
                        break
                    wb += fc
                break
            out["learned_exact_calls"] += 1
            out["learned_exact_work"] += nar
            if c["coll"]:
                if max(c["t0"], c["c0"]) <= min(c["t1"], c["c1"]):
                    out["learned_interval_hit_count"] += 1
                    predicted = True
                    out["first_positive_rank_sum"] += p - b + 1
                    out["cost_before_first_positive_sum"] += wb + nar
                    break
                out["learned_interval_miss_count"] += 1
                out["learned_exact_work"] += full * penalty
                if p - b + 1 >= limit:
                    out["learned_exact_calls"] += 1
                    out["learned_fallback_calls"] += 1
                    out["learned_exact_work"] += full
                    predicted = True
                    out["first_positive_rank_sum"] += p - b + 1
                    out["cost_before_first_positive_sum"] += wb + nar + full
                    break
                wb += nar + full * penalty
                continue
            wb += nar
        out["high_uncertainty_group_count"] += high
        key = ("tp" if predicted else "fn") if truth else ("fp" if predicted else "tn")
        out[key] += 1
        b = e
    return out


# ---- dummy proposal schedules (proposal_policy.cpp:744-858, py_module.cpp:269-361) ----

def _sched_args(c: dict):
    return (c["first_work_item_id"], c["conservative_feature_family_mask"], c["fallback_interval_t0"],
            c["fallback_interval_t1"], c["family_score_threshold"], c["uncertainty_fallback_threshold"],
            c["ood_abs_feature_threshold"], 1 if c["preserve_candidate_order"] else 0)


def _sched_argtypes():
    return [ctypes.c_uint64, ctypes.c_uint32, ctypes.c_double, ctypes.c_double, ctypes.c_float, ctypes.c_float,
            ctypes.c_float, ctypes.c_int]


def _schedule_buffers(n: int):
    from p2cccd_b200.records import (EXACT_WORK_ITEM_DTYPE, FEATURE_ROW_DTYPE, PROPOSAL_OUTPUT_DTYPE,
                                     SCHEDULE_STATS_DTYPE)

    m = max(1, n)
    return (np.zeros(m, EXACT_WORK_ITEM_DTYPE), np.zeros(1, SCHEDULE_STATS_DTYPE), np.zeros(m, FEATURE_ROW_DTYPE),
            np.zeros(m, PROPOSAL_OUTPUT_DTYPE), np.zeros(4, np.int64))


def ref_dummy_schedule(cand, primitive_count, raw_hit_count, compact_candidate_count, masks=None, materialize=True,
                       **cfg):
    """The reference's RunDummyProposalScheduleFromRuntimeCandidates with the
    binding's density: (work items, stats, feature rows, proposal outputs)."""
    c = dict(SCHED_DEFAULTS, **cfg)
    R = ref()
    if not hasattr(R, "_dummy_ready"):
        vp, i64, u64 = ctypes.c_void_p, ctypes.c_int64, ctypes.c_uint64
        R.ref_dummy_schedule.argtypes = [vp, i64, u64, u64, u64, vp, vp, i64] + _sched_argtypes() + \
            [ctypes.c_int, vp, vp, vp, vp, vp]
        R.ref_proxy_last_error.restype = ctypes.c_char_p
        R._dummy_ready = True
    cand = np.ascontiguousarray(cand)
    keys = np.array(sorted((masks or {}).keys()), np.uint64)
    vals = np.array([masks[int(k)] for k in keys], np.uint32)
    items, stats, rows, outs, sizes = _schedule_buffers(len(cand))
    if R.ref_dummy_schedule(_p(cand), len(cand), int(primitive_count), int(raw_hit_count),
                            int(compact_candidate_count), _p(keys) if len(keys) else None,
                            _p(vals) if len(vals) else None, len(keys), *_sched_args(c), int(bool(materialize)),
                            _p(items), _p(stats), _p(rows), _p(outs), _p(sizes)):
        raise ValueError(R.ref_proxy_last_error().decode())
    return items[:sizes[0]], stats[0], rows[:sizes[1]], outs[:sizes[2]]


def ref_external_dummy(batch: dict, materialize=False, **cfg):
    """The binding's GenerateExternalBatchDummyProposalSchedule restated over
    the reference's functions: (candidates, work items, stats, rows, outputs)."""
    from p2cccd_b200.records import CANDIDATE_RECORD_DTYPE

    c = dict(SCHED_DEFAULTS, **cfg)
    R = ref()
    if not hasattr(R, "_ext_dummy_ready"):
        vp = ctypes.c_void_p
        R.ref_external_dummy.argtypes = [ctypes.c_int64] + [vp] * 8 + _sched_argtypes() + [ctypes.c_int] + [vp] * 6
        R.ref_proxy_last_error.restype = ctypes.c_char_p
        R._ext_dummy_ready = True
    a = _external_args(batch)
    n = a[0]
    cand = np.zeros(max(1, n), CANDIDATE_RECORD_DTYPE)
    items, stats, rows, outs, sizes = _schedule_buffers(n)
    if R.ref_external_dummy(n, *[_p(x) for x in a[1:]], *_sched_args(c), int(bool(materialize)), _p(cand),
                            _p(items), _p(stats), _p(rows), _p(outs), _p(sizes)):
        raise ValueError(R.ref_proxy_last_error().decode())
    clean = np.zeros(int(sizes[3]), CANDIDATE_RECORD_DTYPE)  # padding bytes of the reference struct are indeterminate
    for f in CANDIDATE_RECORD_DTYPE.names:
        clean[f] = cand[:int(sizes[3])][f]
    return clean, items[:sizes[0]], stats[0], rows[:sizes[1]], outs[:sizes[2]]


def dummy_schedule(cand, primitive_count, raw_hit_count, compact_candidate_count, masks=None, materialize=True,
                   **cfg):
    """Restatement of RunDummyProposalScheduleFromRuntimeCandidates
    (proposal_policy.cpp:744-858): runtime rows and dummy outputs, the OOD
    fallback, a stable priority sort, ids and checks."""
    from p2cccd_b200.records import EXACT_WORK_ITEM_DTYPE, PROPOSAL_OUTPUT_DTYPE, SCHEDULE_STATS_DTYPE

    c = dict(SCHED_DEFAULTS, **cfg)
    f32 = np.float32
    if primitive_count == 0:
        raise ValueError("CandidateDensityStats.proxy_count must be non-zero")
    def ratio(x, y):
        return float(x) / float(y) if y else 0.0
    cpp = ratio(compact_candidate_count, primitive_count)
    aor = ratio(raw_hit_count, primitive_count // 2 if primitive_count >= 2 else 1)
    avg = ratio(raw_hit_count, compact_candidate_count)
    thr = f32(c["ood_abs_feature_threshold"])
    rows = runtime_feature_rows(cand, primitive_count, raw_hit_count, compact_candidate_count, masks)
    n = len(cand)
    outs = np.zeros(n, PROPOSAL_OUTPUT_DTYPE)
    staged = np.zeros(n, EXACT_WORK_ITEM_DTYPE)
    stats = np.zeros(1, SCHEDULE_STATS_DTYPE)[0]
    for i, r in enumerate(cand):
        base = (masks or {}).get(int(r["query_id"]), 0) or 3
        scal = [1.0, float(r["rt_hit_count"]), float(r["proxy_type_a"]), float(r["proxy_type_b"]), min(1.0, aor),
                cpp, aor, avg]
        ood = any((not math.isfinite(v)) or abs(v) > float(thr) for v in scal) or \
            any((not np.isfinite(v)) or abs(f32(v)) > thr for v in r["motion_bound"])
        stats["fallback_count"] += ood
        stats["ood_fallback_count"] += ood
        act = [k for k in (0, 1) if base & (1 << k)] or [0, 1]
        w = f32(1.0) / f32(len(act))
        fam = [w if k in act else f32(0.0) for k in (0, 1)]
        row = rows[i]
        o = outs[i]
        o["candidate_id"] = r["candidate_id"]
        o["interval_scores"] = row["interval_targets"]
        o["family_scores"][0], o["family_scores"][1] = fam
        o["priority_score"] = max(f32(0.0), row["priority_target"])
        o["cost_score"] = max(f32(0.0), row["cost_target"])
        o["uncertainty_score"] = f32(1.0) if ood else max(f32(0.0), row["uncertainty_target"])
        it = staged[i]
        for k in ("query_id", "slab_id", "patch_a_id", "patch_b_id"):
            it[k] = r[k]
        it["parent_candidate_id"] = r["candidate_id"]
        it["interval_t0"], it["interval_t1"] = c["fallback_interval_t0"], c["fallback_interval_t1"]
        if ood:
            it["feature_family_mask"], it["priority_score"], it["source"] = base, f32(r["rt_hit_count"]), 2
        else:
            m = base | (1 if fam[0] >= f32(c["family_score_threshold"]) else 0) | \
                (2 if fam[1] >= f32(c["family_score_threshold"]) else 0)
            it["feature_family_mask"] = m
            it["priority_score"] = max(f32(0.0), _clamp_feature(min(1.0, 0.5 * float(r["rt_hit_count"]) + 0.5 * cpp)))
            it["source"] = 1
    order = list(range(n))
    if not c["preserve_candidate_order"]:
        order.sort(key=lambda i: -float(staged[i]["priority_score"]))  # stable
    items = staged[order]
    items["work_item_id"] = np.arange(n, dtype=np.uint64) + np.uint64(c["first_work_item_id"])
    stats["raw_candidate_count"] = stats["proposal_output_count"] = stats["work_item_count"] = n
    stats["reordered_count"] = int(np.sum(items["parent_candidate_id"] != np.asarray(cand["candidate_id"])))
    stats["monotonic_safe"] = 1
    clean = np.zeros(n, EXACT_WORK_ITEM_DTYPE)  # zero padding after the fancy-index copy
    for f in EXACT_WORK_ITEM_DTYPE.names:
        clean[f] = items[f]
    if not materialize:
        rows, outs = rows[:0], outs[:0]
    return clean, stats, rows, outs


def ref_compact_raw(sc: dict, raw):
    """The reference's CompactRawCandidates on given raw hits of a proxy scene."""
    from p2cccd_b200.records import CANDIDATE_RECORD_DTYPE, RAW_HIT_DTYPE

    R = ref()
    if not hasattr(R, "_compact_ready"):
        vp, i64 = ctypes.c_void_p, ctypes.c_int64
        R.ref_compact_raw.argtypes = [ctypes.c_uint64, i64] + [vp] * 8 + [vp, i64, vp, vp]
        R.ref_proxy_last_error.restype = ctypes.c_char_p
        R._compact_ready = True
    a = _proxy_args(sc)
    raw = np.ascontiguousarray(raw, dtype=RAW_HIT_DTYPE)
    cand = np.zeros(max(1, len(raw)), CANDIDATE_RECORD_DTYPE)
    n_cand = ctypes.c_int64(0)
    args = [int(sc["query_id"]), int(sc["n"])] + [_p(a[k]) for k in ("object_id", "patch_id", "slab_id", "proxy_type",
                                                                     "t0", "t1", "bounds", "motion_bound")]
    if R.ref_compact_raw(*args, _p(raw) if len(raw) else None, len(raw), _p(cand), ctypes.byref(n_cand)):
        raise ValueError(R.ref_proxy_last_error().decode())
    return cand[:n_cand.value]


def ref_load_mesh(path: str, center: bool = False):
    """The reference's LoadTriangleMesh (and CenterMeshAtAabbCenter): (vertices,
    triangles, patch ids[, center]) or ValueError with its message."""
    R = ref()
    if not hasattr(R, "_mesh_ready"):
        vp = ctypes.c_void_p
        R.ref_load_mesh.argtypes = [ctypes.c_char_p, vp, vp, vp, vp, vp]
        R.ref_proxy_last_error.restype = ctypes.c_char_p
        R._mesh_ready = True
    counts = np.zeros(3, np.int64)
    if R.ref_load_mesh(str(path).encode(), _p(counts), None, None, None, None):
        raise ValueError(R.ref_proxy_last_error().decode())
    v = np.zeros((max(1, counts[0]), 3))
    t = np.zeros((max(1, counts[1]), 3), np.uint32)
    pid = np.zeros(max(1, counts[2]), np.uint32)
    c = np.zeros(3)
    R.ref_load_mesh(str(path).encode(), _p(counts), _p(v), _p(t), _p(pid), _p(c) if center else None)
    out = (v[:counts[0]], t[:counts[1]], pid[:counts[2]])
    return out + (c,) if center else out
