"""Batched external-query candidates (rt_candidate/external_batch_candidate.cpp)
against the reference's GenerateCandidatesForExternalBatch compiled
unchanged: the host encoding and translation around the restated broad phase
on the CPU, the device path on the GPU, byte for byte, with the reference's
error messages."""
from __future__ import annotations

import numpy as np
import pytest

from external_inputs import make_batch

CASES = [(1, 40, {}), (2, 120, {"touching": True}), (3, 7, {"ids": "dense"}), (4, 1, {}),
         (5, 64, {"miss": 0.0, "box_pairs": False}), (6, 300, {"miss": 0.6})]


def _need_ref(oracle_mod):
    if not oracle_mod.ref_available():
        pytest.skip("reference library not built")


@pytest.mark.parametrize("seed,n,kw", CASES)
def test_host_encoding_and_translation_match_reference(oracle_mod, seed, n, kw):
    """encode_scene + the restated CPU broad phase + translate reproduce the
    reference's candidates, runtime ids, counts and recall."""
    from p2cccd_b200 import external as ex

    _need_ref(oracle_mod)
    b = make_batch(n, seed, **kw)
    c1, r1, counts, recall = oracle_mod.ref_external_batch(b)
    scene = ex.encode_scene(b)
    rid = ex.runtime_query_ids(b["query_id"])
    raw, cand = oracle_mod.proxy_candidates(scene)
    c2, active = ex.translate(cand, b, rid)
    assert np.array_equal(r1, rid)
    assert c1.tobytes() == c2.tobytes()
    assert list(counts) == [2 * n, len(raw), len(c2)]
    assert ex.candidate_recall(b, active) == recall


def test_runtime_id_bumps_follow_reference(oracle_mod):
    """A zero source id takes index + 1, bumped past ids that earlier queries
    hold; a later query whose source id was taken by the bump is bumped too."""
    from p2cccd_b200 import external as ex

    _need_ref(oracle_mod)
    b = make_batch(9, 11, ids="dense")
    b["query_id"][:] = [5, 6, 0, 3, 4, 1, 2, 7, 8]  # index 2 asks for 3 (held by index 3 later: not yet taken)
    _, r1, _, _ = oracle_mod.ref_external_batch(b)
    assert np.array_equal(r1, ex.runtime_query_ids(b["query_id"]))
    b["query_id"][:] = [3, 4, 0, 9, 5, 6, 1, 2, 7]  # 3 -> 4 -> 5 taken later: index 4 bumps to 6, ...
    _, r1, _, _ = oracle_mod.ref_external_batch(b)
    assert np.array_equal(r1, ex.runtime_query_ids(b["query_id"]))
    assert len(np.unique(r1)) == 9


@pytest.mark.parametrize("fault", ["t0", "t1", "dup", "t1_then_dup", "dup_then_t0"])
def test_validation_messages_match_reference(oracle_mod, fault):
    from p2cccd_b200 import external as ex

    _need_ref(oracle_mod)
    b = make_batch(12, 21)
    if fault == "t0":
        b["vertices_t0"][5, 2, 1] = np.nan
    elif fault == "t1":
        b["vertices_t1"][3, 0, 0] = np.inf
    elif fault == "dup":
        b["query_id"][7] = b["query_id"][4]
    elif fault == "t1_then_dup":
        b["vertices_t1"][6, 1, 2] = -np.inf
        b["query_id"][8] = b["query_id"][0]
    else:
        b["query_id"][4] = b["query_id"][2]
        b["vertices_t0"][9, 3, 0] = np.nan
    with pytest.raises(ValueError) as ref_err:
        oracle_mod.ref_external_batch(b)
    with pytest.raises(ValueError) as err:
        ex._first_error(b)
    assert str(err.value) == str(ref_err.value)


def test_empty_batch_message(oracle_mod):
    import p2cccd_cpp as cpp
    from p2cccd_b200.external import batch_arrays

    _need_ref(oracle_mod)
    b = batch_arrays([], [], [], np.zeros((0, 4, 3)), np.zeros((0, 4, 3)))
    with pytest.raises(ValueError) as ref_err:
        oracle_mod.ref_external_batch(b)
    with pytest.raises(ValueError) as err:
        cpp.generate_candidates_for_external_batch(b)
    assert str(err.value) == str(ref_err.value)


class _Query:
    def __init__(self, **kw):
        self.__dict__.update(kw)


class _Batch:
    def __init__(self, queries):
        self.queries = queries


def _objects(b: dict) -> _Batch:
    """The column batch as the reference binding's input objects."""
    qs = []
    for k in range(len(b["query_id"])):
        gt = int(b["ground_truth"][k])
        qs.append(_Query(query_id=int(b["query_id"][k]), source_query_index=int(b["source_query_index"][k]),
                         family="vf" if b["family"][k] == 0 else "ee",
                         vertices_t0=b["vertices_t0"][k].tolist(), vertices_t1=b["vertices_t1"][k].tolist(),
                         ground_truth_collides=None if gt < 0 else bool(gt),
                         box_pair=[int(x) for x in b["box_pair"][k]] if b["has_box"][k] else None))
    return _Batch(qs)


def test_binding_parser_round_trip_and_errors():
    """ParseExternalBatchQueries' reading of the batch objects, and its
    messages for a bad family, vertex count, vertex width and box pair."""
    import p2cccd_cpp as cpp

    b = make_batch(10, 31)
    parsed = cpp._external_batch(_objects(b))
    for k in b:
        if k == "box_pair":  # only the pairs that are given
            assert np.array_equal(parsed[k][b["has_box"] == 1], b[k][b["has_box"] == 1])
        else:
            assert np.array_equal(parsed[k], b[k]), k
    bad = _objects(b)
    bad.queries[3].family = "fv"
    with pytest.raises(ValueError, match="unsupported external CCD query family: fv"):
        cpp._external_batch(bad)
    bad = _objects(b)
    bad.queries[2].vertices_t1 = bad.queries[2].vertices_t1[:3]
    with pytest.raises(ValueError, match="vertices_t1 must contain four vertices"):
        cpp._external_batch(bad)
    bad = _objects(b)
    bad.queries[2].vertices_t0[1] = [0.0, 1.0]
    with pytest.raises(ValueError, match="vertices_t0 vertices must be 3D"):
        cpp._external_batch(bad)
    bad = _objects(b)
    bad.queries[0].box_pair = [1, 2, 3]
    with pytest.raises(ValueError, match="box_pair must contain exactly two object ids"):
        cpp._external_batch(bad)
    with pytest.raises(ValueError, match="unsupported candidate backend: rtx"):
        cpp.generate_candidates_for_external_batch(_objects(b), backend_name="rtx")
    with pytest.raises(ValueError, match="built without OptiX"):
        cpp.generate_candidates_for_external_batch(_objects(b), backend_name="optix")


# ---------------------------------------------------------------- on the GPU

@pytest.mark.gpu
@pytest.mark.parametrize("seed,n,kw", CASES)
def test_device_batch_candidates_match_reference(oracle_mod, seed, n, kw):
    from p2cccd_b200 import external as ex

    b = make_batch(n, seed, **kw)
    r = ex.generate(b)
    if oracle_mod.ref_available():
        c1, r1, counts, recall = oracle_mod.ref_external_batch(b)
    else:  # the restated broad phase around the same host encoding
        sc = ex.encode_scene(b)
        raw, cand = oracle_mod.proxy_candidates(sc)
        r1 = ex.runtime_query_ids(b["query_id"])
        c1, active = ex.translate(cand, b, r1)
        counts, recall = [2 * n, len(raw), len(c1)], ex.candidate_recall(b, active)
    assert r["candidates"].tobytes() == c1.tobytes()
    assert np.array_equal(r["runtime_query_ids"], r1)
    assert [r["primitive_count"], r["raw_hit_count"], r["compact_candidate_count"]] == list(counts)
    assert r["candidate_recall"] == recall


@pytest.mark.gpu
def test_mirror_external_batch_objects(oracle_mod):
    import p2cccd_cpp as cpp
    from p2cccd_b200 import external as ex

    b = make_batch(50, 41, touching=True)
    res = cpp.generate_candidates_for_external_batch(_objects(b))
    fb = cpp.generate_candidates_for_external_batch(_objects(b), backend_name="optix", allow_optix_cpu_fallback=True)
    assert res.backend_name == "cpu_reference" and fb.backend_name == "optix_cpu_fallback"
    assert cpp._candidate_array(res.candidates).tobytes() == cpp._candidate_array(fb.candidates).tobytes()
    raw, cand = oracle_mod.proxy_candidates(ex.encode_scene(b))
    want, _ = ex.translate(cand, b, ex.runtime_query_ids(b["query_id"]))
    assert cpp._candidate_array(res.candidates).tobytes() == want.tobytes()
    assert [m.source_query_id for m in res.runtime_query_ids] == b["query_id"].tolist()
    assert res.primitive_count == 100 and res.raw_hit_count == len(raw)
    assert res.timing.total_ms >= res.timing.trace_ms >= 0.0


@pytest.mark.gpu
def test_large_batch_properties():
    """100k queries: one candidate at most per query, ids strictly increasing
    in (query id) order, each candidate's query really overlapping (checked
    on the host from the encoded scene), and queries without a candidate
    really separated."""
    from p2cccd_b200 import external as ex

    n = 100_000
    b = make_batch(n, 51, miss=0.4)
    r = ex.generate(b)
    c = r["candidates"]
    assert r["raw_hit_count"] == len(c) <= n
    assert np.all(np.diff(c["query_id"].astype(np.int64)) > 0)
    assert np.array_equal(c["candidate_id"], c["query_id"] * np.uint64(1_000_003) + np.arange(1, len(c) + 1,
                                                                                             dtype=np.uint64))
    sc = ex.encode_scene(b)
    bnd = sc["bounds"].reshape(n, 2, 6)
    overlap = np.all(~((bnd[:, 0, 3:] < bnd[:, 1, :3]) | (bnd[:, 1, 3:] < bnd[:, 0, :3])), axis=1)
    pos = {int(q): k for k, q in enumerate(r["runtime_query_ids"])}
    hit = np.zeros(n, bool)
    hit[[pos[int(q)] for q in c["query_id"]]] = True
    assert np.array_equal(hit, overlap)
