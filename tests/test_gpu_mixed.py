"""Mixed batches (ovb_rankquant_search_mixed): queries with their own index
(bits) and k in one call, groups on the split-BF16 tensor-core path run
through tuned, graph-captured plans."""
import numpy as np
import pytest

import ordvec_b200 as ob
from test_gpu_parity import check_float_topk

pytestmark = pytest.mark.gpu


def _setup(dim=1024, n=20_000, nq=300, seed=0x0DD5EED3):
    docs = ob.synth_docs(seed, n, dim)
    queries, _ = ob.synth_queries(seed + 1, n, nq, dim)
    indices = []
    for bits in (1, 2, 4):
        rq = ob.RankQuant(dim, bits)
        rq.add(docs)
        indices.append(rq)
    rng = np.random.default_rng(seed)
    sel = rng.integers(0, 3, nq).astype(np.uint32)
    ks = rng.choice([10, 50, 100], nq).astype(np.uint32)
    return docs, queries, indices, sel, ks


def _expected(indices, queries, sel, ks):
    """Per group: one direct batched search at the group's largest k, each row
    truncated to its own k and padded."""
    nq, k_max = len(queries), int(ks.max())
    s = np.full((nq, k_max), -np.inf, np.float32)
    i = np.full((nq, k_max), -1, np.int64)
    for j, rq in enumerate(indices):
        rows = np.flatnonzero(sel == j)
        if rows.size == 0:
            continue
        kg = int(ks[rows].max())
        res = rq.search_asymmetric(queries[rows], kg)
        for r, qi in enumerate(rows):
            keep = min(int(ks[qi]), res.k)
            s[qi, :keep] = res.scores_for_query(r)[:keep]
            i[qi, :keep] = res.indices_for_query(r)[:keep]
    return s, i


def test_mixed_batch_matches_grouped_searches_and_replays_graphs(orc, monkeypatch):
    docs, queries, indices, sel, ks = _setup()
    n, dim = docs.shape
    want_s, want_i = _expected(indices, queries, sel, ks)
    got = ob.search_mixed(indices, sel, ks, queries)  # first call: tune, capture
    k_max = int(ks.max())
    assert got.k == k_max
    assert np.array_equal(got.indices.reshape(-1, k_max), want_i)
    assert np.array_equal(got.scores.reshape(-1, k_max).view(np.uint32), want_s.view(np.uint32))
    again = ob.search_mixed(indices, sel, ks, queries)  # replays the graphs
    assert np.array_equal(again.indices, got.indices)
    assert np.array_equal(again.scores.view(np.uint32), got.scores.view(np.uint32))
    for j, rq in enumerate(indices):
        rows = np.flatnonzero(sel == j)
        info = ob.mixed_plan_info(rq, rows.size, int(ks[rows].max()))
        assert info["q_per_tile"] in (32, 64, 128)
        assert info["candidates"] >= int(ks[rows].max())
        assert info["replays"] >= 1
    # against the FP64 oracle on a few rows
    for qi in (0, 7, 150):
        bits = (1, 2, 4)[sel[qi]]
        packed = orc.rankquant_encode(docs, dim, bits)
        s64 = orc.rq_scores_f64(packed, n, dim, bits, queries[qi])
        k = int(ks[qi])
        check_float_topk(got.indices_for_query(qi)[:k], got.scores_for_query(qi)[:k], np.arange(n), s64, k)
        assert (got.indices_for_query(qi)[k:] == -1).all()
    monkeypatch.setenv("OVB_MIXED_GRAPH", "0")
    plain = ob.search_mixed(indices, sel, ks, queries)
    assert np.array_equal(plain.indices, got.indices)


def test_mixed_batch_other_shapes_and_errors():
    dim, n = 96, 3000  # not a multiple of 64: groups take the CUDA-core path
    docs = ob.synth_docs(77, n, dim)
    queries, _ = ob.synth_queries(78, n, 40, dim)
    a, b = ob.RankQuant(dim, 2), ob.RankQuant(dim, 4)
    a.add(docs)
    b.add(docs)
    sel = np.arange(40, dtype=np.uint32) % 2
    ks = np.where(sel == 0, 5, 12).astype(np.uint32)
    got = ob.search_mixed([a, b], sel, ks, queries)
    want_s, want_i = _expected([a, b], queries, sel, ks)
    assert np.array_equal(got.indices.reshape(-1, 12), want_i)
    with pytest.raises(ob.OrdvecError) as e:
        ob.search_mixed([a, b], np.full(40, 2, np.uint32), ks, queries)
    assert e.value.status == 2
    c = ob.RankQuant(64, 2)
    c.add(docs[:, :64].copy())
    with pytest.raises(ob.OrdvecError) as e:
        ob.search_mixed([a, c], sel, ks, queries)
    assert e.value.status == 7
    with pytest.raises(ob.OrdvecError) as e:
        ob.mixed_plan_info(a, 40, 5)  # never planned
    assert e.value.status == 2


def test_mixed_batch_filtered_plans(monkeypatch):
    """At N large enough for the split-BF16 threshold filter the captured plans
    run the filtered pipeline; results equal the key-matrix plans'."""
    docs, queries, indices, sel, ks = _setup(dim=256, n=150_000, nq=400, seed=0x0DD5EED7)
    got = ob.search_mixed(indices, sel, ks, queries)
    again = ob.search_mixed(indices, sel, ks, queries)  # graph replay
    assert np.array_equal(again.indices, got.indices)
    monkeypatch.setenv("OVB_SPLIT_FILTER", "0")
    monkeypatch.setenv("OVB_MIXED_GRAPH", "0")
    dense = ob.search_mixed(indices, sel, ks, queries)
    assert np.array_equal(dense.indices, got.indices)
    assert np.array_equal(dense.scores.view(np.uint32), got.scores.view(np.uint32))
    for j, rq in enumerate(indices):
        rows = np.flatnonzero(sel == j)
        assert ob.mixed_plan_info(rq, rows.size, int(ks[rows].max()))["replays"] >= 1
