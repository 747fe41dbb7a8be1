"""Size-independent properties the reference's own tests state for this path
(tests/index/two_stage.rs, tests/index/quant.rs), checked on the device path.

* a full candidate set (m = n) makes the subset rerank equal the full search
  (tests/index/two_stage.rs:238-258);
* batched calls equal the same queries searched one at a time
  (tests/index/two_stage.rs:375-425);
* the subset rerank does not depend on the order of the candidate list
  (tests/index/two_stage.rs:457-520);
* RankQuant b=1/2/4 asymmetric top-10 against the float formula
  (tests/index/quant.rs:304-350): scores within 1e-4, identical top-10 set.
"""
import numpy as np
import pytest

import ordvec_b200 as ob

pytestmark = pytest.mark.gpu

DIM, N = 256, 6000


@pytest.fixture(scope="module")
def two_stage():
    docs = ob.synth_docs(0x5EED01, N, DIM)
    queries, _ = ob.synth_queries(0x5EED02, N, 48, DIM)
    sb, rq, fs = ob.SignBitmap(DIM), ob.RankQuant(DIM, 2), ob.RankQuantFastscan(DIM)
    for ix in (sb, rq, fs):
        ix.add(docs)
    return docs, queries, sb, rq, fs


def test_full_candidate_set_equals_full_search(two_stage):
    _, queries, sb, rq, _ = two_stage
    for q in queries[:4]:
        cand = sb.top_m_candidates(q, N)
        assert cand.size == N and np.array_equal(np.sort(cand), np.arange(N))
        full = rq.search_asymmetric(q, 16)
        s, i = rq.search_asymmetric_subset(q, cand, 16)
        assert np.array_equal(i, full.indices)
        assert np.max(np.abs(s - full.scores)) <= 1e-6


def test_batched_equals_looped_single(two_stage):
    _, queries, sb, rq, fs = two_stage
    for s1, m in ((sb, 320), (fs, 500)):
        batched = ob.two_stage_search(rq, s1, queries, m, 10)  # 48 queries: tensor-core stage 1
        for qi in range(0, len(queries), 7):
            one = ob.two_stage_search(rq, s1, queries[qi:qi + 1], m, 10)
            assert np.array_equal(one.indices, batched.indices_for_query(qi)), (type(s1).__name__, qi)
            assert np.array_equal(one.scores, batched.scores_for_query(qi)), (type(s1).__name__, qi)


def test_subset_rerank_is_order_independent(two_stage):
    _, queries, sb, rq, _ = two_stage
    rng = np.random.default_rng(5)
    for q in queries[:4]:
        cand = sb.top_m_candidates(q, 700)
        s0, i0 = rq.search_asymmetric_subset(q, cand, 25)
        for _ in range(3):
            perm = rng.permutation(cand)
            s1, i1 = rq.search_asymmetric_subset(q, perm, 25)
            assert np.array_equal(i0, i1) and np.array_equal(s0, s1)


@pytest.mark.parametrize("bits", [1, 2, 4])
def test_rankquant_asymmetric_matches_float_formula(bits):
    rng = np.random.default_rng(200 + bits)
    docs = rng.standard_normal((2000, DIM)).astype(np.float32)
    q = rng.uniform(-1.0, 1.0, DIM).astype(np.float32)
    rq = ob.RankQuant(DIM, bits)
    rq.add(docs)
    res = rq.search_asymmetric(q, 10)
    # float reference: centred bucket codes against the unit query, over the norm
    ranks = np.argsort(np.argsort(docs, axis=1, kind="stable"), axis=1, kind="stable")
    buckets = (ranks.astype(np.int64) << bits) // DIM
    centred = buckets - ((1 << bits) - 1) / 2.0
    qu = q.astype(np.float64) / np.linalg.norm(q.astype(np.float64))
    norm = np.sqrt(DIM * ((4.0 ** bits - 1.0) / 12.0))
    ref = centred @ qu / norm
    assert np.max(np.abs(res.scores - ref[res.indices])) < 1e-4
    assert set(res.indices.tolist()) == set(np.argsort(-ref, kind="stable")[:10].tolist())
