"""The large-corpus configuration at full size: N=10,000,000 docs, dim 768,
RankQuant b=2 + constant-weight Bitmap n_top=192 + MultiBucketBitmap b=2
resident in HBM, 1,024-query batches, stage-1 top-2,000, rerank top-100.

The device encoders are spot-checked against the oracle on sampled docs; the
scans, the threshold filter and the selects are checked at full size against
the oracle run on the device's own codes (fetched as the persisted payload):
stage-1 candidate ids bit-exact in tie order, reranked top-100 within the
FP64 bar; the batched (tensor-core) form equals the plain one-query form."""
import numpy as np
import pytest

import ordvec_b200 as ob
from test_gpu_parity import check_float_topk

pytestmark = pytest.mark.gpu

N, DIM, SEED, NQ, M, K, N_TOP = 10_000_000, 768, 0x0DD5EED4, 1024, 2000, 100, 192
CHUNK = 1_000_000


@pytest.fixture(scope="module")
def large():
    rq, bm, mb = ob.RankQuant(DIM, 2), ob.Bitmap(DIM, N_TOP), ob.MultiBucketBitmap(DIM, 2)
    samples = {}
    for first in range(0, N, CHUNK):
        d = ob.synth_docs(SEED, min(CHUNK, N - first), DIM, first=first)
        for ix in (rq, bm, mb):
            ix.add(d)
        if first in (0, 9 * CHUNK):  # first and last chunk: 3,000 docs each for the encoder check
            rows = np.r_[0:1000, CHUNK // 2:CHUNK // 2 + 1000, CHUNK - 1000:CHUNK]
            samples[first] = (rows + first, d[rows].copy())
    queries, _ = ob.synth_queries(SEED + 1, N, NQ, DIM)
    return rq, bm, mb, queries, samples


def test_large_encoders_spot_check(orc, large):
    rq, bm, mb, _, samples = large
    words = bm.payload().view(np.uint64).reshape(N, DIM // 64)
    packed = rq.payload().reshape(N, DIM * 2 // 8)
    for rows, docs in samples.values():
        assert np.array_equal(words[rows], orc.bitmap_encode(docs, DIM, N_TOP).reshape(len(rows), -1))
        assert np.array_equal(packed[rows], orc.rankquant_encode(docs, DIM, 2).reshape(len(rows), -1))


def test_large_bitmap_two_stage(orc, large):
    rq, bm, _, queries, _ = large
    res = ob.two_stage_search(rq, bm, queries, M, K)
    # batched (tensor-core scan + threshold filter) == one query per call
    for qi in (0, 511, NQ - 1):
        one = ob.two_stage_search(rq, bm, queries[qi:qi + 1], M, K)
        assert np.array_equal(one.indices, res.indices_for_query(qi))
        assert np.array_equal(one.scores.view(np.uint32), res.scores_for_query(qi).view(np.uint32))
    # stage-1 candidates of a batched call against the oracle on the device's codes
    words = bm.payload().view(np.uint64)
    packed = rq.payload()
    cands = bm.top_m_candidates_batched(queries[:64], M)
    for qi in (0, 63):
        want = orc.bitmap_top_m(words, N, DIM, N_TOP, queries[qi], M)
        assert np.array_equal(cands[qi], want), qi
        s64 = orc.rq_scores_f64_subset(packed, DIM, 2, queries[qi], want)
        check_float_topk(res.indices_for_query(qi), res.scores_for_query(qi), want, s64, K)


def test_large_multibucket_two_stage(orc, large, monkeypatch):
    rq, _, mb, queries, _ = large
    res = ob.two_stage_search(rq, mb, queries[:256], M, K)
    monkeypatch.setenv("OVB_BITMAP_TC", "0")  # the CUDA-core weighted scan
    cc = ob.two_stage_search(rq, mb, queries[:256], M, K)
    monkeypatch.delenv("OVB_BITMAP_TC")
    assert np.array_equal(res.indices, cc.indices)
    assert np.array_equal(res.scores.view(np.uint32), cc.scores.view(np.uint32))
    mwords = mb.payload().view(np.uint64)
    packed = rq.payload()
    w = orc.multibucket_weights(2, "diagonal")
    for qi in (0, 255):
        qbm = orc.multibucket_query(queries[qi], DIM, 2)
        cand = orc.multibucket_top_m(mwords, N, DIM, 2, qbm, w, M)
        s64 = orc.rq_scores_f64_subset(packed, DIM, 2, queries[qi], cand)
        check_float_topk(res.indices_for_query(qi), res.scores_for_query(qi), cand, s64, K)
