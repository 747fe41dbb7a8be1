"""The large-corpus configuration at full size: N=10,000,000 docs, dim 768,
RankQuant b=2 + constant-weight Bitmap n_top=192 + MultiBucketBitmap b=2
resident in HBM, 1,024-query batches, stage-1 top-2,000, rerank top-100 --
the benchmark's headline call.

The oracle encodes the same corpus on the host (one rank transform per doc,
both layouts), independently of the device encoders, and every code byte is
compared.  The headline call (1,024 queries, the benchmark's query seed) is
then checked row by row against the oracle run on the oracle's own codes:
stage-1 candidate rows bit-exact in tie order for all 1,024 queries, and
every row's reranked top-100 within the FP64 bar (ids identical except
between scores closer than 1e-5 relative).  The batched (tensor-core) form
equals the plain one-query form, and the tensor-core multi-bucket path the
CUDA-core weighted path."""
import numpy as np
import pytest

import ordvec_b200 as ob
from test_gpu_parity import check_float_topk

pytestmark = pytest.mark.gpu

N, DIM, SEED, NQ, M, K, N_TOP = 10_000_000, 768, 0x0DD5EED4, 1024, 2000, 100, 192
QPV = DIM // 64
CHUNK = 1_000_000


@pytest.fixture(scope="module")
def large(orc):
    rq, bm, mb = ob.RankQuant(DIM, 2), ob.Bitmap(DIM, N_TOP), ob.MultiBucketBitmap(DIM, 2)
    words = np.empty(N * QPV, np.uint64)
    packed = np.empty(N * DIM // 4, np.uint8)
    for first in range(0, N, CHUNK):
        d = ob.synth_docs(SEED, min(CHUNK, N - first), DIM, first=first)
        for ix in (rq, bm, mb):
            ix.add(d)
        n = d.shape[0]
        orc.encode_bitmap_rankquant(d, DIM, N_TOP, 2, words[first * QPV:(first + n) * QPV],
                                    packed[first * DIM // 4:(first + n) * DIM // 4])
    queries, _ = ob.synth_queries(SEED + 1, N, NQ, DIM)  # the benchmark's rank-0 queries
    return rq, bm, mb, queries, words, packed


@pytest.fixture(scope="module")
def oracle_run(orc, large):
    """The oracle's two-stage run of the whole batch on its own codes: stage-1
    candidate rows (nq x M) and its f32 top-100."""
    _, _, _, queries, words, packed = large
    s, i, cands = orc.cpu_bitmap_two_stage(words, packed, N, DIM, N_TOP, 2, queries, M, K, orc.max_threads(),
                                           want_candidates=True)
    return s, i, cands


def test_large_device_codes_equal_oracle_codes(large):
    rq, bm, mb, _, words, packed = large
    assert np.array_equal(bm.payload().view(np.uint64), words)
    assert np.array_equal(rq.payload(), packed)


def test_large_multibucket_codes_spot_check(orc, large):
    _, _, mb, _, _, _ = large
    mwords = mb.payload().view(np.uint64).reshape(N, 4 * QPV)
    for first in (0, 9 * CHUNK):
        rows = np.r_[0:1000, CHUNK // 2:CHUNK // 2 + 1000, CHUNK - 1000:CHUNK] + first
        d = ob.synth_docs(SEED, CHUNK, DIM, first=first)[rows - first]
        assert np.array_equal(mwords[rows], orc.multibucket_encode(d, DIM, 2).reshape(len(rows), -1))


def test_large_bitmap_headline_call_every_row(orc, large, oracle_run):
    """The benchmark's headline call, 1,024 queries: every stage-1 candidate row
    and every reranked top-100 row against the oracle."""
    rq, bm, _, queries, _, packed = large
    _, _, cands = oracle_run
    got = bm.top_m_candidates_batched(queries, M)
    for qi in range(NQ):
        assert np.array_equal(got[qi], cands[qi]), qi
    res = ob.two_stage_search(rq, bm, queries, M, K)
    for qi in range(NQ):
        s64 = orc.rq_scores_f64_subset(packed, DIM, 2, queries[qi], cands[qi])
        check_float_topk(res.indices_for_query(qi), res.scores_for_query(qi), cands[qi], s64, K)
    # batched (tensor-core scan + threshold filter) == one query per call
    for qi in (0, 511, NQ - 1):
        one = ob.two_stage_search(rq, bm, queries[qi:qi + 1], M, K)
        assert np.array_equal(one.indices, res.indices_for_query(qi))
        assert np.array_equal(one.scores.view(np.uint32), res.scores_for_query(qi).view(np.uint32))


def test_large_multibucket_two_stage(orc, large):
    rq, _, mb, queries, _, packed = large
    import os

    res = ob.two_stage_search(rq, mb, queries[:256], M, K)
    os.environ["OVB_BITMAP_TC"] = "0"  # the CUDA-core weighted scan
    try:
        cc = ob.two_stage_search(rq, mb, queries[:256], M, K)
    finally:
        del os.environ["OVB_BITMAP_TC"]
    assert np.array_equal(res.indices, cc.indices)
    assert np.array_equal(res.scores.view(np.uint32), cc.scores.view(np.uint32))
    mwords = mb.payload().view(np.uint64)
    w = orc.multibucket_weights(2, "diagonal")
    for qi in (0, 255):
        qbm = orc.multibucket_query(queries[qi], DIM, 2)
        cand = orc.multibucket_top_m(mwords, N, DIM, 2, qbm, w, M)
        s64 = orc.rq_scores_f64_subset(packed, DIM, 2, queries[qi], cand)
        check_float_topk(res.indices_for_query(qi), res.scores_for_query(qi), cand, s64, K)
