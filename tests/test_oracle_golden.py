"""Pin the CPU oracle against the reference's own known-answer tests.

Every expectation here is a literal from the reference's test suite (file:line
cited per test) or the reference's own sort-based test oracle restated in
tests/golden/make_golden.py.  Nothing here needs a GPU.
"""
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "tiled_candgen.npz")


def _corpus(orc, kind, dim, n, seed):
    if kind == 0:
        return orc.xorshift_f32(seed, n * dim)
    if kind == 1:
        doc = np.arange(n)[:, None] % 4
        c = np.arange(dim)[None, :]
        return np.where((c + doc) % 3 == 0, -1.0, 1.0).astype(np.float32).reshape(-1)
    return np.tile(orc.xorshift_f32(seed, n * dim), 512)


def golden_cases(orc):
    g = np.load(GOLDEN)
    names = sorted({k.split("__")[0] for k in g.files})
    for name in names:
        meta = [int(x) for x in g[f"{name}__meta"]]
        dim, cn, cseed, qn, qseed, kind = meta[:6]
        ms = meta[6:]
        vec = _corpus(orc, kind, dim, cn, cseed)
        qs = orc.xorshift_f32(qseed, qn * dim)
        assert np.array_equal(vec[:64], g[f"{name}__head"]), name
        assert np.array_equal(qs[:64], g[f"{name}__qhead"]), name
        yield name, dim, vec, qs, ms, g[f"{name}__expected"]


def test_tiled_candgen_single_and_streamed_match_sort_oracle(orc):
    """tests/tiled_candgen.rs:51-175 -- single-query and streamed CSR paths
    equal the (hamming asc, doc_id asc) sort at every m of every case."""
    for name, dim, vec, qs, ms, expected in golden_cases(orc):
        words = orc.sign_encode(vec, dim)
        n = vec.size // dim
        nq = qs.size // dim
        for m in ms:
            me = min(m, n)
            streamed = orc.sign_top_m_streamed(words, n, dim, qs, m)
            for qi in range(nq):
                got = orc.sign_top_m(words, n, dim, qs[qi * dim:(qi + 1) * dim], m)
                assert np.array_equal(got, expected[qi, :me]), (name, m, qi)
                assert np.array_equal(streamed[qi], expected[qi, :me]), (name, m, qi)


def test_rankquant_persisted_payload_golden_bytes(orc):
    """tests/persistence_compat.rs:130-135: RankQuant::new(8, 2) of [0..7]
    packs to 0x05 0xaf."""
    packed = orc.rankquant_encode(np.arange(8, dtype=np.float32), 8, 2)
    assert packed.tolist() == [0x05, 0xAF]


def test_bitmap_and_sign_persisted_payload_golden_bytes(orc):
    """tests/persistence_compat.rs:161-167 (Bitmap::new(64, 2) of [0..63]) and
    :191-200 (SignBitmap of -1 except coords 0 and 63)."""
    bm = orc.bitmap_encode(np.arange(64, dtype=np.float32), 64, 2)
    assert bm.view(np.uint8).tolist() == [0, 0, 0, 0, 0, 0, 0, 0xC0]
    v = -np.ones(64, np.float32)
    v[0] = v[63] = 1.0
    sb = orc.sign_encode(v, 64)
    assert sb.view(np.uint8).tolist() == [1, 0, 0, 0, 0, 0, 0, 0x80]


def test_topk_duplicate_ties_and_score_offset_literals(orc):
    """src/util.rs:658-686 and :732-776."""
    t = orc.TopK(2, tie_keys=[7, 7, 7])
    for i in range(3):
        t.insert(0.0, i)
    s, i = t.finalize()
    assert s.tolist() == [0.0, 0.0] and i.tolist() == [0, 1]

    t = orc.TopK(1, tie_keys=[10, 3])
    t.set_score_offset(16_777_216.0)
    t.insert(1.0, 0)
    t.insert(0.0, 1)
    s, i = t.finalize()
    assert s.tolist() == [16_777_216.0] and i.tolist() == [1]

    t = orc.TopK(2, tie_keys=[10, 20, 30, 40])
    t.insert(1.0, 0)
    t.insert(3.0, 1)
    t.insert(2.0, 2)
    s, i = t.finalize()
    assert i.tolist() == [1, 2]
    t = orc.TopK(2, tie_keys=[10, 20, 30, 40])
    t.insert(5.0, 3)
    t.insert(1.0, 0)
    s, i = t.finalize()
    assert i.tolist() == [3, 0]

    t = orc.TopK(0)
    t.insert(1.0, 0)
    s, i = t.finalize(0)
    assert s.size == 0 and i.size == 0


def test_l2_normalise_threshold_literals(orc):
    """src/util.rs:778-814."""
    eps = np.float32(1e-12)
    assert orc.l2_normalise([3.0, 0.0, 4.0, 0.0]).tolist() == pytest.approx([0.6, 0.0, 0.8, 0.0])
    assert orc.l2_normalise([eps * np.float32(0.5), 0.0]).tolist() == [0.0, 0.0]
    assert orc.l2_normalise([eps, 0.0]).tolist() == [0.0, 0.0]
    assert orc.l2_normalise([eps * np.float32(2.0), 0.0]).tolist() == [1.0, 0.0]
    assert orc.l2_normalise(np.zeros(4)).tolist() == [0.0] * 4


def test_full_search_ties_return_lowest_row_ids(orc):
    """tests/determinism_contract.rs:15-49 and tests/index/quant.rs:246-256."""
    dim = 64
    docs = np.ones((8, dim), np.float32)
    zero = np.zeros(dim, np.float32)
    packed = orc.rankquant_encode(docs, dim, 2)
    s, i = orc.rq_search_asym(packed, 8, dim, 2, zero, 4)
    assert i[0].tolist() == [0, 1, 2, 3] and (s == 0.0).all()
    bm = orc.bitmap_encode(docs, dim, dim // 4)
    s, i = orc.bitmap_search(bm, 8, dim, dim // 4, np.ones(dim, np.float32), 4)
    assert i[0].tolist() == [0, 1, 2, 3] and (s == s[0, 0]).all()
    zdocs = np.zeros((6, dim), np.float32)
    for bits in (1, 2, 4):
        p = orc.rankquant_encode(zdocs, dim, bits)
        _, i = orc.rq_search_asym(p, 6, dim, bits, zero, 6)
        assert i[0].tolist() == [0, 1, 2, 3, 4, 5]


def test_subset_ties_use_global_ids_and_keep_duplicates(orc):
    """tests/determinism_contract.rs:71-125."""
    dim = 64
    packed = orc.rankquant_encode(np.ones((12, dim), np.float32), dim, 2)
    zero = np.zeros(dim, np.float32)
    s, i = orc.rq_subset(packed, 12, dim, 2, zero, [9, 3, 7, 1], 2)
    assert s.tolist() == [0.0, 0.0] and i.tolist() == [1, 3]
    s, i = orc.rq_subset(packed, 12, dim, 2, zero, [7, 8, 7], 2)
    assert i.tolist() == [7, 7]
    s, i = orc.rq_subset_batched(packed, 12, dim, 2, zero, [0, 4], [7, 7, 3, 7], 4)
    assert s[0].tolist() == [0.0] * 4 and i[0].tolist() == [3, 7, 7, 7]


def test_candidate_prefilters_preserve_order(orc):
    """tests/determinism_contract.rs:127-150."""
    dim = 64
    docs = np.ones((10, dim), np.float32)
    q = np.ones(dim, np.float32)
    bm = orc.bitmap_encode(docs, dim, dim // 4)
    assert orc.bitmap_top_m(bm, 10, dim, dim // 4, q, 5).tolist() == [0, 1, 2, 3, 4]
    sw = orc.sign_encode(docs, dim)
    assert orc.sign_top_m(sw, 10, dim, q, 5).tolist() == [0, 1, 2, 3, 4]


def test_ffi_fixture_expectations(orc):
    """ordvec-ffi/src/lib.rs:1022-1049 fixtures and :1135-1271 expectations:
    full search ranks row 0 first; subset [3,1,2] -> [1,2]; duplicates
    [3,1,1,2] -> [1,1,2] for both RankQuant and Bitmap."""
    doc = np.arange(16, dtype=np.float32)
    packed = orc.rankquant_encode(np.tile(doc, 4), 16, 2)
    s, i = orc.rq_search_asym(packed, 4, 16, 2, doc, 2)
    assert i[0, 0] == 0
    # the ABI scores the whole subset then sorts (score desc, row asc) and truncates
    s, i = orc.rq_subset(packed, 4, 16, 2, doc, [3, 1, 2], 3)
    assert i[:2].tolist() == [1, 2]
    s, i = orc.rq_subset(packed, 4, 16, 2, doc, [3, 1, 1, 2], 4)
    assert i[:3].tolist() == [1, 1, 2]
    bdoc = np.zeros(64, np.float32)
    bdoc[:4] = 10.0 + np.arange(4)
    bm = orc.bitmap_encode(np.tile(bdoc, 4), 64, 4)
    s, i = orc.bitmap_search_subset(bm, 4, 64, 4, bdoc, [3, 1, 1, 2], 3)
    assert i.tolist() == [1, 1, 2]


def test_two_stage_policy_literals(orc):
    """tests/index/two_stage.rs:75-89 (N = 256) and the default policy."""
    N = 256
    assert orc.policy_candidate_count(0, N) == 0
    assert orc.policy_candidate_count(1, N) == 256
    assert orc.policy_candidate_count(10, N) == N
    assert orc.policy_candidate_count(10, 100_000) == 320
    big = 2**64 - 1
    assert orc.policy_candidate_count(big, N, 4, big, 37) == 37
    assert orc.policy_candidate_count(10, 9, 4, big, 37) == 9


def test_rank_pack_unpack_roundtrip(orc):
    """src/rank.rs pack/unpack inverse; rank ties break by index (-0.0 == +0.0)."""
    v = np.array([0.5, -0.0, 0.0, -1.0, 0.5, 2.0, 0.0, -0.0], np.float32)
    assert orc.rank_transform(v).tolist() == [5, 1, 2, 0, 6, 7, 3, 4]
    rng = np.random.default_rng(0)
    for bits in (1, 2, 4):
        b = rng.integers(0, 1 << bits, 64).astype(np.uint8)
        assert np.array_equal(orc.unpack_buckets(orc.pack_buckets(b, bits), 64, bits), b)


def test_fastscan_scalar_matches_its_dense_scores(orc):
    """src/fastscan.rs:755-777 corpus (dim 64, n 65, k 9): the TopK search
    equals the dense score sort (score desc under total_cmp, id asc)."""
    dim, n, k = 64, 65, 9
    docs = ((((np.arange(n * dim) * 37 + 11) % 257).astype(np.float32) - 128.0) / 128.0).astype(np.float32)
    qs = ((((np.arange(3 * dim) * 19 + 5) % 193).astype(np.float32) - 96.0) / 96.0).astype(np.float32)
    blocks = orc.fastscan_pack(docs, dim)
    s, i = orc.fastscan_search(blocks, n, dim, qs, k)
    for qi in range(3):
        dense = orc.fastscan_scores(blocks, n, dim, qs[qi * dim:(qi + 1) * dim])
        order = sorted(range(n), key=lambda d: (-dense[d], d))[:k]
        assert i[qi].tolist() == order


def test_multibucket_diag_weights_are_integer_overlaps(orc):
    """src/multi_bucket.rs:142-222: diagonal weights reduce the bilinear score to
    the same-bucket agreement count."""
    dim, bits = 128, 2
    rng = np.random.default_rng(1)
    docs = rng.standard_normal((20, dim)).astype(np.float32)
    words = orc.multibucket_encode(docs, dim, bits)
    q = rng.standard_normal(dim).astype(np.float32)
    qbm = orc.multibucket_query(q, dim, bits)
    w = orc.multibucket_weights(bits, "diagonal")
    s = orc.multibucket_scores(words, 20, dim, bits, qbm, w)
    rq = orc.rankquant_encode(np.concatenate([q[None], docs]), dim, bits)
    codes = np.stack([orc.unpack_buckets(rq[r * dim * bits // 8:(r + 1) * dim * bits // 8], dim, bits) for r in range(21)])
    agree = (codes[1:] == codes[0][None]).sum(axis=1)
    assert np.array_equal(s, agree.astype(np.float32))


def test_rank_and_symmetric_ties_return_lowest_row_ids(orc):
    """tests/determinism_contract.rs:15-38: Rank::search and RankQuant::search
    (symmetric) on 8 identical docs return rows 0..3; Rank::search_asymmetric
    with a zero query scores every doc 0.0."""
    dim = 64
    docs = np.ones((8, dim), np.float32)
    ranks = orc.rank_encode(docs, dim)
    _, i = orc.rank_search(ranks, 8, dim, np.ones(dim, np.float32), 4)
    assert i[0].tolist() == [0, 1, 2, 3]
    s, i = orc.rank_search(ranks, 8, dim, np.zeros(dim, np.float32), 4, asymmetric=True)
    assert i[0].tolist() == [0, 1, 2, 3] and (s == 0.0).all()
    packed = orc.rankquant_encode(docs, dim, 2)
    _, i = orc.rq_search_sym(packed, 8, dim, 2, np.ones(dim, np.float32), 4)
    assert i[0].tolist() == [0, 1, 2, 3]


def test_rank_persisted_payload_golden_bytes(orc):
    """tests/persistence_compat.rs:101-104: Rank::new(4) of [0, 1, 2, 3] stores
    the u16 ranks 0 1 2 3 (payload bytes 0 0 1 0 2 0 3 0)."""
    r = orc.rank_encode(np.arange(4, dtype=np.float32), 4)
    assert r.view(np.uint8).tolist() == [0, 0, 1, 0, 2, 0, 3, 0]


def test_rank_scores_are_spearman_and_centred_cosine(orc):
    """Rank::search is the Spearman correlation of the two rank vectors and
    Rank::search_asymmetric the cosine of the unit query with the centred ranks
    (src/rank.rs:356-482), checked against numpy in float64."""
    rng = np.random.default_rng(7)
    dim, n = 96, 40
    docs = rng.standard_normal((n, dim)).astype(np.float32)
    q = rng.standard_normal(dim).astype(np.float32)
    ranks = orc.rank_encode(docs, dim).reshape(n, dim).astype(np.float64)
    qr = np.argsort(np.argsort(q, kind="stable"), kind="stable").astype(np.float64)
    s, i = orc.rank_search(ranks.astype(np.uint16), n, dim, q, n)
    rho = np.array([np.corrcoef(qr, ranks[d])[0, 1] for d in range(n)])
    assert np.allclose(s[0], rho[i[0]], atol=1e-6)
    s, i = orc.rank_search(ranks.astype(np.uint16), n, dim, q, n, asymmetric=True)
    qu = q.astype(np.float64) / np.linalg.norm(q.astype(np.float64))
    cen = ranks - (dim - 1) / 2.0
    cos = cen @ qu / np.sqrt(dim * (dim * dim - 1) / 12.0)
    assert np.allclose(s[0], cos[i[0]], atol=1e-5)


def test_rankquant_symmetric_scores_are_exact_centre_products(orc):
    """RankQuant::search (src/quant.rs:629-695): the LUT sum of
    centre(q_bucket) * centre(d_bucket) is a multiple of 1/4 below 2^22 quarters,
    so the f32 score is exactly f32(sum) * f32(1 / norm^2), one rounding."""
    rng = np.random.default_rng(8)
    dim, n = 128, 50
    docs = rng.standard_normal((n, dim)).astype(np.float32)
    q = rng.standard_normal(dim).astype(np.float32)
    for bits in (1, 2, 4):
        packed = orc.rankquant_encode(docs, dim, bits)
        s, i = orc.rq_search_sym(packed, n, dim, bits, q, n)
        codes = np.stack([orc.unpack_buckets(packed[r * dim * bits // 8:(r + 1) * dim * bits // 8], dim, bits)
                          for r in range(n)]).astype(np.float64)
        qb = orc.unpack_buckets(orc.rankquant_encode(q, dim, bits), dim, bits).astype(np.float64)
        c = ((1 << bits) - 1) / 2.0
        dot = (codes - c) @ (qb - c)
        nb = float(1 << bits)
        norm = np.float32(np.sqrt(dim * ((nb * nb - 1.0) / 12.0)))
        inv_sq = np.float32(1.0) / (norm * norm)
        want = (dot.astype(np.float32) * inv_sq).astype(np.float32)
        assert np.array_equal(s[0], want[i[0]]), bits
        order = sorted(range(n), key=lambda d: (-want[d], d))
        assert i[0].tolist() == order, bits


def test_rank_transform_is_a_stable_argsort_with_signed_zero_ties(orc):
    """src/rank.rs:38-53 with cmp_finite_f32_then_index (src/util.rs:19-30):
    equal values (-0.0 == +0.0 included) take ranks in index order.  numpy's
    stable argsort orders -0.0 and +0.0 as equal too."""
    rng = np.random.default_rng(11)
    for d in (2, 8, 64, 768, 1024, 4096):
        for trial in range(12):
            v = rng.standard_normal(d).astype(np.float32)
            if trial % 3 == 0:
                v = np.round(v * 2) / 2  # heavy ties
            if trial % 4 == 0:
                v[::5] = -0.0
                v[1::7] = 0.0
            order = np.argsort(v, kind="stable")
            want = np.empty(d, np.uint16)
            want[order] = np.arange(d)
            assert np.array_equal(orc.rank_transform(v), want), (d, trial)


def test_one_pass_encoder_equals_the_separate_encoders(orc):
    docs = orc.synth_docs(5, 700, 768)
    words = np.empty(700 * 12, np.uint64)
    packed = np.empty(700 * 192, np.uint8)
    orc.encode_bitmap_rankquant(docs, 768, 192, 2, words, packed)
    assert np.array_equal(words, orc.bitmap_encode(docs, 768, 192))
    assert np.array_equal(packed, orc.rankquant_encode(docs, 768, 2))
    p4 = np.empty(700 * 384, np.uint8)
    orc.encode_bitmap_rankquant(docs, 768, 100, 4, None, p4)
    assert np.array_equal(p4, orc.rankquant_encode(docs, 768, 4))


def test_cpu_bitmap_two_stage_equals_the_scalar_oracle(orc):
    """The timed CPU restatement (groups of 8 queries on the AVX-512 batched
    scan, then the AVX-512 rerank) against the scalar checker: candidate rows
    bit-exact in (overlap desc, id asc) order, including a final group of 3
    queries; reranked ids equal to the FP64 ordering except within the float
    tolerance."""
    n, dim, n_top, nq, m, k = 9000, 768, 192, 19, 400, 20
    docs = orc.synth_docs(9, n, dim)
    qs, _ = orc.synth_queries(9, n, nq, dim)
    words = orc.bitmap_encode(docs, dim, n_top)
    packed = orc.rankquant_encode(docs, dim, 2)
    s, i, cands = orc.cpu_bitmap_two_stage(words, packed, n, dim, n_top, 2, qs, m, k, 4, want_candidates=True)
    for qi in range(nq):
        want = orc.bitmap_top_m(words, n, dim, n_top, qs[qi], m)
        assert np.array_equal(cands[qi], want), qi
        s64 = orc.rq_scores_f64_subset(packed, dim, 2, qs[qi], want)
        order = np.lexsort((want, -s64))[:k]
        got64 = orc.rq_scores_f64_subset(packed, dim, 2, qs[qi], i[qi].astype(np.uint32))
        tol = 1e-5 * np.maximum(np.abs(s64[order]), 1e-3)
        assert np.all(np.abs(np.sort(got64)[::-1] - s64[order]) <= tol), qi
        np.testing.assert_allclose(s[qi], got64, rtol=1e-5, atol=1e-6)
