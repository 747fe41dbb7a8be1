"""GPU parity: the sm_100a path against the CPU oracle on the same inputs.

Bars (ordvec's determinism contract, docs/determinism.md):
* integer / byte paths (encoders, sign Hamming, bitmap overlap, FastScan
  accumulators and its fixed f32 score, multi-bucket diagonal/outer sums):
  bit-exact, tie order included;
* float asymmetric scores: |s - s64| <= 1e-5 * max(|s64|, 1e-3) against the
  FP64 oracle, ids identical except between entries whose FP64 scores differ by
  less than that tolerance.
"""
import ctypes as C
import os

import numpy as np
import pytest

import ordvec_b200 as ob
from ordvec_b200 import abi
from ordvec_b200._lib import SearchStats, lib

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "tiled_candgen.npz")
REL = 1e-5


def tol(s):
    return REL * max(abs(float(s)), 1e-3)


def check_float_topk(got_ids, got_scores, cand_ids, s64, k):
    """got vs the FP64 ranking of (cand_ids, s64) with ties by id."""
    cand_ids = np.asarray(cand_ids, np.int64)
    order = sorted(range(len(cand_ids)), key=lambda j: (-s64[j], cand_ids[j]))[:k]
    want = cand_ids[order]
    score_of = {}
    for cid, s in zip(cand_ids, s64):
        score_of.setdefault(int(cid), float(s))
    got_ids = np.asarray(got_ids, np.int64)
    assert len(got_ids) == len(want)
    for j, (g, w) in enumerate(zip(got_ids, want)):
        sg = score_of[int(g)]
        assert abs(float(got_scores[j]) - sg) <= tol(sg), (j, got_scores[j], sg)
        if g != w:
            sw = score_of[int(w)]
            assert abs(sg - sw) <= tol(sw), ("id mismatch beyond tolerance", j, g, w, sg, sw)
    return want


@pytest.fixture(scope="module")
def corpus():
    docs = ob.synth_docs(0x0DD5EED1, 5000, 1024)
    queries, _ = ob.synth_queries(0x0DD5EED1, 5000, 8, 1024)
    return docs, queries


# ---------------------------------------------------------------- encoders
@pytest.mark.parametrize("dim", [64, 128, 768, 1024])
def test_encoders_match_oracle(orc, dim):
    rng = np.random.default_rng(dim)
    docs = rng.standard_normal((700, dim)).astype(np.float32)
    docs[::7, : dim // 2] = 0.5  # heavy ties
    docs[::11, :] = 0.0
    docs[3, ::3] = -0.0
    docs[5] = np.tile(np.float32([1.0, -0.0, 0.0, -1.0]), dim // 4)
    for bits in (1, 2, 4):
        rq = ob.RankQuant(dim, bits)
        rq.add(docs[:300])
        rq.add(docs[300:])  # incremental add
        assert np.array_equal(rq.payload(), orc.rankquant_encode(docs, dim, bits)), bits
    sb = ob.SignBitmap(dim)
    sb.add(docs)
    assert np.array_equal(sb.payload().view(np.uint64), orc.sign_encode(docs, dim))
    bm = ob.Bitmap(dim, dim // 4)
    bm.add(docs)
    assert np.array_equal(bm.payload().view(np.uint64), orc.bitmap_encode(docs, dim, dim // 4))
    fs = ob.RankQuantFastscan(dim)
    fs.add(docs)
    assert np.array_equal(fs.payload(), orc.fastscan_pack(docs, dim))
    mb = ob.MultiBucketBitmap(dim, 2)
    mb.add(docs)
    assert np.array_equal(mb.payload().view(np.uint64), orc.multibucket_encode(docs, dim, 2))


def test_fastscan_odd_pair_counts_encode(orc):
    for dim in (4, 20, 100, 132):
        docs = np.random.default_rng(dim).standard_normal((45, dim)).astype(np.float32)
        fs = ob.RankQuantFastscan(dim)
        fs.add(docs)
        assert np.array_equal(fs.payload(), orc.fastscan_pack(docs, dim)), dim


# ------------------------------------------------------- golden candgen
def test_golden_tiled_candgen(orc):
    """tests/tiled_candgen.rs cases against the committed sort-oracle rows."""
    g = np.load(GOLDEN)
    names = sorted({k.split("__")[0] for k in g.files})
    for name in names:
        meta = [int(x) for x in g[f"{name}__meta"]]
        dim, cn, cseed, qn, qseed, kind = meta[:6]
        if kind == 0:
            vec = orc.xorshift_f32(cseed, cn * dim)
        elif kind == 1:
            d = np.arange(cn)[:, None] % 4
            vec = np.where((np.arange(dim)[None, :] + d) % 3 == 0, -1.0, 1.0).astype(np.float32).reshape(-1)
        else:
            vec = np.tile(orc.xorshift_f32(cseed, cn * dim), 512)
        qs = orc.xorshift_f32(qseed, qn * dim)
        n = vec.size // dim
        sb = ob.SignBitmap(dim)
        sb.add(vec)
        exp = g[f"{name}__expected"]
        for m in meta[6:]:
            me = min(m, n)
            cb = sb.top_m_candidates_batched_serial_csr(qs, m)
            assert cb.offsets.tolist() == [i * me for i in range(qn + 1)]
            for qi in range(qn):
                assert np.array_equal(cb.candidates_for_query(qi), exp[qi, :me]), (name, m, qi)
    sb = ob.SignBitmap(64)
    sb.add(orc.xorshift_f32(0x42, 17 * 64))
    cb = sb.top_m_candidates_batched_serial_csr(np.zeros(0, np.float32), 8)
    assert cb.offsets.tolist() == [0] and cb.candidates.size == 0


# ------------------------------------------------ determinism contract
def test_determinism_contract_literals():
    """tests/determinism_contract.rs:15-184 through the GPU path."""
    dim = 64
    docs = np.ones((8, dim), np.float32)
    zero = np.zeros(dim, np.float32)
    rq = ob.RankQuant(dim, 2)
    rq.add(docs)
    r = rq.search_asymmetric(zero, 4)
    assert r.indices_for_query(0).tolist() == [0, 1, 2, 3] and (r.scores == 0.0).all()
    bm = ob.Bitmap(dim, dim // 4)
    bm.add(docs)
    r = bm.search(np.ones(dim, np.float32), 4)
    assert r.indices_for_query(0).tolist() == [0, 1, 2, 3] and (r.scores == r.scores[0]).all()
    rq12 = ob.RankQuant(dim, 2)
    rq12.add(np.ones((12, dim), np.float32))
    s, i = rq12.search_asymmetric_subset(zero, [9, 3, 7, 1], 2)
    assert s.tolist() == [0.0, 0.0] and i.tolist() == [1, 3]
    s, i = rq12.search_asymmetric_subset(zero, [7, 8, 7], 2)
    assert i.tolist() == [7, 7]
    r = rq12.search_asymmetric_subset_batched_serial(zero, [0, 4], [7, 7, 3, 7], 4)
    assert r.scores.tolist() == [0.0] * 4 and r.indices.tolist() == [3, 7, 7, 7]
    ten = np.ones((10, dim), np.float32)
    q2 = np.ones((2, dim), np.float32)
    bm10 = ob.Bitmap(dim, dim // 4)
    bm10.add(ten)
    assert bm10.top_m_candidates(q2[0], 5).tolist() == [0, 1, 2, 3, 4]
    assert [r.tolist() for r in bm10.top_m_candidates_batched(q2, 5)] == [[0, 1, 2, 3, 4]] * 2
    sb = ob.SignBitmap(dim)
    sb.add(ten)
    assert [r.tolist() for r in sb.top_m_candidates_batched(q2, 5)] == [[0, 1, 2, 3, 4]] * 2
    for bits in (1, 2, 4):
        z = ob.RankQuant(dim, bits)
        z.add(np.zeros((6, dim), np.float32))
        assert z.search_asymmetric(zero, 6).indices.tolist() == [0, 1, 2, 3, 4, 5]
    empty = ob.RankQuant(dim, 2)
    r = empty.search_asymmetric(np.ones(dim, np.float32), 10)
    assert r.k == 0 and r.scores.size == 0
    two = ob.RankQuant(dim, 2)
    two.add(np.ones((2, dim), np.float32))
    assert two.search_asymmetric(np.ones(dim, np.float32), 0).k == 0


# ---------------------------------------------------- C ABI v1 fixtures
def _fixture_files(tmp_path):
    rq = ob.RankQuant(16, 2)
    rq.add(np.tile(np.arange(16, dtype=np.float32), 4))
    p_rq = str(tmp_path / "rq.ovrq")
    rq.write(p_rq)
    doc = np.zeros(64, np.float32)
    doc[:4] = 10.0 + np.arange(4)
    bm = ob.Bitmap(64, 4)
    bm.add(np.tile(doc, 4))
    p_bm = str(tmp_path / "bm.ovbm")
    bm.write(p_bm)
    return p_rq, p_bm, doc


def test_abi_v1_fixture_searches(tmp_path):
    """ordvec-ffi/src/lib.rs:1087-1271."""
    small = ob.RankQuant(8, 2)
    small.add(np.arange(8, dtype=np.float32))
    small.write(str(tmp_path / "g.ovrq"))
    assert open(tmp_path / "g.ovrq", "rb").read() == b"OVRQ" + bytes([1, 2, 8, 0, 0, 0, 1, 0, 0, 0, 0x05, 0xAF])
    p_rq, p_bm, doc = _fixture_files(tmp_path)
    L = lib()
    h = abi.index_load(p_rq)
    try:
        info = ob._lib.IndexInfo()
        L.ordvec_index_info_init(C.byref(info))
        assert L.ordvec_index_info(h, C.byref(info)) == 0
        assert (info.kind, info.format_version, info.dim, info.bit_width, info.vector_count) == (1, 1, 16, 2, 4)
        q = np.arange(16, dtype=np.float32)
        stats = SearchStats()
        L.ordvec_search_stats_init(C.byref(stats))
        hits = abi.index_search(h, q, 2, user_tag=77, stats=stats)
        assert len(hits) == 2 and hits[0][0] == 0 and hits[0][0] == hits[0][1]
        assert (stats.user_tag, stats.candidate_count, stats.vectors_scored) == (77, 4, 4)
        assert [x[0] for x in abi.index_search(h, q, 2, candidates=[3, 1, 2])] == [1, 2]
        stats = SearchStats()
        L.ordvec_search_stats_init(C.byref(stats))
        assert [x[0] for x in abi.index_search(h, q, 3, candidates=[3, 1, 1, 2], stats=stats)] == [1, 1, 2]
        assert (stats.candidate_count, stats.vectors_scored) == (4, 4)
    finally:
        L.ordvec_index_free(h)
    h = abi.index_load(p_bm)
    try:
        assert [x[0] for x in abi.index_search(h, doc, 3, candidates=[3, 1, 1, 2])] == [1, 1, 2]
        hits = abi.index_search(h, doc, 4)
        assert [x[0] for x in hits] == [0, 1, 2, 3] and all(x[2] == 4.0 for x in hits)
    finally:
        L.ordvec_index_free(h)


def test_abi_v1_validation_failures(tmp_path):
    """ordvec-ffi/src/lib.rs:1273-1500 statuses, same order."""
    p_rq, _, _ = _fixture_files(tmp_path)
    L = lib()
    h = abi.index_load(p_rq)
    P = ob._lib.SearchParams
    Hit = ob._lib.Hit
    q = np.ones(16, np.float32)
    base = P()
    L.ordvec_search_params_init(C.byref(base))
    base.query = q.ctypes.data_as(C.POINTER(C.c_float))
    base.dim, base.k = 16, 1
    hits = (Hit * 1)()
    ret = C.c_uint64()

    def run(p, hits_ptr=hits, cap=1, ret_ptr=C.byref(ret), stats=None, handle=h):
        return L.ordvec_index_search(handle, C.byref(p) if p is not None else None, hits_ptr, cap, ret_ptr, stats)

    def mod(**kw):
        p = P.from_buffer_copy(base)
        for k, v in kw.items():
            setattr(p, k, v)
        return p

    try:
        assert run(base, handle=None) == 1
        assert run(None) == 1
        assert run(mod(struct_size=127)) == 3
        assert run(mod(flags=1)) == 2
        bad = mod()
        bad.reserved[0] = 1
        assert run(bad) == 2
        assert run(mod(query=None)) == 1
        assert run(mod(dim=15)) == 7
        nan = q.copy()
        nan[0] = np.nan
        assert run(mod(query=nan.ctypes.data_as(C.POINTER(C.c_float)))) == 8
        assert run(base, ret_ptr=None) == 1
        assert run(base, hits_ptr=None) == 1
        assert run(base, cap=0) == 10
        c99 = np.array([99], np.uint32)
        assert run(mod(candidate_rows=c99.ctypes.data_as(C.POINTER(C.c_uint32)), candidate_count=1)) == 9
        assert run(mod(candidate_rows=c99.ctypes.data_as(C.POINTER(C.c_uint32)), candidate_count=0),
                   hits_ptr=None, cap=0) == 2
        assert run(mod(candidate_count=1), hits_ptr=None, cap=0) == 1
        ret.value = 42
        assert run(mod(k=0), hits_ptr=None, cap=0) == 0 and ret.value == 0
        st = SearchStats()
        L.ordvec_search_stats_init(C.byref(st))
        st.struct_size = 183
        assert run(base, stats=C.byref(st)) == 3
    finally:
        L.ordvec_index_free(h)


# -------------------------------------------------- RankQuant float paths
@pytest.mark.parametrize("dim,bits", [(1024, 1), (1024, 2), (1024, 4), (768, 2), (64, 4), (20, 2), (48, 4), (8, 1)])
def test_rankquant_search_matches_fp64(orc, dim, bits):
    n, nq = 3000, 6
    docs = ob.synth_docs(11, n, dim)
    queries, _ = ob.synth_queries(11, n, nq, dim)
    rq = ob.RankQuant(dim, bits)
    rq.add(docs)
    packed = orc.rankquant_encode(docs, dim, bits)
    assert np.array_equal(rq.payload(), packed)
    for k in (10, 100):
        res = rq.search_asymmetric(queries, k)
        for qi in range(nq):
            s64 = orc.rq_scores_f64(packed, n, dim, bits, queries[qi])
            check_float_topk(res.indices_for_query(qi), res.scores_for_query(qi), np.arange(n), s64, k)


def _split_bound(dim, bits, q):
    """The split-BF16 error bound the library states (scan_rank_tc.cu)."""
    qn = np.asarray(q, np.float64)
    qn = qn / np.sqrt((qn * qn).sum())
    inv_norm = 1.0 / np.sqrt(dim * ((4.0 ** bits - 1.0) / 12.0))
    cmax = (2 ** bits - 1) / 2
    return inv_norm * cmax * (2 * dim * 2.0 ** -24 + 2.0 ** -16) * 1.05 * np.abs(qn).sum()


@pytest.mark.parametrize("dim,bits,n", [(1024, 2, 20_000), (1024, 1, 9_000), (768, 4, 7_000), (128, 2, 5_000)])
def test_split_bf16_rank_scan(orc, monkeypatch, dim, bits, n):
    """Tensor-core split-BF16 full search: the exact form (default for >= 64
    queries) meets the FP64 bar; the raw split scores stay within the stated
    error bound; forcing the path on and off changes nothing."""
    nq = 80
    docs = ob.synth_docs(13 + bits, n, dim)
    queries, _ = ob.synth_queries(13 + bits, n, nq, dim)
    rq = ob.RankQuant(dim, bits)
    rq.add(docs)
    packed = orc.rankquant_encode(docs, dim, bits)
    for k in (10, 100):
        res = rq.search_asymmetric(queries, k)
        raw = rq.search_asymmetric_split(queries, k, exact=False)
        worst = 0.0
        for qi in (0, 1, 41, 79):
            s64 = orc.rq_scores_f64(packed, n, dim, bits, queries[qi])
            check_float_topk(res.indices_for_query(qi), res.scores_for_query(qi), np.arange(n), s64, k)
            err = np.abs(raw.scores_for_query(qi).astype(np.float64) - s64[raw.indices_for_query(qi)])
            worst = max(worst, err.max())
            assert err.max() <= _split_bound(dim, bits, queries[qi]), (qi, err.max())
        print(f"split-BF16 dim {dim} b{bits} k {k}: max |split - fp64| = {worst:.3e}")
    monkeypatch.setenv("OVB_RANK_TC", "1")
    a = rq.search_asymmetric(queries[:5], 10)
    monkeypatch.setenv("OVB_RANK_TC", "0")
    b = rq.search_asymmetric(queries[:5], 10)
    assert np.array_equal(a.indices, b.indices)


@pytest.mark.parametrize("bits", [1, 2, 4])
def test_split_bf16_threshold_filter(orc, monkeypatch, bits):
    """Split-BF16 search through the sample-threshold filter (kept docs only,
    no key matrix) returns the key-matrix path's exact top-k, and the oracle's."""
    n, dim, nq = 120_000, 256, 200
    docs = ob.synth_docs(83 + bits, n, dim)
    queries, _ = ob.synth_queries(83 + bits, n, nq, dim)
    rq = ob.RankQuant(dim, bits)
    rq.add(docs)
    packed = orc.rankquant_encode(docs, dim, bits)
    for k in (10, 100):
        filt = rq.search_asymmetric(queries, k)
        monkeypatch.setenv("OVB_SPLIT_FILTER", "0")
        dense = rq.search_asymmetric(queries, k)
        monkeypatch.delenv("OVB_SPLIT_FILTER")
        assert np.array_equal(filt.indices, dense.indices)
        assert np.array_equal(filt.scores.view(np.uint32), dense.scores.view(np.uint32))
        for qi in (0, nq - 1):
            s64 = orc.rq_scores_f64(packed, n, dim, bits, queries[qi])
            check_float_topk(filt.indices_for_query(qi), filt.scores_for_query(qi), np.arange(n), s64, k)


def test_rankquant_large_k_uses_global_select(orc):
    dim, bits, n = 128, 2, 9000
    docs = ob.synth_docs(5, n, dim)
    q, _ = ob.synth_queries(5, n, 2, dim)
    rq = ob.RankQuant(dim, bits)
    rq.add(docs)
    packed = orc.rankquant_encode(docs, dim, bits)
    res = rq.search_asymmetric(q, 6000)
    for qi in range(2):
        s64 = orc.rq_scores_f64(packed, n, dim, bits, q[qi])
        check_float_topk(res.indices_for_query(qi), res.scores_for_query(qi), np.arange(n), s64, 6000)


def test_subset_batched_matches_oracle(orc, corpus):
    docs, queries = corpus
    n, dim = docs.shape
    rng = np.random.default_rng(3)
    for bits in (1, 2, 4):
        rq = ob.RankQuant(dim, bits)
        rq.add(docs)
        packed = orc.rankquant_encode(docs, dim, bits)
        rows = [rng.integers(0, n, 40), np.array([], np.int64), rng.integers(0, n, 3),
                np.array([17, 17, 17, 4]), rng.integers(0, n, 700), rng.integers(0, n, 5),
                rng.permutation(n)[:200], rng.integers(0, n, 1)]
        off = np.cumsum([0] + [len(r) for r in rows]).astype(np.uint64)
        cand = np.concatenate(rows).astype(np.uint32)
        k = 7
        res = rq.search_asymmetric_subset_batched_serial(queries, off, cand, k)
        assert res.k == k
        for qi, row in enumerate(rows):
            got_i, got_s = res.indices_for_query(qi), res.scores_for_query(qi)
            if len(row) == 0:
                assert got_i.tolist() == [-1] * k and np.isneginf(got_s).all()
                continue
            s64 = orc.rq_scores_f64_subset(packed, dim, bits, queries[qi], row.astype(np.uint32))
            m = min(k, len(row))
            check_float_topk(got_i[:m], got_s[:m], row, s64, m)
            assert got_i[m:].tolist() == [-1] * (k - m)


def test_nonfinite_queries_are_rejected(corpus):
    docs, queries = corpus
    rq = ob.RankQuant(1024, 2)
    rq.add(docs[:100])
    bad = queries.copy()
    bad[1, 5] = np.inf
    with pytest.raises(ob.OrdvecError) as e:
        rq.search_asymmetric(bad, 5)
    assert e.value.status == 8
    # a batch above the host-checked size takes the device check
    big = np.tile(queries, (16, 1))
    big[100, 7] = np.nan
    with pytest.raises(ob.OrdvecError) as e:
        rq.search_asymmetric(big, 5)
    assert e.value.status == 8
    assert rq.search_asymmetric(big[:64], 5).k == 5


# ---------------------------------------------------------------- FastScan
@pytest.mark.parametrize("dim,n", [(1024, 5000), (64, 65), (100, 777), (768, 2049)])
def test_fastscan_search_is_bit_exact(orc, dim, n):
    docs = ob.synth_docs(21, n, dim)
    queries, _ = ob.synth_queries(21, n, 5, dim)
    fs = ob.RankQuantFastscan(dim)
    fs.add(docs)
    blocks = orc.fastscan_pack(docs, dim)
    k = min(300, n)
    res = fs.search(queries, k)
    s_ref, i_ref = orc.fastscan_search(blocks, n, dim, queries, k)
    assert np.array_equal(res.indices.reshape(5, k), i_ref)
    assert np.array_equal(res.scores.reshape(5, k).view(np.uint32), s_ref.view(np.uint32))


@pytest.mark.parametrize("dim,n,nq", [(100, 777, 40), (1024, 5000, 300), (64, 65, 33)])
def test_fastscan_tensor_core_path_is_bit_exact(orc, monkeypatch, dim, n, nq):
    """The tcgen05 one-hot GEMM form (>= 32 queries) against the oracle and the
    CUDA-core form: identical ids and score bits, partial query tiles included."""
    docs = ob.synth_docs(23, n, dim)
    queries, _ = ob.synth_queries(23, n, nq, dim)
    fs = ob.RankQuantFastscan(dim)
    fs.add(docs)
    k = min(100, n)
    monkeypatch.setenv("OVB_FASTSCAN_TC", "1")
    tc = fs.search(queries, k)
    monkeypatch.setenv("OVB_FASTSCAN_TC", "0")
    cc = fs.search(queries, k)
    assert np.array_equal(tc.indices, cc.indices)
    assert np.array_equal(tc.scores.view(np.uint32), cc.scores.view(np.uint32))
    s_ref, i_ref = orc.fastscan_search(orc.fastscan_pack(docs, dim), n, dim, queries[:4], k)
    assert np.array_equal(tc.indices.reshape(nq, k)[:4], i_ref)
    assert np.array_equal(tc.scores.reshape(nq, k)[:4].view(np.uint32), s_ref.view(np.uint32))


def _fastscan_modes(monkeypatch, fs, queries, k, **env):
    """Search once per environment setting; returns the results in order."""
    out = []
    for name, settings in env.items():
        for var in ("OVB_FASTSCAN_TC", "OVB_FASTSCAN_FILTER", "OVB_FASTSCAN_SAMPLE_MULT"):
            monkeypatch.delenv(var, raising=False)
        for var, val in settings.items():
            monkeypatch.setenv(var, val)
        out.append(fs.search(queries, k))
    for var in ("OVB_FASTSCAN_TC", "OVB_FASTSCAN_FILTER", "OVB_FASTSCAN_SAMPLE_MULT"):
        monkeypatch.delenv(var, raising=False)
    return out


def _same(a, b):
    assert np.array_equal(a.indices, b.indices)
    assert np.array_equal(a.scores.view(np.uint32), b.scores.view(np.uint32))


@pytest.mark.parametrize(
    "dim,n,nq,k,mult",
    [
        (256, 40_000, 70, 200, None),    # sample stride 4
        (256, 39_950, 40, 64, None),     # last (partial) block is sampled
        (100, 70_001, 300, 333, None),   # two query tiles, odd pair count
        (256, 40_000, 70, 200, "0.02"),  # threshold too tight -> dense redo
        (256, 40_000, 70, 200, "1e6"),   # threshold keeps all -> over capacity -> dense redo
    ],
)
def test_fastscan_threshold_filter_is_exact(orc, monkeypatch, dim, n, nq, k, mult):
    """Sample-threshold filter (TC scan keeping only keys <= a per-query
    threshold) returns exactly the key-matrix result, ids and score bits, and
    its fallback does too."""
    docs = ob.synth_docs(29, n, dim)
    queries, _ = ob.synth_queries(29, n, nq, dim)
    fs = ob.RankQuantFastscan(dim)
    fs.add(docs)
    filt = {"OVB_FASTSCAN_TC": "1", "OVB_FASTSCAN_FILTER": "1"}
    if mult:
        filt["OVB_FASTSCAN_SAMPLE_MULT"] = mult
    f, d, c = _fastscan_modes(
        monkeypatch, fs, queries, k,
        filt=filt,
        dense={"OVB_FASTSCAN_TC": "1", "OVB_FASTSCAN_FILTER": "0"},
        cuda_core={"OVB_FASTSCAN_TC": "0"},
    )
    _same(f, d)
    _same(f, c)
    s_ref, i_ref = orc.fastscan_search(orc.fastscan_pack(docs, dim), n, dim, queries[:3], k)
    assert np.array_equal(f.indices.reshape(nq, k)[:3], i_ref)
    assert np.array_equal(f.scores.reshape(nq, k)[:3].view(np.uint32), s_ref.view(np.uint32))


def test_fastscan_threshold_filter_heavy_ties(orc, monkeypatch):
    """500 distinct rows tiled 80x: the top-k is decided by doc id among equal
    keys; the filter path keeps every tie and orders them like the oracle."""
    dim, base, reps, nq, k = 128, 500, 80, 48, 150
    distinct = ob.synth_docs(37, base, dim)
    docs = np.tile(distinct, (reps, 1))
    n = base * reps
    queries, _ = ob.synth_queries(37, base, nq, dim)
    fs = ob.RankQuantFastscan(dim)
    fs.add(docs)
    f, d = _fastscan_modes(
        monkeypatch, fs, queries, k,
        filt={"OVB_FASTSCAN_TC": "1", "OVB_FASTSCAN_FILTER": "1"},
        dense={"OVB_FASTSCAN_TC": "1", "OVB_FASTSCAN_FILTER": "0"},
    )
    _same(f, d)
    s_ref, i_ref = orc.fastscan_search(orc.fastscan_pack(docs, dim), n, dim, queries[:2], k)
    assert np.array_equal(f.indices.reshape(nq, k)[:2], i_ref)
    assert np.array_equal(f.scores.reshape(nq, k)[:2].view(np.uint32), s_ref.view(np.uint32))


def test_fastscan_reference_formula_corpus(orc):
    """src/fastscan.rs:755-777 corpus (dim 64, n 65, k 9) including a zero query."""
    dim, n, k = 64, 65, 9
    docs = ((((np.arange(n * dim) * 37 + 11) % 257).astype(np.float32) - 128.0) / 128.0).astype(np.float32)
    qs = ((((np.arange(3 * dim) * 19 + 5) % 193).astype(np.float32) - 96.0) / 96.0).astype(np.float32)
    qs = np.concatenate([qs, np.zeros(dim, np.float32)])
    fs = ob.RankQuantFastscan(dim)
    fs.add(docs)
    res = fs.search(qs, k)
    s_ref, i_ref = orc.fastscan_search(orc.fastscan_pack(docs, dim), n, dim, qs, k)
    assert np.array_equal(res.indices.reshape(4, k), i_ref)
    assert np.array_equal(res.scores.reshape(4, k).view(np.uint32), s_ref.view(np.uint32))


def test_fastscan_full_size_property(orc):
    """171,332 docs x dim 1024 (the FastScan two-stage configuration's corpus):
    top-1000 candidate ids and scores bit-identical to the oracle."""
    n, dim = 171_332, 1024
    docs = ob.synth_docs(0x0DD5EED2, n, dim)
    queries, _ = ob.synth_queries(0x0DD5EED2, n, 3, dim)
    fs = ob.RankQuantFastscan(dim)
    fs.add(docs)
    blocks = fs.payload()
    res = fs.search(queries, 1000)
    s_ref, i_ref = orc.fastscan_search(blocks, n, dim, queries, 1000)
    assert np.array_equal(res.indices.reshape(3, 1000), i_ref)
    assert np.array_equal(res.scores.reshape(3, 1000).view(np.uint32), s_ref.view(np.uint32))


def test_fastscan_full_size_batched_filter(orc, monkeypatch):
    """171,332 docs x dim 1024, 300 queries, m = 1000 (the batched two-stage
    candidate step): the default path (TC scan + threshold filter) equals the
    key-matrix path bit for bit, and the oracle on a few rows."""
    n, dim, nq, m = 171_332, 1024, 300, 1000
    docs = ob.synth_docs(0x0DD5EED2, n, dim)
    queries, _ = ob.synth_queries(0x0DD5EED2, n, nq, dim)
    fs = ob.RankQuantFastscan(dim)
    fs.add(docs)
    f, d = _fastscan_modes(
        monkeypatch, fs, queries, m,
        default={},
        dense={"OVB_FASTSCAN_FILTER": "0"},
    )
    _same(f, d)
    s_ref, i_ref = orc.fastscan_search(fs.payload(), n, dim, queries[:2], m)
    assert np.array_equal(f.indices.reshape(nq, m)[:2], i_ref)
    assert np.array_equal(f.scores.reshape(nq, m)[:2].view(np.uint32), s_ref.view(np.uint32))


# ------------------------------------------------------------ Bitmap / sign
def test_bitmap_search_top_m_and_subset_exact(orc):
    n, dim, n_top = 3000, 768, 192
    docs = ob.synth_docs(31, n, dim)
    queries, _ = ob.synth_queries(31, n, 6, dim)
    bm = ob.Bitmap(dim, n_top)
    bm.add(docs)
    words = orc.bitmap_encode(docs, dim, n_top)
    res = bm.search(queries, 50)
    s_ref, i_ref = orc.bitmap_search(words, n, dim, n_top, queries, 50)
    assert np.array_equal(res.indices.reshape(6, 50), i_ref) and np.array_equal(res.scores.reshape(6, 50), s_ref)
    got = bm.top_m_candidates_batched(queries, 500)
    for qi in range(6):
        assert np.array_equal(got[qi], orc.bitmap_top_m(words, n, dim, n_top, queries[qi], 500))
    ids = np.random.default_rng(0).integers(0, n, 300).astype(np.uint32)
    s, i = bm.search_subset(queries[0], ids, 20)
    s_ref, i_ref = orc.bitmap_search_subset(words, n, dim, n_top, queries[0], ids, 20)
    assert i.tolist() == i_ref.tolist() and s.tolist() == s_ref.tolist()


def test_sign_score_all_and_top_m(orc, corpus):
    docs, queries = corpus
    n, dim = docs.shape
    sb = ob.SignBitmap(dim)
    sb.add(docs)
    words = orc.sign_encode(docs, dim)
    ham = orc.sign_hamming_all(words, n, dim, queries[0])
    assert np.array_equal(sb.score_all(queries[0]), dim - ham)
    got = sb.top_m_candidates_batched(queries, 320)
    for qi in range(len(queries)):
        assert np.array_equal(got[qi], orc.sign_top_m(words, n, dim, queries[qi], 320))


_BITMAP_ENV = ("OVB_BITMAP_TC", "OVB_FASTSCAN_FILTER", "OVB_FASTSCAN_SAMPLE_MULT", "OVB_BITMAP_FP4")


def _bitmap_modes(monkeypatch, fn, **env):
    """fn() once per environment setting; returns the results in order."""
    out = []
    for settings in env.values():
        for var in _BITMAP_ENV:
            monkeypatch.delenv(var, raising=False)
        for var, val in settings.items():
            monkeypatch.setenv(var, val)
        out.append(fn())
    for var in _BITMAP_ENV:
        monkeypatch.delenv(var, raising=False)
    return out


_BITMAP_THREE = dict(
    filt={"OVB_BITMAP_TC": "1", "OVB_FASTSCAN_FILTER": "1"},
    dense={"OVB_BITMAP_TC": "1", "OVB_FASTSCAN_FILTER": "0"},
    cuda_core={"OVB_BITMAP_TC": "0"},
)


@pytest.mark.parametrize(
    "dim,n_top,n,nq,m,mult",
    [
        (768, 192, 40_000, 70, 500, None),    # 6 K-blocks, sample stride 4
        (320, 80, 39_950, 40, 300, None),     # odd word count (half K-block), partial last tile
        (64, 16, 70_001, 300, 700, None),     # one word per row, two query tiles, massive key ties
        (768, 192, 40_000, 70, 500, "0.02"),  # threshold too tight -> dense redo
        (768, 192, 40_000, 70, 500, "1e6"),   # keeps everything -> over capacity -> dense redo
    ],
)
def test_bitmap_tensor_core_top_m_is_exact(orc, monkeypatch, dim, n_top, n, nq, m, mult):
    """Constant-weight bitmap candidates from the tensor-core overlap scan
    (sample threshold with a (key, doc) tie bound, and the dense key matrix)
    equal the CUDA-core popcount scan and the oracle, ids in tie order."""
    docs = ob.synth_docs(43, n, dim)
    queries, _ = ob.synth_queries(43, n, nq, dim)
    bm = ob.Bitmap(dim, n_top)
    bm.add(docs)
    env = dict(_BITMAP_THREE)
    if mult:
        env["filt"] = dict(env["filt"], OVB_FASTSCAN_SAMPLE_MULT=mult)
    f, d, c = _bitmap_modes(monkeypatch, lambda: bm.top_m_candidates_batched(queries, m), **env)
    assert np.array_equal(f, d) and np.array_equal(f, c)
    words = orc.bitmap_encode(docs, dim, n_top)
    for qi in (0, nq // 2, nq - 1):
        assert np.array_equal(f[qi], orc.bitmap_top_m(words, n, dim, n_top, queries[qi], m)), qi
    fs, ds = _bitmap_modes(monkeypatch, lambda: bm.search(queries, 50), filt=env["filt"], cuda_core={"OVB_BITMAP_TC": "0"})
    assert np.array_equal(fs.indices, ds.indices) and np.array_equal(fs.scores, ds.scores)


@pytest.mark.parametrize("kind", ["fastscan", "bitmap", "multibucket", "sign"])
def test_cta_pair_scan_matches_single_cta(monkeypatch, kind):
    """The three forms of the tensor-core scans -- one CTA per tile, the
    persistent one-CTA-per-SM kernel, and the persistent CTA-pair kernel
    (cta_group::2, double-buffered accumulators) -- give identical results, on
    the sampled threshold pass, the filter and the dense key matrix, with a
    partial last query tile and a partial last doc tile."""
    n, nq = 70_001, 300
    dim = 256 if kind == "fastscan" else 768
    docs = ob.synth_docs(71, n, dim)
    queries, _ = ob.synth_queries(71, n, nq, dim)
    if kind == "fastscan":
        ix = ob.RankQuantFastscan(dim)
        ix.add(docs)
        run = lambda: ix.search(queries, 333)
    elif kind == "bitmap":
        ix = ob.Bitmap(dim, 192)
        ix.add(docs)
        run = lambda: ix.search(queries, 500)
    elif kind == "sign":
        ix = ob.SignBitmap(dim)
        ix.add(docs)
        run = lambda: np.array(ix.top_m_candidates_batched(queries, 500))
    else:
        ix = ob.MultiBucketBitmap(dim, 2)
        ix.add(docs)
        w = np.eye(4, dtype=np.float32).ravel()
        run = lambda: np.array(ix.top_m_bilinear_batched(queries, w, 500))
    monkeypatch.setenv("OVB_FASTSCAN_TC", "1")
    monkeypatch.setenv("OVB_BITMAP_TC", "1")
    out = {}
    for form in ("tile", "persist", "pair"):
        for filt in ("0", "1"):
            monkeypatch.setenv("OVB_TC_FORM", form)
            monkeypatch.setenv("OVB_FASTSCAN_FILTER", filt)
            out[(form, filt)] = run()
    base = out[("tile", "0")]
    for key, got in out.items():
        if kind in ("multibucket", "sign"):
            assert np.array_equal(got, base), key
        else:
            assert np.array_equal(got.indices, base.indices), key
            assert np.array_equal(got.scores.view(np.uint32), base.scores.view(np.uint32)), key


@pytest.mark.parametrize("kind", ["bitmap", "sign"])
def test_cta_pair_scan_over_query_chunks(monkeypatch, kind):
    """More than 1,024 queries in one call: the CTA-pair kernel stages every
    query's parameters in shared memory and runs query chunks of 1,024; its
    results equal the one-CTA-per-tile kernel's (filter and dense key matrix),
    on a corpus large enough for whole doc tiles per CTA pair and on one small
    enough for the interleaved tile order."""
    for n in (150_000, 9_000):
        dim = 768
        docs = ob.synth_docs(73, n, dim)
        queries, _ = ob.synth_queries(73, n, 1300, dim)
        ix = ob.Bitmap(dim, 192) if kind == "bitmap" else ob.SignBitmap(dim)
        ix.add(docs)
        monkeypatch.setenv("OVB_BITMAP_TC", "1")
        out = {}
        for form in ("tile", "pair"):
            for filt in ("0", "1"):
                monkeypatch.setenv("OVB_TC_FORM", form)
                monkeypatch.setenv("OVB_FASTSCAN_FILTER", filt)
                out[(form, filt)] = np.array(ix.top_m_candidates_batched(queries, 400))
        base = out[("tile", "0")]
        for key, got in out.items():
            assert np.array_equal(got, base), (n, key)


@pytest.mark.parametrize("kind", ["bitmap", "sign", "multibucket"])
def test_bitmap_fp4_filter_matches_int8(orc, monkeypatch, kind):
    """The bitmap filter on the FP4 tensor cores (bits as e2m1 1.0, unit block
    scales, f32 accumulators) keeps exactly the candidates of the int8 scan:
    query counts giving one to six balanced query tiles of <= 224 columns
    (1,300 queries: two launches), rows of 1 to 16 words, a corpus with whole
    doc tiles per CTA pair (A built once per doc tile) and one small enough for
    the interleaved tile order."""
    cases = {
        "bitmap": [(768, 150_000, 1), (768, 150_000, 225), (768, 100_000, 1024), (1024, 9_000, 449), (64, 100_000, 300),
                   (320, 100_000, 1300)],
        "sign": [(768, 100_000, 300), (1024, 9_000, 64), (192, 100_000, 700)],
        "multibucket": [(64, 100_000, 300), (128, 9_000, 250)],
    }[kind]
    for dim, n, nq in cases:
        docs = ob.synth_docs(97, n, dim)
        queries, _ = ob.synth_queries(97, n, nq, dim)
        if kind == "bitmap":
            ix = ob.Bitmap(dim, dim // 4)
            ix.add(docs)
            run = lambda: np.array(ix.top_m_candidates_batched(queries, 400))
        elif kind == "sign":
            ix = ob.SignBitmap(dim)
            ix.add(docs)
            run = lambda: np.array(ix.top_m_candidates_batched(queries, 400))
        else:
            ix = ob.MultiBucketBitmap(dim, 2)
            ix.add(docs)
            w = np.eye(4, dtype=np.float32).ravel()
            run = lambda: np.array(ix.top_m_bilinear_batched(queries, w, 400))
        on = {"OVB_BITMAP_TC": "1", "OVB_FASTSCAN_FILTER": "1", "OVB_TC_FORM": "pair"}
        f4, i8 = _bitmap_modes(monkeypatch, run, fp4=on, int8=dict(on, OVB_BITMAP_FP4="0"))
        monkeypatch.delenv("OVB_TC_FORM", raising=False)
        assert np.array_equal(f4, i8), (dim, n, nq)
        if kind == "bitmap":
            words = orc.bitmap_encode(docs, dim, dim // 4)
            assert np.array_equal(f4[nq - 1], orc.bitmap_top_m(words, n, dim, dim // 4, queries[nq - 1], 400))


@pytest.mark.parametrize("dim,n,nq,m", [(1024, 100_000, 64, 320), (384, 70_001, 300, 700), (192, 40_000, 40, 500)])
def test_sign_tensor_core_top_m_is_exact(orc, monkeypatch, dim, n, nq, m):
    """Sign-bitmap Hamming candidates from the tensor-core overlap scan
    (|q| + |d| - 2 |q AND d|, sampled threshold with the tie bound, and the
    dense key matrix) equal the CUDA-core XOR-popcount scan and the oracle."""
    docs = ob.synth_docs(89, n, dim)
    queries, _ = ob.synth_queries(89, n, nq, dim)
    sb = ob.SignBitmap(dim)
    sb.add(docs)
    f, d, c = _bitmap_modes(monkeypatch, lambda: np.array(sb.top_m_candidates_batched(queries, m)), **_BITMAP_THREE)
    assert np.array_equal(f, d) and np.array_equal(f, c)
    words = orc.sign_encode(docs, dim)
    for qi in (0, nq - 1):
        assert np.array_equal(f[qi], orc.sign_top_m(words, n, dim, queries[qi], m)), qi
    rq = ob.RankQuant(dim, 1)
    rq.add(docs)
    a, b = _bitmap_modes(monkeypatch, lambda: ob.two_stage_search(rq, sb, queries, 0, 10),
                         tc={"OVB_BITMAP_TC": "1"}, cuda_core={"OVB_BITMAP_TC": "0"})
    assert np.array_equal(a.indices, b.indices)
    assert np.array_equal(a.scores.view(np.uint32), b.scores.view(np.uint32))


def test_bitmap_tensor_core_duplicate_rows(orc, monkeypatch):
    """400 distinct rows tiled 100x: every key level holds >= 100 docs, so the
    tie bound alone decides which equal-key docs the filter keeps."""
    dim, n_top, base, reps, nq, m = 256, 64, 400, 100, 48, 1000
    docs = np.tile(ob.synth_docs(47, base, dim), (reps, 1))
    n = len(docs)
    queries, _ = ob.synth_queries(47, base, nq, dim)
    bm = ob.Bitmap(dim, n_top)
    bm.add(docs)
    f, d, c = _bitmap_modes(monkeypatch, lambda: bm.top_m_candidates_batched(queries, m), **_BITMAP_THREE)
    assert np.array_equal(f, d) and np.array_equal(f, c)
    words = orc.bitmap_encode(docs, dim, n_top)
    assert np.array_equal(f[5], orc.bitmap_top_m(words, n, dim, n_top, queries[5], m))


def test_multibucket_identity_weights_tensor_core(orc, monkeypatch):
    """Identity (diagonal) weights take the tensor-core overlap scan: same ids
    as the weighted CUDA-core scan and the oracle; other weights do not change."""
    n, dim, bits, nq, m = 45_000, 768, 2, 64, 600
    docs = ob.synth_docs(53, n, dim)
    queries, _ = ob.synth_queries(53, n, nq, dim)
    mb = ob.MultiBucketBitmap(dim, bits)
    mb.add(docs)
    w = orc.multibucket_weights(bits, "diagonal")
    f, d, c = _bitmap_modes(monkeypatch, lambda: mb.top_m_bilinear_batched(queries, w, m), **_BITMAP_THREE)
    assert np.array_equal(f, d) and np.array_equal(f, c)
    words = orc.multibucket_encode(docs, dim, bits)
    for qi in (0, 33):
        qbm = orc.multibucket_query(queries[qi], dim, bits)
        assert np.array_equal(f[qi], orc.multibucket_top_m(words, n, dim, bits, qbm, w, m)), qi
    wo = orc.multibucket_weights(bits, "outer")
    a, b = _bitmap_modes(monkeypatch, lambda: mb.top_m_bilinear_batched(queries[:40], wo, m),
                         tc={"OVB_BITMAP_TC": "1"}, cuda_core={"OVB_BITMAP_TC": "0"})
    assert np.array_equal(a, b)
    qbm = orc.multibucket_query(queries[1], dim, bits)
    assert np.array_equal(a[1], orc.multibucket_top_m(words, n, dim, bits, qbm, wo, m))


@pytest.mark.parametrize("nq", [1, 3, 16])
def test_wide_select_few_long_rows(orc, monkeypatch, nq):
    """Whole-GPU select for a few rows of >= 2^20 keys (one query per call over
    a large index): heavy key ties, so the id digits decide; equal to the
    cluster / per-row select and to the oracle."""
    n, dim, n_top, m = 1_200_000, 64, 16, 3000
    docs = ob.synth_docs(61, n, dim)
    queries, _ = ob.synth_queries(61, n, nq, dim)
    bm = ob.Bitmap(dim, n_top)
    bm.add(docs)
    wide = np.array(bm.top_m_candidates_batched(queries, m))
    monkeypatch.setenv("OVB_SELECT_WIDE", "0")
    other = np.array(bm.top_m_candidates_batched(queries, m))
    monkeypatch.delenv("OVB_SELECT_WIDE")
    assert np.array_equal(wide, other)
    words = orc.bitmap_encode(docs, dim, n_top)
    for qi in {0, nq - 1}:
        assert np.array_equal(wide[qi], orc.bitmap_top_m(words, n, dim, n_top, queries[qi], m)), qi


def test_wide_select_float_keys(monkeypatch):
    """RankQuant plain search over 1.05M docs (32-bit float keys)."""
    n, dim = 1_050_000, 256
    docs = ob.synth_docs(67, n, dim)
    queries, _ = ob.synth_queries(67, n, 2, dim)
    rq = ob.RankQuant(dim, 2)
    rq.add(docs)
    a = rq.search_asymmetric(queries, 100)
    monkeypatch.setenv("OVB_SELECT_WIDE", "0")
    b = rq.search_asymmetric(queries, 100)
    monkeypatch.delenv("OVB_SELECT_WIDE")
    assert np.array_equal(a.indices, b.indices)
    assert np.array_equal(a.scores.view(np.uint32), b.scores.view(np.uint32))


# ------------------------------------------------------------ multi-bucket
@pytest.mark.parametrize("kind", ["diagonal", "outer", "banded"])
def test_multibucket_top_m_exact(orc, kind):
    n, dim, bits = 2500, 128, 2
    docs = ob.synth_docs(41, n, dim)
    queries, _ = ob.synth_queries(41, n, 4, dim)
    mb = ob.MultiBucketBitmap(dim, bits)
    mb.add(docs)
    words = orc.multibucket_encode(docs, dim, bits)
    w = orc.multibucket_weights(bits, kind, 1)
    got = mb.top_m_bilinear_batched(queries, w, 200)
    for qi in range(4):
        qbm = orc.multibucket_query(queries[qi], dim, bits)
        assert np.array_equal(got[qi], orc.multibucket_top_m(words, n, dim, bits, qbm, w, 200)), qi


# ------------------------------------------------------------- two-stage
def test_two_stage_sign_b1_and_fastscan_b2(orc):
    n, dim, nq, k = 20_000, 1024, 6, 10
    docs = ob.synth_docs(0x0DD5EED1, n, dim)
    queries, _ = ob.synth_queries(0x0DD5EED1, n, nq, dim)
    sb, rq1, fs, rq2 = ob.SignBitmap(dim), ob.RankQuant(dim, 1), ob.RankQuantFastscan(dim), ob.RankQuant(dim, 2)
    for ix in (sb, rq1, fs, rq2):
        ix.add(docs)
    words = orc.sign_encode(docs, dim)
    p1, p2 = orc.rankquant_encode(docs, dim, 1), orc.rankquant_encode(docs, dim, 2)
    blocks = orc.fastscan_pack(docs, dim)
    res = ob.two_stage_search(rq1, sb, queries, 0, k)  # default policy: 320 candidates
    for qi in range(nq):
        cand = orc.sign_top_m(words, n, dim, queries[qi], 320)
        s64 = orc.rq_scores_f64_subset(p1, dim, 1, queries[qi], cand)
        check_float_topk(res.indices_for_query(qi), res.scores_for_query(qi), cand, s64, k)
        s, i = rq1.try_search_with_sign_probe(sb, queries[qi], k)
        check_float_topk(i, s, cand, s64, k)
    res = ob.two_stage_search(rq2, fs, queries, 1000, k)
    _, cands = orc.fastscan_search(blocks, n, dim, queries, 1000)
    for qi in range(nq):
        s64 = orc.rq_scores_f64_subset(p2, dim, 2, queries[qi], cands[qi].astype(np.uint32))
        check_float_topk(res.indices_for_query(qi), res.scores_for_query(qi), cands[qi], s64, k)


def test_sign_b1_two_stage_full_size(orc):
    """The sign-bitmap -> b=1 rerank configuration at full size (N=100,000, dim 1024,
    k=10, default 320 candidates): one query per call equals the batched call, and
    both match the oracle (candidates bit-exact, rerank within the FP64 bar)."""
    n, dim, nq, k = 100_000, 1024, 64, 10
    docs = ob.synth_docs(0x0DD5EED1, n, dim)
    queries, _ = ob.synth_queries(0x0DD5EED1, n, nq, dim)
    sb, rq1 = ob.SignBitmap(dim), ob.RankQuant(dim, 1)
    sb.add(docs)
    rq1.add(docs)
    batched = ob.two_stage_search(rq1, sb, queries, 0, k)
    words = orc.sign_encode(docs, dim)
    p1 = orc.rankquant_encode(docs, dim, 1)
    for qi in range(nq):
        s, i = rq1.try_search_with_sign_probe(sb, queries[qi], k)
        assert np.array_equal(i, batched.indices_for_query(qi))
        assert np.array_equal(s.view(np.uint32), batched.scores_for_query(qi).view(np.uint32))
    for qi in (0, 17, 63):
        cand = orc.sign_top_m(words, n, dim, queries[qi], 320)
        assert np.array_equal(sb.top_m_candidates(queries[qi], 320), cand)
        s64 = orc.rq_scores_f64_subset(p1, dim, 1, queries[qi], cand)
        check_float_topk(batched.indices_for_query(qi), batched.scores_for_query(qi), cand, s64, k)


def test_two_stage_bitmap_and_multibucket(orc):
    n, dim, nq, k, m = 8000, 768, 4, 20, 500
    docs = ob.synth_docs(0x0DD5EED4, n, dim)
    queries, _ = ob.synth_queries(0x0DD5EED4, n, nq, dim)
    rq, bm, mb = ob.RankQuant(dim, 2), ob.Bitmap(dim, 192), ob.MultiBucketBitmap(dim, 2)
    for ix in (rq, bm, mb):
        ix.add(docs)
    p2 = orc.rankquant_encode(docs, dim, 2)
    words = orc.bitmap_encode(docs, dim, 192)
    mwords = orc.multibucket_encode(docs, dim, 2)
    w = orc.multibucket_weights(2, "diagonal")
    r_bm = ob.two_stage_search(rq, bm, queries, m, k)
    r_mb = ob.two_stage_search(rq, mb, queries, m, k)
    for qi in range(nq):
        cand = orc.bitmap_top_m(words, n, dim, 192, queries[qi], m)
        s64 = orc.rq_scores_f64_subset(p2, dim, 2, queries[qi], cand)
        check_float_topk(r_bm.indices_for_query(qi), r_bm.scores_for_query(qi), cand, s64, k)
        cand = orc.multibucket_top_m(mwords, n, dim, 2, orc.multibucket_query(queries[qi], dim, 2), w, m)
        s64 = orc.rq_scores_f64_subset(p2, dim, 2, queries[qi], cand)
        check_float_topk(r_mb.indices_for_query(qi), r_mb.scores_for_query(qi), cand, s64, k)


# ------------------------------------------------------------ persistence
def test_persistence_roundtrip_all_formats(tmp_path, corpus):
    docs, queries = corpus
    docs = docs[:777]
    for make, ext in ((lambda: ob.RankQuant(1024, 4), "ovrq"), (lambda: ob.Bitmap(1024, 256), "ovbm"),
                      (lambda: ob.SignBitmap(1024), "ovsb"), (lambda: ob.RankQuantFastscan(1024), "ovfs")):
        ix = make()
        ix.add(docs)
        p = str(tmp_path / f"x.{ext}")
        ix.write(p)
        back = ob.load(p)
        assert type(back) is type(ix)
        assert np.array_equal(back.payload(), ix.payload()), ext
    fs = ob.load(str(tmp_path / "x.ovfs"))
    a = fs.search(queries, 20)
    b = ob.load(str(tmp_path / "x.ovfs")).search(queries, 20)
    assert np.array_equal(a.indices, b.indices)


@pytest.mark.parametrize("nq", [1, 3, 20])
def test_cluster_select_ties_by_position(orc, monkeypatch, nq):
    """Long rows (>= 32,768 keys) of a few queries go through the 8-CTA cluster
    select; with ids = positions its ties are taken lowest position first.
    Bitmap overlaps tie massively (a few dozen distinct values over 100k docs),
    and duplicate rows add exact ties across the CTAs' slices."""
    monkeypatch.setenv("OVB_BITMAP_TC", "0")  # CUDA-core scan: the key matrix and the select
    monkeypatch.setenv("OVB_SELECT_WIDE", "0")
    dim, n_top, n = 256, 64, 100_003
    rng = np.random.default_rng(77)
    docs = rng.standard_normal((n, dim)).astype(np.float32)
    docs[50_000:50_300] = docs[3]  # duplicates spread over two CTA slices
    qs = rng.standard_normal((nq, dim)).astype(np.float32)
    qs[0] = docs[3]
    bm = ob.Bitmap(dim, n_top)
    bm.add(docs)
    words = orc.bitmap_encode(docs, dim, n_top)
    for m in (1, 257, 1000, 2048):
        got = bm.top_m_candidates_batched(qs, m)
        for qi in range(nq):
            want = orc.bitmap_top_m(words, n, dim, n_top, qs[qi], m)
            assert np.array_equal(np.asarray(got[qi]), want), (m, qi)
