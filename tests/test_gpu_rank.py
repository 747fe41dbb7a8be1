"""GPU parity for the Rank index (src/rank.rs:283-482) and RankQuant's
symmetric search (src/quant.rs:629-695) against the CPU oracle.

Both are bit-exact: Rank::search sums integers, RankQuant::search sums
multiples of 1/4 that f32 holds exactly, and Rank::search_asymmetric follows
the reference's sequential f32 chain per document.
"""
import numpy as np
import pytest

import ordvec_b200 as ob
from ordvec_b200 import abi
from ordvec_b200._lib import OrdvecError

pytestmark = pytest.mark.gpu


def _docs(dim, n, seed):
    rng = np.random.default_rng(seed)
    d = rng.standard_normal((n, dim)).astype(np.float32)
    d[::9, : dim // 3] = 0.25  # tied coordinates
    d[::13] = 0.0
    if n > 4:
        d[4, ::2] = -0.0
    return d


@pytest.mark.parametrize("dim", [64, 100, 768])
def test_rank_encoder_matches_oracle(orc, dim):
    docs = _docs(dim, 500, dim)
    rk = ob.Rank(dim)
    rk.add(docs[:123])
    rk.add(docs[123:])  # incremental add
    assert len(rk) == 500
    assert np.array_equal(rk.payload().view(np.uint16), orc.rank_encode(docs, dim))


@pytest.mark.parametrize("dim,n,nq", [(64, 3000, 1), (100, 2500, 7), (200, 3000, 9), (768, 6000, 70),
                                      (1024, 20000, 3), (2560, 2000, 5)])
def test_rank_search_is_bit_exact(orc, dim, n, nq):
    docs = _docs(dim, n, 11 + dim)
    qs = _docs(dim, nq, 17 + dim)
    qs[0] = docs[5] + 0.0  # an exact match: score 1.0 at row 5
    rk = ob.Rank(dim)
    rk.add(docs)
    ranks = orc.rank_encode(docs, dim)
    for k in (1, 10, 300):
        for asym in (False, True):
            got = (rk.search_asymmetric if asym else rk.search)(qs, k)
            ws, wi = orc.rank_search(ranks, n, dim, qs, k, asymmetric=asym)
            assert got.k == min(k, n)
            assert np.array_equal(got.indices.reshape(nq, -1), wi), (k, asym)
            assert np.array_equal(got.scores.reshape(nq, -1).view(np.uint32), ws.view(np.uint32)), (k, asym)
    top = rk.search(qs[:1], 1)
    assert top.indices[0] == 5 and abs(float(top.scores[0]) - 1.0) < 1e-5


@pytest.mark.parametrize("bits", [1, 2, 4])
@pytest.mark.parametrize("dim,n,nq", [(64, 4000, 1), (768, 30000, 9), (1024, 6000, 70)])
def test_rankquant_symmetric_is_bit_exact(orc, bits, dim, n, nq):
    docs = _docs(dim, n, 31 + dim + bits)
    qs = _docs(dim, nq, 37 + dim)
    rq = ob.RankQuant(dim, bits)
    rq.add(docs)
    packed = orc.rankquant_encode(docs, dim, bits)
    for k in (1, 10, 257):
        got = rq.search(qs, k)
        ws, wi = orc.rq_search_sym(packed, n, dim, bits, qs, k)
        assert np.array_equal(got.indices.reshape(nq, -1), wi), (k,)
        assert np.array_equal(got.scores.reshape(nq, -1).view(np.uint32), ws.view(np.uint32)), (k,)


def test_rank_determinism_literals():
    """tests/determinism_contract.rs:15-38 and 150-160."""
    dim = 64
    docs = np.ones((8, dim), np.float32)
    rk = ob.Rank(dim)
    rk.add(docs)
    assert rk.search(np.ones(dim, np.float32), 4).indices.tolist() == [0, 1, 2, 3]
    r = rk.search_asymmetric(np.zeros(dim, np.float32), 4)
    assert r.indices.tolist() == [0, 1, 2, 3] and (r.scores == 0.0).all()
    rq = ob.RankQuant(dim, 2)
    rq.add(docs)
    assert rq.search(np.ones(dim, np.float32), 4).indices.tolist() == [0, 1, 2, 3]
    empty = ob.Rank(dim).search(np.ones(dim, np.float32), 10)
    assert empty.k == 0 and empty.scores.size == 0 and empty.indices.size == 0
    big = rk.search(np.ones(dim, np.float32), 2**40)  # k clamps to n
    assert big.k == 8


def test_rank_rejects_bad_input():
    with pytest.raises(OrdvecError) as e:
        ob.Rank(1)
    assert e.value.status == 2
    with pytest.raises(OrdvecError):
        ob.Rank(65536)
    rk = ob.Rank(64)
    rk.add(np.ones((3, 64), np.float32))
    q = np.ones(64, np.float32)
    q[3] = np.nan
    for fn in (rk.search, rk.search_asymmetric):
        with pytest.raises(OrdvecError) as e:
            fn(q, 2)
        assert e.value.status == 8
    wide = ob.Rank(20000)  # constructible; the device rank transform stops at 16384
    with pytest.raises(OrdvecError) as e:
        wide.add(np.ones((1, 20000), np.float32))
    assert e.value.status == 11
    sb = ob.SignBitmap(64)
    with pytest.raises(OrdvecError) as e:
        ob._lib.check(ob._lib.lib().ovb_rank_search(sb.handle, None, 0, 1, None, None))
    assert e.value.status == 11


def test_rank_ovr_fixture_bytes_and_roundtrip(tmp_path):
    """tests/persistence_compat.rs:101-125: Rank::new(4) of [0, 1, 2, 3]
    writes OVR1 | 1 | dim 4 | n 1 | ranks 0 1 2 3; trailing bytes and a
    non-permutation row are CORRUPT_INDEX; ABI v1's loader refuses the format."""
    expected = bytes([ord("O"), ord("V"), ord("R"), ord("1"), 1, 4, 0, 0, 0, 1, 0, 0, 0, 0, 0, 1, 0, 2, 0, 3, 0])
    rk = ob.Rank(4)
    rk.add(np.arange(4, dtype=np.float32))
    p = str(tmp_path / "r.ovr")
    rk.write(p)
    assert open(p, "rb").read() == expected
    back = ob.Rank.load(p)
    assert type(back) is ob.Rank and back.dim == 4 and len(back) == 1
    with pytest.raises(OrdvecError) as e:
        abi.index_load(p)
    assert e.value.status == 4
    for bad in (expected + b"\0", expected[:-2] + bytes([2, 0]), expected[:-2] + bytes([4, 0])):
        q = str(tmp_path / "bad.ovr")
        open(q, "wb").write(bad)
        with pytest.raises(OrdvecError) as e:
            ob.load(q)
        assert e.value.status == 5, bad

    docs = _docs(256, 3000, 5)
    rk = ob.Rank(256)
    rk.add(docs)
    p = str(tmp_path / "big.ovr")
    rk.write(p)
    back = ob.load(p)
    assert np.array_equal(back.payload(), rk.payload())
    qs = _docs(256, 4, 6)
    a, b = rk.search(qs, 25), back.search(qs, 25)
    assert np.array_equal(a.indices, b.indices) and np.array_equal(a.scores, b.scores)


@pytest.mark.parametrize("bits", [1, 2, 4])
def test_rankquant_symmetric_tensor_core_batches(orc, monkeypatch, bits):
    """Batches of >= 64 queries take the split-BF16 scan (through the sampled
    threshold filter at this size) with exact rescoring: the same bits as the
    CUDA-core scan and the oracle, heavy score ties included."""
    dim, n, nq = 768, 40000, 64
    docs = _docs(dim, n, 41 + bits)
    docs[100:400] = docs[7]  # 300 duplicate rows: ties across the k-th score
    qs = _docs(dim, nq, 43)
    qs[1] = docs[7]
    rq = ob.RankQuant(dim, bits)
    rq.add(docs)
    packed = orc.rankquant_encode(docs, dim, bits)
    for k in (10, 257):
        monkeypatch.setenv("OVB_RANK_TC", "1")
        tc = rq.search(qs, k)
        monkeypatch.setenv("OVB_RANK_TC", "0")
        plain = rq.search(qs, k)
        assert np.array_equal(tc.indices, plain.indices), k
        assert np.array_equal(tc.scores.view(np.uint32), plain.scores.view(np.uint32)), k
        ws, wi = orc.rq_search_sym(packed, n, dim, bits, qs[:4], k)
        assert np.array_equal(tc.indices.reshape(nq, -1)[:4], wi), k
        assert np.array_equal(tc.scores.reshape(nq, -1)[:4].view(np.uint32), ws.view(np.uint32)), k


def test_search_device_matches_host_entry_points():
    """ovb_index_search_device gives the host entry points' results for every
    kind with a full search, on the caller's stream."""
    import torch

    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev)
    dim, n, nq, k = 256, 5000, 6, 17
    docs = _docs(dim, n, 51)
    qs = _docs(dim, nq, 52)
    rq, rk, bm, fs = ob.RankQuant(dim, 2), ob.Rank(dim), ob.Bitmap(dim, 64), ob.RankQuantFastscan(dim)
    for ix in (rq, rk, bm, fs):
        ix.add(docs)
    d_q = torch.from_numpy(qs).to(dev)
    cases = [(rq, False, rq.search), (rq, True, rq.search_asymmetric), (rk, False, rk.search),
             (rk, True, rk.search_asymmetric), (bm, False, bm.search), (fs, False, fs.search)]
    for ix, asym, host in cases:
        d_s = torch.empty(nq * k, dtype=torch.float32, device=dev)
        d_i = torch.empty(nq * k, dtype=torch.int64, device=dev)
        ob.search_device(ix, d_q.data_ptr(), nq, k, d_s.data_ptr(), d_i.data_ptr(), stream.cuda_stream,
                         asymmetric=asym)
        torch.cuda.synchronize(dev)
        want = host(qs, k)
        name = type(ix).__name__
        assert np.array_equal(d_i.cpu().numpy(), want.indices), (name, asym)
        assert np.array_equal(d_s.cpu().numpy().view(np.uint32), want.scores.view(np.uint32)), (name, asym)
    with pytest.raises(OrdvecError) as e:
        ob.search_device(bm, d_q.data_ptr(), nq, k, 0, 0, stream.cuda_stream, asymmetric=True)
    assert e.value.status == 11
