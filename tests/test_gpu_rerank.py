"""Split-BF16 tensor-core rerank (rerank_tc_kernel) of two-stage candidate rows.

The reference reranks candidates with its asymmetric subset scorer
(src/quant.rs:1126-1281).  The device's default for eligible shapes scores the
candidates with the split-BF16 contraction on tcgen05 and rescores the top
2k + 32 in FP64 after a margin test, so its results must equal the FP64
rerank's bit for bit; the raw split scores must lie within the stated error
bound of the oracle's FP64 scores."""
import numpy as np
import pytest
import torch

import ordvec_b200 as ob
from test_gpu_parity import check_float_topk

pytestmark = pytest.mark.gpu


def _run(rq, s1, queries, m, k, rerank):
    dev = torch.device("cuda", 0)
    nq = queries.shape[0]
    d_q = torch.from_numpy(queries).to(dev)
    d_s = torch.full((nq * k,), float("nan"), dtype=torch.float32, device=dev)
    d_i = torch.full((nq * k,), -7, dtype=torch.int64, device=dev)
    sp = torch.cuda.current_stream(dev).cuda_stream
    ob.two_stage_search_device(rq, s1, d_q.data_ptr(), nq, m, k, d_s.data_ptr(), d_i.data_ptr(), sp, rerank=rerank)
    torch.cuda.synchronize(dev)
    return d_s.view(nq, k).cpu().numpy(), d_i.view(nq, k).cpu().numpy()


@pytest.mark.parametrize("dim,bits,m,k", [(768, 2, 2000, 100), (1024, 2, 1000, 10), (512, 4, 700, 50),
                                          (1024, 1, 500, 10), (128, 2, 300, 10), (256, 4, 333, 20)])
def test_split_rerank_equals_fp64_and_raw_within_bound(orc, dim, bits, m, k):
    n, nq, n_top = 40_000, 80, dim // 4
    docs = ob.synth_docs(0xBEEF + dim + bits, n, dim)
    queries, _ = ob.synth_queries(0xBEEF + dim + bits, n, nq, dim)
    rq, bm = ob.RankQuant(dim, bits), ob.Bitmap(dim, n_top)
    rq.add(docs)
    bm.add(docs)
    s_f, i_f = _run(rq, bm, queries, m, k, "fp64")
    s_x, i_x = _run(rq, bm, queries, m, k, "split")
    s_a, i_a = _run(rq, bm, queries, m, k, "auto")
    assert np.array_equal(i_x, i_f) and np.array_equal(s_x.view(np.uint32), s_f.view(np.uint32))
    assert np.array_equal(i_a, i_f) and np.array_equal(s_a.view(np.uint32), s_f.view(np.uint32))
    s_r, i_r = _run(rq, bm, queries, m, k, "split_raw")
    packed = orc.rankquant_encode(docs, dim, bits)
    words = orc.bitmap_encode(docs, dim, n_top)
    inv_norm = 1.0 / orc.rankquant_norm(dim, bits)
    cmax = ((1 << bits) - 1) / 2
    for qi in range(0, nq, 7):
        cand = orc.bitmap_top_m(words, n, dim, n_top, queries[qi], m)
        s64 = orc.rq_scores_f64_subset(packed, dim, bits, queries[qi], cand)
        check_float_topk(i_f[qi], s_f[qi], cand, s64, k)
        # raw split scores: within the stated bound of FP64, and their ids the
        # FP64 order except between scores closer than twice that bound
        qu = orc.l2_normalise(queries[qi])
        eps = inv_norm * cmax * np.abs(qu).sum() * 1.0001 * (2 * dim * 2.0 ** -24 + 2.0 ** -16) * 1.05
        got64 = orc.rq_scores_f64_subset(packed, dim, bits, queries[qi], i_r[qi].astype(np.uint32))
        assert np.all(np.abs(s_r[qi].astype(np.float64) - got64) <= eps + 4 * np.abs(got64) * 2.0 ** -24), qi
        want = np.sort(s64)[::-1][:k]
        assert np.all(np.abs(np.sort(got64)[::-1] - want) <= 2 * eps), qi


def test_split_rerank_margin_failure_falls_back_to_fp64():
    """A corpus of 40 copies of 500 docs: every candidate score appears 40
    times, so the 2k+32-th split score ties the k-th, the margin test fails
    and the batch is reranked in FP64 -- the same answer as the FP64 mode."""
    dim, bits, base, reps, nq, m, k = 768, 2, 500, 40, 32, 1200, 10
    distinct = ob.synth_docs(77, base, dim)
    docs = np.tile(distinct, (reps, 1))
    queries, _ = ob.synth_queries(77, base, nq, dim)
    rq, bm = ob.RankQuant(dim, bits), ob.Bitmap(dim, 192)
    rq.add(docs)
    bm.add(docs)
    s_f, i_f = _run(rq, bm, queries, m, k, "fp64")
    s_x, i_x = _run(rq, bm, queries, m, k, "split")
    assert np.array_equal(i_x, i_f) and np.array_equal(s_x.view(np.uint32), s_f.view(np.uint32))


def test_split_rerank_on_fastscan_and_sign_stage1(orc):
    """The rerank is shared by every stage-1 kind: FastScan and SignBitmap rows too."""
    dim, n, nq = 1024, 30_000, 48
    docs = ob.synth_docs(909, n, dim)
    queries, _ = ob.synth_queries(909, n, nq, dim)
    rq2, fs = ob.RankQuant(dim, 2), ob.RankQuantFastscan(dim)
    rq1, sb = ob.RankQuant(dim, 1), ob.SignBitmap(dim)
    for ix in (rq2, fs, rq1, sb):
        ix.add(docs)
    for rq, s1, m, k in ((rq2, fs, 1000, 10), (rq1, sb, 640, 20)):
        s_f, i_f = _run(rq, s1, queries, m, k, "fp64")
        s_a, i_a = _run(rq, s1, queries, m, k, "auto")
        assert np.array_equal(i_a, i_f) and np.array_equal(s_a.view(np.uint32), s_f.view(np.uint32))
