"""The FastScan two-stage configuration's whole batch at full size: N=171,332
docs, dim 1024, 1,000 queries, RankQuantFastscan top-1,000 -> RankQuant b=2
rerank top-10 (the call the benchmark's fastscan_two_stage section times).

The oracle packs and encodes the corpus itself (not the device payloads); its
AVX-512 FastScan restatement (bit-identical integer accumulators and the same
three rounded f32 operations as the scalar reference tier) gives every
query's candidate row.  Every row of the device's stage-1 candidates must equal
it in tie order, and every row's reranked top-10 must match the FP64 ordering
of those candidates within the float contract."""
import numpy as np
import pytest

import ordvec_b200 as ob
from test_gpu_parity import check_float_topk

pytestmark = pytest.mark.gpu

N, DIM, NQ, M, K, SEED = 171_332, 1024, 1000, 1000, 10, 0x0DD5EED2


def test_fastscan_two_stage_batch_every_row(orc):
    docs = ob.synth_docs(SEED, N, DIM)
    queries, _ = ob.synth_queries(SEED, N, NQ, DIM)
    rq, fs = ob.RankQuant(DIM, 2), ob.RankQuantFastscan(DIM)
    rq.add(docs)
    fs.add(docs)
    blocks = orc.fastscan_pack(docs, DIM)
    packed = orc.rankquant_encode(docs, DIM, 2)
    assert np.array_equal(fs.payload(), blocks) and np.array_equal(rq.payload(), packed)
    _, _, cands = orc.cpu_fastscan_two_stage(blocks, packed, N, DIM, queries, M, K, orc.max_threads(),
                                             want_candidates=True)
    # the scalar tier on a few rows pins the AVX-512 restatement's candidates
    for qi in (0, 499, NQ - 1):
        _, want = orc.fastscan_search(blocks, N, DIM, queries[qi], M)
        assert np.array_equal(cands[qi], want[0].astype(np.uint32)), qi
    got = fs.search(queries, M)
    assert np.array_equal(got.indices.reshape(NQ, M), cands.astype(np.int64))
    res = ob.two_stage_search(rq, fs, queries, M, K)
    for qi in range(NQ):
        s64 = orc.rq_scores_f64_subset(packed, DIM, 2, queries[qi], cands[qi])
        check_float_topk(res.indices_for_query(qi), res.scores_for_query(qi), cands[qi], s64, K)
