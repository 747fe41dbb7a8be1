"""The allocation-free RankQuant search entry point, called through the C ABI.

ovb_rankquant_search_noalloc exists for callers that must not let a library
allocate device memory -- a serving thread that cannot afford the device-wide
synchronisation cudaMalloc/cudaFree may cause, or a process whose GPU memory is
owned by one budgeted allocator.  Its intermediates live in a fixed 32 MiB
device array inside the library.  This file is named so pytest collects it
last; it must pass alone in a fresh process and after the rest of the suite.
"""
import ctypes as C

import numpy as np
import pytest

import ordvec_b200 as ob
from ordvec_b200._lib import OrdvecError, check, lib

pytestmark = pytest.mark.gpu


def _noalloc(rq, d_q, nq, k, d_s, d_i, stream):
    return lib().ovb_rankquant_search_noalloc(rq.handle, C.c_void_p(d_q), nq, k, C.c_void_p(d_s),
                                              C.c_void_p(d_i), C.c_void_p(stream))


def test_noalloc_search_matches_allocating_entry_point_on_two_calls(orc):
    import torch

    dim, bits, n, nq, k = 768, 2, 6000, 4, 50
    docs = ob.synth_docs(0x5EED, n, dim)
    rq = ob.RankQuant(dim, bits)
    rq.add(docs)
    packed = orc.rankquant_encode(docs, dim, bits)
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev)
    for call in range(2):  # the second call reuses the shared array's stale contents
        queries, _ = ob.synth_queries(0x5EED + call, n, nq, dim)
        d_q = torch.from_numpy(queries).to(dev)
        d_s = torch.full((nq * k,), float("nan"), dtype=torch.float32, device=dev)
        d_i = torch.full((nq * k,), -7, dtype=torch.int64, device=dev)
        check(_noalloc(rq, d_q.data_ptr(), nq, k, d_s.data_ptr(), d_i.data_ptr(), stream.cuda_stream))
        torch.cuda.synchronize(dev)
        got_s, got_i = d_s.cpu().numpy(), d_i.cpu().numpy()
        ref = rq.search_asymmetric(queries, k)
        assert np.array_equal(got_i, ref.indices), call
        np.testing.assert_allclose(got_s, ref.scores, rtol=1e-5, atol=1e-8)
        # and against the oracle's FP64 scores: within 1e-5 relative, ids in
        # (score desc, id asc) order except between scores closer than that
        for qi in range(nq):
            s64 = orc.rq_scores_f64(packed, n, dim, bits, queries[qi])
            want = np.lexsort((np.arange(n), -s64))[:k]
            ids = got_i[qi * k:(qi + 1) * k]
            tol = 1e-5 * np.maximum(np.abs(s64[want]), 1e-3)
            assert np.all(np.abs(s64[ids] - s64[want]) <= tol), (call, qi)
            assert np.all(np.abs(got_s[qi * k:(qi + 1) * k] - s64[ids]) <= tol), (call, qi)


def test_noalloc_search_allocates_no_device_memory():
    import torch

    dim, n, nq, k = 256, 20_000, 8, 20
    rq = ob.RankQuant(dim, 2)
    rq.add(ob.synth_docs(21, n, dim))
    dev = torch.device("cuda", 0)
    queries, _ = ob.synth_queries(21, n, nq, dim)
    d_q = torch.from_numpy(queries).to(dev)
    d_s = torch.empty(nq * k, dtype=torch.float32, device=dev)
    d_i = torch.empty(nq * k, dtype=torch.int64, device=dev)
    sp = torch.cuda.current_stream(dev).cuda_stream
    check(_noalloc(rq, d_q.data_ptr(), nq, k, d_s.data_ptr(), d_i.data_ptr(), sp))  # loads the kernels
    torch.cuda.synchronize(dev)
    free0, _ = torch.cuda.mem_get_info(dev)
    for _ in range(3):
        check(_noalloc(rq, d_q.data_ptr(), nq, k, d_s.data_ptr(), d_i.data_ptr(), sp))
    torch.cuda.synchronize(dev)
    free1, _ = torch.cuda.mem_get_info(dev)
    assert free1 == free0


def test_noalloc_search_rejects_requests_beyond_its_scratch():
    import torch

    dim, n = 64, 70_000  # 70,000 docs x 200 queries x 4 B of keys > 32 MiB
    rq = ob.RankQuant(dim, 2)
    rq.add(ob.synth_docs(3, n, dim))
    nq, k = 200, 10
    d_q = torch.zeros((nq, dim), dtype=torch.float32, device="cuda")
    d_s = torch.empty(nq * k, dtype=torch.float32, device="cuda")
    d_i = torch.empty(nq * k, dtype=torch.int64, device="cuda")
    with pytest.raises(OrdvecError) as e:
        check(_noalloc(rq, d_q.data_ptr(), nq, k, d_s.data_ptr(), d_i.data_ptr(), 0))
    assert e.value.status == 2 and "32 MiB" in e.value.message
    # query counts whose byte sizes overflow 64 bits are rejected, not wrapped
    # (the check runs before any pointer is read or kernel launched)
    for huge in (2 ** 62, 2 ** 64 - 1, (2 ** 64) // (4 * n) + 1):
        with pytest.raises(OrdvecError) as e:
            check(_noalloc(rq, d_q.data_ptr(), huge, k, d_s.data_ptr(), d_i.data_ptr(), 0))
        assert e.value.status == 2, huge
