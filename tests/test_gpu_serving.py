"""Serving loop (ovb_server_*): continuous batching over several device-resident
indices with HBM-budget admission.  Each request's answer must equal the one it
gets alone (bit for bit: every kernel scores a query independently of its batch
mates), whatever it was batched with."""
import threading
import time

import numpy as np
import pytest

import ordvec_b200 as ob

pytestmark = pytest.mark.gpu


def _routes():
    """Scaled-down shapes of the serving configuration: three indices of
    different dim / bits, two-stage and full-search routes."""
    out = []
    d1 = ob.synth_docs(0x0DD5EED5, 12_000, 384)
    sb, r1 = ob.SignBitmap(384), ob.RankQuant(384, 1)
    sb.add(d1)
    r1.add(d1)
    out.append((r1, sb))
    d2 = ob.synth_docs(0x0DD5EED5 + 1, 9_000, 768)
    bm, r2 = ob.Bitmap(768, 192), ob.RankQuant(768, 2)
    bm.add(d2)
    r2.add(d2)
    out.append((r2, bm))
    d3 = ob.synth_docs(0x0DD5EED5 + 2, 6_000, 1024)
    fs, r3 = ob.RankQuantFastscan(1024), ob.RankQuant(1024, 4)
    fs.add(d3)
    r3.add(d3)
    out.append((r3, fs))
    out.append((r3, None))  # full asymmetric search of the b=4 index
    return out


def _requests(routes, n_req, seed):
    rng = np.random.default_rng(seed)
    reqs = []
    for j in range(n_req):
        route = int(rng.integers(len(routes)))
        rq = routes[route][0]
        nq = int(rng.choice([1, 1, 2, 5, 17, 40, 64]))
        k = int(rng.choice([10, 50, 100]))
        q, _ = ob.synth_queries(1000 + j, len(rq), nq, rq.dim)
        reqs.append((route, q, k))
    return reqs


def _alone(routes, route, q, k):
    rq, s1 = routes[route]
    if s1 is None:
        return rq.search_asymmetric(q, k)
    return ob.two_stage_search(rq, s1, q, 0, k)


def test_server_answers_equal_alone_answers():
    routes = _routes()
    reqs = _requests(routes, 120, 7)
    alone = [_alone(routes, r, q, k) for r, q, k in reqs]
    srv = ob.Server(workers=3, max_batch=256)
    ids = [srv.add_route(rq, s1) for rq, s1 in routes]
    assert ids == list(range(len(routes)))
    srv.wait_ready()
    assert srv.stats()["warm_workers"] == 3
    rng = np.random.default_rng(11)
    tickets = [None] * len(reqs)

    def producer():  # Poisson arrivals at ~4k requests/s
        for j, (r, q, k) in enumerate(reqs):
            tickets[j] = srv.submit(r, q, k)
            time.sleep(float(rng.exponential(1 / 4000)))

    th = threading.Thread(target=producer)
    th.start()
    th.join()
    for j, t in enumerate(tickets):
        got, lat = t.wait()
        want = alone[j]
        assert got.k == want.k and got.nq == want.nq
        assert np.array_equal(got.indices, want.indices), j
        assert np.array_equal(got.scores.view(np.uint32), want.scores.view(np.uint32)), j
        assert lat > 0.0
    st = srv.stats()
    assert st["requests"] == len(reqs)
    assert st["queries"] == sum(len(q) for _, q, _ in reqs)
    assert st["batches"] <= st["requests"]
    assert st["p99_ms"] >= st["p50_ms"] > 0.0
    srv.close()


def test_server_batches_pending_requests_of_one_route():
    routes = _routes()[:1]
    rq, sb = routes[0]
    srv = ob.Server(workers=1, max_batch=1024)
    r = srv.add_route(rq, sb)
    qs = [ob.synth_queries(50 + j, len(rq), 3, rq.dim)[0] for j in range(200)]
    tickets = [srv.submit(r, q, 10) for q in qs]  # all arrive at once
    res = [t.wait()[0] for t in tickets]
    st = srv.stats()
    assert st["requests"] == 200 and st["batches"] < 200  # later arrivals were batched
    for q, got in zip(qs, res):
        want = ob.two_stage_search(rq, sb, q, 0, 10)
        assert np.array_equal(got.indices, want.indices)
    srv.close()


def test_server_hbm_budget_admits_one_batch_at_a_time():
    routes = _routes()[2:3]
    rq, fs = routes[0]
    srv = ob.Server(workers=4, max_batch=8, hbm_budget_bytes=1)  # every batch exceeds it
    r = srv.add_route(rq, fs)
    qs = [ob.synth_queries(900 + j, len(rq), 8, rq.dim)[0] for j in range(24)]
    got = [t.wait()[0] for t in [srv.submit(r, q, 20) for q in qs]]
    st = srv.stats()
    assert st["max_concurrent_batches"] == 1  # admitted only when nothing else was in flight
    for q, g in zip(qs, got):
        want = ob.two_stage_search(rq, fs, q, 0, 20)
        assert np.array_equal(g.indices, want.indices)
    srv.close()


def test_server_errors():
    routes = _routes()[3:]
    rq, _ = routes[0]
    srv = ob.Server(workers=1)
    r = srv.add_route(rq)
    bad = np.ones((2, rq.dim), np.float32)
    bad[1, 3] = np.nan
    with pytest.raises(ob.OrdvecError) as e:
        srv.submit(r, bad, 5)
    assert e.value.status == 8
    with pytest.raises(ob.OrdvecError) as e:
        srv.submit(7, bad[:1], 5)
    assert e.value.status == 2
    t = srv.submit(r, np.ones(rq.dim, np.float32), 0)  # k = 0: empty answer
    res, _ = t.wait()
    assert res.k == 0 and res.indices.size == 0
    t = srv.submit(r, np.ones(rq.dim, np.float32), 3)
    t.wait()
    with pytest.raises(ob.OrdvecError) as e:
        t.wait()  # a ticket is collected once
    assert e.value.status == 2
    srv.close()


def test_server_batches_mixed_k_and_m_of_one_route():
    """Requests of one route with different k and candidate counts (explicit m,
    or the default policy's count for their k) share batches; each request's
    rows are a prefix of the batch's rows and equal its answer alone."""
    for rq, s1 in _routes()[1:]:
        srv = ob.Server(workers=1, max_batch=1024)
        r = srv.add_route(rq, s1)
        srv.wait_ready()
        rng = np.random.default_rng(5)
        reqs = []
        for j in range(60):
            q = ob.synth_queries(300 + j, len(rq), int(rng.choice([1, 3, 8])), rq.dim)[0]
            k = int(rng.choice([10, 50, 100]))
            m = 0 if s1 is None else int(rng.choice([0, 0, 400, 1500]))
            reqs.append((q, k, m))
        # four full-size requests occupy the worker (one batch each) while the
        # mixed requests queue up behind them
        big = ob.synth_queries(299, len(rq), 1024, rq.dim)[0]
        blockers = [srv.submit(r, big, 10, 0) for _ in range(4)]
        tickets = [srv.submit(r, q, k, m) for q, k, m in reqs]
        got = [t.wait()[0] for t in tickets]
        for t in blockers:
            t.wait()
        st = srv.stats()
        assert st["requests"] == len(reqs) + 4 and st["batches"] - 4 < len(reqs) // 4
        for (q, k, m), g in zip(reqs, got):
            want = rq.search_asymmetric(q, k) if s1 is None else ob.two_stage_search(rq, s1, q, m, k)
            assert g.k == want.k
            assert np.array_equal(g.indices, want.indices)
            assert np.array_equal(g.scores.view(np.uint32), want.scores.view(np.uint32))
        srv.close()
