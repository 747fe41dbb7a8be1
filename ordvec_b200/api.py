"""Python mirror of ordvec's scan-path API, backed by the B200 kernels.

Class and method names, argument meaning, clamping and result shapes follow
the reference crate (ordvec 0.6.0): ``RankQuant`` (src/quant.rs),
``SignBitmap`` (src/sign_bitmap.rs), ``Bitmap`` (src/bitmap.rs),
``RankQuantFastscan`` (src/fastscan.rs), ``MultiBucketBitmap``
(src/multi_bucket.rs), ``TwoStageCandidatePolicy`` and ``SearchResults``
(src/lib.rs:313-415).  Inputs and outputs are numpy arrays in host memory;
codes live in HBM for the lifetime of the object.  Where the reference
panics on a contract violation this raises ``OrdvecError`` (a ValueError).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np

from . import _lib as _lib_mod
from ._lib import (KIND_BITMAP, KIND_FASTSCAN, KIND_MULTIBUCKET, KIND_RANK, KIND_RANK_QUANT, KIND_SIGN_BITMAP,
                   IndexInfo, OrdvecError, check, lib)


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def _rows(x, dim: int) -> np.ndarray:
    a = np.ascontiguousarray(x, dtype=np.float32).reshape(-1)
    if a.size % dim:
        raise OrdvecError(2, f"queries length {a.size} must be a multiple of dim {dim}")
    return a


@dataclass
class SearchResults:
    """Flat nq*k scores and ids (src/lib.rs:313-415)."""

    scores: np.ndarray
    indices: np.ndarray
    nq: int
    k: int

    def scores_for_query(self, qi: int) -> np.ndarray:
        return self.scores[qi * self.k:(qi + 1) * self.k]

    def indices_for_query(self, qi: int) -> np.ndarray:
        return self.indices[qi * self.k:(qi + 1) * self.k]


@dataclass
class CandidateBatch:
    """CSR candidate rows (src/sign_bitmap.rs:60-86)."""

    candidates: np.ndarray
    offsets: np.ndarray

    def query_count(self) -> int:
        return max(len(self.offsets) - 1, 0)

    def candidates_for_query(self, qi: int) -> Optional[np.ndarray]:
        if qi + 1 >= len(self.offsets):
            return None
        return self.candidates[self.offsets[qi]:self.offsets[qi + 1]]


@dataclass(frozen=True)
class TwoStageCandidatePolicy:
    """src/quant.rs:234-262."""

    min_candidates: int = 256
    k_multiplier: int = 32
    max_candidates: Optional[int] = None

    def candidate_count(self, k: int, search_space: int) -> int:
        if k == 0 or search_space == 0:
            return 0
        count = max(self.min_candidates, min(k * self.k_multiplier, 2**64 - 1))
        if self.max_candidates is not None:
            count = min(count, self.max_candidates)
        return min(count, search_space)


class _Index:
    """Owns one device-resident index handle."""

    _kind = 0

    def __init__(self, handle):
        self._h = handle

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            try:
                lib().ordvec_index_free(h)
            except Exception:
                pass
            self._h = None

    @property
    def handle(self):
        return self._h

    def info(self) -> IndexInfo:
        info = IndexInfo()
        lib().ordvec_index_info_init(C.byref(info))
        check(lib().ordvec_index_info(self._h, C.byref(info)))
        return info

    def __len__(self) -> int:
        return int(self.info().vector_count)

    def len(self) -> int:
        return len(self)

    def is_empty(self) -> bool:
        return len(self) == 0

    @property
    def dim(self) -> int:
        return int(self.info().dim)

    def bytes_per_vec(self) -> int:
        return int(self.info().bytes_per_vec)

    def add(self, vectors) -> None:
        v = _rows(vectors, self.dim)
        check(lib().ovb_index_add(self._h, _ptr(v), v.size // self.dim))

    def add_device(self, device_ptr: int, n: int) -> None:
        check(lib().ovb_index_add_device(self._h, C.c_void_p(device_ptr), n))

    def write(self, path: str) -> None:
        check(lib().ovb_index_write(self._h, str(path).encode()))

    def payload(self) -> np.ndarray:
        """Codes in the reference's persisted payload layout (bytes)."""
        n = C.c_uint64()
        check(lib().ovb_index_payload_bytes(self._h, C.byref(n)))
        out = np.empty(max(n.value, 1), np.uint8)
        check(lib().ovb_index_payload(self._h, _ptr(out), n.value))
        return out[: n.value]

    @classmethod
    def _wrap_loaded(cls, handle):
        obj = cls.__new__(cls)
        _Index.__init__(obj, handle)
        return obj


def _new(fn, *args):
    h = C.c_void_p()
    check(fn(*args, C.byref(h)))
    return h


def load(path: str):
    """Load any of .ovrq / .ovbm / .ovsb / .ovfs / .ovr into HBM (src/rank_io.rs)."""
    h = C.c_void_p()
    check(lib().ovb_index_load_any(str(path).encode(), 0, C.byref(h)))
    info = IndexInfo()
    lib().ordvec_index_info_init(C.byref(info))
    check(lib().ordvec_index_info(h, C.byref(info)))
    cls = {KIND_RANK_QUANT: RankQuant, KIND_BITMAP: Bitmap, KIND_SIGN_BITMAP: SignBitmap,
           KIND_FASTSCAN: RankQuantFastscan, KIND_RANK: Rank}[info.kind]
    return cls._wrap_loaded(h)


def _full_search(fn, h, n: int, dim: int, queries, k: int) -> SearchResults:
    """nq x min(k, n) results of one of the library's full searches."""
    q = _rows(queries, dim)
    nq = q.size // dim
    ke = min(k, n)
    s = np.empty(max(nq * ke, 1), np.float32)
    i = np.empty(max(nq * ke, 1), np.int64)
    check(fn(h, _ptr(q), nq, ke, _ptr(s), _ptr(i)))
    return SearchResults(s[: nq * ke], i[: nq * ke], nq, ke)


class Rank(_Index):
    """Full-precision rank index: one u16 rank per coordinate (src/rank.rs:283-482)."""

    def __init__(self, dim: int):
        super().__init__(_new(lib().ovb_rank_new, dim))

    @classmethod
    def load(cls, path: str) -> "Rank":
        obj = load(path)
        if not isinstance(obj, Rank):
            raise OrdvecError(4, "not a Rank index")
        return obj

    def search(self, queries, k: int) -> SearchResults:
        """Symmetric rank-cosine (Spearman) search, src/rank.rs:364-419."""
        return _full_search(lib().ovb_rank_search, self._h, len(self), self.dim, queries, k)

    def search_asymmetric(self, queries, k: int) -> SearchResults:
        """L2-normalised f32 query against the stored ranks, src/rank.rs:420-482."""
        return _full_search(lib().ovb_rank_search_asymmetric, self._h, len(self), self.dim, queries, k)


class RankQuant(_Index):
    """B-bit bucketed-rank index (src/quant.rs:211-1509)."""

    def __init__(self, dim: int, bits: int):
        super().__init__(_new(lib().ovb_rankquant_new, dim, bits))

    @property
    def bits(self) -> int:
        return int(self.info().bit_width)

    @classmethod
    def load(cls, path: str) -> "RankQuant":
        obj = load(path)
        if not isinstance(obj, RankQuant):
            raise OrdvecError(4, "not a RankQuant index")
        return obj

    def search(self, queries, k: int) -> SearchResults:
        """Symmetric search (src/quant.rs:629-695): the query is rank-bucketed like a document."""
        return _full_search(lib().ovb_rankquant_search_symmetric, self._h, len(self), self.dim, queries, k)

    def search_asymmetric(self, queries, k: int) -> SearchResults:
        """src/quant.rs:713-847: nq x min(k, n), (score desc, id asc)."""
        dim = self.dim
        q = _rows(queries, dim)
        nq = q.size // dim
        ke = min(k, len(self))
        s = np.empty(max(nq * ke, 1), np.float32)
        i = np.empty(max(nq * ke, 1), np.int64)
        check(lib().ovb_rankquant_search(self._h, _ptr(q), nq, ke, _ptr(s), _ptr(i)))
        if ke == 0:
            return SearchResults(np.zeros(0, np.float32), np.full(0, -1, np.int64), nq, 0)
        return SearchResults(s[: nq * ke], i[: nq * ke], nq, ke)

    def search_asymmetric_split(self, queries, k: int, exact: bool = True) -> SearchResults:
        """Full search scored on the tensor cores in split-BF16 (query = hi + lo
        BF16, codes exact in BF16, f32 accumulation).  exact=True rescores
        the candidates within the split error bound in FP64 (same results as
        search_asymmetric); exact=False returns the split-BF16 scores."""
        dim = self.dim
        q = _rows(queries, dim)
        nq = q.size // dim
        ke = min(k, len(self))
        s = np.empty(max(nq * ke, 1), np.float32)
        i = np.empty(max(nq * ke, 1), np.int64)
        check(lib().ovb_rankquant_search_split(self._h, _ptr(q), nq, ke, 1 if exact else 0, _ptr(s), _ptr(i)))
        return SearchResults(s[: nq * ke], i[: nq * ke], nq, ke)

    def search_asymmetric_subset_batched_serial(self, queries, candidate_offsets, candidates, k) -> SearchResults:
        """src/quant.rs:1336-1451: rectangular nq x min(k, n), sentinel padded."""
        dim = self.dim
        q = _rows(queries, dim)
        nq = q.size // dim
        off = np.ascontiguousarray(candidate_offsets, np.uint64)
        cand = np.ascontiguousarray(candidates, np.uint32)
        if off.size != nq + 1:
            raise OrdvecError(2, f"candidate_offsets length {off.size} must be nq+1 ({nq + 1})")
        if off[-1] != cand.size:
            raise OrdvecError(2, "candidate_offsets[nq] must equal candidates.len()")
        out_k = min(k, len(self))
        s = np.empty(max(nq * out_k, 1), np.float32)
        i = np.empty(max(nq * out_k, 1), np.int64)
        c = cand if cand.size else np.zeros(1, np.uint32)
        check(lib().ovb_rankquant_search_subset(self._h, _ptr(q), nq, _ptr(off), _ptr(c), out_k, _ptr(s), _ptr(i)))
        return SearchResults(s[: nq * out_k], i[: nq * out_k], nq, out_k)

    def search_asymmetric_subset(self, query, candidates, k: int):
        """src/quant.rs:1048-1083: returns (scores, ids) of length min(k, m)."""
        cand = np.ascontiguousarray(candidates, np.uint32)
        if cand.size > len(self):
            raise OrdvecError(12, f"search_asymmetric_subset: candidate list length {cand.size} exceeds "
                                  f"n_vectors {len(self)}; deduplicate repeated ids before calling")
        out_k = min(k, cand.size)
        if out_k == 0:
            return np.zeros(0, np.float32), np.zeros(0, np.int64)
        res = self.search_asymmetric_subset_batched_serial(query, [0, cand.size], cand, out_k)
        return res.scores[:out_k].copy(), res.indices[:out_k].copy()

    def try_search_with_sign_probe_with_policy(self, sign_probe: "SignBitmap", query, k: int,
                                               policy: TwoStageCandidatePolicy):
        """src/quant.rs:1467-1498."""
        if sign_probe.dim != self.dim:
            raise OrdvecError(2, f"sign_probe.dim: must match RankQuant dim {self.dim}")
        if len(sign_probe) != len(self):
            raise OrdvecError(2, f"sign_probe.len: must match RankQuant len {len(self)}")
        q = _rows(query, self.dim)
        if q.size != self.dim:
            raise OrdvecError(2, f"query: length {q.size}, expected {self.dim}")
        m = policy.candidate_count(k, len(self))
        cands = sign_probe.top_m_candidates(q, m)
        return self.search_asymmetric_subset(q, cands, k)

    def try_search_with_sign_probe(self, sign_probe: "SignBitmap", query, k: int):
        return self.try_search_with_sign_probe_with_policy(sign_probe, query, k, TwoStageCandidatePolicy())

    search_with_sign_probe = try_search_with_sign_probe


class SignBitmap(_Index):
    """1-bit sign fingerprints, Hamming candidate generation (src/sign_bitmap.rs)."""

    def __init__(self, dim: int):
        super().__init__(_new(lib().ovb_sign_bitmap_new, dim))

    def _top_m(self, queries, m: int) -> np.ndarray:
        dim = self.dim
        q = _rows(queries, dim)
        nq = q.size // dim
        me = min(m, len(self))
        out = np.empty(max(nq * me, 1), np.uint32)
        check(lib().ovb_sign_bitmap_top_m(self._h, _ptr(q), nq, me, _ptr(out)))
        return out[: nq * me].reshape(nq, me)

    def top_m_candidates(self, q, m: int) -> np.ndarray:
        return self._top_m(q, m)[0] if np.size(q) else np.zeros(0, np.uint32)

    def top_m_candidates_batched(self, queries, m: int) -> List[np.ndarray]:
        return list(self._top_m(queries, m))

    def top_m_candidates_batched_serial_csr(self, queries, m: int) -> CandidateBatch:
        rows = self._top_m(queries, m)
        nq, me = rows.shape
        return CandidateBatch(rows.reshape(-1).copy(), np.arange(nq + 1, dtype=np.uint64) * me)

    def score_all(self, q) -> np.ndarray:
        qq = _rows(q, self.dim)
        out = np.empty(max(len(self), 1), np.uint32)
        check(lib().ovb_sign_bitmap_score_all(self._h, _ptr(qq), _ptr(out)))
        return out[: len(self)]


class Bitmap(_Index):
    """Constant-weight top-n_top bitmaps, AND-overlap scoring (src/bitmap.rs)."""

    def __init__(self, dim: int, n_top: int):
        super().__init__(_new(lib().ovb_bitmap_new, dim, n_top))

    @property
    def n_top(self) -> int:
        return int(self.info().n_top)

    def search(self, queries, k: int) -> SearchResults:
        dim = self.dim
        q = _rows(queries, dim)
        nq = q.size // dim
        ke = min(k, len(self))
        s = np.empty(max(nq * ke, 1), np.float32)
        i = np.empty(max(nq * ke, 1), np.int64)
        check(lib().ovb_bitmap_search(self._h, _ptr(q), nq, ke, _ptr(s), _ptr(i)))
        return SearchResults(s[: nq * ke], i[: nq * ke], nq, ke)

    def _top_m(self, queries, m: int) -> np.ndarray:
        dim = self.dim
        q = _rows(queries, dim)
        nq = q.size // dim
        me = min(m, len(self))
        out = np.empty(max(nq * me, 1), np.uint32)
        check(lib().ovb_bitmap_top_m(self._h, _ptr(q), nq, me, _ptr(out)))
        return out[: nq * me].reshape(nq, me)

    def top_m_candidates(self, q, m: int) -> np.ndarray:
        return self._top_m(q, m)[0]

    def top_m_candidates_batched(self, queries, m: int) -> List[np.ndarray]:
        return list(self._top_m(queries, m))

    def search_subset(self, query, doc_ids, k: int):
        """src/bitmap.rs:470-494 through the C ABI subset search."""
        from .abi import index_search

        hits = index_search(self, query, k, candidates=doc_ids)
        return (np.array([h[2] for h in hits], np.float32), np.array([h[0] for h in hits], np.int64))


class RankQuantFastscan(_Index):
    """FastScan b=2 nibble-LUT index (src/fastscan.rs:532-705)."""

    def __init__(self, dim: int):
        super().__init__(_new(lib().ovb_fastscan_new, dim))

    def search(self, queries, k: int) -> SearchResults:
        dim = self.dim
        q = _rows(queries, dim)
        nq = q.size // dim
        ke = min(k, len(self))
        s = np.empty(max(nq * ke, 1), np.float32)
        i = np.empty(max(nq * ke, 1), np.int64)
        check(lib().ovb_fastscan_search(self._h, _ptr(q), nq, ke, _ptr(s), _ptr(i)))
        return SearchResults(s[: nq * ke], i[: nq * ke], nq, ke)


class MultiBucketBitmap(_Index):
    """2^bits bucket bitmaps per document (src/multi_bucket.rs:58-251)."""

    def __init__(self, dim: int, bits: int):
        super().__init__(_new(lib().ovb_multibucket_new, dim, bits))

    @property
    def bits(self) -> int:
        return int(self.info().bit_width)

    def _nb(self):
        return 1 << self.bits

    def diagonal_weights(self) -> np.ndarray:
        nb = self._nb()
        return np.eye(nb, dtype=np.float32).reshape(-1)

    def outer_product_weights(self) -> np.ndarray:
        nb = self._nb()
        c = np.float32((nb - 1.0) / 2.0)
        a = np.arange(nb, dtype=np.float32) - c
        return (a[:, None] * a[None, :]).astype(np.float32).reshape(-1)

    def banded_weights(self, half_width: int) -> np.ndarray:
        nb = self._nb()
        w = self.outer_product_weights().reshape(nb, nb)
        idx = np.arange(nb)
        w[np.abs(idx[:, None] - idx[None, :]) > half_width] = 0.0
        return w.reshape(-1)

    def top_m_bilinear_batched(self, queries, weights, m: int) -> np.ndarray:
        """Query bitmaps from ranks (src/multi_bucket.rs:122-137), then the
        bilinear top-m (src/multi_bucket.rs:228-251), order (score desc, id asc)."""
        dim = self.dim
        q = _rows(queries, dim)
        nq = q.size // dim
        w = np.ascontiguousarray(weights, np.float32)
        if w.size != self._nb() ** 2:
            raise OrdvecError(2, "weights must be nb x nb")
        me = min(m, len(self))
        out = np.empty(max(nq * me, 1), np.uint32)
        check(lib().ovb_multibucket_top_m(self._h, _ptr(q), nq, _ptr(w), me, _ptr(out)))
        return out[: nq * me].reshape(nq, me)


def two_stage_search(rq: RankQuant, stage1: _Index, queries, m: int, k: int) -> SearchResults:
    """Fused candidate generation (sign / FastScan / Bitmap / multi-bucket) and
    RankQuant rerank on the device; m = 0 uses TwoStageCandidatePolicy()."""
    dim = rq.dim
    q = _rows(queries, dim)
    nq = q.size // dim
    me = m if m else TwoStageCandidatePolicy().candidate_count(k, len(rq))
    me = min(me, len(rq))
    ke = min(k, me)
    s = np.empty(max(nq * ke, 1), np.float32)
    i = np.empty(max(nq * ke, 1), np.int64)
    check(lib().ovb_two_stage_search(rq.handle, stage1.handle, _ptr(q), nq, m, k, _ptr(s), _ptr(i)))
    return SearchResults(s[: nq * ke], i[: nq * ke], nq, ke)


def search_mixed(indices: Sequence[RankQuant], index_of_query, k_of_query, queries) -> SearchResults:
    """One call for queries with their own index and k (ovb_rankquant_search_mixed):
    row i holds query i's top-k_of_query[i] in indices[index_of_query[i]],
    padded to max(k_of_query) with (-inf, -1)."""
    if not indices:
        raise OrdvecError(2, "indices must not be empty")
    dim = indices[0].dim
    q = _rows(queries, dim)
    nq = q.size // dim
    sel = np.ascontiguousarray(index_of_query, np.uint32)
    ks = np.ascontiguousarray(k_of_query, np.uint32)
    if sel.size != nq or ks.size != nq:
        raise OrdvecError(2, "index_of_query and k_of_query need one entry per query")
    k_max = int(ks.max()) if nq else 0
    handles = (C.c_void_p * len(indices))(*[ix.handle.value if hasattr(ix.handle, "value") else ix.handle
                                            for ix in indices])
    s = np.empty(max(nq * k_max, 1), np.float32)
    i = np.empty(max(nq * k_max, 1), np.int64)
    check(lib().ovb_rankquant_search_mixed(handles, len(indices), _ptr(sel), _ptr(ks), _ptr(q), nq, k_max,
                                           _ptr(s), _ptr(i)))
    return SearchResults(s[: nq * k_max], i[: nq * k_max], nq, k_max)


def mixed_plan_info(rq: RankQuant, nq: int, k: int) -> dict:
    """Tuned tile (queries per tile), candidate count and graph replays of a plan."""
    qpt, kp, rep = C.c_uint32(), C.c_uint64(), C.c_uint64()
    check(lib().ovb_mixed_plan_info(rq.handle, nq, k, C.byref(qpt), C.byref(kp), C.byref(rep)))
    return {"q_per_tile": qpt.value, "candidates": kp.value, "replays": rep.value}


class Server:
    """Serving loop over device-resident indices (ovb_server_*): requests are
    queued, batched with other pending requests of the same route, k and m
    (continuous batching), admitted under an HBM budget and run by worker
    threads on their own CUDA streams.  A request's result is the one it gets
    alone."""

    def __init__(self, workers: int = 2, max_batch: int = 1024, hbm_budget_bytes: int = 0):
        cfg = _lib_mod.ServerConfig()
        cfg.struct_size = C.sizeof(_lib_mod.ServerConfig)
        cfg.workers, cfg.max_batch, cfg.hbm_budget_bytes = workers, max_batch, hbm_budget_bytes
        h = C.c_void_p()
        check(lib().ovb_server_new(C.byref(cfg), C.byref(h)))
        self._h = h
        self.workers = workers if workers else 2
        self._dims: List[int] = []
        self._keep = []  # indices must outlive the server

    def add_route(self, rq: "RankQuant", stage1: Optional["_Index"] = None) -> int:
        r = C.c_uint32()
        check(lib().ovb_server_add_route(self._h, rq.handle, stage1.handle if stage1 is not None else None,
                                         C.byref(r)))
        self._dims.append(rq.dim)
        self._keep.append((rq, stage1))
        return r.value

    def submit(self, route: int, queries, k: int, m: int = 0) -> "Ticket":
        if not 0 <= route < len(self._dims):
            raise OrdvecError(2, "unknown route")  # the status ovb_server_submit returns
        q = _rows(queries, self._dims[route])
        nq = q.size // self._dims[route]
        t = C.c_uint64()
        check(lib().ovb_server_submit(self._h, route, _ptr(q), nq, k, m, C.byref(t)))
        return Ticket(self, t.value, nq, k)

    def wait_ready(self, timeout_s: float = 60.0) -> None:
        """Block until every worker has sized its buffers for every route."""
        import time

        t_end = time.monotonic() + timeout_s
        while self.stats()["warm_workers"] < self.workers:
            if time.monotonic() > t_end:
                raise TimeoutError("server workers did not finish sizing their buffers")
            time.sleep(0.002)

    def stats(self) -> dict:
        st = _lib_mod.ServerStats()
        st.struct_size = C.sizeof(_lib_mod.ServerStats)
        check(lib().ovb_server_stats(self._h, C.byref(st)))
        return {f: getattr(st, f) for f, _ in _lib_mod.ServerStats._fields_ if f not in ("struct_size", "reserved")}

    def close(self) -> None:
        if self._h:
            lib().ovb_server_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Ticket:
    """A submitted request; wait() blocks until its results are ready."""

    def __init__(self, server: Server, ticket: int, nq: int, k: int):
        self.server, self.ticket, self.nq, self.k = server, ticket, nq, k

    def wait(self):
        cap = max(self.nq * self.k, 1)
        s = np.empty(cap, np.float32)
        i = np.empty(cap, np.int64)
        ko = C.c_uint64()
        lat = C.c_double()
        check(lib().ovb_server_wait(self.server._h, self.ticket, _ptr(s), _ptr(i), cap, C.byref(ko), C.byref(lat)))
        n = self.nq * ko.value
        return SearchResults(s[:n], i[:n], self.nq, ko.value), lat.value


def synth_docs(seed: int, n: int, dim: int, sigma: float = 0.3, first: int = 0) -> np.ndarray:
    out = np.empty((n, dim), np.float32)
    check(lib().ovb_synth_docs(seed, first, n, dim, sigma, _ptr(out)))
    return out


def synth_queries(seed: int, n_docs: int, nq: int, dim: int, doc_sigma: float = 0.3,
                  query_sigma: float = 0.1):
    out = np.empty((nq, dim), np.float32)
    planted = np.empty(nq, np.uint64)
    check(lib().ovb_synth_queries(seed, n_docs, nq, dim, doc_sigma, query_sigma, _ptr(out), _ptr(planted)))
    return out, planted


def last_launch_count() -> int:
    return int(lib().ovb_last_launch_count())


def set_device(device: int) -> None:
    check(lib().ovb_set_device(device))


RERANK_MODES = {"auto": 0, "fp64": 1, "split": 2, "split_raw": 3}


def two_stage_search_device(rq: RankQuant, stage1: _Index, d_queries: int, nq: int, m: int, k: int,
                            d_scores: int, d_ids: int, stream: int, rerank: str = "auto") -> None:
    """Device-pointer two-stage search, asynchronous on `stream` (cudaStream_t as int).
    rerank: "auto" (the FP64 tables, or with OVB_RERANK_TC=1 the split-BF16
    tensor-core rerank with exact FP64 rescoring where eligible), "fp64", "split"
    (force the exact split form) or "split_raw" (the split-BF16 scores themselves)."""
    if rerank == "auto":
        check(lib().ovb_two_stage_search_device(rq.handle, stage1.handle, C.c_void_p(d_queries), nq, m, k,
                                                C.c_void_p(d_scores), C.c_void_p(d_ids), C.c_void_p(stream)))
    else:
        check(lib().ovb_two_stage_search_device_ex(rq.handle, stage1.handle, C.c_void_p(d_queries), nq, m, k,
                                                   C.c_void_p(d_scores), C.c_void_p(d_ids), C.c_void_p(stream),
                                                   RERANK_MODES[rerank]))


def search_device(index: _Index, d_queries: int, nq: int, k: int, d_scores: int, d_ids: int, stream: int,
                  asymmetric: bool = False) -> None:
    """Device-pointer full search, asynchronous on `stream` (cudaStream_t as int):
    the index's `search` (RankQuant / Rank symmetric, Bitmap, RankQuantFastscan),
    or `search_asymmetric` (RankQuant, Rank) with asymmetric=True."""
    check(lib().ovb_index_search_device(index.handle, 1 if asymmetric else 0, C.c_void_p(d_queries), nq, k,
                                        C.c_void_p(d_scores), C.c_void_p(d_ids), C.c_void_p(stream)))


def two_stage_profile(rq: RankQuant, stage1: _Index, d_queries: int, nq: int, m: int, k: int,
                      d_scores: int, d_ids: int, stream: int) -> List[float]:
    """Synchronous device-pointer two-stage search returning per-stage device ms:
    [prep, stage-1 threshold, stage-1 scan, stage-1 select, rerank scoring,
    final select]."""
    ms = (C.c_float * 6)()
    check(lib().ovb_two_stage_profile(rq.handle, stage1.handle, C.c_void_p(d_queries), nq, m, k,
                                      C.c_void_p(d_scores), C.c_void_p(d_ids), C.c_void_p(stream), ms))
    return list(ms)
