"""ctypes/numpy wrapper over oracle/liboracle.so -- TEST INFRASTRUCTURE ONLY.

The oracle is the CPU restatement of ordvec 0.6.0's compressed-scan path
(see ordvec_oracle.h for the per-function reference citations).  Only the
test suite, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this module, and only as the checker / the timed CPU
baseline -- never as the thing measured or shipped.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
u16p = np.ctypeslib.ndpointer(np.uint16, flags="C_CONTIGUOUS")
u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
U32, U64, F32, I = C.c_uint32, C.c_uint64, C.c_float, C.c_int

_SIGS = {
    "orc_rank_transform": (None, [f32p, U32, u16p]),
    "orc_rank_to_bucket": (U32, [U32, U32, U32]),
    "orc_pack_buckets": (None, [u8p, U32, U32, u8p]),
    "orc_unpack_buckets": (None, [u8p, U32, U32, u8p]),
    "orc_bucket_centre": (F32, [U32, U32]),
    "orc_rankquant_norm": (F32, [U32, U32]),
    "orc_l2_normalise": (None, [f32p, U32, f32p]),
    "orc_policy_candidate_count": (U64, [U64, U64, I, U64, U64, U64]),
    "orc_rankquant_encode": (None, [f32p, U64, U32, U32, u8p]),
    "orc_sign_encode": (None, [f32p, U64, U32, u64p]),
    "orc_bitmap_encode": (None, [f32p, U64, U32, U32, u64p]),
    "orc_bitmap_query_fp32": (None, [f32p, U32, U32, u64p]),
    "orc_fastscan_pack": (None, [f32p, U64, U32, u8p]),
    "orc_multibucket_encode": (None, [f32p, U64, U32, U32, u64p]),
    "orc_topk_new": (C.c_void_p, [C.c_void_p, C.c_void_p, U64]),
    "orc_topk_set_score_offset": (None, [C.c_void_p, F32]),
    "orc_topk_insert": (None, [C.c_void_p, F32, U64]),
    "orc_topk_finalize": (None, [C.c_void_p, f32p, i64p, U64]),
    "orc_topk_free": (None, [C.c_void_p]),
    "orc_rq_search_asym": (U64, [u8p, U64, U32, U32, f32p, U64, U64, f32p, i64p]),
    "orc_rq_search_sym": (U64, [u8p, U64, U32, U32, f32p, U64, U64, f32p, i64p]),
    "orc_rank_encode": (None, [f32p, U64, U32, u16p]),
    "orc_rank_search_sym": (U64, [u16p, U64, U32, f32p, U64, U64, f32p, i64p]),
    "orc_rank_search_asym": (U64, [u16p, U64, U32, f32p, U64, U64, f32p, i64p]),
    "orc_rq_scores_f64": (None, [u8p, U64, U32, U32, f32p, f64p]),
    "orc_rq_scores_f64_subset": (None, [u8p, U32, U32, f32p, u32p, U64, f64p]),
    "orc_rq_subset": (U64, [u8p, U64, U32, U32, f32p, u32p, U64, U64, f32p, i64p]),
    "orc_rq_subset_batched": (U64, [u8p, U64, U32, U32, f32p, U64, u64p, u32p, U64, f32p, i64p]),
    "orc_sign_query": (None, [f32p, U32, u64p]),
    "orc_sign_hamming_all": (None, [u64p, U64, U32, f32p, u32p]),
    "orc_sign_top_m": (U64, [u64p, U64, U32, f32p, U64, u32p]),
    "orc_sign_top_m_streamed": (U64, [u64p, U64, U32, f32p, U64, U64, u32p]),
    "orc_bitmap_overlap_all": (None, [u64p, U64, U32, u64p, u32p]),
    "orc_bitmap_top_m": (U64, [u64p, U64, U32, U32, f32p, U64, u32p]),
    "orc_bitmap_search": (U64, [u64p, U64, U32, U32, f32p, U64, U64, f32p, i64p]),
    "orc_bitmap_search_subset": (U64, [u64p, U64, U32, U32, f32p, u32p, U64, U64, f32p, i64p]),
    "orc_fastscan_query": (None, [f32p, U32, u8p, C.POINTER(F32), C.POINTER(F32)]),
    "orc_fastscan_scores": (None, [u8p, U64, U32, f32p, f32p]),
    "orc_fastscan_search": (U64, [u8p, U64, U32, f32p, U64, U64, f32p, i64p]),
    "orc_multibucket_query": (None, [f32p, U32, U32, u64p]),
    "orc_multibucket_weights": (None, [U32, I, U32, f32p]),
    "orc_multibucket_scores": (None, [u64p, U64, U32, U32, u64p, f32p, f32p]),
    "orc_multibucket_top_m": (U64, [u64p, U64, U32, U32, u64p, f32p, U64, u32p]),
    "orc_xorshift_f32": (None, [U64, U64, f32p]),
    "orc_avx512_available": (I, []),
    "orc_max_threads": (I, []),
    "orc_cpu_fastscan_two_stage": (None, [u8p, u8p, U64, U32, f32p, U64, U64, U64, I, f32p, i64p, C.c_void_p]),
    "orc_cpu_sign_two_stage": (None, [u64p, u8p, U64, U32, U32, f32p, U64, U64, U64, I, f32p, i64p]),
    "orc_cpu_rq_search_asym": (None, [u8p, U64, U32, U32, f32p, U64, U64, I, f32p, i64p]),
    "orc_cpu_bitmap_two_stage": (None, [u64p, u8p, U64, U32, U32, U32, f32p, U64, U64, U64, I, f32p, i64p,
                                        C.c_void_p]),
    "orc_synth_docs": (None, [U64, U64, U64, U32, F32, f32p]),
    "orc_synth_queries": (None, [U64, U64, U64, U32, F32, F32, f32p, u64p]),
    "orc_encode_bitmap_rankquant": (None, [f32p, U64, U32, U32, U32, C.c_void_p, C.c_void_p]),
}


def build() -> str:
    """Compile the oracle C restatement (make in this directory)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(
            os.path.join(_HERE, "ordvec_oracle.c")
        ):
            build()
        L = C.CDLL(_LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _rows(a, dim):
    a = _f32(a).reshape(-1)
    assert a.size % dim == 0
    return a, a.size // dim


# ---- math -------------------------------------------------------------------
def rank_transform(v):
    v = _f32(v).reshape(-1)
    out = np.empty(v.size, np.uint16)
    lib().orc_rank_transform(v, v.size, out)
    return out


def pack_buckets(b, bits):
    b = np.ascontiguousarray(b, np.uint8)
    out = np.empty(b.size * bits // 8, np.uint8)
    lib().orc_pack_buckets(b, b.size, bits, out)
    return out


def unpack_buckets(p, dim, bits):
    p = np.ascontiguousarray(p, np.uint8)
    out = np.empty(dim, np.uint8)
    lib().orc_unpack_buckets(p, dim, bits, out)
    return out


def l2_normalise(v):
    v = _f32(v).reshape(-1)
    out = np.empty_like(v)
    lib().orc_l2_normalise(v, v.size, out)
    return out


def rankquant_norm(dim, bits):
    return lib().orc_rankquant_norm(dim, bits)


def policy_candidate_count(k, space, min_candidates=256, k_multiplier=32, max_candidates=None):
    return int(
        lib().orc_policy_candidate_count(
            min_candidates, min(k_multiplier, 2**64 - 1), max_candidates is not None,
            max_candidates or 0, min(k, 2**64 - 1), space,
        )
    )


# ---- encoders ---------------------------------------------------------------
def rankquant_encode(vecs, dim, bits):
    v, n = _rows(vecs, dim)
    out = np.empty(n * dim * bits // 8, np.uint8)
    lib().orc_rankquant_encode(v, n, dim, bits, out)
    return out


def sign_encode(vecs, dim):
    v, n = _rows(vecs, dim)
    out = np.empty(n * dim // 64, np.uint64)
    lib().orc_sign_encode(v, n, dim, out)
    return out


def bitmap_encode(vecs, dim, n_top):
    v, n = _rows(vecs, dim)
    out = np.empty(n * dim // 64, np.uint64)
    lib().orc_bitmap_encode(v, n, dim, n_top, out)
    return out


def bitmap_query(q, dim, n_top):
    out = np.empty(dim // 64, np.uint64)
    lib().orc_bitmap_query_fp32(_f32(q).reshape(-1), dim, n_top, out)
    return out


def fastscan_pack(vecs, dim):
    v, n = _rows(vecs, dim)
    out = np.empty(((n + 31) // 32) * (dim // 2) * 32, np.uint8)
    lib().orc_fastscan_pack(v, n, dim, out)
    return out


def multibucket_encode(vecs, dim, bits):
    v, n = _rows(vecs, dim)
    out = np.empty(n * (1 << bits) * (dim // 64), np.uint64)
    lib().orc_multibucket_encode(v, n, dim, bits, out)
    return out


# ---- TopK -------------------------------------------------------------------
class TopK:
    def __init__(self, k, tie_keys=None):
        self._keep = None
        if tie_keys is not None:
            self._keep = np.ascontiguousarray(tie_keys, np.uint32)
            self.h = lib().orc_topk_new(k, self._keep.ctypes.data, self._keep.size)
        else:
            self.h = lib().orc_topk_new(k, None, 0)
        self.k = k

    def set_score_offset(self, off):
        lib().orc_topk_set_score_offset(self.h, off)

    def insert(self, score, idx):
        lib().orc_topk_insert(self.h, score, idx)

    def finalize(self, length=None):
        n = self.k if length is None else length
        s = np.empty(n, np.float32)
        i = np.empty(n, np.int64)
        lib().orc_topk_finalize(self.h, s, i, n)
        return s, i

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_topk_free(self.h)
            self.h = None


# ---- searches -----------------------------------------------------------------
def rq_search_asym(packed, n, dim, bits, queries, k):
    q, nq = _rows(queries, dim)
    ke = min(k, n)
    s = np.empty(nq * ke, np.float32)
    i = np.empty(nq * ke, np.int64)
    if ke:
        lib().orc_rq_search_asym(np.ascontiguousarray(packed, np.uint8), n, dim, bits, q, nq, k, s, i)
    return s.reshape(nq, ke), i.reshape(nq, ke)


def rq_search_sym(packed, n, dim, bits, queries, k):
    """RankQuant::search (symmetric): (scores, ids) nq x min(k, n)."""
    q, nq = _rows(queries, dim)
    ke = min(k, n)
    s = np.empty(nq * ke, np.float32)
    i = np.empty(nq * ke, np.int64)
    if ke:
        lib().orc_rq_search_sym(np.ascontiguousarray(packed, np.uint8), n, dim, bits, q, nq, k, s, i)
    return s.reshape(nq, ke), i.reshape(nq, ke)


def rank_encode(vecs, dim):
    """Rank index rows: u16 rank per coordinate."""
    v, n = _rows(vecs, dim)
    out = np.empty(max(n * dim, 1), np.uint16)
    lib().orc_rank_encode(v, n, dim, out)
    return out[: n * dim]


def rank_search(ranks, n, dim, queries, k, asymmetric=False):
    """Rank::search / Rank::search_asymmetric: (scores, ids) nq x min(k, n)."""
    q, nq = _rows(queries, dim)
    ke = min(k, n)
    s = np.empty(nq * ke, np.float32)
    i = np.empty(nq * ke, np.int64)
    if ke:
        fn = lib().orc_rank_search_asym if asymmetric else lib().orc_rank_search_sym
        fn(np.ascontiguousarray(ranks, np.uint16), n, dim, q, nq, k, s, i)
    return s.reshape(nq, ke), i.reshape(nq, ke)


def rq_scores_f64(packed, n, dim, bits, query):
    out = np.empty(n, np.float64)
    lib().orc_rq_scores_f64(np.ascontiguousarray(packed, np.uint8), n, dim, bits, _f32(query).reshape(-1), out)
    return out


def rq_scores_f64_subset(packed, dim, bits, query, cands):
    c = np.ascontiguousarray(cands, np.uint32)
    out = np.empty(c.size, np.float64)
    lib().orc_rq_scores_f64_subset(np.ascontiguousarray(packed, np.uint8), dim, bits, _f32(query).reshape(-1), c, c.size, out)
    return out


def rq_subset(packed, n, dim, bits, query, cands, k):
    c = np.ascontiguousarray(cands, np.uint32)
    ke = min(k, c.size)
    s = np.empty(max(ke, 1), np.float32)
    i = np.empty(max(ke, 1), np.int64)
    if ke:
        lib().orc_rq_subset(np.ascontiguousarray(packed, np.uint8), n, dim, bits, _f32(query).reshape(-1), c, c.size, k, s, i)
    return s[:ke], i[:ke]


def rq_subset_batched(packed, n, dim, bits, queries, offsets, cands, k):
    q, nq = _rows(queries, dim)
    out_k = min(k, n)
    s = np.full(max(nq * out_k, 1), np.nan, np.float32)
    i = np.full(max(nq * out_k, 1), -7, np.int64)
    off = np.ascontiguousarray(offsets, np.uint64)
    c = np.ascontiguousarray(cands, np.uint32)
    if c.size == 0:
        c = np.zeros(1, np.uint32)
    lib().orc_rq_subset_batched(np.ascontiguousarray(packed, np.uint8), n, dim, bits, q, nq, off, c, k, s, i)
    return s[: nq * out_k].reshape(nq, out_k), i[: nq * out_k].reshape(nq, out_k)


def sign_hamming_all(words, n, dim, q):
    out = np.empty(n, np.uint32)
    lib().orc_sign_hamming_all(np.ascontiguousarray(words, np.uint64), n, dim, _f32(q).reshape(-1), out)
    return out


def sign_top_m(words, n, dim, q, m):
    me = min(m, n)
    out = np.empty(max(me, 1), np.uint32)
    if me:
        lib().orc_sign_top_m(np.ascontiguousarray(words, np.uint64), n, dim, _f32(q).reshape(-1), m, out)
    return out[:me]


def sign_top_m_streamed(words, n, dim, queries, m):
    q, nq = _rows(queries, dim)
    me = min(m, n)
    out = np.empty(max(nq * me, 1), np.uint32)
    if me and nq:
        lib().orc_sign_top_m_streamed(np.ascontiguousarray(words, np.uint64), n, dim, q, nq, m, out)
    return out[: nq * me].reshape(nq, me)


def bitmap_overlap_all(words, n, dim, qbm):
    out = np.empty(n, np.uint32)
    lib().orc_bitmap_overlap_all(np.ascontiguousarray(words, np.uint64), n, dim, np.ascontiguousarray(qbm, np.uint64), out)
    return out


def bitmap_top_m(words, n, dim, n_top, q, m):
    me = min(m, n)
    out = np.empty(max(me, 1), np.uint32)
    if me:
        lib().orc_bitmap_top_m(np.ascontiguousarray(words, np.uint64), n, dim, n_top, _f32(q).reshape(-1), m, out)
    return out[:me]


def bitmap_search(words, n, dim, n_top, queries, k):
    q, nq = _rows(queries, dim)
    ke = min(k, n)
    s = np.empty(max(nq * ke, 1), np.float32)
    i = np.empty(max(nq * ke, 1), np.int64)
    if ke:
        lib().orc_bitmap_search(np.ascontiguousarray(words, np.uint64), n, dim, n_top, q, nq, k, s, i)
    return s[: nq * ke].reshape(nq, ke), i[: nq * ke].reshape(nq, ke)


def bitmap_search_subset(words, n, dim, n_top, query, ids, k):
    c = np.ascontiguousarray(ids, np.uint32)
    ke = min(k, c.size)
    s = np.empty(max(ke, 1), np.float32)
    i = np.empty(max(ke, 1), np.int64)
    if ke:
        lib().orc_bitmap_search_subset(np.ascontiguousarray(words, np.uint64), n, dim, n_top, _f32(query).reshape(-1), c, c.size, k, s, i)
    return s[:ke], i[:ke]


def fastscan_query(q_unit, dim):
    lut = np.empty(dim * 8, np.uint8)
    b = F32()
    iq = F32()
    lib().orc_fastscan_query(_f32(q_unit).reshape(-1), dim, lut, C.byref(b), C.byref(iq))
    return lut, b.value, iq.value


def fastscan_scores(blocks, n, dim, query):
    out = np.empty(n, np.float32)
    lib().orc_fastscan_scores(np.ascontiguousarray(blocks, np.uint8), n, dim, _f32(query).reshape(-1), out)
    return out


def fastscan_search(blocks, n, dim, queries, k):
    q, nq = _rows(queries, dim)
    ke = min(k, n)
    s = np.empty(max(nq * ke, 1), np.float32)
    i = np.empty(max(nq * ke, 1), np.int64)
    if ke:
        lib().orc_fastscan_search(np.ascontiguousarray(blocks, np.uint8), n, dim, q, nq, k, s, i)
    return s[: nq * ke].reshape(nq, ke), i[: nq * ke].reshape(nq, ke)


def multibucket_query(q, dim, bits):
    out = np.empty((1 << bits) * (dim // 64), np.uint64)
    lib().orc_multibucket_query(_f32(q).reshape(-1), dim, bits, out)
    return out


def multibucket_weights(bits, kind="diagonal", half_width=0):
    k = {"diagonal": 0, "outer": 1, "banded": 2}[kind]
    w = np.empty((1 << bits) ** 2, np.float32)
    lib().orc_multibucket_weights(bits, k, half_width, w)
    return w


def multibucket_scores(words, n, dim, bits, qbm, w):
    out = np.empty(n, np.float32)
    lib().orc_multibucket_scores(np.ascontiguousarray(words, np.uint64), n, dim, bits, np.ascontiguousarray(qbm, np.uint64), _f32(w), out)
    return out


def multibucket_top_m(words, n, dim, bits, qbm, w, m):
    me = min(m, n)
    out = np.empty(max(me, 1), np.uint32)
    if me:
        lib().orc_multibucket_top_m(np.ascontiguousarray(words, np.uint64), n, dim, bits, np.ascontiguousarray(qbm, np.uint64), _f32(w), m, out)
    return out[:me]


def xorshift_f32(seed, count):
    out = np.empty(count, np.float32)
    lib().orc_xorshift_f32(seed, count, out)
    return out


# ---- timed CPU baseline (AVX-512 + OpenMP restatement) -------------------------
def cpu_fastscan_two_stage(blocks, packed_b2, n, dim, queries, n_candidates, k, threads, want_candidates=False):
    """FastScan top-n_candidates -> RankQuant b=2 subset rerank, parallel over
    queries.  Returns (scores, ids) nq x min(k, n_candidates, n) and, with
    want_candidates, the nq x min(n_candidates, n) candidate rows."""
    q, nq = _rows(queries, dim)
    cand = min(n_candidates, n)
    out_k = min(k, cand)
    s = np.empty(nq * out_k, np.float32)
    i = np.empty(nq * out_k, np.int64)
    cands = np.empty(max(nq * cand, 1), np.uint32) if want_candidates else None
    lib().orc_cpu_fastscan_two_stage(np.ascontiguousarray(blocks, np.uint8), np.ascontiguousarray(packed_b2, np.uint8),
                                     n, dim, q, nq, n_candidates, k, threads, s, i,
                                     cands.ctypes.data if cands is not None else None)
    out = (s.reshape(nq, out_k), i.reshape(nq, out_k))
    if want_candidates:
        return out + (cands[: nq * cand].reshape(nq, cand),)
    return out


def cpu_sign_two_stage(sign_words, packed, n, dim, bits, queries, m, k, threads):
    q, nq = _rows(queries, dim)
    out_k = min(k, m, n)
    s = np.empty(nq * out_k, np.float32)
    i = np.empty(nq * out_k, np.int64)
    lib().orc_cpu_sign_two_stage(np.ascontiguousarray(sign_words, np.uint64), np.ascontiguousarray(packed, np.uint8),
                                 n, dim, bits, q, nq, m, k, threads, s, i)
    return s.reshape(nq, out_k), i.reshape(nq, out_k)


def cpu_rq_search_asym(packed, n, dim, bits, queries, k, threads):
    q, nq = _rows(queries, dim)
    ke = min(k, n)
    s = np.empty(nq * ke, np.float32)
    i = np.empty(nq * ke, np.int64)
    lib().orc_cpu_rq_search_asym(np.ascontiguousarray(packed, np.uint8), n, dim, bits, q, nq, k, threads, s, i)
    return s.reshape(nq, ke), i.reshape(nq, ke)


def cpu_bitmap_two_stage(words, packed, n, dim, n_top, bits, queries, m, k, threads, want_candidates=False):
    """Bitmap top-m (batched chunks of 8 queries, AVX-512) -> RankQuant subset
    rerank, parallel over query groups.  Returns (scores, ids) nq x min(k, m, n)
    and, with want_candidates, the nq x min(m, n) candidate rows."""
    q, nq = _rows(queries, dim)
    me = min(m, n)
    out_k = min(k, me)
    s = np.empty(max(nq * out_k, 1), np.float32)
    i = np.empty(max(nq * out_k, 1), np.int64)
    cands = np.empty(max(nq * me, 1), np.uint32) if want_candidates else None
    lib().orc_cpu_bitmap_two_stage(np.ascontiguousarray(words, np.uint64), np.ascontiguousarray(packed, np.uint8),
                                   n, dim, n_top, bits, q, nq, m, k, threads, s, i,
                                   cands.ctypes.data if cands is not None else None)
    out = (s[: nq * out_k].reshape(nq, out_k), i[: nq * out_k].reshape(nq, out_k))
    if want_candidates:
        return out + (cands[: nq * me].reshape(nq, me),)
    return out


# ---- benchmark corpus (the seeded clustered-Gaussian generator) ------------------
DOC_SIGMA, QUERY_SIGMA = 0.3, 0.1


def synth_docs(seed, n, dim, sigma=DOC_SIGMA, first=0):
    """Rows first .. first+n-1 of the benchmark corpus (n x dim float32)."""
    out = np.empty((n, dim), np.float32)
    lib().orc_synth_docs(seed, first, n, dim, sigma, out.reshape(-1))
    return out


def synth_queries(seed, n_docs, nq, dim, doc_sigma=DOC_SIGMA, query_sigma=QUERY_SIGMA):
    """(queries nq x dim float32, planted source doc ids)."""
    out = np.empty((nq, dim), np.float32)
    planted = np.empty(nq, np.uint64)
    lib().orc_synth_queries(seed, n_docs, nq, dim, doc_sigma, query_sigma, out.reshape(-1), planted)
    return out, planted


def encode_bitmap_rankquant(vecs, dim, n_top, bits, bitmap_out=None, rq_out=None):
    """One rank transform per row, both layouts written (each output optional):
    the bytes of bitmap_encode and rankquant_encode."""
    v, n = _rows(vecs, dim)
    if bitmap_out is not None:
        assert bitmap_out.dtype == np.uint64 and bitmap_out.flags.c_contiguous and bitmap_out.size == n * (dim // 64)
    if rq_out is not None:
        assert rq_out.dtype == np.uint8 and rq_out.flags.c_contiguous and rq_out.size == n * dim * bits // 8
    lib().orc_encode_bitmap_rankquant(v, n, dim, n_top, bits,
                                      bitmap_out.ctypes.data if bitmap_out is not None else None,
                                      rq_out.ctypes.data if rq_out is not None else None)


def avx512_available():
    return bool(lib().orc_avx512_available())


def max_threads():
    return int(lib().orc_max_threads())
