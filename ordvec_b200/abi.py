"""Thin ctypes helpers over the ordvec C ABI v1 entry points
(ordvec-ffi/include/ordvec.h), used the way a C or cgo caller would use them."""
from __future__ import annotations

import ctypes as C
from typing import List, Optional, Tuple

import numpy as np

from ._lib import Hit, IndexInfo, SearchParams, SearchStats, check, lib


def index_load(path: str):
    h = C.c_void_p()
    check(lib().ordvec_index_load(str(path).encode(), 0, C.byref(h)))
    return h


def index_probe(path: str) -> IndexInfo:
    info = IndexInfo()
    lib().ordvec_index_info_init(C.byref(info))
    check(lib().ordvec_index_probe(str(path).encode(), 0, C.byref(info)))
    return info


def index_search(index, query, k: int, candidates=None, user_tag: int = 0,
                 stats: Optional[SearchStats] = None) -> List[Tuple[int, int, float]]:
    """ordvec_index_search on one query; returns [(row_id, id, score)]."""
    h = index.handle if hasattr(index, "handle") else index
    q = np.ascontiguousarray(query, np.float32).reshape(-1)
    p = SearchParams()
    lib().ordvec_search_params_init(C.byref(p))
    p.query = q.ctypes.data_as(C.POINTER(C.c_float))
    p.dim = q.size
    p.k = k
    cand = None
    if candidates is not None:
        cand = np.ascontiguousarray(candidates, np.uint32)
        if cand.size:
            p.candidate_rows = cand.ctypes.data_as(C.POINTER(C.c_uint32))
        p.candidate_count = cand.size
    p.user_tag = user_tag
    cap = max(int(k), 1)
    if candidates is not None:
        cap = max(min(int(k), cand.size), 1)
    hits = (Hit * cap)()
    returned = C.c_uint64()
    check(lib().ordvec_index_search(h, C.byref(p), hits, cap, C.byref(returned),
                                    C.byref(stats) if stats is not None else None))
    return [(hits[i].row_id, hits[i].id, hits[i].score) for i in range(returned.value)]
