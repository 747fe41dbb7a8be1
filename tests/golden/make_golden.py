"""Generate tests/golden/tiled_candgen.npz from the reference's own test definitions.

The reference (ordvec 0.6.0, Rust) cannot be built in this environment, so its
candidate-generation contract is pinned through the test that defines it:
``tests/tiled_candgen.rs``.  That test builds its corpora with a self-contained
XorShift generator (lines 12-39) and defines the expected top-m rows with an
implementation-independent oracle: dense sign-agreement scores plus a full
lexicographic sort by ``(hamming asc, doc_id asc)`` (lines 41-49).

This script restates both in pure Python/numpy -- independently of the C oracle
under ``oracle/`` -- and stores, for every case of the test, the first 64
corpus values (to pin the generator) and the expected rows at the largest m of
the case (smaller m are prefixes of the same sorted order).

Run:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import os

import numpy as np

MASK = (1 << 64) - 1


def xorshift_corpus(dim: int, n: int, seed: int) -> np.ndarray:
    """XorShift::next_f32 stream of tests/tiled_candgen.rs:12-27, seed | 1."""
    x = (seed | 1) & MASK
    out = np.empty(n * dim, np.float32)
    for i in range(n * dim):
        x ^= (x << 13) & MASK
        x ^= x >> 7
        x ^= (x << 17) & MASK
        out[i] = np.float32(np.float32(x >> 40) / np.float32(8388608.0)) - np.float32(1.0)
    return out


def tie_heavy_corpus(dim: int, n: int) -> np.ndarray:
    """tie_heavy_corpus of tests/tiled_candgen.rs:32-39."""
    doc = np.arange(n)[:, None] % 4
    c = np.arange(dim)[None, :]
    return np.where((c + doc) % 3 == 0, -1.0, 1.0).astype(np.float32).reshape(-1)


def oracle_top_m(vectors: np.ndarray, queries: np.ndarray, dim: int, m: int) -> np.ndarray:
    """oracle_top_m of tests/tiled_candgen.rs:41-49: sort by (dim - agreement, id)."""
    d = vectors.reshape(-1, dim) > 0.0
    q = queries.reshape(-1, dim) > 0.0
    n = d.shape[0]
    rows = []
    for qi in range(q.shape[0]):
        ham = (d != q[qi][None, :]).sum(axis=1).astype(np.int64)
        order = np.lexsort((np.arange(n), ham))
        rows.append(order[: min(m, n)].astype(np.uint32))
    return np.stack(rows)


CASES = [
    # name, dim, corpus spec, query spec, m values  (tests/tiled_candgen.rs:83-175)
    ("random", 512, ("xs", 10_240, 0xC0FFEE), ("xs", 33, 0xBEEF), [1, 7, 256, 500]),
    ("tie_heavy", 64, ("tie", 4_096, 0), ("xs", 9, 0xABCD), [1, 3, 100, 1_000]),
    ("duplicates", 64, ("dup", 8, 0x1234), ("xs", 5, 0x9999), [10, 100, 513]),
    ("edge", 64, ("xs", 17, 0x42), ("xs", 3, 0x43), [17, 25, 1]),
    ("single_doc", 64, ("xs", 1, 0x77), ("xs", 3, 0x43), [4]),
    ("dim1024", 1024, ("xs", 6_000, 0xA5A5), ("xs", 8, 0x5A5A), [256, 320]),
    ("dim768_tail", 768, ("xs", 3_200, 0x7E57), ("xs", 7, 0x7E58), [64, 320]),
]


def make_corpus(spec, dim):
    kind, n, seed = spec
    if kind == "xs":
        return xorshift_corpus(dim, n, seed)
    if kind == "tie":
        return tie_heavy_corpus(dim, n)
    base = xorshift_corpus(dim, n, seed)  # "dup": 8 distinct rows repeated 512x
    return np.tile(base, 512)


def main():
    out = {}
    for name, dim, cspec, qspec, ms in CASES:
        vec = make_corpus(cspec, dim)
        qs = make_corpus(qspec, dim)
        mmax = max(ms)
        out[f"{name}__expected"] = oracle_top_m(vec, qs, dim, mmax)
        out[f"{name}__head"] = vec[:64].copy()
        out[f"{name}__qhead"] = qs[:64].copy()
        out[f"{name}__meta"] = np.array(
            [dim, cspec[1], cspec[2], qspec[1], qspec[2], {"xs": 0, "tie": 1, "dup": 2}[cspec[0]]]
            + ms, np.uint64)
        print(name, out[f"{name}__expected"].shape)
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tiled_candgen.npz")
    np.savez_compressed(path, **out)
    print("wrote", path)


if __name__ == "__main__":
    main()
