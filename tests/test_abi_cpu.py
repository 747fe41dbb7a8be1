"""C-ABI library checks that need no GPU: it loads, exports every symbol the
header declares, keeps the ordvec.h v1 struct layouts, and validates
arguments and persisted files before touching the device."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import ordvec_b200 as ob
from ordvec_b200 import abi
from ordvec_b200._lib import Hit, IndexInfo, SearchParams, SearchStats, lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "ordvec_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b((?:ordvec|ovb)_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    L = lib()
    names = declared_functions()
    assert len(names) > 30
    for name in names:
        assert hasattr(L, name), name


def test_v1_struct_layouts_match_ordvec_h():
    # ordvec-ffi/src/lib.rs:1060-1066
    assert C.sizeof(IndexInfo) == 128
    assert C.sizeof(SearchParams) == 128
    assert C.sizeof(SearchStats) == 184
    assert C.sizeof(Hit) == 24


def test_version_status_and_init_helpers():
    L = lib()
    assert L.ordvec_abi_version() == 1
    assert L.ordvec_version_string().decode().startswith("0.6.0")
    names = [L.ordvec_status_name(s).decode() for s in range(14)]
    assert names == ["OK", "NULL_POINTER", "BAD_ARGUMENT", "BAD_STRUCT_SIZE", "UNSUPPORTED_FORMAT",
                     "CORRUPT_INDEX", "IO", "DIM_MISMATCH", "NONFINITE_QUERY", "ROW_ID_OUT_OF_RANGE",
                     "BUFFER_TOO_SMALL", "UNSUPPORTED_OPERATION", "PANIC", "INTERNAL"]
    assert L.ordvec_status_name(99).decode() == "UNKNOWN"
    info, p, s = IndexInfo(), SearchParams(), SearchStats()
    L.ordvec_index_info_init(C.byref(info))
    L.ordvec_search_params_init(C.byref(p))
    L.ordvec_search_stats_init(C.byref(s))
    assert (info.struct_size, p.struct_size, s.struct_size, s.abi_version) == (128, 128, 184, 1)
    L.ordvec_index_info_init(None)  # NULL is a no-op


def test_null_pointers_and_flags_are_rejected_before_device_use(tmp_path):
    L = lib()
    out = C.c_void_p()
    assert L.ordvec_index_load(None, 0, C.byref(out)) == 1
    assert L.ordvec_index_load(b"/nonexistent", 0, None) == 1
    assert L.ordvec_index_load(b"/nonexistent", 1, C.byref(out)) == 2
    assert L.ordvec_last_error().decode().startswith("unknown load flags")
    assert L.ordvec_index_load(b"/nonexistent/x.ovrq", 0, C.byref(out)) == 6
    assert L.ordvec_index_search(None, None, None, 0, None, None) == 1
    L.ordvec_index_free(None)


def _write(path, data):
    with open(path, "wb") as f:
        f.write(bytes(data))
    return str(path)


def test_probe_reference_golden_fixture_bytes(tmp_path):
    """tests/persistence_compat.rs:130-185 fixture bytes probe to the same metadata."""
    rq = _write(tmp_path / "a.ovrq", b"OVRQ" + bytes([1, 2, 8, 0, 0, 0, 1, 0, 0, 0, 0x05, 0xAF]))
    info = abi.index_probe(rq)
    assert (info.kind, info.dim, info.bit_width, info.vector_count, info.bytes_per_vec) == (1, 8, 2, 1, 2)
    assert info.source_file_size_bytes == 16 and info.capabilities == 0b1111
    bm = _write(tmp_path / "b.ovbm", b"OVBM" + bytes([1, 64, 0, 0, 0, 2, 0, 0, 0, 1, 0, 0, 0]) + bytes(7) + b"\xc0")
    info = abi.index_probe(bm)
    assert (info.kind, info.dim, info.n_top, info.vector_count, info.bytes_per_vec) == (2, 64, 2, 1, 8)
    legacy = _write(tmp_path / "c.tvrq", b"TVRQ" + bytes([1, 2, 8, 0, 0, 0, 1, 0, 0, 0, 0x05, 0xAF]))
    assert abi.index_probe(legacy).kind == 1


def test_load_maps_unsupported_and_corrupt_formats(tmp_path):
    """ordvec-ffi/src/lib.rs:1502-1553."""
    L = lib()
    rank = _write(tmp_path / "r.ovr", b"OVR1" + bytes([1, 16, 0, 0, 0, 1, 0, 0, 0]) + bytes(32))
    sign = _write(tmp_path / "s.ovsb", b"OVSB" + bytes([1, 64, 0, 0, 0, 1, 0, 0, 0]) + bytes(8))
    fs = _write(tmp_path / "f.ovfs", b"OVFS" + bytes([1, 8, 0, 0, 0, 0, 0, 0, 0]))
    corrupt = _write(tmp_path / "c.ovrq", b"OVRQ\x01")
    for p in (rank, sign, fs):
        out = C.c_void_p()
        assert L.ordvec_index_load(p.encode(), 0, C.byref(out)) == 4, p
        assert not out.value
    out = C.c_void_p()
    assert L.ordvec_index_load(corrupt.encode(), 0, C.byref(out)) == 5
    assert not out.value
    unknown = _write(tmp_path / "u.bin", b"NOPE1234")
    assert L.ordvec_index_load(unknown.encode(), 0, C.byref(out)) == 5


def test_probe_rejects_bad_headers(tmp_path):
    L = lib()
    info = IndexInfo()
    L.ordvec_index_info_init(C.byref(info))
    cases = [
        b"OVRQ" + bytes([1, 3, 8, 0, 0, 0, 0, 0, 0, 0]),          # bits 3
        b"OVRQ" + bytes([1, 2, 6, 0, 0, 0, 0, 0, 0, 0]),          # dim % 4
        b"OVRQ" + bytes([2, 2, 8, 0, 0, 0, 0, 0, 0, 0]),          # version 2
        b"OVRQ" + bytes([1, 2, 8, 0, 0, 0, 1, 0, 0, 0, 0x05]),    # truncated payload
        b"OVRQ" + bytes([1, 2, 8, 0, 0, 0, 1, 0, 0, 0, 5, 5, 5]),  # trailing bytes
        b"OVBM" + bytes([1, 64, 0, 0, 0, 64, 0, 0, 0, 0, 0, 0, 0]),  # n_top == dim
    ]
    for i, data in enumerate(cases):
        p = _write(tmp_path / f"bad{i}", data)
        assert L.ordvec_index_probe(p.encode(), 0, C.byref(info)) == 5, i
    bad_size = IndexInfo()
    bad_size.struct_size = 127
    ok = _write(tmp_path / "ok.ovrq", b"OVRQ" + bytes([1, 2, 8, 0, 0, 0, 1, 0, 0, 0, 0x05, 0xAF]))
    assert L.ordvec_index_probe(ok.encode(), 0, C.byref(bad_size)) == 3


def test_synth_generator_is_deterministic_per_row():
    a = ob.synth_docs(0x0DD5EED1, 20, 128)
    b = ob.synth_docs(0x0DD5EED1, 5, 128, first=10)
    assert np.array_equal(a[10:15], b)
    np.testing.assert_allclose(np.linalg.norm(a, axis=1), 1.0, rtol=1e-5)
    q1, p1 = ob.synth_queries(0x0DD5EED1, 20, 6, 128)
    q2, p2 = ob.synth_queries(0x0DD5EED1, 20, 6, 128)
    assert np.array_equal(q1, q2) and np.array_equal(p1, p2)
    assert (p1 < 20).all()
    # per-coordinate noise sigma=0.1: expected cosine to the planted doc is
    # 1/sqrt(1 + dim * 0.01) = 0.66 at dim 128
    cos = (q1 * a[p1.astype(int)]).sum(axis=1)
    assert (np.abs(cos - 1 / np.sqrt(1 + 128 * 0.01)) < 0.1).all()


def test_oracle_generator_restatement_equals_the_library_generator(orc):
    """The benchmark's CPU legs build their corpus with the oracle's restatement
    of the generator; it must give the library's rows bit for bit (doc rows at
    any offset, queries and their planted source docs)."""
    for seed, n, dim, first in ((0x0DD5EED4, 300, 768, 0), (0x0DD5EED4, 200, 768, 9_999_800), (7, 65, 256, 12)):
        a = ob.synth_docs(seed, n, dim, first=first)
        b = orc.synth_docs(seed, n, dim, first=first)
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
        qa, pa = ob.synth_queries(seed + 1, 10_000_000, 33, dim)
        qb, pb = orc.synth_queries(seed + 1, 10_000_000, 33, dim)
        assert np.array_equal(qa.view(np.uint32), qb.view(np.uint32)) and np.array_equal(pa, pb)


def test_device_entry_points_fail_cleanly_without_a_gpu():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    L = lib()
    assert L.ordvec_init() == 11
    assert "CUDA" in L.ordvec_last_error().decode()
    with pytest.raises(ob.OrdvecError):
        ob.RankQuant(64, 2)


def test_server_config_is_validated_before_device_use():
    from ordvec_b200._lib import ServerConfig, ServerStats

    L = lib()
    assert C.sizeof(ServerConfig) == 64 and C.sizeof(ServerStats) == 104
    h = C.c_void_p()
    assert L.ovb_server_new(None, C.byref(h)) == 1
    cfg = ServerConfig()
    cfg.struct_size = 8
    assert L.ovb_server_new(C.byref(cfg), C.byref(h)) == 3
    cfg.struct_size = C.sizeof(ServerConfig)
    cfg.reserved[2] = 1
    assert L.ovb_server_new(C.byref(cfg), C.byref(h)) == 2
    cfg.reserved[2] = 0
    cfg.workers = 65
    assert L.ovb_server_new(C.byref(cfg), C.byref(h)) == 2
    assert L.ovb_server_submit(None, 0, None, 0, 1, 0, C.byref(C.c_uint64())) == 1
    L.ovb_server_free(None)  # NULL is a no-op


def test_ovr_loader_validates_rows_before_device_use(tmp_path):
    """src/rank_io.rs:581-633: OVR1 rows must be permutations of [0, dim); a
    row with a value >= dim or a repeated value, and trailing bytes, are
    CORRUPT_INDEX.  ABI v1's loader refuses the format outright."""
    L = lib()
    head = b"OVR1" + bytes([1, 4, 0, 0, 0, 1, 0, 0, 0])
    good = head + bytes([0, 0, 1, 0, 2, 0, 3, 0])
    for name, data in (("trailing", good + b"\0"), ("range", head + bytes([0, 0, 1, 0, 2, 0, 4, 0])),
                       ("repeat", head + bytes([0, 0, 1, 0, 1, 0, 3, 0])), ("short", good[:-1])):
        p = _write(tmp_path / f"{name}.ovr", data)
        out = C.c_void_p()
        assert L.ovb_index_load_any(p.encode(), 0, C.byref(out)) == 5, name
        assert not out.value
    p = _write(tmp_path / "good.ovr", good)
    out = C.c_void_p()
    assert L.ordvec_index_load(p.encode(), 0, C.byref(out)) == 4


def test_rank_and_selftest_entry_points_fail_cleanly_without_a_gpu():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    L = lib()
    out = C.c_void_p()
    assert L.ovb_rank_new(1, C.byref(out)) in (2, 11)  # bad dim, or no device first
    assert L.ovb_rank_new(64, None) == 1
    t, w = C.c_uint32(), C.c_uint64()
    assert L.ovb_selftest_bounded_wait(None, None) == 1
    assert L.ovb_selftest_bounded_wait(C.byref(t), C.byref(w)) == 11
    assert L.ovb_index_search_device(None, 0, None, 0, 1, None, None, None) == 1
    # the allocation-free entry point checks for a device before anything else
    assert L.ovb_rankquant_search_noalloc(None, None, 0, 1, None, None, None) == 11
    assert "CUDA" in L.ordvec_last_error().decode()
