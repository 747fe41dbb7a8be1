"""Failure paths of the tensor-core kernels, tested without a GPU fault.

Every mbarrier wait in those kernels is bounded (about one second); a wait that
gives up sets an error word, drains, frees its tensor memory and returns, and the
host entry point reports ORDVEC_STATUS_INTERNAL.  The first test runs that wait
on a barrier nothing arrives at and checks that it gives up and that the context
still works; the second sets the error word from the host and checks that the
next tensor-core search reports it once and the one after succeeds.
"""
import ctypes as C

import numpy as np
import pytest

import ordvec_b200 as ob
from ordvec_b200._lib import OrdvecError, check, lib

pytestmark = pytest.mark.gpu


def _fastscan(n=20000, dim=256, nq=64, seed=3):
    rng = np.random.default_rng(seed)
    fs = ob.RankQuantFastscan(dim)
    fs.add(rng.standard_normal((n, dim)).astype(np.float32))
    return fs, rng.standard_normal((nq, dim)).astype(np.float32)


def test_bounded_wait_gives_up_and_context_survives():
    timed_out, waited = C.c_uint32(), C.c_uint64()
    check(lib().ovb_selftest_bounded_wait(C.byref(timed_out), C.byref(waited)))
    assert timed_out.value == 1
    assert 0.5e9 <= waited.value <= 10e9, waited.value
    fs, q = _fastscan()
    a = fs.search(q, 10)  # 64 queries: the tensor-core scan
    b = fs.search(q, 10)
    assert np.array_equal(a.indices, b.indices)


def test_error_word_reports_internal_once():
    fs, q = _fastscan(seed=4)
    want = fs.search(q, 10)
    check(lib().ovb_selftest_arm_tc_error())
    with pytest.raises(OrdvecError) as e:
        fs.search(q, 10)
    assert e.value.status == 13 and "timed out" in e.value.message
    again = fs.search(q, 10)
    assert np.array_equal(again.indices, want.indices)
    assert np.array_equal(again.scores, want.scores)
