"""Calls made first in a fresh process.  A kernel launch whose static plus
dynamic shared memory passes 48 KiB needs the dynamic-size opt-in even when
the dynamic part alone is small; earlier calls in a long test run can set it
for later ones and hide a missing opt-in, so these calls run in a child
process of their own."""
import os
import subprocess
import sys
import textwrap

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _child(code: str, tmp_path) -> None:
    r = subprocess.run([sys.executable, "-c", textwrap.dedent(code)], cwd=ROOT, capture_output=True, text=True,
                       timeout=600, env=dict(os.environ, OVB_OUT=str(tmp_path)))
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-4000:]


def test_first_call_one_query_bitmap_top_m(orc, tmp_path):
    """One query's top-500 over 60,000 bitmap rows, the process's first
    search: the 8-CTA cluster select stages each CTA's 7,500 keys (30 KB) in
    shared memory beside its 32 KB of static shared memory."""
    _child("""
        import os, numpy as np, ordvec_b200 as ob
        docs = ob.synth_docs(61, 60_000, 768)
        q, _ = ob.synth_queries(61, 60_000, 1, 768)
        bm = ob.Bitmap(768, 192)
        bm.add(docs)
        np.save(os.path.join(os.environ["OVB_OUT"], "got.npy"), np.asarray(bm.top_m_candidates(q[0], 500)))
    """, tmp_path)
    import ordvec_b200 as ob

    docs = ob.synth_docs(61, 60_000, 768)
    q, _ = ob.synth_queries(61, 60_000, 1, 768)
    words = orc.bitmap_encode(docs, 768, 192)
    got = np.load(tmp_path / "got.npy")
    assert np.array_equal(got, orc.bitmap_top_m(words, 60_000, 768, 192, q[0], 500))
