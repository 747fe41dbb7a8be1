"""The multi-GPU (replica) path's host logic, run as two gloo ranks on CPU.

A replica job gives every rank the whole index and its own query shard; the
only collectives are a barrier and the max over ranks of the timed totals.
These tests check that plumbing (ordvec_b200/replicas.py, used by bench.py)
without a GPU: the per-rank compute is the oracle's two-stage search, so the
sharded job must return exactly what one process returns for the same shards.
"""
import json
import os
import socket
import subprocess
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
N, DIM, NQ, M, K = 3000, 128, 6, 64, 5
SEED = 0x5EED


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _env(rank: int, world: int, port: int) -> None:
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))


def _shard_search(rank: int):
    import ordvec_b200 as ob
    from oracle import oracle as orc
    from ordvec_b200.replicas import shard_seed

    docs = ob.synth_docs(SEED, N, DIM)
    queries, _ = ob.synth_queries(shard_seed(SEED, rank), N, NQ, DIM)
    blocks = orc.fastscan_pack(docs, DIM)
    packed = orc.rankquant_encode(docs, DIM, 2)
    return orc.cpu_fastscan_two_stage(blocks, packed, N, DIM, queries, M, K, 1)


def _replica_worker(rank, world, port, out_dir):
    sys.path.insert(0, ROOT)
    _env(rank, world, port)
    from ordvec_b200.replicas import ReplicaGroup, whole_job_rate

    g = ReplicaGroup("gloo", device="cpu", timeout_s=60)
    scores, ids = _shard_search(rank)
    g.barrier()
    slowest = g.max_over_ranks(10.0 * (rank + 1))
    rate = whole_job_rate(NQ, g.world, slowest)
    np.savez(os.path.join(out_dir, f"rank{rank}.npz"), scores=scores, ids=ids)
    with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
        json.dump({"max": slowest, "rate": rate, "root": g.is_root, "world": g.world}, f)
    g.close()


def _dropout_worker(rank, world, port, out_dir):
    sys.path.insert(0, ROOT)
    _env(rank, world, port)
    from ordvec_b200.replicas import ReplicaGroup

    g = ReplicaGroup("gloo", device="cpu", timeout_s=10)
    g.barrier()
    if rank == 1:
        os._exit(0)  # leaves between steps, before the next collective
    status = "ok"
    try:
        g.barrier()
    except Exception as e:  # the survivor learns of it from the collective
        status = "error: " + type(e).__name__
    with open(os.path.join(out_dir, f"rank{rank}.txt"), "w") as f:
        f.write(status)


def test_two_gloo_ranks_match_one_process(orc, tmp_path):
    port = _free_port()
    mp.start_processes(_replica_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    info = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(2)]
    assert [i["max"] for i in info] == [20.0, 20.0]  # max over ranks, seen by both
    assert [i["root"] for i in info] == [True, False]
    assert all(i["world"] == 2 for i in info)
    assert info[0]["rate"] == pytest.approx(2 * NQ / 0.020)
    for r in range(2):
        got = np.load(tmp_path / f"rank{r}.npz")
        want_s, want_i = _shard_search(r)
        assert np.array_equal(got["ids"], want_i)
        assert np.array_equal(got["scores"].view(np.uint32), want_s.view(np.uint32))
    # the shards are different queries
    assert not np.array_equal(np.load(tmp_path / "rank0.npz")["ids"], np.load(tmp_path / "rank1.npz")["ids"])


def test_rank_that_leaves_is_seen_by_the_survivor(tmp_path):
    port = _free_port()
    mp.start_processes(_dropout_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    assert (tmp_path / "rank0.txt").read_text().startswith("error")


def test_single_rank_group_is_a_no_op(monkeypatch):
    from ordvec_b200.replicas import ReplicaGroup, shard_seed, whole_job_rate

    for var in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        monkeypatch.delenv(var, raising=False)
    g = ReplicaGroup("gloo")
    assert (g.rank, g.world, g.is_root) == (0, 1, True)
    g.barrier()
    assert g.max_over_ranks(3.25) == 3.25
    g.close()
    assert shard_seed(7, 0) == 7 and shard_seed(7, 2) == 2007
    assert whole_job_rate(1000, 4, 500.0) == pytest.approx(8000.0)
    with pytest.raises(ValueError):
        whole_job_rate(1, 1, 0.0)


def test_reference_arm_runs_on_rank_zero_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2"],
                       env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0
    assert r.stdout.strip() == ""
