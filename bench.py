"""Benchmark: the large-corpus configuration on B200 -- Bitmap (n_top=192)
top-2,000 candidates -> RankQuant b=2 asymmetric rerank, top-100, over
N=10,000,000 dim-768 docs resident in HBM, batches of 1,024 queries.

One step = one batch of 1,024 synthetic queries through the whole two-stage
path.  Prints ONE JSON line (rank 0).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

value  : device-timed QPS of the batched form (each step's 1,024 queries in one
         fused call), queries resident in HBM; L2 flushed (256 MiB write)
         between steps, outside the timed region (the 0.96 GB of bitmap codes
         and the 1.92 GB of RankQuant codes exceed L2 anyway).
e2e    : the same step through the public C ABI (ovb_two_stage_search) from
         pinned host buffers: H2D of the queries and D2H of the top-100 inside
         the timed region.
plain  : one query per call (device pointers), p50/p99 and QPS, and whether its
         top-100 ids equal the batched form's.
roofline: the dominant kernel, bitmap_pair_kernel (the stage-1 overlap scan as
         a u8 GEMM on tcgen05), timed by the stage events of every timed step.
cpu_baseline / --impl reference: the oracle's AVX-512 + OpenMP restatement of
         the reference path (Bitmap::top_m_candidates_batched_chunked in groups
         of 8 queries, then the AVX-512 subset rerank), all host threads, on a
         bounded query sample; the reference arm builds its inputs with the
         oracle's restatement of the corpus generator and never loads the
         product library.
Extra keys (one GPU): the multi-bucket stage-1 variant of the same corpus, the
FastScan two-stage configuration (N=171,332, dim 1024), the mixed-k/bits batch,
the sign->b1 configuration, the three-index serving loop and the Rank modes.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "QPS & scan HBM GB/s vs peak, batched vs plain GPU @ identical top-10; p50/p99 ms"
# headline workload: the large-corpus configuration
N_DOCS, DIM, NQ, K, M, N_TOP, BITS = 10_000_000, 768, 1024, 100, 2000, 192, 2
QPV = DIM // 64
SEED = 0x0DD5EED4  # corpus; queries use SEED + 1 (+1000 per rank)
BUILD_CHUNK = 1_000_000
STAGES = ["prep", "threshold", "scan", "select", "rerank", "final_select"]
WORKLOAD = (f"large_corpus_bitmap_two_stage: Bitmap n_top={N_TOP} top-{M} -> RankQuant b={BITS} asymmetric "
            f"rerank top-{K}; N={N_DOCS} dim={DIM}; {NQ} queries per step")
# DRAM traffic of one filter launch of bitmap_fp4_pair_kernel at this workload
# (ncu dram__bytes_read.sum 961,795,328 + dram__bytes_write.sum 65,410,304 on the
# full 10M-doc launch): the codes cross HBM once, the rest is the kept candidates.
PAIR_FILTER_DRAM_BYTES = 1_027_205_632
# FastScan two-stage configuration (extra key)
FS_N, FS_DIM, FS_NQ, FS_K, FS_M, FS_SEED = 171_332, 1024, 1000, 10, 1000, 0x0DD5EED2
# DRAM traffic of one filter launch of fastscan_persist_kernel at that workload, from an ncu capture
# (52,310,016 B read + 2,875,392 B written).
FS_TC_FILTER_DRAM_BYTES = 52_310_016 + 2_875_392
# the reference arm keeps its whole run (warm-up + timed steps) near this many seconds
REFERENCE_BUDGET_S = 150.0


def headline_config(world: int) -> dict:
    return {"workload": WORKLOAD, "n_docs": N_DOCS, "dim": DIM, "queries_per_step_per_gpu": NQ, "k": K,
            "candidates": M, "stage1": f"Bitmap n_top={N_TOP} (constant weight)", "rerank": f"RankQuant b={BITS}",
            "form": "batched (one fused two-stage call per step)",
            "l2": "inputs larger than L2 (0.96 GB bitmap + 1.92 GB RankQuant codes) and a 256 MiB device write "
                  "between steps, outside the timed region",
            "parallelism": f"replicas x{world} (queries sharded per rank, no data-path collective)"}


def query_seed(rank: int) -> int:
    return SEED + 1 + 1000 * rank


def measured_peaks():
    """(HBM GB/s, bf16 dense TFLOP/s burst, source)."""
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d.get("hbm_gbs", 6650.0)), float(d.get("bf16_tflops", 1590.0)), "measured"
    return 6650.0, 1590.0, "fallback"


# ----------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.path = tempfile.mktemp(suffix=".csv")
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# ------------------------------------------------------------ CPU helpers
def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def oracle_codes(orc, docs, first, words, packed):
    """Oracle-encode a chunk of docs into the host code arrays (rows first..)."""
    n = docs.shape[0]
    orc.encode_bitmap_rankquant(docs, DIM, N_TOP, BITS, words[first * QPV:(first + n) * QPV],
                                packed[first * DIM * BITS // 8:(first + n) * DIM * BITS // 8])


def topk_agreement(orc, packed, dim, bits, queries, ids_a, ids_b):
    """Compare two top-k id matrices of the same queries.  Returns (identical,
    equal_up_to_fp64_near_ties, rows_differing): rows are ordered by FP64 score
    (desc, id asc) and may differ only at positions whose FP64 scores are within
    1e-5 * max(|s|, 1e-3) of each other (the float contract of the rerank)."""
    same = bool(np.array_equal(ids_a, ids_b))
    if same:
        return True, True, 0
    ok, rows = True, 0
    for qi in range(ids_a.shape[0]):
        a, b = ids_a[qi], ids_b[qi]
        if np.array_equal(a, b):
            continue
        rows += 1
        va, vb = a[a >= 0].astype(np.uint32), b[b >= 0].astype(np.uint32)
        if va.size != vb.size:
            ok = False
            continue
        sa = orc.rq_scores_f64_subset(packed, dim, bits, queries[qi], va)
        sb = orc.rq_scores_f64_subset(packed, dim, bits, queries[qi], vb)
        oa, ob_ = np.lexsort((va, -sa)), np.lexsort((vb, -sb))
        sa, sb = sa[oa], sb[ob_]
        tol = 1e-5 * np.maximum(np.maximum(np.abs(sa), np.abs(sb)), 1e-3)
        if np.any(np.abs(sa - sb) > tol):
            ok = False
    return False, ok, rows


def split_error_stats(orc, packed, dim, bits, queries, ids, scores):
    """Largest |score - FP64 score| and relative error (|d| / max(|s64|, 1e-3))
    of returned (ids, scores) rows against the oracle's FP64 scores."""
    max_abs = max_rel = 0.0
    for qi in range(ids.shape[0]):
        v = ids[qi] >= 0
        s64 = orc.rq_scores_f64_subset(packed, dim, bits, queries[qi], ids[qi][v].astype(np.uint32))
        d = np.abs(scores[qi][v].astype(np.float64) - s64)
        if d.size:
            max_abs = max(max_abs, float(d.max()))
            max_rel = max(max_rel, float((d / np.maximum(np.abs(s64), 1e-3)).max()))
    return max_abs, max_rel


def rerank_report(ob, orc, torch, dev, rq, s1, d_q, queries, m, k, packed, sample, profile):
    """The rerank of a two-stage batch: the split-BF16 tensor-core form
    (OVB_RERANK_TC=1: tcgen05 contraction + margin test + FP64 rescoring of the
    top 2k + 32) beside the default FP64-table rerank -- stage times of the
    split form, and the error against the oracle's FP64 scores of the raw
    split-BF16 scores and of the returned scores, over `sample` queries."""
    nq = d_q.shape[0]
    sp = torch.cuda.current_stream(dev).cuda_stream
    d_s = torch.empty(nq * k, dtype=torch.float32, device=dev)
    d_i = torch.empty(nq * k, dtype=torch.int64, device=dev)
    out = {"default_form": "FP64 per-query nibble tables (CUDA cores)",
           "split_form": "split-BF16 tcgen05 (codes exact in BF16, query hi+lo BF16, f32 accumulation) + margin test "
                         "+ FP64 rescoring of the top 2k+32"}
    os.environ["OVB_RERANK_TC"] = "1"
    try:
        st = profile()
    finally:
        del os.environ["OVB_RERANK_TC"]
    out["split_rerank_ms"], out["split_final_select_ms"] = st[4], st[5]
    if orc is None or packed is None:
        return out
    ob.two_stage_search_device(rq, s1, d_q.data_ptr(), nq, m, k, d_s.data_ptr(), d_i.data_ptr(), sp,
                               rerank="split_raw")
    torch.cuda.synchronize(dev)
    raw_s, raw_i = d_s.view(nq, k).cpu().numpy()[:sample], d_i.view(nq, k).cpu().numpy()[:sample]
    ob.two_stage_search_device(rq, s1, d_q.data_ptr(), nq, m, k, d_s.data_ptr(), d_i.data_ptr(), sp, rerank="split")
    torch.cuda.synchronize(dev)
    ex_s, ex_i = d_s.view(nq, k).cpu().numpy()[:sample], d_i.view(nq, k).cpu().numpy()[:sample]
    dim, bits = rq.dim, rq.bits
    a, r = split_error_stats(orc, packed, dim, bits, queries[:sample], raw_i, raw_s)
    out["split_bf16_max_abs_err_vs_fp64"], out["split_bf16_max_rel_err_vs_fp64"] = a, r
    a, r = split_error_stats(orc, packed, dim, bits, queries[:sample], ex_i, ex_s)
    out["rerank_max_abs_err_vs_fp64"], out["rerank_max_rel_err_vs_fp64"] = a, r
    out["error_sample_queries"] = sample
    return out


def cpu_sample_size(probe_qps: float, budget_s: float, group: int, cap: int) -> int:
    q = int(probe_qps * budget_s) // group * group
    return max(group, min(cap, q))


# ------------------------------------------------------------ reference arm
def cpu_headline_inputs(orc):
    """The headline corpus encoded on the host by the oracle (no product code):
    bitmap words, RankQuant b=2 codes and rank 0's queries."""
    words = np.empty(N_DOCS * QPV, np.uint64)
    packed = np.empty(N_DOCS * DIM * BITS // 8, np.uint8)
    for first in range(0, N_DOCS, BUILD_CHUNK):
        n = min(BUILD_CHUNK, N_DOCS - first)
        oracle_codes(orc, orc.synth_docs(SEED, n, DIM, first=first), first, words, packed)
    queries, _ = orc.synth_queries(query_seed(0), N_DOCS, NQ, DIM)
    return words, packed, queries


def reference_arm(args):
    # the reference path is a CPU path: under torchrun rank 0 alone runs it
    if int(os.environ.get("RANK", "0")) != 0:
        return
    world = int(os.environ.get("WORLD_SIZE", str(args.gpus)))
    from oracle import oracle as orc

    threads = orc.max_threads()
    t0 = time.perf_counter()
    words, packed, queries = cpu_headline_inputs(orc)
    build_s = time.perf_counter() - t0
    run = lambda qs: orc.cpu_bitmap_two_stage(words, packed, N_DOCS, DIM, N_TOP, BITS, qs, M, K, threads)
    # size each step so the whole run stays within a few minutes
    probe = min(NQ, 8 * threads)
    t0 = time.perf_counter()
    run(queries[:probe])
    probe_qps = probe / (time.perf_counter() - t0)
    per_step = cpu_sample_size(probe_qps, REFERENCE_BUDGET_S / max(args.steps + args.warmup, 1), 8, NQ)
    span = NQ - per_step + 1
    for w in range(args.warmup):
        run(queries[:per_step])
    t0 = time.perf_counter()
    done = 0
    for s in range(args.steps):
        off = (s * per_step) % span
        run(queries[off:off + per_step])
        done += per_step
    dt = time.perf_counter() - t0
    qps = done / dt
    line = {"impl": "reference", "metric": METRIC, "value": qps, "unit": "queries/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3 / max(args.steps, 1),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64-popc/f32",
            "data": "synthetic", "config": headline_config(world),
            "cpu_baseline": {"value": qps, "unit": "queries/s", "cores": threads, "kind": "port",
                             "sample": f"{per_step} of each step's {NQ} queries (rotating offsets) x {args.steps} "
                                       f"steps, all host threads", "cpu_model": cpu_model(),
                             "inputs_built_s": build_s},
            "e2e": {"value": qps, "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------- mixed batch
def mixed_run(ob, nq: int, steps: int):
    """The mixed-k / mixed-bits batch configuration: N=1,000,000 synthetic docs,
    dim 1024, RankQuant indices at bits 1, 2 and 4 over the same corpus, nq
    queries each with its own bits and k in {10, 50, 100}, one call per step
    (ovb_rankquant_search_mixed: split-BF16 tensor-core scan + exact FP64
    rescoring, plans with autotuned tiles and CUDA-graph replay).  Host
    buffers in and out; wall time per call after the first (tuning) call."""
    n, dim, seed = 1_000_000, 1024, 0x0DD5EED3
    docs = ob.synth_docs(seed, n, dim)
    queries, _ = ob.synth_queries(seed + 1, n, nq, dim)
    indices = []
    for bits in (1, 2, 4):
        rq = ob.RankQuant(dim, bits)
        rq.add(docs)
        indices.append(rq)
    del docs
    rng = np.random.default_rng(seed)
    sel = rng.integers(0, 3, nq).astype(np.uint32)
    ks = rng.choice([10, 50, 100], nq).astype(np.uint32)
    t0 = time.perf_counter()
    first = ob.search_mixed(indices, sel, ks, queries)
    first_s = time.perf_counter() - t0
    reps = max(1, min(steps, 5))
    times = []
    for _ in range(reps):
        t0 = time.perf_counter()
        res = ob.search_mixed(indices, sel, ks, queries)
        times.append(time.perf_counter() - t0)
    same = bool(np.array_equal(res.indices, first.indices))
    plans = []
    for j, rq in enumerate(indices):
        rows = np.flatnonzero(sel == j)
        if rows.size:
            info = ob.mixed_plan_info(rq, rows.size, int(ks[rows].max()))
            plans.append({"bits": (1, 2, 4)[j], "queries": int(rows.size), **info})
    sec = float(np.median(times))
    flops = 2 * 2 * nq * n * dim  # hi and lo products, multiply + add
    return {"workload": f"N={n} dim={dim} bits {{1,2,4}} k {{10,50,100}}, {nq} mixed queries per call",
            "qps": nq / sec, "s_per_call": sec, "first_call_s": first_s, "calls": reps,
            "split_bf16_tflops_effective": flops / sec / 1e12, "identical_across_calls": same, "plans": plans,
            "form": "host buffers; split-BF16 tcgen05 scan + exact FP64 rescoring; CUDA-graph replay"}


# ------------------------------------------------------ sign -> b=1, plain
def sign_plain_run(ob, torch, dev, plain_queries: int, cpu: bool):
    """The sign-bitmap configuration the reference runs on CPU: N=100,000
    synthetic docs (seed 0x0DD5EED1), dim 1024, SignBitmap top-320 (default
    policy) -> RankQuant b=1 asymmetric rerank, k=10, one query per call
    (device pointers, CUDA events per call), next to the batched form (1,000
    queries in one call) and the CPU oracle (AVX-512 + OpenMP, all threads)."""
    from oracle import oracle as orc

    n, dim, seed, nq, k = 100_000, 1024, 0x0DD5EED1, 1000, 10
    docs = ob.synth_docs(seed, n, dim)
    queries, _ = ob.synth_queries(seed + 1, n, nq, dim)
    sb, rq = ob.SignBitmap(dim), ob.RankQuant(dim, 1)
    sb.add(docs)
    rq.add(docs)
    m = orc.policy_candidate_count(k, n)  # TwoStageCandidatePolicy default: 320 at k=10
    stream = torch.cuda.current_stream(dev)
    sp = stream.cuda_stream
    d_q = torch.from_numpy(queries).to(dev)
    d_s = torch.empty(nq * k, dtype=torch.float32, device=dev)
    d_i = torch.empty(nq * k, dtype=torch.int64, device=dev)
    run = lambda cnt, qp, s_, i_: ob.two_stage_search_device(rq, sb, qp, cnt, 0, k, s_, i_, sp)  # 0: policy
    for _ in range(3):
        run(nq, d_q.data_ptr(), d_s.data_ptr(), d_i.data_ptr())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    reps = 5
    for _ in range(reps):
        run(nq, d_q.data_ptr(), d_s.data_ptr(), d_i.data_ptr())
    e1.record(stream)
    torch.cuda.synchronize(dev)
    batched_ms = e0.elapsed_time(e1) / reps
    ids = d_i.view(nq, k).cpu().numpy()
    P = min(max(plain_queries, 20), nq)
    p_s = torch.empty(P * k, dtype=torch.float32, device=dev)
    p_i = torch.empty(P * k, dtype=torch.int64, device=dev)
    for qi in range(3):
        run(1, d_q[qi].data_ptr(), p_s[qi * k:].data_ptr(), p_i[qi * k:].data_ptr())
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(P)]
    for qi in range(P):
        ev[qi][0].record(stream)
        run(1, d_q[qi].data_ptr(), p_s[qi * k:].data_ptr(), p_i[qi * k:].data_ptr())
        ev[qi][1].record(stream)
    torch.cuda.synchronize(dev)
    plain_ms = [a.elapsed_time(b) for a, b in ev]
    out = {"workload": f"N={n} dim={dim}: SignBitmap top-{m} -> RankQuant b=1 rerank top-{k}",
           "plain_qps": 1e3 / statistics.mean(plain_ms), "plain_p50_ms": float(np.percentile(plain_ms, 50)),
           "plain_p99_ms": float(np.percentile(plain_ms, 99)), "plain_queries": P,
           "plain_launches_per_query": ob.last_launch_count(),
           "batched_qps": nq / (batched_ms * 1e-3), "batched_ms": batched_ms,
           "identical_top10_plain_vs_batched": bool(np.array_equal(p_i.view(P, k).cpu().numpy(), ids[:P]))}
    if cpu:
        words = orc.sign_encode(docs, dim)
        packed = orc.rankquant_encode(docs, dim, 1)
        threads = orc.max_threads()
        sample = min(nq, 200)
        orc.cpu_sign_two_stage(words, packed, n, dim, 1, queries[:8], m, k, threads)
        t0 = time.perf_counter()
        s, i = orc.cpu_sign_two_stage(words, packed, n, dim, 1, queries[:sample], m, k, threads)
        dt = time.perf_counter() - t0
        same, tol_same, rows = topk_agreement(orc, packed, dim, 1, queries[:sample], ids[:sample], i)
        out["cpu_oracle"] = {"qps": sample / dt, "cores": threads, "sample": f"{sample} queries, one batch",
                             "kind": "port (AVX-512 popcount + b1 LUT rerank)",
                             "identical_top10_vs_cpu": same, "equal_up_to_fp64_near_ties": tol_same,
                             "rows_differing": rows}
    return out


# ------------------------------------------------------------- FastScan cfg
def fastscan_run(ob, torch, dev, args, cpu: bool):
    """The FastScan two-stage configuration: N=171,332 synthetic docs (seed
    0x0DD5EED2), dim 1024, RankQuantFastscan top-1,000 -> RankQuant b=2
    asymmetric rerank top-10, 1,000 queries per step.  Batched form
    (device-timed, L2 flushed between steps), e2e through the C ABI from pinned
    host buffers, the plain one-query form, the stage profile and rooflines,
    the serving loop on this route, and the CPU oracle (AVX-512 VPSHUFB
    FastScan + AVX-512 rerank, all host threads) on a bounded sample with the
    identity of its top-10 against the batched GPU result."""
    from ordvec_b200._lib import check, lib

    docs = ob.synth_docs(FS_SEED, FS_N, FS_DIM)
    queries, _ = ob.synth_queries(FS_SEED, FS_N, FS_NQ, FS_DIM)
    rq = ob.RankQuant(FS_DIM, 2)
    rq.add(docs)
    fs = ob.RankQuantFastscan(FS_DIM)
    fs.add(docs)
    d_q = torch.from_numpy(queries).to(dev)
    d_s = torch.empty(FS_NQ * FS_K, dtype=torch.float32, device=dev)
    d_i = torch.empty(FS_NQ * FS_K, dtype=torch.int64, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)
    sp = stream.cuda_stream

    def step(nq=FS_NQ, q_ptr=None, s_ptr=None, i_ptr=None):
        ob.two_stage_search_device(rq, fs, q_ptr or d_q.data_ptr(), nq, FS_M, FS_K, s_ptr or d_s.data_ptr(),
                                   i_ptr or d_i.data_ptr(), sp)

    for _ in range(3):
        step()
    steps = max(args.steps, 5)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    for s in range(steps):
        flush.fill_(s & 0xFF)
        ev[s][0].record(stream)
        step()
        ev[s][1].record(stream)
    torch.cuda.synchronize(dev)
    step_ms = [a.elapsed_time(b) for a, b in ev]
    batched_ids = d_i.view(FS_NQ, FS_K).cpu().numpy()
    # e2e: C ABI, pinned host buffers
    h_q = torch.from_numpy(queries).pin_memory()
    h_s = torch.empty(FS_NQ * FS_K, dtype=torch.float32).pin_memory()
    h_i = torch.empty(FS_NQ * FS_K, dtype=torch.int64).pin_memory()
    e2e_ms = []
    for s in range(3 + 50):
        flush.fill_(s & 0xFF)
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        check(lib().ovb_two_stage_search(rq.handle, fs.handle, C.c_void_p(h_q.data_ptr()), FS_NQ, FS_M, FS_K,
                                         C.c_void_p(h_s.data_ptr()), C.c_void_p(h_i.data_ptr())))
        if s >= 3:
            e2e_ms.append((time.perf_counter() - t0) * 1e3)
    # plain
    P = min(args.plain_queries, FS_NQ)
    pev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(P)]
    p_s = torch.empty(P * FS_K, dtype=torch.float32, device=dev)
    p_i = torch.empty(P * FS_K, dtype=torch.int64, device=dev)
    for qi in range(3):
        step(1, d_q[qi].data_ptr(), p_s[qi * FS_K:].data_ptr(), p_i[qi * FS_K:].data_ptr())
    for qi in range(P):
        flush.fill_(qi & 0xFF)
        pev[qi][0].record(stream)
        step(1, d_q[qi].data_ptr(), p_s[qi * FS_K:].data_ptr(), p_i[qi * FS_K:].data_ptr())
        pev[qi][1].record(stream)
    torch.cuda.synchronize(dev)
    plain_ms = [a.elapsed_time(b) for a, b in pev]
    identical = bool(np.array_equal(p_i.view(P, FS_K).cpu().numpy(), batched_ids[:P]))
    st = ob.two_stage_profile(rq, fs, d_q.data_ptr(), FS_NQ, FS_M, FS_K, d_s.data_ptr(), d_i.data_ptr(), sp)
    st1 = ob.two_stage_profile(rq, fs, d_q.data_ptr(), 1, FS_M, FS_K, d_s.data_ptr(), d_i.data_ptr(), sp)
    hbm_peak, bf16_peak, peak_kind = measured_peaks()
    pairs_pad = ((FS_DIM // 2 + 31) // 32) * 32
    code_bytes = ((FS_N + 31) // 32) * 16 * pairs_pad
    ops = 2 * FS_N * FS_NQ * pairs_pad * 16
    plain_bytes = code_bytes + pairs_pad * 16 + FS_N * 4
    batched_qps = FS_NQ / (statistics.mean(step_ms) * 1e-3)
    out = {"workload": f"fastscan_two_stage: RankQuantFastscan top-{FS_M} -> RankQuant b=2 rerank top-{FS_K}; "
                       f"N={FS_N} dim={FS_DIM}; {FS_NQ} queries per call",
           "batched_qps": batched_qps, "batched_ms": statistics.mean(step_ms),
           "e2e_qps": FS_NQ / (statistics.mean(e2e_ms) * 1e-3), "e2e_calls": len(e2e_ms),
           "e2e_top10_equal_to_device_path": bool(np.array_equal(h_i.numpy().reshape(FS_NQ, FS_K), batched_ids)),
           "plain": {"qps": 1e3 / statistics.mean(plain_ms), "p50_ms": float(np.percentile(plain_ms, 50)),
                     "p99_ms": float(np.percentile(plain_ms, 99)), "queries": P,
                     "identical_top10_vs_batched": identical},
           "stages_ms": dict(zip(STAGES, st)), "stages_ms_plain": dict(zip(STAGES, st1)),
           "roofline_batched_scan": {"bound": "tensor", "kernel": "fastscan_persist_kernel (filter epilogue)",
                                     "achieved": ops / (st[2] * 1e-3) / 1e12, "peak": 2 * bf16_peak,
                                     "unit": "TOPS (int8)", "frac": ops / (st[2] * 1e-3) / 1e12 / (2 * bf16_peak),
                                     "traffic": FS_TC_FILTER_DRAM_BYTES,
                                     "peak_source": f"2 x {peak_kind} bf16 dense TFLOP/s (burst)"},
           "roofline_plain_scan": {"bound": "hbm", "kernel": "fastscan_scan_kernel",
                                   "achieved": plain_bytes / (st1[2] * 1e-3) / 1e9, "peak": hbm_peak, "unit": "GB/s",
                                   "frac": plain_bytes / (st1[2] * 1e-3) / 1e9 / hbm_peak,
                                   "peak_source": f"{peak_kind} HBM copy"}}
    if args.serve_seconds > 0:
        out["serving"] = serving_run(ob, rq, fs, queries, batched_ids, args.serve_seconds, args.serve_rate)
    if cpu:
        from oracle import oracle as orc

        blocks = orc.fastscan_pack(docs, FS_DIM)
        packed = orc.rankquant_encode(docs, FS_DIM, 2)
        out["codes_identical_to_oracle"] = bool(np.array_equal(fs.payload(), blocks)
                                                and np.array_equal(rq.payload(), packed))
        threads = orc.max_threads()
        probe = min(FS_NQ, max(threads, 8))
        t0 = time.perf_counter()
        orc.cpu_fastscan_two_stage(blocks, packed, FS_N, FS_DIM, queries[:probe], FS_M, FS_K, threads)
        sample = cpu_sample_size(probe / (time.perf_counter() - t0), args.cpu_seconds / 2, 8, FS_NQ)
        t0 = time.perf_counter()
        s, i = orc.cpu_fastscan_two_stage(blocks, packed, FS_N, FS_DIM, queries[:sample], FS_M, FS_K, threads)
        dt = time.perf_counter() - t0
        same, tol_same, rows = topk_agreement(orc, packed, FS_DIM, 2, queries[:sample], batched_ids[:sample], i)
        out["cpu_oracle"] = {"qps": sample / dt, "cores": threads, "kind": "port",
                             "sample": f"first {sample} of the {FS_NQ} queries, all host threads",
                             "identical_top10_vs_cpu": same, "equal_up_to_fp64_near_ties": tol_same,
                             "rows_differing": rows}
        out["rerank"] = rerank_report(
            ob, orc, torch, dev, rq, fs, d_q, queries, FS_M, FS_K, packed, 128,
            lambda: ob.two_stage_profile(rq, fs, d_q.data_ptr(), FS_NQ, FS_M, FS_K, d_s.data_ptr(), d_i.data_ptr(),
                                         sp))
        out["rerank"]["fp64_rerank_ms"], out["rerank"]["fp64_final_select_ms"] = st[4], st[5]
    return out


# ----------------------------------------------------- Rank and symmetric
def rank_modes_run(ob, torch, dev, plain_queries: int):
    """The Rank (u16) index and RankQuant's symmetric search, device-timed
    through ob.search_device: Rank(768) over N=1,000,000 synthetic docs
    (1.54 GB of ranks) and a RankQuant b=2 dim-1024 index over N=171,332, one
    query per call (plain) and a batch per call.  For the plain calls the whole
    call's time is set against the bytes the scan must read (ranks or codes
    once, plus the 4-byte key row), a lower bound on the scan kernel's HBM
    rate."""
    hbm_peak, _, peak_kind = measured_peaks()
    stream = torch.cuda.current_stream(dev)
    sp = stream.cuda_stream
    out = {}

    def timed(ix, d_q, nq, k, asym, reps):
        d_s = torch.empty(nq * k, dtype=torch.float32, device=dev)
        d_i = torch.empty(nq * k, dtype=torch.int64, device=dev)
        run = lambda qp: ob.search_device(ix, qp, nq, k, d_s.data_ptr(), d_i.data_ptr(), sp, asymmetric=asym)
        for r in range(3):
            run(d_q[r * nq].data_ptr() if nq == 1 else d_q.data_ptr())
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(reps)]
        for r in range(reps):
            ev[r][0].record(stream)
            run(d_q[r * nq].data_ptr() if nq == 1 else d_q.data_ptr())
            ev[r][1].record(stream)
        torch.cuda.synchronize(dev)
        return [a.elapsed_time(b) for a, b in ev]

    def roof(nbytes, ms):
        gbs = nbytes / (ms * 1e-3) / 1e9
        return {"bound": "hbm", "achieved": gbs, "peak": hbm_peak, "unit": "GB/s", "frac": gbs / hbm_peak,
                "peak_source": f"{peak_kind} HBM copy"}

    n, dim, k, nb = 1_000_000, 768, 100, 64
    rk = ob.Rank(dim)
    for first in range(0, n, 250_000):
        rk.add(ob.synth_docs(0x0DD5EED6, 250_000, dim, first=first))
    q, _ = ob.synth_queries(0x0DD5EED7, n, nb, dim)
    d_q = torch.from_numpy(q).to(dev)
    P = max(4, min(plain_queries, 32))
    for asym in (False, True):
        plain = timed(rk, d_q, 1, k, asym, P)
        batch = timed(rk, d_q, nb, k, asym, 3)
        out["rank_asymmetric" if asym else "rank_symmetric"] = {
            "workload": f"Rank dim={dim} N={n} top-{k}", "plain_qps": 1e3 / statistics.mean(plain),
            "plain_p50_ms": float(np.percentile(plain, 50)), "batched_qps": nb / (statistics.median(batch) * 1e-3),
            "batch_queries": nb, "roofline_plain_call": roof(n * dim * 2 + 4 * n, statistics.median(plain))}
    del rk
    rq = ob.RankQuant(FS_DIM, 2)
    rq.add(ob.synth_docs(FS_SEED, FS_N, FS_DIM))
    queries, _ = ob.synth_queries(FS_SEED, FS_N, 1000, FS_DIM)
    nr = len(rq)
    d_q = torch.from_numpy(queries).to(dev)
    plain = timed(rq, d_q, 1, 10, False, P)
    batch = timed(rq, d_q, 1000, 10, False, 3)
    out["rankquant_symmetric"] = {
        "workload": f"RankQuant b={rq.bits} dim={rq.dim} N={nr} symmetric top-10",
        "plain_qps": 1e3 / statistics.mean(plain), "plain_p50_ms": float(np.percentile(plain, 50)),
        "batched_qps": 1000 / (statistics.median(batch) * 1e-3), "batch_queries": 1000,
        "roofline_plain_call": roof(nr * rq.dim * rq.bits // 8 + 4 * nr, statistics.median(plain))}
    return out


# ------------------------------------------------------------------ serving
def serving_run(ob, rq, fs, queries, batched_ids, seconds: float, rate_qps: float):
    """The serving loop on the FastScan route: seeded Poisson request arrivals
    offering `rate_qps` queries/s, 1-256 queries per request, k=10, m=1000;
    answered by ob.Server (continuous batching, 3 worker streams).  Reports
    completed QPS, request latency p50/p99 and whether every answer equals the
    batched form's top-10."""
    import threading

    rng = np.random.default_rng(FS_SEED)
    mean_size = 128.5
    n_req = max(int(seconds * rate_qps / mean_size), 8)
    sizes = rng.integers(1, 257, n_req)
    offs = rng.integers(0, FS_NQ - 256, n_req)
    gaps = rng.exponential(mean_size / rate_qps, n_req)
    srv = ob.Server(workers=3, max_batch=1024)
    route = srv.add_route(rq, fs)
    srv.wait_ready()  # workers have sized their buffers for the route
    tickets, done_at, lat = [None] * n_req, [0.0] * n_req, [0.0] * n_req
    same = [True]

    def collect():
        for j in range(n_req):
            while tickets[j] is None:
                time.sleep(20e-6)
            res, lat[j] = tickets[j].wait()
            done_at[j] = time.perf_counter()
            o, sz = int(offs[j]), int(sizes[j])
            if not np.array_equal(res.indices.reshape(sz, FS_K), batched_ids[o:o + sz]):
                same[0] = False

    th = threading.Thread(target=collect)
    th.start()
    t0 = time.perf_counter()
    due = t0
    for j in range(n_req):
        due += gaps[j]
        while time.perf_counter() < due:
            pass
        o, sz = int(offs[j]), int(sizes[j])
        tickets[j] = srv.submit(route, queries[o:o + sz], FS_K, FS_M)
    th.join()
    wall = max(done_at) - t0
    st = srv.stats()
    srv.close()
    n_q = int(sizes.sum())
    return {"offered_qps": rate_qps, "completed_qps": n_q / wall, "requests": n_req, "queries": n_q,
            "request_queries": "uniform 1-256", "k": FS_K, "candidates": FS_M,
            "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "mean_ms": float(np.mean(lat)), "batches": st["batches"],
            "max_concurrent_batches": st["max_concurrent_batches"], "workers": 3,
            "arrivals": "seeded Poisson", "latency": "submit -> results ready, per request",
            "identical_top10_vs_batched": same[0]}


# ------------------------------------------------------- profiling cases
def profile_case(case: str):
    """Small single-kernel workloads for ncu captures (no timing, no JSON):
      bitmap    Bitmap(768, 192) top-2000 of 1024 queries, N=2M (bitmap_pair_kernel)
      bitmap10m the same at N=10M (the headline's stage-1 index only, 0.96 GB)
      popc      the 2M index, one query per call (popc_rows_kernel, wide select)
      rank      RankQuant(1024, 2) exact top-100 of 1024 queries, N=1M (rank_tc_kernel)
      fastscan  the FastScan configuration's top-1000 of 1000 queries (fastscan_tc_kernel)
      plain     the FastScan two-stage search, one query per call, 12 calls
                (fastscan_scan_kernel, select_rows_cluster_kernel, rerank)
      rankfull  Rank(768) N=1M top-100: symmetric then asymmetric, 1 query and 64
                queries per call (rank_tile_kernel)
      multibucket MultiBucketBitmap(768, 2) N=2M: diagonal-weight top-2000 of 1
                query per call (multibucket_rows_kernel), 3 calls
      encode    RankQuant(768, 2).add of 1M docs, twice (rank_encode_kernel)
      rerank    Bitmap(768, 192) top-2000 -> RankQuant b=2 top-100 of 1024 queries,
                N=2M, twice (rerank_tc_kernel, asym_table_kernel rescoring)
    Each search runs more than once so captures can skip the first call."""
    import ordvec_b200 as ob

    if case in ("bitmap", "popc", "bitmap10m"):
        n = 10_000_000 if case == "bitmap10m" else 2_000_000
        bm = ob.Bitmap(768, 192)
        for first in range(0, n, 1_000_000):
            bm.add(ob.synth_docs(0x0DD5EED4, 1_000_000, 768, first=first))
        q, _ = ob.synth_queries(0x0DD5EED5, n, 1024, 768)
        for _ in range(3 if case == "popc" else 2):
            bm.top_m_candidates(q[0], 2000) if case == "popc" else bm.top_m_candidates_batched(q, 2000)
    elif case == "multibucket":
        n = 2_000_000
        mb = ob.MultiBucketBitmap(768, 2)
        for first in range(0, n, 1_000_000):
            mb.add(ob.synth_docs(0x0DD5EED4, 1_000_000, 768, first=first))
        q, _ = ob.synth_queries(0x0DD5EED5, n, 4, 768)
        for i in range(3):
            mb.top_m_bilinear_batched(q[i:i + 1], mb.diagonal_weights(), 2000)
    elif case == "rerank":
        n = 2_000_000
        rq, bm = ob.RankQuant(768, 2), ob.Bitmap(768, 192)
        for first in range(0, n, 1_000_000):
            d = ob.synth_docs(0x0DD5EED4, 1_000_000, 768, first=first)
            rq.add(d)
            bm.add(d)
        q, _ = ob.synth_queries(0x0DD5EED5, n, 1024, 768)
        for _ in range(2):
            ob.two_stage_search(rq, bm, q, 2000, 100)
    elif case == "encode":
        rq = ob.RankQuant(768, 2)
        d = ob.synth_docs(0x0DD5EED4, 1_000_000, 768)
        for _ in range(2):
            rq.add(d)
    elif case == "rank":
        n = 1_000_000
        rq = ob.RankQuant(1024, 2)
        rq.add(ob.synth_docs(0x0DD5EED3, n, 1024))
        q, _ = ob.synth_queries(0x0DD5EED4, n, 1024, 1024)
        for _ in range(2):
            rq.search_asymmetric(q, 100)
    elif case == "fastscan":
        fs = ob.RankQuantFastscan(FS_DIM)
        fs.add(ob.synth_docs(FS_SEED, FS_N, FS_DIM))
        q, _ = ob.synth_queries(FS_SEED + 1, FS_N, FS_NQ, FS_DIM)
        for _ in range(2):
            fs.search(q, FS_M)
    elif case == "plain":
        rq, fs = ob.RankQuant(FS_DIM, 2), ob.RankQuantFastscan(FS_DIM)
        docs = ob.synth_docs(FS_SEED, FS_N, FS_DIM)
        rq.add(docs)
        fs.add(docs)
        q, _ = ob.synth_queries(FS_SEED + 1, FS_N, 12, FS_DIM)
        for i in range(12):
            ob.two_stage_search(rq, fs, q[i:i + 1], FS_M, FS_K)
    elif case == "rankfull":
        n = 1_000_000
        rk = ob.Rank(768)
        for first in range(0, n, 250_000):
            rk.add(ob.synth_docs(0x0DD5EED6, 250_000, 768, first=first))
        q, _ = ob.synth_queries(0x0DD5EED7, n, 64, 768)
        for fn in (rk.search, rk.search_asymmetric):
            for _ in range(2):
                fn(q[:1], 100)
                fn(q, 100)
    else:
        raise SystemExit(f"unknown profile case {case}")
    print(f"profile case {case}: done", flush=True)


# ------------------------------------------------------ serving, 3 indices
def serving_multi_run(ob, seconds: float, rates):
    """The serving configuration: three device-resident indices -- (dim 384,
    N=2M, b=1), (768, 5M, b=2), (1024, 1M, b=4) -- each behind a sign-bitmap
    stage 1 (two-stage route, default candidate policy), seeded Poisson request
    streams offering each rate in `rates` queries/s with 1-256 queries per
    request, k in {10, 50, 100} and a uniformly drawn index; ob.Server with 3
    workers (continuous batching, HBM-budget admission).  Per rate: completed
    QPS and request latency p50/p99.  Beside it the plain per-request form (one
    request at a time through ob.two_stage_search) and whether sampled
    requests' answers in the mix equal their answers alone."""
    import threading

    specs = [(384, 2_000_000, 1), (768, 5_000_000, 2), (1024, 1_000_000, 4)]
    seed = 0x0DD5EED5
    t0 = time.perf_counter()
    routes, pools = [], []
    srv = ob.Server(workers=3, max_batch=1024)
    keep = []
    for j, (dim, n, bits) in enumerate(specs):
        rq, sb = ob.RankQuant(dim, bits), ob.SignBitmap(dim)
        for first in range(0, n, 1_000_000):
            d = ob.synth_docs(seed + j, min(1_000_000, n - first), dim, first=first)
            rq.add(d)
            sb.add(d)
        q, _ = ob.synth_queries(seed + 16 + j, n, 2048, dim)
        pools.append(q)
        routes.append(srv.add_route(rq, sb))
        keep.append((rq, sb))
    build_s = time.perf_counter() - t0
    srv.wait_ready()
    rng = np.random.default_rng(seed)
    out = {"workload": "3 indices: (384, 2M, b1), (768, 5M, b2), (1024, 1M, b4), each SignBitmap -> RankQuant; "
                       "requests of 1-256 queries, k in {10,50,100}, seeded Poisson arrivals",
           "build_s": build_s, "workers": 3, "rates": []}
    sample_ans = {}
    for rate in rates:
        mean_size = 128.5
        n_req = max(int(seconds * rate / mean_size), 16)
        sizes = rng.integers(1, 257, n_req)
        which = rng.integers(0, 3, n_req)
        ks = rng.choice([10, 50, 100], n_req)
        offs = rng.integers(0, 2048 - 256, n_req)
        gaps = rng.exponential(mean_size / rate, n_req)
        tickets, lat, done_at = [None] * n_req, [0.0] * n_req, [0.0] * n_req

        def collect():
            for i in range(n_req):
                while tickets[i] is None:
                    time.sleep(20e-6)
                res, lat[i] = tickets[i].wait()
                done_at[i] = time.perf_counter()
                if i % 97 == 0:
                    sample_ans[(rate, i)] = (int(which[i]), int(offs[i]), int(sizes[i]), int(ks[i]), res.indices.copy())

        th = threading.Thread(target=collect)
        th.start()
        start = time.perf_counter()
        due = start
        for i in range(n_req):
            due += gaps[i]
            while time.perf_counter() < due:
                pass
            j, o, sz = int(which[i]), int(offs[i]), int(sizes[i])
            tickets[i] = srv.submit(routes[j], pools[j][o:o + sz], int(ks[i]), 0)
        th.join()
        wall = max(done_at) - start
        nq = int(sizes.sum())
        out["rates"].append({"offered_qps": rate, "completed_qps": nq / wall, "requests": n_req, "queries": nq,
                             "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                             "mean_ms": float(np.mean(lat))})
    st = srv.stats()
    out["batches"], out["max_concurrent_batches"] = st["batches"], st["max_concurrent_batches"]
    srv.close()
    # plain per-request form: one request at a time, host buffers; this thread's
    # buffers are first sized by one untimed largest request per index (the
    # server's workers do the same before serving)
    for j in range(3):
        for sz in (7, 31, 256):
            ob.two_stage_search(keep[j][0], keep[j][1], pools[j][:sz], 0, 100)
    rng2 = np.random.default_rng(seed + 1)
    plain_lat, plain_q = [], 0
    for i in range(120):
        j, sz, k = int(rng2.integers(0, 3)), int(rng2.integers(1, 257)), int(rng2.choice([10, 50, 100]))
        o = int(rng2.integers(0, 2048 - 256))
        rq, sb = keep[j]
        t1 = time.perf_counter()
        ob.two_stage_search(rq, sb, pools[j][o:o + sz], 0, k)
        plain_lat.append((time.perf_counter() - t1) * 1e3)
        plain_q += sz
    out["plain_per_request"] = {"qps": plain_q / (sum(plain_lat) * 1e-3), "p50_ms": float(np.percentile(plain_lat, 50)),
                                "p99_ms": float(np.percentile(plain_lat, 99)), "requests": 120,
                                "form": "one request at a time, ob.two_stage_search, host buffers"}
    same = True
    for (rate, i), (j, o, sz, k, ids) in list(sample_ans.items())[:24]:
        rq, sb = keep[j]
        alone = ob.two_stage_search(rq, sb, pools[j][o:o + sz], 0, k)
        same &= bool(np.array_equal(alone.indices, ids))
    out["identical_in_mix_vs_alone"] = same
    out["checked_requests"] = min(len(sample_ans), 24)
    return out


# ------------------------------------------------------------ headline build
def build_headline(ob, orc, with_multibucket: bool):
    """The headline indices built on the device in 1M-doc chunks; with an oracle
    module, the same chunks are also encoded on the host by the oracle (bitmap
    words and RankQuant b=2 codes, for the CPU leg and the code identity check)."""
    rq, bm = ob.RankQuant(DIM, BITS), ob.Bitmap(DIM, N_TOP)
    mb = ob.MultiBucketBitmap(DIM, BITS) if with_multibucket else None
    words = np.empty(N_DOCS * QPV, np.uint64) if orc else None
    packed = np.empty(N_DOCS * DIM * BITS // 8, np.uint8) if orc else None
    for first in range(0, N_DOCS, BUILD_CHUNK):
        d = ob.synth_docs(SEED, min(BUILD_CHUNK, N_DOCS - first), DIM, first=first)
        for ix in (rq, bm, mb):
            if ix is not None:
                ix.add(d)
        if orc:
            oracle_codes(orc, d, first, words, packed)
    return rq, bm, mb, words, packed


def second_stage1_run(ob, torch, dev, rq, s1, name, words_per_doc, d_q, queries, plain_queries):
    """Batched vs plain for one more stage-1 kind on the headline corpus."""
    hbm_peak, bf16_peak, peak_kind = measured_peaks()
    stream = torch.cuda.current_stream(dev)
    sp = stream.cuda_stream
    nq = d_q.shape[0]
    d_s = torch.empty(nq * K, dtype=torch.float32, device=dev)
    d_i = torch.empty(nq * K, dtype=torch.int64, device=dev)
    run = lambda cnt, qp, s_, i_: ob.two_stage_search_device(rq, s1, qp, cnt, M, K, s_, i_, sp)
    for _ in range(2):
        run(nq, d_q.data_ptr(), d_s.data_ptr(), d_i.data_ptr())
    reps = 3
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(reps)]
    for r in range(reps):
        ev[r][0].record(stream)
        run(nq, d_q.data_ptr(), d_s.data_ptr(), d_i.data_ptr())
        ev[r][1].record(stream)
    torch.cuda.synchronize(dev)
    batch_ms = statistics.median(a.elapsed_time(b) for a, b in ev)
    ids = d_i.view(nq, K).cpu().numpy()
    P = max(4, min(plain_queries, 16))
    p_s = torch.empty(P * K, dtype=torch.float32, device=dev)
    p_i = torch.empty(P * K, dtype=torch.int64, device=dev)
    run(1, d_q[0].data_ptr(), p_s.data_ptr(), p_i.data_ptr())
    pev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(P)]
    for qi in range(P):
        pev[qi][0].record(stream)
        run(1, d_q[qi].data_ptr(), p_s[qi * K:].data_ptr(), p_i[qi * K:].data_ptr())
        pev[qi][1].record(stream)
    torch.cuda.synchronize(dev)
    plain_ms = [a.elapsed_time(b) for a, b in pev]
    st = ob.two_stage_profile(rq, s1, d_q.data_ptr(), nq, M, K, d_s.data_ptr(), d_i.data_ptr(), sp)
    st1 = ob.two_stage_profile(rq, s1, d_q.data_ptr(), 1, M, K, p_s.data_ptr(), p_i.data_ptr(), sp)
    ops = 2 * N_DOCS * nq * words_per_doc * 64
    plain_gbs = N_DOCS * words_per_doc * 8 / (st1[2] * 1e-3) / 1e9
    return {"workload": f"{name} top-{M} -> RankQuant b={BITS} rerank top-{K}; N={N_DOCS} dim={DIM}; "
                        f"{nq} queries per batch",
            "batched_qps": nq / (batch_ms * 1e-3), "batch_ms": batch_ms,
            "plain_qps": 1e3 / statistics.mean(plain_ms), "plain_p50_ms": float(np.percentile(plain_ms, 50)),
            "plain_p99_ms": float(np.percentile(plain_ms, 99)), "plain_queries": P,
            "batched_over_plain": nq / (batch_ms * 1e-3) * statistics.mean(plain_ms) * 1e-3,
            "identical_top100_batched_vs_plain": bool(np.array_equal(p_i.view(P, K).cpu().numpy(), ids[:P])),
            "stages_ms": dict(zip(STAGES, st)), "stages_ms_plain": dict(zip(STAGES, st1)),
            "roofline_batched_scan": {"bound": "tensor", "kernel": "bitmap_pair_kernel (filter epilogue)",
                                      "achieved": ops / (st[2] * 1e-3) / 1e12, "peak": 2 * bf16_peak,
                                      "unit": "TOPS (int8)", "frac": ops / (st[2] * 1e-3) / 1e12 / (2 * bf16_peak),
                                      "peak_source": f"2 x {peak_kind} bf16 dense TFLOP/s (burst)"},
            "roofline_plain_scan": {"bound": "hbm", "kernel": "multibucket_rows_kernel",
                                    "achieved": plain_gbs, "peak": hbm_peak, "unit": "GB/s",
                                    "frac": plain_gbs / hbm_peak, "peak_source": f"{peak_kind} HBM copy"}}


# ------------------------------------------------------------------ GPU arm
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--plain-queries", type=int, default=100)
    ap.add_argument("--cpu-seconds", type=float, default=20.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--serve-seconds", type=float, default=2.0)
    ap.add_argument("--serve-rate", type=float, default=200_000.0, help="offered queries/s")
    ap.add_argument("--mixed-queries", type=int, default=-1,
                    help="also run the mixed-k/bits batch (N=1M, dim 1024) with this many queries; "
                         "0 = skip, -1 = 4096 on a single GPU")
    ap.add_argument("--extras", default="auto", choices=["auto", "on", "off"],
                    help="the extra configurations (auto: on a single GPU only)")
    ap.add_argument("--profile-case",
                    choices=["bitmap", "bitmap10m", "popc", "rank", "fastscan", "plain", "rankfull", "multibucket",
                             "encode", "rerank"],
                    help="run one small kernel workload for an ncu capture and exit")
    args = ap.parse_args()
    if args.profile_case:
        return profile_case(args.profile_case)
    if args.impl == "reference":
        return reference_arm(args)

    import torch

    import ordvec_b200 as ob
    from ordvec_b200._lib import check, lib

    from ordvec_b200.replicas import ReplicaGroup, rank_env, whole_job_rate

    rank, world, local = rank_env()
    extras = (world == 1) if args.extras == "auto" else args.extras == "on"
    mixed_q = args.mixed_queries if args.mixed_queries >= 0 else (4096 if extras else 0)
    cpu = rank == 0 and not args.no_cpu
    torch.cuda.set_device(local)
    ob.set_device(local)
    dev = torch.device("cuda", local)
    group = ReplicaGroup("nccl", device=dev, sync=lambda: torch.cuda.synchronize(dev))
    orc = None
    if cpu:
        from oracle import oracle as orc

    t0 = time.perf_counter()
    rq, bm, mb, h_words, h_packed = build_headline(ob, orc, extras)
    build_s = time.perf_counter() - t0
    queries, _ = ob.synth_queries(query_seed(rank), N_DOCS, NQ, DIM)

    d_q = torch.from_numpy(queries).to(dev)
    d_s = torch.empty(NQ * K, dtype=torch.float32, device=dev)
    d_i = torch.empty(NQ * K, dtype=torch.int64, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)
    sp = stream.cuda_stream

    def step_device(nq=NQ, q_ptr=None, s_ptr=None, i_ptr=None):
        ob.two_stage_search_device(rq, bm, q_ptr or d_q.data_ptr(), nq, M, K, s_ptr or d_s.data_ptr(),
                                   i_ptr or d_i.data_ptr(), sp)

    barrier = group.barrier
    max_over_ranks = group.max_over_ranks

    for _ in range(args.warmup):
        step_device()
    barrier()

    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    # ---- value: device-timed batched steps; every step records its stage
    # events (ovb_two_stage_profile: the same pipeline plus CUDA events between
    # the stages on the launching stream), so the dominant kernel's launch time
    # is measured inside the timed region
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    stage_rows = []
    barrier()
    for s in range(args.steps):
        flush.fill_(s & 0xFF)
        ev[s][0].record(stream)
        stage_rows.append(ob.two_stage_profile(rq, bm, d_q.data_ptr(), NQ, M, K, d_s.data_ptr(), d_i.data_ptr(), sp))
        ev[s][1].record(stream)
    barrier()
    launches_per_step = ob.last_launch_count()
    step_ms = [a.elapsed_time(b) for a, b in ev]
    total_ms = max_over_ranks(sum(step_ms))
    batched_ids = d_i.view(NQ, K).cpu().numpy()
    batched_scores = d_s.view(NQ, K).cpu().numpy()
    stages = [statistics.mean(r[j] for r in stage_rows) for j in range(6)]

    # ---- e2e: public C ABI, pinned host buffers, H2D + D2H inside the timed region
    h_q = torch.from_numpy(queries).pin_memory()
    h_s = torch.empty(NQ * K, dtype=torch.float32).pin_memory()
    h_i = torch.empty(NQ * K, dtype=torch.int64).pin_memory()
    e2e_ms = []
    e2e_steps = max(args.steps, 30)
    for s in range(args.warmup + e2e_steps):
        flush.fill_(s & 0xFF)
        barrier()
        t0 = time.perf_counter()
        check(lib().ovb_two_stage_search(rq.handle, bm.handle, C.c_void_p(h_q.data_ptr()), NQ, M, K,
                                         C.c_void_p(h_s.data_ptr()), C.c_void_p(h_i.data_ptr())))
        dt = (time.perf_counter() - t0) * 1e3
        if s >= args.warmup:
            e2e_ms.append(dt)
    e2e_total = max_over_ranks(sum(e2e_ms))
    e2e_same = bool(np.array_equal(h_i.numpy().reshape(NQ, K), batched_ids))

    # ---- plain: one query per call
    P = min(args.plain_queries, NQ)
    pev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(P)]
    p_s = torch.empty(P * K, dtype=torch.float32, device=dev)
    p_i = torch.empty(P * K, dtype=torch.int64, device=dev)
    for qi in range(3):
        step_device(1, d_q[qi].data_ptr(), p_s[qi * K:].data_ptr(), p_i[qi * K:].data_ptr())
    barrier()
    for qi in range(P):
        flush.fill_(qi & 0xFF)
        pev[qi][0].record(stream)
        step_device(1, d_q[qi].data_ptr(), p_s[qi * K:].data_ptr(), p_i[qi * K:].data_ptr())
        pev[qi][1].record(stream)
    barrier()
    plain_ms = [a.elapsed_time(b) for a, b in pev]
    plain_launches = ob.last_launch_count()
    identical = bool(np.array_equal(p_i.view(P, K).cpu().numpy(), batched_ids[:P]))
    stages1 = ob.two_stage_profile(rq, bm, d_q.data_ptr(), 1, M, K, p_s.data_ptr(), p_i.data_ptr(), sp)
    multibucket = second_stage1_run(ob, torch, dev, rq, mb, "MultiBucketBitmap b=2 (diagonal weights)", 4 * QPV,
                                    d_q, queries, args.plain_queries) if mb is not None else None
    clock_info = clocks.stop()

    hbm_peak, bf16_peak, peak_kind = measured_peaks()
    code_bytes = N_DOCS * QPV * 8

    fp4 = os.environ.get("OVB_BITMAP_FP4", "1") != "0"

    def roof_batched(ms):
        """The filter scan: the overlap popcount(q AND d) of every (doc, query)
        pair as an exact tensor-core GEMM on 0/1 operands.  Default form
        bitmap_fp4_pair_kernel (kind::mxf4: bits as e2m1 1.0 / 0 with unit
        block scales, f32 sums; peak = 4 x the measured dense bf16 rate, the
        ratio of the nominal dense FP4 and bf16 rates); with OVB_BITMAP_FP4=0
        bitmap_pair_kernel (kind::i8 on 0/1 bytes; peak = 2 x measured bf16).
        Algorithmic ops = 2 * docs * queries * 768 either way."""
        ops = 2 * N_DOCS * NQ * QPV * 64
        achieved = ops / (ms * 1e-3) / 1e12
        peak = (4 if fp4 else 2) * bf16_peak
        return {"bound": "tensor", "achieved": achieved, "peak": peak,
                "unit": "TOPS (0/1 operands; FP4 e2m1 MMAs)" if fp4 else "TOPS (int8)",
                "frac": achieved / peak, "frac_of_int8_peak": achieved / (2 * bf16_peak),
                "traffic": PAIR_FILTER_DRAM_BYTES,
                "traffic_unit": "DRAM bytes per launch (ncu dram__bytes_read.sum + dram__bytes_write.sum)",
                "algorithmic_hbm_bytes_per_launch": code_bytes + NQ * QPV * 64,
                "codes_gbs": code_bytes / (ms * 1e-3) / 1e9,
                "kernel": ("bitmap_fp4_pair_kernel" if fp4 else "bitmap_pair_kernel") + " (filter epilogue)",
                "queries_per_launch": NQ,
                "algorithmic_ops_per_launch": ops, "launch_ms": ms, "launches_timed": len(stage_rows),
                "timing": "mean of the scan-stage CUDA events of every timed step (launching stream)",
                "peak_source": f"{4 if fp4 else 2} x {peak_kind} bf16 dense TFLOP/s (burst)"}

    def roof_plain(ms):
        """One query: popc_rows_kernel (CUDA cores), bound by HBM: the codes
        once plus the 4-byte key row."""
        b = code_bytes + N_DOCS * 4
        achieved = b / (ms * 1e-3) / 1e9
        return {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s", "frac": achieved / hbm_peak,
                "kernel": "popc_rows_kernel", "queries_per_launch": 1, "algorithmic_bytes_per_launch": b,
                "launch_ms": ms, "peak_source": f"{peak_kind} HBM copy bandwidth"}

    value = whole_job_rate(NQ * args.steps, world, total_ms)
    e2e = whole_job_rate(NQ * e2e_steps, world, e2e_total)
    plain_qps = 1e3 / statistics.mean(plain_ms)
    line = {
        "metric": METRIC, "value": value, "unit": "queries/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": ("e2m1-bits/f32-acc" if fp4 else "u8-bits/s32-acc") + " + f64 rerank", "data": "synthetic",
        "config": headline_config(world),
        "e2e": {"value": e2e, "unit": "queries/s", "h2d_bytes_per_step": NQ * DIM * 4,
                "d2h_bytes_per_step": NQ * K * (4 + 8), "ms_per_step": e2e_total / e2e_steps, "steps": e2e_steps,
                "call": "ovb_two_stage_search (C ABI, pinned host buffers)",
                "top100_equal_to_device_path": e2e_same},
        "gpu_launches": launches_per_step * args.steps,
        "plain": {"qps": plain_qps, "p50_ms": float(np.percentile(plain_ms, 50)),
                  "p99_ms": float(np.percentile(plain_ms, 99)), "queries": P, "launches_per_query": plain_launches,
                  "identical_top100_vs_batched": identical, "batched_over_plain": value / world / plain_qps},
        "stages_ms": dict(zip(STAGES, stages)),
        "stages_ms_plain": dict(zip(STAGES, stages1)),
        "roofline": roof_batched(stages[2]),
        "roofline_plain": roof_plain(stages1[2]),
        "multibucket": multibucket,
        "build_s": build_s,
        "clocks": clock_info,
    }
    line["rerank"] = rerank_report(
        ob, orc, torch, dev, rq, bm, d_q, queries, M, K, h_packed, 128,
        lambda: ob.two_stage_profile(rq, bm, d_q.data_ptr(), NQ, M, K, d_s.data_ptr(), d_i.data_ptr(), sp))
    line["rerank"]["fp64_rerank_ms"], line["rerank"]["fp64_final_select_ms"] = stages[4], stages[5]
    if cpu:
        line["codes_identical_to_oracle"] = bool(np.array_equal(bm.payload().view(np.uint64), h_words)
                                                 and np.array_equal(rq.payload(), h_packed))
        threads = orc.max_threads()
        run = lambda qs: orc.cpu_bitmap_two_stage(h_words, h_packed, N_DOCS, DIM, N_TOP, BITS, qs, M, K, threads)
        probe = min(NQ, 8 * threads)
        t0 = time.perf_counter()
        run(queries[:probe])
        probe_qps = probe / (time.perf_counter() - t0)
        sample = cpu_sample_size(probe_qps, args.cpu_seconds, 8, NQ)
        t0 = time.perf_counter()
        cs, ci = run(queries[:sample])
        dt = time.perf_counter() - t0
        same, tol_same, rows = topk_agreement(orc, h_packed, DIM, BITS, queries[:sample], batched_ids[:sample], ci)
        line["cpu_baseline"] = {"value": sample / dt, "unit": "queries/s", "cores": threads, "kind": "port",
                                "sample": f"first {sample} of the step's {NQ} queries, all host threads",
                                "cpu_model": cpu_model(), "identical_top100_vs_cpu": same,
                                "equal_up_to_fp64_near_ties": tol_same, "rows_differing": rows}
        line["identical_top100_vs_cpu"] = same
    if extras:
        del mb, multibucket

        def extra(name, fn):
            """One optional side workload: an error in it is recorded in the line
            (the headline above stands on its own)."""
            try:
                line[name] = fn()
            except Exception as exc:  # noqa: BLE001 -- reported, not hidden
                line[name] = {"error": f"{type(exc).__name__}: {exc}"}

        extra("fastscan_two_stage", lambda: fastscan_run(ob, torch, dev, args, cpu))
        extra("mixed_batch", lambda: mixed_run(ob, mixed_q, args.steps) if mixed_q > 0 else None)
        extra("sign_b1_plain", lambda: sign_plain_run(ob, torch, dev, args.plain_queries, cpu))
        extra("serving_multi", lambda: serving_multi_run(ob, args.serve_seconds, [20_000.0, 100_000.0, args.serve_rate])
              if args.serve_seconds > 0 else None)
        extra("rank_modes", lambda: rank_modes_run(ob, torch, dev, args.plain_queries))
    group.close()
    if rank == 0:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
