"""Benchmark of the HNSW query path: batched persistent CUDA search on one B200 per rank.

Workload (default): 1M x 128 SIFT-like float32 base (seeded synthetic stand-in for SIFT1M),
10K queries, space l2, M=16, efConstruction=200, k=10, efSearch swept over
{16, 32, 64, 128, 256, 512}; the headline efSearch is the smallest one whose recall@10 reaches
0.95 against exact float64 neighbours. One step = one batch of 10K queries through the engine.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0). ``value`` is device-timed throughput with queries resident in HBM;
``e2e`` is the same metric through the public Python API with host arrays (H2D of the queries and
D2H of ids/distances/counts inside the timed region). ``--impl reference`` times the reference's
own CPU knnQueryBatch (built from its sources into oracle/_ref) on the same index and queries.
Multi-GPU runs are replicas (the query path has no exchange step): each rank searches its own
batch against its own copy of the index and ``value`` sums the queries of all ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = "c2_sift1m_d128_l2"
EF_SWEEP = (16, 32, 64, 128, 256, 512)
K = 10
EFC = 200
RECALL_TARGET = 0.95
# smallest swept efSearch whose recall@10 reaches RECALL_TARGET on this workload (measured by
# the sweep, which is reported with every run); both arms time this setting
HEADLINE_EF = 64
CACHE_DIR = os.path.join(tempfile.gettempdir(), "nmslib_b200_bench")
METRIC = "HNSW QPS at recall@10>=0.95 (1M x 128 SIFT-like l2, batched persistent kernel)"


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# ------------------------------------------------------------------ distributed plumbing
def dist_init(n_gpus):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    return rank, world, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ------------------------------------------------------------------ data and index
def workload_data():
    from nmslib_b200.datasets import workload
    base, queries, space, m = workload(WORKLOAD)
    return base, queries, space, m


def index_path(m):
    return os.path.join(CACHE_DIR, f"{WORKLOAD}_M{m}_efc{EFC}_seed0.hnsw")


def ensure_index(base, space, m, rank, world):
    """Rank 0 builds the index with the engine's host builder (all host cores) unless a copy is
    cached on this machine; the other ranks wait and load the same file."""
    from nmslib_b200 import SPACES, _capi
    path = index_path(m)
    if rank == 0 and not os.path.exists(path):
        os.makedirs(CACHE_DIR, exist_ok=True)
        t0 = time.time()
        _capi.build_index(base, SPACES[space], m, EFC, nthreads=0, seed=0, out_path=path + ".tmp")
        os.replace(path + ".tmp", path)
        log(f"[bench] built {path} in {time.time() - t0:.1f}s")
    barrier(world)
    return path


def ground_truth(base, queries, k):
    """Exact float64 neighbours on the GPU (measurement only): ids [nq, k] and the k-th distance."""
    import torch
    b = torch.from_numpy(base).cuda().double()
    bsq = (b * b).sum(1)
    kth = np.empty(len(queries))
    ids = np.empty((len(queries), k), np.int64)
    for s in range(0, len(queries), 512):
        q = torch.from_numpy(queries[s:s + 512]).cuda().double()
        d = (q * q).sum(1, keepdim=True) - 2 * q @ b.T + bsq[None, :]
        v, i = torch.topk(d, k, dim=1, largest=False)
        ids[s:s + 512] = i.cpu().numpy()
        kth[s:s + 512] = v[:, -1].cpu().numpy()
    del b
    torch.cuda.empty_cache()
    return ids, kth


def recall_at_k(found_d, counts, kth, k):
    """ann-benchmarks recall: a returned neighbour counts when its distance is within the true
    k-th distance (so equal-distance alternatives are not penalised)."""
    valid = np.arange(found_d.shape[1])[None, :k] < np.minimum(counts, k)[:, None]
    ok = found_d[:, :k] <= (kth * (1 + 1e-6) + 1e-6)[:, None]
    return float(np.sum(valid & ok)) / (k * len(kth))


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi clock/throttle samples every 100 ms while the timed region runs."""
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")
    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.out = None

    def __enter__(self):
        try:
            self.out = tempfile.TemporaryFile(mode="w+")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.out, stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            time.sleep(0.15)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        rows = []
        if self.out is not None:
            self.out.seek(0)
            rows = [[c.strip() for c in ln.split(",")] for ln in self.out.read().splitlines() if ln.strip()]
        num = lambda v: float(v) if v.replace(".", "", 1).isdigit() else None  # noqa: E731
        sm = [num(r[0]) for r in rows if r and num(r[0]) is not None]
        mx = [num(r[1]) for r in rows if len(r) > 1 and num(r[1]) is not None]
        reasons = sorted({self.NAMES[i] for r in rows for i in range(4) if len(r) > 3 + i and r[3 + i] == "Active"})
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# ------------------------------------------------------------------ ncu traffic record
def recorded_traffic():
    """DRAM bytes per launch of the search kernel from the committed ncu summary, if present."""
    p = os.path.join(ROOT, "profiles", "hnsw_search_batched_c2.md")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        m = re.search(r"traffic_bytes_per_launch_full_batch:\s*([0-9.eE+]+)", f.read())
    return float(m.group(1)) if m else None


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ------------------------------------------------------------------ reference (CPU) arm
def cpu_reference_qps(path, queries, ef, k, target_seconds=3.0, space="l2"):
    """The reference's own knnQueryBatch on all host cores over a bounded sample of the batch
    (sized to about `target_seconds` per run, best of 3 runs as benchmark/eval.py:489-508 does).
    Returns (qps, sample_size, kind, cores)."""
    from oracle.oracle import OracleIndex, reference_module
    cores = os.cpu_count() or 1
    ref = reference_module()
    if ref is not None:
        idx = ref.init(method="hnsw", space=space)
        idx.loadIndex(path)
        idx.setQueryTimeParams({"efSearch": ef})
        run = lambda q: idx.knnQueryBatch(q, k=k, num_threads=cores)  # noqa: E731
        kind = "reference"
    else:
        oix = OracleIndex(path)
        run = lambda q: oix.search(q, k=k, ef=ef, nthreads=cores)  # noqa: E731
        kind = "port"
    n = min(len(queries), 1000)
    t0 = time.perf_counter()
    run(queries[:n])  # warm-up and sizing
    dt = time.perf_counter() - t0
    n = int(min(len(queries), max(n, n * target_seconds / max(dt, 1e-6))))
    best = None
    for _ in range(3):
        t0 = time.perf_counter()
        run(queries[:n])
        dt = time.perf_counter() - t0
        best = dt if best is None else min(best, dt)
    return n / best, n, kind, cores


# ------------------------------------------------------------------ main
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--profile-case", type=int, default=0, metavar="NQ",
                    help="profiling run: only NQ queries at the headline efSearch, no sweep, no baselines")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3

    rank, world, local = dist_init(args.gpus)
    base, queries, space, m = workload_data()

    if args.impl == "reference":
        if rank != 0:
            return
        path = ensure_index(base, space, m, 0, 1)
        ef = HEADLINE_EF
        qps, n, kind, cores = cpu_reference_qps(path, queries, ef, K, space=space)
        ms = 1e3 * len(queries) / qps
        line = {"metric": METRIC, "value": qps, "unit": "queries/s", "n_gpus": 1, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
                "config": {"workload": WORKLOAD, "n_base": len(base), "nq": len(queries), "dim": base.shape[1],
                           "M": m, "efConstruction": EFC, "efSearch": ef, "k": K},
                "cpu_baseline": {"value": qps, "unit": "queries/s", "cores": cores, "kind": kind,
                                 "sample": f"best of repeated knnQueryBatch over {n} of the {len(queries)} queries"},
                "e2e": {"value": qps, "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    import torch

    import nmslib_b200 as nmslib
    from nmslib_b200 import _capi
    from nmslib_b200.build import build
    build()
    torch.cuda.set_device(local)
    path = ensure_index(base, space, m, rank, world)
    index = nmslib.init(method="hnsw", space=space, device=local)
    index.loadIndex(path)
    lib = _capi.load()
    nq, dim = queries.shape
    dq = torch.from_numpy(queries).cuda()
    d_ids = torch.empty((nq, K), dtype=torch.int32, device="cuda")
    d_dists = torch.empty((nq, K), dtype=torch.float32, device="cuda")
    d_counts = torch.empty((nq,), dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream()

    def run_device(plain=False):
        rc = lib.nmsg_knn_batch(index._h, dq.data_ptr(), nq, dim, K, None, None, K, d_ids.data_ptr(),
                                d_dists.data_ptr(), d_counts.data_ptr(), None,
                                _capi.FLAG_DEVICE_PTRS | (_capi.FLAG_PLAIN_KERNEL if plain else 0),
                                stream.cuda_stream)
        _capi.check(rc)

    def time_device(steps, plain=False):
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        start.record(stream)
        for _ in range(steps):
            run_device(plain)
        end.record(stream)
        torch.cuda.synchronize()
        return start.elapsed_time(end) / steps

    if args.profile_case:
        # a small launch of the same kernel for ncu: the full index, a slice of the queries
        index.setQueryTimeParams({"efSearch": HEADLINE_EF})
        nq = min(nq, args.profile_case)
        for _ in range(args.warmup + args.steps):
            run_device()
        torch.cuda.synchronize()
        log(f"[bench] profile case: {args.warmup + args.steps} launches of {nq} queries")
        return

    # ---- untimed: recall / throughput sweep, headline ef
    gt_ids, kth = ground_truth(base, queries, K)
    sweep = []
    for ef in EF_SWEEP:
        index.setQueryTimeParams({"efSearch": ef})
        ids, dd, cnt = index.knnQueryBatchArrays(queries, K)
        rec = recall_at_k(dd, cnt, kth, K)
        run_device()
        ms_b = time_device(3)
        run_device(plain=True)
        ms_p = time_device(2, plain=True)
        sweep.append({"efSearch": ef, "recall@10": round(rec, 4), "qps_batched": round(nq / ms_b * 1e3),
                      "qps_plain": round(nq / ms_p * 1e3)})
        log(f"[bench] ef={ef} recall={rec:.4f} batched={nq / ms_b * 1e3:.0f} q/s plain={nq / ms_p * 1e3:.0f} q/s")
    head = next(s for s in sweep if s["efSearch"] == HEADLINE_EF)
    ef = HEADLINE_EF
    index.setQueryTimeParams({"efSearch": ef})
    _, _, _, st = index.knnQueryBatchArrays(queries, K, stats=True)
    alg_bytes = float(st[:, 3].sum())
    n_dist = float(st[:, 0].sum())

    # ---- timed: device-resident batches
    for _ in range(args.warmup):
        run_device()
    barrier(world)
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(stream)
        for _ in range(args.steps):
            run_device()
        end.record(stream)
        torch.cuda.synchronize()
    barrier(world)
    ms = start.elapsed_time(end) / args.steps
    ms_max = max_over_ranks(ms, world)
    value = world * nq / (ms_max * 1e-3)

    # ---- timed: end to end through the public API with host arrays
    h_q = np.ascontiguousarray(queries)
    for _ in range(2):
        index.knnQueryBatchArrays(h_q, K)
    barrier(world)
    torch.cuda.synchronize()
    e2e_steps = max(3, args.steps // 2)
    e_start, e_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e_start.record(stream)
    for _ in range(e2e_steps):
        ids, dd, cnt = index.knnQueryBatchArrays(h_q, K)  # synchronous: H2D, search, D2H
    e_end.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e_start.elapsed_time(e_end) / e2e_steps
    e2e_ms = max_over_ranks(e2e_ms, world)
    e2e = world * nq / (e2e_ms * 1e-3)

    peak, peak_kind = peaks()
    achieved = alg_bytes / (ms * 1e-3) / 1e9
    traffic = recorded_traffic()
    cpu = None
    if rank == 0 and world == 1:
        qps, n, kind, cores = cpu_reference_qps(path, queries, ef, K, space=space)
        cpu = {"value": qps, "unit": "queries/s", "cores": cores, "kind": kind,
               "sample": f"best of repeated knnQueryBatch(num_threads={cores}) over {n} of the {nq} queries, "
                         f"efSearch={ef}"}
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "queries/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_max, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded SIFT-like mixture)",
                "config": {"workload": WORKLOAD, "n_base": len(base), "nq_per_gpu": nq, "dim": dim, "M": m,
                           "efConstruction": EFC, "efSearch": ef, "k": K, "recall@10": head["recall@10"],
                           "parallelism": f"replicas x{world}", "l2_flush": "no: index (512 MB) > L2 (126 MB)",
                           "index_builder": "nmslib_b200 host builder"},
                "e2e": {"value": e2e, "unit": "queries/s", "h2d_bytes_per_step": int(h_q.nbytes),
                        "d2h_bytes_per_step": int(nq * K * 8 + nq * 4)},
                "gpu_launches": args.steps,
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                             "frac": achieved / peak, "peak_kind": peak_kind,
                             "traffic": traffic,
                             "algorithmic_bytes_per_launch": alg_bytes,
                             "distances_per_launch": n_dist},
                "cpu_baseline": cpu,
                "clocks": clk.summary(),
                "sweep": sweep}
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
