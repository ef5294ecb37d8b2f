"""Benchmark of the HNSW query path: batched persistent CUDA search on one B200 per rank.

Workload (default): 1M x 128 SIFT-like float32 base (seeded synthetic stand-in for SIFT1M),
10K queries, space l2, M=16, efConstruction=200, k=10, efSearch swept over
{16, 32, 64, 128, 256, 512}; the headline efSearch is the smallest one whose recall@10 reaches
0.95 against exact float64 neighbours. One step = one batch of 10K queries through the engine.
The index is built by the reference's own createIndex and written by its saveIndex (cached per
machine); both arms load that same file.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0). ``value`` is device-timed throughput with queries resident in HBM;
``e2e`` is the same metric through the public Python API with host arrays (H2D of the queries from
a page-locked host array and D2H of ids/distances/counts inside the timed region; the same call on
pageable arrays, staged and direct, and the list-returning knnQueryBatch are reported beside it). ``parity`` compares the engine's lists with
the reference's knnQueryBatch on the same file at full size. ``--impl reference`` times the
reference's own CPU knnQueryBatch (built from its sources into oracle/_ref) on the same index and
queries, and loads nothing of the engine. Multi-GPU runs are replicas (the query path has no
exchange step): each rank searches its own batch against its own copy of the index and ``value``
sums the queries of all ranks.
"""
from __future__ import annotations

import argparse
import importlib.util
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
    """Max of a per-rank scalar over all ranks (NCCL tensors on the GPU, gloo on the CPU)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(nq_per_rank, ms_per_rank, world):
    """Whole-job queries/s of `world` replicas that each searched nq_per_rank queries: the job
    takes as long as its slowest rank."""
    return world * nq_per_rank / (max_over_ranks(ms_per_rank, world) * 1e-3)


# ------------------------------------------------------------------ data and index
def _datasets():
    """nmslib_b200/datasets.py loaded by file path, so the reference arm imports nothing of the
    engine's package."""
    spec = importlib.util.spec_from_file_location("_bench_datasets", os.path.join(ROOT, "nmslib_b200", "datasets.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def workload_data(name=WORKLOAD):
    return _datasets().workload(name)


def index_path(name, m):
    return os.path.join(CACHE_DIR, f"{name}_M{m}_efc{EFC}_reference_build.hnsw")


BUILD_INFO = {}


def reference_module_or_none():
    from oracle.oracle import reference_module
    return reference_module()


def ensure_index(name, base, space, m, rank, world):
    """Rank 0 builds the index with the reference's own createIndex (all host cores) and writes it
    with its saveIndex, unless a copy is cached on this machine; the other ranks wait and load the
    same file. Returns the path, or None when the reference module is not available."""
    path = index_path(name, m)
    if rank == 0 and not os.path.exists(path):
        ref = reference_module_or_none()
        if ref is not None:
            os.makedirs(CACHE_DIR, exist_ok=True)
            threads = os.cpu_count() or 1
            t0 = time.time()
            idx = ref.init(method="hnsw", space=space)
            idx.addDataPointBatch(base)
            idx.createIndex({"M": m, "efConstruction": EFC, "indexThreadQty": threads}, print_progress=False)
            idx.saveIndex(path + ".tmp", save_data=False)
            del idx
            os.replace(path + ".tmp", path)
            BUILD_INFO[name] = {"seconds": round(time.time() - t0, 1), "threads": threads}
            log(f"[bench] reference createIndex {name}: {BUILD_INFO[name]}")
    barrier(world)
    return path if os.path.exists(path) else None


def engine_built_index(name, base, space, m):
    """Fallback when the reference module is missing: the engine's host builder (labelled so)."""
    from nmslib_b200 import SPACES, _capi
    path = os.path.join(CACHE_DIR, f"{name}_M{m}_efc{EFC}_engine_build.hnsw")
    if not os.path.exists(path):
        os.makedirs(CACHE_DIR, exist_ok=True)
        _capi.build_index(base, SPACES[space], m, EFC, nthreads=0, seed=0, out_path=path + ".tmp")
        os.replace(path + ".tmp", path)
    return path


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("model name"):
                    return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def ground_truth(base, queries, k):
    """Exact float64 neighbours on the GPU (measurement only): ids [nq, k], the k-th distance and
    the k smallest squared distances [nq, k] (ascending)."""
    import torch
    b = torch.from_numpy(base).cuda().double()
    bsq = (b * b).sum(1)
    kth = np.empty(len(queries))
    ids = np.empty((len(queries), k), np.int64)
    dk = np.empty((len(queries), k))
    for s in range(0, len(queries), 512):
        q = torch.from_numpy(queries[s:s + 512]).cuda().double()
        d = (q * q).sum(1, keepdim=True) - 2 * q @ b.T + bsq[None, :]
        v, i = torch.topk(d, k, dim=1, largest=False)
        ids[s:s + 512] = i.cpu().numpy()
        kth[s:s + 512] = v[:, -1].cpu().numpy()
        dk[s:s + 512] = v.cpu().numpy()
    del b
    torch.cuda.empty_cache()
    return ids, kth, dk


def recall_at_k(found_d, counts, kth, k):
    """ann-benchmarks recall: a returned neighbour counts when its distance is within the true
    k-th distance (so equal-distance alternatives are not penalised)."""
    valid = np.arange(found_d.shape[1])[None, :k] < np.minimum(counts, k)[:, None]
    ok = found_d[:, :k] <= (kth * (1 + 1e-6) + 1e-6)[:, None]
    return float(np.sum(valid & ok)) / (k * len(kth))


def list_parity(ids_a, d_a, cnt_a, ids_b, d_b, cnt_b):
    """Result lists a (the engine) against b (the reference), both ascending by distance:
    identical lists; lists whose ids differ only inside runs of equal distance (including the run
    cut by k, where either side may keep any of the tied items); and the largest relative distance
    difference position by position."""
    n = len(cnt_a)
    identical = tie_only = other = 0
    max_rel = 0.0
    for r in range(n):
        ca, cb = int(cnt_a[r]), int(cnt_b[r])
        if ca != cb:
            other += 1
            continue
        da, db = d_a[r, :ca].astype(np.float64), d_b[r, :cb].astype(np.float64)
        if ca:
            max_rel = max(max_rel, float((np.abs(da - db) / np.maximum(np.abs(db), 1e-30)).max()))
        ia, ib = ids_a[r, :ca], ids_b[r, :cb]
        if (ia == ib).all():
            identical += 1
            continue
        ok = bool((da == db).all())
        s0 = 0
        while ok and s0 < ca:
            e = s0
            while e < ca and db[e] == db[s0]:
                e += 1
            if e < ca and sorted(ia[s0:e].tolist()) != sorted(ib[s0:e].tolist()):
                ok = False
            s0 = e
        if ok:
            tie_only += 1
        else:
            other += 1
    return {"queries": n, "identical_lists_frac": identical / max(1, n), "tie_only_frac": tie_only / max(1, n),
            "other_frac": other / max(1, n), "max_rel_dist": max_rel}


def reference_arrays(ref_index, queries, k, threads):
    """The reference's knnQueryBatch as dense arrays (ids, dists, counts), ascending."""
    res = ref_index.knnQueryBatch(queries, k=k, num_threads=threads)
    ids = np.full((len(res), k), -1, np.int32)
    dd = np.full((len(res), k), np.inf, np.float32)
    cnt = np.zeros(len(res), np.int32)
    for r, (i, d) in enumerate(res):
        ids[r, :len(i)] = i
        dd[r, :len(d)] = d
        cnt[r] = len(i)
    return ids, dd, cnt


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi clock/throttle samples every 100 ms while the timed region runs."""
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap,clocks.mem")
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
        mem = [num(r[7]) for r in rows if len(r) > 7 and num(r[7]) is not None]
        reasons = sorted({self.NAMES[i] for r in rows for i in range(4) if len(r) > 3 + i and r[3 + i] == "Active"})
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "mem_mhz": statistics.median(mem) if mem else None, "reasons": reasons, "samples": len(rows)}


# ------------------------------------------------------------------ ncu traffic record
def recorded_traffic():
    """DRAM bytes of one 10K-query search step (the lean kernel's descent and level-0 launches)
    from the committed ncu summary, if present."""
    p = os.path.join(ROOT, "profiles", "search_lean_kernel_c2.md")
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
def cpu_reference_qps(path, queries, ef, k, target_seconds=3.0, space="l2", one_thread=True):
    """The reference's own knnQueryBatch on the host cores over a bounded sample of the batch
    (sized to about `target_seconds` per run, best of 3 runs as benchmark/eval.py:489-508 does),
    with every core and, when `one_thread`, with one thread. Returns a dict."""
    from oracle.oracle import OracleIndex, reference_module
    cores = os.cpu_count() or 1
    ref = reference_module()
    if ref is not None:
        idx = ref.init(method="hnsw", space=space)
        idx.loadIndex(path)
        idx.setQueryTimeParams({"efSearch": ef})
        run = lambda q, t: idx.knnQueryBatch(q, k=k, num_threads=t)  # noqa: E731
        kind = "reference"
    else:
        oix = OracleIndex(path)
        run = lambda q, t: oix.search(q, k=k, ef=ef, nthreads=t)  # noqa: E731
        kind = "port"

    def best_qps(threads, seconds):
        n = min(len(queries), 1000 if threads > 1 else 200)
        t0 = time.perf_counter()
        run(queries[:n], threads)  # warm-up and sizing
        dt = time.perf_counter() - t0
        n = int(min(len(queries), max(n, n * seconds / max(dt, 1e-6))))
        best = None
        for _ in range(3):
            t0 = time.perf_counter()
            run(queries[:n], threads)
            dt = time.perf_counter() - t0
            best = dt if best is None else min(best, dt)
        return n / best, n

    qps, n = best_qps(cores, target_seconds)
    out = {"value": qps, "unit": "queries/s", "cores": cores, "kind": kind, "cpu_model": cpu_model(),
           "sample": f"best of 3 knnQueryBatch(num_threads={cores}) over {n} of the {len(queries)} queries, "
                     f"efSearch={ef}"}
    if one_thread:
        q1, n1 = best_qps(1, 1.0)
        out["one_thread"] = {"value": q1, "sample": f"best of 3 knnQueryBatch(num_threads=1) over {n1} queries"}
    return out


# ------------------------------------------------------------------ serving and brute force
def serve_sweep(index, queries, rates_qps=(250e3, 500e3, 1e6), seconds=1.0, seed=11, workload=WORKLOAD):
    """p50/p99 request latency and achieved QPS of the continuous-batching server at several
    offered loads (queries per second), open-loop Poisson arrivals. The memory budget holds 32 x 256
    search slots (one visited byte per base vector each) shared by 64 lanes; a request takes one
    slot per query."""
    from nmslib_b200.serving import Server
    rng = np.random.default_rng(seed)
    n = index.info["n"]
    budget = max(8 << 30, int(32 * 256 * ((n + 15) // 16 * 16 + 1) * 1.05))
    srv = Server(index, memory_budget_bytes=budget, max_batch=256, max_k=100, max_lanes=64)
    out = []
    try:
        for qps in rates_qps:
            mean_batch = (256 - 1) / np.log(256)
            n_req = int(qps * seconds / mean_batch)
            sizes = np.minimum(256, np.floor(np.exp(rng.uniform(0, np.log(257), n_req)))).astype(np.int32)
            ks = rng.choice([10, 100], n_req).astype(np.int32)
            efs = rng.choice([100, 400], n_req).astype(np.int32)
            offs = rng.integers(0, len(queries) - 256, n_req)
            arrivals = np.cumsum(rng.exponential(mean_batch / qps, n_req))
            lat, wall = srv.run_trace(queries, offs, sizes, ks, efs, arrivals)
            small = sizes <= 256
            out.append({"offered_qps": qps, "requests": n_req, "achieved_qps": round(float(sizes.sum()) / wall),
                        "p50_ms": round(float(np.percentile(lat[small], 50)) * 1e3, 3),
                        "p99_ms": round(float(np.percentile(lat[small], 99)) * 1e3, 3), "lanes": srv.lanes})
            log(f"[bench] serving {qps:.0f} q/s offered: {out[-1]}")
    finally:
        srv.close()
    return {"workload": workload + " index, request mix of the 5M serving config", "points": out,
            "memory_budget_bytes": budget}


def brute_force_measure(index, queries, k=10, reps=3, base=None, true_d=None, space="l2"):
    """Exact k-NN of the whole batch over every stored vector: time and throughput. The tensor-core
    path (l2 / cosine / negdot, dim <= 256) reports 2 * nq * n * padded dim BF16 FLOP per batch; the
    exact CUDA-core scan (L1, LInf, wider rows) 2 * nq * n * dim FP32 FLOP. With `base` and the
    float64 top-k distances `true_d` [nq, k] (l2), every query's returned set is checked: the
    float64 distances of the returned ids must be the float64 top-k distances (exact top-k up to
    the choice among equal distances)."""
    import torch
    ids, d, c, st = index.bruteForceBatchArrays(queries, k, stats=True)  # builds the BF16 copy
    t = []
    for _ in range(reps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        index.bruteForceBatchArrays(queries, k)
        t.append(time.perf_counter() - t0)
    best = min(t)
    n, dim = index.info["n"], index.info["dim"]
    if st[0] == 0:  # the exact CUDA-core scan
        flops = 2.0 * len(queries) * n * dim
        res = {"path": "exact CUDA-core scan", "queries": len(queries), "k": k, "ms_end_to_end": round(best * 1e3, 3),
               "qps": round(len(queries) / best), "fp32_tflops": round(flops / best / 1e12, 1)}
    else:
        kp = (dim + 63) // 64 * 64
        flops = 2.0 * len(queries) * n * kp
        res = {"path": "tensor-core BF16 + exact rerank", "queries": len(queries), "k": k,
               "ms_end_to_end": round(best * 1e3, 3), "qps": round(len(queries) / best),
               "tensor_tflops": round(flops / best / 1e12, 1), "sample_rows": int(st[0]),
               "max_rows_reranked": int(st[1]), "rescanned": int(st[2])}
    if base is not None and true_d is not None and space == "l2":
        res["verify_fp64"] = bf_verify_l2(base, queries, ids, c, true_d)
        res["bf16_key_error"] = bf16_key_error_l2(base, queries[:256])
    log(f"[bench] brute force: {res}")
    return res


def bf_verify_l2(base, queries, ids, counts, true_d):
    """Float64 squared distances of the returned ids against the float64 top-k: the fraction of
    queries whose returned distances equal the true k smallest, position by position."""
    import torch
    b = torch.from_numpy(base).cuda()
    exact = 0
    worst = 0.0
    k = true_d.shape[1]
    for s0 in range(0, len(queries), 1024):
        q = torch.from_numpy(queries[s0:s0 + 1024]).cuda().double()
        i = torch.from_numpy(ids[s0:s0 + 1024, :k].astype(np.int64)).cuda()
        x = b[i.clamp_min(0)].double()
        d = ((x - q[:, None, :]) ** 2).sum(-1)
        d = torch.where(i >= 0, d, torch.full_like(d, float("inf")))
        d, _ = torch.sort(d, dim=1)
        t = torch.from_numpy(true_d[s0:s0 + 1024]).cuda()
        ok = (d == t).all(dim=1) & torch.from_numpy(counts[s0:s0 + 1024] == k).cuda()
        exact += int(ok.sum().item())
        worst = max(worst, float(((d - t).abs() / t.abs().clamp_min(1e-30)).max().item()))
    del b
    torch.cuda.empty_cache()
    return {"queries": len(queries), "exact_topk_frac": exact / max(1, len(queries)), "max_rel_dist_err": worst}


def bf16_key_error_l2(base, queries):
    """Largest |BF16 key - float64 key| of the tensor-core pass over every base row for a sample of
    queries: key = 2 q.x - |x|^2 with q and x rounded to BF16 and the product summed in FP32 (the
    GEMM's inputs and accumulator type), against the same key in float64. The rerank removes this
    error; the bound the kernel uses to pick candidates covers it."""
    import torch
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    try:
        b32 = torch.from_numpy(base).cuda()
        bb = b32.bfloat16().float()
        xn = (b32 * b32).sum(1)
        b64 = b32.double()
        xn64 = (b64 * b64).sum(1)
        worst = 0.0
        scale = 0.0
        for s0 in range(0, len(queries), 64):
            q = torch.from_numpy(queries[s0:s0 + 64]).cuda()
            kb = 2.0 * (q.bfloat16().float() @ bb.T) - xn[None, :]
            k64 = 2.0 * (q.double() @ b64.T) - xn64[None, :]
            worst = max(worst, float((kb.double() - k64).abs().max().item()))
            scale = max(scale, float(k64.abs().max().item()))
    finally:
        torch.backends.cuda.matmul.allow_tf32 = prev
    torch.cuda.empty_cache()
    return {"queries": len(queries), "max_abs_key_err": worst, "max_abs_key": scale,
            "key": "2 q.x - |x|^2, BF16 inputs, FP32 accumulation"}


def profile_scan(n, calls, dim=960, nq=200):
    """The exact CUDA-core scan (negdot rows wider than 256) through the public API, for ncu:
    n x dim standard-normal rows and nq queries (seed 0), indexed by a small device-built graph
    (M 4, efConstruction 8: the scan never reads it)."""
    import torch
    import nmslib_b200 as nmslib
    from nmslib_b200 import _capi
    from nmslib_b200.build import build
    build()
    rng = np.random.default_rng(0)
    base = rng.standard_normal((n, dim), dtype=np.float32)
    q = rng.standard_normal((nq, dim), dtype=np.float32)
    os.makedirs(CACHE_DIR, exist_ok=True)
    path = os.path.join(CACHE_DIR, f"scan_profile_{n}_{dim}.hnsw")
    _capi.build_index(base, 2, 4, 8, nthreads=0, seed=0, out_path=path, device=0)
    index = nmslib.init(method="hnsw", space="negdotprod")
    index.loadIndex(path)
    t = []
    for _ in range(calls):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        index.bruteForceBatchArrays(q, K)
        t.append(time.perf_counter() - t0)
    best = min(t)
    log(f"[bench] scan profile case: {calls} calls of {nq} queries over {n} x {dim}; best {best * 1e3:.2f} ms "
        f"({2.0 * nq * n * dim / best / 1e12:.1f} TFLOP/s end to end)")


def build_compare(base, space, m, queries, kth, ref_recall, device):
    """The same index built by the engine with the level-0 construction searches on the GPU: wall
    time and recall@10 at the headline efSearch, beside the reference build's."""
    import nmslib_b200 as nmslib
    from nmslib_b200 import SPACES, _capi
    path = os.path.join(CACHE_DIR, f"{WORKLOAD}_M{m}_efc{EFC}_device_build.hnsw")
    t0 = time.time()
    _capi.build_index(base, SPACES[space], m, EFC, nthreads=0, seed=0, out_path=path, device=device)
    dt = time.time() - t0
    idx = nmslib.init(method="hnsw", space=space, device=device)
    idx.loadIndex(path)
    idx.setQueryTimeParams({"efSearch": HEADLINE_EF})
    _, dd, cnt = idx.knnQueryBatchArrays(queries, K)
    rec = recall_at_k(dd, cnt, kth, K)
    del idx
    os.remove(path)
    ref_build = BUILD_INFO.get(WORKLOAD)
    res = {"reference_build_s": ref_build["seconds"] if ref_build else None,
           "device_build_s": round(dt, 2), "host_threads": os.cpu_count(),
           f"recall@10_ef{HEADLINE_EF}": {"reference_build": round(ref_recall, 4), "device_build": round(rec, 4)}}
    log(f"[bench] index build: {res}")
    return res


# ------------------------------------------------------------------ the other workloads
AUX = {"c3": "c3_glove1m_d100_cos", "c4": "c4_abs1m_d960_negdot", "c5": "c5_unit5m_d96_l2"}


def fp64_truth(base, queries, k, space):
    """Exact float64 top-k keys on the GPU (measurement only): k-th best distance per query."""
    import torch
    b = torch.from_numpy(base).cuda().double()
    if space == "cosinesimil":
        b = b / b.norm(dim=1, keepdim=True).clamp_min(1e-300)
    bsq = (b * b).sum(1)
    kth = np.empty(len(queries))
    for s0 in range(0, len(queries), 256):
        q = torch.from_numpy(queries[s0:s0 + 256]).cuda().double()
        if space == "cosinesimil":
            q = q / q.norm(dim=1, keepdim=True).clamp_min(1e-300)
            d = 1 - q @ b.T
        elif space == "negdotprod":
            d = -(q @ b.T)
        else:
            d = (q * q).sum(1, keepdim=True) - 2 * q @ b.T + bsq[None, :]
        v, _ = torch.topk(d, k, dim=1, largest=False)
        kth[s0:s0 + 256] = v[:, -1].cpu().numpy()
    del b
    torch.cuda.empty_cache()
    return kth


def aux_workload(which, device=0, serving_rates=(250e3, 500e3, 1e6)):
    """One of the other benchmark configurations, measured on this GPU, as a dict:
    c3 = 1M x 100 cosine (M 24): HNSW efSearch sweep with recall@10 against float64, the reference's
         CPU knnQueryBatch at efSearch 200, and the tensor-core brute force of 10K queries checked
         against float64; c4 = 1M x 960 negdot (M 16): one launch of 8K queries with per-query
         k in {1, 10, 100} and efSearch in [64, 1024] (SearchOld at 1000 and above), the reference
         on a sample of the same mix, and the streamed tensor-core brute force of 1K queries;
    c5 = 5M x 96 l2 (M 32): the serving loop under open-loop Poisson arrivals of requests of
         1-256 queries (k in {10, 100}, efSearch in {100, 400}), p50 / p99 latency.
    Indices are built by the engine's device-assisted builder (the reference's createIndex on these
    sizes takes minutes to tens of minutes) and cached on this machine."""
    import torch

    import nmslib_b200 as nmslib
    from nmslib_b200 import SPACES, _capi
    name = AUX[which]
    t_start = time.time()
    base, queries, space, m = workload_data(name)
    path = os.path.join(CACHE_DIR, f"{name}_M{m}_efc{EFC}_device_build.hnsw")
    build_s = None
    if not os.path.exists(path):
        os.makedirs(CACHE_DIR, exist_ok=True)
        t0 = time.time()
        _capi.build_index(base, SPACES[space], m, EFC, nthreads=0, seed=0, out_path=path + ".tmp", device=device)
        os.replace(path + ".tmp", path)
        build_s = round(time.time() - t0, 1)
    index = nmslib.init(method="hnsw", space=space, device=device)
    index.loadIndex(path)
    out = {"workload": name, "n_base": len(base), "nq": len(queries), "dim": base.shape[1], "M": m,
           "efConstruction": EFC, "space": space, "index_builder": "nmslib_b200 device-assisted build",
           "index_build_s": build_s}

    def timed(fn, reps=3):
        fn()
        best = None
        for _ in range(reps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            r = fn()
            dt = time.perf_counter() - t0
            best = dt if best is None else min(best, dt)
        return best, r

    if which == "c3":
        qs = queries[:10_000]
        kth = fp64_truth(base, qs, 10, space)
        rows = []
        for ef in (50, 100, 200, 400):
            index.setQueryTimeParams({"efSearch": ef})
            dt, (ids, d, cnt) = timed(lambda: index.knnQueryBatchArrays(qs, 10))
            rows.append({"efSearch": ef, "recall@10": round(recall_at_k(d.astype(np.float64), cnt, kth, 10), 4),
                         "qps_e2e": round(len(qs) / dt)})
            log(f"[bench] {name} ef={ef}: {rows[-1]}")
        out["hnsw"] = rows
        cpu = cpu_reference_qps(path, qs, 200, 10, space=space, one_thread=False)
        out["cpu_reference"] = {"efSearch": 200, "qps": round(cpu["value"]), "cores": cpu["cores"],
                                "kind": cpu["kind"], "sample": cpu["sample"]}
        out["bruteforce"] = brute_force_measure(index, qs)
        out["bruteforce"]["verify_fp64"] = bf_verify_keys(base, qs, index, space)
    elif which == "c4":
        rng = np.random.default_rng(4)
        nq = len(queries)
        k = rng.choice([1, 10, 100], nq).astype(np.int32)
        ef = rng.integers(64, 1025, nq).astype(np.int32)
        dt, (ids, d, cnt) = timed(lambda: index.knnQueryBatchArrays(queries, k, ef=ef))
        # the same launch with each way of fetching the 3840-byte rows: staged in shared memory 8
        # per round by one bulk copy (TMA unit) per row (the default) or by 16-byte copies spread
        # over the lanes, or gathered into registers, one row per 8-lane group
        row_copy = {"default_ms": round(dt * 1e3, 2)}
        for label, cfg in (("staged_bulk_ms", dict(stage_rows=8, row_copy=2)),
                           ("staged_cp16_ms", dict(stage_rows=8, row_copy=1)),
                           ("register_rows_ms", dict(stage_rows=-1, rows_per_group=1))):
            index.setLaunchConfig(**cfg)
            dts, (ids_s, _, _) = timed(lambda: index.knnQueryBatchArrays(queries, k, ef=ef))
            index.setLaunchConfig()
            assert np.array_equal(ids_s, ids), f"{label}: results differ from the default launch"
            row_copy[label] = round(dts * 1e3, 2)
        truth10 = fp64_truth(base, queries, 10, space)
        sel = k == 10
        out["mixed_batch"] = {"queries": nq, "qps_e2e": round(nq / dt), "ms": round(dt * 1e3, 2),
                              "row_copy": row_copy,
                              "searchold_queries": int((ef >= 1000).sum()),
                              "recall@10_of_k10_queries": round(
                                  recall_at_k(d[sel][:, :10].astype(np.float64), cnt[sel], truth10[sel], 10), 4)}
        log(f"[bench] {name} mixed batch: {out['mixed_batch']}")
        ref = reference_module_or_none()
        if ref is not None:
            r = ref.init(method="hnsw", space=space)
            r.loadIndex(path)
            sample = np.arange(min(nq, 2000))
            t_total = 0.0
            for kk in (1, 10, 100):
                for e in np.unique(ef[sample][k[sample] == kk]):
                    rows = sample[(k[sample] == kk) & (ef[sample] == e)]
                    r.setQueryTimeParams({"efSearch": int(e)})
                    t0 = time.perf_counter()
                    r.knnQueryBatch(queries[rows], k=int(kk), num_threads=os.cpu_count())
                    t_total += time.perf_counter() - t0
            out["cpu_reference"] = {"qps": round(len(sample) / t_total), "cores": os.cpu_count(),
                                    "kind": "reference",
                                    "sample": f"{len(sample)} queries of the mixed batch, grouped by (k, efSearch)"}
        out["bruteforce"] = brute_force_measure(index, queries[:1000])
        out["bruteforce"]["verify_fp64"] = bf_verify_keys(base, queries[:1000], index, space)
    elif which == "c5":
        qs = queries[:10_000]
        kth = fp64_truth(base, qs, 10, space)
        rows = []
        for efs in (100, 400):
            index.setQueryTimeParams({"efSearch": efs})
            dt, (ids, d, cnt) = timed(lambda: index.knnQueryBatchArrays(qs, 10))
            rows.append({"efSearch": efs, "recall@10": round(recall_at_k(d.astype(np.float64), cnt, kth, 10), 4),
                         "qps_e2e": round(len(qs) / dt)})
            log(f"[bench] {name} ef={efs}: {rows[-1]}")
        out["hnsw"] = rows
        out["serving"] = serve_sweep(index, queries, rates_qps=serving_rates, workload=name)
    del index
    torch.cuda.empty_cache()
    out["seconds"] = round(time.time() - t_start, 1)
    return out


def bf_verify_keys(base, queries, index, space, k=10):
    """Brute-force results against float64 for any space: the float64 distances of the returned ids
    equal the float64 top-k distances (to 1e-9 relative, the float64 sums of the two being in
    different orders), and the fraction of queries whose sets agree that way."""
    import torch
    ids, d, cnt = index.bruteForceBatchArrays(queries, k)
    b = torch.from_numpy(base).cuda().double()
    if space == "cosinesimil":
        b = b / b.norm(dim=1, keepdim=True).clamp_min(1e-300)
    bsq = (b * b).sum(1)
    ok = 0
    for s0 in range(0, len(queries), 256):
        q = torch.from_numpy(queries[s0:s0 + 256]).cuda().double()
        if space == "cosinesimil":
            q = q / q.norm(dim=1, keepdim=True).clamp_min(1e-300)
            full = 1 - q @ b.T
        elif space == "negdotprod":
            full = -(q @ b.T)
        else:
            full = (q * q).sum(1, keepdim=True) - 2 * q @ b.T + bsq[None, :]
        top, _ = torch.topk(full, k, dim=1, largest=False)
        got = torch.gather(full, 1, torch.from_numpy(ids[s0:s0 + 256, :k].astype(np.int64)).cuda())
        got, _ = torch.sort(got, dim=1)
        tol = 1e-9 * top.abs().clamp_min(1.0)
        ok += int(((got - top).abs() <= tol).all(dim=1).sum().item())
    del b
    torch.cuda.empty_cache()
    return {"queries": len(queries), "exact_topk_frac": ok / max(1, len(queries))}


def run_aux(args):
    from nmslib_b200.build import build
    build()
    print(json.dumps(aux_workload(args.workload)))


# ------------------------------------------------------------------ main
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--profile-case", type=int, default=0, metavar="NQ",
                    help="profiling run: only NQ queries at the headline efSearch, no sweep, no baselines")
    ap.add_argument("--profile-bruteforce", type=int, default=0, metavar="NQ",
                    help="profiling run: exact brute force (k=10) of NQ queries over the base, warmup + steps calls")
    ap.add_argument("--profile-scan", type=int, default=0, metavar="N",
                    help="profiling run: the exact CUDA-core scan alone (200 queries, k=10) over N x 960 normal "
                         "rows (negdot, a small device-built graph), warmup + steps calls")
    ap.add_argument("--no-aux", action="store_true",
                    help="skip the c3 / c4 / c5 sections of the default line")
    ap.add_argument("--workload", choices=["c2", "c3", "c4", "c5"], default="c2",
                    help="c2 (default, the headline line); c3 cosine 1M x 100 + brute force; c4 negdot "
                         "1M x 960 mixed k/ef batch; c5 l2 5M x 96 serving")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.profile_scan:
        profile_scan(args.profile_scan, args.warmup + args.steps)
        return
    if args.workload != "c2":
        run_aux(args)
        return

    rank, world, local = dist_init(args.gpus)
    base, queries, space, m = workload_data()

    if args.impl == "reference":
        # the reference alone: its createIndex builds the file (or a cached copy is read), its
        # knnQueryBatch is timed; nothing of the engine is imported or loaded
        if rank != 0:
            return
        if reference_module_or_none() is None:
            print(json.dumps({"impl": "reference", "unavailable": "reference module not built (oracle/_ref)"}))
            return
        path = ensure_index(WORKLOAD, base, space, m, 0, 1)
        ef = HEADLINE_EF
        cpu = cpu_reference_qps(path, queries, ef, K, space=space)
        qps = cpu["value"]
        ms = 1e3 * len(queries) / qps
        line = {"metric": METRIC, "value": qps, "unit": "queries/s", "n_gpus": 1, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
                "config": {"workload": WORKLOAD, "n_base": len(base), "nq": len(queries), "dim": base.shape[1],
                           "M": m, "efConstruction": EFC, "efSearch": ef, "k": K,
                           "index_builder": "reference createIndex", "index_build": BUILD_INFO.get(WORKLOAD)},
                "cpu_baseline": cpu,
                "e2e": {"value": qps, "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    import torch

    import nmslib_b200 as nmslib
    from nmslib_b200 import _capi
    from nmslib_b200.build import build
    build()
    torch.cuda.set_device(local)
    path = ensure_index(WORKLOAD, base, space, m, rank, world)
    index_builder = "reference createIndex"
    if path is None:  # no reference module on this machine: the engine's own builder, labelled so
        index_builder = "nmslib_b200 host builder (reference module unavailable)"
        if rank == 0:
            engine_built_index(WORKLOAD, base, space, m)
        barrier(world)
        path = engine_built_index(WORKLOAD, base, space, m)
    index = nmslib.init(method="hnsw", space=space, device=local)
    index.loadIndex(path)
    lib = _capi.load()
    nq, dim = queries.shape
    dq = torch.from_numpy(queries).cuda()
    d_ids = torch.empty((nq, K), dtype=torch.int32, device="cuda")
    d_dists = torch.empty((nq, K), dtype=torch.float32, device="cuda")
    d_counts = torch.empty((nq,), dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream()

    def run_device(plain=False, graph=False):
        flags = _capi.FLAG_DEVICE_PTRS | (_capi.FLAG_PLAIN_KERNEL if plain else 0) | (
            _capi.FLAG_CUDA_GRAPH if graph else 0)
        rc = lib.nmsg_knn_batch(index._h, dq.data_ptr(), nq, dim, K, None, None, K, d_ids.data_ptr(),
                                d_dists.data_ptr(), d_counts.data_ptr(), None, flags, stream.cuda_stream)
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

    if args.profile_bruteforce:
        # the tensor-core brute force alone, through the public API, for ncu
        qs = queries[:args.profile_bruteforce]
        for _ in range(args.warmup + args.steps):
            index.bruteForceBatchArrays(qs, K)
        torch.cuda.synchronize()
        log(f"[bench] brute-force profile case: {args.warmup + args.steps} calls of {len(qs)} queries")
        return

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
    gt_ids, kth, true_d = ground_truth(base, queries, K)
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
    # launch shape picked by the autotuner on this batch (untimed); the timed steps use it
    from nmslib_b200.autotune import autotune
    best_shape, tune_table = autotune(index, queries, K, ef)
    log(f"[bench] autotune: best {best_shape} " + " ".join(f"{s}:{ms:.3f}ms" for s, ms in tune_table))

    # ---- timed: device-resident batches, each step one replay of the captured launch
    for _ in range(args.warmup):
        run_device(graph=True)
    barrier(world)
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(stream)
        for _ in range(args.steps):
            run_device(graph=True)
        end.record(stream)
        torch.cuda.synchronize()
    barrier(world)
    ms = start.elapsed_time(end) / args.steps
    launches_per_step = lib.nmsg_last_kernel_launches(index._h)  # descent, order, level 0 when split
    ms_max = max_over_ranks(ms, world)
    value = world * nq / (ms_max * 1e-3)  # == replica_throughput(nq, ms, world)

    # ---- timed: end to end through the public API with host arrays: the queries in page-locked
    # host memory (h_qp), and for comparison in pageable memory (h_q)
    h_q = np.ascontiguousarray(queries)
    h_qp = torch.empty(queries.shape, dtype=torch.float32, pin_memory=True).numpy()
    h_qp[:] = queries
    e2e_steps = max(3, args.steps // 2)

    def time_e2e(arr):
        for _ in range(2):
            index.knnQueryBatchArrays(arr, K)
        barrier(world)
        torch.cuda.synchronize()
        e_start, e_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e_start.record(stream)
        for _ in range(e2e_steps):
            index.knnQueryBatchArrays(arr, K)  # synchronous: H2D, search, D2H
        e_end.record(stream)
        torch.cuda.synchronize()
        return max_over_ranks(e_start.elapsed_time(e_end) / e2e_steps, world)

    # pageable queries copied directly (host_copy 1), then through the default page-locked staging,
    # then the page-locked queries the line reports
    shape_kw = dict(warps_per_block=best_shape[0], rows_per_group=best_shape[1], visited_hash_log2=best_shape[2],
                    stage_rows=best_shape[3], queries_per_warp=best_shape[4], row_copy=best_shape[5])
    index.setLaunchConfig(**shape_kw, host_copy=1)
    e2e_direct_ms = time_e2e(h_q)
    index.setLaunchConfig(**shape_kw)
    e2e_pageable_ms = time_e2e(h_q)
    e2e_ms = time_e2e(h_qp)
    e2e = world * nq / (e2e_ms * 1e-3)
    # the reference's own call, knnQueryBatch: a list of per-query (ids, distances) arrays
    index.knnQueryBatch(h_q, K)
    torch.cuda.synchronize()
    t_list = time.perf_counter()
    for _ in range(e2e_steps):
        index.knnQueryBatch(h_q, K)
    list_ms = max_over_ranks((time.perf_counter() - t_list) * 1e3 / e2e_steps, world)

    # ---- full-size parity against the reference's knnQueryBatch on the same file (checker)
    parity = None
    if rank == 0 and world == 1:
        parity = full_size_parity(index, path, queries, space, (HEADLINE_EF, 256))
        parity["c1_gauss10k_d128_l2"] = c1_parity(local)

    # ---- serving: open-loop Poisson arrivals of the serving mix (batch 1..256 log-uniform,
    # k in {10, 100}, efSearch in {100, 400}) against the same resident index
    serving = serve_sweep(index, queries) if world == 1 else None

    # ---- exact brute force on the tensor cores (same queries and vectors), checked against float64
    brute = brute_force_measure(index, queries, base=base, true_d=true_d, space=space) if world == 1 else None

    # ---- the index built again with the construction searches on the GPU
    build_info = build_compare(base, space, m, queries, kth, head["recall@10"], local) if world == 1 else None

    # ---- the other configurations (cosine + brute force, wide mixed batch, 5M serving)
    aux = None
    if world == 1 and not args.no_aux:
        del index
        torch.cuda.empty_cache()
        aux = {}
        for which in ("c3", "c4", "c5"):
            try:
                aux[which] = aux_workload(which, local)
            except Exception as e:  # noqa: BLE001 - reported in the line, the headline stands
                aux[which] = {"error": f"{type(e).__name__}: {e}"}
                log(f"[bench] {which} failed: {e}")

    peak, peak_kind = peaks()
    achieved = alg_bytes / (ms * 1e-3) / 1e9
    traffic = recorded_traffic()
    cpu = None
    if rank == 0 and world == 1:
        cpu = cpu_reference_qps(path, queries, ef, K, space=space)
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "queries/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_max, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded SIFT-like mixture)",
                "config": {"workload": WORKLOAD, "n_base": len(base), "nq_per_gpu": nq, "dim": dim, "M": m,
                           "efConstruction": EFC, "efSearch": ef, "k": K, "recall@10": head["recall@10"],
                           "parallelism": f"replicas x{world}", "l2_flush": "no: index (512 MB) > L2 (126 MB)",
                           "index_builder": index_builder, "index_build": BUILD_INFO.get(WORKLOAD)},
                "e2e": {"value": e2e, "unit": "queries/s", "h2d_bytes_per_step": int(h_q.nbytes),
                        "d2h_bytes_per_step": int(nq * K * 8 + nq * 4),
                        "inputs": "queries in a page-locked host array; results into new numpy arrays",
                        "pageable_value": world * nq / (e2e_pageable_ms * 1e-3),
                        "direct_copies_value": world * nq / (e2e_direct_ms * 1e-3),
                        "knnQueryBatch_list_value": world * nq / (list_ms * 1e-3)},
                "gpu_launches": args.steps * launches_per_step,
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                             "frac": achieved / peak, "peak_kind": peak_kind,
                             "traffic": traffic,
                             "algorithmic_bytes_per_launch": alg_bytes,
                             "distances_per_launch": n_dist},
                "cpu_baseline": cpu,
                "clocks": clk.summary(),
                "parity": parity,
                "sweep": sweep,
                "launch": {"autotuned_shape": {"warps_per_block": best_shape[0], "rows_per_group": best_shape[1],
                                               "visited_hash_log2": best_shape[2], "stage_rows": best_shape[3],
                                               "queries_per_warp": best_shape[4], "row_copy": best_shape[5]},
                           "cuda_graph": True},
                "serving": serving,
                "bruteforce": brute,
                "index_build": build_info,
                "aux": aux}
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def full_size_parity(index, path, queries, space, efs):
    """The engine's lists against the reference's knnQueryBatch on the same index file and
    queries, at each efSearch of `efs` (the whole batch, all host threads)."""
    ref = reference_module_or_none()
    if ref is None:
        return {"unavailable": "reference module not built (oracle/_ref)"}
    r = ref.init(method="hnsw", space=space)
    r.loadIndex(path)
    out = {}
    for ef in efs:
        index.setQueryTimeParams({"efSearch": ef})
        ids, dd, cnt = index.knnQueryBatchArrays(queries, K)
        r.setQueryTimeParams({"efSearch": ef})
        ri, rd, rc = reference_arrays(r, queries, K, os.cpu_count() or 1)
        out[f"ef{ef}"] = list_parity(ids, dd, cnt, ri, rd, rc)
        log(f"[bench] parity ef={ef}: {out[f'ef{ef}']}")
    index.setQueryTimeParams({"efSearch": HEADLINE_EF})
    return out


def c1_parity(device):
    """The plain small configuration: 10K x 128 Gaussian mixture, l2, M 16, efConstruction 200,
    built by the reference's createIndex; efSearch 100, k 10, 1K queries. The engine against the
    reference's knnQueryBatch on that file, and recall@10 against exact float64 neighbours."""
    import nmslib_b200 as nmslib
    name = "c1_gauss10k_d128_l2"
    base, queries, space, m = workload_data(name)
    path = ensure_index(name, base, space, m, 0, 1)
    ref = reference_module_or_none()
    if path is None or ref is None:
        return {"unavailable": "reference module not built (oracle/_ref)"}
    idx = nmslib.init(method="hnsw", space=space, device=device)
    idx.loadIndex(path)
    idx.setQueryTimeParams({"efSearch": 100})
    ids, dd, cnt = idx.knnQueryBatchArrays(queries, K)
    r = ref.init(method="hnsw", space=space)
    r.loadIndex(path)
    r.setQueryTimeParams({"efSearch": 100})
    ri, rd, rc = reference_arrays(r, queries, K, os.cpu_count() or 1)
    _, kth, _ = ground_truth(base, queries, K)
    out = list_parity(ids, dd, cnt, ri, rd, rc)
    out.update({"efSearch": 100, "k": K, "recall@10": round(recall_at_k(dd, cnt, kth, K), 4),
                "recall@10_reference": round(recall_at_k(rd, rc, kth, K), 4),
                "index_build": BUILD_INFO.get(name)})
    log(f"[bench] c1 parity: {out}")
    return out


if __name__ == "__main__":
    main()
