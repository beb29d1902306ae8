#!/usr/bin/env python
"""Headline benchmark: the angular IVF-PQ fast-scan + RefineIndex workload.

Workload (synthetic stand-in for a GloVe-100-angular-shaped set; the real set
is not available offline): 2,000 centres ~ N(0, I_100), cluster c drawn with
p ~ (c + 1)^-1.1, row = centre + 0.3 * N(0, I), L2-normalised; 1,200,000 base
rows (seed 0) and 10,000 queries (seed 1) from the same mixture; cosine;
IVFIndex(nlist 4096) + PQ 50 x 4-bit fast-scan trained with e-means (seed 1),
RefineIndex(k_factor 10), k = 10. The operating point is swept: nprobe over
8..256 at k_factor 10 (the configured re-rank depth) and at larger k_factors;
recall@10 is measured against exact FP64 brute force, and the metric is
queries per second at the smallest nprobe that reaches 0.95 at any swept
k_factor (ties to the smaller k_factor). The configured k_factor's own point
is reported beside it.

One step = one batch_query of the 10,000 queries. `value` is measured with
the queries already in HBM (device-resident search, CUDA events on the
launching stream, L2 flushed between steps); `e2e` is the same metric through
the public Python API with host arrays (copies in and out inside the timed
region). `cpu_baseline` times the reference's own C++ build (oracle/_ref) on
the host cores on the index this library built, and compares its results
with this library's query by query (`reference_parity`).

`--impl reference` is the reference's CPU path alone: its library trains and
fills the index itself (minutes, once per box; cached), sweeps the same
operating points and answers the queries on all host cores.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl qann_b200|reference]

For N > 1 every rank holds a replica of the index and serves its own 10,000
queries (seed 1 + rank): weak scaling with no collective on the data path;
the step time is the max over ranks.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import pathlib
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))
os.environ.setdefault("QANN_DISABLE_AVX512", "1")

# nprobe is swept over 8..256 as the workload names it. At the configured
# k_factor 10 recall@10 saturates below 0.95 on this set (0.919 at nprobe
# 256, 0.933 at 1024), so the sweep also runs larger k_factors (the
# RefineIndex's re-rank depth, a query-time setting of the same index), and
# the metric is taken at the smallest nprobe <= 256 that reaches 0.95 at any
# of them (ties to the smaller k_factor).
FULL = dict(n=1_200_000, d=100, centres=2000, zipf=1.1, sigma=0.3, nq=10_000, nlist=4096, m=50, k=10, kf=10,
            train_seed=1, nprobes=[8, 16, 32, 64, 128, 256], kfs=[10, 20, 40, 80], target=0.95)
SMALL = dict(FULL, n=120_000, nq=2_000, nlist=512)   # --small: a quick functional check, not a bench line
CACHE = pathlib.Path(os.environ.get("QANN_B200_BENCH_CACHE", pathlib.Path(tempfile.gettempdir()) / "qann_b200_bench"))
L2_FLUSH_BYTES = 256 << 20   # twice the B200's 126 MB L2
METRIC = "QPS@recall10>=0.95 (angular 1.2Mx100, IVF4096-PQ50x4fs + refine)"


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# ---- data --------------------------------------------------------------------------------

def mixture(cfg, seed_rows, nrows):
    c_rng = np.random.default_rng(12345)
    centres = c_rng.standard_normal((cfg["centres"], cfg["d"]), dtype=np.float32)
    p = (np.arange(cfg["centres"]) + 1.0) ** -cfg["zipf"]
    p /= p.sum()
    rng = np.random.default_rng(seed_rows)
    lab = rng.choice(cfg["centres"], size=nrows, p=p)
    x = centres[lab] + np.float32(cfg["sigma"]) * rng.standard_normal((nrows, cfg["d"]), dtype=np.float32)
    x /= np.linalg.norm(x, axis=1, keepdims=True)
    return np.ascontiguousarray(x, dtype=np.float32)


def tag(cfg):
    return f"angular_{cfg['n']}x{cfg['d']}_nl{cfg['nlist']}_m{cfg['m']}_kf{cfg['kf']}"


def build_or_load(cfg, base, rank, world, barrier):
    import qann_b200 as qb
    CACHE.mkdir(parents=True, exist_ok=True)
    path = CACHE / f"{tag(cfg)}.qann"
    if rank == 0 and not path.exists():
        t = time.time()
        ivf = qb.IVFIndex(cfg["d"], cfg["nlist"], 16, metric=qb.Metric.Cosine)
        ivf.enable_pq(cfg["m"], fast_scan=True)
        ivf.train(base, seed=cfg["train_seed"])
        t_train = time.time() - t
        r = qb.RefineIndex(ivf, cfg["kf"])
        r.add(base)
        t_add = time.time() - t - t_train
        r.save(str(path) + ".part")
        os.replace(str(path) + ".part", path)
        log(f"built index on the GPU: train {t_train:.1f}s add {t_add:.1f}s "
            f"(cosine_inner_product={ivf.cosine_inner_product})")
    barrier()
    return qb.load(path), path


def ground_truth(cfg, base, queries, dev):
    """Exact top-k by cosine: fp32 similarities on the GPU to pick 64 candidates,
    rescored in fp64 (measurement only)."""
    import torch
    digest = hashlib.sha1(queries[:16].tobytes()).hexdigest()[:12]
    path = CACHE / f"{tag(cfg)}_gt_{queries.shape[0]}_{digest}.npy"
    if path.exists():
        return np.load(path)
    torch.backends.cuda.matmul.allow_tf32 = False
    b = torch.from_numpy(base).to(dev)
    out = np.empty((queries.shape[0], cfg["k"]), np.int64)
    for s in range(0, queries.shape[0], 1000):
        q = torch.from_numpy(queries[s:s + 1000]).to(dev)
        cand = torch.topk(q @ b.T, 64, dim=1).indices
        exact = torch.einsum("qd,qcd->qc", q.double(), b[cand].double())
        order = torch.argsort(-exact, dim=1, stable=True)[:, :cfg["k"]]
        out[s:s + 1000] = torch.gather(cand, 1, order).cpu().numpy()
    del b
    np.save(path, out)
    return out


def recall(ids, gt):
    k = gt.shape[1]
    return float(np.mean([len(set(a[:k]) & set(b)) / k for a, b in zip(ids, gt)]))


def sweep_operating_points(cfg, index, queries, gt, cache_name):
    """recall@k over nprobe 8..256 at each k_factor of cfg["kfs"] (10, the
    configured value, first), each row stopping at the first nprobe that
    reaches the target. The operating point is the smallest nprobe that
    reaches it at any swept k_factor, ties to the smaller k_factor: the scan
    of the probed lists is most of a query's work in both implementations,
    and the rule needs no timing, so both arms pick the same point from the
    same recalls. "configured" is k_factor 10's own point (the nprobe that
    reaches the target, else the largest swept). Works on any index with the
    RefineIndex API (this library's or the reference's)."""
    path = CACHE / f"{tag(cfg)}_{cache_name}_sweep2.json"
    if path.exists():
        return json.loads(path.read_text())
    ivf = index.base
    sweep, chosen, own = {}, None, None
    for kf in cfg["kfs"]:
        index.k_factor = kf
        row = {}
        for npb in [p for p in cfg["nprobes"] if p <= cfg["nlist"]]:
            if chosen and npb >= chosen["nprobe"]:
                break   # (cannot beat the point found)
            ivf.nprobe = npb
            ids, _ = index.batch_query(queries, cfg["k"])
            row[str(npb)] = round(recall(ids, gt), 4)
            log(f"k_factor {kf} nprobe {npb}: recall@{cfg['k']} {row[str(npb)]}")
            if row[str(npb)] >= cfg["target"]:
                chosen = {"k_factor": kf, "nprobe": npb}
                break
        sweep[str(kf)] = row
        if kf == cfg["kf"]:
            last = list(row)[-1]
            own = {"k_factor": kf, "nprobe": int(last), "recall": row[last], "target_met": row[last] >= cfg["target"]}
    index.k_factor = cfg["kf"]
    res = {"sweep": sweep, "chosen": chosen, "target_met": chosen is not None,
           "rule": "smallest nprobe reaching the target at any swept k_factor, ties to the smaller k_factor",
           "configured": own}
    if chosen is None:   # the target is out of reach: report the configured k_factor's last point
        res["chosen"] = {"k_factor": own["k_factor"], "nprobe": own["nprobe"]}
    path.write_text(json.dumps(res))
    return res


# ---- measurement helpers ---------------------------------------------------------------------

class Clocks:
    """nvidia-smi samples during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                       "-lms", "50", "-i", str(self.gpu)], stdout=subprocess.PIPE,
                                      stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.p = None
        time.sleep(0.1)
        return self

    def __exit__(self, *exc):
        time.sleep(0.1)
        self.out = ""
        if self.p:
            self.p.terminate()
            try:
                self.out, _ = self.p.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()
                self.out, _ = self.p.communicate()

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in (self.out or "").splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak(key, fallback):
    try:
        return float(json.loads((ROOT / "MEASURED_PEAKS.json").read_text())[key]), "measured"
    except Exception:
        return fallback, "fallback"


def alu_roofline(alg_bytes, launch_ms, clocks, dev):
    """The scan against the integer pipe: 4-bit lookups per second over the
    peak rate of the lookup core. Every probed vector costs m lookups (m / 2
    code bytes, so lookups = 2 x the algorithmic bytes). The core spends one
    integer op per lookup (two byte permutes and one three-input add per four
    lookups, and the 16-bit widening of the byte sums), and an SM issues 64
    integer lane-ops per clock (32-bit add, logic, permute), so the peak is
    SMs x 64 x the median SM clock sampled during the timed region."""
    import torch
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    mhz = (clocks or {}).get("sm_mhz") or 1965.0
    lookups = 2 * alg_bytes
    achieved = lookups / (launch_ms / 1e3) / 1e12
    peak = sms * 64 * mhz * 1e6 / 1e12
    return {"bound": "integer pipe", "achieved": round(achieved, 3), "peak": round(peak, 3),
            "unit": "T lookups/s", "frac": round(achieved / peak, 4), "lookups_per_launch": lookups,
            "ops_per_lookup": 1.0, "sms": sms, "sm_mhz": mhz}


def scan_traffic():
    """dram bytes per scan launch from the committed ncu summary, when present."""
    p = ROOT / "profiles" / "scan_traffic.txt"
    if not p.exists():
        return None
    for line in p.read_text().splitlines():
        if line.startswith("bytes_per_launch="):
            return float(line.split("=", 1)[1])
    return None


def algorithmic_scan_bytes(cfg, index, queries, nprobe, dev):
    """Code bytes the scan must read per launch: for every (query, probed
    list), the list's vectors x m/2 bytes (4-bit codes)."""
    import torch
    ivf = index.base
    sizes = torch.from_numpy(ivf.list_sizes().astype(np.int64)).to(dev)
    cent = torch.from_numpy(ivf.centroids()).to(dev)
    total = 0
    for s in range(0, queries.shape[0], 2000):
        q = torch.from_numpy(queries[s:s + 2000]).to(dev)
        d2 = (q * q).sum(1, keepdim=True) - 2 * q @ cent.T + (cent * cent).sum(1)[None]
        probes = torch.topk(d2, nprobe, dim=1, largest=False).indices
        total += int(sizes[probes].sum())
    return total * cfg["m"] // 2


# ---- the reference arm -------------------------------------------------------------------------

def reference_build(cfg):
    """The reference library's own train + add of the workload's index (no
    part of this library involved), saved once per box. Its e-means
    assignment runs on one core without BLAS, so this takes minutes."""
    from oracle import ref
    CACHE.mkdir(parents=True, exist_ok=True)
    path = CACHE / f"{tag(cfg)}_reference.qann"
    if not path.exists():
        base = mixture(cfg, 0, cfg["n"])
        ref.set_num_threads(os.cpu_count() or 1)
        t = time.time()
        ivf = ref.IVFIndex(cfg["d"], cfg["nlist"], 16, metric=ref.COSINE)
        ivf.enable_pq(cfg["m"], fast_scan=True)
        ivf.train(base, seed=cfg["train_seed"])
        t_train = time.time() - t
        r = ref.RefineIndex(ivf, cfg["kf"])
        r.add(base)
        log(f"reference library built the index on the CPU: train {t_train:.1f}s add {time.time() - t - t_train:.1f}s")
        r.save(str(path) + ".part")
        os.replace(str(path) + ".part", path)
    return path


def time_reference(r, queries, k, steps, warmup, seconds_per_step=2.0):
    """QPS of the reference library's batch_query on bounded samples of the
    queries: each step one call on ~seconds_per_step of CPU work."""
    t = time.time()
    r.batch_query(queries[:200], k)
    per_q = max((time.time() - t) / 200, 1e-6)
    sample = int(min(queries.shape[0], max(200, seconds_per_step / per_q)))
    for _ in range(warmup):
        r.batch_query(queries[:sample], k)
    times = []
    for s in range(steps):
        off = (s * sample) % max(1, queries.shape[0] - sample + 1)
        t = time.perf_counter()
        r.batch_query(queries[off:off + sample], k)
        times.append(time.perf_counter() - t)
    return sample * len(times) / sum(times), sample, times


def reference_arm(args, cfg):
    """The reference's own CPU path end to end: its library (oracle/_ref,
    compiled from the reference sources) trains and fills the index, picks
    the operating point by the same sweep, and answers the queries on all
    host cores. This library is not imported; ground truth is torch FP64."""
    from oracle import ref
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    if not ref.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libqann_ref.so was not built"}))
        return 0
    import torch
    dev = torch.device("cuda:0") if torch.cuda.is_available() else torch.device("cpu")
    path = reference_build(cfg)
    base = mixture(cfg, 0, cfg["n"])
    queries = mixture(cfg, 1, cfg["nq"])
    gt = ground_truth(cfg, base, queries, dev)
    del base
    r = ref.load(path)
    cores = os.cpu_count() or 1
    ref.set_num_threads(cores)
    sel = sweep_operating_points(cfg, r, queries, gt, "reference")
    op = sel["chosen"]
    # the configured k_factor's own point, one timed pass over the queries
    own = sel["configured"]
    r.k_factor, r.base.nprobe = own["k_factor"], own["nprobe"]
    own_qps, _, _ = time_reference(r, queries, cfg["k"], 1, 1)
    r.k_factor, r.base.nprobe = op["k_factor"], op["nprobe"]
    qps, sample, times = time_reference(r, queries, cfg["k"], args.steps, args.warmup)
    ids, _ = r.batch_query(queries, cfg["k"])
    rec = recall(ids, gt)
    line = {
        "impl": "reference", "metric": METRIC,
        "value": round(qps, 1), "unit": "queries/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(1e3 * sum(times) / len(times), 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
        "config": {"workload": tag(cfg), "nq": cfg["nq"], "k": cfg["k"], "k_factor": op["k_factor"],
                   "nprobe": op["nprobe"], "recall@10": round(rec, 4), "recall_target": cfg["target"],
                   "target_met": sel["target_met"], "sweep": sel["sweep"], "queries_per_step": sample,
                   "threads": cores,
                   "index": "trained and filled by the reference library on the host (train(seed=1) + add), "
                            "loaded and queried by it",
                   "configured_k_factor": {"k_factor": own["k_factor"], "nprobe": own["nprobe"],
                                           "recall@10": own["recall"], "target_met": own["target_met"],
                                           "qps": round(own_qps, 1)}},
        "cpu_baseline": {"value": round(qps, 1), "unit": "queries/s", "cores": cores, "kind": "reference",
                         "sample": f"{sample} queries per step, one batch_query on {cores} threads"},
        "e2e": {"value": round(qps, 1), "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


# ---- our arm -------------------------------------------------------------------------------------

def served(index, queries, k, nprobe, batch_ids,
           rates=(25_000, 50_000, 100_000, 200_000, 225_000, 250_000, 275_000, 300_000, 350_000, 400_000, 450_000,
                  500_000, 600_000),
           per_rate=20_000, slots=2, max_batch=512):
    """Open-loop Poisson arrivals through the continuous-batching server:
    achieved QPS and p50 / p99 latency (arrival to results) per offered rate;
    every served result must equal the batch path's."""
    import qann_b200 as qb
    nq = queries.shape[0]
    rng = np.random.default_rng(3)
    out = []
    same = True
    with qb.Server(index, slots=slots, max_batch=max_batch) as srv:
        srv.replay(queries[:2000], np.full(2000, k, np.int32), np.zeros(2000),
                   nprobes=np.full(2000, nprobe, np.int32))   # warm-up
        for rate in rates:
            n = per_rate
            rows = np.arange(n) % nq
            arrivals = np.cumsum(rng.exponential(1.0 / rate, size=n))
            t = time.perf_counter()
            ids, _, lat = srv.replay(queries[rows], np.full(n, k, np.int32), arrivals,
                                     nprobes=np.full(n, nprobe, np.int32))
            wall = time.perf_counter() - t
            same &= bool(np.array_equal(ids, batch_ids[rows]))
            lat_ms = np.sort(lat) * 1e3
            # served throughput of the stream: requests / (start of the arrival
            # schedule to the last result); the call's wall time also holds the
            # trace's copy-in and lead-in, reported beside it
            span = float(np.max(arrivals + lat))
            out.append({"offered_qps": rate, "achieved_qps": round(n / span, 1),
                        "p50_ms": round(float(lat_ms[n // 2]), 3), "p99_ms": round(float(lat_ms[int(0.99 * n)]), 3),
                        "requests": n, "replay_call_s": round(wall, 4)})
            log(f"served at {rate}/s: {out[-1]}")
        st = srv.stats()
    ok = [r for r in out if r["p99_ms"] <= 2.0]
    best = max(ok, key=lambda r: r["achieved_qps"]) if ok else None
    return {"slots": slots, "max_batch": max_batch, "k": k, "nprobe": nprobe, "arrivals": "Poisson, open loop",
            "latency": "arrival to results on the host", "rates": out, "mean_batch": round(st["completed"] / st["batches"], 1),
            "results_equal_batch_path": same, "best_qps_at_p99_le_2ms": best["achieved_qps"] if best else None}


def plain_fp32_qps(base, queries, k, metric):
    """The plain FP32 GPU batch path on the same rows: exact flat search with
    FP32 tiles only (no tensor cores, no index), through the public API."""
    import qann_b200 as qb
    flat = qb.FlatIndex(base.shape[1], metric=metric)
    flat.add(base)
    qb.set_tensor_filter(0)
    try:
        flat.batch_query(queries[:200], k)   # warm-up
        n = min(2000, queries.shape[0])
        best = 0.0
        for _ in range(3):   # the best of three, in the baseline's favour
            t = time.perf_counter()
            flat.batch_query(queries[:n], k)
            best = max(best, n / (time.perf_counter() - t))
        return best
    finally:
        qb.set_tensor_filter(1)


def fp32_ivf_batch_qps(index, queries, k):
    """The same IVF fast-scan + refine batch path with the tensor cores off
    (the coarse step in exact FP32 tiles), through the public API: the best
    of three batch_query calls on all queries."""
    import qann_b200 as qb
    qb.set_tensor_filter(0)
    try:
        index.batch_query(queries[:1000], k)   # warm-up
        best = 0.0
        for _ in range(3):
            t = time.perf_counter()
            index.batch_query(queries, k)
            best = max(best, queries.shape[0] / (time.perf_counter() - t))
        return best
    finally:
        qb.set_tensor_filter(1)


# ---- other workloads (--workload): flat search, index training, served stream -------------------

def gaussian_mixture(n, d, centres, sigma, seed_rows, seed_centres=12345):
    """Uniform choice among `centres` N(0, I) centres plus sigma * N(0, I) noise."""
    c = np.random.default_rng(seed_centres).standard_normal((centres, d), dtype=np.float32)
    rng = np.random.default_rng(seed_rows)
    x = np.empty((n, d), np.float32)
    for s in range(0, n, 1 << 20):
        e = min(n, s + (1 << 20))
        x[s:e] = c[rng.integers(0, centres, e - s)] + np.float32(sigma) * rng.standard_normal((e - s, d), dtype=np.float32)
    return x


def device_steps(index, q_dev, nq, k, steps, warmup, flush=None):
    """CUDA-event times (ms) of `steps` device-resident searches of the nq queries."""
    import torch
    oi = torch.empty((nq, k), dtype=torch.int64, device=q_dev.device)
    od = torch.empty((nq, k), dtype=torch.float32, device=q_dev.device)
    st = torch.cuda.current_stream()
    for _ in range(warmup):
        index.search_device(q_dev.data_ptr(), nq, k, oi.data_ptr(), od.data_ptr(), st.cuda_stream)
    torch.cuda.synchronize()
    times = []
    for _ in range(steps):
        if flush is not None:
            flush.fill_(1.0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        index.search_device(q_dev.data_ptr(), nq, k, oi.data_ptr(), od.data_ptr(), st.cuda_stream)
        e1.record(st)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    return times, oi, od


def small_workload(args):
    """The reference's own CPU-scale case: base 100,000 x 128 uniform [0, 1)
    (seeded), squared L2, nlist 256 k-means (seed 1), PQ 64 x 4-bit fast-scan,
    nprobe 16, RefineIndex k_factor 10, 1,000 queries of the same law, k = 10."""
    import torch
    import qann_b200 as qb
    from qann_b200 import profiling
    n, d, nq, k = 100_000, 128, 1_000, 10
    x = np.random.default_rng(0).random((n, d), dtype=np.float32)
    q = np.random.default_rng(1).random((nq, d), dtype=np.float32)
    ivf = qb.IVFIndex(d, 256, 16)
    ivf.enable_pq(64, fast_scan=True)
    ivf.train(x, seed=1)
    index = qb.RefineIndex(ivf, 10)
    index.add(x)
    dev = torch.device("cuda:0")
    q_dev = torch.from_numpy(q).to(dev)
    profiling.enable(True)
    launches0 = profiling.launch_count()
    times, oi, _ = device_steps(index, q_dev, nq, k, args.steps, args.warmup)
    launches = profiling.launch_count() - launches0
    profiling.enable(False)
    ids = oi.cpu().numpy()
    xt = torch.from_numpy(x).to(dev)
    gt = torch.topk(torch.cdist(q_dev.double(), xt.double()), k, largest=False).indices.cpu().numpy()
    rec = recall(ids, gt)
    t = time.perf_counter()
    e_ids, _ = index.batch_query(q, k)
    e2e = nq / (time.perf_counter() - t)
    cpu, same = None, None
    if not args.no_cpu_baseline:
        from oracle import ref
        if ref.available():
            path = CACHE / "small_100000x128.qann"
            CACHE.mkdir(parents=True, exist_ok=True)
            index.save(path)
            r = ref.load(path)
            cores = os.cpu_count() or 1
            ref.set_num_threads(cores)
            t = time.perf_counter()
            r_ids, _ = r.batch_query(q, k)
            dt = time.perf_counter() - t
            same = bool(np.array_equal(r_ids, e_ids))
            cpu = {"value": round(nq / dt, 1), "unit": "queries/s", "cores": cores, "kind": "reference",
                   "sample": f"all {nq} queries, one batch_query on {cores} threads, the same .qann index"}
    total = sum(times)
    print(json.dumps({
        "metric": "QPS (100k x 128 uniform, IVF256-PQ64x4fs + refine kf10, nprobe 16, k=10)",
        "value": round(nq * args.steps / (total / 1e3), 1), "unit": "queries/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(total / args.steps, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
        "config": {"workload": "small_100000x128_nl256_m64_kf10", "nprobe": 16, "recall@10": round(rec, 4),
                   "results_equal_reference": same},
        "e2e": {"value": round(e2e, 1), "unit": "queries/s", "h2d_bytes_per_step": nq * d * 4,
                "d2h_bytes_per_step": nq * k * 12},
        "gpu_launches": launches, "cpu_baseline": cpu}))
    return 0


def flat_workload(args):
    """Exact flat search as a GEMM: 10,000,000 x 96 float32 (N(0,1) per
    dimension, rows scaled by LogNormal(0, 0.25)), 10,000 queries of the same
    law, k = 100, squared L2 and inner product. Exact results through the BF16
    tensor-core filter and FP32 recheck; per-distance error against FP64."""
    import torch
    import qann_b200 as qb
    from qann_b200 import profiling
    n, d, nq, k = (1_000_000, 96, 2_000, 100) if args.small else (10_000_000, 96, 10_000, 100)
    rng = np.random.default_rng(0)
    x = rng.standard_normal((n, d), dtype=np.float32)
    x *= np.exp(rng.normal(0.0, 0.25, size=(n, 1))).astype(np.float32)
    rq = np.random.default_rng(1)
    q = rq.standard_normal((nq, d), dtype=np.float32) * np.exp(rq.normal(0.0, 0.25, size=(nq, 1))).astype(np.float32)
    dev = torch.device("cuda:0")
    q_dev = torch.from_numpy(q).to(dev)
    per_metric = {}
    peak, peak_src = measured_peak("bf16_tflops", 1590.0)
    for metric, name in ((qb.Metric.L2, "l2"), (qb.Metric.InnerProduct, "ip")):
        idx = qb.FlatIndex(d, metric=metric)
        idx.add(x)
        profiling.enable(True)
        profiling.reset()
        launches0 = profiling.launch_count()
        times, oi, od = device_steps(idx, q_dev, nq, k, args.steps, args.warmup)
        launches = profiling.launch_count() - launches0
        mm_ms, mm_n = profiling.get("mm_filter")
        profiling.enable(False)
        total = sum(times)
        ids, dist = oi.cpu().numpy(), od.cpu().numpy()
        # the exact FP32 path on a sample: identical results
        qb.set_tensor_filter(0)
        i0, d0 = idx.batch_query(q[:32], k)
        qb.set_tensor_filter(1)
        same = bool(np.array_equal(i0, ids[:32]) and d0.tobytes() == dist[:32].tobytes())
        # per-distance error against FP64 on a sample
        s = 256
        rows = torch.from_numpy(x[ids[:s].ravel()].reshape(s, k, d)).to(dev).double()
        qq = q_dev[:s].double()[:, None, :]
        d64 = ((qq - rows) ** 2).sum(-1) if name == "l2" else -(qq * rows).sum(-1)
        err = (torch.from_numpy(dist[:s]).to(dev).double() - d64).abs() / d64.abs().clamp_min(1e-30)
        t = time.perf_counter()
        idx.batch_query(q, k)
        e2e = nq / (time.perf_counter() - t)
        flops = 2.0 * nq * n * d
        per_metric[name] = {
            "qps": round(nq * args.steps / (total / 1e3), 1), "ms_per_step": round(total / args.steps, 2),
            "e2e_qps": round(e2e, 1), "identical_to_exact_fp32": same,
            "rel_err_vs_fp64": {"max": float(err.max()), "mean": float(err.mean())},
            "tensor_tflops": round(flops / (total / args.steps / 1e3) / 1e12, 1),
            "filter_kernel_tflops": round(flops * args.steps / (mm_ms / 1e3) / 1e12, 1) if mm_ms else None,
            "gpu_launches": launches}
        del idx
        log(f"flat {name}: {per_metric[name]}")
    cpu = None
    if not args.no_cpu_baseline:
        from oracle import ref
        if ref.available():
            cores = os.cpu_count() or 1
            ref.set_num_threads(cores)
            r = ref.FlatIndex(d)
            r.add(x)
            sample = 16
            t = time.perf_counter()
            r.batch_query(q[:sample], k)
            dt = time.perf_counter() - t
            cpu = {"value": round(sample / dt, 2), "unit": "queries/s", "cores": cores, "kind": "reference",
                   "sample": f"{sample} queries, L2, one batch_query on {cores} threads"}
    l2 = per_metric["l2"]
    print(json.dumps({
        "metric": "exact flat search QPS (10M x 96, k=100)", "value": l2["qps"], "unit": "queries/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": l2["ms_per_step"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "bf16 filter + f32 recheck", "data": "synthetic",
        "config": {"workload": f"flat_{n}x{d}_k{k}", "nq": nq, "l2": "inputs larger than L2 (3.84 GB rows)"},
        "per_metric": per_metric,
        "roofline": {"bound": "tensor", "achieved": l2["tensor_tflops"], "peak": peak, "unit": "TFLOP/s",
                     "frac": round(l2["tensor_tflops"] / peak, 4), "traffic": None, "peak_source": peak_src},
        "e2e": {"value": l2["e2e_qps"], "unit": "queries/s", "h2d_bytes_per_step": nq * d * 4,
                "d2h_bytes_per_step": nq * k * 12},
        "gpu_launches": l2["gpu_launches"], "filter_schedule": qb.filter_options(), "cpu_baseline": cpu}))
    return 0


def train_workload(args):
    """Index training, batched: 2,000,000 x 128 Gaussian mixture (8,192
    centres, sigma 0.2, uniform sizes); coarse k-means nlist 16,384 for 20
    Lloyd iterations, then PQ 64 x 4-bit; seed 1."""
    import torch
    import qann_b200 as qb
    n, nlist = (200_000, 2048) if args.small else (2_000_000, 16384)
    d, m, iters = 128, 64, 20
    x = gaussian_mixture(n, d, 8192, 0.2, seed_rows=0)
    # warm-up: context, kernels and pools on a small problem
    w = qb.IVFIndex(d, 256, 8)
    w.enable_pq(m, fast_scan=True)
    w.train(x[:20000], max_iters=2, seed=1, clustering=qb.Clustering.Lloyd)
    del w
    torch.cuda.synchronize()
    ivf = qb.IVFIndex(d, nlist, 16)
    ivf.enable_pq(m, fast_scan=True)
    t = time.perf_counter()
    ivf.train(x, max_iters=iters, seed=1, clustering=qb.Clustering.Lloyd)
    torch.cuda.synchronize()
    secs = time.perf_counter() - t
    pairs = float(n) * nlist * (iters + 1)   # assignments: every iteration plus the final one
    cpu = None
    if not args.no_cpu_baseline:
        from oracle import ref
        if ref.available():
            cores = os.cpu_count() or 1
            ref.set_num_threads(cores)
            sample = 50_000
            r = ref.IVFIndex(d, nlist, 16)
            r.enable_pq(m, fast_scan=True)
            t = time.perf_counter()
            r.train(x[:sample], max_iters=1, seed=1, clustering=ref.LLOYD)
            dt = time.perf_counter() - t
            rate = 2.0 * sample * nlist / dt   # one iteration and the final assignment
            cpu = {"value": round(pairs / rate, 1), "unit": "s (extrapolated)", "cores": cores, "kind": "reference",
                   "sample": f"train() of {sample} points, 1 Lloyd iteration, {dt:.1f} s: "
                             f"{rate:.3g} point-list pairs/s extrapolated to the full training"}
    print(json.dumps({
        "metric": "IVF training time (2M x 128, nlist 16384, 20 Lloyd iterations, PQ 64x4)", "value": round(secs, 2),
        "unit": "s", "n_gpus": 1, "steps": 1, "warmup": 1, "ms_per_step": round(secs * 1e3, 1),
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "bf16 filter + f32/f64",
        "data": "synthetic", "config": {"workload": f"train_{n}x{d}_nl{nlist}_lloyd{iters}_pq{m}"},
        "assign_pairs_per_s": round(pairs / secs, 1), "filter_schedule": qb.filter_options(), "cpu_baseline": cpu}))
    return 0


def served_workload(args):
    """Served stream over a device-resident IVF-PQ fast-scan + refine index of
    5,000,000 x 128 (Gaussian mixture, 8,192 centres, sigma 0.2), nlist 16,384,
    PQ 64 x 4-bit, k_factor 10: Poisson arrivals at 5k-300k queries/s, k in
    {10, 100}, nprobe log-uniform in 8..256, 30% of requests with an allowed-id
    bitmap of selectivity uniform in [1%, 50%]; p50 / p99 latency per rate."""
    import torch
    import qann_b200 as qb
    n, nlist = (500_000, 2048) if args.small else (5_000_000, 16384)
    d, m, kf = 128, 64, 10
    path = CACHE / f"served_{n}x{d}_nl{nlist}_m{m}_kf{kf}.qann"
    CACHE.mkdir(parents=True, exist_ok=True)
    x = gaussian_mixture(n, d, 8192, 0.2, seed_rows=0)
    if not path.exists():
        t = time.time()
        ivf = qb.IVFIndex(d, nlist, 32)
        ivf.enable_pq(m, fast_scan=True)
        ivf.train(x, seed=1)
        r = qb.RefineIndex(ivf, kf)
        r.add(x)
        r.save(str(path) + ".part")
        os.replace(str(path) + ".part", path)
        log(f"built the served index on the GPU in {time.time() - t:.1f} s")
        del r, ivf
    index = qb.load(path)
    nreq = 20_000
    q = gaussian_mixture(nreq, d, 8192, 0.2, seed_rows=1)
    if args.scan_shape != "auto":
        qb.set_scan_options(autotune=False, variant={"global": 0, "staged": 1, "dense": 2}[args.scan_shape])
    batch = batch_scan_roofline(index, q[:10_000], m, (args.nprobe,) if args.nprobe else (32, 256),
                                max(3, args.steps // 10), max(3, args.warmup))
    if args.no_served:   # the batch measurement alone
        print(json.dumps({
            "metric": "batch QPS of the served index (5M x 128 IVF16384-PQ64x4fs + refine kf10, k 10)",
            "value": batch[-1]["qps"], "unit": "queries/s", "n_gpus": 1, "steps": max(3, args.steps // 10),
            "warmup": max(3, args.warmup), "ms_per_step": round(10_000 / batch[-1]["qps"] * 1e3, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
            "config": {"workload": f"served_{n}x{d}_nl{nlist}_m{m}_kf{kf}", "nq": 10_000, "k": 10,
                       "nprobe": batch[-1]["nprobe"], "l2": "flushed between steps (256 MB write)"},
            "batch_scan": batch}))
        return 0
    rng = np.random.default_rng(2)
    pool = []
    for _ in range(16):
        sel = rng.uniform(0.01, 0.5)
        bits = rng.random(n) < sel
        pool.append(bits)
    rates = (5_000, 10_000, 20_000, 50_000, 100_000, 200_000, 300_000)
    out = []
    same = True
    with qb.Server(index, slots=2, max_batch=512, mem_budget=4 << 30) as srv:
        fids = [srv.add_filter(np.packbits(np.concatenate([b, np.zeros((-n) % 64, bool)]), bitorder="little")
                               .view(np.uint64)) for b in pool]
        arng = np.random.default_rng(3)
        ks = arng.choice(np.array([10, 100], np.int32), size=nreq)
        npb = np.rint(np.exp(arng.uniform(np.log(8), np.log(256), size=nreq))).astype(np.int32)
        filt = np.where(arng.random(nreq) < 0.3, arng.integers(0, len(fids), nreq), -1)
        fid = np.array([fids[f] if f >= 0 else -1 for f in filt], np.int32)
        srv.replay(q[:2000], ks[:2000], np.zeros(2000), nprobes=npb[:2000], filter_ids=fid[:2000])   # warm-up
        from qann_b200 import profiling
        kind = np.where(filt >= 0, np.where(ks == 100, "filtered_k100", "filtered_k10"),
                        np.where(ks == 100, "k100", "k10"))

        def by_kind(lat):
            return {kd: {"requests": int((kind == kd).sum()),
                         "p50_ms": round(float(np.median(lat[kind == kd])) * 1e3, 3),
                         "p99_ms": round(float(np.quantile(lat[kind == kd], 0.99)) * 1e3, 3)}
                    for kd in sorted(set(kind.tolist()))}

        # kernel time per batch at the lowest rate (a separate replay: the
        # per-kernel timers cost host time, so the reported rates run without them)
        profiling.enable(True)
        profiling.reset()
        b0 = srv.stats()["batches"]
        srv.replay(q[:4000], ks[:4000], np.cumsum(arng.exponential(1.0 / rates[0], size=4000)),
                   nprobes=npb[:4000], filter_ids=fid[:4000])
        nb = max(1, srv.stats()["batches"] - b0)
        kernel_per_batch = {kk: round(v[0] / nb, 4) for kk in profiling.KERNELS for v in [profiling.get(kk)] if v[1]}
        profiling.enable(False)
        for ri, rate in enumerate(rates):
            arrivals = np.cumsum(arng.exponential(1.0 / rate, size=nreq))
            t = time.perf_counter()
            ids, dists, lat = srv.replay(q, ks, arrivals, nprobes=npb, filter_ids=fid)
            if ri == 0:
                err64 = fp64_error_l2(x, q, ids, dists)
            wall = time.perf_counter() - t
            lat_ms = np.sort(lat) * 1e3
            span = float(np.max(arrivals + lat))   # arrival schedule start to the last result
            out.append({"offered_qps": rate, "achieved_qps": round(nreq / span, 1),
                        "p50_ms": round(float(lat_ms[nreq // 2]), 3),
                        "p99_ms": round(float(lat_ms[int(0.99 * nreq)]), 3), "replay_call_s": round(wall, 4),
                        "by_kind": by_kind(lat)})
            log(f"served at {rate}/s: {out[-1]}")
        # each kind alone, one request at a time (the floor of its latency)
        solo = {}
        for kd in sorted(set(kind.tolist())):
            rows = np.flatnonzero(kind == kd)[:200]
            t_ms = []
            for i in rows:
                t = time.perf_counter()
                srv.result(srv.submit(q[i], int(ks[i]), nprobe=int(npb[i]),
                                      filter_id=int(fid[i]) if fid[i] >= 0 else -1))
                t_ms.append((time.perf_counter() - t) * 1e3)
            solo[kd] = {"p50_ms": round(float(np.median(t_ms)), 3), "p99_ms": round(float(np.quantile(t_ms, 0.99)), 3)}
        # a sample of requests against the same search run alone
        base = index.base
        for i in range(0, nreq, nreq // 64):
            base.nprobe = int(npb[i])
            allowed = np.flatnonzero(pool[filt[i]]) if filt[i] >= 0 else None
            si, _ = index.batch_query(q[i:i + 1], int(ks[i]), allowed=allowed)
            same &= bool(np.array_equal(si[0], ids[i, :ks[i]]))
        st = srv.stats()
    # the plain FP32 GPU batch path on the same rows: exact flat search, no tensor cores
    flat = qb.FlatIndex(d)
    flat.add(x)
    qb.set_tensor_filter(0)
    t = time.perf_counter()
    flat.batch_query(q[:1000], 10)
    fp32_qps = 1000 / (time.perf_counter() - t)
    qb.set_tensor_filter(1)
    del flat
    # the same IVF fast-scan + refine batch path with the tensor cores off (k 10, nprobe 64)
    index.base.nprobe = 64
    fp32_ivf = fp32_ivf_batch_qps(index, q[:10_000], 10)
    best = max(out, key=lambda r: r["achieved_qps"] if r["p99_ms"] <= 2.0 else 0)
    # sustained: the highest offered rate the server keeps up with (achieved >= 98 % of offered)
    kept = [r for r in out if r["achieved_qps"] >= 0.98 * r["offered_qps"]]
    sus = max(kept, key=lambda r: r["achieved_qps"]) if kept else None
    print(json.dumps({
        "metric": "served stream: highest sustained QPS (achieved >= 98% of offered) with p50/p99 per offered rate "
                  "(5M x 128 IVF16384-PQ64x4fs + refine kf10, mixed k / nprobe / filters)",
        "value": sus["achieved_qps"] if sus else None, "unit": "queries/s", "n_gpus": 1,
        "p50_ms_at_value": sus["p50_ms"] if sus else None, "p99_ms_at_value": sus["p99_ms"] if sus else None,
        "qps_at_p99_le_2ms": best["achieved_qps"] if best["p99_ms"] <= 2.0 else None,
        "steps": len(rates), "warmup": 1, "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8", "data": "synthetic",
        "config": {"workload": f"served_{n}x{d}_nl{nlist}_m{m}_kf{kf}", "requests_per_rate": nreq,
                   "k": [10, 100], "nprobe": "log-uniform 8..256", "filtered": 0.3, "selectivity": [0.01, 0.5],
                   "slots": 2, "max_batch": 512},
        "rates": out, "results_equal_solo_searches": same, "mean_batch": round(st["completed"] / st["batches"], 1),
        "rel_err_vs_fp64": err64,
        "at_lowest_rate": {"kernel_ms_per_batch": kernel_per_batch}, "one_at_a_time": solo,
        "plain_fp32_gpu_flat_qps": round(fp32_qps, 1),
        "fp32_ivf_batch_qps": {"qps": round(fp32_ivf, 1), "nq": 10_000, "k": 10, "nprobe": 64,
                               "path": "IVF fast-scan + refine batch, tensor cores off"},
        "batch_scan": batch}))
    return 0


def batch_scan_roofline(index, queries, m, nprobes, steps, warmup):
    """Device-resident batches of the served index at fixed nprobe, k 10: QPS
    and the scan's algorithmic code bytes per second against the HBM peak.
    The codes (n x m / 2 bytes: 160 MB at 5M x 64) exceed the 126 MB L2, so
    this is the scan's HBM-bound case; the L2 is flushed between steps."""
    import torch
    from qann_b200 import profiling
    dev = torch.device("cuda:0")
    nq, k = queries.shape[0], 10
    q_dev = torch.from_numpy(queries).to(dev)
    ids = torch.empty((nq, k), dtype=torch.int64, device=dev)
    dists = torch.empty((nq, k), dtype=torch.float32, device=dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream()
    peak, peak_src = measured_peak("hbm_gbs", 6650.0)
    base = index.base
    old = base.nprobe
    out = []
    for p in nprobes:
        base.nprobe = p
        for _ in range(warmup):
            index.search_device(q_dev.data_ptr(), nq, k, ids.data_ptr(), dists.data_ptr(), stream.cuda_stream)
        torch.cuda.synchronize()
        profiling.enable(True)
        profiling.reset()
        step_ms = []
        for _ in range(steps):
            flush.fill_(1.0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            index.search_device(q_dev.data_ptr(), nq, k, ids.data_ptr(), dists.data_ptr(), stream.cuda_stream)
            e1.record(stream)
            e1.synchronize()
            step_ms.append(e0.elapsed_time(e1))
        scan_ms, scan_n = profiling.get("scan")
        profiling.enable(False)
        per_launch = scan_ms / max(1, scan_n)
        alg = algorithmic_scan_bytes({"m": m}, index, queries, p, dev)
        achieved = alg / (per_launch / 1e3) / 1e9
        out.append({"nprobe": p, "nq": nq, "k": k, "qps": round(nq * steps / (sum(step_ms) / 1e3), 1),
                    "scan_launch_ms": round(per_launch, 4), "algorithmic_bytes_per_launch": alg,
                    "achieved_gbs": round(achieved, 1), "peak_gbs": peak, "frac": round(achieved / peak, 4),
                    "peak_source": peak_src, "scan_shape": qb_last_shape()})
        log(f"batch scan at nprobe {p}: {out[-1]}")
    base.nprobe = old
    return out


def qb_last_shape():
    import qann_b200 as qb
    so = qb.scan_options()["last_shape"]
    return {"warps": so // 1000, "lists_per_group": (so % 1000) // 10,
            "codes": {0: "global", 1: "staged", 2: "global, dense"}.get(so % 10)}


def reference_check(path, queries, k, op, ids, dists):
    """The reference library on the index this library built (loaded from
    its .qann) at the same operating point: QPS on the host cores (the CPU
    baseline) and whether its results equal this library's, query by query
    (ids, and distance bits)."""
    from oracle import ref
    if not ref.available():
        return None, None
    r = ref.load(path)
    r.k_factor, r.base.nprobe = op["k_factor"], op["nprobe"]
    cores = os.cpu_count() or 1
    ref.set_num_threads(cores)
    r.batch_query(queries[:200], k)   # warm-up
    t = time.perf_counter()
    r_ids, r_d = r.batch_query(queries, k)
    dt = time.perf_counter() - t
    id_diff = ~np.all(r_ids == ids, axis=1)
    d_diff = ~np.all(r_d.view(np.uint32) == dists.view(np.uint32), axis=1)
    cpu = {"value": round(queries.shape[0] / dt, 1), "unit": "queries/s", "cores": cores, "kind": "reference",
           "sample": f"all {queries.shape[0]} queries, one batch_query on {cores} threads, on the index this "
                     "library built (loaded from its .qann)"}
    cmp = {"results_equal_reference": bool(not id_diff.any() and not d_diff.any()),
           "queries_compared": int(queries.shape[0]), "queries_with_different_ids": int(id_diff.sum()),
           "queries_with_different_distance_bits": int(d_diff.sum())}
    return cpu, cmp


def fp64_error(base, queries, ids, dists, sample=2000):
    """Relative error of the returned re-ranked distances against FP64: the
    cosine distance 0.5 * |q/|q| - x/|x||^2 of the raw rows, in FP64."""
    s = min(sample, queries.shape[0])
    q = queries[:s].astype(np.float64)
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    x = base[ids[:s].ravel()].astype(np.float64).reshape(s, ids.shape[1], -1)
    x /= np.linalg.norm(x, axis=2, keepdims=True)
    d64 = 0.5 * ((q[:, None, :] - x) ** 2).sum(-1)
    err = np.abs(dists[:s].astype(np.float64) - d64) / np.maximum(np.abs(d64), 1e-30)
    return {"max": float(err.max()), "mean": float(err.mean()), "sample": f"{s} queries x {ids.shape[1]} results",
            "fp64": "0.5 * |q/|q| - x/|x||^2 of the raw rows"}


def fp64_error_l2(base, queries, ids, dists, sample=2000):
    """Relative error of served squared-L2 distances against FP64 over the
    first `sample` requests' results (ids of -1 past a request's own k are
    skipped)."""
    s = min(sample, queries.shape[0])
    ok = ids[:s] >= 0
    qi = np.nonzero(ok)[0]
    x = base[ids[:s][ok]].astype(np.float64)
    d64 = ((queries[:s].astype(np.float64)[qi] - x) ** 2).sum(-1)
    err = np.abs(dists[:s][ok].astype(np.float64) - d64) / np.maximum(np.abs(d64), 1e-30)
    return {"max": float(err.max()), "mean": float(err.mean()), "sample": f"{int(ok.sum())} results of {s} requests",
            "fp64": "|q - x|^2 of the raw rows"}


def index_matches_reference_build(path, cfg):
    """Whether the .qann this library wrote equals the reference library's
    own build of the same workload: the SHA-256 pinned in the golden
    fixtures (tests/golden/scale/, written by make_scale_golden.py)."""
    meta = ROOT / "tests" / "golden" / "scale" / "angular.json"
    if not meta.exists() or cfg is not FULL:
        return None
    want = json.loads(meta.read_text())["qann_sha256"]
    h = hashlib.sha256()
    with open(path, "rb") as f:
        for chunk in iter(lambda: f.read(1 << 24), b""):
            h.update(chunk)
    return h.hexdigest() == want


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="qann_b200", choices=["qann_b200", "reference"])
    ap.add_argument("--small", action="store_true", help="a quick functional run on a 10x smaller set")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-served", action="store_true", help="skip the continuous-batching server measurement")
    ap.add_argument("--nprobe", type=int, default=0, help="use this nprobe instead of the recall sweep (profiling)")
    ap.add_argument("--kf", type=int, default=0, help="use this k_factor instead of the recall sweep (profiling)")
    ap.add_argument("--tensor-scan", type=int, default=1, choices=[0, 1, 2],
                    help="fast-scan on the tensor cores: 0 never, 1 when it pays (default), 2 whenever it applies")
    ap.add_argument("--scan-shape", default="auto", choices=["auto", "global", "staged", "dense"],
                    help="fast-scan kernel shape: autotuned (default) or fixed (profiling)")
    ap.add_argument("--workload", default="angular", choices=["angular", "small", "flat", "train", "served"],
                    help="angular: the headline line; small / flat / train / served: the other configurations")
    args = ap.parse_args()
    if args.workload != "angular" and args.impl == "qann_b200":
        import torch
        torch.cuda.set_device(0)
        return {"small": small_workload, "flat": flat_workload, "train": train_workload,
                "served": served_workload}[args.workload](args)
    cfg = SMALL if args.small else FULL
    if args.impl == "reference":
        return reference_arm(args, cfg)

    import torch
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device(f"cuda:{local}")
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    def barrier():
        if dist is not None:
            dist.barrier()

    import qann_b200 as qb
    from qann_b200 import profiling

    if args.scan_shape != "auto":
        qb.set_scan_options(autotune=False, variant={"global": 0, "staged": 1, "dense": 2}[args.scan_shape])
    qb.set_tensor_scan(args.tensor_scan)
    base = mixture(cfg, 0, cfg["n"])
    queries = mixture(cfg, 1 + rank, cfg["nq"])
    index, path = build_or_load(cfg, base, rank, world, barrier)
    gt = ground_truth(cfg, base, queries, dev) if rank == 0 else None
    if args.nprobe or args.kf:
        op = {"k_factor": args.kf or cfg["kf"], "nprobe": args.nprobe or cfg["nprobes"][-1]}
        sel = {"sweep": {}, "chosen": op, "target_met": None, "configured": None}
    elif rank == 0:
        sel = sweep_operating_points(cfg, index, queries, gt, "qann_b200")
    barrier()
    if rank != 0 and not (args.nprobe or args.kf):
        sel = json.loads((CACHE / f"{tag(cfg)}_qann_b200_sweep2.json").read_text())
    op = sel["chosen"]
    nq, k = cfg["nq"], cfg["k"]

    # ---- device-resident steps ----
    q_dev = torch.from_numpy(queries).to(dev)
    out_ids = torch.empty((nq, k), dtype=torch.int64, device=dev)
    out_d = torch.empty((nq, k), dtype=torch.float32, device=dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream()

    # the configured k_factor's own point (below the target on this set)
    own = None
    if sel.get("configured") and sel["configured"]["k_factor"] != op["k_factor"]:
        c = sel["configured"]
        index.k_factor, index.base.nprobe = c["k_factor"], c["nprobe"]
        profiling.enable(True)   # (its scan time, for the same roofline at this point)
        profiling.reset()
        times, _, _ = device_steps(index, q_dev, nq, k, max(3, args.steps // 5), args.warmup, flush)
        own_scan_ms, own_scan_n = profiling.get("scan")
        profiling.enable(False)
        t = time.perf_counter()
        index.batch_query(queries, k)
        own = {"k_factor": c["k_factor"], "nprobe": c["nprobe"], "recall@10": c["recall"],
               "target_met": c["target_met"], "qps": round(nq * len(times) / (sum(times) / 1e3), 1),
               "e2e_qps": round(nq / (time.perf_counter() - t), 1),
               "scan_launch_ms": round(own_scan_ms / max(1, own_scan_n), 4)}

    index.k_factor, index.base.nprobe = op["k_factor"], op["nprobe"]
    for _ in range(args.warmup):
        index.search_device(q_dev.data_ptr(), nq, k, out_ids.data_ptr(), out_d.data_ptr(), stream.cuda_stream)
    torch.cuda.synchronize()
    profiling.enable(True)
    profiling.reset()
    coarse0 = qb.tensor_filter_counts()
    tscan0 = qb.tensor_scan_counts()
    launches0 = profiling.launch_count()
    step_ms = []
    barrier()
    with Clocks(local) as clk:
        for _ in range(args.steps):
            flush.fill_(1.0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            index.search_device(q_dev.data_ptr(), nq, k, out_ids.data_ptr(), out_d.data_ptr(), stream.cuda_stream)
            e1.record(stream)
            e1.synchronize()
            step_ms.append(e0.elapsed_time(e1))
    torch.cuda.synchronize()
    barrier()
    launches = profiling.launch_count() - launches0
    coarse1 = qb.tensor_filter_counts()
    profiling.enable(False)
    cq = coarse1["coarse_queries"] - coarse0["coarse_queries"]
    coarse = {"path": "f16 tensor-core estimates + exact FP32 recheck" if cq else "exact FP32",
              "queries": cq, "redone_exactly": coarse1["coarse_redone"] - coarse0["coarse_redone"],
              "lists_rescored_per_query": round((coarse1["coarse_candidates"] - coarse0["coarse_candidates"]) / cq, 1)
              if cq else None}
    tscan1 = qb.tensor_scan_counts()
    # the fast-scan stage per step: the query-major kernel (all probes, or the
    # first wave of the tensor-core path) and the tensor-core wave with its
    # preparation and final cut
    stage = {kname: profiling.get(kname) for kname in ("scan", "tscan_prep", "tscan", "tscan_final")}
    scan_ms = sum(v[0] for v in stage.values())
    scan_n = args.steps
    kernel_ms = {kname: profiling.get(kname) for kname in profiling.KERNELS}
    tensor_scan = {"used": tscan1["calls"] > tscan0["calls"], "searches": tscan1["calls"] - tscan0["calls"],
                   "queries_redone": tscan1["redone"] - tscan0["redone"],
                   "work_per_search": {kk: round((tscan1[kk] - tscan0[kk]) / max(1, tscan1["calls"] - tscan0["calls"]))
                                       for kk in ("pairs", "pairs_kept", "units", "tiles", "luts_live",
                                                  "luts_hopeless", "candidates")},
                   "ms_per_step": {kname: round(v[0] / args.steps, 4) for kname, v in stage.items() if v[1]}}
    total_ms = float(sum(step_ms))
    if dist is not None:
        t = torch.tensor([total_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    value = nq * args.steps * world / (total_ms / 1e3)
    got = out_ids.cpu().numpy()
    got_d = out_d.cpu().numpy()

    # ---- end to end through the public API, host arrays ----
    e2e_times = []
    for _ in range(max(3, args.steps // 5)):
        torch.cuda.synchronize()
        t = time.perf_counter()
        ids_h, d_h = index.batch_query(queries, k)
        e2e_times.append(time.perf_counter() - t)
    e2e_qps = nq * len(e2e_times) / sum(e2e_times)
    if dist is not None:
        t = torch.tensor([sum(e2e_times)], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_qps = nq * len(e2e_times) * world / float(t.item())

    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return 0

    so = qb.scan_options()["last_shape"]
    scan_shape = {"warps": so // 1000, "lists_per_group": (so % 1000) // 10,
                  "codes": {0: "global", 1: "staged", 2: "global, dense"}[so % 10],
                  "autotuned": bool(qb.scan_options()["autotune"])}
    rec = recall(got, gt)
    assert np.array_equal(got, ids_h) and got_d.tobytes() == d_h.tobytes(), \
        "device-resident and host-API results differ"
    alg_bytes = algorithmic_scan_bytes(cfg, index, queries, op["nprobe"], dev)
    per_launch_ms = scan_ms / max(1, scan_n)
    achieved = alg_bytes / (per_launch_ms / 1e3) / 1e9
    peak, peak_src = measured_peak("hbm_gbs", 6650.0)
    if own is not None and own["nprobe"] == op["nprobe"] and own["scan_launch_ms"] > 0:
        # the configured k_factor scans the same lists: the same algorithmic bytes
        own_gbs = alg_bytes / (own["scan_launch_ms"] / 1e3) / 1e9
        own["scan_roofline"] = {"achieved": round(own_gbs, 1), "peak": peak, "unit": "GB/s",
                                "frac": round(own_gbs / peak, 4), "peak_source": peak_src}
    traffic = scan_traffic()
    serving = None
    if not args.no_served:
        serving = served(index, queries, k, op["nprobe"], ids_h)
        serving["k_factor"] = op["k_factor"]
        fp32 = plain_fp32_qps(base, queries, k, qb.Metric.Cosine)
        serving["plain_fp32_gpu_batch_qps"] = round(fp32, 1)
        ivf32 = fp32_ivf_batch_qps(index, queries, k)
        serving["fp32_ivf_batch_qps"] = round(ivf32, 1)
        if serving["best_qps_at_p99_le_2ms"]:
            serving["served_over_plain_fp32"] = round(serving["best_qps_at_p99_le_2ms"] / fp32, 1)
            serving["served_over_fp32_ivf_batch"] = round(serving["best_qps_at_p99_le_2ms"] / ivf32, 2)
    cpu, cmp = (None, None) if (args.no_cpu_baseline or world > 1) else \
        reference_check(path, queries, k, op, ids_h, d_h)
    clocks = clk.summary()
    alu = alu_roofline(alg_bytes, per_launch_ms, clocks, dev)
    srt = sorted(step_ms)
    line = {
        "metric": METRIC,
        "value": round(value, 1), "unit": "queries/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(total_ms / args.steps, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8", "data": "synthetic",
        "config": {"workload": tag(cfg), "nq": nq, "k": k, "k_factor": op["k_factor"], "nprobe": op["nprobe"],
                   "recall@10": round(rec, 4), "recall_target": cfg["target"], "target_met": sel.get("target_met"),
                   "sweep": sel["sweep"], "l2": "flushed between steps (256 MB write)",
                   "parallelism": f"replicas x{world}", "batch_latency_ms": {
                       "p50": round(srt[len(srt) // 2], 4), "p99": round(srt[min(len(srt) - 1, int(0.99 * len(srt)))], 4)},
                   "kernel_ms_total": {kk: round(v[0], 3) for kk, v in kernel_ms.items() if v[1]},
                   "scan_shape": scan_shape, "coarse": coarse,
                   "index_equals_reference_build": index_matches_reference_build(path, cfg),
                   "configured_k_factor": own},
        "reference_parity": cmp,
        "rel_err_vs_fp64": fp64_error(base, queries, ids_h, d_h),
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "traffic": traffic, "peak_source": peak_src,
                     "kernel": "fast-scan stage (k_scan; with the tensor-core path k_scan on the first 16 probes "
                               "+ k_tscan on the rest)" if tensor_scan["used"] else "k_scan",
                     "algorithmic_bytes_per_launch": alg_bytes, "launch_ms": round(per_launch_ms, 4),
                     "note": "algorithmic bytes count every probed list's codes; the codes (33 MB) stay in L2 and "
                             "lists that cannot beat a query's bound are skipped, so this is not a DRAM rate"},
        "alu_roofline": alu,
        "tensor_scan": tensor_scan,
        "e2e": {"value": round(e2e_qps, 1), "unit": "queries/s", "h2d_bytes_per_step": nq * cfg["d"] * 4,
                "d2h_bytes_per_step": nq * k * 12, "timing": "host wall clock around the blocking batch_query"},
        "gpu_launches": launches, "clocks": clocks, "cpu_baseline": cpu, "served": serving,
    }
    print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
