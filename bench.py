#!/usr/bin/env python3
"""Benchmark of the B200 symmetric-deletion neighbour search.

One step = one full nearest-neighbour search (pack, variant generation, key grouping,
candidate emission, pair dedup and sort, verification, compaction) over the workload's
sequences, inputs resident in HBM (`value`); `e2e` is the same search through the C ABI's
host-buffer entry point (xtn_context_perform) with the host->device copy of the sequences
and the device->host copy of the result pairs inside the timed region.

Workload (default): 10,000,000 synthetic CDR3 sequences, 20% in mutant clusters, 2% exact
duplicates, Levenshtein d = 2, seeded generator (xtn.synth_clusters). The 1,000,000-sequence
workload of the same generator is measured too and reported under "extra_workloads".

The reference arm (--impl reference) times the reference's own library entry point,
xtn_perform, built from its sources for sm_100a (oracle/_ref/ref_perform), as a call in one
process after a warm-up call, on workload files written by a separate generator process.

  python bench.py [--gpus N --steps K --warmup W] [--impl ours|reference] [--workload NAME]

With N > 1 (under torchrun) every rank runs an independent replica of the workload on its
own GPU (the search does not shard); `value` is the sum over ranks divided by the slowest
rank's time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "xt-neighbor_b200")
sys.path.insert(0, PKG)

# expect_out: the output length on the workload, which the reference binary's and this
# build's outputs share byte for byte (tests/test_gpu_reference_full_size.py); the reference
# arm compares its own count with it
WORKLOADS = {
    "nn_1m_leven_d2": dict(kind="clusters", n=1_000_000, d=2, measure=0, seed=20241, expect_out=314_584),
    "nn_10k_leven_d1": dict(kind="mutants", n=10_000, d=1, measure=0, seed=20240),
    "nn_10m_leven_d2": dict(kind="clusters", n=10_000_000, d=2, measure=0, seed=20242, expect_out=3_182_141),
    "nn_10m_hamming_d2": dict(kind="clusters", n=10_000_000, d=2, measure=1, seed=20242, expect_out=890_373),
    # repertoire overlap: 64 repertoires, sizes log-uniform in [1e4, 2e6] (23.9M rows with this
    # seed), 5% of each drawn from a shared pool, power-law duplicate counts; Levenshtein d = 1
    "overlap_64rep_leven_d1": dict(kind="repertoires", n_reps=64, min=1e4, max=2e6, shared=0.05, d=1, measure=0,
                                   seed=20244),
}
# serving: resident d = 2 index over 5M generator sequences; query requests drawn from a further
# 1M rows of the same generator run (rows are shuffled, so clusters span index and pool)
SERVE_WORKLOADS = {
    "serve_5m_d2": dict(n_index=5_000_000, n_pool=1_000_000, seed=20245, rates=(10, 100, 1000), seconds=3.0,
                        max_size=100_000, p_d1=0.7),
}
DEFAULT_WORKLOAD = "nn_10m_leven_d2"
EXTRA_WORKLOADS = {"nn_10m_leven_d2": ["nn_1m_leven_d2"]}
SYNTH_CLI = os.path.join(PKG, "bin", "xtn_synth")
REF_PERFORM = os.path.join(ROOT, "oracle", "_ref", "ref_perform")
# the reference arm stops repeating the search once its timed calls have taken this long
REF_MAX_SECONDS = 60.0
METRIC = "seqs/s (symmetric-deletion NN search, whole job)"
L2_FLUSH_BYTES = 256 << 20


def gen_workload(w):
    """(chars, offsets, info or None, repertoire sizes or None)."""
    import xtn

    if w["kind"] == "repertoires":
        return xtn.synth_repertoires(w["seed"], w["n_reps"], w["min"], w["max"], w["shared"])
    if w["kind"] == "clusters":
        return (*xtn.synth_clusters(w["seed"], w["n"], 0.20, 0.02), None, None)
    return (*xtn.synth_mutants(w["seed"], w["n"], 0.10), None, None)


def measured_peak_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            j = json.load(f)
        return float(j["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """SM clock and clock-event reasons of one GPU while the timed steps run: NVML read-only
    queries every 10 ms from a thread (nvidia-smi every 200 ms when NVML is unavailable)."""

    REASONS = {0x8: "hw_slowdown", 0x40: "hw_thermal_slowdown", 0x20: "sw_thermal_slowdown", 0x4: "sw_power_cap",
               0x80: "hw_power_brake_slowdown"}
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int, period: float = 0.01):
        self.device = device
        self.period = period
        self.sm, self.reasons, self.max_mhz = [], set(), None
        self.thread = self.proc = self.path = None
        self.stop_flag = False

    def _nvml_handle(self):
        import pynvml
        import torch

        pynvml.nvmlInit()
        try:
            uuid = str(torch.cuda.get_device_properties(self.device).uuid)
            return pynvml, pynvml.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.device)

    def start(self):
        import threading

        try:
            nv, h = self._nvml_handle()
            self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))

            def loop():
                while not self.stop_flag:
                    self.sm.append(float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)))
                    r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                    self.reasons.update(name for bit, name in self.REASONS.items() if r & bit)
                    time.sleep(self.period)

            self.thread = threading.Thread(target=loop, daemon=True)
            self.thread.start()
            return
        except Exception:
            self.thread = None
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if self.thread:
            self.stop_flag = True
            self.thread.join(timeout=5)
            return {"sm_mhz": statistics.median(self.sm) if self.sm else None, "sm_max_mhz": self.max_mhz,
                    "reasons": sorted(self.reasons), "samples": len(self.sm), "source": "nvml, 10 ms"}
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["clock sampling unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    mx.append(float(parts[2]))
                except ValueError:
                    continue
                for nm, v in zip(names, parts[5:9]):
                    if v.lower() == "active":
                        reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm), "source": "nvidia-smi, 200 ms"}


def algorithmic_bytes(kernel: str, st: dict, n: int, n_chars: int) -> float | None:
    """Compulsory HBM bytes of all launches of `kernel` in one step (divided by the launch count
    by the caller). V = deletion variants, P = candidate pairs, n = sequences."""
    V, Pc = st["n_variants"], st["n_candidates"]
    if kernel == "bucket_scatter":
        # each 8-byte record written once; per sequence its 19-word key table (152 B), run info,
        # variant and task offsets (8 B each) and key length (1 B) read once
        return 8.0 * V + 177.0 * n
    if kernel == "bucket_gen":
        # two-pass first level, generation: each 8-byte record written once; per sequence the
        # same 177 bytes read as the one-pass scatter
        return 8.0 * V + 177.0 * n
    if kernel == "bucket_partition":
        return 16.0 * V  # each record read once and written once
    if kernel == "bucket_group":
        return 8.0 * V + 8.0 * Pc  # each record read once; candidate pairs written
    if kernel == "bucket_split":
        return 16.0 * V  # records of split buckets read once and written once
    if kernel == "bucket_count":
        return 161.0 * n  # key table (152 B), run info (8 B) and key length (1 B) of each sequence
    if kernel == "key_sort_downsweep":
        return 16.0 * V  # sort engine: read + write each 8-byte record once
    if kernel == "key_sort_upsweep":
        return 8.0 * V
    if kernel == "gen":
        return 8.0 * V + 25.0 * n
    if kernel == "find_groups":
        return 8.0 * V
    U = st.get("n_unique") or Pc  # pairs sorted and verified (distinct ones after the hash set)
    if kernel == "pair_dedup":
        return 8.0 * Pc + 16.0 * U  # candidates read; each distinct pair written to its slot and the list
    if kernel == "pair_sort_pass":
        passes = -(-2 * st["id_bits"] // 8)
        return 16.0 * U * passes  # each pass reads and writes every key
    if kernel == "verify":
        return 10.0 * U + 2.0 * (n_chars / max(n, 1) + 8.0) * U
    return None


def serve_trace(ix, pool_c, pool_o, w, rate, rng, slots=2):
    """One Poisson trace against a resident index: `rate` req/s for w["seconds"] seconds,
    request sizes log-uniform in [1, max_size], d = 1 with probability p_d1 else 2,
    Levenshtein. Latency = completion - arrival of each request (host clock, the request's
    pairs delivered to the host)."""
    import numpy as np

    n_pool = len(pool_o) - 1
    n_req = max(5, int(rate * w["seconds"]))
    arrivals = np.cumsum(rng.exponential(1.0 / rate, n_req))
    sizes = np.minimum(np.exp(rng.uniform(0, np.log(w["max_size"]), n_req)).astype(np.int64), w["max_size"])
    sizes = np.maximum(sizes, 1)
    dists = np.where(rng.random(n_req) < w["p_d1"], 1, 2)
    reqs = []
    for k in range(n_req):
        a = int(rng.integers(0, n_pool - sizes[k] + 1))
        o = (pool_o[a : a + sizes[k] + 1] - pool_o[a]).astype(np.uint32)
        reqs.append((pool_c[pool_o[a] : pool_o[a + sizes[k]]], o, int(dists[k]), 0, float(arrivals[k])))
    # warm-up, untimed: the three largest requests of each distance
    warm = [reqs[k] for dd in (1, 2) for k in np.argsort(-sizes * (dists == dd))[:3]]
    ix.serve(warm, realtime=False, keep_results=False, slots=slots)
    stats, _ = ix.serve(reqs, realtime=True, keep_results=False, slots=slots)
    lat = np.array([(st["done_s"] - t) * 1e3 for st, (_, _, _, _, t) in zip(stats, reqs)])
    span = max(st["done_s"] for st in stats) - float(arrivals[0])
    small_d1 = np.array([l for l, (_, o, d, _, _) in zip(lat, reqs) if d == 1 and len(o) - 1 <= 1000])
    return {
        "rate_req_per_s": rate,
        "slots": slots,
        "requests": n_req,
        "p50_ms": float(np.percentile(lat, 50)),
        "p99_ms": float(np.percentile(lat, 99)),
        "p50_ms_d1": float(np.percentile(lat[dists == 1], 50)),
        "p99_ms_d1": float(np.percentile(lat[dists == 1], 99)),
        "p99_ms_d2": float(np.percentile(lat[dists == 2], 99)) if (dists == 2).any() else None,
        "p99_ms_d1_le_1k_seqs": float(np.percentile(small_d1, 99)) if len(small_d1) else None,
        "seqs_per_s": float(sizes.sum() / span),
        "batches": len({st["batch"] for st in stats}),
        "pairs": int(sum(st["n_out"] for st in stats)),
        "slowest": [{"seqs": int(sizes[k]), "d": int(dists[k]), "queue_ms": (stats[k]["admitted_s"] - arrivals[k]) * 1e3,
                     "service_ms": (stats[k]["done_s"] - stats[k]["admitted_s"]) * 1e3, "batch": stats[k]["batch"]}
                    for k in np.argsort(-lat)[:5]],
    }


def serve_setup(w, device):
    """The resident index over the first n_index generator rows and the request pool."""
    import numpy as np

    import xtn

    chars, offs = xtn.synth_clusters(w["seed"], w["n_index"] + w["n_pool"], 0.20, 0.02)
    ni = w["n_index"]
    t0 = time.perf_counter()
    ix = xtn.Index(chars[: offs[ni]], offs[: ni + 1], max_distance=2, device=device)
    build_wall = time.perf_counter() - t0
    pool_c, pool_o = chars[offs[ni] :], (offs[ni:] - offs[ni]).astype(np.uint32)
    return ix, pool_c, pool_o, build_wall


def run_serve(args, w):
    """Serving loop on a resident deletion index (xtn_index_serve) at each rate of the workload."""
    import numpy as np
    import torch

    world, rank, local = dist_setup()
    if rank != 0:
        return None
    torch.cuda.set_device(local)
    ix, pool_c, pool_o, build_wall = serve_setup(w, local)
    info = ix.info()
    rng = np.random.default_rng(w["seed"] + 1)
    sampler = ClockSampler(local)
    sampler.start()
    per_rate = {str(rate): serve_trace(ix, pool_c, pool_o, w, rate, rng) for rate in w["rates"]}
    clocks = sampler.stop()
    ix.close()
    top = per_rate[str(max(w["rates"]))]
    return {
        "metric": "served query latency p99 (resident 5M-sequence d=2 index), ms",
        "value": per_rate[str(w["rates"][len(w["rates"]) // 2])]["p99_ms"],
        "unit": "ms",
        "n_gpus": 1,
        "steps": len(w["rates"]),
        "warmup": 1,
        "ms_per_step": None,
        "higher_is_better": False,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "u64",
        "data": "synthetic (seeded CDR3 generator)",
        "config": {"workload": args.workload, "index_seqs": w["n_index"], "index_max_distance": 2,
                   "request_sizes": f"log-uniform 1..{w['max_size']}", "p_d1": w["p_d1"],
                   "rates_req_per_s": list(w["rates"]), "seconds_per_rate": w["seconds"],
                   "value_is": f"p99 at {w['rates'][len(w['rates']) // 2]} req/s"},
        "per_rate": per_rate,
        "seqs_per_s_at_top_rate": top["seqs_per_s"],
        "index": {"records": info["n_records"], "bytes": info["bytes"], "directory_bits": info["directory_bits"],
                  "build_ms_device": info["ms_build"], "build_s_wall": build_wall},
        "clocks": clocks,
    }


def serving_line(local):
    """The serving configuration at one rate (100 req/s, 3 s), for the default bench line."""
    import numpy as np

    w = SERVE_WORKLOADS["serve_5m_d2"]
    ix, pool_c, pool_o, build_wall = serve_setup(w, local)
    out = serve_trace(ix, pool_c, pool_o, w, 100, np.random.default_rng(w["seed"] + 1))
    out["index_seqs"] = w["n_index"]
    out["index_build_ms_device"] = ix.info()["ms_build"]
    ix.close()
    return out


def ncu_traffic(kernel: str, workload: str):
    """DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum) of `kernel` on
    `workload`, from the committed ncu summary profiles/<kernel>_<workload>.md (its line
    `traffic_bytes_per_launch: N`), or None."""
    path = os.path.join(ROOT, "profiles", f"{kernel}_{workload}.md")
    try:
        with open(path) as f:
            for line in f:
                if line.strip().startswith("traffic_bytes_per_launch:"):
                    return float(line.split(":", 1)[1].strip())
    except OSError:
        pass
    return None


def reduce_max(values, pg, device):
    """Element-wise maximum over the ranks of a process group (None: one process). Every rank
    calls it with the same number of values; the replicas' step time is the slowest rank's."""
    if pg is None:
        return [float(v) for v in values]
    import torch

    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return [float(x) for x in t.cpu()]


def replica_throughput(units_per_rank: int, world: int, ms_max: float) -> float:
    """Whole-job throughput of `world` independent replicas: all ranks' units over the slowest
    rank's time."""
    return world * units_per_rank / (ms_max / 1e3)


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def run_ours(args, w):
    import datetime

    import numpy as np
    import torch

    import xtn

    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
        pg = dist
    chars, offs, info, reps = gen_workload(w)
    overlap = info is not None
    n = len(offs) - 1
    opts = {k: int(v) for k, v in (o.split("=", 1) for o in args.opt)}
    opts.setdefault("engine", 1 if args.engine == "sort" else 0)
    ctx = xtn.Context(local, **opts)
    ctx.set_profiling(True)
    d_chars = torch.from_numpy(chars).cuda()
    d_offs = torch.from_numpy(offs.view(np.int32)).cuda()
    d_info = torch.from_numpy(np.ascontiguousarray(info)).cuda() if overlap else None
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")
    ext = torch.cuda.ExternalStream(ctx.stream())
    torch.cuda.synchronize()
    tuned = None
    if args.autotune and not overlap:  # outside the timed region
        tuned = ctx.autotune(d_chars.data_ptr(), d_offs.data_ptr(), n, w["d"], w["measure"])

    def step():
        if overlap:
            return ctx.overlap_device(d_chars.data_ptr(), d_offs.data_ptr(), n, d_info.data_ptr(), len(reps), w["d"],
                                      w["measure"])
        return ctx.nn_device(d_chars.data_ptr(), d_offs.data_ptr(), n, w["d"], w["measure"])

    for _ in range(args.warmup):
        step()
    # one more step with every launch bracketed by events, outside the timed region: the
    # per-kernel breakdown; the timed steps bracket only the dominant kernel (for the roofline)
    flush.zero_()
    torch.cuda.synchronize()
    step()
    breakdown = ctx.kernel_times()
    dom_name = max(breakdown.items(), key=lambda kv: kv[1][0])[0]
    ctx.set_profiling(True, only=dom_name)
    sampler = ClockSampler(local)
    if rank == 0:
        sampler.start()
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    times, ktimes, launches, n_out, stats = [], {}, 0, 0, None
    for _ in range(args.steps):
        flush.zero_()  # L2 flush between steps (outside the timed window)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(ext)
        n_out = step()
        e1.record(ext)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
        for k, (ms, cnt) in ctx.kernel_times().items():
            a, b = ktimes.get(k, (0.0, 0))
            ktimes[k] = (a + ms, b + cnt)
        stats = ctx.stats()
        launches += stats["n_launches"]
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    clocks = sampler.stop() if rank == 0 else None
    ms_step = sum(times) / len(times)

    # end to end through the host-buffer entry point: H2D + search + D2H each step
    pin_c = torch.from_numpy(chars).pin_memory()
    pin_o = torch.from_numpy(offs.view(np.int32)).pin_memory()
    hc, ho = pin_c.numpy(), pin_o.numpy().view(np.uint32)
    e2e_times = []
    res = None
    for i in range(args.warmup + args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(ext)
        if overlap:
            res = ctx.perform(hc, ho, distance=w["d"], measure=w["measure"], info=info, n_reps=len(reps))
        else:
            res = ctx.perform(hc, ho, distance=w["d"], measure=w["measure"])
        e1.record(ext)
        e1.synchronize()
        if i >= args.warmup:
            e2e_times.append(e0.elapsed_time(e1))
    e2e_ms = sum(e2e_times) / len(e2e_times)
    assert len(res.pairs) == n_out

    ms_step, e2e_ms = reduce_max([ms_step, e2e_ms], pg, "cuda")
    if rank != 0:
        ctx.close()
        if pg:
            pg.destroy_process_group()
        return None

    peak, peak_kind = measured_peak_hbm()
    dom_ms, dom_launches = ktimes[dom_name]
    per_launch_ms = dom_ms / dom_launches
    launches_per_step = dom_launches / args.steps
    ab = algorithmic_bytes(dom_name, stats, n, len(chars))
    achieved = (ab / launches_per_step) / (per_launch_ms / 1e3) / 1e9 if ab else None
    total_kernel_ms = sum(v[0] for v in breakdown.values())
    line = {
        "metric": METRIC,
        "value": replica_throughput(n, world, ms_step),
        "unit": "seqs/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_step,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "u64",
        "data": "synthetic (seeded CDR3 generator)",
        "config": {
            "workload": args.workload,
            "n_seqs": n,
            "distance": w["d"],
            "measure": "hamming" if w["measure"] else "leven",
            "mode": "overlap" if overlap else "nn",
            "repertoires": len(reps) if overlap else None,
            "parallelism": f"replicas x{world}",
            "engine": args.engine,
            "options": {o.split("=", 1)[0]: int(o.split("=", 1)[1]) for o in args.opt},
            "l2": "flushed between steps (256 MiB write)",
            "autotuned": tuned,
        },
        "pairs_per_s": None if overlap else world * n_out / (ms_step / 1e3),
        "verified_pairs": stats["n_verified_pairs"] if overlap else n_out,
        "output_entries": n_out,
        "counts": {k: stats[k] for k in ("n_variants", "n_groups", "n_fallback", "n_candidates", "n_unique", "n_out")},
        "e2e": {
            "value": replica_throughput(n, world, e2e_ms),
            "unit": "seqs/s",
            "ms_per_step": e2e_ms,
            "h2d_bytes_per_step": int(len(chars) + 4 * len(offs) + (12 * n if overlap else 0)),
            "d2h_bytes_per_step": int(n_out * (16 if overlap else 9)),
        },
        "gpu_launches": int(launches),
        "roofline": {
            "kernel": dom_name,
            "bound": "hbm",
            "achieved": achieved,
            "peak": peak,
            "peak_kind": peak_kind,
            "unit": "GB/s",
            "frac": (achieved / peak) if achieved else None,
            "traffic": ncu_traffic(dom_name, args.workload),
            "algorithmic_bytes_per_launch": (ab / launches_per_step) if ab else None,
            "launch_ms": per_launch_ms,
            "share_of_kernel_time": breakdown[dom_name][0] / total_kernel_ms,
        },
        # one profiled step outside the timed region (every launch bracketed by events)
        "kernels_ms_per_step": {k: round(v[0], 4) for k, v in sorted(breakdown.items(), key=lambda kv: -kv[1][0])},
        "clocks": clocks,
    }
    # the plain form (above: one launch sequence per search, sizes read back between stages)
    # against the batched/persistent form (the search captured once into a CUDA graph and
    # replayed, every size read on the device), same inputs, same timing
    if not args.no_forms:
        line["forms"] = measure_forms(ctx, w, n, d_chars, d_offs, args, flush, ext, ms_step, n_out,
                                      (d_info, len(reps)) if overlap else None)
    extras = {}
    for name in ([] if args.no_extra else EXTRA_WORKLOADS.get(args.workload, [])):
        extras[name] = measure_extra(ctx, WORKLOADS[name], args, flush, ext)
    if extras:
        line["extra_workloads"] = extras
    if world == 1 and not args.no_serving and not overlap:
        line["serving"] = serving_line(local)
    if world == 1 and not args.no_cli:
        line["cli_process"] = cli_process(args, w, n)
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(chars, offs, w, info, reps)
    ctx.close()
    if pg:
        pg.destroy_process_group()
    return line


def measure_forms(ctx, w, n, d_chars, d_offs, args, flush, ext, plain_ms, plain_out, overlap=None):
    """The plain form (the headline's search: one launch sequence per search that reads sizes
    back between its stages, default shapes) against the batched/persistent form (shapes from
    the autotuner, which also picks between the plain and the CUDA-graph form; the graph form is
    the whole search captured once and replayed with every size read on the device), same
    inputs and timing, in a second context. Overlap mode (overlap = (device info, repertoires)):
    the graph form of the whole overlap sequence, default shapes."""
    import torch

    import xtn

    ctx.set_profiling(False)
    if overlap:
        b = xtn.Context(ctx_device(ctx), graph=1)
        report = "graph=1 (overlap mode: string merge, diagonal, search, cross term and matrix in one graph)"
        d_info, R = overlap
        fn = lambda: b.overlap_device(d_chars.data_ptr(), d_offs.data_ptr(), n, d_info.data_ptr(), R, w["d"],
                                      w["measure"])
    else:
        b = xtn.Context(ctx_device(ctx))
        report = b.autotune(d_chars.data_ptr(), d_offs.data_ptr(), n, w["d"], w["measure"], repeats=2)
        fn = lambda: b.nn_device(d_chars.data_ptr(), d_offs.data_ptr(), n, w["d"], w["measure"])
    times, out = [], None
    for i in range(1 + args.warmup + args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        bext = torch.cuda.ExternalStream(b.stream())
        e0.record(bext)
        out = fn()
        e1.record(bext)
        e1.synchronize()
        if i > args.warmup:
            times.append(e0.elapsed_time(e1))
    st = b.stats()
    b.close()
    assert out == plain_out, "batched and plain forms differ in output length"
    g = sum(times) / len(times)
    return {"plain": {"value": n / (plain_ms / 1e3), "ms_per_step": plain_ms,
                      "what": "one launch sequence per search, four host reads of sizes, default shapes"},
            "batched": {"value": n / (g / 1e3), "ms_per_step": g, "launches": st["n_launches"],
                        "autotuned": report,
                        "what": "autotuned shapes; with graph=1 the whole search captured once in a CUDA graph, "
                                "sizes read on the device, grouping by persistent CTAs, one host read per search"},
            "batched_over_plain": plain_ms / g}


def ctx_device(ctx):
    import torch

    return torch.cuda.current_device()


def measure_extra(ctx, w, args, flush, ext):
    """A further nearest-neighbour workload on the same context, timed like the headline:
    device-resident search (`value`) and host-buffer search with both copies (`e2e`)."""
    import numpy as np
    import torch

    chars, offs, _, _ = gen_workload(w)
    n = len(offs) - 1
    d_chars = torch.from_numpy(chars).cuda()
    d_offs = torch.from_numpy(offs.view(np.int32)).cuda()
    torch.cuda.synchronize()
    ctx.set_profiling(False)

    def timed(fn, count):
        out, ms = None, []
        for _ in range(count):
            flush.zero_()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(ext)
            out = fn()
            e1.record(ext)
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
        return out, ms

    dev = lambda: ctx.nn_device(d_chars.data_ptr(), d_offs.data_ptr(), n, w["d"], w["measure"])
    timed(dev, args.warmup)
    n_out, ms = timed(dev, args.steps)
    pin_c = torch.from_numpy(chars).pin_memory()
    pin_o = torch.from_numpy(offs.view(np.int32)).pin_memory()
    hc, ho = pin_c.numpy(), pin_o.numpy().view(np.uint32)
    host = lambda: ctx.perform(hc, ho, distance=w["d"], measure=w["measure"])
    timed(host, args.warmup)
    res, ems = timed(host, args.steps)
    assert len(res.pairs) == n_out
    st = ctx.stats()
    m, em = sum(ms) / len(ms), sum(ems) / len(ems)
    return {"value": n / (m / 1e3), "unit": "seqs/s", "ms_per_step": m, "steps": args.steps,
            "n_seqs": n, "distance": w["d"], "measure": "hamming" if w["measure"] else "leven",
            "pairs_per_s": n_out / (m / 1e3), "output_entries": n_out,
            "counts": {k: st[k] for k in ("n_variants", "n_candidates", "n_unique", "n_out")},
            "e2e": {"value": n / (em / 1e3), "unit": "seqs/s", "ms_per_step": em,
                    "h2d_bytes_per_step": int(len(chars) + 4 * len(offs)), "d2h_bytes_per_step": int(n_out * 9)}}


def cpu_baseline(chars, offs, w, info=None, reps=None, max_seqs=2_000_000):
    """The CPU oracle (multithreaded restatement of the reference algorithm) on a bounded sample
    of the workload: its first max_seqs sequences in nearest-neighbour mode (the whole input
    when it is smaller), the leading repertoires up to about max_seqs rows in overlap mode."""
    import numpy as np

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc

    n = len(offs) - 1
    t0 = time.perf_counter()
    if info is None:
        k = min(n, max_seqs)
        sub_o = offs[: k + 1]
        orc.nn_search(chars[: sub_o[-1]], sub_o, w["d"], w["measure"])
        sample = k
        what = (f"whole workload ({n} seqs), one search" if k == n else
                f"first {k} of the workload's {n} sequences, one search")
    else:
        k = max(1, int(np.searchsorted(np.cumsum(reps), max_seqs, side="right")))
        rows = int(np.sum(reps[:k]))
        sub_info = np.ascontiguousarray(info[:rows])
        orc.overlap_search(chars[: offs[rows]], offs[: rows + 1], sub_info, w["d"], w["measure"])
        sample, what = rows, f"first {k} repertoires ({rows} rows), one overlap search"
    dt = time.perf_counter() - t0
    return {
        "value": sample / dt,
        "unit": "seqs/s",
        "cores": orc.threads(),
        "kind": "port",
        "sample": what,
        "seconds": dt,
    }


def cli_process(args, w, n):
    """The xt_neighbor CLI as a whole process on the workload files (parse + search, no -o),
    timed like the reference's published harness: wall clock around the process. Its -V
    stage lines (start-up, parse, search, output) give the breakdown of the last run."""
    import xtn

    with tempfile.TemporaryDirectory() as td:
        cmd = [xtn.CLI_PATH] + workload_files(td, w)
        runs = 3 if n <= 2_000_000 else 2
        times, stages = [], None
        for i in range(1 + runs):
            t0 = time.perf_counter()
            p = subprocess.run(cmd + ["-V"], capture_output=True, text=True, timeout=1800)
            dt = time.perf_counter() - t0
            if p.returncode != 0:
                return {"error": p.stderr[-200:]}
            if i >= 1:
                times.append(dt)
                stages = cli_stage_times(p.stdout)
    s = sum(times) / len(times)
    return {"value": n / s, "unit": "seqs/s", "ms_per_run": s * 1e3, "runs": len(times),
            "stages_ms": stages, "what": "xt_neighbor CLI process: CSV parse + search, no -o, wall clock"}


def cli_stage_times(stdout: str):
    """The `xtn_b200 stage <name> <ms>` lines the CLI prints under -V, as a dict."""
    out = {}
    for line in stdout.splitlines():
        parts = line.split()
        if len(parts) == 4 and parts[0] == "xtn_b200" and parts[1] == "stage":
            try:
                out[parts[2]] = float(parts[3])
            except ValueError:
                pass
    return out or None


def workload_files(td, w, prefix_rows: int = 0, max_len: int = 0):
    """Writes the workload in the CLI's input format under td with the generator command
    (bin/xtn_synth: a separate process, so the caller loads no library of this build);
    returns the CLI arguments. With prefix_rows, also writes the first rows to warm.csv; with
    max_len (repertoires only), rows longer than max_len residues are left out."""
    path = os.path.join(td, "seqs.csv")
    if w["kind"] == "repertoires":
        ipath = os.path.join(td, "info.csv")
        cmd = [SYNTH_CLI, "repertoires", str(w["seed"]), str(w["n_reps"]), repr(w["min"]), repr(w["max"]),
               repr(w["shared"]), path, ipath] + ([str(max_len)] if max_len else [])
    elif w["kind"] == "clusters":
        cmd = [SYNTH_CLI, "clusters", str(w["seed"]), str(w["n"]), "0.2", "0.02", path]
    else:
        cmd = [SYNTH_CLI, "mutants", str(w["seed"]), str(w["n"]), "0.1", path]
    if prefix_rows and w["kind"] != "repertoires":
        cmd += [str(prefix_rows), os.path.join(td, "warm.csv")]
    p = subprocess.run(cmd, capture_output=True, text=True, check=True, timeout=1800)
    n = int(p.stdout.strip().splitlines()[-1])
    args = ["-i", path, "-n", str(n), "-d", str(w["d"])] + (["-m", "hamming"] if w["measure"] else [])
    if w["kind"] == "repertoires":
        with open(os.path.join(td, "info.csv")) as f:
            n_reps = sum(1 for line in f) - 1
        args += ["-I", os.path.join(td, "info.csv"), "-N", str(n_reps)]
    return args


def run_reference(args, w):
    """The reference XTNeighbor-streaming's own library entry point, xtn_perform, built from its
    sources for sm_100a (oracle/_ref/ref_perform), timed as a call in one process: one warm-up
    call on the workload's first 10,000 sequences, then up to --steps calls on the workload,
    stopping once the timed calls have taken REF_MAX_SECONDS (at least one always runs). The
    workload files come from the generator command, a separate process: this process loads no
    library of this build. Rank 0 alone runs under torchrun."""
    world, rank, local = dist_setup()
    if rank != 0:
        return None
    if w["kind"] == "repertoires":
        return {"impl": "reference", "unavailable": "the in-process reference arm covers nearest-neighbour workloads"}
    if not os.path.exists(REF_PERFORM):
        return {"impl": "reference", "unavailable": "reference build oracle/_ref/ref_perform missing"}
    warm_rows = 10_000
    with tempfile.TemporaryDirectory() as td:
        cli = workload_files(td, w, prefix_rows=warm_rows)
        n = int(cli[cli.index("-n") + 1])
        cmd = [REF_PERFORM, os.path.join(td, "warm.csv"), str(min(warm_rows, n)), cli[cli.index("-i") + 1], str(n),
               str(w["d"]), str(w["measure"]), str(max(1, args.steps)), str(REF_MAX_SECONDS)]
        env = dict(os.environ, CUDA_VISIBLE_DEVICES=os.environ.get("CUDA_VISIBLE_DEVICES", str(local)))
        t0 = time.perf_counter()
        p = subprocess.run(cmd, capture_output=True, text=True, env=env, timeout=3600)
        wall = time.perf_counter() - t0
    steps, outputs, parse_s = [], [], None
    for line in p.stdout.splitlines():
        parts = line.split()
        if parts and parts[0] == "step":
            steps.append(float(parts[1]))
            outputs.append(int(parts[2]))
        elif parts and parts[0] == "parse":
            parse_s = float(parts[1])
    if p.returncode != 0 or not steps or "Cuda error" in p.stdout:
        return {"impl": "reference", "unavailable": f"reference exited {p.returncode}: {(p.stderr or p.stdout)[-200:]}"}
    sec = sum(steps) / len(steps)
    v = n / sec
    expect = w.get("expect_out")
    return {
        "impl": "reference",
        "metric": METRIC,
        "value": v,
        "unit": "seqs/s",
        "n_gpus": 1,
        "steps": len(steps),
        "warmup": 1,
        "ms_per_step": sec * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "u32",
        "data": "synthetic (seeded CDR3 generator)",
        "config": {"workload": args.workload, "n_seqs": n, "distance": w["d"],
                   "measure": "hamming" if w["measure"] else "leven", "mode": "nn",
                   "parallelism": "single process", "steps_requested": args.steps,
                   "warmup_call": f"first {min(warm_rows, n)} sequences of the workload",
                   "stop_after_s": REF_MAX_SECONDS},
        # the reference's Levenshtein on sequences longer than 18 residues frees its DP column
        # before reading the result (xtneighbor_streaming/src/kernel.cu:263-278), so its output
        # length on a workload with such sequences varies between runs; this build's is exact
        "outputs": outputs[-1],
        "outputs_this_build": expect,
        "outputs_difference": (outputs[-1] - expect) if expect is not None else None,
        "parse_s": parse_s,
        "process_wall_s": wall,
        "cpu_baseline": {"value": v, "unit": "seqs/s", "cores": 1, "kind": "reference",
                         "sample": f"reference xtn_perform (its CUDA build, sm_100a, on this GPU; one host thread) "
                                   f"on the whole workload, {len(steps)} timed call(s) after a warm-up call"},
        "e2e": {"value": v, "unit": "seqs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def run_sharded(args, w):
    """The nearest-neighbour search sharded by first-level hash buckets (options shard_count /
    shard_index, xtn.nn_sharded): under torchrun every rank (one GPU each) searches its share of
    the buckets of the same input, the verified pairs are exchanged by owner over NCCL and
    merged; with --shard-by sequences (xtn.nn_sharded_exchange) every rank generates its own
    sequences' records and sends them to the bucket owners first; one step is the whole search over all ranks (strong scaling), timed on the device
    from the search's start to the merge's end, slowest rank. On one process, --shards K runs
    the K shards one after another on the one GPU and exchanges on the device with the same
    splits (per-shard and merge times reported): what each rank of a K-GPU run would compute,
    without the collective."""
    import datetime

    import numpy as np
    import torch

    import xtn

    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    K = world if world > 1 else args.shards
    pg = None
    if world > 1:
        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
        pg = dist
    chars, offs, info, _ = gen_workload(w)
    if info is not None:
        raise SystemExit("sharding covers the nearest-neighbour workloads only")
    n = len(offs) - 1
    opts = {k: int(v) for k, v in (o.split("=", 1) for o in args.opt)}
    ctx = xtn.Context(local, **opts)
    d_chars = torch.from_numpy(chars).cuda()
    d_offs = torch.from_numpy(offs.view(np.int32)).cuda()
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")
    ext = torch.cuda.ExternalStream(ctx.stream())
    torch.cuda.synchronize()
    unsharded = ctx.nn_device(d_chars.data_ptr(), d_offs.data_ptr(), n, w["d"], w["measure"])

    by_seq = args.shard_by == "sequences"

    def one_rank():
        search = xtn.nn_sharded_exchange if by_seq else xtn.nn_sharded
        return search(ctx, d_chars.data_ptr(), d_offs.data_ptr(), n, w["d"], w["measure"])

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(ext)
        r = fn()
        e1.record(ext)
        e1.synchronize()
        return r, e0.elapsed_time(e1)

    def emulated_exchange():
        """Sequence sharding: every rank's generate, then every owner's search over the pieces
        the ranks send it, then every owner's merge, in sequence on the one GPU. A rank's records
        are copied out of the context before the next rank's generate reuses its buffer; that copy
        and the gathering of an owner's pieces stand in for the all-to-all and are not timed."""
        gen_ms, sent_recs, counts = [], [], []
        for r in range(K):
            (cnt, ptr, nrec), ms = timed(lambda: ctx.shard_generate(d_chars.data_ptr(), d_offs.data_ptr(), n, w["d"],
                                                                    w["measure"], r, K))
            gen_ms.append(ms)
            counts.append(cnt.astype(np.int64))
            sent_recs.append(torch.as_tensor(xtn._DeviceWords(ptr, nrec), device="cuda").clone() if nrec else None)
        bounds = xtn.owner_ranges(sum(counts), K)
        cums = [np.concatenate([[0], np.cumsum(c)]) for c in counts]
        search_ms, sent_keys, remote = [], [], 0
        for k in range(K):
            lo, hi = bounds[k], bounds[k + 1]
            parts = [sent_recs[r][int(cums[r][lo]): int(cums[r][hi])] for r in range(K)
                     if sent_recs[r] is not None and cums[r][hi] > cums[r][lo]]
            remote += sum(int(cums[r][hi] - cums[r][lo]) for r in range(K) if r != k)
            got = torch.cat(parts) if parts else torch.zeros(1, dtype=torch.int64, device="cuda")
            pcs = np.stack([c[lo:hi] for c in counts]).astype(np.uint64)
            torch.cuda.synchronize()

            def search():
                m = ctx.shard_search(d_chars.data_ptr(), d_offs.data_ptr(), n, w["d"], w["measure"], got.data_ptr(), pcs)
                keys = torch.empty(max(m, 1), dtype=torch.int64, device="cuda")
                return keys, ctx.result_keys(n, keys.data_ptr(), keys.numel(), K)

            kst, ms = timed(search)
            search_ms.append(ms)
            sent_keys.append(kst)
            del got
        del sent_recs
        merge_ms, total = [], 0
        for dst in range(K):
            got = torch.cat([keys[st[dst]: st[dst + 1]] for keys, st in sent_keys])
            u, ms = timed(lambda: ctx.merge_keys(n, got.data_ptr(), got.numel()))
            total += u
            merge_ms.append(ms)
        return total, gen_ms, search_ms, merge_ms, remote * 8

    def emulated():
        shard_ms, sent = [], []
        ctx.set_option("shard_count", K)
        for k in range(K):
            ctx.set_option("shard_index", k)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(ext)
            m = ctx.nn_device(d_chars.data_ptr(), d_offs.data_ptr(), n, w["d"], w["measure"])
            keys = torch.empty(max(m, 1), dtype=torch.int64, device="cuda")
            starts = ctx.result_keys(n, keys.data_ptr(), keys.numel(), K)
            e1.record(ext)
            e1.synchronize()
            shard_ms.append(e0.elapsed_time(e1))
            sent.append((keys, starts))
        merge_ms, total = [], 0
        for dst in range(K):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(ext)
            got = torch.cat([keys[st[dst]: st[dst + 1]] for keys, st in sent])
            total += ctx.merge_keys(n, got.data_ptr(), got.numel())
            e1.record(ext)
            e1.synchronize()
            merge_ms.append(e0.elapsed_time(e1))
        return total, shard_ms, merge_ms

    times, out, detail = [], 0, None
    for i in range(args.warmup + args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        if pg:
            pg.barrier()
        if world > 1:
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(ext)
            out = one_rank()
            e1.record()
            e1.synchronize()
            ms = e0.elapsed_time(e1)
        elif by_seq:
            out, gen_ms, search_ms, merge_ms, sent_bytes = emulated_exchange()
            ms = sum(gen_ms) + sum(search_ms) + sum(merge_ms)
            if i >= args.warmup:
                detail = (detail or [np.zeros(K), np.zeros(K), np.zeros(K), 0])
                detail[0] += np.array(gen_ms) / args.steps
                detail[1] += np.array(search_ms) / args.steps
                detail[2] += np.array(merge_ms) / args.steps
                detail[3] = sent_bytes
        else:
            out, shard_ms, merge_ms = emulated()
            ms = sum(shard_ms) + sum(merge_ms)
            if i >= args.warmup:
                detail = (detail or [np.zeros(K), np.zeros(K)])
                detail[0] += np.array(shard_ms) / args.steps
                detail[1] += np.array(merge_ms) / args.steps
        if i >= args.warmup:
            times.append(ms)
    ms_step = reduce_max([sum(times) / len(times)], pg, "cuda")[0]
    if pg:
        import torch.distributed as dist

        t = torch.tensor([out], dtype=torch.int64, device="cuda")
        dist.all_reduce(t)
        out = int(t.item())
    ctx.close()
    if pg:
        pg.destroy_process_group()
    if rank != 0:
        return None
    line = {
        "metric": METRIC,
        "value": n / (ms_step / 1e3),
        "unit": "seqs/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_step,
        "higher_is_better": True,
        "scaling": "strong",
        "vs_baseline": None,
        "dtype": "u64",
        "data": "synthetic (seeded CDR3 generator)",
        "config": {"workload": args.workload, "n_seqs": n, "distance": w["d"],
                   "measure": "hamming" if w["measure"] else "leven", "mode": "nn",
                   "parallelism": f"shards x{K} by {args.shard_by}" + ("" if world > 1 else " run in sequence on one GPU"),
                   "l2": "flushed between steps (256 MiB write)"},
        "output_entries": out,
        "output_matches_unsharded": out == unsharded,
    }
    if detail is not None and by_seq:
        line["shards_one_gpu"] = {
            "generate_ms": [round(float(x), 3) for x in detail[0]],
            "search_ms": [round(float(x), 3) for x in detail[1]],
            "merge_ms": [round(float(x), 3) for x in detail[2]],
            "records_sent_to_other_ranks_bytes": int(detail[3]),
            "what": "each rank's generate of its own sequences' records, each owner's search over the "
                    "records sent to it + key packing, then each owner's merge, one after another on one "
                    "GPU (the two all-to-alls between them are not run)"}
    elif detail is not None:
        line["shards_one_gpu"] = {
            "shard_ms": [round(float(x), 3) for x in detail[0]],
            "merge_ms": [round(float(x), 3) for x in detail[1]],
            "what": "each shard's search + key packing, then each owner's merge of the keys it receives, "
                    "one after another on one GPU (the collective between them is not run)"}
    return line


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS) + sorted(SERVE_WORKLOADS), default=DEFAULT_WORKLOAD)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--engine", choices=["bucket", "sort"], default="bucket",
                    help="key grouping: shared-memory hash buckets (default) or full radix sort")
    ap.add_argument("--no-cli", action="store_true", help="skip timing the xt_neighbor CLI process")
    ap.add_argument("--no-extra", action="store_true", help="skip the extra workloads measured beside the headline")
    ap.add_argument("--no-forms", action="store_true", help="skip the plain-vs-graph form comparison")
    ap.add_argument("--no-serving", action="store_true", help="skip the serving trace in the default line")
    ap.add_argument("--autotune", action="store_true",
                    help="pick the bucket-engine shape by timing on the workload first (xtn_context_autotune)")
    ap.add_argument("--opt", action="append", default=[], metavar="NAME=VALUE",
                    help="context option (xtn_context_set_option), repeatable")
    ap.add_argument("--shards", type=int, default=0,
                    help="sharded search: under torchrun one shard per rank (any value > 0); on one process, "
                         "this many shards run in sequence on the one GPU")
    ap.add_argument("--shard-by", choices=["buckets", "sequences"], default="buckets",
                    help="sharding: every rank generates all variants and keeps its first-level buckets "
                         "(buckets), or generates its own sequences' variants and sends records to the "
                         "bucket owners (sequences)")
    args = ap.parse_args()
    if args.workload in SERVE_WORKLOADS:
        if args.impl == "reference":
            line = {"impl": "reference", "unavailable": "the reference has no query-serving mode (offline searches only)"}
        else:
            line = run_serve(args, SERVE_WORKLOADS[args.workload])
    else:
        w = WORKLOADS[args.workload]
        if args.impl == "reference":
            line = run_reference(args, w)
        elif args.shards > 0:
            line = run_sharded(args, w)
        else:
            line = run_ours(args, w)
    if line is not None:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
