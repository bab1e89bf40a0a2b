#!/usr/bin/env python
"""Benchmark: HTRIP queryAllPairs on one B200 (per-call path), bit-exact.

Workload: 512 x 512 recursive-backtracker maze with 1-cell corridors and walls
(256 x 256 lattice), fully revealed, leaf b = 16, group 2 x 2 (H = 5), k = 256
viewpoints drawn uniformly from free cells.  One step = one queryAllPairs.

  value   k*k entries/s with viewpoints, flags and the output resident in HBM
          (htrip_query_all_pairs_dev), CUDA events on the index's stream,
          L2 flushed (256 MB write) before every timed query.
  e2e     the same metric through the C ABI with HOST buffers
          (htrip_query_all_pairs: host viewpoints and grid in, host matrix out).
  roofline  the query kernel's algorithmic HBM bytes (htrip_query_work) per
          launch / its event-timed duration, against the measured copy bandwidth.
  cpu_baseline  the reference's own MinPlusOracle::queryAllPairs (oracle/_ref,
          compiled from the reference sources) on one host core, same inputs.

`--impl reference` times the reference's CPU queryAllPairs with one query per
host thread per step (all host threads), same workload and metric.
Multi-GPU (torchrun): every rank runs an independent replica with its own
viewpoints (weak scaling, no collective on the data path).
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

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = dict(name="maze512-w1", side=512, corridor=1, maze_seed=2, b=16, g=2, k=256, vp_seed=7)
METRIC = "k×k entries/s (queryAllPairs, bit-exact)"


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def make_inputs(rank: int):
    from htrip_b200 import workloads as W
    grid = W.maze_grid(WORKLOAD["side"], WORKLOAD["corridor"], WORKLOAD["maze_seed"])
    vps = W.sample_free(grid, WORKLOAD["k"], WORKLOAD["vp_seed"] + rank)
    return grid, vps


def config_dict(extra=None):
    d = {"workload": "queryAllPairs, 512x512 maze (corridor 1, wall 1), b=16, g=2, k=256",
         "grid": WORKLOAD["side"], "b": WORKLOAD["b"], "g": WORKLOAD["g"], "k": WORKLOAD["k"],
         "l2": "256 MB L2 flush before every timed query"}
    if extra:
        d.update(extra)
    return d


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        rows = []
        try:
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) >= 9:
                    rows.append(f)
        except OSError:
            pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def profile_traffic():
    """Per-launch DRAM bytes of the query kernel from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "query_kernel_maze512_k256.json")
    try:
        return json.load(open(path)).get("dram_bytes_per_launch")
    except (OSError, ValueError):
        return None


def cpu_baseline_reference(grid, vps, seconds=10.0):
    """The reference's queryAllPairs on one host core (oracle/_ref), bounded sample."""
    from oracle.ref import PortOracle, RefOracle, ref_available
    k = len(vps)
    if ref_available():
        ref = RefOracle(WORKLOAD["b"], WORKLOAD["g"])
        ref.set_grid(grid)
        assert ref.build()
        sec, out = ref.time_query(vps, 1, 1)
        reps = max(1, min(200, int(seconds / max(sec, 1e-4))))
        sec, out = ref.time_query(vps, 1, reps)
        return {"value": reps * k * k / sec, "unit": "entries/s", "cores": 1, "kind": "reference",
                "sample": f"{reps} queryAllPairs calls (k={k}) on one core, same grid and viewpoints"}, out
    po = PortOracle(WORKLOAD["b"], WORKLOAD["g"])
    po.build(grid)
    t = time.perf_counter()
    out = po.query(vps, grid)
    sec = time.perf_counter() - t
    return {"value": k * k / sec, "unit": "entries/s", "cores": 1, "kind": "port",
            "sample": f"1 queryAllPairs call (k={k}) of the C restatement on one core"}, out


def run_reference(args, rank, world):
    if rank != 0:
        return 0
    from oracle.ref import PortOracle, RefOracle, ref_available
    grid, vps = make_inputs(0)
    k = len(vps)
    nthreads = os.cpu_count() or 1
    kind = "reference" if ref_available() else "port"
    if kind == "reference":
        ref = RefOracle(WORKLOAD["b"], WORKLOAD["g"])
        ref.set_grid(grid)
        assert ref.build()
        for _ in range(args.warmup):
            ref.time_query(vps, nthreads, 1)
        times = [ref.time_query(vps, nthreads, 1)[0] for _ in range(args.steps)]
    else:
        po = PortOracle(WORKLOAD["b"], WORKLOAD["g"])
        po.build(grid)
        nthreads = 1
        for _ in range(args.warmup):
            po.query(vps, grid)
        times = []
        for _ in range(args.steps):
            t = time.perf_counter()
            po.query(vps, grid)
            times.append(time.perf_counter() - t)
    total = sum(times)
    value = args.steps * nthreads * k * k / total
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "entries/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u16",
            "data": "synthetic", "config": config_dict({"threads": nthreads}),
            "cpu_baseline": {"value": value, "unit": "entries/s", "cores": nthreads, "kind": kind,
                             "sample": f"each step: {nthreads} concurrent queryAllPairs calls (k={k}), one per thread"},
            "e2e": {"value": value, "unit": "entries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    from htrip_b200.minplus_oracle import HierarchyConfig, MinPlusOracle

    torch.cuda.set_device(local_rank)
    grid, vps = make_inputs(rank)
    k = len(vps)
    idx = MinPlusOracle(HierarchyConfig(WORKLOAD["b"], WORKLOAD["g"], WORKLOAD["g"]), device=local_rank)
    t0 = time.perf_counter()
    assert idx.build(grid)
    build_s = time.perf_counter() - t0
    out_host = np.empty((k, k), dtype=np.uint16)
    idx.queryAllPairs(vps, grid, out_host)

    # parity of this rank's matrix against the CPU checker (rank 0 also times it)
    parity = None
    cpu = None
    if rank == 0:
        cpu, ref_out = cpu_baseline_reference(grid, vps)
        parity = "bit-exact" if np.array_equal(ref_out, out_host) else "MISMATCH"
        if parity != "bit-exact":
            log("parity check FAILED against", cpu["kind"])

    stream = torch.cuda.ExternalStream(idx.stream(), device=local_rank)
    vd = torch.from_numpy(vps).to(f"cuda:{local_rank}")
    pf = torch.ones(k, dtype=torch.uint8, device=f"cuda:{local_rank}")
    od = torch.empty((k, k), dtype=torch.int16, device=f"cuda:{local_rank}")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local_rank}")
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    ev2 = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            idx.queryAllPairsDevice(vd.data_ptr(), pf.data_ptr(), k, od.data_ptr())
        barrier()
        kern_ms = []
        with ClockSampler(local_rank) as clk:
            for i in range(args.steps):
                flush.zero_()
                ev[i][0].record(stream)
                idx.queryAllPairsDevice(vd.data_ptr(), pf.data_ptr(), k, od.data_ptr())
                ev[i][1].record(stream)
                kern_ms.append(idx.lastQueryKernelMs())
            barrier()
        dev_ms = sum(a.elapsed_time(b) for a, b in ev) / args.steps
        # e2e: host viewpoints / grid in, host matrix out, through the C ABI
        for _ in range(args.warmup):
            idx.queryAllPairs(vps, grid, out_host)
        barrier()
        for i in range(args.steps):
            flush.zero_()
            ev2[i][0].record(stream)
            idx.queryAllPairs(vps, grid, out_host)
            ev2[i][1].record(stream)
        barrier()
        e2e_ms = sum(a.elapsed_time(b) for a, b in ev2) / args.steps
    if not np.array_equal(od.cpu().numpy().view(np.uint16), out_host):
        parity = "MISMATCH (device path)"

    t = torch.tensor([dev_ms, e2e_ms, float(np.mean(kern_ms))], dtype=torch.float64, device=f"cuda:{local_rank}")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dev_ms, e2e_ms, kern_ms_avg = (float(x) for x in t.cpu())
    if rank != 0:
        return 0
    alg_bytes, alg_ops = idx.queryWork(vps, grid)
    peak, peak_kind = measured_peaks()
    achieved = alg_bytes / (kern_ms_avg * 1e-3) / 1e9
    h2d, d2h = idx.lastQueryIO()
    line = {
        "metric": METRIC, "value": world * k * k / (dev_ms * 1e-3), "unit": "entries/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dev_ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u16", "data": "synthetic",
        "config": config_dict({"parallelism": f"replicas x{world}", "build_s": round(build_s, 4)}),
        "e2e": {"value": world * k * k / (e2e_ms * 1e-3), "unit": "entries/s", "ms_per_step": e2e_ms,
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": profile_traffic(), "peak_source": peak_kind,
                     "kernel": "q_persistent_kernel", "kernel_ms": kern_ms_avg,
                     "alg_bytes_per_launch": alg_bytes, "alg_minplus_ops_per_launch": alg_ops,
                     "minplus_gops": alg_ops / (kern_ms_avg * 1e-3) / 1e9},
        "cpu_baseline": cpu,
        "clocks": clk.summary(),
        "gpu_launches": args.steps,
        "parity": parity,
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        return run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
