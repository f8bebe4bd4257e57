"""Benchmark: MarchingCubesCutCell update_cache! at 512^3 on one B200 (cells/s).

Workload: the CSG body (sphere r=0.45 offset by a seeded U(+-0.05), box half extents
(0.3,0.2,0.6), torus R=0.5 r=0.12 under a seeded random rotation) over [-1,1]^3 at 512^3 cells,
Float32 (the headline) and Float64. A step is one update of the whole cache: every node sampled,
every cell's CutCellData written (14.23 GB per Float32 update, 28.19 GB per Float64 update -- far
larger than the 126 MB L2, so no flush is needed between steps).

* ``value``: cells/s of the update with the cache resident in HBM, CUDA events on the launching
  stream, max over ranks.
* ``e2e``: the same metric through the public API as a user calls it: the body is flattened and
  uploaded from the host every step, update_cache blocks, and the cut-cell report is read back.
* ``roofline``: algorithmic bytes (output columns + phi) / average update duration against the
  measured HBM copy bandwidth.
* ``cpu_baseline`` / ``--impl reference``: the oracle (a C++ restatement of the reference's CPU
  path, all host threads) on a bounded slab of the same workload -- the reference itself is Julia
  and cannot run here.

Multi-GPU: the path has no exchange step; ``--gpus N`` runs N independent replicas (weak scaling).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm = [float(r[1]) for r in self.rows if len(r) > 8 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 8 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows if len(r) > 8 for i in range(4) if r[5 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def cpu_port_rate(n, prec, seconds=8.0, slab=8):
    """Oracle throughput (cells/s) on a slab of the workload with every host thread."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as po
    from __graft_entry__ import load_package
    cc = load_package()
    threads = os.cpu_count() or 1
    po.set_threads(threads)
    g = cc.workloads.csg_grid(n)
    # a slab through the middle of the body: n x n x slab cells
    sub = cc.CartesianGrid((g.x0[0], g.x0[1], -slab / 2 * g.d[2]), (n, n, slab), g.d)
    tape = cc.flatten(cc.workloads.csg_body(0), 3)
    table = cc.mc_tables.project_table()
    t0 = time.perf_counter()
    cells = 0
    reps = 0
    while True:
        po.mc_update(sub, tape, table, prec)
        cells += sub.ncell
        reps += 1
        if time.perf_counter() - t0 >= seconds:
            break
    dt = time.perf_counter() - t0
    return cells / dt, threads, f"{reps} x oracle mc_update of a {n}x{n}x{slab} slab of the workload ({dt:.1f} s)"


def run_reference(args, rank, world):
    if rank != 0:
        return
    prec = 0 if args.prec == "f32" else 1
    rates = []
    for _ in range(args.warmup):
        cpu_port_rate(args.n, prec, seconds=0.5)
    for _ in range(args.steps):
        r, threads, sample = cpu_port_rate(args.n, prec, seconds=2.0)
        rates.append(r)
    v = statistics.median(rates)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "cells/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": args.n ** 3 / v * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": args.prec,
            "data": "synthetic", "config": config(args),
            "cpu_baseline": {"value": v, "unit": "cells/s", "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": "cells/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


METRIC = "MarchingCubesCutCell update_cache! cells/s at 512^3 (Float32)"


def config(args):
    return {"workload": f"MarchingCubesCutCell update_cache! {args.n}^3 {'Float32' if args.prec == 'f32' else 'Float64'}, "
                        "CSG union sphere+box+rotated torus over [-1,1]^3, seed 0",
            "grid": [args.n] * 3, "method": "MarchingCubesCutCell", "parallelism": f"replicas x{args.gpus}",
            "l2": "each step writes >14 GB (outputs larger than L2), no flush needed"}


def run_ours(args, rank, world, dist):
    import ctypes as C
    import torch
    from __graft_entry__ import load_package
    cc = load_package()
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
    torch.cuda.set_device(dev)
    n = args.n
    g = cc.workloads.csg_grid(n)
    body = cc.workloads.csg_body(0)
    tape = cc.flatten(body, 3)
    peak, peak_kind = measured_peak()

    def timed_updates(dtype):
        cache = cc.allocate_cache(g, cc.MarchingCubesCutCell(), dtype=dtype, device=dev)
        s = torch.cuda.current_stream(dev)
        for _ in range(args.warmup):
            cc.update_cache(cache, tape, g, sync=False)
        torch.cuda.synchronize(dev)
        if dist:
            dist.barrier()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        with ClockSampler(dev.index) as clk:
            torch.cuda.synchronize(dev)
            t0 = torch.cuda.Event(enable_timing=True)
            t1 = torch.cuda.Event(enable_timing=True)
            t0.record(s)
            for a, b in ev:
                a.record(s)
                cc.update_cache(cache, tape, g, sync=False)
                b.record(s)
            t1.record(s)
            torch.cuda.synchronize(dev)
        total_ms = t0.elapsed_time(t1)
        per = [a.elapsed_time(b) for a, b in ev]
        return cache, total_ms, per, clk.summary()

    cache, total_ms, per, clocks = timed_updates(torch.float32)
    if dist:
        t = torch.tensor([total_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    ms = total_ms / args.steps
    value = world * n ** 3 / (ms * 1e-3)
    elem = 4
    bytes_per = cc.workloads.mc_bytes_per_update(n, elem)
    avg = statistics.mean(per)
    achieved = bytes_per / (avg * 1e-3) / 1e9

    # end to end through the public API: host body -> tape upload, blocking update, report back
    rep = None
    torch.cuda.synchronize(dev)
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        cc.update_cache(cache, body, g)  # flattens the host body and uploads it every step
        rep = cc.cut_cell_report(cache)
    e2e_s = (time.perf_counter() - t0) / args.steps
    if dist:
        t = torch.tensor([e2e_s], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    ops_bytes = tape.ops.nbytes + tape.params.nbytes
    del cache
    torch.cuda.empty_cache()

    # Float64 at the same size
    cache64, total64, per64, _ = timed_updates(torch.float64)
    del cache64
    torch.cuda.empty_cache()
    ms64 = total64 / args.steps
    bytes64 = cc.workloads.mc_bytes_per_update(n, 8)

    if rank != 0:
        return
    line = {"metric": METRIC, "value": value, "unit": "cells/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded CSG body, no dataset)",
            "config": config(args),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": None, "peak_source": peak_kind,
                         "algorithmic_bytes_per_launch": bytes_per},
            "e2e": {"value": world * n ** 3 / e2e_s, "unit": "cells/s", "h2d_bytes_per_step": int(ops_bytes),
                    "d2h_bytes_per_step": 48},
            "gpu_launches": args.steps,
            "clocks": clocks,
            "fp64": {"value": world * n ** 3 / (ms64 * 1e-3), "ms_per_step": ms64,
                     "roofline_frac": bytes64 / (statistics.mean(per64) * 1e-3) / 1e9 / peak},
            "report": rep}
    if not args.no_cpu and world == 1:
        v, threads, sample = cpu_port_rate(n, 0)
        line["cpu_baseline"] = {"value": v, "unit": "cells/s", "cores": threads, "kind": "port", "sample": sample}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=512)
    ap.add_argument("--prec", default="f32", choices=["f32", "f64"])
    ap.add_argument("--no-cpu", action="store_true")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dist = None
    if world > 1 and args.impl == "ours":
        import datetime
        import torch
        import torch.distributed as tdist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = tdist
    try:
        if args.impl == "reference":
            run_reference(args, rank, world)
        else:
            run_ours(args, rank, world, dist)
    finally:
        if dist:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
