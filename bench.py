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
* ``fp64``: the same update in Float64; ``mixed``: in mixed precision (Float32 columns and
  arithmetic with Float64 islands). ``precision``: every column's max / mean absolute error of
  the Float32 and mixed updates against the Float64 one, and the cells whose kind or ambiguous
  flag differ.
* ``learned``: the learned volume-fraction correction (packaged weights) on an unseen seeded
  smooth-min body (``workloads.smooth_blob(5002)``, 4..12 spheres in [0,1]^3) at the same size,
  Float32: the cut cells' volume-fraction L1 error against marching cubes at 8x sub-refinement,
  plain and learned, the fallback rate, and the plain and learned update times on the same cache
  (CUDA events). Equal error: plain marching cubes' convergence order p is measured between n/2
  and n on the same body; plain reaches the learned error at n * (L1_plain / L1_learned)^(1/p)
  cells per axis, which costs (that / n)^3 plain updates at n.
* ``batch``: the batched marching-squares workloads -- 256 updates of a translating circle
  (radius 0.3, velocity (0.4, 0.1), dt 1e-3), update i on its own n_i x n_i grid of [-1,1]^2,
  n_i ~ U{64..1024}, Float32 and Float64; and a quadtree refined from level 4 to 12 toward a star
  curve -- as per-update launches against one autotuned, graph-captured batched launch (CUDA
  events, the same caches).
* ``plic``: PLICCutCell over [0,1]^3 at the same n, a union of 64 seeded spheres: update times
  in Float32, Float64 and mixed precision, the resolved face fractions' single-valuedness, the
  errors against Float64, calc_volume against a 10^8-point Monte Carlo estimate, and
  ``surface_f32``: generate_mesh of the Float32 cache (every cell's plane clipped to its cell).
* ``mesh``: generate_mesh (count and emit) of the Float32 CSG cache on the device, and the oracle's
  serial march of a bounded slab of the same field.
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
    """nvidia-smi clocks and throttle reasons, sampled every period_ms while the timed regions run."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index, period_ms=200):
        self.index = index
        self.period_ms = period_ms
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", str(self.period_ms)],
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


def slab_range(n, slab=8):
    """The middle z-slab of cell layers the CPU legs sample: layers k0..k0+slab-1 of the n^3 grid."""
    k0 = max(n // 2 - slab // 2, 0)
    return k0, min(k0 + slab, n)


def cpu_port_rate(n, prec, seconds=8.0, slab=8):
    """Oracle throughput (cells/s) on the middle slab of the workload with every host thread; the
    slab is evaluated with the full grid's node coordinates, so its output is the whole-grid
    oracle's for those layers. Returns (rate, threads, sample, (phi, columns) of the last run)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as po
    from __graft_entry__ import load_package
    cc = load_package()
    threads = os.cpu_count() or 1
    po.set_threads(threads)
    g = cc.workloads.csg_grid(n)
    k0, k1 = slab_range(n, slab)
    tape = cc.flatten(cc.workloads.csg_body(0), 3)
    table = cc.mc_tables.project_table()
    t0 = time.perf_counter()
    cells = 0
    reps = 0
    while True:
        out = po.mc_update_slab(g, tape, table, prec, k0, k1)
        cells += n * n * (k1 - k0)
        reps += 1
        if time.perf_counter() - t0 >= seconds:
            break
    dt = time.perf_counter() - t0
    sample = (f"{reps} x oracle mc_update of cell layers {k0}..{k1 - 1} of the {n}^3 workload ({n}x{n}x{k1 - k0} "
              f"cells, full-grid node coordinates, {dt:.1f} s); cells/s of that sample, extrapolated to the "
              f"whole grid only in ms_per_step")
    return cells / dt, threads, sample, out


def slab_of_cache(cache, n, slab=8):
    """Host copies of the middle slab's phi (node layers k0..k1) and columns (cell layers k0..k1-1)."""
    k0, k1 = slab_range(n, slab)
    lay, nlay = n * n, (n + 1) * (n + 1)
    cols = {f: getattr(cache.cells, f)[lay * k0:lay * k1].cpu().numpy() for f in CELL_FIELDS}
    return cache.phi[nlay * k0:nlay * (k1 + 1)].cpu().numpy(), cols


CELL_FIELDS = ("kind", "ambiguous", "volume_fraction", "centroid", "face_fraction", "face_centroid_local",
               "interface_centroid")


def same_bits(dev, ref):
    """Device slab (phi, columns) equal to the oracle's bit for bit."""
    import numpy as np

    def eq(a, b):
        return np.array_equal(np.ascontiguousarray(a).view(np.uint8), np.ascontiguousarray(b).view(np.uint8))
    return bool(eq(dev[0], ref[0]) and all(eq(dev[1][f], ref[1][f]) for f in CELL_FIELDS))


def run_reference(args, rank, world):
    if rank != 0:
        return
    prec = 0 if args.prec == "f32" else 1
    rates = []
    for _ in range(args.warmup):
        cpu_port_rate(args.n, prec, seconds=0.5)
    for _ in range(args.steps):
        r, threads, sample, _ = cpu_port_rate(args.n, prec, seconds=2.0)
        rates.append(r)
    v = statistics.median(rates)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "cells/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": args.n ** 3 / v * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": args.prec,
            "data": "synthetic", "config": config(args),
            "cpu_baseline": {"value": v, "unit": "cells/s", "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": "cells/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


METRIC = "MC cells/s at 512\u00b3 FP32 vs FP64 and learned vs plain at equal vol-frac L1 error"


def config(args):
    return {"workload": f"MarchingCubesCutCell update_cache! {args.n}^3 {'Float32' if args.prec == 'f32' else 'Float64'}, "
                        "CSG union sphere+box+rotated torus over [-1,1]^3, seed 0",
            "grid": [args.n] * 3, "method": "MarchingCubesCutCell", "parallelism": f"replicas x{args.gpus}",
            "l2": "each step writes >14 GB (outputs larger than L2), no flush needed"}


def max_over_ranks(x: float, dist, device) -> float:
    """The largest of every rank's x: a multi-GPU time is the slowest rank's. Every rank must call
    it at the same point (it is a collective); alone, x itself."""
    if not dist:
        return x
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(world: int, cells_per_rank: int, seconds: float) -> float:
    """Whole-job cells/s: every rank updates its own replica of cells_per_rank cells (weak scaling),
    in the slowest rank's time."""
    return world * cells_per_rank / seconds


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

    def timed_updates(dtype, precision="plain"):
        cache = cc.allocate_cache(g, cc.MarchingCubesCutCell(), dtype=dtype, device=dev, precision=precision)
        s = torch.cuda.current_stream(dev)
        for _ in range(args.warmup):
            cc.update_cache(cache, tape, g, sync=False)
        torch.cuda.synchronize(dev)
        if dist:
            dist.barrier()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
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
        return cache, total_ms, per

    # clocks are sampled over every timed region (Float32, end to end, Float64, learned)
    clk = ClockSampler(dev.index, period_ms=100).__enter__()
    cache, total_ms, per = timed_updates(torch.float32)
    total_ms = max_over_ranks(total_ms, dist, dev)
    ms = total_ms / args.steps
    value = job_rate(world, n ** 3, ms * 1e-3)
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
    e2e_s = max_over_ranks((time.perf_counter() - t0) / args.steps, dist, dev)
    ops_bytes = tape.ops.nbytes + tape.params.nbytes

    # Float64 and mixed precision at the same size, then every field's error against Float64
    cache64, total64, per64 = timed_updates(torch.float64)
    ms64 = max_over_ranks(total64, dist, dev) / args.steps
    bytes64 = cc.workloads.mc_bytes_per_update(n, 8)
    cachem, totalm, perm = timed_updates(torch.float32, "mixed")
    msm = max_over_ranks(totalm, dist, dev) / args.steps
    precision = precision_report(cc, g, cache, cache64, cachem, dev)
    # the middle slab of each cache, for the oracle check of the CPU-baseline leg below
    slabs = {"float32": slab_of_cache(cache, n), "float64": slab_of_cache(cache64, n),
             "mixed": slab_of_cache(cachem, n)} if (not args.no_cpu and world == 1) else None
    del cache, cache64, cachem
    torch.cuda.empty_cache()
    precision["degenerate_deciders"] = degenerate_decider_errors(cc, dev)

    sizes = sizes_block(args, dev, cc)
    learned = None if args.no_learned else learned_block(args, dev, cc)
    batched = None if args.no_batch else batch_block(args, dev, cc, k=args.batch_updates)
    mesh = mesh_block(args, dev, cc)
    plic = None if args.no_plic else plic_block(args, dev, cc)
    clk.__exit__(None, None, None)
    clocks = clk.summary()

    if rank != 0:
        return
    line = {"metric": METRIC, "value": value, "unit": "cells/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded CSG body, no dataset)",
            "config": config(args),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic_per_update(n), "peak_source": peak_kind,
                         "algorithmic_bytes_per_launch": bytes_per,
                         "per": "one update (fill + cut-band launch), CUDA events",
                         "traffic_source": "ncu dram__bytes_read+write of fill and cut at 256^3, scaled by cells"},
            "e2e": {"value": job_rate(world, n ** 3, e2e_s), "unit": "cells/s", "h2d_bytes_per_step": int(ops_bytes),
                    "d2h_bytes_per_step": 48,
                    "note": "per step: the host body flattened and uploaded, a blocking update_cache, the cut-cell "
                            "report read back; the columns stay on the device, as the reference's CuArray cache "
                            "does"},
            "gpu_launches": 2 * args.steps,  # per update: the fill kernel and the cut-band kernel
            "clocks": clocks,
            "fp64": {"value": job_rate(world, n ** 3, ms64 * 1e-3), "ms_per_step": ms64,
                     "roofline_frac": bytes64 / (statistics.mean(per64) * 1e-3) / 1e9 / peak},
            "mixed": {"value": job_rate(world, n ** 3, msm * 1e-3), "ms_per_step": msm,
                      "roofline_frac": bytes_per / (statistics.mean(perm) * 1e-3) / 1e9 / peak},
            "precision": precision,
            "sizes": sizes,
            "learned": learned,
            "batch": batched,
            "mesh": mesh,
            "plic": plic,
            "report": rep}
    if slabs is not None:
        v, threads, sample, ref32 = cpu_port_rate(n, 0)
        line["cpu_baseline"] = {"value": v, "unit": "cells/s", "cores": threads, "kind": "port", "sample": sample}
        # the timed oracle's own output checks the device's Float32 slab; one more oracle run each
        # checks the Float64 and mixed slabs
        _, _, _, ref64 = cpu_port_rate(n, 1, seconds=0.0)
        _, _, _, refm = cpu_port_rate(n, 2, seconds=0.0)
        k0, k1 = slab_range(n)
        precision["oracle_check"] = {
            "slab": f"cell layers {k0}..{k1 - 1} of {n}^3 ({n * n * (k1 - k0)} cells), every column and phi",
            "float32_bitwise": same_bits(slabs["float32"], ref32),
            "float64_bitwise": same_bits(slabs["float64"], ref64),
            "mixed_bitwise": same_bits(slabs["mixed"], refm)}
    else:
        precision["oracle_check"] = "not run (--no-cpu or more than one rank)"
    print(json.dumps(line), flush=True)


def field_errors(c, ref, chunk=1 << 23, keep=None):
    """Max and mean absolute error of every column of cache ``c`` against cache ``ref`` (same
    grid), over all cells and over the cells whose eight corner values classify the same in both
    (marching cubes' nudged signs, phi > -eps(T): there the difference is the arithmetic's;
    elsewhere a value within eps(Float32) of zero, or a sampled value near zero, flipped side),
    and the cells whose kind or ambiguous flag differ. ``keep`` (a bool per cell) restricts the
    "same signs" statistics further. Computed on the device in chunks."""
    import torch
    import torch.nn.functional as F
    n = c.cells.kind.numel()
    nn = [x + 1 for x in c.n]
    # the signs marching cubes classifies by: nudge_zeros(phi) >= 0, i.e. phi > -eps(T)
    e_c, e_r = torch.finfo(c.phi.dtype).eps, torch.finfo(ref.phi.dtype).eps
    flip = ((c.phi > -e_c) != (ref.phi > -e_r)).reshape(1, 1, nn[2], nn[1], nn[0]).float()
    same = (F.max_pool3d(flip, 2, stride=1) == 0).reshape(-1)
    del flip
    out = {"cells_with_a_flipped_corner_sign": int(n - same.sum().item())}
    if keep is not None:
        same &= keep
    out["cells_in_same_signs_stats"] = int(same.sum().item())
    for f in ("volume_fraction", "centroid", "face_fraction", "face_centroid_local", "interface_centroid"):
        a = getattr(c.cells, f).reshape(n, -1)
        b = getattr(ref.cells, f).reshape(n, -1)
        mx = sm = mxs = sms = 0.0
        for s0 in range(0, n, chunk):
            d = (a[s0:s0 + chunk].double() - b[s0:s0 + chunk]).abs()
            mx = max(mx, d.max().item())
            sm += d.sum().item()
            ds = d[same[s0:s0 + chunk]]
            if ds.numel():
                mxs = max(mxs, ds.max().item())
                sms += ds.sum().item()
        out[f] = {"max": mx, "mean": sm / a.numel(), "max_same_signs": mxs,
                  "mean_same_signs": sms / max(int(same.sum().item()) * a.shape[1], 1)}
    d = (c.phi.double() - ref.phi).abs()
    out["phi"] = {"max": d.max().item(), "mean": d.mean().item()}
    del d
    out["kind_mismatch"] = int((c.cells.kind != ref.cells.kind).sum().item())
    out["ambiguous_mismatch"] = int((c.cells.ambiguous != ref.cells.ambiguous).sum().item())
    return out


def cells_differ(a, b, chunk=1 << 23):
    """Per cell: does any column of cache ``a`` differ from cache ``b`` (same dtype) bit for bit."""
    import torch
    n = a.cells.kind.numel()
    out = torch.zeros(n, dtype=torch.bool, device=a.cells.kind.device)
    for f in ("kind", "ambiguous", "volume_fraction", "centroid", "face_fraction", "face_centroid_local",
              "interface_centroid"):
        x = getattr(a.cells, f).reshape(n, -1)
        y = getattr(b.cells, f).reshape(n, -1)
        iv = torch.int8 if x.element_size() == 1 else (torch.int32 if x.element_size() == 4 else torch.int64)
        for s0 in range(0, n, chunk):
            out[s0:s0 + chunk] |= (x[s0:s0 + chunk].view(iv) != y[s0:s0 + chunk].view(iv)).any(dim=1)
    return out


def near_zero_cells(c):
    """Per cell: does a corner of cache ``c``'s phi lie within eps(T) of zero, where nudge_zeros
    replaces it by eps(T) (src/marching_cubes/marching_cubes.jl:240-243)."""
    import torch
    import torch.nn.functional as F
    nn = [x + 1 for x in c.n]
    near = (c.phi.abs() < torch.finfo(c.phi.dtype).eps).reshape(1, 1, nn[2], nn[1], nn[0]).float()
    return (F.max_pool3d(near, 2, stride=1) > 0).reshape(-1)


def decider_threshold_cells(c, chunk=32):
    """Per cell: does one of its faces have alternating corner signs and an asymptotic-decider
    determinant |A C - B D| below eps(Float32) (src/marching_cubes/marching_cubes.jl:401-406)? There
    a Float32 or mixed update decides by the threshold, face >= 0, where Float64, whose threshold is
    eps(Float64), decides by the determinant's sign: the two tile the cell differently. Computed in
    Float64 on the cache's phi nudged as Float32 nudges it."""
    import torch
    n0, n1, n2 = c.n
    phi = c.phi.reshape(n2 + 1, n1 + 1, n0 + 1)
    e = float(torch.finfo(torch.float32).eps)
    out = torch.zeros(n2, n1, n0, dtype=torch.bool, device=phi.device)

    def amb(a, b, cc_, d):
        pa, pb, pc, pd = a >= 0, b >= 0, cc_ >= 0, d >= 0
        return (pa == pc) & (pb == pd) & (pa != pb) & ((a * cc_ - b * d).abs() < e)
    for k0 in range(0, n2, chunk):
        k1 = min(k0 + chunk, n2)
        v = phi[k0:k1 + 1].double()
        v = torch.where(v.abs() < e, torch.full_like(v, e), v)
        fx = amb(v[:-1, :-1, :], v[:-1, 1:, :], v[1:, 1:, :], v[1:, :-1, :])    # faces normal to x
        fy = amb(v[:-1, :, :-1], v[:-1, :, 1:], v[1:, :, 1:], v[1:, :, :-1])    # normal to y
        fz = amb(v[:, :-1, :-1], v[:, :-1, 1:], v[:, 1:, 1:], v[:, 1:, :-1])    # normal to z
        out[k0:k1] = (fx[:, :, :-1] | fx[:, :, 1:]) | (fy[:, :-1, :] | fy[:, 1:, :]) | (fz[:-1] | fz[1:])
        del v, fx, fy, fz
    return out.reshape(-1)


def precision_report(cc, g, c32, c64, cm, dev):
    """Every column's error of the Float32 and mixed updates against Float64, split into its
    sources. ``c64_on_32`` is the Float64 cell construction run on the Float32 update's phi: against
    the Float64 update it isolates the error of sampling phi in Float32 (corner signs and the
    deciders' inputs move). On the same phi, two things still differ before any arithmetic:
    nudge_zeros lifts a corner within eps(Float32) of zero to eps(Float32) in Float32 but leaves it
    in Float64 (near-zero cells), and a Float32 decider can decide otherwise than Float64 (the cells
    where Float32 and mixed differ, mixed's deciders being Float64). The arithmetic-only
    statistics leave both out."""
    import torch
    c64on32 = cc.allocate_cache(g, cc.MarchingCubesCutCell(), dtype=torch.float64, device=dev)
    cc.update_cache(c64on32, cc.NodalField(c32.phi.double()), g)
    flips = cells_differ(c32, cm)
    near = near_zero_cells(c32)
    thresh = decider_threshold_cells(c32)
    out = {"reference": "the Float64 update of the same body and grid",
           "float32": field_errors(c32, c64), "mixed": field_errors(cm, c64),
           "input_rounding": {"what": "Float64 cells from the Float32 phi, against the Float64 update",
                              **field_errors(c64on32, c64)},
           "float32_decider_flip_cells": int(flips.sum().item()),
           "near_zero_corner_cells": int(near.sum().item()),
           "decider_threshold_cells": int(thresh.sum().item()),
           "decider_threshold": {"what": "Float32 against Float64 cells on the same Float32 phi, cells with a "
                                         "face decided by the eps(Float32) threshold, not the determinant's sign",
                                 **field_errors(c32, c64on32, keep=thresh)},
           "near_zero": {"what": "Float32 against Float64 cells on the same Float32 phi, cells with a corner "
                                 "within eps(Float32) of zero (nudged in Float32 only)",
                         **field_errors(c32, c64on32, keep=near)},
           "float32_arithmetic": {"what": "Float32 against Float64 cells on the same Float32 phi, cells with the "
                                          "same decisions as mixed, no corner within eps(Float32) of zero and no "
                                          "face at the decider threshold",
                                  **field_errors(c32, c64on32, keep=~flips & ~near & ~thresh)},
           "mixed_arithmetic": {"what": "mixed against Float64 cells on the same Float32 phi, no corner within "
                                        "eps(Float32) of zero, no face at the decider threshold",
                                **field_errors(cm, c64on32, keep=~near & ~thresh)}}
    del c64on32, flips, near, thresh
    torch.cuda.empty_cache()
    return out


def degenerate_decider_errors(cc, dev, n=128, seed=7):
    """Marching cubes from a nodal field built to stress the asymptotic deciders -- corner values
    +-(4096 + k 2^-11), k < 64, random signs, so every ambiguous face's determinant is a
    difference of nearly equal products -- in Float32 and mixed precision, against Float64 on the
    same (Float32) values."""
    import numpy as np
    import torch
    rng = np.random.default_rng(seed)
    m = (n + 1) ** 3
    mag = 4096.0 + rng.integers(0, 64, m) * 2.0 ** -11
    v32 = torch.as_tensor((np.where(rng.random(m) < 0.5, -1.0, 1.0) * mag).astype(np.float32), device=dev)
    g = cc.CartesianGrid((0.0, 0.0, 0.0), (n, n, n), (1.0, 1.0, 1.0))
    caches = {}
    for name, dt, prec in (("f64", torch.float64, "plain"), ("float32", torch.float32, "plain"),
                           ("mixed", torch.float32, "mixed")):
        c = cc.allocate_cache(g, cc.MarchingCubesCutCell(), dtype=dt, device=dev, precision=prec)
        cc.update_cache(c, cc.NodalField(v32.to(dt)), g)
        caches[name] = c
    out = {"field": f"{n}^3 nodal field +-(4096 + k 2^-11), seed {seed}"}
    for name in ("float32", "mixed"):
        e = field_errors(caches[name], caches["f64"])
        out[name] = {k: e[k] for k in ("volume_fraction", "face_fraction", "kind_mismatch", "ambiguous_mismatch")}
    return out


def sizes_block(args, dev, cc, sizes=(256, 200, 500)):
    """The Float32 update of the same CSG body at other sizes: 256^3 (a configuration of its own) and
    two grids whose x extent is not a multiple of 16 cells (200^3, the reference README's example
    size, and 500^3), whose kind/ambiguous rows TMA cannot address. CUDA events, the roofline
    fraction of each against the measured copy bandwidth."""
    import torch
    peak = measured_peak()[0]
    out = {}
    for m in sizes:
        g = cc.workloads.csg_grid(m)
        tape = cc.flatten(cc.workloads.csg_body(0), 3)
        cache = cc.allocate_cache(g, cc.MarchingCubesCutCell(), dtype=torch.float32, device=dev)
        s = torch.cuda.current_stream(dev)
        for _ in range(max(args.warmup, 3)):
            cc.update_cache(cache, tape, g, sync=False)
        torch.cuda.synchronize(dev)
        reps = max(args.steps, 10)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(s)
        for _ in range(reps):
            cc.update_cache(cache, tape, g, sync=False)
        b.record(s)
        torch.cuda.synchronize(dev)
        ms = a.elapsed_time(b) / reps
        byts = cc.workloads.mc_bytes_per_update(m, 4)
        out[f"{m}^3"] = {"ms": ms, "cells_per_s": m ** 3 / (ms * 1e-3), "algorithmic_bytes": byts,
                         "roofline_frac": byts / (ms * 1e-3) / 1e9 / peak,
                         "x_multiple_of_16": m % 16 == 0}
        del cache
        torch.cuda.empty_cache()
    return out


def traffic_per_update(n):
    """DRAM bytes of one Float32 update of the CSG workload, from one ncu capture of the fill and
    cut-band kernels at 256^3 (fill 1.7377 GB written + 3.9 MB read; cut 21.3 MB for 99,771 cut
    cells), scaled by cells (x8 per doubling of n for the fill, x4 for the cut band's surface)."""
    if n < 64:
        return None
    s = n / 256.0
    return (1.7377e9 + 3.9e6) * s ** 3 + 21.3e6 * s ** 2


# Per-cell counts of the PLIC Float32 update (fit + face pass) on the 64-sphere union. Warp
# instructions from one ncu capture at 512^3 (sm__inst_executed.sum, one pass: 1812.4 M + 1372.8 M
# over 134,217,728 cells). FP32 flops (FADD + FMUL + 2 FFMA thread instructions) from a capture at
# 256^3 (3756 M + 266 M over 16,777,216 cells), scaled to 512^3 by the two sizes' ratio of
# instructions per cell (23.73 / 30.37).
PLIC_F32_WARP_INSTS_PER_CELL = (1812.37e6 + 1372.79e6) / 134217728
PLIC_F32_FLOPS_PER_CELL = (((1307.33 + 475.00 + 2 * 986.78) + (109.12 + 105.61 + 2 * 25.52)) * 1e6 / 16777216
                           * PLIC_F32_WARP_INSTS_PER_CELL / ((316.58e6 + 192.88e6) / 16777216))
B200_SMS, B200_MHZ = 148, 1965.0


def plic_rooflines(cells, ms, peak_gbs, bytes_per_cell=46):
    """The PLIC update against the three rooflines that could bound it: HBM (the bytes it must
    write), the FP32 pipe (128 lanes per SM, FFMA two flops) and instruction issue (4 warp
    instructions per SM per cycle), at B200's 148 SMs and 1965 MHz."""
    t = ms * 1e-3
    fp32_peak = B200_SMS * 128 * 2 * B200_MHZ * 1e6
    issue_peak = B200_SMS * 4 * B200_MHZ * 1e6
    hbm = cells * bytes_per_cell / t / 1e9 / peak_gbs
    fp32 = cells * PLIC_F32_FLOPS_PER_CELL / t / fp32_peak
    issue = cells * PLIC_F32_WARP_INSTS_PER_CELL / t / issue_peak
    return {"hbm_frac": hbm, "fp32_pipe_frac": fp32, "issue_frac": issue,
            "bound": max((("hbm", hbm), ("fp32 pipe", fp32), ("instruction issue", issue)), key=lambda x: x[1])[0],
            "fp32_flops_per_cell": PLIC_F32_FLOPS_PER_CELL, "warp_instructions_per_cell": PLIC_F32_WARP_INSTS_PER_CELL,
            "counts_source": "ncu: instructions at 512^3, flops at 256^3 scaled (profiles/plic_fit_face_f32_256_fp.md)"}


def plic_block(args, dev, cc):
    """PLIC over [0,1]^3 at n^3, a union of 64 seeded spheres: update times (Float32, Float64,
    mixed), the resolved face fractions' single-valuedness, every precision's error against
    Float64, and calc_volume against a 10^8-point Monte Carlo estimate."""
    import math
    import torch
    n = args.n
    g = cc.workloads.unit_grid(n)
    body = cc.workloads.sphere_cloud(0, 64)
    tape = cc.flatten(body, 3)
    s = torch.cuda.current_stream(dev)

    def timed(fn, reps):
        for _ in range(max(args.warmup, 1)):
            fn()
        torch.cuda.synchronize(dev)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(s)
        for _ in range(reps):
            fn()
        b.record(s)
        torch.cuda.synchronize(dev)
        return a.elapsed_time(b) / reps

    def faces_single_valued(c):
        ff = c.cells.face_fraction.reshape(n, n, n, 6)
        bad = 0
        for ax, dim in ((0, 2), (1, 1), (2, 0)):  # x, y, z (the tensor is [z, y, x, dir])
            lo = ff.narrow(dim, 1, n - 1)[..., 2 * ax]
            hi = ff.narrow(dim, 0, n - 1)[..., 2 * ax + 1]
            bad += int((lo.view(torch.int32 if ff.dtype == torch.float32 else torch.int64) !=
                        hi.view(torch.int32 if ff.dtype == torch.float32 else torch.int64)).sum().item())
        return bad

    out = {"grid": f"[0,1]^3 at {n}^3", "body": "union of 64 spheres, centres U[0.1,0.9]^3, radii U[0.02,0.08], seed 0"}
    ref = cc.allocate_cache(g, cc.PLICCutCell(), dtype=torch.float64, device=dev)
    ms64 = timed(lambda: cc.update_cache(ref, tape, g, sync=False), args.steps)
    out["f64"] = {"ms": ms64, "cells_per_s": n ** 3 / (ms64 * 1e-3), "shared_face_mismatches": faces_single_valued(ref)}
    for name, prec in (("f32", "plain"), ("mixed", "mixed")):
        c = cc.allocate_cache(g, cc.PLICCutCell(), dtype=torch.float32, device=dev, precision=prec)
        ms = timed(lambda: cc.update_cache(c, tape, g, sync=False), args.steps)
        vf = (c.cells.volume_fraction.double() - ref.cells.volume_fraction).abs()
        fd = (c.cells.face_fraction.double() - ref.cells.face_fraction).abs()
        out[name] = {"ms": ms, "cells_per_s": n ** 3 / (ms * 1e-3),
                     "roofline_frac": n ** 3 * 46 / (ms * 1e-3) / 1e9 / measured_peak()[0],
                     "rooflines": plic_rooflines(n ** 3, ms, measured_peak()[0]),
                     "shared_face_mismatches": faces_single_valued(c),
                     "is_valid_differs_from_f64": int((c.is_valid != ref.is_valid).sum().item()),
                     "kind_differs_from_f64": int((c.cells.kind != ref.cells.kind).sum().item()),
                     "vf_err_vs_f64": {"max": vf.max().item(), "mean": vf.mean().item()},
                     "face_fraction_err_vs_f64": {"max": fd.max().item(), "mean": fd.mean().item()}}
        if name == "f32":
            out["surface_f32"] = plic_surface_timing(c, g, dev)
        del c, vf, fd
        torch.cuda.empty_cache()
    del ref
    torch.cuda.empty_cache()
    vols = {}
    for name, dt, prec in (("f64", torch.float64, "plain"), ("f32", torch.float32, "plain"),
                           ("mixed", torch.float32, "mixed")):
        t0 = time.perf_counter()
        vols[name] = cc.calc_volume(tape, g, dtype=dt, precision=prec)
        vols[name + "_ms"] = (time.perf_counter() - t0) * 1e3
    t0 = time.perf_counter()
    mc, inside = cc.monte_carlo_volume(body, (0.0, 0.0, 0.0), (1.0, 1.0, 1.0), 100_000_000, 0)
    mc_ms = (time.perf_counter() - t0) * 1e3
    sigma = math.sqrt(mc * (1 - mc) / 1e8)
    out["calc_volume"] = dict(vols, monte_carlo={"points": 100_000_000, "seed": 0, "volume": mc, "std_error": sigma,
                                                 "ms": mc_ms},
                              f64_minus_mc_in_sigmas=(vols["f64"] - mc) / sigma)
    return out


def plic_surface_timing(cache, g, dev, reps=5):
    """generate_mesh of a PLIC cache (every cell's plane clipped to its cell; count, scan, emit),
    timed on the host around the blocking call."""
    import importlib
    import torch
    S = importlib.import_module("cutcell_b200.surface")
    for _ in range(2):
        m = S.generate_mesh(cache, g)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    for _ in range(reps):
        m = S.generate_mesh(cache, g)
    torch.cuda.synchronize(dev)
    ms = (time.perf_counter() - t0) / reps * 1e3
    ncell = cache.intercepts.shape[0]
    # per cell the count pass reads the plane (D+1 values) and the flag; the emit pass reads only
    # the survivors the count kept (counted with the output, below the rounding of this figure)
    plane_bytes = ncell * (cache.intercepts.element_size() * (g.dim + 1) + 1)
    out_bytes = m.nodes.numel() * m.nodes.element_size() + m.elements.numel() * 4 + m.cells.numel() * 8
    r = {"ms": ms, "cells_per_s": ncell / (ms * 1e-3), "nodes": int(m.nodes.shape[0]),
         "triangles": int(m.elements.shape[0]), "algorithmic_gb": (plane_bytes + out_bytes) / 1e9,
         "roofline_frac": (plane_bytes + out_bytes) / (ms * 1e-3) / 1e9 / measured_peak()[0]}
    del m
    return r


def mesh_block(args, dev, cc):
    """generate_mesh of the Float32 CSG cache at n^3 on the device, against the oracle's serial
    march of a bounded slab of the same field."""
    import importlib
    import numpy as np
    import torch
    S = importlib.import_module("cutcell_b200.surface")
    n = args.n
    g = cc.workloads.csg_grid(n)
    cache = cc.update_cache(cc.allocate_cache(g, cc.MarchingCubesCutCell(), dtype=torch.float32, device=dev),
                            cc.workloads.csg_body(0), g)
    for _ in range(max(args.warmup, 2)):
        m = S.generate_mesh(cache, g)
    torch.cuda.synchronize(dev)
    reps = 5
    t0 = time.perf_counter()
    for _ in range(reps):
        m = S.generate_mesh(cache, g)
    torch.cuda.synchronize(dev)
    ms = (time.perf_counter() - t0) / reps * 1e3
    out = {"grid": f"{n}^3 CSG body, Float32", "ms": ms, "vertices": int(m.nodes.shape[0]),
           "triangles": int(m.elements.shape[0]), "cells_per_s": n ** 3 / (ms * 1e-3)}
    if not args.no_cpu:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import pyoracle as po
        slab = 8
        k0 = n // 2 - slab // 2
        nx = n + 1
        phi = cache.phi.reshape(n + 1, nx, nx)[k0:k0 + slab + 1].cpu().numpy().reshape(-1)
        sub = cc.CartesianGrid((g.x0[0], g.x0[1], g.x0[2] + k0 * g.d[2]), (n, n, slab), g.d)
        table = cc.mc_tables.project_table()
        t0 = time.perf_counter()
        po.mc_mesh(sub, phi, table, 0)
        dt = time.perf_counter() - t0
        out["cpu_oracle_serial"] = {"cells_per_s": n * n * slab / dt, "sample": f"oracle mc_mesh of a {n}x{n}x{slab} slab"}
    del cache, m
    torch.cuda.empty_cache()
    return out


def batch_block(args, dev, cc, k=256):
    """Batched updates against per-update launches (the moving-circle and quadtree workloads)."""
    import importlib
    import torch
    Bm = importlib.import_module("cutcell_b200.batch")
    W = cc.workloads
    s = torch.cuda.current_stream(dev)

    def timed(fn, reps):
        for _ in range(max(args.warmup, 2)):
            fn()
        torch.cuda.synchronize(dev)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(s)
        for _ in range(reps):
            fn()
        b.record(s)
        torch.cuda.synchronize(dev)
        return a.elapsed_time(b) / reps

    out = {}
    for dtype, name in ((torch.float32, "f32"), (torch.float64, "f64")):
        ups = W.moving_circle_updates(k, seed=0)
        tapes = [cc.flatten(body, 2) for _, body, _ in ups]
        caches = [cc.allocate_cache(g, cc.MarchingSquaresCutCell(), dtype=dtype, device=dev) for g, _, _ in ups]
        cells = sum(g.ncell for g, _, _ in ups)
        nodes = sum(g.nnode for g, _, _ in ups)
        elem = 4 if dtype == torch.float32 else 8
        algo = cells * (2 + 13 * elem) + nodes * elem  # kind, ambiguous, vf, c 2, ff 4, fcl 4, ic 2

        def per_update():
            for c, (g, _, _), t in zip(caches, ups, tapes):
                cc.update_cache(c, t, g, sync=False)
        ms_single = timed(per_update, 3)
        b = Bm.Batch(dtype=dtype, device=dev)
        for c, (g, _, _), t in zip(caches, ups, tapes):
            b.add(c, t, g)
        cfg, tune_ms = b.autotune(reps=2)
        ms_graph = timed(lambda: b.run(sync=False), 5)
        # the tuned shape with band compaction switched the other way (off if tuned on, always on if off)
        other_band = 0 if cfg["band_percent"] > 0 else 100
        b.configure(band_percent=other_band)
        ms_other_band = timed(lambda: b.run(sync=False), 5)
        b.configure(band_percent=cfg["band_percent"], use_graph=0)
        ms_direct = timed(lambda: b.run(sync=False), 5)
        out[name] = {"updates": k, "cells": cells, "grids": "n x n, n ~ U{64..1024}, over [-1,1]^2",
                     "ms_per_update_launches": ms_single, "ms_batched_graph": ms_graph, "ms_batched_direct": ms_direct,
                     "speedup": ms_single / ms_graph, "cells_per_s_batched": cells / (ms_graph * 1e-3),
                     "roofline_frac": algo / (ms_graph * 1e-3) / 1e9 / measured_peak()[0],
                     "algorithmic_bytes": algo, "autotuned": cfg,
                     "band_compaction": {"tuned_percent": cfg["band_percent"], "other_percent": other_band,
                                         "ms_batched_graph_other": ms_other_band}}
        del b, caches
        torch.cuda.empty_cache()
    tree, amp, ph = cc.star_curve_tree(0, 4, 12)
    body = cc.flatten(W.star_body(amp, ph), 2)
    tc = cc.allocate_cache(tree, cc.MarchingSquaresCutCell(), dtype=torch.float32, device=dev)
    ms_tree = timed(lambda: cc.update_cache(tc, body, tree, sync=False), 5)
    bt = Bm.Batch(dtype=torch.float32, device=dev)
    bt.add(tc, body, tree)
    cfg, _ = bt.autotune(reps=3)
    ms_tree_b = timed(lambda: bt.run(sync=False), 10)
    out["quadtree"] = {"leaves": tree.nleaves, "levels": "4..12 toward a star curve (seed 0)",
                       "ms_single_update": ms_tree, "ms_batched_graph": ms_tree_b,
                       "leaves_per_s_batched": tree.nleaves / (ms_tree_b * 1e-3), "autotuned": cfg}
    return out


def learned_block(args, dev, cc):
    """Accuracy and cost of the learned correction against plain marching cubes (see the module
    docstring)."""
    import importlib
    import math
    import torch
    L = importlib.import_module("cutcell_b200.learned")
    n, seed, bound = args.n, 5002, 0.05
    m = L.pretrained(dev)
    g = cc.workloads.unit_grid(n)
    body = cc.workloads.smooth_blob(seed)
    tape = cc.flatten(body, 3)
    f, lab, pl, idx = L.body_samples(seed, n, dev, with_index=True)
    _, lab2, pl2 = L.body_samples(seed, n // 2, dev)
    cache = cc.allocate_cache(g, cc.MarchingCubesCutCell(), dtype=torch.float32, device=dev)
    nfb = L.update_cache_learned(cache, tape, g, m, bound=bound)
    vf = cache.cells.volume_fraction.reshape(-1)[idx]
    l1p = (lab - pl).abs().mean().item()
    l1l = (lab - vf).abs().mean().item()
    l1p_half = (lab2 - pl2).abs().mean().item()
    s = torch.cuda.current_stream(dev)

    def timed(fn):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize(dev)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(s)
        for _ in range(args.steps):
            fn()
        b.record(s)
        torch.cuda.synchronize(dev)
        return a.elapsed_time(b) / args.steps

    ms_plain = timed(lambda: cc.update_cache(cache, tape, g, sync=False))
    ms_learned = timed(lambda: L.update_cache_learned(cache, tape, g, m, bound=bound, count_fallback=False))
    order = math.log2(l1p_half / l1p)
    n_eq = n * (l1p / l1l) ** (1.0 / order)
    cost_eq = (n_eq / n) ** 3 * ms_plain
    del cache
    torch.cuda.empty_cache()
    return {"body": f"workloads.smooth_blob({seed}) over [0,1]^3 at {n}^3, Float32 (not a training body)",
            "weights": os.path.basename(L.default_weights_path()), "cut_cells": int(f.shape[0]),
            "l1_plain": l1p, "l1_learned": l1l, "gain": l1p / l1l, "fallback": int(nfb),
            "fallback_rate": nfb / f.shape[0], "bound": bound,
            "ms_plain": ms_plain, "ms_learned": ms_learned, "time_ratio": ms_learned / ms_plain,
            "cells_per_s_plain": n ** 3 / (ms_plain * 1e-3), "cells_per_s_learned": n ** 3 / (ms_learned * 1e-3),
            "equal_error": {"plain_l1_at_half_n": l1p_half, "plain_order": order, "plain_n_for_learned_l1": n_eq,
                            "plain_ms_at_that_n": cost_eq, "learned_speedup_at_equal_l1": cost_eq / ms_learned}}


def run_only(args):
    """One block alone: the marching-cubes update of the CSG body at --n and --prec, the
    marching-cubes mesh of the Float32 CSG cache or the PLIC surface of the Float32 64-sphere cache
    at --n, or the batched marching-squares workloads (--batch-updates)."""
    import torch
    from __graft_entry__ import load_package
    cc = load_package()
    dev = torch.device("cuda", 0)
    if args.only == "update":
        # the marching-cubes update alone (CSG body, --n, --prec), --warmup then --steps launches
        # of the fill and cut-band kernels: the bounded command to profile
        dtype = torch.float32 if args.prec == "f32" else torch.float64
        g = cc.workloads.csg_grid(args.n)
        tape = cc.flatten(cc.workloads.csg_body(0), 3)
        cache = cc.allocate_cache(g, cc.MarchingCubesCutCell(), dtype=dtype, device=dev)
        s = torch.cuda.current_stream(dev)
        for _ in range(args.warmup):
            cc.update_cache(cache, tape, g, sync=False)
        torch.cuda.synchronize(dev)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(s)
        for _ in range(args.steps):
            cc.update_cache(cache, tape, g, sync=False)
        b.record(s)
        torch.cuda.synchronize(dev)
        ms = a.elapsed_time(b) / max(args.steps, 1)
        byts = cc.workloads.mc_bytes_per_update(args.n, 4 if args.prec == "f32" else 8)
        out = {"grid": f"{args.n}^3 CSG body, {args.prec}", "ms": ms, "cells_per_s": args.n ** 3 / (ms * 1e-3),
               "roofline_frac": byts / (ms * 1e-3) / 1e9 / measured_peak()[0]}
    elif args.only == "mesh":
        args.no_cpu = True
        out = mesh_block(args, dev, cc)
    elif args.only == "batch":
        out = batch_block(args, dev, cc, k=args.batch_updates)
    else:
        g = cc.workloads.unit_grid(args.n)
        c = cc.allocate_cache(g, cc.PLICCutCell(), dtype=torch.float32, device=dev)
        cc.update_cache(c, cc.flatten(cc.workloads.sphere_cloud(0, 64), 3), g)
        out = dict(plic_surface_timing(c, g, dev), grid=f"[0,1]^3 at {args.n}^3, union of 64 spheres, Float32")
    print(json.dumps({"only": args.only, **out}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=512)
    ap.add_argument("--prec", default="f32", choices=["f32", "f64"])
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-learned", action="store_true")
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--no-plic", action="store_true")
    ap.add_argument("--batch-updates", type=int, default=256, help="updates in the batched marching-squares block")
    ap.add_argument("--only", choices=["update", "mesh", "plic-surface", "batch"],
                    help="run one block alone at --n and print its JSON (for profiling)")
    args = ap.parse_args()
    if args.only:
        run_only(args)
        return
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
