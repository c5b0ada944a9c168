#!/usr/bin/env python
"""Benchmark of the wildfire hot path (fire behaviour + arrival-time
propagation) on B200.

Default workload: the large heterogeneous single scenario (4096 x 4096 cells
at 5 m, ridged terrain up to 45 deg, 12 % non-burnable lakes and roads,
smooth random wind 0-15 m/s, per-cell moisture jitter, 20 ignitions,
max_time 43200 s), seeded synthetic inputs.  A step = fire behaviour over
every cell + boundaries + propagation + post mask for that scenario.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME]
  python bench.py --impl reference ...   # the CPU implementation of the path

The JSON line carries: value (scenarios/s with inputs resident in HBM),
e2e (same metric through the C-ABI host-buffer entry point, copies inside
the timed region), per-step latency percentiles, roofline of the dominant
kernel (propagation) against the measured HBM peak, the fire kernel's
roofline, the CPU baseline and the SM clocks seen during the timed region.
N > 1 runs one replica per GPU (the single-scenario path does not shard).
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "propag-hidalgo_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "scenarios/s & p50/p99 latency, batched vs plain on 1 B200; cells/s vs HBM roofline"
UNIT = "scenarios/s"
FIRE_BYTES_PER_CELL = 49  # 37 B in (u8 fuel + 9 f32) + 12 B out (3 f32)
# propagation: 20 B per cell evaluation + 8 B per improvement + 4 B per
# reference-time gather (algorithmic, neighbours reused on chip)


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def _rank_env():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def _workload(name: str):
    from py_propag import scenarios as S
    if name == "config1":
        return S.config1(size=4096), "config1: 4096x4096 heterogeneous, 20 ignitions, 43200 s"
    if name == "config0":
        return S.config0(size=1024), "config0: 1024x1024 hills/voronoi, 1 ignition, 36000 s"
    if name.startswith("config1-"):
        n = int(name.split("-")[1])
        return S.config1(size=n), f"config1 style at {n}x{n}"
    raise SystemExit(f"unknown workload {name}")


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, index: int):
        self.proc = None
        self.path = os.path.join(ROOT, "gpurun_out", f"clocks_{os.getpid()}.csv")
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={index}",
                 "--query-gpu=clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 8:
                    continue
                try:
                    sm.append(float(parts[0]))
                    mx.append(float(parts[1]))
                except ValueError:
                    continue
                for nm, v in zip(names, parts[4:8]):
                    if v.lower() == "active":
                        reasons.add(nm)
        try:
            os.remove(self.path)
        except OSError:
            pass
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": float(max(mx)) if mx else None,
                "samples": len(sm), "reasons": sorted(reasons)}


def cpu_baseline(sc, evaluations_full: int, threads: int, budget_s: float = 20.0) -> dict:
    """Times the CPU restatement (oracle) on a bounded crop of the workload and
    scales by the propagation work (cell evaluations) of the full scenario."""
    from oracle import oracle as O
    t0 = time.perf_counter()
    ncell = sc.width * sc.height
    # fire behaviour: FP64 restatement over a 1/16 sample of the cells
    k = max(1, ncell // 16)
    samp = {kk: np.ascontiguousarray(v.ravel()[:k]) for kk, v in sc.terrain.items()}
    tf = time.perf_counter()
    O.burn_f64(samp)
    fire_s = (time.perf_counter() - tf) * (ncell / k)
    # propagation: crop around the first ignition, growing until the budget
    crop = 256
    cx, cy = sc.ignitions[0][0], sc.ignitions[0][1]
    prop_rate = None
    while True:
        x0 = int(min(max(cx - crop // 2, 0), sc.width - crop))
        y0 = int(min(max(cy - crop // 2, 0), sc.height - crop))
        sub = {kk: np.ascontiguousarray(v[y0:y0 + crop, x0:x0 + crop]) for kk, v in sc.terrain.items()}
        f, _ = O.burn_f64(sub)
        ign = [(x - x0, y - y0, t) for (x, y, t) in sc.ignitions
               if x0 <= x < x0 + crop and y0 <= y < y0 + crop]
        tp = time.perf_counter()
        r = O.propagate(crop, crop, sc.dx, sc.dy, sc.max_time, f[:, 4].astype(np.float32),
                        f[:, 5].astype(np.float32), f[:, 6].astype(np.float32), ign,
                        tile=323, threads=threads)
        dt = time.perf_counter() - tp
        prop_rate = r.stats["evaluations"] / dt
        if time.perf_counter() - t0 > budget_s / 3 or crop >= 1024:
            break
        crop *= 2
    prop_s = evaluations_full / prop_rate
    return {"value": 1.0 / (fire_s + prop_s), "unit": UNIT, "cores": threads, "kind": "port",
            "sample": (f"CPU restatement (oracle/): FP64 fire behaviour on {k} cells scaled to "
                       f"{ncell}; propagation on a {crop}x{crop} crop around the first ignition "
                       f"({prop_rate:.3g} cell evaluations/s on {threads} threads) scaled to the "
                       f"full scenario's {evaluations_full} evaluations"),
            "fire_s": fire_s, "propagation_s": prop_s}


def run_reference(args):
    rank, world, _ = _rank_env()
    if rank != 0:
        return
    sc, desc = _workload(args.workload)
    threads = os.cpu_count() or 1
    # the full scenario's propagation work, measured on B200 with the same
    # schedule (bit-identical evaluations on both sides)
    evals = {"config1": 1.0e9}.get(args.workload)
    vals = []
    for i in range(args.warmup + args.steps):
        cb = cpu_baseline(sc, int(evals or 0) or 10_000_000, threads, budget_s=10.0)
        if i >= args.warmup:
            vals.append(cb["value"])
    v = float(np.median(vals))
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "config": {"workload": desc}, "dtype": "f32", "data": "synthetic",
            "cpu_baseline": dict(cb, value=v),
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default="config1")
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--tile", type=int, default=0)
    ap.add_argument("--cluster", type=int, default=0)
    ap.add_argument("--no-cpu", action="store_true")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)

    import torch
    import torch.distributed as dist

    import py_propag as pp
    from py_propag import _lib as L

    rank, world, local = _rank_env()
    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", init_method="env://",
                                timeout=__import__("datetime").timedelta(seconds=600))
    dev = torch.device("cuda", torch.cuda.current_device())
    lib = L.lib()
    sc, desc = _workload(args.workload)
    N = sc.width * sc.height
    words = (N + 31) // 32

    # device-resident inputs and outputs
    t_dev = {k: torch.from_numpy(np.ascontiguousarray(v).ravel()).to(dev) for k, v in sc.terrain.items()}
    ptrs = L.PropagTerrainPtrs(*[t_dev[k].data_ptr() for k in L.TERRAIN_FIELDS])
    fire = [torch.empty(N, dtype=torch.float32, device=dev) for _ in range(3)]
    ign_np = np.array([(x, y, t) for (x, y, t) in sc.ignitions],
                      dtype=[("x", "<u4"), ("y", "<u4"), ("t", "<f4")])
    ign_dev = torch.from_numpy(np.frombuffer(ign_np.tobytes(), np.uint8).copy()).to(dev)
    time_d = torch.empty(N, dtype=torch.float32, device=dev)
    rx_d = torch.empty(N, dtype=torch.int16, device=dev)
    ry_d = torch.empty(N, dtype=torch.int16, device=dev)
    bnd_d = torch.empty(words, dtype=torch.int32, device=dev)
    job = L.PropagJob()
    job.width, job.height, job.dx, job.dy = sc.width, sc.height, sc.dx, sc.dy
    job.max_time, job.tile = sc.max_time, args.tile
    job.speed_max, job.azimuth_max, job.eccentricity = (f.data_ptr() for f in fire)
    job.ignitions, job.n_ignitions = ign_dev.data_ptr(), len(sc.ignitions)
    job.time, job.refs_x, job.refs_y, job.boundaries = (time_d.data_ptr(), rx_d.data_ptr(),
                                                        ry_d.data_ptr(), bnd_d.data_ptr())
    opt = L.PropagOptions(args.tile, args.cluster, 0, -1)
    eng = lib.propag_engine_create(C.byref(opt))
    if not eng:
        raise RuntimeError(L.last_error())
    stream = torch.cuda.current_stream(dev)
    sptr = C.c_void_p(stream.cuda_stream)

    def step(stats=None):
        rc = lib.propag_fire_simple_device(N, C.byref(ptrs), fire[0].data_ptr(), fire[1].data_ptr(),
                                           fire[2].data_ptr(), sptr)
        if rc:
            raise RuntimeError(L.last_error())
        rc = lib.propag_engine_run(eng, C.byref(job), 1, sptr, stats)
        if rc:
            raise RuntimeError(L.last_error())

    st = L.PropagStats()
    step(C.byref(st))  # first run: allocations + statistics of the workload
    stats = st.as_dict()
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()

    ev_fire = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(args.steps)]
    ev_step = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(args.steps)]
    eng_ms = []
    clocks = Clocks(torch.cuda.current_device())
    torch.cuda.synchronize()
    t_all0 = torch.cuda.Event(enable_timing=True)
    t_all1 = torch.cuda.Event(enable_timing=True)
    t_all0.record(stream)
    for i in range(args.steps):
        ev_step[i][0].record(stream)
        ev_fire[i][0].record(stream)
        rc = lib.propag_fire_simple_device(N, C.byref(ptrs), fire[0].data_ptr(), fire[1].data_ptr(),
                                           fire[2].data_ptr(), sptr)
        ev_fire[i][1].record(stream)
        rc |= lib.propag_engine_run(eng, C.byref(job), 1, sptr, None)
        ev_step[i][1].record(stream)
        if rc:
            raise RuntimeError(L.last_error())
        ms = (C.c_float * 3)()
        lib.propag_engine_last_times(eng, ms)  # waits for this step
        eng_ms.append(list(ms))
    t_all1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    total_ms = t_all0.elapsed_time(t_all1)
    if world > 1:
        tt = torch.tensor([total_ms], device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        total_ms = float(tt.item())
    step_ms = [a.elapsed_time(b) for a, b in ev_step]
    fire_ms = [a.elapsed_time(b) for a, b in ev_fire]
    prop_ms = [m[1] for m in eng_ms]
    value = world * args.steps / (total_ms / 1e3)

    # end to end through the C-ABI host entry point (pinned host buffers)
    pin = {k: torch.from_numpy(np.ascontiguousarray(v).ravel()).pin_memory() for k, v in sc.terrain.items()}
    hptrs = L.PropagTerrainPtrs(*[pin[k].data_ptr() for k in L.TERRAIN_FIELDS])
    out_t = torch.empty(N, dtype=torch.float32).pin_memory()
    out_rx = torch.empty(N, dtype=torch.int16).pin_memory()
    out_ry = torch.empty(N, dtype=torch.int16).pin_memory()
    out_b = torch.empty(words, dtype=torch.int32).pin_memory()
    g = pp.PyGeoReference(sc.width, sc.height, "+proj=utm +zone=30 +units=m",
                          [0.0, sc.dx, 0.0, 0.0, 0.0, sc.dy])
    settings = pp.PySettings(g, sc.max_time).inner
    ign_arr = (L.PropagIgnition * len(sc.ignitions))(*[L.PropagIgnition(x, y, t) for (x, y, t) in sc.ignitions])
    hopt = L.PropagOptions(args.tile, args.cluster, 0, -1)

    def e2e_step():
        rc = lib.propag_run_host(C.byref(settings), C.byref(hptrs), ign_arr, len(sc.ignitions),
                                 C.byref(hopt), out_t.data_ptr(), out_rx.data_ptr(), out_ry.data_ptr(),
                                 out_b.data_ptr(), None)
        if rc:
            raise RuntimeError(L.last_error())

    for _ in range(max(1, args.warmup)):
        e2e_step()
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    e2e_s = time.perf_counter() - t0
    if world > 1:
        tt = torch.tensor([e2e_s], device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e2e_s = float(tt.item())
    same = np.array_equal(out_t.numpy().view(np.uint32), time_d.cpu().numpy().view(np.uint32))
    h2d = N * 37 + len(sc.ignitions) * 12
    d2h = N * 4 + N * 4 + words * 4

    peak, peak_kind = _peaks()
    prop_bytes = 20 * stats["evaluations"] + 8 * stats["improvements"] + 4 * stats["gathers"]
    prop_s = float(np.mean(prop_ms)) / 1e3
    fire_s = float(np.mean(fire_ms)) / 1e3
    ach = prop_bytes / prop_s / 1e9
    fire_ach = FIRE_BYTES_PER_CELL * N / fire_s / 1e9
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": desc, "cells": N, "tile": args.tile or 323, "cluster": args.cluster,
                   "l2": "inputs larger than L2 (620 MB terrain, 16.8M-cell state)",
                   "parallelism": "replicas" if world > 1 else "single"},
        "latency_ms": {"p50": float(np.percentile(step_ms, 50)), "p99": float(np.percentile(step_ms, 99)),
                       "fire_kernel": float(np.mean(fire_ms)), "propagation_kernel": float(np.mean(prop_ms)),
                       "prep": float(np.mean([m[0] for m in eng_ms])),
                       "post": float(np.mean([m[2] for m in eng_ms]))},
        "cells_per_s": N * world * args.steps / (total_ms / 1e3),
        "e2e": {"value": world * args.steps / e2e_s, "unit": UNIT, "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "matches_device_path": bool(same)},
        "roofline": {"bound": "hbm", "kernel": "propagation engine", "achieved": ach, "peak": peak,
                     "unit": "GB/s", "frac": ach / peak, "traffic": None,
                     "algorithmic_bytes": prop_bytes, "peak_source": peak_kind},
        "kernels": {"fire_behaviour": {"achieved": fire_ach, "peak": peak, "unit": "GB/s",
                                       "frac": fire_ach / peak, "bytes": FIRE_BYTES_PER_CELL * N}},
        "workload_stats": stats,
        "gpu_launches": 5 * args.steps,
        "clocks": clk,
    }
    if rank == 0 and not args.no_cpu:
        line["cpu_baseline"] = cpu_baseline(sc, stats["evaluations"], os.cpu_count() or 1)
    lib.propag_engine_destroy(eng)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
