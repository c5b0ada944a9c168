#!/usr/bin/env python
"""Benchmark of the wildfire hot path (fire behaviour + arrival-time
propagation) on B200.

Headline workload: the large heterogeneous single scenario (4096 x 4096
cells at 5 m, ridged terrain up to 45 deg, 12 % non-burnable lakes and
roads, smooth random wind 0-15 m/s, per-cell moisture jitter, 20 ignitions,
max_time 43200 s), seeded synthetic inputs.  A step = fire behaviour over
every cell + boundaries + propagation + post mask for that scenario.

Batched legs: ``batched`` -- the 256-member ensemble on a shared 1024 x 1024
terrain (per-member wind, dead moisture and ignition, max_time 21600 s);
``batched_uneven`` -- 64 independent scenarios, square grids 128..2048 at
5-30 m with their own terrain.  Each: all jobs in one persistent launch
captured as a CUDA graph (cluster size from the autotuner), against the same
jobs run one by one through the plain path, with per-scenario latency.

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

# Propagation work of the full workloads (cell evaluations), as counted on the
# device by the engine in group mode (first sweeps over the pending cells
# only) and identically by the CPU restatement in the same mode (full=2; same
# schedule, bit-identical results).  The CPU legs time a bounded crop in that
# mode and scale by it; the GPU leg reports whether its own count still agrees.
WORK_EVALUATIONS = {"config1": 163488517}

# DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum) from
# one single-pass ncu capture of the full-size workload; the command and the
# figures are in profiles/dram_traffic_config1-4096.md.
DRAM_TRAFFIC = {"config1": {"engine_kernel": 988.88e6 + 348.53e6,
                            "fire_kernel": 558.02e6 + 181.39e6}}


def _log(msg: str) -> None:
    """Progress on stderr (the JSON line alone goes to stdout)."""
    print(f"[bench {time.strftime('%H:%M:%S')}] {msg}", file=sys.stderr, flush=True)


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


def max_over_ranks(value: float, world: int, dev) -> float:
    """The largest of every rank's value (all ranks call it at the same
    point); the value itself on one rank.  `dev` is the device of the
    reduction tensor: the GPU under NCCL, the CPU under gloo."""
    if world <= 1:
        return float(value)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


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
        import tempfile
        fd, self.path = tempfile.mkstemp(prefix="propag_clocks_", suffix=".csv")
        os.close(fd)
        try:
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


def _parallel(fn, terrain: dict, threads: int):
    """Runs a CPU fire-behaviour function over the cells in `threads` slices
    on as many threads (the ctypes calls release the GIL; every call builds
    its own fuel catalog)."""
    from concurrent.futures import ThreadPoolExecutor
    n = next(iter(terrain.values())).size
    cuts = np.linspace(0, n, threads + 1).astype(np.int64)
    parts = [{k: np.ascontiguousarray(v.ravel()[a:b]) for k, v in terrain.items()}
             for a, b in zip(cuts[:-1], cuts[1:]) if b > a]
    with ThreadPoolExecutor(max_workers=threads) as ex:
        list(ex.map(fn, parts))


def cpu_baseline(sc, evaluations_full: int, threads: int, budget_s: float = 20.0,
                 use_firelib_c: bool = False) -> dict:
    """Times the CPU path on this host's cores.

    Fire behaviour: the reference's own fireLib.c when asked and built (else
    the FP64 restatement) on a quarter of the workload's cells, on `threads`
    threads, scaled to all cells.  Propagation (the reference has none on the
    CPU): the CPU restatement of its kernel, in the engine's work-skipping
    mode (same schedule and results as whole-tile sweeps), timed on a crop
    of the workload around its first ignition and scaled by the full
    workload's recorded cell evaluations (an extrapolation, labelled as one);
    beside it, the whole 1024 x 1024 single-ignition scenario measured end to
    end, and the evaluation rate of the reference's own whole-tile sweeps
    (every cell of a tile in every sweep) on a 512 x 512 crop."""
    from oracle import oracle as O
    from py_propag import scenarios as S
    ncell = sc.width * sc.height
    k = max(threads, ncell // 4)
    samp = {kk: np.ascontiguousarray(v.ravel()[:k]) for kk, v in sc.terrain.items()}
    c_fire = use_firelib_c and O.have_firelib_c()
    fire_kind = "fireLib.c (reference)" if c_fire else "FP64 restatement"
    tf = time.perf_counter()
    _parallel(O.burn_firelib_c if c_fire else O.burn_f64, samp, threads)
    fire_s = (time.perf_counter() - tf) * (ncell / k)

    def fire_fields(t):
        f, _ = O.burn_f64(t)
        return f[:, 4].astype(np.float32), f[:, 5].astype(np.float32), f[:, 6].astype(np.float32)

    # the workload's own evaluation rate, on a 1024 x 1024 crop around its
    # first ignition
    crop = min(1024, sc.width, sc.height)
    cx, cy = sc.ignitions[0][0], sc.ignitions[0][1]
    x0 = int(min(max(cx - crop // 2, 0), sc.width - crop))
    y0 = int(min(max(cy - crop // 2, 0), sc.height - crop))
    sub = {kk: np.ascontiguousarray(v[y0:y0 + crop, x0:x0 + crop]) for kk, v in sc.terrain.items()}
    sp, az, ec = fire_fields(sub)
    ign = [(x - x0, y - y0, t) for (x, y, t) in sc.ignitions if x0 <= x < x0 + crop and y0 <= y < y0 + crop]
    tp = time.perf_counter()
    rc = O.propagate(crop, crop, sc.dx, sc.dy, sc.max_time, sp, az, ec, ign, tile=323,
                     threads=threads, full=2, trig=2)
    prop_rate = rc.stats["evaluations"] / (time.perf_counter() - tp)
    prop_s = evaluations_full / prop_rate
    # the whole 1024 x 1024 single-ignition scenario, end to end
    c0 = S.config0(size=1024)
    sp, az, ec = fire_fields(c0.terrain)
    tp = time.perf_counter()
    r0 = O.propagate(c0.width, c0.height, c0.dx, c0.dy, c0.max_time, sp, az, ec, c0.ignitions,
                     tile=323, threads=threads, full=2, trig=2)
    c0_s = time.perf_counter() - tp
    half = 512
    x0 = y0 = int(c0.ignitions[0][0]) - half // 2
    sub = {kk: np.ascontiguousarray(v[y0:y0 + half, x0:x0 + half]) for kk, v in c0.terrain.items()}
    sp2, az2, ec2 = fire_fields(sub)
    tp = time.perf_counter()
    r1 = O.propagate(half, half, c0.dx, c0.dy, c0.max_time, sp2, az2, ec2,
                     [(half // 2, half // 2, 0.0)], tile=323, threads=threads, full=1, trig=2)
    full_rate = r1.stats["evaluations"] / (time.perf_counter() - tp)
    return {"value": 1.0 / (fire_s + prop_s), "unit": UNIT, "cores": threads,
            # the propagation (over 95 % of the time) is always the CPU restatement
            "kind": "port",
            "sample": (f"fire behaviour: {fire_kind} on {k} of {ncell} cells on {threads} threads, "
                       f"scaled; propagation: CPU restatement of propag.cu (the reference has no CPU "
                       f"propagation), {prop_rate:.3g} cell evaluations/s on {threads} threads "
                       f"(work-skipping sweeps) timed on a {crop}x{crop} crop around the first "
                       f"ignition and extrapolated to the full scenario's {evaluations_full} "
                       f"evaluations"),
            "fire_s": fire_s, "propagation_s": prop_s,
            "config0_measured": {"value": 1.0 / c0_s, "unit": "scenarios/s (propagation only)",
                                 "evaluations": r0.stats["evaluations"], "seconds": c0_s},
            "reference_schedule": {"evaluations_per_s": full_rate,
                                   "note": "whole-tile sweeps as the reference runs them (every cell "
                                           "of the tile in every sweep), 512x512 crop of config 0; "
                                           "same results, far more evaluations"}}


def run_reference(args):
    """The reference's CPU implementation of the path on this host's cores:
    its own fireLib.c for fire behaviour when it was built here (oracle/_ref),
    and the CPU restatement of its propagation kernel."""
    rank, world, _ = _rank_env()
    if rank != 0:
        return
    sc, desc = _workload(args.workload)
    threads = os.cpu_count() or 1
    evals = WORK_EVALUATIONS.get(args.workload)
    if evals is None:
        raise SystemExit(f"no recorded propagation work for workload {args.workload}")
    vals = []
    cb = None
    for i in range(args.warmup + args.steps):
        cb = cpu_baseline(sc, evals, threads, use_firelib_c=True)
        if i >= args.warmup:
            vals.append(cb["value"])
    v = float(np.median(vals))
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "config": {"workload": desc}, "dtype": "f32", "data": "synthetic",
            "cpu_baseline": dict(cb, value=v),
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def serve_leg(lib, L, pp, dev, master, seconds: float, rate: float, budget_gb: float,
              check_every: int = 10, cap_requests: int = 1000) -> dict:
    """Serving loop: Poisson arrivals of window requests cut from a
    device-resident master terrain, submitted to a continuous-batching server
    as they arrive; latency = submit to done (host clock).  Every
    `check_every`-th request's served arrival times are kept on the host, and
    after the run the same requests are re-run alone through the plain path
    and compared bit for bit.  Capacity: the first `cap_requests` requests
    again, closed loop with 32 outstanding."""
    import torch
    from py_propag import scenarios as S
    from py_propag.batches import device_jobs
    reqs = S.config4_requests(master["fuel_code"], seconds=seconds, rate=rate)
    H, W = master["fuel_code"].shape
    mt = {k: torch.from_numpy(np.ascontiguousarray(v)).to(dev) for k, v in master.items()}
    prep = torch.cuda.Stream(dev)
    torch.cuda.empty_cache()
    free, _ = torch.cuda.mem_get_info(dev)
    # the server reserves its budget up front; requests' own buffers (inputs,
    # fire rasters, outputs) need room beside it
    # (the server adds its slot scratch, about 2.6 GB, to the budget)
    budget = int(max(min(budget_gb * 1e9, free - 45e9), 8e9))
    srv = pp.Server(hbm_budget=budget, lanes=4, max_batch=64)
    try:
        return _serve(srv, lib, L, torch, dev, reqs, mt, prep, W, H, seconds, rate, budget,
                      check_every, cap_requests, device_jobs)
    finally:
        srv.close()  # the dispatcher thread must stop before the process exits


def _serve(srv, lib, L, torch, dev, reqs, mt, prep, W, H, seconds, rate, budget, check_every,
           cap_requests, device_jobs):
    keep, res, served = {}, {}, {}

    def make(i, r):
        n, x0, y0 = r["size"], r["x0"], r["y0"]
        with torch.cuda.stream(prep):
            t = {k: v[y0:y0 + n, x0:x0 + n].contiguous().view(-1) for k, v in mt.items()}
            t["wind_speed"] = torch.full((n * n,), r["wind_speed"], dtype=torch.float32, device=dev)
            t["wind_azimuth"] = torch.full((n * n,), r["wind_azimuth"], dtype=torch.float32, device=dev)
            for k in ("d1hr", "d10hr", "d100hr"):
                t[k] = t[k] + np.float32(r["dead_offset"])
            (jobs, terrains, kp) = device_jobs(L, dev, [(n, n, 5.0, 5.0, r["max_time"], 0,
                                                         [r["ignition"]], t)])
        prep.synchronize()
        return jobs[0], terrains[0], kp

    def collect(block=False, check=True):
        for rid in list(keep):
            out = srv.wait(rid, 120_000) if block else srv.poll(rid)
            if block and out is None:
                raise RuntimeError(f"serving: request {rid} not done after 120 s")
            if out is not None:
                res[rid] = out
                i = keep[rid][3]
                if check and i % check_every == 0:
                    served[i] = keep[rid][2][0][3].cpu().numpy()
                del keep[rid]
                srv.release(rid)

    t_start = time.perf_counter()
    ids = []
    overloaded = None
    _log(f"serving: {len(reqs)} requests over {seconds:g} s, budget {budget / 1e9:.0f} GB")
    for i, r in enumerate(reqs):
        while time.perf_counter() - t_start < r["arrival"]:
            collect()
            time.sleep(0.0005)
        if len(keep) > 64:  # the server falls behind the arrivals: stop offering
            overloaded = i
            _log(f"serving: {len(keep)} requests outstanding at request {i}; arrivals stopped")
            break
        if i % 500 == 0:
            _log(f"serving: request {i}, {len(keep)} outstanding")
        job, terr, kp = make(i, r)
        rid = srv.submit(job, terr)
        ids.append(rid)
        keep[rid] = (job, terr, kp, i)
    collect(block=True)
    n_req = len(ids)
    lat = np.array([(res[r]["done_ns"] - res[r]["submit_ns"]) / 1e6 for r in ids])
    span = (max(res[r]["done_ns"] for r in ids) - min(res[r]["submit_ns"] for r in ids)) / 1e9
    _log("serving: open loop done; capacity run")
    # capacity: the first requests again, closed loop with 32 outstanding
    cap_ids = []
    n_cap = min(len(reqs), cap_requests)
    t_cap = time.perf_counter()
    for i, r in enumerate(reqs[:n_cap]):
        while len(keep) >= 32:
            collect(check=False)
            time.sleep(0.0002)
        job, terr, kp = make(i, r)
        rid = srv.submit(job, terr)
        cap_ids.append(rid)
        keep[rid] = (job, terr, kp, i)
    collect(block=True, check=False)
    capacity = n_cap / (time.perf_counter() - t_cap)
    cap_batch = float(np.mean([res[r]["batch_size"] for r in cap_ids]))
    srv.close()
    _log(f"serving: capacity done; {len(served)} requests re-run alone")
    # the checked requests alone through the plain path
    eng = lib.propag_engine_create(C.byref(L.PropagOptions(0, 0, 0, -1)))
    sptr = C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    same = True
    for i, times in served.items():
        job, terr, kp = make(i, reqs[i])
        if lib.propag_fire_simple_device(job.width * job.height, C.byref(terr), job.speed_max,
                                         job.azimuth_max, job.eccentricity, sptr) or \
                lib.propag_engine_run(eng, C.byref(job), 1, sptr, None):
            raise RuntimeError(L.last_error())
        torch.cuda.synchronize()
        same &= bool(np.array_equal(times.view(np.uint32), kp[0][3].cpu().numpy().view(np.uint32)))
        del kp
    lib.propag_engine_destroy(eng)
    sizes = np.array([r["size"] for r in reqs])
    return {
        "workload": (f"config4: Poisson arrivals at {rate:g}/s for {seconds:g} s ({n_req} requests"
                     + (f" of {len(reqs)}: arrivals stopped when 64 requests were outstanding"
                        if overloaded is not None else "")
                     + "), "
                     f"windows {sizes.min()}..{sizes.max()} square from a device-resident "
                     f"{W}x{H} master terrain, per-request wind/moisture/ignition, 1-12 h, "
                     f"HBM budget {budget / 1e9:.0f} GB of engine scratch reserved by the server"),
        "value": n_req / span, "unit": UNIT, "offered_rate": rate,
        "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                       "max": float(lat.max())},
        "batch_size_mean": float(np.mean([res[r]["batch_size"] for r in ids])),
        "capacity": {"value": capacity, "unit": UNIT, "batch_size_mean": cap_batch, "requests": n_cap,
                     "note": "the first requests again, closed loop with 32 outstanding (host wall "
                             "clock, request preparation included)"},
        "matches_plain_bitwise": same, "checked_alone": len(served),
        "fell_behind_at_s": (None if overloaded is None else float(reqs[overloaded]["arrival"])),
        "server": "4 streams, continuous batching (requests admitted while earlier batches run)",
    }


def batched_leg(lib, L, pp, stream, batch, desc, steps, warmup, plain_jobs) -> dict:
    """All jobs of a batch in one persistent launch, captured as a CUDA graph
    with the cluster size the autotuner picks, against the plain path: each
    job alone (its fire pass + a one-job engine run), one after another."""
    import torch
    jobs, terrains, keep = batch
    sptr = C.c_void_p(stream.cuda_stream)
    eng = lib.propag_engine_create(C.byref(L.PropagOptions(0, 0, 0, -1)))
    if not eng:
        raise RuntimeError(L.last_error())
    arr = (L.PropagJob * len(jobs))(*jobs)

    def plain_one(i):
        j = jobs[i]
        if lib.propag_fire_simple_device(j.width * j.height, C.byref(terrains[i]), j.speed_max,
                                         j.azimuth_max, j.eccentricity, sptr):
            raise RuntimeError(L.last_error())
        p = C.cast(C.addressof(arr) + i * C.sizeof(L.PropagJob), C.POINTER(L.PropagJob))
        if lib.propag_engine_run(eng, p, 1, sptr, None):
            raise RuntimeError(L.last_error())

    plain_jobs = min(plain_jobs, len(jobs))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    plain_one(0)
    torch.cuda.synchronize()
    plain_ms, plain_out = [], []
    for i in range(plain_jobs):
        e0.record(stream)
        plain_one(i)
        e1.record(stream)
        torch.cuda.synchronize()
        plain_ms.append(e0.elapsed_time(e1))
        plain_out.append(keep[i][3].clone())
    lib.propag_engine_destroy(eng)
    # batched: autotuned cluster size, one CUDA graph replayed per batch
    best, tune_ms = pp.autotune(jobs, terrains, stream=stream.cuda_stream, repeats=1)
    g = pp.Graph(jobs, terrains, cluster=best["cluster"])
    for _ in range(warmup):
        g.launch(stream.cuda_stream)
    torch.cuda.synchronize()
    step_ms = []
    for _ in range(steps):
        e0.record(stream)
        g.launch(stream.cuda_stream)
        e1.record(stream)
        torch.cuda.synchronize()
        step_ms.append(e0.elapsed_time(e1))
    st = g.stats(stream.cuda_stream)
    g.close()
    same = all(torch.equal(plain_out[i], keep[i][3]) for i in range(plain_jobs))
    t0 = min(s["t_start_ns"] for s in st)
    batch_ms = float(np.median(step_ms))
    fire_prep_ms = batch_ms - (max(s["t_done_ns"] for s in st) - t0) / 1e6
    lat = np.array([(s["t_done_ns"] - t0) / 1e6 + max(fire_prep_ms, 0.0) for s in st])
    batched = len(jobs) / (batch_ms / 1e3)
    plain = len(plain_ms) / (float(np.sum(plain_ms)) / 1e3)
    return {
        "workload": desc, "value": batched, "unit": UNIT, "ms_per_batch": batch_ms,
        "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                       "note": "batch start to each job's propagation end (device clock), "
                               "plus the batch's fire/prep time"},
        "plain": {"value": plain, "unit": UNIT, "jobs_timed": len(plain_ms),
                  "latency_ms": {"p50": float(np.percentile(plain_ms, 50)),
                                 "p99": float(np.percentile(plain_ms, 99))}},
        "speedup_vs_plain": batched / plain,
        "matches_plain_bitwise": bool(same),
        "graph": "fire passes + one persistent propagation launch, captured once, replayed per batch",
        "autotuned": {"cluster": best["cluster"], "tuning_ms": tune_ms},
        "gpu_launches_per_batch": len(jobs) + 4,
        "sweeps_mean": float(np.mean([s["sweeps"] for s in st])),
        "evaluations": int(sum(s["evaluations"] for s in st)),
    }


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
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--ensemble", type=int, default=256, help="members of the ensemble leg (0 = skip)")
    ap.add_argument("--uneven", type=int, default=64, help="scenarios of the uneven leg (0 = skip)")
    ap.add_argument("--serve-seconds", type=float, default=30.0,
                    help="length of the serving leg's arrival stream (0 = skip)")
    ap.add_argument("--serve-only", action="store_true",
                    help="run the serving leg alone and print its JSON object (the main run "
                         "starts it so, in a child process with a time limit)")
    ap.add_argument("--serve-terrain", default="",
                    help="with --serve-only: .npz of the master terrain (else it is generated)")
    ap.add_argument("--serve-rate", type=float, default=20.0, help="serving arrivals per second")
    ap.add_argument("--plain-members", type=int, default=256,
                    help="ensemble members timed one by one on the plain path")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.warmup < 0 or args.steps < 1:
        raise SystemExit("--steps >= 1 and --warmup >= 0")
    if args.serve_only:
        return serve_only(args)
    bench_b200(args)


def serve_only(args):
    """The serving leg on its own (config 4 on the 4096^2 master terrain)."""
    import torch

    import py_propag as pp
    from py_propag import _lib as L
    from py_propag import scenarios as S
    dev = torch.device("cuda", torch.cuda.current_device())
    if args.serve_terrain:
        with np.load(args.serve_terrain) as z:
            master = {k: z[k] for k in z.files}
    else:
        master = S.config1(size=4096).terrain
    # The server reserves its budget up front; the requests' own buffers
    # (terrain windows, fire rasters, outputs: up to 1 GB each, dozens in
    # flight) need the rest of the device, so the budget is well below
    # config 4's 150 GB, which this device could not hold beside them.
    res = serve_leg(L.lib(), L, pp, dev, master, args.serve_seconds, args.serve_rate, 60.0)
    print(json.dumps(res), flush=True)


def serving_child(args, terrain: dict) -> dict:
    """Runs the serving leg in a child process with a time limit, so that a
    server that falls behind its arrivals (config 4's windows reach 4096^2,
    a quarter of them 2048^2 or more) cannot stall the benchmark."""
    import tempfile
    limit = args.serve_seconds + 240.0
    with tempfile.TemporaryDirectory(prefix="propag_serve_") as tmp:
        path = os.path.join(tmp, "master.npz")
        np.savez(path, **terrain)
        cmd = [sys.executable, os.path.abspath(__file__), "--serve-only", "--serve-seconds",
               str(args.serve_seconds), "--serve-rate", str(args.serve_rate), "--serve-terrain", path]
        try:
            out = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=None, text=True, timeout=limit)
        except subprocess.TimeoutExpired:
            return {"unavailable": f"the serving run did not finish within {limit:.0f} s"}
    lines = [x for x in out.stdout.splitlines() if x.startswith("{")]
    if out.returncode != 0 or not lines:
        return {"unavailable": f"the serving run failed (exit {out.returncode})"}
    return json.loads(lines[-1])


def bench_b200(args):
    import torch
    import torch.distributed as dist

    import py_propag as pp
    from py_propag import _lib as L
    from py_propag.batches import ensemble_batch, uneven_batch

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
    eng = lib.propag_engine_create(C.byref(L.PropagOptions(args.tile, args.cluster, 0, -1)))
    if not eng:
        raise RuntimeError(L.last_error())
    stream = torch.cuda.current_stream(dev)
    sptr = C.c_void_p(stream.cuda_stream)

    def fire_pass():
        if lib.propag_fire_simple_device(N, C.byref(ptrs), fire[0].data_ptr(), fire[1].data_ptr(),
                                         fire[2].data_ptr(), sptr):
            raise RuntimeError(L.last_error())

    def step(stats=None):
        fire_pass()
        if lib.propag_engine_run(eng, C.byref(job), 1, sptr, stats):
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
        fire_pass()
        ev_fire[i][1].record(stream)
        if lib.propag_engine_run(eng, C.byref(job), 1, sptr, None):
            raise RuntimeError(L.last_error())
        ev_step[i][1].record(stream)
        ms = (C.c_float * 3)()
        lib.propag_engine_last_times(eng, ms)  # waits for this step
        eng_ms.append(list(ms))
    t_all1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    total_ms = max_over_ranks(t_all0.elapsed_time(t_all1), world, dev)
    step_ms = [a.elapsed_time(b) for a, b in ev_step]
    fire_ms = [a.elapsed_time(b) for a, b in ev_fire]
    prop_ms = [m[1] for m in eng_ms]
    value = world * args.steps / (total_ms / 1e3)
    dev_time = time_d.cpu().numpy()

    e2e = None
    if not args.no_e2e:
        _log("end-to-end leg ...")
        e2e = e2e_leg(lib, L, pp, sc, args, world, dev, dev_time)

    peak, peak_kind = _peaks()
    prop_bytes = 20 * stats["evaluations"] + 8 * stats["improvements"] + 4 * stats["gathers"]
    prop_s = float(np.mean(prop_ms)) / 1e3
    fire_s = float(np.mean(fire_ms)) / 1e3
    ach = prop_bytes / prop_s / 1e9
    fire_ach = FIRE_BYTES_PER_CELL * N / fire_s / 1e9
    known = WORK_EVALUATIONS.get(args.workload)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": desc, "cells": N, "tile": args.tile or 323, "cluster": args.cluster,
                   "l2": "inputs larger than L2 (terrain 37 B/cell, 620 MB at 4096^2)",
                   "parallelism": "replicas" if world > 1 else "single"},
        "latency_ms": {"p50": float(np.percentile(step_ms, 50)), "p99": float(np.percentile(step_ms, 99)),
                       "fire_kernel": float(np.mean(fire_ms)), "propagation_kernel": float(np.mean(prop_ms)),
                       "prep": float(np.mean([m[0] for m in eng_ms])),
                       "post": float(np.mean([m[2] for m in eng_ms]))},
        "cells_per_s": N * world * args.steps / (total_ms / 1e3),
        "e2e": e2e,
        "roofline": {"bound": "hbm", "kernel": "engine_kernel (propagation)", "achieved": ach,
                     "peak": peak, "unit": "GB/s", "frac": ach / peak,
                     "traffic": DRAM_TRAFFIC.get(args.workload, {}).get("engine_kernel"),
                     "algorithmic_bytes": prop_bytes, "peak_source": peak_kind,
                     "cell_updates_per_s": stats["evaluations"] / prop_s,
                     "sweeps": stats["sweeps"],
                     "bytes_per_sweep": prop_bytes / max(1, stats["sweeps"]),
                     "full_grid_bytes_per_sweep": 20 * N},
        "kernels": {"fire_kernel": {"achieved": fire_ach, "peak": peak, "unit": "GB/s",
                                    "frac": fire_ach / peak, "bytes": FIRE_BYTES_PER_CELL * N,
                                    "traffic": DRAM_TRAFFIC.get(args.workload, {}).get("fire_kernel")}},
        "workload_stats": stats,
        "work_matches_recorded": (stats["evaluations"] == known) if known else None,
        "gpu_launches": 5 * args.steps,
        "clocks": clk,
    }
    lib.propag_engine_destroy(eng)
    del t_dev, fire, time_d, rx_d, ry_d, bnd_d
    if args.ensemble > 0:
        batch, bdesc = ensemble_batch(L, dev, args.ensemble)
        _log("batched leg ...")
        line["batched"] = batched_leg(lib, L, pp, stream, batch, bdesc, args.steps, args.warmup,
                                      args.plain_members)
        del batch
    if args.uneven > 0:
        batch, bdesc = uneven_batch(L, dev, args.uneven)
        _log("uneven batch leg ...")
        line["batched_uneven"] = batched_leg(lib, L, pp, stream, batch, bdesc, args.steps,
                                             args.warmup, args.uneven)
        del batch
    if args.serve_seconds > 0 and args.workload == "config1":
        _log("serving leg ...")
        torch.cuda.synchronize()
        torch.cuda.empty_cache()  # the child reserves most of the device for its server
        line["serving"] = serving_child(args, sc.terrain)
    if rank == 0 and not args.no_cpu:
        _log("CPU baseline ...")
        line["cpu_baseline"] = cpu_baseline(sc, stats["evaluations"], os.cpu_count() or 1)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def e2e_leg(lib, L, pp, sc, args, world, dev, dev_time):
    """The same metric through the C-ABI host entry point (propag_run_host):
    pinned host inputs copied in and results copied out inside the timed
    region, every step."""
    import torch
    import torch.distributed as dist
    N = sc.width * sc.height
    words = (N + 31) // 32
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
        if lib.propag_run_host(C.byref(settings), C.byref(hptrs), ign_arr, len(sc.ignitions),
                               C.byref(hopt), out_t.data_ptr(), out_rx.data_ptr(), out_ry.data_ptr(),
                               out_b.data_ptr(), None):
            raise RuntimeError(L.last_error())

    for _ in range(max(1, args.warmup)):
        e2e_step()
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    e2e_s = max_over_ranks(time.perf_counter() - t0, world, dev)
    same = np.array_equal(out_t.numpy().view(np.uint32), dev_time.view(np.uint32))
    return {"value": world * args.steps / e2e_s, "unit": UNIT,
            "h2d_bytes_per_step": N * 37 + len(sc.ignitions) * 12,
            "d2h_bytes_per_step": N * 4 + N * 4 + words * 4, "matches_device_path": bool(same),
            "note": "propag_run_host: pinned host terrain in, times/refs/boundaries out, "
                    "fire + propagation on the device, wall clock"}


if __name__ == "__main__":
    main()
