"""TEST INFRASTRUCTURE ONLY -- how far the arrival times move between the
propagation's float arithmetics, measured with the CPU restatement.

The reference's time_from (crates/propag/src/propag.cu:269-294) calls CUDA's
atan2f and __cosf and is compiled with nvcc's default multiply-add
contraction (crates/propag/build.rs:48-69).  The CPU restatement runs in
three modes (oracle/propag_oracle.c): trig 0 = the portable cosine and
arctangent, every operation rounded on its own; trig 1 = libm's cosf/atan2f;
trig 2 = libm's cosf/atan2f and the three fused multiply-adds.  This script
runs the same scenario in two modes and reports, against the tolerance
max(0.5 s, 1e-4 t):

  * the fraction of burned cells whose times differ by more than it;
  * burned/unburned mismatches away from max_time (a cell burned in one run
    and not the other, its burned time below max_time minus the tolerance);
  * the largest deviation, and the number of cells whose reference differs.

Usage: python oracle/measure_arith.py [--sizes 1024,4096] [--modes 0,2]
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
# run as a script, this folder is first on the path and would shadow the package
sys.path[:] = [p for p in sys.path if os.path.abspath(p or ".") != HERE]
for p in (ROOT, os.path.join(ROOT, "propag-hidalgo_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)

from oracle import oracle as O  # noqa: E402
from py_propag import scenarios as S  # noqa: E402

FMAX = np.finfo(np.float32).max


def tolerance(t):
    return np.maximum(0.5, 1e-4 * np.abs(t))


def compare(a: O.OracleResult, b: O.OracleResult, max_time: float) -> dict:
    """Deviation of run b from run a (post-masked times)."""
    ta, tb = a.time.astype(np.float64), b.time.astype(np.float64)
    ba, bb = a.time < FMAX, b.time < FMAX
    both = ba & bb
    dev = np.abs(ta - tb)
    tol = tolerance(np.where(both, ta, 0.0))
    out_tol = both & (dev > tol)
    edge = max_time - tolerance(max_time)
    mask_mismatch = (ba != bb) & (np.where(ba, ta, tb) < edge)
    return dict(
        burned_a=int(ba.sum()), burned_b=int(bb.sum()),
        cells_outside_tolerance=int(out_tol.sum()),
        frac_outside_tolerance=float(out_tol.sum() / max(both.sum(), 1)),
        mask_mismatch_away_from_max_time=int(mask_mismatch.sum()),
        mask_mismatch_total=int((ba != bb).sum()),
        max_abs_dev_s=float(dev[both].max()) if both.any() else 0.0,
        max_rel_dev=float((dev[both] / np.maximum(ta[both], 1e-30)).max()) if both.any() else 0.0,
        cells_bitwise_different=int((a.time.view(np.uint32) != b.time.view(np.uint32)).sum()),
        refs_different=int(((a.refs_x != b.refs_x) | (a.refs_y != b.refs_y)).sum()),
    )


def scenario(size: int):
    if size <= 1024:
        return S.config0(size=size)
    return S.config1(size=size)


def fire_fields(sc):
    fields, _ = O.burn_f64(sc.terrain)
    f = fields.astype(np.float32)
    return f[:, 4].copy(), f[:, 5].copy(), f[:, 6].copy()


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--sizes", default="1024,4096")
    ap.add_argument("--modes", default="0,2")
    ap.add_argument("--tile", type=int, default=323)
    ap.add_argument("--threads", type=int, default=0)
    args = ap.parse_args()
    modes = [int(m) for m in args.modes.split(",")]
    for size in (int(s) for s in args.sizes.split(",")):
        sc = scenario(size)
        sp, az, ec = fire_fields(sc)
        runs = {}
        for m in modes:
            t0 = time.time()
            runs[m] = O.propagate(sc.width, sc.height, sc.dx, sc.dy, sc.max_time, sp, az, ec,
                                  sc.ignitions, tile=args.tile, full=2, trig=m, threads=args.threads)
            print(f"# {sc.name} trig={m}: {time.time() - t0:.1f} s, sweeps {runs[m].stats['sweeps']}",
                  file=sys.stderr, flush=True)
        base = modes[0]
        for m in modes[1:]:
            rep = dict(scenario=sc.name, tile=args.tile, modes=[base, m],
                       sweeps=[runs[base].stats["sweeps"], runs[m].stats["sweeps"]])
            rep.update(compare(runs[base], runs[m], sc.max_time))
            print(json.dumps(rep), flush=True)


if __name__ == "__main__":
    main()
