"""Generates tests/golden/firelib_c_golden.npz: fire-behaviour outputs of the
reference's own C fireLib (crates/firelib-sys/fireLib.c, compiled from the
reference sources by oracle/Makefile into oracle/_ref/) on seeded terrains,
driven the way the reference's quickcheck harness drives it
(crates/firelib/src/lib.rs:312-367).

Run in a checkout where the reference sources exist:
    python tests/golden/make_firelib_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from conftest import random_terrain  # noqa: E402
from oracle import oracle as O  # noqa: E402


def main():
    O.build()
    parts = [random_terrain(1000, 101, quickcheck=True), random_terrain(1000, 102, quickcheck=False)]
    terrain = {k: np.concatenate([p[k] for p in parts]) for k in parts[0]}
    # codes 14..15 of the realistic set have no model in fireLib's standard
    # catalog of 13: keep them (both sides give no fire)
    out = O.burn_firelib_c(terrain)
    np.savez_compressed(os.path.join(HERE, "firelib_c_golden.npz"), outputs=out,
                        **{k: np.asarray(v) for k, v in terrain.items()})
    print("wrote", out.shape)


if __name__ == "__main__":
    main()
