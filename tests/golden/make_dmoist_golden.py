"""Generates tests/golden/dmoist_fixtures.npz from the reference's dmoist
fixture files (crates/dmoist/fixtures/*.txt), parsed the way the
reference's own tests parse them (crates/dmoist/src/lib.rs:725-811): lines
"(p0, p1, ...) -> result", "[month] + range(6) -> result" (precipitation
0..5 mm on the six days) and "(month,) -> result"; comment and malformed
lines are skipped.  The wind files have no test in the reference; their
"u, v -> value" lines (with or without parentheses) are kept as well.

Run where the reference sources exist ($PROPAG_REFERENCE, else a
`reference` folder beside this repository):
    python tests/golden/make_dmoist_golden.py
"""
import os
import re

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REFERENCE = os.environ.get("PROPAG_REFERENCE") or os.path.join(HERE, "..", "..", "..", "reference")
FIXTURES = os.path.join(REFERENCE, "crates", "dmoist", "fixtures")

FILES = {
    "hcb": "hcb.txt",
    "hcb_shading": "corrige_hcb_por_sombreado.txt",
    "prob_precip": "corrige_prob_por_pp.txt",
    "d1hr": "d1hr.txt",
    "max_precip": "efecto_precipitacion_maximo.txt",
    "x10hr": "hco_x10hr.txt",
    "live": "humedad_vivo.txt",
    "prob_ign": "probabilidad_ignicion.txt",
    "shading": "sombreado.txt",
    "wind_speed": "mod_viento.txt",
    "wind_dir": "dir_viento.txt",
}


def parse(name, text):
    rows = []
    for line in text.splitlines():
        line = line.strip()
        if not line or line.startswith("#") or " -> " not in line:
            continue
        left, right = (s.strip() for s in line.split(" -> ", 1))
        m = re.fullmatch(r"\[(-?\d+)\] \+ range\(6\)", left)
        if m:
            rows.append(([float(m.group(1))], float(right)))
            continue
        wind = name.startswith("wind")
        if left.startswith("(") and left.endswith(")"):
            inner = left[1:-1].rstrip(",")
        elif wind:
            inner = left
        else:
            continue  # the reference's parser skips it
        rows.append(([float(v) for v in inner.split(",")], float(right)))
    return rows


def main():
    out = {}
    for key, fname in FILES.items():
        with open(os.path.join(FIXTURES, fname)) as f:
            rows = parse(key, f.read())
        k = max(len(p) for p, _ in rows)
        params = np.array([p + [np.nan] * (k - len(p)) for p, _ in rows], dtype=np.float64)
        out[key + "_params"] = params
        out[key + "_expected"] = np.array([r for _, r in rows], dtype=np.float64)
        print(key, params.shape)
    np.savez_compressed(os.path.join(HERE, "dmoist_fixtures.npz"), **out)


if __name__ == "__main__":
    main()
