"""Pins of the CPU oracles (no GPU needed).

* The FP64 fire-behaviour restatement against the reference's own C fireLib:
  the committed golden vectors (tests/golden/firelib_c_golden.npz, made by
  tests/golden/make_firelib_golden.py from the compiled reference sources)
  and, where the reference checkout is present, live runs.
* The propagation restatement: its work-skipping mode against full sweeps,
  the README demo of the reference (crates/propag README.md:94-112), the
  directed-rounding emulation and the portable trig functions.
"""
import os
from fractions import Fraction

import numpy as np
import pytest

from conftest import random_terrain

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "firelib_c_golden.npz")
FIELDS = ("rx_int", "speed0", "hpua", "phi_eff_wind", "speed_max", "azimuth_max",
          "eccentricity", "residence_time", "byrams_max", "flame_max")


def _golden():
    d = np.load(GOLDEN)
    terrain = {k: d[k] for k in ("fuel_code", "d1hr", "d10hr", "d100hr", "herb", "wood",
                                 "wind_speed", "wind_azimuth", "slope", "aspect")}
    return terrain, d["outputs"]


def test_fp64_restatement_matches_firelib_c_golden(oracle):
    """Codes >= 14 are outside the standard catalog (no fire on both sides).
    Code 13 is left out: the reference's GPU path uses the Rust catalog,
    whose NFFL13 10-h load is 0.0580 lb/ft2 (crates/firelib/src/lib.rs:256-266)
    where fireLib.c has 1.0580 (crates/firelib-sys/fireLib.c:1316); the
    reference's own equivalence property draws codes 0..12 only."""
    terrain, c_out = _golden()
    ours, _ = oracle.burn_f64(terrain)
    keep = terrain["fuel_code"] != 13
    ours, c_out = ours[keep], c_out[keep]
    for k, name in enumerate(FIELDS):
        a, b = ours[:, k], c_out[:, k]
        if name == "azimuth_max":
            d = np.abs(np.angle(np.exp(1j * (a - b))))
            moving = c_out[:, 4] >= 0.00508  # reference excuses speed_max < 1 ft/min
            assert np.max(d[moving], initial=0) < 1e-6, name
        else:
            rel = np.abs(a - b) / np.maximum(np.abs(b), 1e-12)
            assert np.max(np.where(np.abs(b) > 1e-9, rel, np.abs(a - b))) < 1e-9, name


def test_reference_bar_on_quickcheck_terrains(oracle):
    """The reference's own property (crates/firelib/src/lib.rs:295-302): abs
    1e-2 or rel 2e-2 in imperial units; here on the golden set it holds for
    every cell and every field."""
    terrain, c_out = _golden()
    ours, _ = oracle.burn_f64(terrain)
    keep = terrain["fuel_code"] != 13
    ours, c_out = ours[keep], c_out[keep]
    to_imp = {"speed_max": 1 / 0.00508, "speed0": 1 / 0.00508, "eccentricity": 1.0,
              "phi_eff_wind": 1.0}
    for name, f in to_imp.items():
        k = FIELDS.index(name)
        a, b = ours[:, k] * f, c_out[:, k] * f
        d = np.abs(a - b)
        ok = (d < 1e-2) | (d / np.maximum(np.minimum(np.abs(a), np.abs(b)), 1e-30) < 2e-2)
        assert ok.all(), name


def test_live_firelib_c_when_reference_present(oracle):
    if not oracle.have_firelib_c():
        pytest.skip("reference fireLib.c not built here")
    t = random_terrain(5000, 7, quickcheck=True)
    ours, _ = oracle.burn_f64(t)
    c = oracle.burn_firelib_c(t)
    rel = np.abs(ours[:, 4] - c[:, 4]) / np.maximum(np.abs(c[:, 4]), 1e-12)
    assert np.max(rel[c[:, 4] > 1e-9]) < 1e-9


def test_nffl13_follows_the_rust_catalog(oracle):
    """Only NFFL13 differs from fireLib.c, and only through its 10-h load."""
    terrain, c_out = _golden()
    ours, _ = oracle.burn_f64(terrain)
    is13 = terrain["fuel_code"] == 13
    assert is13.sum() > 0
    diff = np.any(np.abs(ours - c_out) > 1e-6 * np.maximum(np.abs(c_out), 1.0), axis=1)
    assert not np.any(diff & ~is13)
    cat = oracle.catalog_f64()
    assert cat[13, 0] > 0


@pytest.mark.parametrize("quickcheck", [True, False])
def test_live_firelib_c_with_the_rust_nffl13_load(oracle, quickcheck):
    """With NFFL13's 10-h dead load set to the Rust catalog's value inside
    fireLib.c (its surface area follows), the FP64 restatement equals the
    reference's C fireLib on every fuel code, NFFL13 included, to ~1e-13 in
    every field: that one catalog entry is the whole difference."""
    if not oracle.have_firelib_c():
        pytest.skip("reference fireLib.c not built here")
    t = random_terrain(20_000, 9, quickcheck=quickcheck)
    t["fuel_code"][::3] = 13
    ours, _ = oracle.burn_f64(t)
    c = oracle.burn_firelib_c(t, rust_nffl13=True)
    for k, name in enumerate(FIELDS):
        a, b = ours[:, k], c[:, k]
        if name == "azimuth_max":
            d = np.abs(np.angle(np.exp(1j * (a - b))))
            assert np.max(d[c[:, 4] >= 0.00508], initial=0) < 1e-6, name
        else:
            err = np.where(np.abs(b) > 1e-9, np.abs(a - b) / np.maximum(np.abs(b), 1e-12), np.abs(a - b))
            assert np.max(err) < 1e-12, name
    plain = oracle.burn_firelib_c(t)
    is13 = t["fuel_code"] == 13
    moved = np.any(np.abs(plain - c) > 1e-9 * np.maximum(np.abs(c), 1.0), axis=1)
    assert np.array_equal(moved & ~is13, np.zeros_like(moved)) and moved[is13].mean() > 0.5


def test_no_fire_codes(oracle):
    t = random_terrain(64, 8)
    t["fuel_code"][:] = np.array([0, 14, 19, 20, 255, 1, 13, 7], np.uint8)[np.arange(64) % 8]
    out, sit = oracle.burn_f64(t)
    none = np.isin(t["fuel_code"], [0, 14, 19, 20, 255])
    assert np.all(out[none] == 0) and np.all(sit[none] == -1)
    assert np.all(sit[~none] >= 0)


def test_catalog_sanity(oracle):
    cat = oracle.catalog_f64()
    assert cat[0, 0] == 0 and all(cat[i, 0] > 0 for i in range(1, 14))
    assert np.all(cat[14:, 0] == 0)
    # NFFL01: one dead particle, sigma = savr 3500
    assert abs(cat[1, 1] - 3500.0) < 1e-9
    assert np.all(cat[1:14, 3] > 0) and np.all(cat[1:14, 5] > 0)


# ---------------------------------------------------------------- propag ----

def _scenario(size, kind, seed=0):
    from py_propag import scenarios as S
    return S.config0(size=size, seed=seed) if kind == 0 else S.config1(size=size, seed=seed, n_ign=4, max_time=9000.0)


@pytest.mark.parametrize("size,kind,tile", [(96, 0, 0), (96, 0, 31), (120, 1, 0), (120, 1, 50), (90, 1, 19)])
def test_work_skipping_equals_full_sweeps(oracle, size, kind, tile):
    sc = _scenario(size, kind, seed=3)
    f, _ = oracle.burn_f64(sc.terrain)
    sp, az, ec = (f[:, k].astype(np.float32) for k in (4, 5, 6))
    a = oracle.propagate(sc.width, sc.height, sc.dx, sc.dy, sc.max_time, sp, az, ec, sc.ignitions, tile=tile)
    b = oracle.propagate(sc.width, sc.height, sc.dx, sc.dy, sc.max_time, sp, az, ec, sc.ignitions,
                         tile=tile, full=True)
    assert np.array_equal(a.time_raw.view(np.uint32), b.time_raw.view(np.uint32))
    assert np.array_equal(a.refs_x, b.refs_x) and np.array_equal(a.refs_y, b.refs_y)
    for k in ("rounds", "launches", "sweeps", "improvements"):
        assert a.stats[k] == b.stats[k], k
    assert a.stats["evaluations"] < b.stats["evaluations"]


@pytest.mark.parametrize("size,kind,tile,north_up", [(96, 0, 31, False), (120, 1, 50, False),
                                                     (120, 1, 19, True), (150, 1, 37, False),
                                                     (96, 0, 0, False)])
def test_first_sweep_skipping_equals_full_sweeps(oracle, size, kind, tile, north_up):
    """full = 2: a launch's first sweep evaluates only the cells whose inputs
    changed since their last evaluation (grid-wide pending bitmap, referrer
    boxes scanned whole): same times, references and schedule as evaluating
    every cell, with fewer evaluations when there are several tiles."""
    sc = _scenario(size, kind, seed=5)
    dy = -sc.dy if north_up else sc.dy
    f, _ = oracle.burn_f64(sc.terrain)
    sp, az, ec = (f[:, k].astype(np.float32) for k in (4, 5, 6))
    runs = [oracle.propagate(sc.width, sc.height, sc.dx, dy, sc.max_time, sp, az, ec, sc.ignitions,
                             tile=tile, full=m) for m in (1, 0, 2)]
    full, skip, skip2 = runs
    for r in (skip, skip2):
        assert np.array_equal(r.time_raw.view(np.uint32), full.time_raw.view(np.uint32))
        assert np.array_equal(r.refs_x, full.refs_x) and np.array_equal(r.refs_y, full.refs_y)
        for k in ("rounds", "launches", "sweeps", "improvements"):
            assert r.stats[k] == full.stats[k], k
    assert skip2.stats["evaluations"] <= skip.stats["evaluations"]
    if full.stats["launches"] > 1 and full.stats["improvements"] > 0:
        assert skip2.stats["evaluations"] < skip.stats["evaluations"]


def test_readme_demo_soft_pin(oracle, pp):
    """Reference demo (crates/propag/src/main.rs:12-55): 1024 x 1024 at 5 m,
    uniform NFFL 1, moistures 0.1, wind 5 m/s toward azimuth 0, flat, one
    ignition at (500, 500), max_time 36000 s.  The reference README reports
    447822 burned cells and a maximum time of 35999.9 s (from an older build
    with 24 x 24 blocks); the restatement must agree within 1 %."""
    w = h = 1024
    t = pp.demo_terrain(w, h)
    f, _ = oracle.burn_f64(t)
    sp, az, ec = (f[:, k].astype(np.float32) for k in (4, 5, 6))
    r = oracle.propagate(w, h, 5.0, 5.0, 36000.0, sp, az, ec, [(500, 500, 0.0)], tile=264)
    burned = int(np.sum(r.time < np.finfo(np.float32).max))
    assert abs(burned - 447822) / 447822 < 0.01, burned
    assert 35990.0 < float(r.time[r.time < 3e38].max()) <= 36000.0


def test_uniform_fire_is_schedule_independent(oracle, pp):
    """With a uniform fire every cell references the ignition, so the tile
    schedule does not change the times beyond float noise."""
    w = h = 160
    t = pp.demo_terrain(w, h)
    f, _ = oracle.burn_f64(t)
    sp, az, ec = (f[:, k].astype(np.float32) for k in (4, 5, 6))
    a = oracle.propagate(w, h, 5.0, 5.0, 5000.0, sp, az, ec, [(70, 70, 0.0)], tile=0)
    b = oracle.propagate(w, h, 5.0, 5.0, 5000.0, sp, az, ec, [(70, 70, 0.0)], tile=19)
    m = a.time < 3e38
    assert np.array_equal(m, b.time < 3e38)
    assert np.max(np.abs(a.time[m] - b.time[m])) < 0.01


def _exact_f32(v):
    return Fraction(float(v))


def test_directed_rounding_emulation(oracle):
    rng = np.random.default_rng(9)
    x = np.concatenate([rng.uniform(1e-3, 1e3, 3000), rng.uniform(0.05, 2.0, 3000),
                        [1.0, 2.0, 3.0, 0.1, 1e-30, 3.4e38, 7.0]]).astype(np.float32)
    r, s = oracle.rounding_batch(x)
    for xi, ri, si in zip(x[:800], r[:800], s[:800]):
        q = 1 / _exact_f32(xi)
        assert _exact_f32(ri) <= q < _exact_f32(np.nextafter(ri, np.float32(np.inf)))
        assert _exact_f32(si) ** 2 <= _exact_f32(xi) < _exact_f32(np.nextafter(si, np.float32(np.inf))) ** 2
    # spot checks on the rest against numpy's round-to-nearest neighbour
    rn = (1.0 / x.astype(np.float64)).astype(np.float32)
    assert np.all((r == rn) | (r == np.nextafter(rn, np.float32(-np.inf))))


def test_portable_trig_accuracy(oracle):
    rng = np.random.default_rng(10)
    a = np.concatenate([rng.uniform(0, 10, 20000), np.linspace(0, 3 * np.pi, 2000)]).astype(np.float32)
    b = rng.uniform(-50, 50, a.size).astype(np.float32)
    y = rng.uniform(-50, 50, a.size).astype(np.float32)
    c, _ = oracle.trig_batch(a, b)
    _, t = oracle.trig_batch(y, b)
    ulp_c = np.abs(c.astype(np.float64) - np.cos(a.astype(np.float64))) / np.spacing(np.float32(1.0))
    assert np.max(ulp_c) < 4
    exact = np.arctan2(y.astype(np.float64), b.astype(np.float64))
    ulp_t = np.abs(t - exact) / np.spacing(np.abs(exact).astype(np.float32) + np.float32(1e-30))
    assert np.max(ulp_t) < 4


@pytest.mark.parametrize("fx,fy,tx,ty", [(0, 0, 5, 2), (3, 3, 0, 0), (2, 0, 2, 4), (0, 0, 10, 1),
                                         (7, 1, 1, 6), (0, 5, 0, 0), (4, 4, 9, 4)])
def test_dda_walk_visits_from_to_inclusive(oracle, fx, fy, tx, ty):
    cells = [(int(a), int(b)) for a, b in oracle.dda_cells(fx, fy, tx, ty)]
    assert cells[0] == (fx, fy) and cells[-1] == (tx, ty)
    for (a, b), (c, d) in zip(cells, cells[1:]):
        assert max(abs(c - a), abs(d - b)) == 1  # 8-connected steps
    xs, ys = [c[0] for c in cells], [c[1] for c in cells]
    assert min(xs) >= min(fx, tx) and max(xs) <= max(fx, tx)
    assert min(ys) >= min(fy, ty) and max(ys) <= max(fy, ty)


# Known answers of the reference's line walk (crates/geometry/src/lib.rs:
# 508-649, the host DDA's tests): (from, to) -> cells visited.  The device
# walk the propagation uses (crates/propag/src/propag.h:91-135, which the
# oracle restates) visits the same cells on every one of them.
DDA_KNOWN = [
    ((0, 0), (0, 2), [(0, 0), (0, 1), (0, 2)]),
    ((0, 0), (0, 1), [(0, 0), (0, 1)]),
    ((0, 0), (0, -2), [(0, 0), (0, -1), (0, -2)]),
    ((0, 0), (0, -1), [(0, 0), (0, -1)]),
    ((0, 0), (2, 0), [(0, 0), (1, 0), (2, 0)]),
    ((0, 0), (-2, 0), [(0, 0), (-1, 0), (-2, 0)]),
    ((0, 0), (-2, -2), [(0, 0), (-1, -1), (-2, -2)]),
    ((0, 0), (-2, 2), [(0, 0), (-1, 1), (-2, 2)]),
    ((0, 0), (2, -2), [(0, 0), (1, -1), (2, -2)]),
    ((0, 0), (1, -1), [(0, 0), (1, -1)]),
    ((0, 0), (2, 2), [(0, 0), (1, 1), (2, 2)]),
]


@pytest.mark.parametrize("frm,to,cells", DDA_KNOWN)
def test_dda_known_answers_of_the_reference(oracle, frm, to, cells):
    got = [(int(a), int(b)) for a, b in oracle.dda_cells(frm[0], frm[1], to[0], to[1])]
    assert got == cells


def _boundaries_numpy(speed, az, ecc):
    """find_boundaries (crates/propag/src/propag.cu:345-375) restated over
    whole arrays: a cell is a boundary when some in-grid neighbour's fire is
    not similar to its own (similar_fires, :296-302: float differences, taken
    in float and compared with the double thresholds 0.1 m/s, 5 degrees in
    radians and 0.05) and the neighbour spreads faster."""
    H, W = speed.shape
    out = np.zeros((H, W), bool)
    for j in (-1, 0, 1):
        for i in (-1, 0, 1):
            if i == 0 and j == 0:
                continue
            ys, xs = slice(max(0, -j), H - max(0, j)), slice(max(0, -i), W - max(0, i))
            yn, xn = slice(max(0, j), H + min(0, j)), slice(max(0, i), W + min(0, i))
            s_me, s_nb = speed[ys, xs], speed[yn, xn]
            similar = ((np.abs(s_nb - s_me).astype(np.float64) < 0.1)
                       & (np.abs(az[yn, xn] - az[ys, xs]).astype(np.float64) < 5.0 * (2 * np.pi) / 360.0)
                       & (np.abs(ecc[yn, xn] - ecc[ys, xs]).astype(np.float64) < 0.05))
            out[ys, xs] |= ~similar & (s_me < s_nb)
    return out


@pytest.mark.parametrize("seed", range(4))
def test_find_boundaries_restated(oracle, seed):
    """The oracle's boundary bits against the rule restated in numpy, on
    fields drawn from lattices whose steps put many neighbour differences
    exactly at (or one float rounding from) the thresholds, with non-burnable
    (all-zero) cells and grids of one row or column."""
    rng = np.random.default_rng(seed)
    for H, W in ((17, 23), (1, 40), (31, 1), (64, 64)):
        speed = (rng.integers(0, 8, (H, W)) * np.float32(0.05)).astype(np.float32)
        az = (rng.integers(0, 12, (H, W)) * np.float32(2.5 * np.pi / 180)).astype(np.float32)
        ecc = (rng.integers(0, 20, (H, W)) * np.float32(0.025)).astype(np.float32)
        dead = rng.random((H, W)) < 0.1
        speed[dead] = az[dead] = ecc[dead] = 0.0
        bits = oracle.find_boundaries(W, H, speed, az, ecc)
        got = np.unpackbits(bits.view(np.uint8), bitorder="little")[: H * W].reshape(H, W).astype(bool)
        want = _boundaries_numpy(speed, az, ecc)
        assert np.array_equal(got, want), (seed, H, W)
        assert want.any() and not want.all()


def test_find_boundaries_takes_differences_in_float(oracle):
    """0.1f - 2e-9f is 0.09999999949 exactly, below the double 0.1, but
    rounds to 0.1f = 0.10000000149 in float: the speeds are not similar, so
    the slower cell is a boundary, as the reference's float subtraction
    decides (propag.cu:296-302)."""
    speed = np.array([[np.float32(2e-9), np.float32(0.1)]], np.float32)
    zeros = np.zeros_like(speed)
    bits = oracle.find_boundaries(2, 1, speed, zeros, zeros)
    assert int(bits[0]) & 3 == 1
    assert _boundaries_numpy(speed, zeros, zeros).tolist() == [[True, False]]


def test_dda_special_case_propag(oracle):
    """The reference's special_case_propag: the second cell of the walk from
    (499, 99) to (500, 100) is (500, 100)."""
    assert [tuple(int(v) for v in c) for c in oracle.dda_cells(499, 99, 500, 100)][1] == (500, 100)


def test_dda_second_cell_is_the_neighbour_in_direction(oracle):
    """The reference's neighbor_in_direction_same_as_line_to property
    (crates/geometry/src/lib.rs:477-495, 511-521) on offsets within 300
    cells: the walk's second cell is the neighbour in the direction of the
    target (diagonal on |dx| = |dy|, else along the longer axis)."""
    rng = np.random.default_rng(12)
    for x, y in rng.integers(-300, 301, size=(4000, 2)):
        x, y = int(x), int(y)
        if x == 0 or y == 0:
            continue
        sx, sy = (x > 0) - (x < 0), (y > 0) - (y < 0)
        want = (sx, sy) if abs(x) == abs(y) else ((sx, 0) if abs(x) > abs(y) else (0, sy))
        got = tuple(int(v) for v in oracle.dda_cells(0, 0, x, y)[1])
        assert got == want, (x, y, got, want)


def test_arithmetic_moves_the_fixpoint(oracle):
    """The reference kernel's float operations matter to the last bit: the
    same scenario in the portable arithmetic (trig 0) and with libm's
    cosine/arctangent and the reference's fused multiply-adds (trig 2)
    adopts other references in some cells and moves their times by more
    than max(0.5 s, 1e-4 t) -- which is why the engine's default arithmetic
    is the reference's own (oracle/measure_arith.py measures it at full
    size)."""
    from py_propag import scenarios as S
    sc = S.config0(size=256, seed=3)
    f, _ = oracle.burn_f64(sc.terrain)
    sp, az, ec = (f[:, k].astype(np.float32) for k in (4, 5, 6))
    runs = [oracle.propagate(sc.width, sc.height, sc.dx, sc.dy, sc.max_time, sp, az, ec, sc.ignitions,
                             tile=57, full=2, trig=t) for t in (0, 2)]
    a, b = (r.time.astype(np.float64) for r in runs)
    fmax = np.finfo(np.float32).max
    both = (runs[0].time < fmax) & (runs[1].time < fmax)
    assert both.sum() > 1000
    assert (runs[0].time.view(np.uint32) != runs[1].time.view(np.uint32)).any()
    assert ((runs[0].refs_x != runs[1].refs_x) | (runs[0].refs_y != runs[1].refs_y)).any()
    dev = np.abs(a - b)[both]
    assert np.median(dev) < 0.5  # most cells agree closely ...
    assert (dev > np.maximum(0.5, 1e-4 * a[both])).any()  # ... some do not
