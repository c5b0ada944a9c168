"""Seeded synthetic wildfire scenarios (terrain, fuel, weather, ignitions).

The reference ships no dataset; its demo (crates/propag/src/main.rs:12-55)
is a constant terrain.  These generators build the five workloads the
benchmarks and parity tests use, from a seed, with the shapes and value
ranges of the reference's inputs (``TerrainCuda`` SoA, crates/firelib/src/
firelib.rs:98-109):

* fuel_code      u8   NFFL model 1..13, 0 = non-burnable
* d1hr .. wood   f32  moisture ratios
* wind_speed     f32  m/s
* wind_azimuth   f32  rad, the bearing the wind blows TOWARD (compass)
* slope          f32  rise / run
* aspect         f32  rad, downslope compass azimuth

Rasters are (H, W) row-major, south-up (row index grows with y, geo
transform ``[0, dx, 0, 0, 0, dy]``, dy > 0) like the reference demo.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

TERRAIN_KEYS = ("fuel_code", "d1hr", "d10hr", "d100hr", "herb", "wood",
                "wind_speed", "wind_azimuth", "slope", "aspect")


@dataclass
class Scenario:
    width: int
    height: int
    dx: float
    dy: float
    max_time: float
    terrain: dict
    ignitions: list = field(default_factory=list)  # [(x, y, t)]
    name: str = ""

    @property
    def cells(self) -> int:
        return self.width * self.height


# ---------------------------------------------------------------- terrain ----

def dem_hills(width: int, height: int, cell: float, rng, n_hills: int = 30,
              zmax: float = 800.0) -> np.ndarray:
    """Sum of Gaussian hills (separable), rescaled to [0, zmax] metres."""
    xs = (np.arange(width) + 0.5) * cell
    ys = (np.arange(height) + 0.5) * cell
    z = np.zeros((height, width), dtype=np.float64)
    for _ in range(n_hills):
        cx = rng.uniform(0, width * cell)
        cy = rng.uniform(0, height * cell)
        sig = rng.uniform(150.0, 1500.0)
        h = rng.uniform(0.2, 1.0)
        gx = np.exp(-0.5 * ((xs - cx) / sig) ** 2)
        gy = np.exp(-0.5 * ((ys - cy) / sig) ** 2)
        z += h * np.outer(gy, gx)
    z -= z.min()
    if z.max() > 0:
        z *= zmax / z.max()
    return z


def _value_noise(width: int, height: int, period: float, rng) -> np.ndarray:
    """Smooth value noise: random lattice every `period` cells, bicubic-ish
    (smoothstep) interpolation."""
    gw = int(math.ceil(width / period)) + 2
    gh = int(math.ceil(height / period)) + 2
    lat = rng.uniform(-1.0, 1.0, (gh, gw))
    fx = (np.arange(width) + 0.5) / period
    fy = (np.arange(height) + 0.5) / period
    ix = np.floor(fx).astype(np.int64)
    iy = np.floor(fy).astype(np.int64)
    tx = fx - ix
    ty = fy - iy
    sx = tx * tx * (3 - 2 * tx)
    sy = ty * ty * (3 - 2 * ty)
    a = lat[np.ix_(iy, ix)]
    b = lat[np.ix_(iy, ix + 1)]
    c = lat[np.ix_(iy + 1, ix)]
    d = lat[np.ix_(iy + 1, ix + 1)]
    top = a + (b - a) * sx[None, :]
    bot = c + (d - c) * sx[None, :]
    return top + (bot - top) * sy[:, None]


def dem_ridged(width: int, height: int, cell: float, rng, octaves: int = 6,
               max_slope: float = 1.0) -> np.ndarray:
    """Ridged fractal noise, scaled so that the steepest slope is max_slope."""
    z = np.zeros((height, width), dtype=np.float64)
    period = max(width, height) / 4.0
    amp = 1.0
    for _ in range(octaves):
        n = 1.0 - np.abs(_value_noise(width, height, period, rng))
        z += amp * n * n
        period /= 2.0
        amp *= 0.5
        if period < 2:
            break
    s, _ = slope_aspect(z, cell, cell)
    smax = float(s.max())
    if smax > 0:
        z *= max_slope / smax
    return z


def slope_aspect(dem: np.ndarray, dx: float, dy: float):
    """Central differences.  slope = |grad z| (rise/run); aspect = compass
    azimuth of -grad z in [0, 2 pi) (rows grow northward: south-up)."""
    dzdx = np.gradient(dem, dx, axis=1)
    dzdy = np.gradient(dem, dy, axis=0)
    slope = np.hypot(dzdx, dzdy)
    aspect = np.arctan2(-dzdx, -dzdy)
    aspect = np.where(aspect < 0, aspect + 2 * np.pi, aspect)
    aspect = np.where(slope == 0, 0.0, aspect)
    return slope.astype(np.float32), aspect.astype(np.float32)


def fuel_voronoi(width: int, height: int, rng, n_seeds: int = 256,
                 nonburn_frac: float = 0.05) -> np.ndarray:
    """Voronoi patches of NFFL 1..13; whole patches become code 0 until about
    nonburn_frac of the cells are non-burnable."""
    from scipy.spatial import cKDTree

    pts = np.column_stack([rng.uniform(0, width, n_seeds), rng.uniform(0, height, n_seeds)])
    codes = rng.integers(1, 14, n_seeds).astype(np.uint8)
    yy, xx = np.mgrid[0:height, 0:width]
    q = np.column_stack([xx.ravel() + 0.5, yy.ravel() + 0.5])
    _, idx = cKDTree(pts).query(q, workers=-1)
    idx = idx.reshape(height, width)
    sizes = np.bincount(idx.ravel(), minlength=n_seeds)
    target = nonburn_frac * width * height
    burned_off = 0
    for p in rng.permutation(n_seeds):
        if burned_off >= target:
            break
        if burned_off + sizes[p] > 1.6 * target and burned_off > 0:
            continue
        codes[p] = 0
        burned_off += sizes[p]
    return codes[idx]


def _stamp_disc(mask: np.ndarray, cx: float, cy: float, r: float) -> None:
    h, w = mask.shape
    x0, x1 = max(int(cx - r), 0), min(int(cx + r) + 2, w)
    y0, y1 = max(int(cy - r), 0), min(int(cy + r) + 2, h)
    if x0 >= x1 or y0 >= y1:
        return
    yy, xx = np.mgrid[y0:y1, x0:x1]
    mask[y0:y1, x0:x1] |= (xx + 0.5 - cx) ** 2 + (yy + 0.5 - cy) ** 2 <= r * r


def lakes_and_roads(width: int, height: int, rng, frac: float = 0.12) -> np.ndarray:
    """Non-burnable mask: seeded lake discs plus 2-3 cell wide road polylines."""
    mask = np.zeros((height, width), dtype=bool)
    # roads first: a handful of long polylines
    n_roads = max(2, int(round(6 * max(width, height) / 4096)))
    for _ in range(n_roads):
        x, y = rng.uniform(0, width), rng.uniform(0, height)
        heading = rng.uniform(0, 2 * np.pi)
        half = rng.uniform(1.0, 1.5)
        for _seg in range(int(rng.integers(4, 9))):
            heading += rng.normal(0, 0.5)
            length = rng.uniform(0.1, 0.3) * max(width, height)
            steps = int(length / 0.7) + 1
            for s in range(steps):
                _stamp_disc(mask, x, y, half)
                x += 0.7 * math.sin(heading)
                y += 0.7 * math.cos(heading)
                if not (0 <= x < width and 0 <= y < height):
                    break
    target = frac * width * height
    while mask.sum() < target:
        r = rng.uniform(0.01, 0.05) * max(width, height)
        _stamp_disc(mask, rng.uniform(0, width), rng.uniform(0, height), r)
    return mask


def _burnable_cells(fuel: np.ndarray, rng, k: int, margin: int = 0):
    h, w = fuel.shape
    out = []
    while len(out) < k:
        x = int(rng.integers(margin, w - margin))
        y = int(rng.integers(margin, h - margin))
        if fuel[y, x] != 0:
            out.append((x, y))
    return out


def _full(shape, v):
    return np.full(shape, v, dtype=np.float32)


# -------------------------------------------------------------- workloads ----

def config0(size: int = 1024, seed: int = 0, cell: float = 5.0) -> Scenario:
    """Plain single scenario (the reference demo shape): Gaussian hills, NFFL
    Voronoi patches with 5 % non-burnable, uniform wind 5 m/s from 225 deg,
    moisture 6/7/8/60/90 %, one ignition at (500, 500) scaled to the size,
    max_time 36000 s."""
    rng = np.random.default_rng(seed)
    w = h = size
    dem = dem_hills(w, h, cell, rng)
    slope, aspect = slope_aspect(dem, cell, cell)
    fuel = fuel_voronoi(w, h, rng, n_seeds=max(16, int(256 * (size / 1024) ** 2)))
    shp = (h, w)
    ix = iy = int(round(500 * size / 1024))
    if fuel[iy, ix] == 0:
        fuel[max(iy - 1, 0):iy + 2, max(ix - 1, 0):ix + 2] = 1
    terrain = dict(fuel_code=fuel, d1hr=_full(shp, 0.06), d10hr=_full(shp, 0.07),
                   d100hr=_full(shp, 0.08), herb=_full(shp, 0.60), wood=_full(shp, 0.90),
                   wind_speed=_full(shp, 5.0), wind_azimuth=_full(shp, np.deg2rad(45.0)),
                   slope=slope, aspect=aspect)
    return Scenario(w, h, cell, cell, 36000.0, terrain, [(ix, iy, 0.0)], f"config0-{size}")


def config1(size: int = 4096, seed: int = 1, cell: float = 5.0, n_ign: int = 20,
            max_time: float = 43200.0) -> Scenario:
    """Large heterogeneous scenario: ridged fBm terrain (max slope 45 deg),
    12 % non-burnable lakes and roads, smooth random wind 0-15 m/s from
    225 +- 60 deg, per-cell moisture +- 2 points, 20 ignitions."""
    rng = np.random.default_rng(seed)
    w = h = size
    dem = dem_ridged(w, h, cell, rng, max_slope=1.0)
    slope, aspect = slope_aspect(dem, cell, cell)
    fuel = fuel_voronoi(w, h, rng, n_seeds=max(16, int(256 * (size / 1024) ** 2)), nonburn_frac=0.0)
    fuel[lakes_and_roads(w, h, rng, 0.12)] = 0
    shp = (h, w)
    wn = _value_noise(w, h, max(w, h) / 3.0, rng)
    ws = (7.5 + 7.5 * wn).clip(0.0, 15.0).astype(np.float32)
    dn = _value_noise(w, h, max(w, h) / 3.0, rng)
    wind_from = np.deg2rad(225.0 + 60.0 * dn)
    waz = np.mod(wind_from + np.pi, 2 * np.pi).astype(np.float32)

    def jitter(base):
        return (base + rng.uniform(-0.02, 0.02, shp)).astype(np.float32)

    terrain = dict(fuel_code=fuel, d1hr=jitter(0.06), d10hr=jitter(0.07), d100hr=jitter(0.08),
                   herb=jitter(0.60), wood=jitter(0.90), wind_speed=ws, wind_azimuth=waz,
                   slope=slope, aspect=aspect)
    ign = [(x, y, 0.0) for (x, y) in _burnable_cells(fuel, rng, n_ign)]
    return Scenario(w, h, cell, cell, max_time, terrain, ign, f"config1-{size}")


def ensemble_members(base: Scenario, n: int = 256, seed: int = 2, max_time: float = 21600.0):
    """Ensemble over a shared terrain/fuel: per member wind speed
    lognormal(median 6 m/s, sigma 0.3), direction 225 +- 30 deg, dead moisture
    offset +- 0.02 and one ignition over burnable cells.  Returns a list of
    dicts with the per-member scalars."""
    rng = np.random.default_rng(seed)
    fuel = base.terrain["fuel_code"]
    out = []
    for _ in range(n):
        speed = float(np.exp(np.log(6.0) + 0.3 * rng.standard_normal()))
        wind_from = 225.0 + rng.uniform(-30.0, 30.0)
        off = float(rng.uniform(-0.02, 0.02))
        (x, y), = _burnable_cells(fuel, rng, 1)
        out.append(dict(wind_speed=speed, wind_azimuth=float(np.deg2rad((wind_from + 180.0) % 360.0)),
                        dead_offset=off, ignition=(x, y, 0.0), max_time=max_time))
    return out


def member_scenario(base: Scenario, m: dict) -> Scenario:
    """Materialises one ensemble member as a full scenario."""
    t = dict(base.terrain)
    shp = t["slope"].shape
    t["wind_speed"] = _full(shp, m["wind_speed"])
    t["wind_azimuth"] = _full(shp, m["wind_azimuth"])
    for k in ("d1hr", "d10hr", "d100hr"):
        t[k] = (base.terrain[k] + np.float32(m["dead_offset"])).astype(np.float32)
    return Scenario(base.width, base.height, base.dx, base.dy, m["max_time"], t,
                    [m["ignition"]], base.name + "-member")


def config2(n: int = 256, size: int = 1024, seed: int = 2):
    base = config0(size=size, seed=0)
    return base, ensemble_members(base, n=n, seed=seed)


def config3(n: int = 64, seed: int = 3, min_size: int = 128, max_size: int = 2048):
    """Uneven batch: square grids log-uniform in [min_size, max_size], cell
    size U(5, 30) m, config-0 style terrain/fuel per scenario seed, 1-10
    ignitions, max_time U(3600, 43200) s."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        size = int(round(math.exp(rng.uniform(math.log(min_size), math.log(max_size)))))
        cell = float(rng.uniform(5.0, 30.0))
        s_seed = int(rng.integers(0, 2**31 - 1))
        r2 = np.random.default_rng(s_seed)
        dem = dem_hills(size, size, cell, r2)
        slope, aspect = slope_aspect(dem, cell, cell)
        fuel = fuel_voronoi(size, size, r2, n_seeds=max(16, int(256 * (size / 1024) ** 2)))
        shp = (size, size)
        wind_from = 225.0 + r2.uniform(-30, 30)
        terrain = dict(fuel_code=fuel, d1hr=_full(shp, 0.06), d10hr=_full(shp, 0.07),
                       d100hr=_full(shp, 0.08), herb=_full(shp, 0.60), wood=_full(shp, 0.90),
                       wind_speed=_full(shp, float(np.exp(np.log(6.0) + 0.3 * r2.standard_normal()))),
                       wind_azimuth=_full(shp, np.deg2rad((wind_from + 180.0) % 360.0)),
                       slope=slope, aspect=aspect)
        k = int(r2.integers(1, 11))
        ign = [(x, y, 0.0) for (x, y) in _burnable_cells(fuel, r2, k)]
        out.append(Scenario(size, size, cell, cell, float(rng.uniform(3600.0, 43200.0)), terrain,
                            ign, f"config3-{i}-{size}"))
    return out


def config4_requests(master_fuel: np.ndarray, seconds: float = 300.0, rate: float = 20.0,
                     seed: int = 4, min_size: int = 256, max_size: int = 4096):
    """Serving workload: Poisson arrivals at `rate` per second for `seconds`;
    each request is a square window, side log-uniform in [min_size, max_size],
    cut from a master terrain/fuel atlas at a random offset, with its own wind
    speed (lognormal, median 6 m/s, sigma 0.3), direction (225 +- 30 deg),
    dead-moisture offset (+-0.02), one ignition over burnable cells of the
    window and max_time U(1, 12) h.  Returns a list of dicts sorted by
    arrival time (s)."""
    rng = np.random.default_rng(seed)
    H, W = master_fuel.shape
    out, t = [], 0.0
    while True:
        t += float(rng.exponential(1.0 / rate))
        if t > seconds:
            break
        n = int(round(math.exp(rng.uniform(math.log(min_size), math.log(max_size)))))
        n = min(n, W, H)
        x0 = int(rng.integers(0, W - n + 1))
        y0 = int(rng.integers(0, H - n + 1))
        win = master_fuel[y0:y0 + n, x0:x0 + n]
        if not np.any(win):
            continue
        (ix, iy), = _burnable_cells(win, rng, 1)
        out.append(dict(arrival=t, size=n, x0=x0, y0=y0,
                        wind_speed=float(np.exp(np.log(6.0) + 0.3 * rng.standard_normal())),
                        wind_azimuth=float(np.deg2rad((225.0 + rng.uniform(-30.0, 30.0) + 180.0) % 360.0)),
                        dead_offset=float(rng.uniform(-0.02, 0.02)), ignition=(ix, iy, 0.0),
                        max_time=float(rng.uniform(3600.0, 43200.0))))
    return out
