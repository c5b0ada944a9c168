"""TEST INFRASTRUCTURE ONLY -- ctypes front-end of the CPU oracles.

Loaded by the tests, by ``__graft_entry__.smoke()`` and by ``bench.py``'s
CPU-baseline leg, as the checker.  Nothing in the product imports this module.

* ``burn_f64``      -- FP64 restatement of the reference's Rust firelib
                       (oracle/firelib_oracle.c)
* ``burn_firelib_c``-- the reference's own C fireLib compiled from source
                       (oracle/_ref/libfirelib_ref.so), driven like the
                       reference's quickcheck harness
* ``find_boundaries``, ``propagate``, ``post`` -- CPU restatement of the
                       propagation kernel with the reference's tile schedule
                       (oracle/propag_oracle.c)
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
FIELDS = ("rx_int", "speed0", "hpua", "phi_eff_wind", "speed_max", "azimuth_max",
          "eccentricity", "residence_time", "byrams_max", "flame_max")
STAT_NAMES = ("rounds", "launches", "sweeps", "evaluations", "improvements", "gathers",
              "dda_steps", "refbox_scans", "refbox_cells", "tiles_x", "tiles_y")

_lib = None
_ref = None


def reference_root() -> str:
    """The reference checkout: $PROPAG_REFERENCE, else a `reference` folder
    beside this repository."""
    return os.environ.get("PROPAG_REFERENCE") or os.path.join(os.path.dirname(HERE), "..", "reference")


def build(reference: str | None = None) -> None:
    """Compiles liboracle.so and, when the reference checkout exists, _ref/."""
    args = ["make", "-s", "-C", HERE, "all"]
    subprocess.run(args, check=True)
    ref_root = os.path.abspath(reference or reference_root())
    if os.path.isdir(os.path.join(ref_root, "crates", "firelib-sys")):
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REFERENCE={ref_root}"], check=True)


def _load():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        _lib = C.CDLL(path)
        f32p = C.POINTER(C.c_float)
        _lib.ofl_burn_f64.restype = C.c_int64
        _lib.ops_propagate.restype = C.c_int
        _lib.ops_find_boundaries.restype = C.c_int64
        _lib.ops_post.restype = C.c_int64
        _lib.ops_post.argtypes = [C.c_int64, f32p, C.c_float, f32p]
    return _lib


def have_firelib_c() -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", "libfirelib_ref.so"))


def _load_ref():
    global _ref
    if _ref is None:
        _ref = C.CDLL(os.path.join(HERE, "_ref", "libfirelib_ref.so"))
        _ref.ref_burn_c.restype = C.c_int64
        if hasattr(_ref, "ref_burn_c_rust_catalog"):  # absent from builds of older harnesses
            _ref.ref_burn_c_rust_catalog.restype = C.c_int64
    return _ref


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


TERRAIN_KEYS = ("fuel_code", "d1hr", "d10hr", "d100hr", "herb", "wood",
                "wind_speed", "wind_azimuth", "slope", "aspect")


def _terrain_args(t):
    fuel = np.ascontiguousarray(t["fuel_code"], dtype=np.uint8).ravel()
    rest = [np.ascontiguousarray(t[k], dtype=np.float32).ravel() for k in TERRAIN_KEYS[1:]]
    n = fuel.size
    for r in rest:
        assert r.size == n
    return n, fuel, rest


def burn_f64(terrain: dict) -> tuple[np.ndarray, np.ndarray]:
    """Returns (fields[n, 10] float64, situation[n] int32)."""
    lib = _load()
    n, fuel, rest = _terrain_args(terrain)
    out = np.zeros((n, 10), dtype=np.float64)
    sit = np.zeros(n, dtype=np.int32)
    lib.ofl_burn_f64(C.c_int64(n), _ptr(fuel), *[_ptr(r) for r in rest], _ptr(out), _ptr(sit))
    return out, sit


def burn_firelib_c(terrain: dict, rust_nffl13: bool = False) -> np.ndarray:
    """The reference's fireLib.c on each cell (10 SI fields).  rust_nffl13:
    with NFFL13's 10-h dead load set to the Rust catalog's 0.0580 instead of
    fireLib.c's 1.0580 (the one entry where the two catalogs differ)."""
    lib = _load_ref()
    n, fuel, rest = _terrain_args(terrain)
    out = np.zeros((n, 10), dtype=np.float64)
    fn = lib.ref_burn_c_rust_catalog if rust_nffl13 else lib.ref_burn_c
    fn(C.c_int64(n), _ptr(fuel), *[_ptr(r) for r in rest], _ptr(out))
    return out


def catalog_f64() -> np.ndarray:
    lib = _load()
    out = np.zeros((20, 17), dtype=np.float64)
    lib.ofl_catalog_f64(_ptr(out), C.c_int(17))
    return out


class _Settings(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("dx", C.c_float),
                ("dy", C.c_float), ("max_time", C.c_float)]


def find_boundaries(width: int, height: int, speed, az, ecc) -> np.ndarray:
    lib = _load()
    n = width * height
    bits = np.zeros((n + 31) // 32, dtype=np.uint32)
    s, a, e = (np.ascontiguousarray(x, dtype=np.float32).ravel() for x in (speed, az, ecc))
    lib.ops_find_boundaries(C.c_uint32(width), C.c_uint32(height), _ptr(s), _ptr(a), _ptr(e),
                            _ptr(bits))
    return bits


@dataclass
class OracleResult:
    time: np.ndarray        # (H, W) float32 after the post mask
    time_raw: np.ndarray    # (H, W) float32 before the post mask
    refs_x: np.ndarray
    refs_y: np.ndarray
    boundaries: np.ndarray  # uint32 bit words
    stats: dict


def initial_state(width: int, height: int, ignitions):
    """ignitions: iterable of (x, y, t).  Mirrors propag.rs:433-449: ignited
    cells reference themselves, the rest hold 0xFFFF and f32::MAX."""
    time = np.full(width * height, np.finfo(np.float32).max, dtype=np.float32)
    rx = np.full(width * height, 0xFFFF, dtype=np.uint16)
    ry = np.full(width * height, 0xFFFF, dtype=np.uint16)
    for (x, y, t) in ignitions:
        i = int(x) + int(y) * width
        time[i] = np.float32(t)
    ign = np.nonzero(time < np.finfo(np.float32).max)[0]
    rx[ign] = (ign % width).astype(np.uint16)
    ry[ign] = (ign // width).astype(np.uint16)
    return time, rx, ry


def propagate(width: int, height: int, dx: float, dy: float, max_time: float,
              speed, az, ecc, ignitions=None, *, time0=None, refs0=None, tile: int = 0,
              full: int = 0, trig: int = 0, threads: int = 0) -> OracleResult:
    """Runs the CPU restatement.  tile = cells per side of one cooperative
    launch (block * grid_w); 0 = one tile (global Jacobi).  full: 0 = the
    engine's work skipping (whole tile in a launch's first sweep), 1 = every
    cell in every sweep, 2 = skipping in first sweeps too (grid-wide pending
    bitmap); all three give the same results.  trig: the arithmetic of
    time_from -- 0 portable (the engine's PROPAG_ARITH_PORTABLE), 1 libm
    cosine/arctangent, 2 libm plus the reference's fused multiply-adds, 3 as 2
    with the GPU's __cosf/atan2f tables (the engine's PROPAG_ARITH_REFERENCE;
    see set_device_tables)."""
    lib = _load()
    s_arr, a_arr, e_arr = (np.ascontiguousarray(x, dtype=np.float32).ravel() for x in (speed, az, ecc))
    if time0 is None:
        time, rx, ry = initial_state(width, height, ignitions or [])
    else:
        time = np.array(time0, dtype=np.float32).ravel().copy()
        rx = np.array(refs0[0], dtype=np.uint16).ravel().copy()
        ry = np.array(refs0[1], dtype=np.uint16).ravel().copy()
    bits = find_boundaries(width, height, s_arr, a_arr, e_arr)
    st = _Settings(width, height, dx, dy, max_time)
    stats = np.zeros(len(STAT_NAMES), dtype=np.int64)
    rc = lib.ops_propagate(C.byref(st), _ptr(s_arr), _ptr(a_arr), _ptr(e_arr), _ptr(time), _ptr(rx),
                           _ptr(ry), _ptr(bits), C.c_int(tile), C.c_int(int(full)), C.c_int(trig),
                           C.c_int(threads), _ptr(stats))
    if rc != 0:
        raise RuntimeError(f"ops_propagate failed: {rc}")
    raw = time.copy()
    lib.ops_post(C.c_int64(time.size), s_arr.ctypes.data_as(C.POINTER(C.c_float)),
                 C.c_float(max_time), time.ctypes.data_as(C.POINTER(C.c_float)))
    return OracleResult(time.reshape(height, width), raw.reshape(height, width),
                        rx.reshape(height, width), ry.reshape(height, width), bits,
                        dict(zip(STAT_NAMES, (int(v) for v in stats))))


_tables = None  # keeps the arrays given to ops_set_tables alive


def set_device_tables(cos_tab, cos_lo: int, cos_below: float, atan_tab, max_a: int,
                      max_b: int) -> None:
    """Installs the GPU's __cosf values -- cos_tab[i] for the float with bits
    cos_lo + i, and the constant cos_below for every float with smaller bits
    -- and its atan2f values over integer pairs (|a| <= max_a, |b| <= max_b)
    for trig = 3; cos_tab None uninstalls them."""
    global _tables
    lib = _load()
    lib.ops_set_tables.argtypes = [C.c_void_p, C.c_uint32, C.c_uint64, C.c_float, C.c_void_p,
                                   C.c_int, C.c_int]
    if cos_tab is None:
        _tables = None
        lib.ops_set_tables(None, 0, 0, 1.0, None, -1, -1)
        return
    c = np.ascontiguousarray(cos_tab, dtype=np.float32)
    a = np.ascontiguousarray(atan_tab, dtype=np.float32)
    assert a.size == (2 * max_a + 1) * (2 * max_b + 1)
    _tables = (c, a)
    lib.ops_set_tables(_ptr(c), C.c_uint32(cos_lo), C.c_uint64(c.size), C.c_float(cos_below), _ptr(a),
                       int(max_a), int(max_b))


# Range of the trig = 3 tables.  The cosine's argument is |bearing -
# azimuth_max|, in [0, 3 pi] (bearings in [-pi, pi], azimuths in [0, 2 pi));
# the bearings are atan2f of cell offsets.
COS_TABLE_LO = 0x35800000  # 2^-20: below it __cosf must be one constant (checked)
COS_TABLE_HI = 0x41180000  # 9.5 > 3 pi


def install_device_tables(lib, max_offset: int = 4095) -> None:
    """Builds the trig = 3 tables from the device (libpropag's
    propag_selftest_cosf_table / propag_selftest_atan2f_table, given as the
    ctypes library `lib`) and installs them: __cosf of every float with bits
    in [lo, COS_TABLE_HI), lo = COS_TABLE_LO unless the device's values below
    it are not all one constant, and atan2f of every integer pair within
    max_offset (grids up to max_offset + 1 cells per side)."""
    chunk = 1 << 26
    below = None
    lo = COS_TABLE_LO
    buf = np.empty(chunk, np.float32)
    for o in range(0, COS_TABLE_LO, chunk):
        m = min(chunk, COS_TABLE_LO - o)
        if lib.propag_selftest_cosf_table(o, m, buf.ctypes.data) != 0:
            raise RuntimeError("propag_selftest_cosf_table failed")
        t = buf[:m]
        if below is None:
            below = t[0]
        bad = np.nonzero(t != below)[0]
        if bad.size:  # not constant there: the table starts at the first other value
            lo = o + int(bad[0])
            break
    tab = np.empty(COS_TABLE_HI - lo, np.float32)
    if lib.propag_selftest_cosf_table(lo, tab.size, tab.ctypes.data) != 0:
        raise RuntimeError("propag_selftest_cosf_table failed")
    w = 2 * max_offset + 1
    atan = np.empty(w * w, np.float32)
    if lib.propag_selftest_atan2f_table(max_offset, max_offset, atan.ctypes.data) != 0:
        raise RuntimeError("propag_selftest_atan2f_table failed")
    set_device_tables(tab, lo, float(below), atan, max_offset, max_offset)


def table_misses() -> int:
    """Look-ups outside the trig = 3 tables since they were installed."""
    lib = _load()
    lib.ops_table_misses.restype = C.c_int64
    return int(lib.ops_table_misses())


def time_from_batch(dx, dy, fx, fy, ftime, tx, ty, smax, azmax, ecc, trig=0):
    lib = _load()
    st = _Settings(0, 0, dx, dy, 0.0)
    arrs = [np.ascontiguousarray(a, dtype=t) for a, t in
            ((fx, np.int32), (fy, np.int32), (ftime, np.float32), (tx, np.int32), (ty, np.int32),
             (smax, np.float32), (azmax, np.float32), (ecc, np.float32))]
    n = arrs[0].size
    out = np.zeros(n, dtype=np.float32)
    lib.ops_time_from_batch(C.byref(st), C.c_int64(n), *[_ptr(a) for a in arrs], C.c_int(trig), _ptr(out))
    return out


def trig_batch(a, b):
    lib = _load()
    a = np.ascontiguousarray(a, dtype=np.float32)
    b = np.ascontiguousarray(b, dtype=np.float32)
    c = np.zeros_like(a)
    t = np.zeros_like(a)
    lib.ops_trig_batch(C.c_int64(a.size), _ptr(a), _ptr(b), _ptr(c), _ptr(t))
    return c, t


def rounding_batch(x):
    """(round-down reciprocal, round-toward-zero square root) of float32 x."""
    lib = _load()
    x = np.ascontiguousarray(x, dtype=np.float32)
    r = np.zeros_like(x)
    s = np.zeros_like(x)
    lib.ops_rounding_batch(C.c_int64(x.size), _ptr(x), _ptr(r), _ptr(s))
    return r, s


# ---- dmoist (crates/dmoist/src/lib.rs) --------------------------------------

_F, _I = C.c_float, C.c_int
_DMOIST = {  # name -> (C function, argument types); float result
    "hcb": ("odm_humidity_content_base", (_F, _F, _I), C.c_int),
    "hcb_shading": ("odm_correct_hcb_for_shading", (_F, _F, _I, _F, _F, _I, _I), _F),
    "prob_precip": ("odm_correct_probability_for_precipitation", (_F, _F), _F),
    "d1hr": ("odm_d1hr", (_F, _F, _F), _F),
    "x10hr": ("odm_moisture_by_10hr", (_I, _F, _F, _F), _F),
    "live": ("odm_live_moisture", (_I,), _F),
    "prob_ign": ("odm_ignition_probability", (_F, _F, _F, _I), _F),
    "shading": ("odm_shading", (_F, _I), _F),
    "wind_speed": ("odm_wind_speed", (C.c_double, C.c_double), C.c_double),
    "wind_dir": ("odm_wind_direction", (C.c_double, C.c_double), C.c_double),
}


def dmoist_fn(name: str, params) -> np.ndarray:
    """Evaluates one dmoist function row by row (params: rows x arguments)."""
    lib = _load()
    fname, argt, rest = _DMOIST[name]
    fn = getattr(lib, fname)
    fn.restype = rest
    fn.argtypes = list(argt)
    out = []
    for row in np.asarray(params, dtype=np.float64):
        args = [int(v) if t is _I else float(v) for v, t in zip(row, argt)]
        out.append(float(fn(*args)))
    return np.array(out)


def dmoist_max_precip(month: int, pp) -> float:
    lib = _load()
    lib.odm_maximum_precipitation_effect.restype = C.c_float
    a = np.ascontiguousarray(pp, dtype=np.float32)
    return float(lib.odm_maximum_precipitation_effect(C.c_int(month), _ptr(a)))


def dmoist_hourly(t, rh, cc, slope, aspect, pp, month, fuel):
    """calculate_hourly_fuel_moisture for one site: (d1, d10, d100), 24 each."""
    lib = _load()
    arrs = [np.ascontiguousarray(a, dtype=np.float32) for a in (t, rh, cc, pp)]
    out = [np.zeros(24, np.float32) for _ in range(3)]
    lib.odm_hourly(_ptr(arrs[0]), _ptr(arrs[1]), _ptr(arrs[2]), C.c_float(slope), C.c_float(aspect),
                   _ptr(arrs[3]), C.c_int(month), C.c_int(fuel), *[_ptr(o) for o in out])
    return tuple(out)


def dmoist_cells(hour, month, t, rh, cc, slope, aspect, fuel, pp):
    """Per-cell moisture at one hour: weather (24, n), precipitation (6, n)."""
    lib = _load()
    n = np.asarray(slope).size
    t, rh, cc, pp = (np.ascontiguousarray(a, dtype=np.float32) for a in (t, rh, cc, pp))
    slope, aspect = (np.ascontiguousarray(a, dtype=np.float32).ravel() for a in (slope, aspect))
    fuel = np.ascontiguousarray(fuel, dtype=np.uint8).ravel()
    out = [np.zeros(n, np.float32) for _ in range(3)]
    lib.odm_cells(C.c_int64(n), C.c_int(hour), C.c_int(month), _ptr(t), _ptr(rh), _ptr(cc), _ptr(slope),
                  _ptr(aspect), _ptr(fuel), _ptr(pp), *[_ptr(o) for o in out])
    return tuple(out)


def dda_cells(fx, fy, tx, ty):
    """Cells visited by the line-of-sight walk (propag.h:91-135)."""
    lib = _load()
    lib.ops_dda_cells.restype = C.c_int64
    cap = abs(tx - fx) + abs(ty - fy) + 4
    out = np.zeros(2 * cap, dtype=np.int32)
    n = lib.ops_dda_cells(C.c_int(fx), C.c_int(fy), C.c_int(tx), C.c_int(ty), _ptr(out), C.c_int64(cap))
    return [tuple(p) for p in out[: 2 * min(n, cap)].reshape(-1, 2)]
