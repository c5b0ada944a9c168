"""py_propag -- Python drop-in for the reference's ``py_propag`` module, backed
by libpropag.so (hand-written CUDA for sm_100a).

Same names, arguments, validation rules and exception types as the
reference's pyo3 module (crates/py-propag/src/lib.rs:12-15,174-839,
crates/py-propag/py_propag/__init__.py), with two differences:

* ``propagate`` runs the real propagation (the reference's returns a mock of
  all-``inf`` times, lib.rs:676-691) and writes the arrival-time GeoTIFF to
  ``output_path``.  Unburned cells hold ``f32::MAX``, as the C path writes.
* ``propagate`` takes an optional keyword ``terrain=`` (dict of the ten
  ``TerrainCuda`` rasters, shape (H, W)); without it the reference's constant
  demo terrain is used (fuel 1, moistures 0.1, wind 5 m/s toward azimuth 0,
  flat: crates/propag/src/main.rs:44-55).  ``tile=`` selects the super-grid
  tile side (default 323, -1 = whole grid).

Extras for B200 work: ``fire_behaviour`` (the per-cell fire pass),
``propagate_arrays`` (propagation without files), ``Engine`` (batched
propagation over device-resident scenarios).
"""
from __future__ import annotations

import ctypes as C
import os
import shutil
import subprocess
from dataclasses import dataclass

import numpy as np

from . import _lib as L

__version__ = "0.1.0"

FLT_MAX = float(np.finfo(np.float32).max)
TERRAIN_FIELDS = L.TERRAIN_FIELDS
FIRE_FIELDS = L.FIRE_FIELDS


class PropagCudaError(RuntimeError):
    pass


class PropagGdalError(RuntimeError):
    pass


class PropagValidationError(ValueError):
    pass


class PropagMPIError(RuntimeError):
    pass


def _raise(rc: int, what: str):
    msg = f"{what}: {L.last_error()}"
    if rc == L.PROPAG_ERR_INVALID:
        raise PropagValidationError(msg)
    raise PropagCudaError(msg)


# --------------------------------------------------------------- geometry ----

def _gt_invert(gt):
    """GT::invert (crates/geometry/src/lib.rs:84-124) in f32."""
    f = np.float32
    x0, dx, rx, y0, ry, dy = (f(v) for v in gt)
    with np.errstate(all="ignore"):
        if rx == 0 and ry == 0 and dx != 0 and dy != 0:
            return [-x0 / dx, f(1) / dx, f(0), -y0 / dy, f(0), f(1) / dy]
        det = dx * dy - rx * ry
        mag = max(abs(dx), abs(rx), abs(ry), abs(dy))
        if not abs(det) > f(1e-10) * mag * mag:
            return None
        inv = f(1) / det
        return [(rx * y0 - x0 * dy) * inv, dy * inv, -rx * inv, (-dx * y0 + x0 * ry) * inv,
                -ry * inv, dx * inv]


class PyGeoReference:
    """Grid size, projection and transform (crates/py-propag/src/lib.rs:236-380)."""

    def __init__(self, width: int, height: int, proj: str, transform):
        if width == 0 or height == 0:
            raise PropagValidationError("Grid dimensions must be positive (width > 0, height > 0)")
        if width > 32768 or height > 32768:
            raise PropagValidationError("Grid dimensions too large (max 32768x32768)")
        if not proj:
            raise PropagValidationError("Projection string cannot be empty")
        pb = proj.encode()
        if len(pb) >= 1024:
            raise PropagValidationError("Projection string too large (max 1023 characters)")
        t = np.asarray(transform, dtype=np.float64).ravel()
        if t.size != 6:
            raise PropagValidationError(
                "Geo transform must have exactly 6 elements [x_origin, pixel_width, x_rotation, "
                "y_origin, y_rotation, pixel_height]")
        if t[1] == 0.0 or t[5] == 0.0:
            raise PropagValidationError("Invalid geo transform: pixel size cannot be zero")
        inv = _gt_invert(t.astype(np.float32))
        if inv is None:
            raise PropagValidationError(
                "Invalid geo transform parameters - ensure pixel sizes are non-zero and finite")
        g = L.GeoReference()
        g.width, g.height = int(width), int(height)
        C.memmove(g.proj, pb, len(pb))
        g.transform.gt = L.GT(*[float(np.float32(v)) for v in t])
        g.transform.inv = L.GT(*[float(v) for v in inv])
        self.inner = g

    @classmethod
    def _wrap(cls, g: "L.GeoReference") -> "PyGeoReference":
        obj = cls.__new__(cls)
        obj.inner = g
        return obj

    @classmethod
    def south_up(cls, x0, y0, x1, y1, dx, dy, proj: str) -> "PyGeoReference":
        g = L.GeoReference()
        if not L.lib().GeoReference_south_up(x0, y0, x1, y1, dx, dy, proj.encode(), C.byref(g)):
            raise PropagValidationError("GeoReference_south_up failed")
        return cls._wrap(g)

    @classmethod
    def north_up(cls, x0, y0, x1, y1, dx, dy, proj: str) -> "PyGeoReference":
        g = L.GeoReference()
        if not L.lib().GeoReference_north_up(x0, y0, x1, y1, dx, dy, proj.encode(), C.byref(g)):
            raise PropagValidationError("GeoReference_north_up failed")
        return cls._wrap(g)

    @property
    def width(self) -> int:
        return int(self.inner.width)

    @property
    def height(self) -> int:
        return int(self.inner.height)

    @property
    def proj(self) -> str:
        raw = bytes(self.inner.proj)
        return raw.split(b"\0", 1)[0].decode()

    @property
    def transform(self) -> np.ndarray:
        t = self.inner.transform.gt
        return np.array([t.x0, t.dx, t.rx, t.y0, t.ry, t.dy], dtype=np.float64)


class PySettings:
    """Settings{geo_ref, max_time} (crates/py-propag/src/lib.rs:172-234)."""

    def __init__(self, geo_ref: PyGeoReference, max_time: float):
        self._check(max_time)
        self.geo_ref = geo_ref
        self._max_time = float(np.float32(max_time))

    @staticmethod
    def _check(max_time):
        if max_time <= 0.0:
            raise PropagValidationError("Maximum simulation time must be positive")
        if not np.isfinite(max_time):
            raise PropagValidationError("Maximum simulation time must be a finite number")
        if max_time > 10.0 * 365.0 * 24.0 * 3600.0:
            raise PropagValidationError("Maximum simulation time too large (limit: 10 years)")

    @property
    def max_time(self) -> float:
        return self._max_time

    @max_time.setter
    def max_time(self, v: float):
        self._check(v)
        self._max_time = float(np.float32(v))

    @property
    def inner(self) -> "L.Settings":
        s = L.Settings()
        s.geo_ref = self.geo_ref.inner
        s.max_time = self._max_time
        return s


class PyTimeFeature:
    """An ignition: WKB geometry + time in seconds (lib.rs:381-433)."""

    def __init__(self, time: float, geom_wkb: bytes):
        if time < 0.0:
            raise PropagValidationError("Time must be non-negative")
        if not np.isfinite(time):
            raise PropagValidationError("Time must be a finite number")
        if len(geom_wkb) == 0:
            raise PropagValidationError("Geometry WKB cannot be empty")
        if len(geom_wkb) < 9:
            raise PropagValidationError("Invalid geometry WKB - too short for valid geometry")
        self.time = float(np.float32(time))
        self.geom_wkb = bytes(geom_wkb)


@dataclass
class PyPropagResults:
    """Results (lib.rs:434-486): arrival_times (H, W) f32, boundary_change
    (bit words u32), refs_x / refs_y (u16, row-major), geo_ref, shape."""
    arrival_times: np.ndarray
    boundary_change: np.ndarray
    refs_x: np.ndarray
    refs_y: np.ndarray
    geo_ref: PyGeoReference
    stats: dict

    @property
    def shape(self):
        return self.arrival_times.shape


Settings = PySettings
GeoReference = PyGeoReference
TimeFeature = PyTimeFeature
PropagResults = PyPropagResults


def check_cuda_available() -> bool:
    """True when libpropag sees a CUDA device."""
    try:
        return L.lib().propag_device_count() > 0
    except L.LibraryMissing:
        return False


def point_wkb(x: float, y: float) -> bytes:
    """Little-endian WKB POINT."""
    return b"\x01\x01\x00\x00\x00" + np.array([x, y], dtype="<f8").tobytes()


def _validate_path(path, name):
    if not path:
        raise PropagValidationError(f"{name} cannot be empty")
    if ".." in path:
        raise PropagValidationError(f"{name} contains invalid path components (..): {path}")
    if os.path.isabs(path) and path.startswith(("/etc", "/sys", "/proc")):
        raise PropagValidationError(f"{name} attempts to access restricted system directory: {path}")


def demo_terrain(width: int, height: int) -> dict:
    """The reference's constant loader (crates/propag/src/main.rs:44-55)."""
    shp = (height, width)
    t = {k: np.full(shp, 0.1, dtype=np.float32) for k in ("d1hr", "d10hr", "d100hr", "herb", "wood")}
    t.update(fuel_code=np.ones(shp, dtype=np.uint8), wind_speed=np.full(shp, 5.0, np.float32),
             wind_azimuth=np.zeros(shp, np.float32), slope=np.zeros(shp, np.float32),
             aspect=np.zeros(shp, np.float32))
    return t


def _terrain_host(terrain: dict, n: int):
    arrs = {}
    for k in TERRAIN_FIELDS:
        if k not in terrain:
            raise PropagValidationError(f"terrain is missing '{k}'")
        dt = np.uint8 if k == "fuel_code" else np.float32
        a = np.ascontiguousarray(terrain[k], dtype=dt).ravel()
        if a.size != n:
            raise PropagValidationError(f"terrain '{k}' has {a.size} cells, expected {n}")
        arrs[k] = a
    ptrs = L.PropagTerrainPtrs(*[arrs[k].ctypes.data for k in TERRAIN_FIELDS])
    return arrs, ptrs


def _time_features(features):
    bufs = []
    arr = (L.FFITimeFeature * max(len(features), 1))()
    for i, f in enumerate(features):
        b = (C.c_uint8 * len(f.geom_wkb)).from_buffer_copy(f.geom_wkb)
        bufs.append(b)
        arr[i].time = f.time
        arr[i].geom_wkb = C.cast(b, C.POINTER(C.c_uint8))
        arr[i].geom_wkb_len = len(f.geom_wkb)
    return arr, bufs


def rasterize_ignitions(geo_ref: PyGeoReference, features) -> np.ndarray:
    """TimeFeatures -> structured array of ignited cells (x, y, time)."""
    lib = L.lib()
    arr, keep = _time_features(features)
    n = lib.propag_rasterize_ignitions(C.byref(geo_ref.inner), arr, len(features), None, 0)
    if n < 0:
        _raise(int(n), "rasterize_ignitions")
    out = (L.PropagIgnition * max(int(n), 1))()
    lib.propag_rasterize_ignitions(C.byref(geo_ref.inner), arr, len(features), out, n)
    del keep
    return np.ctypeslib.as_array(out)[: int(n)].copy() if n else np.zeros(0, np.dtype(
        [("x", "<u4"), ("y", "<u4"), ("time", "<f4")]))


def _ignition_array(ignitions):
    if isinstance(ignitions, np.ndarray) and ignitions.dtype.names:
        a = np.ascontiguousarray(ignitions)
        return (L.PropagIgnition * max(len(a), 1)).from_buffer_copy(a.tobytes() or bytes(12)), len(a)
    items = list(ignitions)
    arr = (L.PropagIgnition * max(len(items), 1))()
    for i, (x, y, t) in enumerate(items):
        arr[i].x, arr[i].y, arr[i].time = int(x), int(y), float(t)
    return arr, len(items)


ARITH_REFERENCE = L.PROPAG_ARITH_REFERENCE
ARITH_PORTABLE = L.PROPAG_ARITH_PORTABLE


def _options(tile, cluster=0, threads=0, device=-1, arith=ARITH_REFERENCE):
    return L.PropagOptions(int(tile or 0), int(cluster or 0), int(threads or 0), int(device),
                           int(arith))


def propagate_arrays(settings: PySettings, terrain: dict, ignitions, *, tile=None, cluster=0,
                     threads=0, arith=ARITH_REFERENCE) -> PyPropagResults:
    """Fire behaviour + propagation for one grid, no files.  ignitions:
    iterable of (x, y, t) cells or the output of ``rasterize_ignitions``.
    arith: the float arithmetic of the propagation's time_from --
    ARITH_REFERENCE (the reference kernel's operations, the default) or
    ARITH_PORTABLE (operations a CPU reproduces bit for bit)."""
    lib = L.lib()
    g = settings.geo_ref
    n = g.width * g.height
    _arrs, ptrs = _terrain_host(terrain, n)
    ign, n_ign = _ignition_array(ignitions)
    time = np.empty(n, np.float32)
    rx = np.empty(n, np.uint16)
    ry = np.empty(n, np.uint16)
    bnd = np.empty((n + 31) // 32, np.uint32)
    st = L.PropagStats()
    opt = _options(tile, cluster, threads, arith=arith)
    s = settings.inner
    rc = lib.propag_run_host(C.byref(s), C.byref(ptrs), ign, n_ign, C.byref(opt),
                             time.ctypes.data, rx.ctypes.data, ry.ctypes.data, bnd.ctypes.data,
                             C.byref(st))
    if rc != 0:
        _raise(rc, "propagate")
    return PyPropagResults(time.reshape(g.height, g.width), bnd, rx, ry, g, st.as_dict())


def propagate(settings: PySettings, output_path: str, initial_ignited_elements,
              initial_ignited_elements_crs: str, refs_output_path=None,
              block_boundaries_out_path=None, grid_boundaries_out_path=None, *, terrain=None,
              tile=None) -> PyPropagResults:
    """Runs the propagation (crates/py-propag/src/lib.rs:595-700 signature)."""
    _validate_path(output_path, "output_path")
    for p, name in ((refs_output_path, "refs_output_path"),
                    (block_boundaries_out_path, "block_boundaries_out_path"),
                    (grid_boundaries_out_path, "grid_boundaries_out_path")):
        if p is not None:
            _validate_path(p, name)
    if not initial_ignited_elements_crs:
        raise PropagValidationError("Coordinate reference system (CRS) cannot be empty")
    if len(initial_ignited_elements_crs) > 2048:
        raise PropagValidationError("CRS string too long (max 2048 characters)")
    if not initial_ignited_elements:
        raise PropagValidationError("At least one ignition element is required")
    if len(initial_ignited_elements) > 10000:
        raise PropagValidationError("Too many ignition elements (max 10,000)")
    if not check_cuda_available():
        raise PropagCudaError(
            "CUDA is not available. Ensure NVIDIA GPU drivers and CUDA runtime are installed.")
    g = settings.geo_ref
    if initial_ignited_elements_crs.split() != g.proj.split():
        raise PropagGdalError("ignition CRS differs from the grid CRS; this build does not reproject")
    ign = rasterize_ignitions(g, initial_ignited_elements)
    t = terrain if terrain is not None else demo_terrain(g.width, g.height)
    res = propagate_arrays(settings, t, ign, tile=tile)
    write_geotiff(output_path, g, res.arrival_times)
    return res


def write_geotiff(path: str, geo_ref: PyGeoReference, data: np.ndarray) -> None:
    """Tiled float32 GeoTIFF, nodata f32::MAX (crates/propag/src/propag.rs:576-600)."""
    a = np.ascontiguousarray(data, dtype=np.float32)
    if a.size != geo_ref.width * geo_ref.height:
        raise PropagValidationError("raster size does not match the grid")
    rc = L.lib().propag_write_geotiff(C.byref(geo_ref.inner), a.ctypes.data, path.encode())
    if rc != 0:
        raise PropagGdalError(L.last_error())


def load_terrain_data(width, height, proj, transform, elevation=None, slope=None, aspect=None,
                      fuel_model=None) -> PyGeoReference:
    """Validates terrain rasters and returns their PyGeoReference
    (crates/py-propag/src/lib.rs:505-579)."""
    if width == 0 or height == 0:
        raise PropagValidationError("Grid dimensions must be positive")
    if width * height > 100_000_000:
        raise PropagValidationError(
            "Grid too large (limit: 100 million cells). Consider using smaller tiles.")

    def check(a, name, lo, hi):
        a = np.asarray(a)
        if a.shape != (height, width):
            raise PropagValidationError(
                f"{name} array shape mismatch: expected ({height}, {width}), got {a.shape}")
        if lo is not None and np.any(a < lo):
            r, c = np.argwhere(a < lo)[0]
            raise PropagValidationError(f"{name} value {a[r, c]} at position ({r}, {c}) is below minimum {lo}")
        if hi is not None and np.any(a > hi):
            r, c = np.argwhere(a > hi)[0]
            raise PropagValidationError(f"{name} value {a[r, c]} at position ({r}, {c}) exceeds maximum {hi}")

    if elevation is not None:
        check(elevation, "Elevation", -1000.0, 9000.0)
    if slope is not None:
        check(slope, "Slope", 0.0, 90.0)
    if aspect is not None:
        check(aspect, "Aspect", 0.0, 360.0)
    if fuel_model is not None:
        check(fuel_model, "Fuel model", None, None)
        fm = np.asarray(fuel_model)
        bad = np.argwhere(fm > 13)
        if bad.size:
            r, c = bad[0]
            raise PropagValidationError(
                f"Invalid fuel model ID {fm[r, c]} at position ({r}, {c}). Valid NFFL fuel models are 1-13.")
    return PyGeoReference(width, height, proj, transform)


# ------------------------------------------------------------ B200 extras ----

def fire_behaviour(terrain: dict, full: bool = False) -> dict:
    """The per-cell fire pass over host arrays (cuda_standard_simple_burn, or
    every FireCuda field + Byram + flame when full)."""
    lib = L.lib()
    shape = np.asarray(terrain["fuel_code"]).shape
    n = int(np.prod(shape))
    _arrs, ptrs = _terrain_host(terrain, n)
    names = FIRE_FIELDS if full else ("speed_max", "azimuth_max", "eccentricity")
    out = {k: np.empty(n, np.float32) for k in names}
    if full:
        f = L.PropagFireFields(*[out[k].ctypes.data for k in FIRE_FIELDS])
        rc = lib.propag_fire_full_host(n, C.byref(ptrs), C.byref(f))
    else:
        rc = lib.propag_fire_simple_host(n, C.byref(ptrs), out["speed_max"].ctypes.data,
                                         out["azimuth_max"].ctypes.data, out["eccentricity"].ctypes.data)
    if rc != 0:
        _raise(rc, "fire_behaviour")
    return {k: v.reshape(shape) for k, v in out.items()}


def dead_fuel_moisture(temperature, humidity, cloud_cover, precipitation, slope, aspect, fuel_code,
                       hour: int, month: int, scale: float = 1.0) -> dict:
    """Hourly dead fuel moisture per cell (the dmoist model) over host
    arrays: weather (24, ...) per hour, precipitation (6, ...) per day, the
    rest per cell.  Returns d1hr/d10hr/d100hr in the model's percent units
    times ``scale`` (0.01 for the fractions fire_behaviour takes)."""
    lib = L.lib()
    shape = np.asarray(slope).shape
    n = int(np.prod(shape))
    w = [np.ascontiguousarray(a, dtype=np.float32).reshape(k, n)
         for a, k in ((temperature, 24), (humidity, 24), (cloud_cover, 24), (precipitation, 6))]
    sl, asp = (np.ascontiguousarray(a, dtype=np.float32).ravel() for a in (slope, aspect))
    fu = np.ascontiguousarray(fuel_code, dtype=np.uint8).ravel()
    if sl.size != n or asp.size != n or fu.size != n:
        raise PropagValidationError("slope, aspect and fuel_code must have one value per cell")
    ptrs = L.PropagWeatherPtrs(*[a.ctypes.data for a in w])
    out = {k: np.empty(n, np.float32) for k in ("d1hr", "d10hr", "d100hr")}
    rc = lib.propag_dmoist_host(n, int(hour), int(month), C.byref(ptrs), sl.ctypes.data, asp.ctypes.data,
                                fu.ctypes.data, float(scale), out["d1hr"].ctypes.data,
                                out["d10hr"].ctypes.data, out["d100hr"].ctypes.data)
    if rc != 0:
        _raise(rc, "dead_fuel_moisture")
    return {k: v.reshape(shape) for k, v in out.items()}


class Engine:
    """Batched propagation over device-resident scenarios (propag_engine_*).
    Jobs are ``PropagJob`` structures holding device pointers."""

    def __init__(self, tile=None, cluster=0, threads=0, device=-1):
        lib = L.lib()
        opt = _options(tile, cluster, threads, device)
        self._h = lib.propag_engine_create(C.byref(opt))
        if not self._h:
            _raise(L.PROPAG_ERR_CUDA, "propag_engine_create")

    def run(self, jobs, stream=0, want_stats=True):
        arr = (L.PropagJob * len(jobs))(*jobs)
        stats = (L.PropagStats * len(jobs))() if want_stats else None
        rc = L.lib().propag_engine_run(self._h, arr, len(jobs), C.c_void_p(int(stream)), stats)
        if rc != 0:
            _raise(rc, "propag_engine_run")
        return [s.as_dict() for s in stats] if want_stats else None

    def close(self):
        if getattr(self, "_h", None):
            L.lib().propag_engine_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Graph:
    """A batch (fire passes + one persistent propagation launch) captured as
    a CUDA graph (propag_graph_*).  ``jobs``: ``PropagJob`` structures with
    device pointers; ``terrains``: one ``PropagTerrainPtrs`` (device) per job,
    or None when the fire rasters are inputs."""

    def __init__(self, jobs, terrains=None, tile=None, cluster=0, threads=0, device=-1):
        lib = L.lib()
        n = len(jobs)
        self.n = n
        arr = (L.PropagJob * n)(*jobs)
        tarr = (L.PropagTerrainPtrs * n)(*terrains) if terrains is not None else None
        opt = _options(tile, cluster, threads, device)
        self._h = lib.propag_graph_create(C.byref(opt), arr, tarr, n)
        if not self._h:
            _raise(L.PROPAG_ERR_CUDA, "propag_graph_create")

    def launch(self, stream=0):
        rc = L.lib().propag_graph_launch(self._h, C.c_void_p(int(stream)))
        if rc != 0:
            _raise(rc, "propag_graph_launch")

    def stats(self, stream=0):
        st = (L.PropagStats * self.n)()
        rc = L.lib().propag_graph_stats(self._h, C.c_void_p(int(stream)), st)
        if rc != 0:
            _raise(rc, "propag_graph_stats")
        return [s.as_dict() for s in st]

    def close(self):
        if getattr(self, "_h", None):
            L.lib().propag_graph_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Continuous-batching server (propag_server_*): submit device-resident
    scenarios from any thread; a dispatcher batches what is waiting onto free
    streams.  Results are dicts with the job's statistics, host times (ns)
    and the batch size it ran in."""

    def __init__(self, hbm_budget=0, lanes=0, max_batch=0, device=-1):
        opt = L.PropagServerOptions(int(hbm_budget), int(lanes), int(max_batch), int(device), 0)
        self._h = L.lib().propag_server_create(C.byref(opt))
        if not self._h:
            _raise(L.PROPAG_ERR_CUDA, "propag_server_create")

    def submit(self, job, terrain=None, device_bytes=0) -> int:
        rid = L.lib().propag_server_submit(self._h, C.byref(job),
                                           C.byref(terrain) if terrain is not None else None,
                                           int(device_bytes))
        if rid < 0:
            _raise(int(rid), "propag_server_submit")
        return int(rid)

    @staticmethod
    def _result(r):
        if r.status < 0:
            raise PropagCudaError(f"request failed ({r.status}): {r.message.decode()}")
        d = r.stats.as_dict()
        d.update(submit_ns=int(r.submit_ns), start_ns=int(r.start_ns), done_ns=int(r.done_ns),
                 batch_size=int(r.batch_size))
        return d

    def poll(self, rid):
        r = L.PropagServerResult()
        rc = L.lib().propag_server_poll(self._h, int(rid), C.byref(r))
        if rc < 0:
            _raise(rc, "propag_server_poll")
        return self._result(r) if rc == 1 else None

    def wait(self, rid, timeout_ms=600_000):
        r = L.PropagServerResult()
        rc = L.lib().propag_server_wait(self._h, int(rid), C.byref(r), int(timeout_ms))
        if rc < 0:
            _raise(rc, "propag_server_wait")
        if rc == 0:
            raise TimeoutError(f"request {rid} not done after {timeout_ms} ms")
        return self._result(r)

    def release(self, rid):
        L.lib().propag_server_release(self._h, int(rid))

    def close(self):
        if getattr(self, "_h", None):
            L.lib().propag_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def autotune(jobs, terrains=None, stream=0, repeats=1):
    """Fastest cluster size for this batch (propag_autotune): returns
    (options dict, milliseconds)."""
    n = len(jobs)
    arr = (L.PropagJob * n)(*jobs)
    tarr = (L.PropagTerrainPtrs * n)(*terrains) if terrains is not None else None
    best = L.PropagOptions()
    ms = C.c_float()
    rc = L.lib().propag_autotune(arr, tarr, n, C.c_void_p(int(stream)), int(repeats), C.byref(best),
                                 C.byref(ms))
    if rc != 0:
        _raise(rc, "propag_autotune")
    return {"tile": best.tile, "cluster": best.cluster, "threads": best.threads}, float(ms.value)


def build(force: bool = False) -> str:
    """Compiles libpropag.so for sm_100a with nvcc (make in csrc/)."""
    if force and os.path.exists(L.LIB_PATH):
        os.remove(L.LIB_PATH)
    make = shutil.which("make") or "make"
    subprocess.run([make, "-s", "-C", os.path.join(L.PKG_DIR, "csrc")], check=True)
    return L.LIB_PATH


__all__ = [
    "Settings", "PySettings", "GeoReference", "PyGeoReference", "TimeFeature", "PyTimeFeature",
    "PropagResults", "PyPropagResults", "propagate", "load_terrain_data", "check_cuda_available",
    "PropagCudaError", "PropagGdalError", "PropagValidationError", "PropagMPIError",
    "fire_behaviour", "propagate_arrays", "rasterize_ignitions", "write_geotiff", "point_wkb",
    "demo_terrain", "Engine", "Graph", "Server", "autotune", "dead_fuel_moisture", "build",
]
