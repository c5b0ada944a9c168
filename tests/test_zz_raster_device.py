"""Rasterisation on the device (raster.cu) against the host rasteriser, bit
for bit: the time raster of TimeFeatures (the reference's rasterize_times,
crates/propag/src/propag.rs:837-890: FLT_MAX where nothing burns, the last
feature over earlier ones), the fuel raster of FuelFeatures (rasterize_fuels,
:929-982, nodata 255), and the ignition list of a time raster, which must
start a propagation exactly like the host rasteriser's list.  The host
rasteriser itself is pinned to a scanline restatement in tests/test_raster.py
(on the CPU)."""
import ctypes as C

import numpy as np
import pytest

from test_raster import GRIDS, PROJ, georef, random_geometries, wkb_line, wkb_point, wkb_polygon

pytestmark = pytest.mark.gpu
FMAX = np.float32(np.finfo(np.float32).max)


@pytest.fixture(scope="module")
def L():
    from py_propag import _lib
    return _lib


def _time_features(L, items):
    arr = (L.FFITimeFeature * max(len(items), 1))()
    keep = []
    for i, (t, wkb) in enumerate(items):
        b = (C.c_uint8 * len(wkb)).from_buffer_copy(wkb)
        keep.append(b)
        arr[i].time, arr[i].geom_wkb, arr[i].geom_wkb_len = t, C.cast(b, C.POINTER(C.c_uint8)), len(wkb)
    return arr, keep


def _fuel_features(L, items):
    arr = (L.FFIFuelFeature * max(len(items), 1))()
    keep = []
    for i, (code, wkb) in enumerate(items):
        b = (C.c_uint8 * len(wkb)).from_buffer_copy(wkb)
        keep.append(b)
        arr[i].code, arr[i].geom_wkb, arr[i].geom_wkb_len = code, C.cast(b, C.POINTER(C.c_uint8)), len(wkb)
    return arr, keep


def _host_times(L, g, arr, n):
    lib = L.lib()
    k = lib.propag_rasterize_ignitions(C.byref(g), arr, n, None, 0)
    assert k >= 0
    out = (L.PropagIgnition * max(k, 1))()
    lib.propag_rasterize_ignitions(C.byref(g), arr, n, out, k)
    t = np.full(g.width * g.height, FMAX, np.float32)
    for i in range(k):  # in burn order: the last one wins
        t[out[i].x + out[i].y * g.width] = out[i].time
    return t, [(out[i].x, out[i].y, out[i].time) for i in range(k)]


def _device_times(L, g, arr, n):
    import torch
    d = torch.empty(g.width * g.height, dtype=torch.float32, device="cuda")
    rc = L.lib().propag_rasterize_times_device(C.byref(g), arr, n, d.data_ptr(), None)
    assert rc == 0, L.last_error()
    torch.cuda.synchronize()
    return d


def _features(rng, g, n):
    feats = random_geometries(rng, g, n)
    times = rng.uniform(0, 3600, n).astype(np.float32)
    return [(float(times[i]), wkb) for i, (wkb, _) in enumerate(feats)]


@pytest.mark.parametrize("grid", range(len(GRIDS)))
@pytest.mark.parametrize("seed", range(4))
def test_times_raster_equals_host(L, grid, seed):
    w, h, gt = GRIDS[grid]
    g = georef(L, w, h, gt)
    items = _features(np.random.default_rng(700 + 10 * grid + seed), g, 24)
    items.append((5.0, b"\x01\x07\x00\x00\x00garbage!"))  # invalid WKB: skipped
    items.append((6.0, b""))
    arr, keep = _time_features(L, items)
    expect, _ = _host_times(L, g, arr, len(items))
    got = _device_times(L, g, arr, len(items)).cpu().numpy()
    assert np.array_equal(got.view(np.uint32), expect.view(np.uint32))


def test_times_raster_no_features(L):
    g = georef(L, 33, 7, GRIDS[0][2])
    arr, keep = _time_features(L, [])
    got = _device_times(L, g, arr, 0).cpu().numpy()
    assert np.all(got == FMAX)


@pytest.mark.parametrize("w,h", [(65534, 3), (4099, 2050)])
def test_wide_grids(L, w, h):
    """Rows of up to 65534 cells (eight mask words per thread, carries across
    all eight warps), and a grid of 8.4 M cells.  The host's time raster is
    read off its fuel raster with feature k burnt as code k."""
    g = georef(L, w, h, (0.0, 2.0, 0.0, 0.0, 0.0, 2.0))
    rng = np.random.default_rng(w)
    items = []
    for k in range(12):  # world x = 2 col: vertices on a half-cell lattice
        xs = rng.integers(-40, 2 * w + 40, 6).astype(float)
        ys = rng.integers(-4, 2 * h + 4, 6).astype(float)
        ring = [(float(x), float(y)) for x, y in zip(xs, ys)]
        items.append((float(k) + 0.5, wkb_polygon([ring + [ring[0]]])))
    items.append((20.5, wkb_line([(-100.0, 1.0), (2.0 * w + 50.0, 2.0 * h - 1.0)])))
    items.append((21.5, wkb_point(2.0 * w - 1.0, 2.0 * h - 1.0)))
    fuels, fkeep = _fuel_features(L, [(k, wkb) for k, (_, wkb) in enumerate(items)])
    winner = _check_fuels(L, g, fuels, len(items))
    value = np.array([t for t, _ in items] + [FMAX] * (256 - len(items)), np.float32)
    expect = value[winner]
    assert np.count_nonzero(winner != 255) > w
    arr, keep = _time_features(L, items)
    got = _device_times(L, g, arr, len(items)).cpu().numpy()
    assert np.array_equal(got.view(np.uint32), expect.view(np.uint32))


def _check_fuels(L, g, arr, n):
    import torch
    lib = L.lib()
    N = g.width * g.height
    expect = np.zeros(N, np.uint8)
    err = C.create_string_buffer(256)
    assert lib.propag_rasterize_fuels(arr, n, PROJ.encode(), C.byref(g), expect.ctypes.data, err, 256)
    d = torch.zeros(N, dtype=torch.uint8, device="cuda")
    rc = lib.propag_rasterize_fuels_device(arr, n, PROJ.encode(), C.byref(g), d.data_ptr(), None)
    assert rc == 0, L.last_error()
    torch.cuda.synchronize()
    assert np.array_equal(d.cpu().numpy(), expect)
    return expect


@pytest.mark.parametrize("seed", range(3))
def test_fuels_raster_equals_host(L, seed):
    w, h, gt = GRIDS[seed % 2]
    g = georef(L, w, h, gt)
    feats = random_geometries(np.random.default_rng(900 + seed), g, 30)
    arr, keep = _fuel_features(L, [(i % 14, wkb) for i, (wkb, _) in enumerate(feats)])
    _check_fuels(L, g, arr, len(feats))


def test_fuels_device_rejects_other_crs(L):
    import torch
    g = georef(L, 8, 8, GRIDS[0][2])
    arr, keep = _fuel_features(L, [(1, wkb_point(1001.0, 2001.0))])
    d = torch.zeros(64, dtype=torch.uint8, device="cuda")
    rc = L.lib().propag_rasterize_fuels_device(arr, 1, b"EPSG:4326", C.byref(g), d.data_ptr(), None)
    assert rc == L.PROPAG_ERR_INVALID and "CRS" in L.last_error()
    # an empty CRS means "already in the grid CRS"
    assert L.lib().propag_rasterize_fuels_device(arr, 1, b"", C.byref(g), d.data_ptr(), None) == 0
    torch.cuda.synchronize()
    assert d.cpu().numpy()[0] == 1 and (d.cpu().numpy()[1:] == 255).all()


def _device_list(L, times, w, h, max_out=None):
    import torch
    lib = L.lib()
    n = lib.propag_ignitions_from_times_device(times.data_ptr(), w, h, None, 0, None)
    assert n >= 0, L.last_error()
    cap = n if max_out is None else max_out
    out = torch.zeros(max(cap, 1) * 3, dtype=torch.int32, device="cuda")
    k = lib.propag_ignitions_from_times_device(times.data_ptr(), w, h, out.data_ptr(), cap, None)
    assert k == n
    a = out.cpu().numpy()[: 3 * min(cap, n)].reshape(-1, 3)
    return n, a[:, 0].astype(np.uint32), a[:, 1].astype(np.uint32), a[:, 2].view(np.float32)


def test_ignition_list_row_major(L):
    import torch
    rng = np.random.default_rng(4)
    w, h = 4099, 37
    t = np.full(w * h, FMAX, np.float32)
    on = rng.random(w * h) < 0.02
    t[on] = rng.uniform(0, 100, on.sum()).astype(np.float32)
    t[5] = np.nan
    d = torch.from_numpy(t).cuda()
    n, x, y, tt = _device_list(L, d, w, h)
    idx = np.flatnonzero(t != FMAX)
    assert n == idx.size
    assert np.array_equal(x, idx % w) and np.array_equal(y, idx // w)
    assert np.array_equal(tt.view(np.uint32), t[idx].view(np.uint32))
    n2, x2, y2, _ = _device_list(L, d, w, h, max_out=10)  # truncated: the first 10
    assert n2 == n and np.array_equal(x2, x[:10]) and np.array_equal(y2, y[:10])


def test_device_ignitions_start_the_same_propagation(L, pp):
    """Host list (with repeats, in burn order) and device list (one entry per
    burning cell, row-major) give bit-identical propagations."""
    from conftest import random_terrain
    w, h = 96, 80
    gt = (0.0, 4.0, 0.0, 0.0, 0.0, 4.0)
    g = georef(L, w, h, gt)
    items = [(0.0, wkb_point(41.0, 33.0)),
             (600.0, wkb_line([(8.0, 300.0), (200.0, 250.0), (370.0, 300.0)])),
             (120.0, wkb_polygon([[(250.0, 40.0), (330.0, 40.0), (330.0, 90.0), (250.0, 90.0),
                                   (250.0, 40.0)]])),
             (60.0, wkb_point(41.0, 33.0)),  # the same cell again, later feature wins
             (900.0, wkb_polygon([[(100.0, 100.0), (180.0, 140.0), (120.0, 200.0)]]))]
    arr, keep = _time_features(L, items)
    _, host_list = _host_times(L, g, arr, len(items))
    d = _device_times(L, g, arr, len(items))
    n, x, y, tt = _device_list(L, d, w, h)
    dev_list = list(zip(x.tolist(), y.tolist(), tt.tolist()))
    assert n == len({(a, b) for a, b, _ in host_list}) < len(host_list)
    terrain = random_terrain(w * h, 11)
    terrain["fuel_code"][:] = 2
    s = pp.PySettings(pp.PyGeoReference._wrap(g), 7200.0)
    a = pp.propagate_arrays(s, terrain, host_list)
    b = pp.propagate_arrays(s, terrain, dev_list)
    assert np.array_equal(a.arrival_times.view(np.uint32), b.arrival_times.view(np.uint32))
    assert np.array_equal(a.refs_x, b.refs_x) and np.array_equal(a.refs_y, b.refs_y)
    assert np.array_equal(a.boundary_change, b.boundary_change)
    assert (a.arrival_times < FMAX).sum() > 100
