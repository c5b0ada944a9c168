"""The rasterisation kernels' own source, run on the CPU.

tests/emul/cuda_host_emul.hpp executes CUDA kernel source on the host (the
threads of a block as coroutines meeting at every barrier);
tests/emul/raster_emul.cpp compiles csrc/raster_kernels.cuh -- the file the
device build compiles -- against it, behind the same passes as raster.cu's
launchers, with the kernels' own 256-thread blocks.  Its rasters and
ignition lists must equal the host rasteriser's bit for bit: random mixed
geometries on the four test grids, rows of 65 534 cells (eight mask words per
thread, carries across all eight warps), several grid sizes (grid-stride
loops), and the row-major ignition list with NaN times and truncation.  The
same comparisons run on the GPU in tests/test_zz_raster_device.py."""
import ctypes as C
import os
import shutil
import subprocess

import numpy as np
import pytest

from test_raster import GRIDS, PROJ, georef, random_geometries, wkb_line, wkb_point, wkb_polygon

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
FMAX = np.float32(np.finfo(np.float32).max)


@pytest.fixture(scope="module")
def L():
    from py_propag import _lib
    return _lib


@pytest.fixture(scope="module")
def emul(tmp_path_factory):
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("no C++ compiler")
    out = str(tmp_path_factory.mktemp("emul") / "libraster_emul.so")
    csrc = os.path.join(ROOT, "propag-hidalgo_b200", "csrc")
    cmd = [cxx, "-std=c++20", "-O2", "-fPIC", "-shared", "-I" + os.path.join(ROOT, "include"),
           "-I" + csrc, "-I" + os.path.join(ROOT, "tests", "emul"),
           os.path.join(ROOT, "tests", "emul", "raster_emul.cpp"), os.path.join(csrc, "io.cpp"),
           "-o", out]
    subprocess.run(cmd, check=True, capture_output=True)
    E = C.CDLL(out)
    E.emul_rasterize_times.argtypes = [C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint]
    E.emul_rasterize_fuels.argtypes = [C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p, C.c_uint]
    E.emul_ignitions_from_times.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p, C.c_uint64,
                                            C.c_uint]
    E.emul_ignitions_from_times.restype = C.c_int64
    return E


def _features(L, ctype, items, value_field):
    arr = (ctype * max(len(items), 1))()
    keep = []
    for i, (v, wkb) in enumerate(items):
        b = (C.c_uint8 * max(len(wkb), 1)).from_buffer_copy(wkb or b"\0")
        keep.append(b)
        setattr(arr[i], value_field, v)
        arr[i].geom_wkb, arr[i].geom_wkb_len = C.cast(b, C.POINTER(C.c_uint8)), len(wkb)
    return arr, keep


def _host_times(L, g, arr, n):
    lib = L.lib()
    k = lib.propag_rasterize_ignitions(C.byref(g), arr, n, None, 0)
    out = (L.PropagIgnition * max(k, 1))()
    lib.propag_rasterize_ignitions(C.byref(g), arr, n, out, k)
    t = np.full(g.width * g.height, FMAX, np.float32)
    for i in range(k):
        t[out[i].x + out[i].y * g.width] = out[i].time
    return t


def _host_fuels(L, g, arr, n):
    out = np.zeros(g.width * g.height, np.uint8)
    err = C.create_string_buffer(256)
    assert L.lib().propag_rasterize_fuels(arr, n, PROJ.encode(), C.byref(g), out.ctypes.data, err, 256)
    return out


@pytest.mark.parametrize("grid", range(len(GRIDS)))
@pytest.mark.parametrize("seed", range(3))
def test_emulated_kernels_equal_host_rasteriser(L, emul, grid, seed):
    w, h, gt = GRIDS[grid]
    g = georef(L, w, h, gt)
    rng = np.random.default_rng(700 + 10 * grid + seed)
    feats = random_geometries(rng, g, 24)
    times = rng.uniform(0, 3600, len(feats)).astype(np.float32)
    items = [(float(times[i]), wkb) for i, (wkb, _) in enumerate(feats)]
    items += [(5.0, b"\x01\x07\x00\x00\x00garbage!"), (6.0, b"")]
    arr, keep = _features(L, L.FFITimeFeature, items, "time")
    got = np.empty(w * h, np.float32)
    emul.emul_rasterize_times(C.addressof(g), C.addressof(arr), len(items), got.ctypes.data, 1 + seed)
    assert np.array_equal(got.view(np.uint32), _host_times(L, g, arr, len(items)).view(np.uint32))
    fuel_items = [(i % 14, wkb) for i, (_, wkb) in enumerate(items)]
    farr, fkeep = _features(L, L.FFIFuelFeature, fuel_items, "code")
    fgot = np.empty(w * h, np.uint8)
    emul.emul_rasterize_fuels(C.addressof(farr), len(items), C.addressof(g), fgot.ctypes.data, 2)
    assert np.array_equal(fgot, _host_fuels(L, g, farr, len(items)))


def test_emulated_kernels_on_wide_rows(L, emul):
    w, h = 65534, 3
    g = georef(L, w, h, (0.0, 2.0, 0.0, 0.0, 0.0, 2.0))
    rng = np.random.default_rng(w)
    items = []
    for k in range(12):
        xs = rng.integers(-40, 2 * w + 40, 6).astype(float)
        ys = rng.integers(-4, 2 * h + 4, 6).astype(float)
        ring = [(float(x), float(y)) for x, y in zip(xs, ys)]
        items.append((k, wkb_polygon([ring + [ring[0]]])))
    items.append((12, wkb_line([(-100.0, 1.0), (2.0 * w + 50.0, 2.0 * h - 1.0)])))
    items.append((13, wkb_point(2.0 * w - 1.0, 2.0 * h - 1.0)))
    # feature k burns code k, so the host's fuel raster names each cell's winner
    farr, fkeep = _features(L, L.FFIFuelFeature, items, "code")
    expect = _host_fuels(L, g, farr, len(items))
    got = np.empty(w * h, np.uint8)
    emul.emul_rasterize_fuels(C.addressof(farr), len(items), C.addressof(g), got.ctypes.data, 2)
    assert np.array_equal(got, expect) and np.count_nonzero(expect != 255) > w
    tarr, tkeep = _features(L, L.FFITimeFeature, [(k + 0.5, wkb) for k, wkb in items], "time")
    value = np.array([k + 0.5 for k, _ in items] + [FMAX] * (256 - len(items)), np.float32)
    tgot = np.empty(w * h, np.float32)
    emul.emul_rasterize_times(C.addressof(g), C.addressof(tarr), len(items), tgot.ctypes.data, 3)
    assert np.array_equal(tgot.view(np.uint32), value[expect].view(np.uint32))


@pytest.mark.parametrize("w,h,density", [(4099, 5, 0.05), (1, 1, 1.0), (33, 1000, 0.001)])
def test_emulated_ignition_list(emul, w, h, density):
    rng = np.random.default_rng(w * h)
    t = np.full(w * h, FMAX, np.float32)
    on = rng.random(w * h) < density
    t[on] = rng.uniform(0, 100, on.sum()).astype(np.float32)
    if w * h > 10:
        t[5] = np.nan
    idx = np.flatnonzero(t != FMAX)
    out = np.zeros(3 * max(idx.size, 1), np.int32)
    n = emul.emul_ignitions_from_times(t.ctypes.data, w, h, out.ctypes.data, idx.size, 3)
    a = out[: 3 * idx.size].reshape(-1, 3)
    assert n == idx.size
    assert np.array_equal(a[:, 0], idx % w) and np.array_equal(a[:, 1], idx // w)
    assert np.array_equal(a[:, 2].view(np.uint32), t[idx].view(np.uint32))
    few = np.zeros(30, np.int32)
    assert emul.emul_ignitions_from_times(t.ctypes.data, w, h, few.ctypes.data, 10, 2) == n
    k = min(10, idx.size)
    assert np.array_equal(few.reshape(-1, 3)[:k, 0], idx[:k] % w)
