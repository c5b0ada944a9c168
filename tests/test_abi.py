"""The C-ABI library on a machine without a GPU: it loads, exports every
function the headers declare, and its host-side logic (geo-references,
rasterisation of WKB ignitions and fuels, error reporting of the plugin entry
point, the GeoTIFF writer) behaves like the reference's
(crates/geometry/src/lib.rs, crates/propag/src/propag.rs).  No compute call
reaches a device here: the GPU entry points must fail with an error."""
import ctypes as C
import glob
import os
import re
import struct

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PROJ = "+proj=utm +zone=30 +ellps=GRS80 +units=m +no_defs"


@pytest.fixture(scope="module")
def L():
    from py_propag import _lib
    return _lib


@pytest.fixture(scope="module")
def lib(L):
    return L.lib()


def _declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        src = re.sub(r"//[^\n]*", "", src)
        src = re.sub(r"^\s*#.*$", "", src, flags=re.M)
        src = re.sub(r"\{[^{}]*\}", "", src)
        src = re.sub(r"typedef[^;]*;", "", src)
        for m in re.finditer(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\([^;{]*\)\s*;", src):
            names.add(m.group(1))
    return sorted(names)


def test_headers_declare_the_reference_entry_points():
    names = _declared_functions()
    for ref in ("FFIPropagation_run", "propag_rasterize_fuels", "create_plugin", "create_settings",
                "create_fire", "GeoReference_len", "GeoReference_south_up", "GeoReference_north_up"):
        assert ref in names
    assert len(names) >= 25


def test_library_exports_every_declared_function(lib, L):
    for name in _declared_functions():
        assert hasattr(lib, name), name
        assert name in L.SIGNATURES, name  # the ctypes binding covers it too


def test_version_and_no_device(lib, pp):
    assert b"sm_100a" in lib.propag_version()
    if not pp.check_cuda_available():
        assert lib.propag_device_count() == 0


def test_struct_layouts(L):
    # repr(C) layouts of the reference (crates/geometry/src/lib.rs:20-28,127-131,180-187)
    assert C.sizeof(L.GT) == 24 and C.sizeof(L.GeoTransform) == 48
    assert C.sizeof(L.GeoReference) == 4 + 4 + 1024 + 48
    assert C.sizeof(L.Settings) == C.sizeof(L.GeoReference) + 4
    assert C.sizeof(L.FireSimpleCuda) == 12
    assert C.sizeof(L.FFITimeFeature) == 24 and C.sizeof(L.FFIFuelFeature) == 24
    assert C.sizeof(L.PluginT) == 16
    assert C.sizeof(L.PropagIgnition) == 12


def _header_defines():
    out = {}
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        for m in re.finditer(r"^#define\s+(PROPAG_[A-Z_0-9]+)\s+\(?(-?\d+)[uU]?\)?", open(h).read(), re.M):
            out[m.group(1)] = int(m.group(2))
    return out


def test_extension_structs_and_constants_match_the_header(L):
    # PropagStats (include/propag_b200.h): 13 u64 counters, status and
    # max_walk u32, then 4 u64 (start/done clocks, scan cells, barrier wait)
    assert C.sizeof(L.PropagStats) == 13 * 8 + 2 * 4 + 4 * 8
    names = [f[0] for f in L.PropagStats._fields_]
    assert names[-6:] == ["status", "max_walk", "t_start_ns", "t_done_ns", "scan_cells", "cyc_wait"]
    d = _header_defines()
    assert d["PROPAG_CLUSTER_GROUPS"] == L.PROPAG_CLUSTER_GROUPS == -1
    assert d["PROPAG_DEFAULT_TILE"] == L.PROPAG_DEFAULT_TILE
    assert d["PROPAG_ERR_TIMEOUT"] == L.PROPAG_ERR_TIMEOUT


def test_group_wait_selftest_needs_a_device(lib, L, pp):
    if pp.check_cuda_available():
        pytest.skip("a GPU is present")
    st = C.c_uint32(7)
    assert lib.propag_selftest_group_wait(C.byref(st)) == L.PROPAG_ERR_NO_DEVICE
    assert lib.propag_selftest_group_wait(None) != L.PROPAG_OK


def _georef(pp, w=100, h=80, gt=(1000.0, 5.0, 0.0, 2000.0, 0.0, 5.0)):
    return pp.PyGeoReference(w, h, PROJ, list(gt))


def test_georeference_extent_functions(lib, pp):
    g = _georef(pp)
    assert lib.GeoReference_len(C.byref(g.inner)) == 8000
    assert lib.GeoReference_x0(C.byref(g.inner)) == 1000.0
    assert lib.GeoReference_x1(C.byref(g.inner)) == 1500.0
    assert lib.GeoReference_y0(C.byref(g.inner)) == 2000.0
    assert lib.GeoReference_y1(C.byref(g.inner)) == 2400.0
    n = _georef(pp, gt=(1000.0, 5.0, 0.0, 2400.0, 0.0, -5.0))
    assert lib.GeoReference_y0(C.byref(n.inner)) == 2000.0
    assert lib.GeoReference_y1(C.byref(n.inner)) == 2400.0


def test_south_up_and_north_up_constructors(pp):
    s = pp.PyGeoReference.south_up(0.0, 0.0, 500.0, 250.0, 5.0, 5.0, PROJ)
    assert (s.width, s.height) == (100, 50)
    assert list(s.transform) == [0.0, 5.0, 0.0, 0.0, 0.0, 5.0]
    n = pp.PyGeoReference.north_up(0.0, 0.0, 500.0, 250.0, 5.0, 5.0, PROJ)
    assert (n.width, n.height) == (100, 50)
    assert n.transform[3] == 250.0 and n.transform[5] == -5.0
    assert s.proj == PROJ
    with pytest.raises(pp.PropagValidationError):
        pp.PyGeoReference.south_up(0.0, 0.0, -500.0, 250.0, 5.0, 5.0, PROJ)


def test_create_settings_and_fire(lib, pp):
    g = _georef(pp)
    s = lib.create_settings(g.inner, C.c_float(3600.0))
    assert s.max_time == 3600.0 and s.geo_ref.width == 100
    f = lib.create_fire(1.5, 0.25, 0.5)
    assert (f.speed_max, f.azimuth_max, f.eccentricity) == (1.5, 0.25, 0.5)
    p = lib.create_plugin()
    assert p.run and p.rasterize_fuels


# ---------------------------------------------------------------- WKB -------

def wkb_point(x, y, big=False, srid=None, z=None):
    o = ">" if big else "<"
    t = 1
    extra = b""
    if z is not None:
        t = 1001
    if srid is not None:
        t = (0x20000000 | 1)
        extra = struct.pack(o + "I", srid)
    body = struct.pack(o + "dd", x, y) + (struct.pack(o + "d", z) if z is not None else b"")
    return bytes([0 if big else 1]) + struct.pack(o + "I", t) + extra + body


def wkb_line(pts):
    return b"\x01" + struct.pack("<II", 2, len(pts)) + b"".join(struct.pack("<dd", *p) for p in pts)


def wkb_polygon(rings):
    out = b"\x01" + struct.pack("<II", 3, len(rings))
    for r in rings:
        out += struct.pack("<I", len(r)) + b"".join(struct.pack("<dd", *p) for p in r)
    return out


def wkb_multi(kind, parts):
    return b"\x01" + struct.pack("<II", kind, len(parts)) + b"".join(parts)


def _cells(pp, g, feats):
    ign = pp.rasterize_ignitions(g, feats)
    return sorted((int(a["x"]), int(a["y"]), float(a["time"])) for a in ign)


def test_rasterize_points(pp):
    g = _georef(pp)
    feats = [pp.PyTimeFeature(10.0, wkb_point(1012.5, 2007.5)),
             pp.PyTimeFeature(20.0, wkb_point(1012.5, 2007.5, big=True)),
             pp.PyTimeFeature(30.0, wkb_point(1022.5, 2007.5, srid=25830)),
             pp.PyTimeFeature(40.0, wkb_point(1032.5, 2007.5, z=55.0)),
             pp.PyTimeFeature(50.0, wkb_point(999.0, 2007.5)),       # outside: dropped
             pp.PyTimeFeature(60.0, b"\x01\x07\x00\x00\x00garbage!")]  # invalid: dropped
    assert _cells(pp, g, feats) == [(2, 1, 10.0), (2, 1, 20.0), (4, 1, 30.0), (6, 1, 40.0)]


def test_rasterize_north_up_point(pp):
    g = _georef(pp, gt=(1000.0, 5.0, 0.0, 2400.0, 0.0, -5.0))
    assert _cells(pp, g, [pp.PyTimeFeature(0.0, wkb_point(1002.0, 2398.0))]) == [(0, 0, 0.0)]
    assert _cells(pp, g, [pp.PyTimeFeature(0.0, wkb_point(1002.0, 2001.0))]) == [(0, 79, 0.0)]


def test_rasterize_line_and_polygon(pp):
    g = _georef(pp)
    line = wkb_line([(1002.5, 2002.5), (1027.5, 2002.5)])
    got = _cells(pp, g, [pp.PyTimeFeature(5.0, line)])
    assert sorted({(x, y) for x, y, _ in got}) == [(c, 0) for c in range(6)]
    # square covering cell centres of columns 2..5 and rows 3..4
    poly = wkb_polygon([[(1010.0, 2015.0), (1030.0, 2015.0), (1030.0, 2025.0), (1010.0, 2025.0),
                         (1010.0, 2015.0)]])
    got = {(x, y) for x, y, _ in _cells(pp, g, [pp.PyTimeFeature(0.0, poly)])}
    assert got == {(c, r) for c in range(2, 6) for r in range(3, 5)}
    # a hole removes its cells (even-odd)
    holed = wkb_polygon([[(1000.0, 2000.0), (1050.0, 2000.0), (1050.0, 2050.0), (1000.0, 2050.0),
                          (1000.0, 2000.0)],
                         [(1020.0, 2020.0), (1030.0, 2020.0), (1030.0, 2030.0), (1020.0, 2030.0),
                          (1020.0, 2020.0)]])
    got = {(x, y) for x, y, _ in _cells(pp, g, [pp.PyTimeFeature(0.0, holed)])}
    assert len(got) == 100 - 4 and (4, 4) not in got and (0, 0) in got
    multi = wkb_multi(4, [wkb_point(1002.0, 2002.0), wkb_point(1497.0, 2397.0)])
    assert {(x, y) for x, y, _ in _cells(pp, g, [pp.PyTimeFeature(0.0, multi)])} == {(0, 0), (99, 79)}


def _fuel_features(L, items):
    arr = (L.FFIFuelFeature * len(items))()
    keep = []
    for i, (code, wkb) in enumerate(items):
        b = (C.c_uint8 * len(wkb)).from_buffer_copy(wkb)
        keep.append(b)
        arr[i].code, arr[i].geom_wkb, arr[i].geom_wkb_len = code, C.cast(b, C.POINTER(C.c_uint8)), len(wkb)
    return arr, keep


def test_rasterize_fuels(lib, L, pp):
    g = _georef(pp, w=20, h=10)
    poly = wkb_polygon([[(1000.0, 2000.0), (1050.0, 2000.0), (1050.0, 2050.0), (1000.0, 2050.0),
                         (1000.0, 2000.0)]])
    arr, keep = _fuel_features(L, [(7, poly)])
    out = np.zeros(200, np.uint8)
    err = C.create_string_buffer(256)
    assert lib.propag_rasterize_fuels(arr, 1, PROJ.encode(), C.byref(g.inner), out.ctypes.data, err, 256)
    grid = out.reshape(10, 20)
    assert np.all(grid[:, :10] == 7) and np.all(grid[:, 10:] == 255)  # nodata 255
    # an empty CRS means "already in the grid CRS"
    assert lib.propag_rasterize_fuels(arr, 1, b"", C.byref(g.inner), out.ctypes.data, err, 256)
    assert not lib.propag_rasterize_fuels(arr, 1, b"EPSG:4326", C.byref(g.inner), out.ctypes.data, err, 256)
    assert b"CRS" in err.value


def _propagation(L, pp, out, loader, crs=PROJ, n_ign=1, w=32, h=32):
    g = _georef(pp, w=w, h=h)
    p = L.FFIPropagation()
    p.settings = L.Settings(g.inner, 3600.0)
    p.output_path = out.encode() if out is not None else None
    feats = (L.FFITimeFeature * 1)()
    wkb = wkb_point(1050.0, 2050.0)
    buf = (C.c_uint8 * len(wkb)).from_buffer_copy(wkb)
    feats[0].time, feats[0].geom_wkb, feats[0].geom_wkb_len = 0.0, C.cast(buf, C.POINTER(C.c_uint8)), len(wkb)
    p.initial_ignited_elements, p.initial_ignited_elements_len = feats, n_ign
    p.initial_ignited_elements_crs = crs.encode()
    p.terrain_loader = L.FFITerrainLoader(loader, None)
    return p, (feats, buf, loader)


def test_plugin_run_error_paths(lib, L, pp, tmp_path):
    calls = []

    def refuse(ctx, g, t):
        calls.append(g.contents.width)
        return False

    refuse_fn = L.LoadFn(refuse)
    err = C.create_string_buffer(128)
    p, keep = _propagation(L, pp, str(tmp_path / "a.tif"), refuse_fn)
    assert not lib.FFIPropagation_run(p, 128, err)
    assert err.value == b"load_extent_error" and calls == [32]

    p, keep = _propagation(L, pp, str(tmp_path / "a.tif"), refuse_fn, crs="EPSG:4326")
    assert not lib.FFIPropagation_run(p, 128, err)
    assert b"CRS" in err.value

    p, keep = _propagation(L, pp, None, refuse_fn)
    assert not lib.FFIPropagation_run(p, 128, err)
    assert b"output_path" in err.value

    # strncpy semantics (propag.rs:295-306): a short buffer is filled, unterminated
    small = C.create_string_buffer(b"\xaa" * 8, 8)
    p, keep = _propagation(L, pp, str(tmp_path / "a.tif"), refuse_fn)
    assert not lib.FFIPropagation_run(p, 4, small)
    assert small.raw[:4] == b"load" and small.raw[4:] == b"\xaa" * 4


def test_plugin_run_without_gpu_fails_loudly(lib, L, pp, tmp_path):
    if pp.check_cuda_available():
        pytest.skip("a GPU is present")

    def fill(ctx, g, t):
        n = g.contents.width * g.contents.height
        for k in ("d1hr", "d10hr", "d100hr", "herb", "wood"):
            C.memmove(getattr(t.contents, k), np.full(n, 0.1, np.float32).ctypes.data, 4 * n)
        C.memset(t.contents.fuel_code, 1, n)
        return True

    fn = L.LoadFn(fill)
    p, keep = _propagation(L, pp, str(tmp_path / "b.tif"), fn)
    err = C.create_string_buffer(256)
    assert not lib.FFIPropagation_run(p, 256, err)
    assert b"no CUDA device" in err.value
    assert not os.path.exists(tmp_path / "b.tif")


def test_device_entry_points_fail_without_gpu(lib, L, pp):
    if pp.check_cuda_available():
        pytest.skip("a GPU is present")
    assert lib.propag_engine_create(None) is None
    assert "no CUDA device" in L.last_error()
    assert lib.propag_server_create(None) is None
    assert "no CUDA device" in L.last_error()
    with pytest.raises(pp.PropagCudaError):
        pp.Server()
    t = pp.demo_terrain(4, 4)
    with pytest.raises(pp.PropagCudaError, match="no CUDA device"):
        pp.fire_behaviour(t)
    g = pp.PyGeoReference(4, 4, PROJ, [0, 5, 0, 0, 0, 5])
    with pytest.raises(pp.PropagCudaError):
        pp.propagate_arrays(pp.PySettings(g, 100.0), t, [(0, 0, 0.0)])


# ------------------------------------------------------------ GeoTIFF -------

def _read_tiff(path):
    b = open(path, "rb").read()
    assert b[:4] == b"II*\x00"
    ifd = struct.unpack_from("<I", b, 4)[0]
    n = struct.unpack_from("<H", b, ifd)[0]
    size = {1: 1, 2: 1, 3: 2, 4: 4, 12: 8}
    fmt = {1: "B", 2: "c", 3: "H", 4: "I", 12: "d"}
    tags = {}
    for i in range(n):
        tag, typ, cnt, val = struct.unpack_from("<HHII", b, ifd + 2 + 12 * i)
        nbytes = size[typ] * cnt
        at = ifd + 2 + 12 * i + 8 if nbytes <= 4 else val
        raw = b[at:at + nbytes]
        tags[tag] = raw.rstrip(b"\0").decode() if typ == 2 else struct.unpack("<" + fmt[typ] * cnt, raw)
    return b, tags


@pytest.mark.parametrize("w,h", [(300, 270), (100, 80), (256, 256), (257, 1)])
def test_geotiff_round_trip(pp, tmp_path, w, h):
    """Several tiles with ragged edges, a single tile (its offset inline in
    the IFD entry), exactly one full tile, a one-row grid."""
    g = pp.PyGeoReference(w, h, PROJ, [500000.0, 5.0, 0.0, 4000000.0, 0.0, -5.0])
    data = np.arange(w * h, dtype=np.float32).reshape(h, w) * 0.5
    data[min(5, h - 1), 7] = np.finfo(np.float32).max
    path = str(tmp_path / "t.tif")
    pp.write_geotiff(path, g, data)
    b, tags = _read_tiff(path)
    assert tags[256] == (w,) and tags[257] == (h,) and tags[258] == (32,) and tags[339] == (3,)
    assert tags[322] == (256,) and tags[323] == (256,)
    assert tags[42113] == "3.40282346638529e+38"
    mt = tags[34264]
    assert mt[0] == 5.0 and mt[3] == 500000.0 and mt[5] == -5.0 and mt[7] == 4000000.0
    assert PROJ in tags[34737]
    offs = tags[324]
    tx, ty = (w + 255) // 256, (h + 255) // 256
    assert len(offs) == tx * ty
    out = np.empty((h, w), np.float32)
    for t, off in enumerate(offs):
        tile = np.frombuffer(b, dtype="<f4", count=256 * 256, offset=off).reshape(256, 256)
        r0, c0 = (t // tx) * 256, (t % tx) * 256
        rr, cc = min(256, h - r0), min(256, w - c0)
        out[r0:r0 + rr, c0:c0 + cc] = tile[:rr, :cc]
        assert np.all(tile[rr:, :] == np.finfo(np.float32).max)
    assert np.array_equal(out, data)
    with pytest.raises(pp.PropagValidationError):
        pp.write_geotiff(path, g, data.ravel()[:10])


def _gpkg_geoms(path, layer):
    """(geometry type name, srs id, [(x, y), ...] per feature) read back with
    SQLite, decoding the GeoPackage blob header and the little-endian WKB."""
    import sqlite3
    import struct
    db = sqlite3.connect(path)
    assert db.execute("PRAGMA application_id").fetchone()[0] == 0x47504B47
    (gtype, srs), = db.execute("SELECT geometry_type_name, srs_id FROM gpkg_geometry_columns "
                               "WHERE table_name = ?", (layer,)).fetchall()
    assert db.execute("SELECT data_type FROM gpkg_contents WHERE table_name = ?",
                      (layer,)).fetchone()[0] == "features"
    out = []
    for (blob,) in db.execute(f'SELECT geom FROM "{layer}" ORDER BY fid'):
        assert blob[:2] == b"GP" and blob[3] == 0x03
        assert struct.unpack_from("<i", blob, 4)[0] == srs
        wkb = blob[8 + 32:]
        order, typ = wkb[0], struct.unpack_from("<I", wkb, 1)[0]
        assert order == 1
        o = 5
        if typ == 3:
            assert struct.unpack_from("<I", wkb, o)[0] == 1
            o += 4
        n = struct.unpack_from("<I", wkb, o)[0]
        pts = struct.unpack_from(f"<{2 * n}d", wkb, o + 4)
        out.append(list(zip(pts[0::2], pts[1::2])))
    db.close()
    return gtype, srs, out


def test_refs_geopackage(lib, pp, tmp_path):
    """propag_write_refs_gpkg: one LineString per burned cell, from its
    reference's centre to its own, columns outer (propag.rs:699-750)."""
    g = _georef(pp, w=4, h=3)
    time = np.full(12, np.finfo(np.float32).max, np.float32)
    rx = np.zeros(12, np.uint16)
    ry = np.zeros(12, np.uint16)
    burned = [(0, 0, 0, 0), (2, 1, 0, 0), (1, 2, 2, 1)]  # (x, y, ref x, ref y)
    for (x, y, a, b) in burned:
        time[x + y * 4] = 10.0
        rx[x + y * 4], ry[x + y * 4] = a, b
    path = str(tmp_path / "refs.gpkg")
    assert lib.propag_write_refs_gpkg(C.byref(g.inner), time.ctypes.data, rx.ctypes.data,
                                      ry.ctypes.data, path.encode()) == 0
    gtype, srs, geoms = _gpkg_geoms(path, "fire_references")
    assert gtype == "LINESTRING"
    centre = lambda c, r: (1000.0 + (c + 0.5) * 5.0, 2000.0 + (r + 0.5) * 5.0)
    want = [[centre(a, b), centre(x, y)] for (x, y, a, b) in sorted(burned)]
    assert geoms == want
    # a second call replaces the file
    time[:] = np.finfo(np.float32).max
    assert lib.propag_write_refs_gpkg(C.byref(g.inner), time.ctypes.data, rx.ctypes.data,
                                      ry.ctypes.data, path.encode()) == 0
    assert _gpkg_geoms(path, "fire_references")[2] == []


def _wkt_balanced(w):
    depth = 0
    for ch in w:
        depth += {"[": 1, "]": -1}.get(ch, 0)
        if depth < 0:
            return False
    return depth == 0 and w.count('"') % 2 == 0


@pytest.mark.parametrize("crs,srs_id,org,has", [
    (PROJ, 100000, "NONE", ['PROJCS["unknown"', 'SPHEROID["GRS 1980",6378137,298.257222101',
                            'PARAMETER["central_meridian",-3]', 'PARAMETER["false_northing",0]']),
    ("+proj=utm +zone=33 +south +datum=WGS84 +units=m +no_defs", 100000, "NONE",
     ['GEOGCS["WGS 84"', 'PARAMETER["central_meridian",15]', 'PARAMETER["false_northing",10000000]']),
    ("EPSG:25830", 25830, "EPSG", ['PROJCS["ETRS89 / UTM zone 30N"', 'AUTHORITY["EPSG","4258"]',
                                  'AUTHORITY["EPSG","25830"]']),
    ("epsg:32733", 32733, "EPSG", ['PROJCS["WGS 84 / UTM zone 33S"', 'PARAMETER["false_northing",10000000]']),
    ("EPSG:4326", 4326, "EPSG", ['GEOGCS["WGS 84"']),
    ("+proj=longlat +ellps=GRS80 +no_defs", 100000, "NONE", ['GEOGCS["unknown"', 'GRS 1980']),
    ("+proj=lcc +lat_1=40 +ellps=GRS80", 100000, "NONE", None),  # needs a projection library
    ("EPSG:2062", 100000, "NONE", None),                         # needs the EPSG database
])
def test_geopackage_crs_rows(lib, pp, tmp_path, crs, srs_id, org, has):
    """The layer's srs row: WKT for the CRSs that need no database (EPSG:4326,
    WGS 84 and ETRS89 UTM zones, PROJ strings of UTM / longlat on WGS 84 or
    GRS 1980), "undefined" otherwise; the projection string stays in the
    description, and the layer and its geometries carry the row's id."""
    import sqlite3
    g = pp.PyGeoReference(4, 3, crs, [1000.0, 5.0, 0.0, 2000.0, 0.0, 5.0])
    time = np.full(12, 1.0, np.float32)
    zeros = np.zeros(12, np.uint16)
    path = str(tmp_path / "refs.gpkg")
    assert lib.propag_write_refs_gpkg(C.byref(g.inner), time.ctypes.data, zeros.ctypes.data,
                                      zeros.ctypes.data, path.encode()) == 0
    _, srs, geoms = _gpkg_geoms(path, "fire_references")
    assert srs == srs_id and len(geoms) == 12
    db = sqlite3.connect(path)
    rows = db.execute("SELECT organization, organization_coordsys_id, definition, description "
                      "FROM gpkg_spatial_ref_sys WHERE srs_id = ?", (srs_id,)).fetchall()
    assert db.execute("SELECT srs_id FROM gpkg_contents").fetchone()[0] == srs_id
    db.close()
    assert len(rows) == 1
    o, oid, definition, description = rows[0]
    assert o == org and oid == srs_id
    if srs_id != 4326:
        assert description == crs
    if has is None:
        assert definition == "undefined"
    else:
        assert _wkt_balanced(definition)
        for piece in has:
            assert piece in definition, piece


def test_boundaries_geopackage(lib, pp, tmp_path):
    """propag_write_boundaries_gpkg: the super-grid tiles ("grids") and their
    19 x 19 thread blocks ("blocks") as closed polygons (propag.rs:601-697)."""
    g = _georef(pp, w=100, h=80)
    gp, bp = str(tmp_path / "grids.gpkg"), str(tmp_path / "blocks.gpkg")
    assert lib.propag_write_boundaries_gpkg(C.byref(g.inner), 57, gp.encode(), bp.encode()) == 0
    gtype, _, grids = _gpkg_geoms(gp, "grids")
    assert gtype == "POLYGON" and len(grids) == 2 * 2
    assert grids[0] == [(1000.0, 2000.0), (1285.0, 2000.0), (1285.0, 2285.0), (1000.0, 2285.0),
                        (1000.0, 2000.0)]
    _, _, blocks = _gpkg_geoms(bp, "blocks")
    assert len(blocks) == 4 * 3 * 3
    assert blocks[1][0] == (1000.0 + 19 * 5.0, 2000.0)
    assert lib.propag_write_boundaries_gpkg(C.byref(g.inner), 0, gp.encode(), None) == 0
    assert len(_gpkg_geoms(gp, "grids")[2]) == 1
