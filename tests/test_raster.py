"""Rasterisation of WKB geometries without a GPU.

1. The host rasteriser (propag_rasterize_ignitions / propag_rasterize_fuels)
   against a scanline restatement of GDALRasterizeGeometries' default burn
   rules written here in plain Python: the cell holding a point; along a
   segment, ceil(max(|dcol|, |drow|)) equal steps and the cell under each
   sample; for a polygon, on each row's centre line the sorted crossings of
   all (closed) rings paired up, and the cells whose centre lies in
   [x0, x1), [x2, x3), ...  Burn order and repeats must agree one for one.
   Coordinates sit on a quarter-cell lattice, so crossings and samples fall
   exactly on cell edges and centres: the tie rules are what is tested.
2. The bit logic of the device kernels (raster.cu), restated step for step
   with the kernels' own constants (256 threads, 8 warps, 4096-cell chunks):
   the polygon kernel's row mask (toggles -> per-thread word ranges, warp
   ballots and carries -> inclusive prefix XOR) against a cumulative XOR,
   the binary search over `before` against searchsorted, and the ignition
   list's count / scan / ballot-compaction against np.flatnonzero.
The kernels' own source runs on the CPU against the host rasteriser in
tests/test_raster_kernels_emulated.py, and on the device in
tests/test_zz_raster_device.py."""
import ctypes as C
import math
import struct

import numpy as np
import pytest

PROJ = "+proj=utm +zone=30 +ellps=GRS80 +units=m +no_defs"


@pytest.fixture(scope="module")
def L():
    from py_propag import _lib
    return _lib


# ---------------------------------------------------------------- WKB -------
def wkb_point(x, y):
    return b"\x01" + struct.pack("<Idd", 1, x, y)


def wkb_line(pts):
    return b"\x01" + struct.pack("<II", 2, len(pts)) + b"".join(struct.pack("<dd", *p) for p in pts)


def wkb_polygon(rings):
    out = b"\x01" + struct.pack("<II", 3, len(rings))
    for r in rings:
        out += struct.pack("<I", len(r)) + b"".join(struct.pack("<dd", *p) for p in r)
    return out


def wkb_multi(kind, parts):
    return b"\x01" + struct.pack("<II", kind, len(parts)) + b"".join(parts)


def georef(L, w, h, gt):
    """A GeoReference with an exactly invertible transform (power-of-two
    pixel sizes, no rotation)."""
    g = L.GeoReference()
    g.width, g.height = w, h
    pb = PROJ.encode()
    C.memmove(g.proj, pb, len(pb))
    x0, dx, _, y0, _, dy = gt
    g.transform.gt = L.GT(x0, dx, 0.0, y0, 0.0, dy)
    g.transform.inv = L.GT(-x0 / dx, 1.0 / dx, 0.0, -y0 / dy, 0.0, 1.0 / dy)
    return g


# ------------------------------------------------------ Python restatement --
def _pix(g, x, y):
    v = g.transform.inv
    return v.x0 + x * v.dx + y * v.rx, v.y0 + x * v.ry + y * v.dy


def scanline(g, geom):
    """Cells burnt by one geometry, in the host's order: points, line
    segments sample by sample, polygons row by row.  geom = (points, lines,
    polygons) in world coordinates."""
    W, H = g.width, g.height
    out = []

    def put(c, r):
        if 0 <= c < W and 0 <= r < H:
            out.append((c, r))

    points, lines, polys = geom
    for x, y in points:
        c, r = _pix(g, x, y)
        put(math.floor(c), math.floor(r))
    for line in lines:
        for a, b in zip(line, line[1:]):
            c0, r0 = _pix(g, *a)
            c1, r1 = _pix(g, *b)
            dc, dr = c1 - c0, r1 - r0
            steps = math.ceil(max(abs(dc), abs(dr)))
            if steps == 0:
                put(math.floor(c0), math.floor(r0))
                continue
            for s in range(steps + 1):
                t = s / steps
                put(math.floor(c0 + t * dc), math.floor(r0 + t * dr))
    for rings in polys:
        px = [[_pix(g, *p) for p in ring] for ring in rings]
        edges = []
        for ring in px:
            edges += list(zip(ring, ring[1:]))
            if len(ring) >= 2 and ring[0] != ring[-1]:
                edges.append((ring[-1], ring[0]))
        ys = [p[1] for ring in px for p in ring]
        if not edges or not ys:
            continue
        for r in range(max(0, math.floor(min(ys))), min(H - 1, math.ceil(max(ys))) + 1):
            yc = r + 0.5
            xs = sorted(a[0] + (yc - a[1]) * (b[0] - a[0]) / (b[1] - a[1])
                        for a, b in edges if (a[1] <= yc < b[1]) or (b[1] <= yc < a[1]))
            for k in range(0, len(xs) - 1, 2):
                ca, cb = math.ceil(xs[k] - 0.5), math.ceil(xs[k + 1] - 0.5) - 1
                for c in range(max(ca, 0), min(cb, W - 1) + 1):
                    put(c, r)
    return out


def random_geometries(rng, g, n):
    """n features of mixed kinds on a quarter-cell lattice around the grid
    (some reaching outside it); returns [(wkb, (points, lines, polygons))]."""
    W, H = g.width, g.height
    x0, dx, y0, dy = g.transform.gt.x0, g.transform.gt.dx, g.transform.gt.y0, g.transform.gt.dy

    def pt(margin=6):
        c = rng.integers(-4 * margin, 4 * (W + margin)) / 4.0
        r = rng.integers(-4 * margin, 4 * (H + margin)) / 4.0
        return (x0 + c * dx, y0 + r * dy)

    out = []
    for _ in range(n):
        kind = rng.integers(0, 7)
        if kind == 0:
            p = pt(0)
            out.append((wkb_point(*p), ([p], [], [])))
        elif kind == 1:
            ps = [pt(0) for _ in range(rng.integers(2, 6))]
            out.append((wkb_multi(4, [wkb_point(*p) for p in ps]), (ps, [], [])))
        elif kind == 2:
            line = [pt() for _ in range(rng.integers(2, 5))]
            out.append((wkb_line(line), ([], [line], [])))
        elif kind == 3:  # a rectangle, edges on lattice lines, sometimes with a hole
            a, b = pt(), pt()
            ring = [(a[0], a[1]), (b[0], a[1]), (b[0], b[1]), (a[0], b[1]), (a[0], a[1])]
            rings = [ring]
            if rng.random() < 0.5:
                m = ((a[0] + b[0]) / 2, (a[1] + b[1]) / 2)
                q = (m[0] + (b[0] - a[0]) / 4, m[1] + (b[1] - a[1]) / 4)
                rings.append([(m[0], m[1]), (q[0], m[1]), (q[0], q[1]), (m[0], q[1]), (m[0], m[1])])
            out.append((wkb_polygon(rings), ([], [], [rings])))
        elif kind == 4:  # a random star-shaped or self-intersecting ring
            k = rng.integers(3, 9)
            ring = [pt() for _ in range(k)]
            if rng.random() < 0.7:
                ring.append(ring[0])  # closed; the others are closed by the rasteriser
            out.append((wkb_polygon([ring]), ([], [], [[ring]])))
        elif kind == 5:  # multipolygon of two triangles
            polys = [[[pt(), pt(), pt()]] for _ in range(2)]
            for p in polys:
                p[0].append(p[0][0])
            out.append((wkb_multi(6, [wkb_polygon(p) for p in polys]), ([], [], polys)))
        else:  # a collection of a point, a line and a polygon
            p, line, tri = pt(0), [pt(), pt()], [pt(), pt(), pt()]
            tri.append(tri[0])
            wkb = wkb_multi(7, [wkb_point(*p), wkb_line(line), wkb_polygon([tri])])
            out.append((wkb, ([p], [line], [[tri]])))
    return out


GRIDS = [(41, 29, (1000.0, 4.0, 0.0, 2000.0, 0.0, 4.0)),        # south-up
         (37, 23, (1000.0, 0.5, 0.0, 2000.0 + 23 * 0.5, 0.0, -0.5)),  # north-up
         (1, 17, (0.0, 2.0, 0.0, 0.0, 0.0, 2.0)),
         (19, 1, (0.0, 2.0, 0.0, 0.0, 0.0, -2.0))]


def _time_features(L, items):
    arr = (L.FFITimeFeature * max(len(items), 1))()
    keep = []
    for i, (t, wkb) in enumerate(items):
        b = (C.c_uint8 * len(wkb)).from_buffer_copy(wkb)
        keep.append(b)
        arr[i].time, arr[i].geom_wkb, arr[i].geom_wkb_len = t, C.cast(b, C.POINTER(C.c_uint8)), len(wkb)
    return arr, keep


def _host_ignitions(L, g, arr, n):
    lib = L.lib()
    k = lib.propag_rasterize_ignitions(C.byref(g), arr, n, None, 0)
    assert k >= 0
    out = (L.PropagIgnition * max(k, 1))()
    assert lib.propag_rasterize_ignitions(C.byref(g), arr, n, out, k) == k
    return [(out[i].x, out[i].y, out[i].time) for i in range(k)]


@pytest.mark.parametrize("grid", range(len(GRIDS)))
@pytest.mark.parametrize("seed", range(6))
def test_host_rasteriser_matches_scanline_restatement(L, grid, seed):
    w, h, gt = GRIDS[grid]
    g = georef(L, w, h, gt)
    rng = np.random.default_rng(1000 * grid + seed)
    feats = random_geometries(rng, g, 24)
    expect = []
    for i, (_, geom) in enumerate(feats):
        expect += [(c, r, float(i)) for c, r in scanline(g, geom)]
    arr, keep = _time_features(L, [(float(i), wkb) for i, (wkb, _) in enumerate(feats)])
    got = _host_ignitions(L, g, arr, len(feats))
    assert got == expect
    del keep


def test_host_rasteriser_tie_rules(L):
    """Crossings exactly on a cell centre open the span there and close it
    there (half-open [x0, x1)); rows whose centre line passes through a
    vertex count the edge above it, not the one below (y0 <= y < y1)."""
    g = georef(L, 10, 10, (0.0, 1.0, 0.0, 0.0, 0.0, 1.0))
    sq = [(2.5, 2.5), (6.5, 2.5), (6.5, 6.5), (2.5, 6.5), (2.5, 2.5)]
    arr, keep = _time_features(L, [(0.0, wkb_polygon([sq]))])
    cells = {(x, y) for x, y, _ in _host_ignitions(L, g, arr, 1)}
    assert cells == {(c, r) for c in range(2, 6) for r in range(2, 6)}
    diamond = [(5.0, 1.5), (8.5, 5.0), (5.0, 8.5), (1.5, 5.0), (5.0, 1.5)]
    arr, keep = _time_features(L, [(0.0, wkb_polygon([diamond]))])
    got = _host_ignitions(L, g, arr, 1)
    assert [(x, y) for x, y, _ in got] == scanline(g, ([], [], [[diamond]]))
    # an unclosed ring is closed
    arr, keep = _time_features(L, [(0.0, wkb_polygon([sq[:-1]]))])
    assert {(x, y) for x, y, _ in _host_ignitions(L, g, arr, 1)} == cells
    del keep


def test_host_line_far_outside_is_clipped(L):
    """A segment that starts a million cells away burns the same cells as the
    full sampling, without taking a million steps (samples are clipped to
    the ones that can reach the grid)."""
    g = georef(L, 64, 48, (0.0, 1.0, 0.0, 0.0, 0.0, 1.0))
    line = [(-1.0e6 + 0.25, -0.75e6 + 0.5), (63.25, 47.75)]
    arr, keep = _time_features(L, [(3.0, wkb_line(line))])
    got = _host_ignitions(L, g, arr, 1)
    # the full sampling restated over the samples near the grid only
    c0, r0 = line[0]
    dc, dr = line[1][0] - c0, line[1][1] - r0
    steps = math.ceil(max(abs(dc), abs(dr)))
    exp = []
    for s in range(steps - 200, steps + 1):
        t = s / steps
        c, r = math.floor(c0 + t * dc), math.floor(r0 + t * dr)
        if 0 <= c < 64 and 0 <= r < 48:
            exp.append((c, r, 3.0))
    assert got == exp and len(got) >= 48
    # lines beyond 2^40 cells are left out
    arr, keep = _time_features(L, [(3.0, wkb_line([(-2.0 ** 41, 0.5), (10.5, 0.5)]))])
    assert _host_ignitions(L, g, arr, 1) == []
    del keep


@pytest.mark.parametrize("seed", range(3))
def test_host_fuels_last_feature_wins(L, seed):
    w, h, gt = GRIDS[0]
    g = georef(L, w, h, gt)
    rng = np.random.default_rng(50 + seed)
    feats = random_geometries(rng, g, 30)
    expect = np.full((h, w), 255, np.uint8)
    for i, (_, geom) in enumerate(feats):
        for c, r in scanline(g, geom):
            expect[r, c] = i % 14
    arr = (L.FFIFuelFeature * len(feats))()
    keep = []
    for i, (wkb, _) in enumerate(feats):
        b = (C.c_uint8 * len(wkb)).from_buffer_copy(wkb)
        keep.append(b)
        arr[i].code, arr[i].geom_wkb, arr[i].geom_wkb_len = i % 14, C.cast(b, C.POINTER(C.c_uint8)), len(wkb)
    out = np.zeros(w * h, np.uint8)
    err = C.create_string_buffer(256)
    assert L.lib().propag_rasterize_fuels(arr, len(feats), PROJ.encode(), C.byref(g), out.ctypes.data, err, 256)
    assert np.array_equal(out.reshape(h, w), expect)


# ------------------------------------------- the device kernels' bit logic --
THREADS, WARPS, CHUNK = 256, 8, 4096


def _popc(x):
    return bin(x).count("1")


def row_mask_as_kernel(toggles, W):
    """polygon_kernel's steps after the toggles: words per thread, ballot of
    per-thread parities, warp parities, carries, shifts-and-XOR prefix."""
    nw = (W + 31) // 32
    mask = [0] * nw
    for c in toggles:
        mask[c >> 5] ^= 1 << (c & 31)
    per = (nw + THREADS - 1) // THREADS
    rng_ = [(min(nw, t * per), min(nw, min(nw, t * per) + per)) for t in range(THREADS)]
    par = [0] * THREADS
    for t, (a, b) in enumerate(rng_):
        for w in range(a, b):
            par[t] ^= _popc(mask[w]) & 1
    votes = [sum(par[32 * k + l] << l for l in range(32)) for k in range(WARPS)]
    warp_parity = [_popc(v) & 1 for v in votes]
    out = list(mask)
    for t, (a, b) in enumerate(rng_):
        lane, wid = t & 31, t >> 5
        carry = _popc(votes[wid] & ((1 << lane) - 1)) & 1
        for k in range(wid):
            carry ^= warp_parity[k]
        for w in range(a, b):
            m = mask[w]
            for sh in (1, 2, 4, 8, 16):
                m ^= (m << sh) & 0xFFFFFFFF
            out[w] = (~m & 0xFFFFFFFF) if carry else m
            carry ^= _popc(mask[w]) & 1
    return np.array([(out[c >> 5] >> (c & 31)) & 1 for c in range(W)], bool)


@pytest.mark.parametrize("W", [1, 31, 33, 1000, 8199, 32768, 65534])
def test_row_mask_logic(W):
    rng = np.random.default_rng(W)
    for n in (0, 1, 2, 7, 64):
        toggles = rng.integers(0, W, n)
        got = row_mask_as_kernel(list(toggles), W)
        bits = np.zeros(W, np.int64)
        np.add.at(bits, toggles, 1)
        expect = (np.cumsum(bits) & 1).astype(bool)
        assert np.array_equal(got, expect), (W, n)


def find_part_as_kernel(before, i):
    lo, hi = 0, len(before) - 1
    while lo < hi:
        mid = lo + (hi - lo + 1) // 2
        if before[mid] <= i:
            lo = mid
        else:
            hi = mid - 1
    return lo


def test_find_part_logic():
    rng = np.random.default_rng(3)
    for n in (1, 2, 3, 10, 257):
        sizes = rng.integers(1, 20, n)
        before = np.concatenate([[0], np.cumsum(sizes)[:-1]])
        for i in range(int(sizes.sum())):
            assert find_part_as_kernel(list(before), i) == np.searchsorted(before, i, side="right") - 1


def burning_list_as_kernel(t):
    """count_burning_kernel + scan_counts_kernel + write_burning_kernel."""
    n = t.size
    fmax = np.float32(np.finfo(np.float32).max)
    chunks = (n + CHUNK - 1) // CHUNK
    counts = [int(np.count_nonzero(t[ch * CHUNK:(ch + 1) * CHUNK] != fmax)) for ch in range(chunks)]
    per = (chunks + 1023) // 1024
    part = []
    for tid in range(1024):
        a = min(chunks, tid * per)
        b = min(chunks, a + per)
        part.append(sum(counts[a:b]))
    incl = np.cumsum(part)
    offsets = [0] * (chunks + 1)
    for tid in range(1024):
        a = min(chunks, tid * per)
        b = min(chunks, a + per)
        run = int(incl[tid] - part[tid])
        for k in range(a, b):
            offsets[k] = run
            run += counts[k]
    offsets[chunks] = int(incl[-1])
    out = [None] * offsets[chunks]
    for ch in range(chunks):
        at = offsets[ch]
        for j0 in range(0, CHUNK, THREADS):
            idx = ch * CHUNK + j0 + np.arange(THREADS)
            v = np.where(idx < n, t[np.minimum(idx, n - 1)], fmax)
            hit = v != fmax
            votes = [sum(int(hit[32 * k + l]) << l for l in range(32)) for k in range(WARPS)]
            counts_w = [_popc(x) for x in votes]
            for tid in np.flatnonzero(hit):
                lane, wid = tid & 31, tid >> 5
                ahead = _popc(votes[wid] & ((1 << lane) - 1)) + sum(counts_w[:wid])
                out[at + ahead] = int(idx[tid])
            at += sum(counts_w)
    return offsets[chunks], out


@pytest.mark.parametrize("n,density", [(1, 1.0), (4095, 0.3), (4097, 0.01), (3 * 4096 + 5, 0.5)])
def test_burning_list_logic(n, density):
    rng = np.random.default_rng(n)
    t = np.full(n, np.finfo(np.float32).max, np.float32)
    on = rng.random(n) < density
    t[on] = rng.uniform(0, 100, on.sum()).astype(np.float32)
    if n > 10:
        t[7] = np.nan  # NaN != FLT_MAX: listed
    total, order = burning_list_as_kernel(t)
    expect = np.flatnonzero(t != np.finfo(np.float32).max)
    assert total == expect.size and order == list(expect)


def test_device_rasterisers_need_a_device(L):
    """Without a GPU the device entry points report PROPAG_ERR_NO_DEVICE
    (the host rasterisers above keep working)."""
    import py_propag
    if py_propag.check_cuda_available():
        pytest.skip("a GPU is present")
    lib = L.lib()
    g = georef(L, 8, 8, GRIDS[0][2])
    assert lib.propag_rasterize_times_device(C.byref(g), None, 0, None, None) == L.PROPAG_ERR_NO_DEVICE
    assert lib.propag_rasterize_fuels_device(None, 0, b"", C.byref(g), None, None) == L.PROPAG_ERR_NO_DEVICE
    assert lib.propag_ignitions_from_times_device(None, 8, 8, None, 0, None) == L.PROPAG_ERR_NO_DEVICE
