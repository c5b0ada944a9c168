"""Propagation kernels vs the CPU restatement of the reference kernel.

Both sides run the reference's schedule (super-grid tiles of T cells, Jacobi
sweeps inside a tile, tiles in row-major order, passes until no tile
improves) on the same fire fields, with the same float arithmetic, so the
comparison is exact: arrival times, references and boundary bits bit for bit,
and the schedule counters (rounds, tile launches, sweeps, improvements)
equal.  Each test runs in the engine's two arithmetics: the reference's
(PROPAG_ARITH_REFERENCE, against the restatement with the device's
__cosf/atan2f tables, trig = 3) and the portable one (PROPAG_ARITH_PORTABLE,
against the restatement's own portable functions, trig = 0).
"""
import ctypes as C

import numpy as np
import pytest

from conftest import trig_for

pytestmark = pytest.mark.gpu

FMAX = np.finfo(np.float32).max
ARITHS = [pytest.param(0, id="ref-arith"), pytest.param(1, id="portable")]


@pytest.fixture
def oracle(ref_oracle):
    """The restatement with the device's trig tables installed; every run
    here must stay inside them."""
    before = ref_oracle.table_misses()
    yield ref_oracle
    assert ref_oracle.table_misses() == before, "a trig = 3 look-up fell outside the device tables"


SCHEDULE = ("rounds", "launches", "sweeps", "improvements")
WORK = ("evaluations", "dda_steps", "gathers")


def _check_counts(res, o, rerun, keys=SCHEDULE + WORK):
    """Schedule counters equal the oracle's; the work counters equal the
    oracle's in the mode the engine used: whole first sweeps (shared-memory
    tiles, oracle full=0) or first sweeps over the pending cells only
    (global-memory tiles, oracle full=2; `rerun(full)` runs the oracle)."""
    for k in keys:
        if k not in WORK:
            assert res.stats[k] == o.stats[k], (k, res.stats[k], o.stats[k])
    work = [k for k in keys if k in WORK]
    if all(res.stats[k] == o.stats[k] for k in work):
        return 0
    o2 = rerun(2)
    for k in work:
        assert res.stats[k] == o2.stats[k], (k, res.stats[k], o.stats[k], o2.stats[k])
    return 2


def _fire(pp, terrain):
    f = pp.fire_behaviour(terrain, full=False)
    return f["speed_max"], f["azimuth_max"], f["eccentricity"]


def _settings(pp, w, h, dx, dy, max_time):
    gt = [0.0, dx, 0.0, 0.0 if dy > 0 else h * -dy, 0.0, dy]
    g = pp.PyGeoReference(w, h, "+proj=utm +zone=30 +ellps=GRS80 +units=m +no_defs", gt)
    return pp.PySettings(g, max_time)


def _check(pp, oracle, terrain, w, h, dx, dy, max_time, ignitions, tile, arith=0):
    s = _settings(pp, w, h, dx, dy, max_time)
    res = pp.propagate_arrays(s, terrain, ignitions, tile=tile, arith=arith)
    sp, az, ec = _fire(pp, terrain)
    def run(full=0):
        return oracle.propagate(w, h, dx, dy, max_time, sp, az, ec, ignitions,
                                tile=(0 if tile == -1 else tile), full=full, trig=trig_for(arith))
    o = run()
    assert np.array_equal(res.boundary_change, o.boundaries), "boundary bits"
    t_gpu = res.arrival_times.view(np.uint32)
    t_ref = o.time.view(np.uint32)
    diff = t_gpu != t_ref
    if diff.any():
        i = np.argwhere(diff)[0]
        pytest.fail(f"{diff.sum()} times differ, first at {tuple(i)}: gpu={res.arrival_times[tuple(i)]} "
                    f"ref={o.time[tuple(i)]}")
    assert np.array_equal(res.refs_x.reshape(h, w), o.refs_x)
    assert np.array_equal(res.refs_y.reshape(h, w), o.refs_y)
    _check_counts(res, o, run)
    assert res.stats["burned"] == int(np.sum(o.time < FMAX))
    return res, o


@pytest.mark.parametrize("arith", ARITHS)
def test_uniform_demo(pp, oracle, arith):
    w = h = 96
    t = pp.demo_terrain(w, h)
    _check(pp, oracle, t, w, h, 5.0, 5.0, 3000.0, [(40, 40, 0.0)], tile=-1, arith=arith)


@pytest.mark.parametrize("arith", ARITHS)
@pytest.mark.parametrize("tile", [-1, 57, 19])
def test_hills_voronoi(pp, oracle, tile, arith):
    from py_propag import scenarios as S
    sc = S.config0(size=128)
    _check(pp, oracle, sc.terrain, sc.width, sc.height, sc.dx, sc.dy, sc.max_time,
           sc.ignitions, tile, arith)


@pytest.mark.parametrize("arith", ARITHS)
@pytest.mark.parametrize("tile", [-1, 64, 323])
def test_ridges_lakes_roads_many_ignitions(pp, oracle, tile, arith):
    from py_propag import scenarios as S
    sc = S.config1(size=160, n_ign=6, max_time=7200.0)
    res, o = _check(pp, oracle, sc.terrain, sc.width, sc.height, sc.dx, sc.dy, sc.max_time,
                    sc.ignitions, tile, arith)
    assert res.stats["improvements"] > 0


@pytest.mark.parametrize("arith", ARITHS)
@pytest.mark.parametrize("cluster", [1, 2, 16, -1])
def test_shared_memory_and_global_tiles(pp, oracle, cluster, arith):
    """The same scenario with the tile resident in the cluster's shared
    memory (when it fits) and in global memory (cluster 1 cannot hold a
    130 x 130 halo'd tile; group mode, -1, always uses global memory): all
    bit-exact against the restatement."""
    from py_propag import scenarios as S
    sc = S.config1(size=128, seed=5, n_ign=4, max_time=10000.0)
    s = _settings(pp, sc.width, sc.height, sc.dx, sc.dy, sc.max_time)
    res = pp.propagate_arrays(s, sc.terrain, sc.ignitions, tile=-1, cluster=cluster, arith=arith)
    sp, az, ec = _fire(pp, sc.terrain)
    def run(full=0):
        return oracle.propagate(sc.width, sc.height, sc.dx, sc.dy, sc.max_time, sp, az, ec,
                                sc.ignitions, tile=0, full=full, trig=trig_for(arith))
    o = run()
    assert np.array_equal(res.arrival_times.view(np.uint32), o.time.view(np.uint32))
    assert np.array_equal(res.refs_x.reshape(sc.height, sc.width), o.refs_x)
    _check_counts(res, o, run, ("sweeps", "improvements") + WORK)


@pytest.mark.parametrize("arith", ARITHS)
@pytest.mark.parametrize("tile,cluster", [(300, 16), (300, 8), (323, 0), (300, -1), (64, -1)])
def test_wide_tiles_several_launches(pp, oracle, tile, cluster, arith):
    """Tiles wider than 254 cells keep their staged referrer boxes at
    two-cell granularity; over several tile launches and rounds the scans
    must still find every referrer (exact evaluation counts)."""
    from py_propag import scenarios as S
    sc = S.config1(size=640, seed=17, n_ign=8, max_time=14400.0)
    s = _settings(pp, sc.width, sc.height, sc.dx, sc.dy, sc.max_time)
    res = pp.propagate_arrays(s, sc.terrain, sc.ignitions, tile=tile, cluster=cluster, arith=arith)
    sp, az, ec = _fire(pp, sc.terrain)
    def run(full=0):
        return oracle.propagate(sc.width, sc.height, sc.dx, sc.dy, sc.max_time, sp, az, ec,
                                sc.ignitions, tile=tile, full=full, trig=trig_for(arith))
    o = run()
    assert res.stats["launches"] > 4
    assert np.array_equal(res.arrival_times.view(np.uint32), o.time.view(np.uint32))
    assert np.array_equal(res.refs_x.reshape(sc.height, sc.width), o.refs_x)
    mode = _check_counts(res, o, run)
    # shared-memory clusters evaluate whole first sweeps, global-memory tiles
    # (group mode) only the pending cells
    assert mode == (0 if cluster > 0 else 2)


@pytest.mark.parametrize("cluster", [1, 2])
def test_shared_memory_list_overflow(pp, oracle, cluster):
    """Hundreds of ignitions in one shared-memory tile: the first sweeps
    produce more work-list and update-list entries than a CTA holds in
    shared memory (4096 / 2048), so entries spill to the global overflow."""
    from py_propag import scenarios as S
    sc = S.config1(size=110, seed=9, n_ign=900, max_time=3000.0)
    s = _settings(pp, sc.width, sc.height, sc.dx, sc.dy, sc.max_time)
    res = pp.propagate_arrays(s, sc.terrain, sc.ignitions, tile=-1, cluster=cluster)
    sp, az, ec = _fire(pp, sc.terrain)
    def run(full=0):
        return oracle.propagate(sc.width, sc.height, sc.dx, sc.dy, sc.max_time, sp, az, ec,
                                sc.ignitions, tile=0, full=full, trig=3)
    o = run()
    assert res.stats["improvements"] > 2048 * cluster
    assert np.array_equal(res.arrival_times.view(np.uint32), o.time.view(np.uint32))
    assert np.array_equal(res.refs_x.reshape(sc.height, sc.width), o.refs_x)
    assert np.array_equal(res.refs_y.reshape(sc.height, sc.width), o.refs_y)
    _check_counts(res, o, run, ("sweeps", "improvements") + WORK)


@pytest.mark.parametrize("arith", ARITHS)
def test_north_up_and_staggered_ignition_times(pp, oracle, arith):
    from py_propag import scenarios as S
    sc = S.config0(size=96, seed=4)
    ign = [(10, 10, 0.0), (80, 70, 600.0), (50, 20, 1200.0), (10, 10, 30.0)]  # repeated cell
    _check(pp, oracle, sc.terrain, 96, 96, 5.0, -5.0, 20000.0, ign, tile=-1, arith=arith)


@pytest.mark.parametrize("arith", ARITHS)
def test_rectangular_and_degenerate_grids(pp, oracle, arith):
    for (w, h) in [(1, 1), (1, 37), (53, 1), (33, 70)]:
        t = pp.demo_terrain(w, h)
        _check(pp, oracle, t, w, h, 5.0, 5.0, 5000.0, [(0, 0, 0.0)], tile=-1, arith=arith)


def test_no_ignition_and_non_burnable_ignition(pp, oracle):
    w = h = 40
    t = pp.demo_terrain(w, h)
    res, _ = _check(pp, oracle, t, w, h, 5.0, 5.0, 5000.0, [], tile=-1)
    assert res.stats["burned"] == 0
    t["fuel_code"][20, 20] = 0
    res, _ = _check(pp, oracle, t, w, h, 5.0, 5.0, 5000.0, [(20, 20, 0.0)], tile=-1)
    assert res.stats["burned"] == 0  # a non-burnable ignition never spreads


def _job(L, w, h, dx, dy, max_time, dev, tile=0, arith=0):
    j = L.PropagJob()
    j.width, j.height, j.dx, j.dy, j.max_time, j.tile = w, h, dx, dy, max_time, tile
    j.arith = arith
    j.speed_max, j.azimuth_max, j.eccentricity = (dev[k].data_ptr() for k in ("sp", "az", "ec"))
    j.ignitions, j.n_ignitions = dev["ign"].data_ptr(), dev["n_ign"]
    j.time, j.refs_x, j.refs_y, j.boundaries = (dev[k].data_ptr() for k in ("time", "rx", "ry", "bnd"))
    return j


def _device_scenario(pp, sc):
    import torch
    sp, az, ec = _fire(pp, sc.terrain)
    n = sc.width * sc.height
    ign = np.array([(x, y, t) for (x, y, t) in sc.ignitions],
                   dtype=[("x", "<u4"), ("y", "<u4"), ("t", "<f4")])
    dev = dict(sp=torch.from_numpy(sp.ravel().copy()).cuda(), az=torch.from_numpy(az.ravel().copy()).cuda(),
               ec=torch.from_numpy(ec.ravel().copy()).cuda(),
               ign=torch.from_numpy(np.frombuffer(ign.tobytes() or bytes(12), np.uint8).copy()).cuda(),
               n_ign=len(sc.ignitions),
               time=torch.empty(n, dtype=torch.float32, device="cuda"),
               rx=torch.empty(n, dtype=torch.int16, device="cuda"),
               ry=torch.empty(n, dtype=torch.int16, device="cuda"),
               bnd=torch.empty((n + 31) // 32, dtype=torch.int32, device="cuda"))
    return dev


@pytest.mark.parametrize("cluster", [1, 4, 16, -1, -2])
def test_batch_equals_single_runs(pp, oracle, cluster):
    """Uneven scenarios in one persistent launch give each scenario's own
    result, whatever the cluster size (-1: group mode, four teams; -2: teams
    of 2+ CTAs)."""
    import torch
    from py_propag import _lib as L
    from py_propag import scenarios as S
    scs = [S.config0(size=64, seed=11), S.config1(size=96, seed=12, n_ign=3, max_time=3600.0),
           S.config0(size=80, seed=13), S.config1(size=48, seed=14, n_ign=2, max_time=1800.0)]
    devs = [_device_scenario(pp, sc) for sc in scs]
    # the jobs alternate between the two arithmetics (a per-job choice)
    jobs = [_job(L, sc.width, sc.height, sc.dx, sc.dy, sc.max_time, d,
                 tile=(-1 if i % 2 == 0 else 37), arith=(i // 2) % 2)
            for i, (sc, d) in enumerate(zip(scs, devs))]
    eng = pp.Engine(cluster=cluster)
    stats = eng.run(jobs)
    torch.cuda.synchronize()
    for i, (sc, d, st) in enumerate(zip(scs, devs, stats)):
        sp, az, ec = (d[k].cpu().numpy() for k in ("sp", "az", "ec"))
        o = oracle.propagate(sc.width, sc.height, sc.dx, sc.dy, sc.max_time, sp, az, ec,
                             sc.ignitions, tile=(0 if i % 2 == 0 else 37), trig=trig_for((i // 2) % 2))
        assert np.array_equal(d["time"].cpu().numpy().view(np.uint32), o.time.ravel().view(np.uint32)), i
        assert np.array_equal(d["rx"].cpu().numpy().view(np.uint16), o.refs_x.ravel()), i
        assert st["sweeps"] == o.stats["sweeps"] and st["improvements"] == o.stats["improvements"], i
    eng.close()


def test_repeated_calls_are_deterministic(pp):
    from py_propag import scenarios as S
    sc = S.config0(size=100, seed=21)
    s = _settings(pp, sc.width, sc.height, sc.dx, sc.dy, sc.max_time)
    a = pp.propagate_arrays(s, sc.terrain, sc.ignitions, tile=-1)
    b = pp.propagate_arrays(s, sc.terrain, sc.ignitions, tile=-1)
    assert np.array_equal(a.arrival_times.view(np.uint32), b.arrival_times.view(np.uint32))
    # schedule counters are deterministic; cycle counts and the number of
    # referrer scans (which may or may not see a reference adopted in the
    # same sweep) are not
    keys = ("rounds", "launches", "sweeps", "evaluations", "improvements", "dda_steps", "gathers",
            "burned")
    assert {k: a.stats[k] for k in keys} == {k: b.stats[k] for k in keys}


def test_group_wait_gives_up_and_device_stays_usable(pp, oracle):
    """Group mode's team barrier is a bounded wait: a team that counts one
    CTA more than its launch holds gives up after the limit, the call fails
    with PROPAG_ERR_TIMEOUT and the job reports status 2; afterwards the
    device runs group mode normally (bit-exact)."""
    import time
    from py_propag import _lib as L
    from py_propag import scenarios as S
    st = C.c_uint32(0)
    t0 = time.perf_counter()
    rc = L.lib().propag_selftest_group_wait(C.byref(st))
    dt = time.perf_counter() - t0
    assert rc == L.PROPAG_ERR_TIMEOUT, L.last_error()
    assert st.value == 2
    assert "group barrier" in L.last_error()
    assert 1.5 < dt < 30.0
    sc = S.config0(size=96, seed=3)
    s = _settings(pp, sc.width, sc.height, sc.dx, sc.dy, sc.max_time)
    res = pp.propagate_arrays(s, sc.terrain, sc.ignitions, tile=0, cluster=-1)
    sp, az, ec = _fire(pp, sc.terrain)
    o = oracle.propagate(sc.width, sc.height, sc.dx, sc.dy, sc.max_time, sp, az, ec,
                         sc.ignitions, tile=0, trig=3)
    assert np.array_equal(res.arrival_times.view(np.uint32), o.time.view(np.uint32))
