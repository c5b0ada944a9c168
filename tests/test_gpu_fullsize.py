"""Propagation parity at the benchmark workloads' full sizes.

The engine against the CPU restatement of the reference kernel, on:
  * the 1024 x 1024 single scenario (config 0: hills, Voronoi fuel patches,
    one ignition at (500, 500), 36 000 s; the reference demo's shape,
    crates/propag/src/main.rs:12-55) in both arithmetics;
  * the 4096 x 4096 heterogeneous scenario (config 1: ridges, lakes and
    roads, variable wind and moisture, 20 ignitions, 43 200 s);
  * members of the 256-member ensemble (config 2) taken from one batched
    CUDA-graph run.
Times, references and boundary bits bit for bit, schedule counters equal;
the engine in the reference's arithmetic against the restatement fed with
the device's __cosf/atan2f tables (trig = 3).
"""
import numpy as np
import pytest

from conftest import trig_for

pytestmark = pytest.mark.gpu

TILE = 323  # the engine's default super-grid tile on a 148-SM B200


@pytest.fixture
def oracle(ref_oracle):
    before = ref_oracle.table_misses()
    yield ref_oracle
    assert ref_oracle.table_misses() == before, "a trig = 3 look-up fell outside the device tables"


def _settings(pp, sc):
    g = pp.PyGeoReference(sc.width, sc.height, "+proj=utm +zone=30 +ellps=GRS80 +units=m +no_defs",
                          [0.0, sc.dx, 0.0, 0.0, 0.0, sc.dy])
    return pp.PySettings(g, sc.max_time)


def _compare(res, o, w, h):
    t_gpu = res.arrival_times.view(np.uint32)
    t_ref = o.time.view(np.uint32)
    diff = t_gpu != t_ref
    assert not diff.any(), f"{diff.sum()} of {diff.size} arrival times differ"
    assert np.array_equal(res.refs_x.reshape(h, w), o.refs_x)
    assert np.array_equal(res.refs_y.reshape(h, w), o.refs_y)
    assert np.array_equal(res.boundary_change, o.boundaries)
    for k in ("rounds", "launches", "sweeps", "improvements", "evaluations", "dda_steps", "gathers"):
        assert res.stats[k] == o.stats[k], (k, res.stats[k], o.stats[k])
    assert res.stats["burned"] == int(np.sum(o.time < np.finfo(np.float32).max))


def _run(pp, oracle, sc, arith):
    res = pp.propagate_arrays(_settings(pp, sc), sc.terrain, sc.ignitions, tile=TILE, arith=arith)
    f = pp.fire_behaviour(sc.terrain, full=False)
    # the engine's default (group) mode evaluates first sweeps over the
    # pending cells only: the restatement's full = 2
    o = oracle.propagate(sc.width, sc.height, sc.dx, sc.dy, sc.max_time, f["speed_max"],
                         f["azimuth_max"], f["eccentricity"], sc.ignitions, tile=TILE, full=2,
                         trig=trig_for(arith))
    _compare(res, o, sc.width, sc.height)
    return res


@pytest.mark.parametrize("arith", [pytest.param(0, id="ref-arith"), pytest.param(1, id="portable")])
def test_config0_1024(pp, oracle, arith):
    from py_propag import scenarios as S
    res = _run(pp, oracle, S.config0(size=1024), arith)
    assert res.stats["burned"] > 100_000


def test_config1_4096(pp, oracle):
    from py_propag import scenarios as S
    res = _run(pp, oracle, S.config1(size=4096), 0)
    assert res.stats["burned"] > 1_000_000


def test_config2_ensemble_members_from_a_batched_graph(pp, oracle):
    """All 256 members in one graph-captured persistent launch; eight of
    them, drawn at random, equal the restatement."""
    import torch
    from py_propag import _lib as L
    from py_propag.batches import ensemble_batch
    (jobs, terrains, keep), _ = ensemble_batch(L, "cuda", 256)
    g = pp.Graph(jobs, terrains)
    g.launch()
    torch.cuda.synchronize()
    stats = g.stats()
    rng = np.random.default_rng(20)
    for i in sorted(rng.choice(len(jobs), 8, replace=False)):
        j = jobs[i]
        t, fire, ign_d, out, rx, ry, bnd = keep[i]
        sp, az, ec = (f.cpu().numpy() for f in fire)
        ign = np.frombuffer(ign_d.cpu().numpy().tobytes(), dtype=[("x", "<u4"), ("y", "<u4"), ("t", "<f4")])
        ign = [(int(a["x"]), int(a["y"]), float(a["t"])) for a in ign[: j.n_ignitions]]
        o = oracle.propagate(j.width, j.height, j.dx, j.dy, j.max_time, sp, az, ec, ign, tile=TILE,
                             full=2, trig=3)
        got = out.cpu().numpy()
        assert np.array_equal(got.view(np.uint32), o.time.ravel().view(np.uint32)), i
        assert np.array_equal(rx.cpu().numpy().view(np.uint16), o.refs_x.ravel()), i
        assert np.array_equal(ry.cpu().numpy().view(np.uint16), o.refs_y.ravel()), i
        assert np.array_equal(bnd.cpu().numpy().view(np.uint32), o.boundaries), i
        for k in ("rounds", "launches", "sweeps", "improvements"):
            assert stats[i][k] == o.stats[k], (i, k, stats[i][k], o.stats[k])
    g.close()
