"""Uneven batches in one persistent launch, captured as a CUDA graph, and
the autotuner: every scenario's result equals the same scenario propagated
alone (bit for bit), whatever the capture, the replay count or the cluster
size the tuner picks."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _device_batch(pp, L, scs, tiles):
    """Device terrains, fire rasters (outputs of the graph's fire pass) and
    outputs for a list of scenarios; returns jobs, terrains, buffers."""
    import torch
    jobs, terrains, keep = [], [], []
    for sc, tile in zip(scs, tiles):
        n = sc.width * sc.height
        t = {k: torch.from_numpy(np.ascontiguousarray(v).ravel()).cuda() for k, v in sc.terrain.items()}
        ign = np.array([(x, y, tt) for (x, y, tt) in sc.ignitions],
                       dtype=[("x", "<u4"), ("y", "<u4"), ("t", "<f4")])
        b = dict(terrain=t,
                 fire=[torch.full((n,), -1.0, dtype=torch.float32, device="cuda") for _ in range(3)],
                 ign=torch.from_numpy(np.frombuffer(ign.tobytes() or bytes(12), np.uint8).copy()).cuda(),
                 time=torch.empty(n, dtype=torch.float32, device="cuda"),
                 rx=torch.empty(n, dtype=torch.int16, device="cuda"),
                 ry=torch.empty(n, dtype=torch.int16, device="cuda"),
                 bnd=torch.empty((n + 31) // 32, dtype=torch.int32, device="cuda"))
        j = L.PropagJob()
        j.width, j.height, j.dx, j.dy, j.max_time, j.tile = sc.width, sc.height, sc.dx, sc.dy, sc.max_time, tile
        j.speed_max, j.azimuth_max, j.eccentricity = (f.data_ptr() for f in b["fire"])
        j.ignitions, j.n_ignitions = b["ign"].data_ptr(), len(sc.ignitions)
        j.time, j.refs_x, j.refs_y, j.boundaries = (b[k].data_ptr() for k in ("time", "rx", "ry", "bnd"))
        jobs.append(j)
        terrains.append(L.PropagTerrainPtrs(*[t[k].data_ptr() for k in L.TERRAIN_FIELDS]))
        keep.append(b)
    return jobs, terrains, keep


def _alone(pp, sc, tile):
    gt = [0.0, sc.dx, 0.0, 0.0, 0.0, sc.dy]
    s = pp.PySettings(pp.PyGeoReference(sc.width, sc.height, "+proj=utm", gt), sc.max_time)
    return pp.propagate_arrays(s, sc.terrain, sc.ignitions, tile=tile)


def _uneven(n=6, seed=41):
    from py_propag import scenarios as S
    return S.config3(n=n, seed=seed, min_size=48, max_size=360)


@pytest.mark.parametrize("cluster", [0, 16, -1, -4])
def test_graph_replays_equal_single_runs(pp, cluster):
    """Six uneven scenarios captured once and replayed twice, with the
    automatic choice (group mode), 16-CTA clusters, group mode with the
    automatic team size and with teams of 4 CTAs (a cooperative launch inside
    the graph)."""
    import torch
    from py_propag import _lib as L
    scs = _uneven()
    tiles = [0 if i % 3 else 57 for i in range(len(scs))]
    jobs, terrains, keep = _device_batch(pp, L, scs, tiles)
    g = pp.Graph(jobs, terrains, cluster=cluster)
    alone = [_alone(pp, sc, t) for sc, t in zip(scs, tiles)]
    for rep in range(2):
        for b in keep:
            b["time"].fill_(-1.0)
        g.launch()
        torch.cuda.synchronize()
        st = g.stats()
        for i, (b, a) in enumerate(zip(keep, alone)):
            assert np.array_equal(b["time"].cpu().numpy().view(np.uint32),
                                  a.arrival_times.ravel().view(np.uint32)), (rep, i)
            assert np.array_equal(b["rx"].cpu().numpy().view(np.uint16), a.refs_x), (rep, i)
            # (evaluations are not compared: group-mode runs evaluate only
            # the pending cells in first sweeps, shared-memory clusters all)
            for k in ("sweeps", "improvements", "burned"):
                assert st[i][k] == a.stats[k], (rep, i, k)
    g.close()


def test_graph_reads_current_buffer_contents(pp):
    """A replay reads the buffers as they are at launch: a new ignition time
    written into the same device buffer is propagated."""
    import torch
    from py_propag import _lib as L
    from py_propag import scenarios as S
    sc = S.config0(size=96, seed=5)
    jobs, terrains, keep = _device_batch(pp, L, [sc], [0])
    g = pp.Graph(jobs, terrains)
    g.launch()
    torch.cuda.synchronize()
    x, y, _ = sc.ignitions[0]
    late = np.array([(x, y, 900.0)], dtype=[("x", "<u4"), ("y", "<u4"), ("t", "<f4")])
    keep[0]["ign"].copy_(torch.from_numpy(np.frombuffer(late.tobytes(), np.uint8).copy()))
    g.launch()
    torch.cuda.synchronize()
    sc.ignitions = [(x, y, 900.0)]
    a = _alone(pp, sc, 0)
    assert np.array_equal(keep[0]["time"].cpu().numpy().view(np.uint32), a.arrival_times.ravel().view(np.uint32))
    g.close()


def test_autotune_picks_a_fitting_cluster_and_results_do_not_change(pp):
    import torch
    from py_propag import _lib as L
    scs = _uneven(n=5, seed=43)
    tiles = [0] * len(scs)
    jobs, terrains, keep = _device_batch(pp, L, scs, tiles)
    opts, ms = pp.autotune(jobs, terrains, repeats=1)
    # cluster sizes whose shared memory holds the tiles, the automatic choice
    # (0: group mode) and group-mode teams of 24, 16, 8 or 4 CTAs
    assert opts["cluster"] in (1, 2, 4, 8, 16, 0, -24, -16, -8, -4) and ms > 0
    g = pp.Graph(jobs, terrains, cluster=opts["cluster"])
    g.launch()
    torch.cuda.synchronize()
    for b, sc in zip(keep, scs):
        a = _alone(pp, sc, 0)
        assert np.array_equal(b["time"].cpu().numpy().view(np.uint32), a.arrival_times.ravel().view(np.uint32))
    g.close()


def test_graph_rejects_bad_jobs(pp):
    from py_propag import _lib as L
    j = L.PropagJob()
    j.width, j.height, j.dx, j.dy, j.max_time = 0, 10, 5.0, 5.0, 100.0
    with pytest.raises((pp.PropagValidationError, pp.PropagCudaError), match="width/height"):
        pp.Graph([j])
