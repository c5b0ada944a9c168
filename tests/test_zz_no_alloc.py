"""propag_run_device_static (the allocation-free propagation entry point)
against propag_engine_run on the same device-resident scenarios.

The file name sorts last so that the fixed scratch is exercised after every
other GPU test has used the library; it passes alone as well.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DET_KEYS = ("rounds", "launches", "sweeps", "evaluations", "improvements", "dda_steps", "gathers",
            "burned", "status")


def _device_job(pp, L, sc, tile):
    import torch
    f = pp.fire_behaviour(sc.terrain, full=False)
    n = sc.width * sc.height
    ign = np.array([(x, y, t) for (x, y, t) in sc.ignitions],
                   dtype=[("x", "<u4"), ("y", "<u4"), ("t", "<f4")])
    keep = dict(
        sp=torch.from_numpy(f["speed_max"].ravel().copy()).cuda(),
        az=torch.from_numpy(f["azimuth_max"].ravel().copy()).cuda(),
        ec=torch.from_numpy(f["eccentricity"].ravel().copy()).cuda(),
        ign=torch.from_numpy(np.frombuffer(ign.tobytes() or bytes(12), np.uint8).copy()).cuda(),
        time=torch.empty(n, dtype=torch.float32, device="cuda"),
        rx=torch.empty(n, dtype=torch.int16, device="cuda"),
        ry=torch.empty(n, dtype=torch.int16, device="cuda"),
        bnd=torch.empty((n + 31) // 32, dtype=torch.int32, device="cuda"))
    j = L.PropagJob()
    j.width, j.height, j.dx, j.dy, j.max_time, j.tile = sc.width, sc.height, sc.dx, sc.dy, sc.max_time, tile
    j.speed_max, j.azimuth_max, j.eccentricity = (keep[k].data_ptr() for k in ("sp", "az", "ec"))
    j.ignitions, j.n_ignitions = keep["ign"].data_ptr(), len(sc.ignitions)
    j.time, j.refs_x, j.refs_y, j.boundaries = (keep[k].data_ptr() for k in ("time", "rx", "ry", "bnd"))
    return j, keep


def _outputs(keep):
    return {k: keep[k].cpu().numpy().copy() for k in ("time", "rx", "ry", "bnd")}


def _static(L, job, with_stats=True):
    st = L.PropagStats()
    rc = L.lib().propag_run_device_static(C.byref(job), None, C.byref(st) if with_stats else None)
    assert rc == 0, L.last_error()
    return st.as_dict()


def _same(a, b):
    for k in ("time", "rx", "ry", "bnd"):
        assert np.array_equal(a[k].view(np.uint8), b[k].view(np.uint8)), k


def test_static_equals_engine_on_consecutive_calls(pp):
    import torch
    from py_propag import _lib as L
    from py_propag import scenarios as S
    a_sc = S.config1(size=256, seed=31, n_ign=4, max_time=7200.0)
    b_sc = S.config0(size=200, seed=32)
    a, ka = _device_job(pp, L, a_sc, 0)
    b, kb = _device_job(pp, L, b_sc, 57)

    # two calls in a row through the fixed scratch, different grids
    st_a = _static(L, a)
    out_a = _outputs(ka)
    st_b = _static(L, b)
    out_b = _outputs(kb)

    # the existing entry point on the same jobs, on a 16-CTA cluster as the
    # fixed-scratch path runs (the same results in every mode; the work
    # counters are those of cluster mode)
    eng = pp.Engine(cluster=16)
    ref_a = eng.run([a])[0]
    ea = _outputs(ka)
    ref_b = eng.run([b])[0]
    eb = _outputs(kb)
    eng.close()

    _same(out_a, ea)
    _same(out_b, eb)
    assert {k: st_a[k] for k in DET_KEYS} == {k: ref_a[k] for k in DET_KEYS}
    assert {k: st_b[k] for k in DET_KEYS} == {k: ref_b[k] for k in DET_KEYS}
    assert st_a["burned"] > 0 and st_b["burned"] > 0

    # again after the other grid used the scratch, without statistics (async)
    ka["time"].fill_(-1.0)
    _static(L, a, with_stats=False)
    torch.cuda.synchronize()
    _same(_outputs(ka), ea)


def test_static_allocates_no_device_memory(pp):
    """Net device usage is unchanged by calls after the first (which takes
    the scratch's address): free device memory before and after two calls is
    the same.  This sees allocations still held at the end; the entry point's
    source makes no cudaMalloc/cudaFree/cudaMallocHost call at all."""
    import torch
    from py_propag import _lib as L
    from py_propag import scenarios as S
    sc = S.config1(size=192, seed=33, n_ign=3, max_time=5400.0)
    job, keep = _device_job(pp, L, sc, 0)
    first = _static(L, job)  # set-up happens in the first call on a device
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(2):
        st = _static(L, job)
        assert {k: st[k] for k in DET_KEYS} == {k: first[k] for k in DET_KEYS}
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0


def test_static_rejects_jobs_beyond_its_limits(pp):
    import torch
    from py_propag import _lib as L
    lib = L.lib()
    assert L.PROPAG_STATIC_MAX_CELLS == 1 << 20
    j = L.PropagJob()
    j.width, j.height, j.dx, j.dy, j.max_time = 1025, 1024, 5.0, 5.0, 100.0
    assert lib.propag_run_device_static(C.byref(j), None, None) == L.PROPAG_ERR_INVALID
    assert "exceeds its fixed scratch of 1048576 cells" in L.last_error()
    # a whole-grid tile of 600 x 600 cells does not fit a 16-CTA cluster
    buf = torch.zeros(600 * 600, dtype=torch.float32, device="cuda")
    j.width, j.height, j.tile = 600, 600, -1
    j.speed_max = j.azimuth_max = j.eccentricity = j.time = buf.data_ptr()
    assert lib.propag_run_device_static(C.byref(j), None, None) == L.PROPAG_ERR_INVALID
    assert "does not fit" in L.last_error()
    assert lib.propag_run_device_static(None, None, None) == L.PROPAG_ERR_INVALID


def test_static_status_without_stats(pp, monkeypatch):
    """A caller that runs without `stats` (stream-ordered) reads the job's
    outcome afterwards: a job stopped by the sweep limit (PROPAG_MAX_SWEEPS,
    read at each call) reports it, and the next call clears it."""
    from py_propag import _lib as L
    from py_propag import scenarios as S
    lib = L.lib()
    sc = S.config0(size=96, seed=34)
    job, keep = _device_job(pp, L, sc, 0)
    monkeypatch.setenv("PROPAG_MAX_SWEEPS", "3")
    assert lib.propag_run_device_static(C.byref(job), None, None) == 0, L.last_error()
    st = L.PropagStats()
    assert lib.propag_static_last_status(None, C.byref(st)) == L.PROPAG_ERR_TIMEOUT
    assert st.status == 1 and "sweep limit" in L.last_error()
    assert lib.propag_run_device_static(C.byref(job), None, C.byref(L.PropagStats())) == \
        L.PROPAG_ERR_TIMEOUT
    monkeypatch.delenv("PROPAG_MAX_SWEEPS")
    assert lib.propag_run_device_static(C.byref(job), None, None) == 0, L.last_error()
    assert lib.propag_static_last_status(None, C.byref(st)) == 0, L.last_error()
    assert st.status == 0 and st.burned > 0
