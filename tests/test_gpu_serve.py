"""The serving loop (continuous batching): requests submitted while others
run are admitted onto free streams, and every request's result equals the
same scenario propagated alone, bit for bit, whatever batch it lands in."""
import time

import numpy as np
import pytest

from test_gpu_batch import _alone, _device_batch, _uneven

pytestmark = pytest.mark.gpu


def test_results_equal_alone_in_any_mix(pp):
    from py_propag import _lib as L
    scs = _uneven(n=8, seed=51)
    jobs, terrains, keep = _device_batch(pp, L, scs, [0] * len(scs))
    srv = pp.Server(lanes=1, max_batch=8)
    ids = []
    for i, (j, t) in enumerate(zip(jobs, terrains)):
        ids.append(srv.submit(j, t))
        if i == 3:
            time.sleep(0.002)
    res = [srv.wait(r) for r in ids]
    srv.close()
    # with one lane, requests that arrive while a batch runs wait for it and
    # go out together
    assert max(r["batch_size"] for r in res) > 1
    assert sum(1 for r in res) == len(scs)
    for i, (sc, b, r) in enumerate(zip(scs, keep, res)):
        a = _alone(pp, sc, 0)
        assert np.array_equal(b["time"].cpu().numpy().view(np.uint32),
                              a.arrival_times.ravel().view(np.uint32)), i
        assert r["burned"] == a.stats["burned"] and r["sweeps"] == a.stats["sweeps"], i
        assert r["submit_ns"] <= r["start_ns"] <= r["done_ns"]


def test_concurrent_lanes_and_resubmission(pp):
    """Several lanes in flight; the same buffers submitted again after their
    first request finished give the same results."""
    from py_propag import _lib as L
    scs = _uneven(n=6, seed=52)
    jobs, terrains, keep = _device_batch(pp, L, scs, [0] * len(scs))
    srv = pp.Server(lanes=3, max_batch=2)
    first = [srv.wait(srv.submit(j, t)) for j, t in zip(jobs, terrains)]
    outs = [b["time"].cpu().numpy().copy() for b in keep]
    for b in keep:
        b["time"].fill_(-1.0)
    ids = [srv.submit(j, t) for j, t in zip(jobs, terrains)]
    second = [srv.wait(r) for r in ids]
    for r in ids:
        srv.release(r)
    srv.close()
    for i, b in enumerate(keep):
        assert np.array_equal(b["time"].cpu().numpy().view(np.uint32), outs[i].view(np.uint32)), i
        assert first[i]["evaluations"] == second[i]["evaluations"], i


def test_budget_and_bad_requests(pp):
    from py_propag import _lib as L
    scs = _uneven(n=2, seed=53)
    jobs, terrains, keep = _device_batch(pp, L, scs, [0, 0])
    # each of the two lanes reserves half the budget: room for the smaller
    # request's engine scratch, not the larger one's
    small = min(L.lib().propag_engine_job_bytes(sc.width, sc.height) for sc in scs)
    srv = pp.Server(hbm_budget=2 * small, lanes=2)
    big = int(np.argmax([sc.width * sc.height for sc in scs]))
    rid = srv.submit(jobs[big], terrains[big])
    with pytest.raises(pp.PropagCudaError, match="budget"):
        srv.wait(rid)
    ok = 1 - big
    r = srv.wait(srv.submit(jobs[ok], terrains[ok]))
    assert r["burned"] == _alone(pp, scs[ok], 0).stats["burned"]
    bad = L.PropagJob()
    with pytest.raises(pp.PropagValidationError):
        srv.submit(bad)
    srv.close()
