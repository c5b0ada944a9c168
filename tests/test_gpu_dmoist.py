"""The per-cell dmoist kernel against the CPU restatement (itself pinned to
the reference's fixtures in test_dmoist.py): equal bit for bit, every
output hour, over random weather, terrain and fuel."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _inputs(n, seed):
    rng = np.random.default_rng(seed)
    return dict(
        temperature=rng.uniform(-10, 48, (24, n)).astype(np.float32),
        humidity=rng.uniform(0, 100, (24, n)).astype(np.float32),
        cloud_cover=rng.uniform(0, 100, (24, n)).astype(np.float32),
        precipitation=(rng.uniform(0, 50, (6, n)) * (rng.random((6, n)) < 0.4)).astype(np.float32),
        slope=rng.uniform(0, 1.6, n).astype(np.float32),
        aspect=rng.uniform(0, 2 * np.pi, n).astype(np.float32),
        fuel_code=rng.integers(0, 14, n).astype(np.uint8))


@pytest.mark.parametrize("month", [1, 4, 7, 10])
def test_dmoist_kernel_equals_restatement(pp, oracle, month):
    n = 20_011
    x = _inputs(n, month)
    for hour in (0, 6, 9, 15, 23):
        g = pp.dead_fuel_moisture(hour=hour, month=month, **x)
        c = oracle.dmoist_cells(hour, month, x["temperature"], x["humidity"], x["cloud_cover"],
                                x["slope"], x["aspect"], x["fuel_code"], x["precipitation"])
        for k, ref in zip(("d1hr", "d10hr", "d100hr"), c):
            assert np.array_equal(g[k].view(np.uint32), ref.view(np.uint32)), (month, hour, k)


def test_dmoist_scale_and_validation(pp):
    x = _inputs(1000, 9)
    a = pp.dead_fuel_moisture(hour=12, month=7, **x)
    b = pp.dead_fuel_moisture(hour=12, month=7, scale=0.01, **x)
    for k in a:
        assert np.array_equal(b[k], (a[k] * np.float32(0.01)).astype(np.float32))
    assert np.all(a["d1hr"][x["fuel_code"] == 0] == 0)
    with pytest.raises(pp.PropagValidationError):
        pp.dead_fuel_moisture(hour=24, month=7, **x)


@pytest.mark.parametrize("hour,month", [(14, 7), (3, 1)])
def test_fused_moisture_fire_equals_two_passes(pp, hour, month):
    """propag_fire_weather_device (moisture and fire behaviour in one pass)
    gives the bits of the moisture pass (scale 0.01) followed by the fire
    pass on the moistures it wrote."""
    import ctypes as C
    import torch
    from conftest import random_terrain
    from py_propag import _lib as L
    n = 50_003
    x = _inputs(n, 40 + month)
    t = random_terrain(n, 41 + month)
    t["fuel_code"], t["slope"], t["aspect"] = x["fuel_code"], x["slope"], x["aspect"]
    d = pp.dead_fuel_moisture(hour=hour, month=month, scale=0.01, **x)
    two = pp.fire_behaviour(dict(t, **d), full=False)
    dev = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in dict(t, **x).items()}
    w = L.PropagWeatherPtrs(*[dev[k].data_ptr() for k in ("temperature", "humidity", "cloud_cover",
                                                           "precipitation")])
    ter = L.PropagTerrainPtrs(*[(0 if k in ("d1hr", "d10hr", "d100hr") else dev[k].data_ptr())
                                for k in L.TERRAIN_FIELDS])
    out = [torch.empty(n, dtype=torch.float32, device="cuda") for _ in range(3)]
    rc = L.lib().propag_fire_weather_device(n, hour, month, C.byref(w), C.byref(ter),
                                            *[o.data_ptr() for o in out], None)
    assert rc == 0, L.last_error()
    torch.cuda.synchronize()
    for o, k in zip(out, ("speed_max", "azimuth_max", "eccentricity")):
        assert np.array_equal(o.cpu().numpy().view(np.uint32), two[k].ravel().view(np.uint32)), k
    assert (two["speed_max"] > 0).mean() > 0.3
    assert L.lib().propag_fire_weather_device(n, 24, month, C.byref(w), C.byref(ter),
                                              *[o.data_ptr() for o in out], None) == L.PROPAG_ERR_INVALID
