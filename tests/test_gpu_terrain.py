"""Slope and aspect from a DEM on the device against numpy's definition
(np.gradient in double from the float DEM, hypot, arctan2 mapped to
[0, 2 pi), 0 where flat): within one float32 ulp (both round a double
result; the double atan2/hypot of the two libraries may differ in the last
bit)."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _numpy(dem, dx, dy):
    d = dem.astype(np.float64)
    gx = np.gradient(d, dx, axis=1) if d.shape[1] > 1 else np.zeros_like(d)
    gy = np.gradient(d, dy, axis=0) if d.shape[0] > 1 else np.zeros_like(d)
    s = np.hypot(gx, gy)
    a = np.arctan2(-gx, -gy)
    a = np.where(a < 0, a + 2 * np.pi, a)
    a = np.where(s == 0, 0.0, a)
    return s.astype(np.float32), a.astype(np.float32)


@pytest.mark.parametrize("shape,dx,dy", [((257, 300), 5.0, 5.0), ((128, 96), 30.0, -30.0),
                                         ((1, 50), 5.0, 5.0), ((40, 1), 2.0, -2.0)])
def test_slope_aspect_matches_numpy(pp, shape, dx, dy):
    import torch
    from py_propag import _lib as L
    from py_propag import scenarios as S
    rng = np.random.default_rng(7)
    h, w = shape
    dem = (S.dem_hills(w, h, abs(dx), rng) if min(shape) > 1 else rng.uniform(0, 500, shape))
    dem = np.asarray(dem, dtype=np.float32)
    dem[0, 0] = dem[0, min(1, w - 1)]  # a flat spot on an edge
    d = torch.from_numpy(dem.ravel().copy()).cuda()
    s = torch.empty_like(d)
    a = torch.empty_like(d)
    rc = L.lib().propag_slope_aspect_device(w, h, dx, dy, d.data_ptr(), s.data_ptr(), a.data_ptr(), None)
    assert rc == 0, L.last_error()
    torch.cuda.synchronize()
    ns, na = _numpy(dem, dx, dy)
    gs, ga = s.cpu().numpy().reshape(shape), a.cpu().numpy().reshape(shape)
    assert np.all(np.abs(gs - ns) <= np.spacing(np.maximum(np.abs(ns), 1e-30)))
    da = np.abs(ga - na)
    da = np.minimum(da, 2 * np.pi - da)  # 0 and 2 pi are the same direction
    assert np.all(da <= 2 * np.spacing(np.float32(2 * np.pi)))
    assert np.all((ga >= 0) & (ga <= np.float32(2 * np.pi)))


def test_slope_aspect_rejects_bad_sizes(pp):
    from py_propag import _lib as L
    assert L.lib().propag_slope_aspect_device(0, 5, 5.0, 5.0, None, None, None, None) == L.PROPAG_ERR_INVALID
