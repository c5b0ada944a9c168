"""The propagation's time_from arithmetic against the reference's own.

The reference evaluates time_from (crates/propag/src/propag.cu:269-294) with
CUDA's atan2f, the __cosf intrinsic, __frcp_rd, __fsqrt_rz and whatever
multiply-adds nvcc contracts under its default flags
(crates/propag/build.rs:48-69).  oracle/_ref/libref_time_from.so is that
source compiled the way the reference builds it; the engine's
PROPAG_ARITH_REFERENCE arithmetic must give the same bits on every case.
The CPU restatement's trig = 3 mode (the GPU's __cosf/atan2f values in
tables, fused multiply-adds) must give them too, which is what lets the
whole-propagation tests compare the engine with it bit for bit.
"""
import ctypes as C
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_SO = os.path.join(ROOT, "oracle", "_ref", "libref_time_from.so")


def _cases(seed: int, n_far: int = 200_000):
    """Offsets from the source cell to the evaluated cell: every offset within
    40 cells, then random ones up to 4095 cells; eccentricities from 0 to
    0.999 (0 and the extremes included), speeds over five decades, azimuths
    over [0, 2 pi), start times from 0 to 12 h."""
    rng = np.random.default_rng(seed)
    g = np.arange(-40, 41)
    ddx, ddy = (a.ravel() for a in np.meshgrid(g, g))
    keep = (ddx != 0) | (ddy != 0)
    ddx, ddy = ddx[keep], ddy[keep]
    ddx = np.concatenate([ddx, rng.integers(-4095, 4096, n_far)]).astype(np.int32)
    ddy = np.concatenate([ddy, rng.integers(-4095, 4096, n_far)]).astype(np.int32)
    n = ddx.size
    ecc = rng.uniform(0.0, 0.999, n).astype(np.float32)
    ecc[::17] = 0.0
    ecc[5::17] = np.float32(0.999)
    smax = np.exp(rng.uniform(np.log(1e-3), np.log(1e2), n)).astype(np.float32)
    az = rng.uniform(0.0, 2 * np.pi, n).astype(np.float32)
    az[3::11] = 0.0
    ftime = rng.uniform(0.0, 43200.0, n).astype(np.float32)
    ftime[::7] = 0.0
    return ddx, ddy, ftime, smax, az, ecc


def _ref_time_from(ddx, ddy, ftime, smax, az, ecc, dx, dy):
    if not os.path.exists(REF_SO):
        pytest.skip("oracle/_ref/libref_time_from.so not built (needs the reference checkout)")
    lib = C.CDLL(REF_SO)
    lib.ref_time_from_batch.restype = C.c_int
    lib.ref_time_from_batch.argtypes = [C.c_int64] + [C.c_void_p] * 6 + [C.c_float, C.c_float] + \
        [C.c_void_p] * 3
    n = ddx.size
    out = np.empty(n, np.float32)
    tx = np.empty(n, np.int32)
    ty = np.empty(n, np.int32)
    rc = lib.ref_time_from_batch(n, *[a.ctypes.data for a in (ddx, ddy, ftime, smax, az, ecc)],
                                 dx, dy, out.ctypes.data, tx.ctypes.data, ty.ctypes.data)
    assert rc == 0, f"reference harness: CUDA error {rc}"
    return out, tx, ty


def _device_time_from(L, arith, fx, fy, ftime, tx, ty, smax, az, ecc, dx, dy):
    out = np.empty(fx.size, np.float32)
    rc = L.lib().propag_selftest_time_from(arith, fx.size, *[a.ctypes.data for a in
                                                             (fx, fy, ftime, tx, ty, smax, az, ecc)],
                                           dx, dy, out.ctypes.data)
    assert rc == 0, L.last_error()
    return out


GRIDS = [(5.0, 5.0), (5.0, -5.0), (30.0, -12.5), (2.0, 7.5)]


@pytest.mark.parametrize("dx,dy", GRIDS)
def test_reference_arith_equals_reference_source(pp, dx, dy):
    """PROPAG_ARITH_REFERENCE gives the reference kernel's own bits (south-up
    and north-up, square and oblong cells)."""
    from py_propag import _lib as L
    ddx, ddy, ftime, smax, az, ecc = _cases(int(abs(dx * 10 + dy)))
    ref, tx, ty = _ref_time_from(ddx, ddy, ftime, smax, az, ecc, dx, dy)
    fx, fy = (tx + ddx).astype(np.int32), (ty + ddy).astype(np.int32)
    got = _device_time_from(L, L.PROPAG_ARITH_REFERENCE, fx, fy, ftime, tx, ty, smax, az, ecc, dx, dy)
    diff = got.view(np.uint32) != ref.view(np.uint32)
    assert not diff.any(), (f"{diff.sum()} of {diff.size} differ; first case {np.argmax(diff)}: "
                            f"{got[diff][:3]} vs {ref[diff][:3]}")
    # the portable arithmetic is a different rounding of the same quantity:
    # __cosf's absolute error (about 2^-21.4) grows by e / (1 - e cos) in
    # the elliptical factor, up to 1000 times at e = 0.999
    port = _device_time_from(L, L.PROPAG_ARITH_PORTABLE, fx, fy, ftime, tx, ty, smax, az, ecc, dx, dy)
    rel = np.abs(port.astype(np.float64) - ref) / np.maximum(np.abs(ref.astype(np.float64)), 1e-30)
    assert rel.max() < 1e-3
    assert np.median(rel) < 1e-6


@pytest.mark.parametrize("dx,dy", GRIDS[:2])
def test_oracle_tables_follow_reference_arith(pp, ref_oracle, dx, dy):
    """The CPU restatement with the device's __cosf/atan2f tables (trig = 3)
    gives the engine's reference-arithmetic bits; without them (trig = 2,
    libm) it does not in general."""
    from py_propag import _lib as L
    ddx, ddy, ftime, smax, az, ecc = _cases(7)
    tx = np.full(ddx.size, 5000, np.int32)
    ty = np.full(ddx.size, 5000, np.int32)
    fx, fy = (tx + ddx).astype(np.int32), (ty + ddy).astype(np.int32)
    got = _device_time_from(L, L.PROPAG_ARITH_REFERENCE, fx, fy, ftime, tx, ty, smax, az, ecc, dx, dy)
    misses = ref_oracle.table_misses()
    cpu = ref_oracle.time_from_batch(dx, dy, fx, fy, ftime, tx, ty, smax, az, ecc, trig=3)
    assert ref_oracle.table_misses() == misses
    assert np.array_equal(cpu.view(np.uint32), got.view(np.uint32))
    port = _device_time_from(L, L.PROPAG_ARITH_PORTABLE, fx, fy, ftime, tx, ty, smax, az, ecc, dx, dy)
    cpu0 = ref_oracle.time_from_batch(dx, dy, fx, fy, ftime, tx, ty, smax, az, ecc, trig=0)
    assert np.array_equal(cpu0.view(np.uint32), port.view(np.uint32))
