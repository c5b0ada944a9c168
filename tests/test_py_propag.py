"""The Python drop-in's validation and host logic, mirroring the reference's
own py_propag tests (crates/py-propag/tests/test_basic.py,
crates/py-propag/tests/test_validation.py) against this implementation's
real checks rather than restated conditions.  No GPU needed."""
import math

import numpy as np
import pytest

GT = np.array([0.0, 1.0, 0.0, 0.0, 0.0, -1.0], dtype=np.float64)
WKB = bytes([1, 1, 0, 0, 0, 0, 0, 0, 0, 0, 0, 240, 63, 0, 0, 0, 0, 0, 0, 0, 64])


def test_check_cuda_available_is_bool(pp):
    assert isinstance(pp.check_cuda_available(), bool)


def test_geo_reference(pp):
    g = pp.PyGeoReference(100, 200, "EPSG:4326", GT)
    assert (g.width, g.height, g.proj) == (100, 200, "EPSG:4326")
    assert list(g.transform) == list(GT)
    with pytest.raises(pp.PropagValidationError, match="Grid dimensions must be positive"):
        pp.PyGeoReference(0, 100, "EPSG:4326", GT)
    with pytest.raises(pp.PropagValidationError, match="too large"):
        pp.PyGeoReference(40000, 100, "EPSG:4326", GT)
    with pytest.raises(pp.PropagValidationError, match="exactly 6 elements"):
        pp.PyGeoReference(100, 200, "EPSG:4326", [0.0, 1.0, 0.0])
    for bad in ([0.0, 0.0, 0.0, 0.0, 0.0, -1.0], [0.0, 1.0, 0.0, 0.0, 0.0, 0.0]):
        with pytest.raises(pp.PropagValidationError, match="pixel size cannot be zero"):
            pp.PyGeoReference(10, 10, "EPSG:4326", bad)
    # a singular rotated transform has no inverse (GT::invert,
    # crates/geometry/src/lib.rs:107-113); an infinite pixel size without
    # rotation passes the reference's checks and passes here too
    with pytest.raises(pp.PropagValidationError, match="non-zero and finite"):
        pp.PyGeoReference(10, 10, "EPSG:4326", [0.0, 1.0, 1.0, 0.0, 1.0, 1.0])
    pp.PyGeoReference(10, 10, "EPSG:4326", [0.0, float("inf"), 0.0, 0.0, 0.0, -1.0])
    for t in ([-180.0, 0.1, 0.0, 90.0, 0.0, -0.1], [500000.0, 30.0, 0.0, 4000000.0, 0.0, -30.0]):
        pp.PyGeoReference(10, 10, "EPSG:4326", t)


def test_projection_edge_cases(pp):
    with pytest.raises(pp.PropagValidationError, match="Projection string cannot be empty"):
        pp.PyGeoReference(100, 200, "", GT)
    ok = "EPSG:4326+" + "a" * 1013
    assert pp.PyGeoReference(100, 200, ok, GT).proj == ok
    with pytest.raises(pp.PropagValidationError, match=r"Projection string too large \(max 1023 characters\)"):
        pp.PyGeoReference(100, 200, ok + "a", GT)
    uni = "EPSG:4326 with émojis 🌍 and spëcial chars: αβγ"
    assert pp.PyGeoReference(100, 200, uni, GT).proj == uni
    mb = "EPSG:4326+" + "é" * 506 + "a"
    assert len(mb.encode()) == 1023
    pp.PyGeoReference(100, 200, mb, GT)
    with pytest.raises(pp.PropagValidationError, match="too large"):
        pp.PyGeoReference(100, 200, "EPSG:4326+" + "€" * 338, GT)


def test_settings(pp):
    g = pp.PyGeoReference(100, 200, "EPSG:4326", GT)
    s = pp.PySettings(g, 3600.0)
    assert s.max_time == 3600.0
    for bad, msg in ((-1.0, "must be positive"), (0.0, "must be positive"),
                     (float("inf"), "finite number"), (10.1 * 365 * 24 * 3600.0, "10 years")):
        with pytest.raises(pp.PropagValidationError, match=msg):
            pp.PySettings(g, bad)
    with pytest.raises(pp.PropagValidationError):
        s.max_time = -5.0
    s.max_time = 31536000.0
    assert s.max_time == 31536000.0
    assert s.inner.geo_ref.width == 100


def test_time_feature(pp):
    f = pp.PyTimeFeature(300.0, WKB)
    assert f.time == 300.0 and f.geom_wkb == WKB
    with pytest.raises(pp.PropagValidationError, match="non-negative"):
        pp.PyTimeFeature(-1.0, WKB)
    with pytest.raises(pp.PropagValidationError, match="finite number"):
        pp.PyTimeFeature(float("inf"), WKB)
    with pytest.raises(pp.PropagValidationError, match="cannot be empty"):
        pp.PyTimeFeature(300.0, b"")
    for short in (b"short", b"x" * 8):
        with pytest.raises(pp.PropagValidationError, match="too short"):
            pp.PyTimeFeature(300.0, short)


def test_load_terrain_data(pp):
    rng = np.random.default_rng(0)
    w, h = 10, 10
    g = pp.load_terrain_data(w, h, "EPSG:4326", GT,
                             rng.uniform(0, 1000, (h, w)).astype(np.float32),
                             rng.uniform(0, 45, (h, w)).astype(np.float32),
                             rng.uniform(0, 360, (h, w)).astype(np.float32),
                             rng.integers(1, 14, (h, w)).astype(np.uint8))
    assert (g.width, g.height) == (w, h)
    with pytest.raises(pp.PropagValidationError, match="must be positive"):
        pp.load_terrain_data(0, 10, "EPSG:4326", GT, None, None, None, None)
    with pytest.raises(pp.PropagValidationError, match="100 million"):
        pp.load_terrain_data(50000, 50000, "EPSG:4326", GT)
    cases = [("elevation", np.full((h, w), 15000.0), "exceeds maximum"),
             ("elevation", np.full((h, w), -2000.0), "below minimum"),
             ("slope", np.full((h, w), 120.0), "exceeds maximum"),
             ("slope", np.full((h, w), -10.0), "below minimum"),
             ("aspect", np.full((h, w), 400.0), "exceeds maximum"),
             ("aspect", np.full((h, w), -45.0), "below minimum"),
             ("fuel_model", np.full((h, w), 20, np.uint8), "Invalid fuel model ID"),
             ("elevation", np.zeros((h + 10, w)), "shape mismatch")]
    for name, arr, msg in cases:
        with pytest.raises(pp.PropagValidationError, match=msg):
            pp.load_terrain_data(w, h, "EPSG:4326", GT, **{name: arr})


def test_propagate_argument_validation(pp, tmp_path):
    g = pp.PyGeoReference(16, 16, "EPSG:4326", GT)
    s = pp.PySettings(g, 100.0)
    f = [pp.PyTimeFeature(0.0, WKB)]
    out = str(tmp_path / "o.tif")
    for path in ("", "../etc/passwd", "data/../../../etc/hosts", "/etc/shadow", "/sys/kernel/config",
                 "/proc/version"):
        with pytest.raises(pp.PropagValidationError):
            pp.propagate(s, path, f, "EPSG:4326")
    with pytest.raises(pp.PropagValidationError):
        pp.propagate(s, out, f, "EPSG:4326", refs_output_path="../x.csv")
    with pytest.raises(pp.PropagValidationError, match="CRS"):
        pp.propagate(s, out, f, "")
    with pytest.raises(pp.PropagValidationError, match="too long"):
        pp.propagate(s, out, f, "x" * 3000)
    with pytest.raises(pp.PropagValidationError, match="At least one"):
        pp.propagate(s, out, [], "EPSG:4326")
    with pytest.raises(pp.PropagValidationError, match="Too many"):
        pp.propagate(s, out, f * 10001, "EPSG:4326")


def test_propagate_without_gpu_raises_cuda_error(pp, tmp_path):
    if pp.check_cuda_available():
        pytest.skip("a GPU is present")
    g = pp.PyGeoReference(16, 16, "EPSG:4326", GT)
    with pytest.raises(pp.PropagCudaError, match="CUDA is not available"):
        pp.propagate(pp.PySettings(g, 100.0), str(tmp_path / "o.tif"),
                     [pp.PyTimeFeature(0.0, WKB)], "EPSG:4326")


def test_exception_hierarchy(pp):
    assert issubclass(pp.PropagCudaError, RuntimeError)
    assert issubclass(pp.PropagGdalError, RuntimeError)
    assert issubclass(pp.PropagMPIError, RuntimeError)
    assert issubclass(pp.PropagValidationError, ValueError)
    assert pp.Settings is pp.PySettings and pp.GeoReference is pp.PyGeoReference


def test_terrain_validation(pp):
    t = pp.demo_terrain(8, 8)
    del t["slope"]
    with pytest.raises(pp.PropagValidationError, match="missing 'slope'"):
        pp._terrain_host(t, 64)
    t = pp.demo_terrain(8, 8)
    t["aspect"] = np.zeros(10, np.float32)
    with pytest.raises(pp.PropagValidationError, match="has 10 cells"):
        pp._terrain_host(t, 64)


def test_scenarios_are_deterministic_and_in_range(pp):
    from py_propag import scenarios as S
    a, b = S.config1(size=96, seed=3, n_ign=5), S.config1(size=96, seed=3, n_ign=5)
    for k in a.terrain:
        assert np.array_equal(a.terrain[k], b.terrain[k]), k
    assert a.ignitions == b.ignitions and len(a.ignitions) == 5
    t = a.terrain
    assert t["fuel_code"].dtype == np.uint8 and t["fuel_code"].max() <= 13
    assert np.all(t["slope"] >= 0) and np.all(t["slope"] <= math.tan(math.radians(45.0)) + 1e-5)
    assert np.all((t["aspect"] >= 0) & (t["aspect"] < 2 * np.pi + 1e-5))
    assert np.all((t["wind_speed"] >= 0) & (t["wind_speed"] <= 15.0 + 1e-5))
    assert np.mean(t["fuel_code"] == 0) < 0.3
    c = S.config1(size=96, seed=4, n_ign=5)
    assert not np.array_equal(a.terrain["fuel_code"], c.terrain["fuel_code"])
    z = S.config0(size=64)
    assert len(z.ignitions) == 1 and z.width == z.height == 64
