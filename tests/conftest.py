import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "propag-hidalgo_b200")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


def has_gpu() -> bool:
    try:
        import py_propag
        return py_propag.check_cuda_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O._load()
    return O


def trig_for(arith: int) -> int:
    """The oracle's trig mode that follows the engine's arithmetic `arith`:
    3 (the device's __cosf/atan2f tables) for PROPAG_ARITH_REFERENCE, 0 for
    PROPAG_ARITH_PORTABLE."""
    return 3 if arith == 0 else 0


@pytest.fixture(scope="session")
def ref_oracle():
    """The oracle with the device's __cosf and atan2f values installed (use
    trig=3 for PROPAG_ARITH_REFERENCE results; grids up to 4096 cells a side)."""
    from oracle import oracle
    from py_propag import _lib as L
    oracle._load()
    oracle.install_device_tables(L.lib(), 4095)
    yield oracle
    oracle.set_device_tables(None, 0, 1.0, None, 0, 0)


@pytest.fixture(scope="session")
def pp():
    import py_propag
    return py_propag


def random_terrain(n: int, seed: int, quickcheck: bool = False) -> dict:
    """Terrains like the reference's quickcheck generator
    (crates/firelib/src/lib.rs:415-448) or realistic ranges."""
    rng = np.random.default_rng(seed)
    if quickcheck:
        return dict(fuel_code=rng.integers(0, 13, n).astype(np.uint8),
                    d1hr=(rng.integers(0, 101, n) / 100).astype(np.float32),
                    d10hr=(rng.integers(0, 101, n) / 100).astype(np.float32),
                    d100hr=(rng.integers(0, 101, n) / 100).astype(np.float32),
                    herb=(rng.integers(0, 101, n) / 100).astype(np.float32),
                    wood=(rng.integers(0, 101, n) / 100).astype(np.float32),
                    wind_speed=(rng.integers(0, 101, n) / 10).astype(np.float32),
                    wind_azimuth=np.deg2rad(rng.integers(0, 3601, n) / 10).astype(np.float32),
                    slope=(rng.integers(0, 1001, n) / 1000).astype(np.float32),
                    aspect=np.deg2rad(rng.integers(0, 3601, n) / 10).astype(np.float32))
    return dict(fuel_code=rng.integers(0, 16, n).astype(np.uint8),
                d1hr=rng.uniform(0.02, 0.2, n).astype(np.float32),
                d10hr=rng.uniform(0.03, 0.25, n).astype(np.float32),
                d100hr=rng.uniform(0.04, 0.3, n).astype(np.float32),
                herb=rng.uniform(0.3, 2.0, n).astype(np.float32),
                wood=rng.uniform(0.5, 2.0, n).astype(np.float32),
                wind_speed=rng.uniform(0, 15, n).astype(np.float32),
                wind_azimuth=rng.uniform(0, 2 * np.pi, n).astype(np.float32),
                slope=rng.uniform(0, 1.2, n).astype(np.float32),
                aspect=rng.uniform(0, 2 * np.pi, n).astype(np.float32))
