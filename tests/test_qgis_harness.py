"""A C program that binds libpropag.so exactly as the reference's QGIS
provider does (dlopen + dlsym, C terrain loader callback; see
tests/qgis_harness.c).  Without a GPU the call must fail with a message;
with one it must write the arrival-time GeoTIFF."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(ROOT, "propag-hidalgo_b200", "libpropag.so")


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    exe = str(tmp_path_factory.mktemp("qgis") / "qgis_harness")
    subprocess.run([cc, "-O1", "-std=c11", "-I", os.path.join(ROOT, "include"), "-o", exe,
                    os.path.join(HERE, "qgis_harness.c"), "-ldl"], check=True)
    return exe


def _run(harness, out):
    p = subprocess.run([harness, LIB, out], capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr
    return p.stdout.strip()


def test_harness_without_gpu_reports_error(harness, tmp_path, pp):
    if pp.check_cuda_available():
        pytest.skip("a GPU is present")
    out = _run(harness, str(tmp_path / "t.tif"))
    assert out.startswith("error:") and "CUDA" in out
    assert not os.path.exists(tmp_path / "t.tif")


@pytest.mark.gpu
def test_harness_runs_propagation(harness, tmp_path):
    out = _run(harness, str(tmp_path / "t.tif"))
    assert out == "ok loads=1", out
    data = open(tmp_path / "t.tif", "rb").read()
    assert data[:4] == b"II*\x00" and len(data) > 128 * 128 * 4
