"""Shared fixtures.  Tests marked ``gpu`` need a B200; everything else runs on
the CPU (the oracle, the host mesh builder, the C ABI's exports and its
error handling)."""
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle():
    import pyoracle
    pyoracle.build()
    return pyoracle.Oracle()


@pytest.fixture(scope="session")
def lib():
    from fesom2_tracer_dwarf_b200 import _lib
    if not _lib.LIB_PATH.exists():
        subprocess.run(["make", "-s", "-C", str(ROOT / "fesom2_tracer_dwarf_b200")], check=True)
    return _lib.load()


@pytest.fixture()
def api(lib):
    from fesom2_tracer_dwarf_b200 import FESOMTracerAdvection
    t = FESOMTracerAdvection()
    t.cleanup()
    yield t
    t.cleanup()


def f64(a):
    return np.asfortranarray(np.asarray(a, dtype=np.float64))


@pytest.fixture(scope="session")
def pi_mesh_dir(tmp_path_factory):
    """The reference's ASCII pi mesh (tests/golden/pi/*.out.gz, byte copies),
    unpacked into a temporary mesh directory."""
    import gzip
    d = tmp_path_factory.mktemp("pi_mesh")
    for gz in (ROOT / "tests" / "golden" / "pi").glob("*.out.gz"):
        target = d / gz.name[:-3].replace("__", "/")  # dist_8__rpart.out -> dist_8/rpart.out
        target.parent.mkdir(exist_ok=True)
        target.write_bytes(gzip.decompress(gz.read_bytes()))
    return d
