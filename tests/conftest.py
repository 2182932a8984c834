"""pytest set-up: the `gpu` marker, the golden-vector manifest, the oracle and the library."""
import json
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
GOLDEN = ROOT / "tests" / "golden"
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (a B200)")


def manifest():
    return json.loads((GOLDEN / "manifest.json").read_text())


@pytest.fixture(scope="session")
def oracle_bin():
    """The CPU oracle (test infrastructure), built from oracle/ if needed."""
    subprocess.run(["make", "-s", "-C", str(ROOT / "oracle")], check=True)
    return ROOT / "oracle" / "_build" / "twins_oracle"


@pytest.fixture(scope="session")
def native_lib():
    """The product library, built in-tree if needed."""
    from twins_b200 import build
    build.build()
    return build.SO


@pytest.fixture(scope="session")
def rdma_kat():
    """The reference's known answers for the RDMA rules."""
    import rdma_shim
    return rdma_shim.load_kat()


@pytest.fixture(scope="session")
def rdma_lib(tmp_path_factory):
    """The RDMA rules' C shim, built with g++ (the CPU build of the rules)."""
    import shutil
    import rdma_shim
    if shutil.which("g++") is None:
        pytest.skip("g++ is not here")
    return rdma_shim.build(tmp_path_factory.mktemp("rdma_shim"))
