import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the product kernels")


def _build(target_dir):
    subprocess.run(["make", "-s", f"-j{os.cpu_count() or 1}", "-C", os.path.join(ROOT, target_dir)], check=True)


@pytest.fixture(scope="session", autouse=True)
def built_libraries():
    """Builds the oracle and the product library in place (no-ops when up to date)."""
    if os.environ.get("NEBULA_SKIP_BUILD") != "1":
        _build("oracle")
        _build(os.path.join("edge_rs_b200", "csrc"))
    yield
