"""Shared pytest set-up: the `gpu` marker, import paths, and the native library
(built on demand; there is no CPU fallback, so GPU tests fail loudly if it is
missing)."""

import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def native():
    from reformulation_b200 import build, _native
    build.build()
    return _native.lib()


@pytest.fixture(scope="session")
def oracle_lib():
    import subprocess
    subprocess.run(["make", "-s", "-C", str(ROOT / "oracle")], check=True)
    import oracle
    return oracle
