import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

ORACLE_SO = os.path.join(ROOT, "oracle", "lib", "liboracle_gint.so")
REF_HOST_SO = os.path.join(ROOT, "oracle", "_ref", "libref_host.so")
REF_GINT_SO = os.path.join(ROOT, "oracle", "_ref", "libref_gint.so")
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (runs the CUDA engine)")


def _ensure_built():
    from libgint_b200.build import build_engine, build_driver
    build_driver()
    try:
        build_engine()
    except Exception:
        # a prebuilt engine is fine where nvcc is absent
        if not os.path.exists(os.path.join(ROOT, "libgint_b200", "lib", "libgint_b200.so")):
            raise
    if not os.path.exists(ORACLE_SO):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle")], check=True, capture_output=True)


_ensure_built()


@pytest.fixture(scope="session")
def oracle_path():
    return ORACLE_SO


@pytest.fixture(scope="session")
def engine_so():
    from libgint_b200.capi import engine_path
    return engine_path()
