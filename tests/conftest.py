import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "precision-study_b200")
for p in (PKG, os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) GPU")
    config.addinivalue_line("markers", "slow: long CPU run; set PMHD_SLOW=1 to run")


def pytest_collection_modifyitems(config, items):
    if os.environ.get("PMHD_SLOW") == "1":
        return
    skip = pytest.mark.skip(reason="slow; set PMHD_SLOW=1")
    for it in items:
        if "slow" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def oracle():
    import oracle_lib
    if not os.path.exists(oracle_lib.LIB_PATH):
        oracle_lib.build()
    return oracle_lib


@pytest.fixture(scope="session")
def pmhd_lib():
    lib = os.path.join(PKG, "libpmhd.so")
    if not os.path.exists(lib):
        subprocess.run(["make", "-s", "-C", PKG, "-j4"], check=True)
    import pmhd
    pmhd.load()
    return pmhd
