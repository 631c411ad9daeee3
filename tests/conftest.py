import os
import subprocess
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(REPO, "tests", "golden")
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def pytest_collection_modifyitems(config, items):
    # keep files in name order so that tests/test_zz_* runs last
    items.sort(key=lambda it: (os.path.basename(str(it.fspath)), 0))


@pytest.fixture(scope="session")
def oracle_lib():
    import pso

    if not os.path.exists(pso.LIB):
        subprocess.run(["make", "-s", "-C", os.path.join(REPO, "oracle")], check=True)
    return pso


@pytest.fixture(scope="session")
def native():
    """The product library; built here when absent (the GPU box gets the
    prebuilt one)."""
    import periodsearch_b200 as ps

    if not os.path.exists(ps.LIB_PATH):
        from periodsearch_b200 import build

        build.build()
    return ps


def golden_path(name, f="period_search_in"):
    return os.path.join(GOLDEN, name, f)
