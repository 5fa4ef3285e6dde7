"""Shared pytest configuration.

Markers: ``gpu`` tests need a CUDA device (a B200) and call the product
through its C-ABI; everything else runs on CPU.  ``slow`` tests run only with
OLAP_SLOW=1 (minutes of single-threaded CPU work).
"""
import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU; calls the sm_100a library")
    config.addinivalue_line("markers", "slow: minutes of CPU work; runs only with OLAP_SLOW=1")


def pytest_collection_modifyitems(config, items):
    if os.environ.get("OLAP_SLOW") == "1":
        return
    skip = pytest.mark.skip(reason="slow test: set OLAP_SLOW=1")
    for it in items:
        if "slow" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def golden_queries():
    import json
    return json.loads((ROOT / "tests" / "golden" / "olapcore_queries.json").read_text())


@pytest.fixture(scope="session")
def golden_sf1_groups():
    import json
    return json.loads((ROOT / "tests" / "golden" / "olapcore_sf1_groups.json").read_text())


@pytest.fixture(scope="session")
def ctx():
    from memory_database_b200 import olapcore
    c = olapcore.Context(0)
    yield c
    c.close()
