"""Test configuration: paths to the engine package and the oracle, GPU marker."""
import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "deleglise-rivat_b200")
ORACLE = os.path.join(ROOT, "oracle")
GOLDEN = os.path.join(ROOT, "tests", "golden")
for p in (PKG, ORACLE):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU (run with -m gpu)")
    config.addinivalue_line("markers", "slow: long-running parity case")


def load_golden(name):
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def oracle():
    from oracle_py import Oracle

    return Oracle()


@pytest.fixture(scope="session")
def reference():
    from oracle_py import Reference

    if not Reference.available():
        pytest.skip("reference build (oracle/_ref) not present")
    return Reference()


@pytest.fixture(scope="session")
def engine():
    import dr_b200

    e = dr_b200.Engine(0)
    yield e
    e.close()
