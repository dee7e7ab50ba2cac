import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "c-mc_electron_b200"))
sys.path.insert(0, os.path.join(ROOT, "tests"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); parity tests through the C ABI")


@pytest.fixture(scope="session")
def oracle_tables():
    from oracle_bridge import ORACLE_TABLES

    if not os.path.exists(os.path.join(ORACLE_TABLES, "bs.si.asc")):
        pytest.skip("oracle tables not staged (build the oracle first)")
    return ORACLE_TABLES
