import os
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.dirname(HERE))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle():
    import mhd_cases as M
    if not M.oracle_available():
        pytest.skip("oracle library not built (python __graft_entry__.py build)")
    return M.OracleLib()


@pytest.fixture(scope="session")
def ref():
    import mhd_cases as M
    if not M.ref_available():
        pytest.skip("reference CPU build absent (oracle/build_ref.sh)")
    return M.RefLib()
