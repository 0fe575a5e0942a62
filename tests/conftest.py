import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) GPU")
    config.addinivalue_line("markers", "ref: needs the reference built from source (oracle/_ref)")
    config.addinivalue_line("markers", "slow: takes minutes (a full-size oracle solve on one host core)")


def pytest_collection_modifyitems(config, items):
    from oracle import oracle as O
    have_ref = O.REF_LIB.exists()
    for it in items:
        if "ref" in it.keywords and not have_ref:
            it.add_marker(pytest.mark.skip(reason="oracle/_ref not built (reference tree absent)"))


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.clib()
    return O


@pytest.fixture(scope="session")
def sys0():
    """The 32x32-interior 2D P1-FEM system (n = 1024) with its x_true."""
    from project_xplus_b200 import generators as g
    return g.system_2d_small()


@pytest.fixture(scope="session")
def gpu():
    import project_xplus_b200 as xp
    if xp.device_count() == 0:
        pytest.fail("gpu test collected but no sm_100 device is visible")
    return xp
