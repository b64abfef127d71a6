import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "lxmf-vanity_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (runs the sm_100a kernels through the C ABI)")
    config.addinivalue_line("markers", "slow: takes more than a few seconds")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.lib()
    return O


@pytest.fixture(scope="session")
def lx():
    import lxmfv
    lxmfv.lib()
    return lxmfv


@pytest.fixture(scope="session", params=["group", "xadd"])
def backend(lx, request):
    """One open device per walk for the GPU tests (a small walker count)."""
    walk = lx.WALK_GROUP if request.param == "group" else lx.WALK_XADD
    b = lx.Backend(device=0, lanes=4096, batch=64, walk=walk)
    yield b
    b.close()
