import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libnewton_b200.so")
    config.addinivalue_line("markers", "product_build: runs on the product build (FMA contraction) of the library "
                                       "and compares at a stated tolerance; every other test runs on the parity "
                                       "build, which agrees with the oracle bit for bit")


@pytest.fixture(autouse=True)
def _library_build(request):
    """Bit-exact comparisons with the oracle use the parity build (--fmad=false); tests marked
    product_build check the product build at tolerance."""
    from newton_custom_contact_b200 import _lib

    prev = _lib.use_build("product" if request.node.get_closest_marker("product_build") else "exact")
    yield
    _lib.use_build(prev)


@pytest.fixture(scope="session")
def orc():
    import oracle

    oracle.build()
    return oracle


@pytest.fixture(scope="session")
def cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from newton_custom_contact_b200 import _lib

    _lib.load()
    return torch.device("cuda")
