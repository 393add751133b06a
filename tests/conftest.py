import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (sm_100a); parity tests through the C ABI")


@pytest.fixture(scope="session")
def orc():
    from oracle import oracle
    oracle.lib()
    return oracle


@pytest.fixture(scope="session")
def ref(orc):
    if orc.ref_lib() is None:
        pytest.skip("reference kernels (oracle/_ref) not built")
    return orc


@pytest.fixture(scope="session")
def xlib():
    from xpulse_recon_b200 import _lib
    return _lib.lib()


@pytest.fixture(scope="session")
def ctx():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from xpulse_recon_b200.projector import Context
    c = Context(0)
    yield c
    c.close()
