import os
import sys

import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
PKG = os.path.join(ROOT, "ocudu-dapp-platform_b200")
ORACLE = os.path.join(ROOT, "oracle")
GOLDEN = os.path.join(ROOT, "tests", "golden")
for p in (PKG, ORACLE):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU (B200)")


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def port():
    from oracle import Port
    return Port()


@pytest.fixture(scope="session")
def ref():
    """The reference's own compiled CPU code, when it was built (oracle/_ref travels with the tree)."""
    from oracle import REF_SO, Ref
    if not os.path.exists(REF_SO):
        pytest.skip("oracle/_ref not built")
    return Ref()


@pytest.fixture(scope="session")
def ctx():
    from pusch_b200 import _native
    c = _native.Context(device=0, max_codeblocks=1024)
    yield c
    c.close()


@pytest.fixture(scope="session")
def batch_decoder(ctx):
    from pusch_b200.ldpc import LdpcBatchDecoder
    return LdpcBatchDecoder(context=ctx)
