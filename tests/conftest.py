import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: larger parity cases")


def _ensure_built():
    from exclucene_b200 import build as b

    b.build()
    import oracle

    oracle.build(ref=oracle.have_reference_tree())


_ensure_built()


def have_reference() -> bool:
    import oracle

    return oracle.have_reference_tree()


@pytest.fixture(scope="session")
def gpu_ctx():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import exclucene_b200 as ex

    ctx = ex.Context(0, max_queries=65536, max_keys=1 << 24)
    yield ctx
    ctx.close()
