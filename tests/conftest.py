import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def engine_lib():
    from fasterstereocuda_b200.build import build_engine
    build_engine()
    import fasterstereocuda_b200 as fsc
    return fsc.load_library()


@pytest.fixture(scope="session")
def oracle_mod():
    from fasterstereocuda_b200.build import build_oracle
    build_oracle()
    from oracle import oracle
    return oracle


def cuda_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
