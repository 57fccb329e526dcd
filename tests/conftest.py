import json
import os
import sys
import tempfile
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))

import __graft_entry__ as graft  # noqa: E402


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA (B200) device")
    # keep the kernel-variant tuning cache of the tests out of the user's home
    os.environ.setdefault("FE_B200_TUNE_CACHE",
                          os.path.join(tempfile.mkdtemp(prefix="fe_b200_tune_"), "tune.txt"))


def cuda_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def fe():
    """The package (fixedeffects.jl_b200/) with its CUDA library loaded."""
    mod = graft.load_package()
    mod._lib.load()
    return mod


@pytest.fixture(scope="session")
def fe_host():
    """The package without touching the CUDA library (host-side helpers)."""
    return graft.load_package()


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.build()
    return O


@pytest.fixture(scope="session")
def golden():
    return json.loads((ROOT / "tests" / "golden" / "solve_jl.json").read_text())


@pytest.fixture(scope="session")
def synth():
    graft.load_package()
    import fe_b200.synth as S
    return S
