import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session", autouse=True)
def _built_libraries():
    """Builds the generators and the oracle when missing (CPU only, seconds);
    the CUDA library is built by __graft_entry__.build() / cumat_b200/build.py.
    The build script is loaded by path, so that this works before the CUDA
    library (which the package loads on import) exists."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("_cumat_build", ROOT / "cumat_b200" / "build.py")
    build = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(build)
    build.build_problems()
    if not (ROOT / "oracle" / "liboracle.so").exists():
        build.build_oracle()
    yield


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def cuda():
    if not gpu_available():
        pytest.skip("no CUDA device")
    import torch
    return torch.device("cuda", 0)
