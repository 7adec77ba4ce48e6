import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def reference_checkout():
    """The reference's checkout, for the CPU tests that compare against its scene files: the
    directory named by TOASTER_REFERENCE, else a `reference` directory beside this repository.
    The tests that use it skip when neither exists."""
    env = os.environ.get("TOASTER_REFERENCE")
    return Path(env) if env else ROOT.parent / "reference"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) GPU and the built CUDA library")


def _gpu_available() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _gpu_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device in this environment")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


@pytest.fixture(scope="session")
def native_lib():
    from toaster_b200 import build, native

    build.build()
    return native.load_library()


@pytest.fixture(scope="session")
def renderer(native_lib):
    from toaster_b200.renderer import GpuRenderer

    r = GpuRenderer(int(os.environ.get("TC_DEVICE", "0")))
    yield r
    r.close()
