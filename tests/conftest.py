"""Shared fixtures.  GPU tests are marked `gpu`; everything else runs on CPU.  The default library of the
test process is the parity build (BTE_LIBRARY=parity)."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
# Bit-exact tests run on the parity build of the library; tests of the product build ask for variant="fast".
os.environ.setdefault("BTE_LIBRARY", "parity")
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def _has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _has_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle as O
    if not (os.path.exists(os.path.join(ROOT, "oracle", "liboracle.so")) and
            os.path.exists(os.path.join(ROOT, "oracle", "liboracle_libm.so"))):
        O.build(ref=True)
    return O


@pytest.fixture(scope="session")
def bte():
    import bluetruthengine_b200 as B
    B.load_library()
    return B


@pytest.fixture(scope="session")
def cornell_scene(bte):
    from bluetruthengine_b200 import scenes
    return bte.load_scene(scenes.cornell())


@pytest.fixture(scope="session")
def random_scene(bte):
    from bluetruthengine_b200 import scenes
    return bte.load_scene(scenes.random_scene(5))


@pytest.fixture(scope="session")
def renderer(bte):
    return bte.Renderer()


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)
