import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


def rel_l2(x, ref) -> float:
    x, ref = np.asarray(x), np.asarray(ref)
    dt = np.complex128 if (np.iscomplexobj(x) or np.iscomplexobj(ref)) else np.float64
    x = x.astype(dt)
    ref = ref.astype(dt)
    return float(np.linalg.norm((x - ref).ravel()) / np.linalg.norm(ref.ravel()))


@pytest.fixture(scope="session")
def ctx():
    import cudaem_b200 as cb
    c = cb.Context(0)
    yield c
    c.close()


@pytest.fixture(scope="session", autouse=True)
def _built_library():
    # the engine library is built in-tree; build it if a checkout lacks it
    from cudaem_b200 import build
    build.build()
    yield
