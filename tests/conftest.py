import glob
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the engine through the C ABI")


def golden_names():
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "*.npz")))


def load_golden(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    return {k: z[k] for k in z.files}


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle as O
    O.build()
    return O


@pytest.fixture(scope="session")
def pbrcm():
    import parallelbatchrcm_b200 as P
    from parallelbatchrcm_b200 import _lib
    _lib.lib()  # raises if libpbrcm.so has not been built
    return P


@pytest.fixture(scope="session")
def gpu_ctx(pbrcm):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    ctx = pbrcm.Context(0)
    yield ctx
    ctx.close()


@pytest.fixture(scope="session")
def gpu_ctx_team(pbrcm):
    """A context that runs every single matrix on the team engine
    (PBRCM_ENGINE=team: neither the shared-memory engine nor the hand-over
    to the level-synchronous one)."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    old = os.environ.get("PBRCM_ENGINE")
    os.environ["PBRCM_ENGINE"] = "team"
    try:
        ctx = pbrcm.Context(0)
    finally:
        if old is None:
            del os.environ["PBRCM_ENGINE"]
        else:
            os.environ["PBRCM_ENGINE"] = old
    yield ctx
    ctx.close()
