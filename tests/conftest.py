import glob
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs libdipl_bvh.so kernels")


@pytest.fixture(scope="session")
def orc():
    import oracle as O
    if not os.path.exists(O.ORC_LIB):
        O.build()
    return O.Oracle()


@pytest.fixture(scope="session")
def ref():
    import oracle as O
    if not os.path.exists(O.REF_LIB):
        pytest.skip("reference harness not built (oracle/_ref is produced where the reference tree exists)")
    return O.RefOracle()


def load_golden(name):
    with np.load(os.path.join(GOLDEN, name + ".npz")) as z:
        return {k: z[k] for k in z.files}


# triangle + ray fixtures (obj_*.npz hold scene-loader outputs instead)
GOLDEN_NAMES = sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "*.npz"))
                      if not os.path.basename(p).startswith("obj_"))


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)
