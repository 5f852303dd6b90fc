import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running CPU test")


@pytest.fixture(scope="session")
def golden32():
    import numpy as np
    return dict(np.load(os.path.join(ROOT, "tests", "golden", "c0_32.npz")))


@pytest.fixture(scope="session")
def golden64():
    import numpy as np
    path = os.path.join(ROOT, "tests", "golden", "c1_64.npz")
    if not os.path.exists(path):
        pytest.skip("64^3 golden fixture not generated")
    return dict(np.load(path))


@pytest.fixture(scope="session")
def golden_rot():
    import numpy as np
    return dict(np.load(os.path.join(ROOT, "tests", "golden", "rot20.npz")))


@pytest.fixture(scope="session")
def golden_rotinterp():
    import numpy as np
    return dict(np.load(os.path.join(ROOT, "tests", "golden", "rotinterp12.npz")))
