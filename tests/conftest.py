import os
import sys

import numpy as np
import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
HERE = os.path.dirname(os.path.abspath(__file__))
if HERE not in sys.path:
    sys.path.insert(0, HERE)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the sm_100a library")


@pytest.fixture(scope="session")
def cube_lib():
    """The sm_100a library, built in-tree if stale (nvcc cross-compiles without a GPU)."""
    from cube2_b200 import build as B
    B.build()
    from cube2_b200 import kick
    return kick.lib()


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle import oracle as O
    O.build_oracle()
    return O.lib()


@pytest.fixture(scope="session")
def gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from cube2_b200 import build as B
    B.build()
    return torch.device("cuda:0")


def load_golden(name):
    """Image + reference outputs of tests/golden/pp_<name>.npz."""
    from cube2_b200.layout import Image, Layout
    from oracle.layouts import LAYOUTS
    z = np.load(os.path.join(HERE, "golden", f"pp_{name}.npz"))
    L = Layout(**LAYOUTS[str(z["layout"])])
    img = Image(L, z["xp"], z["vp"], z["rhoc"], z["idx_b_r"], np.zeros(z["xp"].shape[0], np.int64), z["active"],
                n_particles=int(z["active"].sum()))
    return img, z
