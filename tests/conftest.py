import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libemfem_b200.so")


@pytest.fixture(scope="session")
def mt_small():
    from emfem_b200 import meshgen as mg
    return mg.mt_halfspace_block(4000, freqs=(0.1, 1.0, 10.0), name="mt-small")


@pytest.fixture(scope="session")
def mt_aniso():
    from emfem_b200 import meshgen as mg
    return mg.mt_halfspace_block(4000, with_block=False, n_bodies=3, topo_height=500.0,
                                 freqs=(0.01, 1.0), seed=5, name="mt-aniso")


@pytest.fixture(scope="session")
def csem_small():
    from emfem_b200 import meshgen as mg
    return mg.marine_csem(5000, freqs=(0.25, 1.25), name="csem-small")
