import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs on the B200 box)")


@pytest.fixture(scope="session")
def water_case():
    from subsecondpbs_b200 import phantoms

    return phantoms.water_phantom_case()


@pytest.fixture(scope="session")
def hetero_small_case():
    from subsecondpbs_b200 import phantoms

    return phantoms.heterogeneous_case(dims=(96, 96, 64), n_layers=4, target_radius_mm=20.0)


@pytest.fixture(scope="session")
def hetero_case():
    from subsecondpbs_b200 import phantoms

    return phantoms.heterogeneous_case()
