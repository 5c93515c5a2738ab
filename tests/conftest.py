import sys
from pathlib import Path

import pytest

sys.path.insert(0, str(Path(__file__).resolve().parent))
sys.path.insert(0, str(Path(__file__).resolve().parent.parent))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 (B200) GPU")
    config.addinivalue_line("markers", "slow: long-running")


@pytest.fixture(scope="session")
def gpu_available():
    from openlb_b200 import lbx
    return lbx.device_count() > 0


@pytest.fixture(autouse=True)
def _require_gpu(request):
    if request.node.get_closest_marker("gpu") is not None:
        from openlb_b200 import lbx
        if lbx.device_count() == 0:
            pytest.fail("GPU test selected but no sm_100 device is visible")
