import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "gpumd-sus2-sh_b200")
ORACLE = os.path.join(REPO, "oracle")
for p in (PKG, ORACLE):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); parity tests through the C-ABI")


@pytest.fixture(scope="session")
def model_dir(tmp_path_factory):
    return str(tmp_path_factory.mktemp("models"))


@pytest.fixture(scope="session")
def l3k3_path(model_dir):
    from sus2sh import models
    return models.preset_model("l3k3", model_dir)


@pytest.fixture(scope="session")
def l4k4_path(model_dir):
    from sus2sh import models
    return models.preset_model("l4k4", model_dir)


def cuda_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
