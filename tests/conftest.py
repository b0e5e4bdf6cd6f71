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
    # one-program CG kernel builds are kept on disk; the test session (and the
    # processes it starts) shares a fresh cache instead of the user's
    if "SUS2SH_CACHE_DIR" not in os.environ:
        import tempfile
        os.environ["SUS2SH_CACHE_DIR"] = tempfile.mkdtemp(prefix="sus2sh_cache_")


@pytest.fixture(scope="session")
def model_dir(tmp_path_factory):
    return str(tmp_path_factory.mktemp("models"))


@pytest.fixture(scope="session")
def l3k3_path(model_dir):
    from sus2sh import models
    return models.preset_model("l3k3", model_dir)


@pytest.fixture(scope="session")
def laguerre_path(model_dir):
    """An l3k3 Cu-Zr model on the Laguerre-log1p radial basis (rho 3.5 A)."""
    import os
    from sus2sh import models
    path = os.path.join(model_dir, "l3k3_laguerre.mtp")
    if not os.path.exists(path):
        models.write_model(path, laguerre=True, seed=20260404)
    return path


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
