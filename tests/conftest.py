import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libgg_b200.so")


def _ensure_oracle():
    lib = os.path.join(ROOT, "oracle", "liboracle.so")
    if not os.path.exists(lib):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "restatement"], check=True,
                       capture_output=True)
    return lib


@pytest.fixture(scope="session")
def oracle():
    _ensure_oracle()
    import pyoracle

    return pyoracle


@pytest.fixture(scope="session")
def gpu():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import gragles_3d_b200 as gg

    gg.load_library()  # fails loudly if the extension is missing
    return gg
