"""pytest configuration: the `gpu` marker and shared helpers.

CPU tests (-m "not gpu") cover the oracle against the golden fixtures, the host
logic and the library's exported ABI; GPU tests (-m gpu) are the parity tests
of the CUDA path through the C ABI.
"""
import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")
GOLDEN_CASES = ["grid16_pm", "hernquist2048_iso", "mix1500_pm", "grid12_ewald", "mns2000_pm"]


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and runs the CUDA library")


def load_golden(name):
    z = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    d = {k: z[k] for k in z.files}
    d["params"] = json.loads(str(d["params"]))
    return d


@pytest.fixture(scope="session")
def cuda_lib():
    """Builds (if stale) and loads libarepo_gpugrav; GPU tests only."""
    from arepo_b200 import build as B
    from arepo_b200 import _lib

    B.build()
    return _lib.load()
