import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden", "reference_vectors.npz")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def golden():
    return np.load(GOLDEN)


def golden_solve_names(npz):
    return sorted(k[len("ccg_"):-len("_config")] for k in npz.files
                  if k.startswith("ccg_") and k.endswith("_config"))


def golden_config(npz, name):
    return json.loads(str(npz[f"ccg_{name}_config"]))


def golden_operator_names(npz):
    return sorted(k[len("op_"):-len("_config")] for k in npz.files
                  if k.startswith("op_") and k.endswith("_config"))


def golden_operator_config(npz, name):
    return json.loads(str(npz[f"op_{name}_config"]))
