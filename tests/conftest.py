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


def golden_pipeline_names(npz):
    return sorted(k[len("pipe_"):-len("_config")] for k in npz.files
                  if k.startswith("pipe_") and k.endswith("_config"))


def golden_pipeline_case(npz, name):
    """(heights, physical sizes, periodic, keyword arguments of contact_mechanics)
    of a recorded automated sweep."""
    cfg = json.loads(str(npz[f"pipe_{name}_config"]))
    kw = {k: cfg[k] for k in ("nsteps", "offsets", "pressures", "maxiter", "optimizer_kwargs",
                              "hardness") if k in cfg and cfg[k] is not None}
    return npz[f"pipe_{name}_heights"], tuple(cfg["physical_sizes"]), cfg["periodic"], kw


PIPELINE_OUTPUTS = ("mean_pressure", "area", "mean_displacement", "mean_gap", "converged")
