"""The oracle's k-space operators and energies against the reference's own
outputs (tests/golden/kspace_vectors.npz, from tests/golden/make_golden.py)."""
import json
import os

import numpy as np
import pytest

from oracle import contact_oracle as oc

KS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "kspace_vectors.npz")
_npz = np.load(KS)
CASES = sorted(k[2:-7] for k in _npz.files if k.startswith("k_") and k.endswith("_config"))


def oracle_substrate(cfg):
    nb, sizes = tuple(cfg["nb_grid_pts"]), tuple(cfg["physical_sizes"])
    if cfg["kind"] == "free":
        return oc.FreeSubstrate(nb, cfg["young"], sizes)
    return oc.PeriodicSubstrate(nb, cfg["young"], sizes, **cfg["kwargs"])


@pytest.mark.parametrize("name", CASES)
def test_kspace_oracle_vs_reference(name):
    cfg = json.loads(str(_npz[f"k_{name}_config"]))
    s = oracle_substrate(cfg)
    f, u = _npz[f"k_{name}_f"], _npz[f"k_{name}_u"]
    for key, got in (("kdisp", s.evaluate_k_disp(f)), ("kforce", s.evaluate_k_force(u)),
                     ("kforce_k", s.evaluate_k_force_k(_npz[f"k_{name}_kdisp"]))):
        ref = _npz[f"k_{name}_{key}"]
        np.testing.assert_allclose(got, ref, rtol=0, atol=1e-13 * abs(ref).max(), err_msg=key)
    ka, kb = _npz[f"k_{name}_kdisp"], _npz[f"k_{name}_kforce"]
    np.testing.assert_allclose(s.evaluate_scalar_product_k_space(ka, kb), _npz[f"k_{name}_dot"],
                               rtol=1e-12)
    np.testing.assert_allclose(s.evaluate_energy_k(u), _npz[f"k_{name}_energy_k"], rtol=1e-12)
    # the power theorem: the k-space product equals the real-space one
    da = s._apply(s.greens_function, -f, 1.0 / s.area_per_pt)
    fb = s._apply(s.surface_stiffness, u, -s.area_per_pt)
    np.testing.assert_allclose(s.evaluate_scalar_product_k_space(ka, kb),
                               float(np.sum(da * fb)), rtol=1e-10)
