"""The FP64 form against the oracle over long windows at full lattice size:
configuration 2 (1601 x 641, MDF + Peskin-4, TRT and CM-MRT) for 2 000 steps,
configuration 3 (1281 x 1281, oscillating DFC) for one period of 10 000 steps,
and configuration 5 (321 x 1281, two settling discs, coupled MDF, CM-MRT) for
5 000 steps.  The oracle's results are committed as SHA-256 digests
(tests/golden/make_golden_long.py, run on the host), so nothing here runs the
oracle: every final field must hash to the same digest (bit for bit), the Cd /
Cl histories agree to 1e-12 (the device sums forces in another order) and the
particles' positions, velocities and forces are equal."""
import hashlib
import json
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(__file__), "golden")
NAMES = ["C2_trt_2000", "C2_cmmrt_2000", "C3_10000", "C5_5000"]


@pytest.fixture(scope="module")
def torch():
    import torch
    assert torch.cuda.is_available()
    return torch


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.float64).tobytes()).hexdigest()


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_fp64_long_window_matches_oracle_digest(torch, name):
    path = os.path.join(GOLD, f"long_{name}.npz")
    if not os.path.exists(path):
        pytest.skip(f"{path} has not been generated")
    from iblbm_b200 import run
    from tests.test_gpu_parity import _cfg
    g = np.load(path)
    kw = json.loads(bytes(g["config_json"]).decode())
    cfg = _cfg(kw)
    res = run(cfg, verbose=False)
    assert res["engine"].status() == 0
    assert res["final_step"] == int(g["final_step"][0])
    st = res["state"]
    for k in ("ro", "U", "fib", "fstar", "feq"):
        assert _sha(getattr(st, k)) == bytes(g[f"sha_{k}"]).hex(), k
    np.testing.assert_allclose(res["Cd_history"], g["Cd_history"], rtol=1e-12, atol=1e-15)
    np.testing.assert_allclose(res["Cl_history"], g["Cl_history"], rtol=1e-12, atol=1e-13)
    if "particles" in g:
        got = np.array([[*p.pos, *p.vel, *p.force] for p in st.particles])
        np.testing.assert_array_equal(got, g["particles"])
