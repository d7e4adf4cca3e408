"""The single-particle sedimentation runtime (iblbm/runtime/scenarios/
sedimentation_single.py) against the reference's own runs of it
(tests/golden/sed1_*.npz, written by tests/golden/make_golden.py): every field
bit for bit (SHA-256), the disc's position, velocity, force and rotation, and
the history records, on the FP64 form."""
import hashlib
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden")
CASES = sorted(f[5:-4] for f in os.listdir(GOLD) if f.startswith("sed1_") and f.endswith(".npz"))


@pytest.fixture(scope="module")
def torch():
    import torch
    assert torch.cuda.is_available()
    return torch


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(np.asarray(a, dtype=np.float64)).tobytes()).hexdigest()


@pytest.mark.parametrize("name", CASES)
def test_single_particle_runtime_matches_reference(torch, name):
    from iblbm_b200 import run
    from iblbm_b200.config import SimConfig
    g = dict(np.load(os.path.join(GOLD, f"sed1_{name}.npz")))
    kw = json.loads(bytes(g["config_json"]).decode())
    kw["cylinder_center"] = tuple(kw["cylinder_center"])
    if kw.get("prescribed_velocity") is not None:
        kw["prescribed_velocity"] = tuple(kw["prescribed_velocity"])
    res = run(SimConfig(**kw), verbose=False)
    st = res["state"]
    assert res["engine"].status() == 0
    for k in ("ro", "U", "fib", "fstar", "feq"):
        assert _sha(getattr(st, k)) == bytes(g[f"sha_{k}"]).hex(), k
    got = np.array([*st.particle_pos, *st.particle_vel, *st.particle_force])
    np.testing.assert_array_equal(got, g["particle"])
    np.testing.assert_array_equal(np.array([st.particle_omega, st.particle_angle, st.particle_torque]), g["rotation"])
    assert res["sedimentation_history"] == json.loads(bytes(g["history_json"]).decode())
    assert res["final_step"] == int(g["final_step"][0])
    assert res["termination_reason"] == bytes(g["termination"]).decode()


@pytest.mark.parametrize("name", CASES)
def test_single_particle_runtime_on_the_device(torch, name):
    """The same runs with the disc stepped by the device particle step (forces
    summed over the band field, or over the markers under DFC, in numpy's order;
    the semi-implicit marker velocity from the half-kicked omega; the
    prescribed-velocity mode): the disc
    within 1e-12 relative of the reference's run (equal bits without rotation,
    whose device cos and sin may round differently from numpy's)."""
    from iblbm_b200 import run
    from iblbm_b200.config import SimConfig
    from iblbm_b200.engine import Engine
    g = dict(np.load(os.path.join(GOLD, f"sed1_{name}.npz")))
    kw = json.loads(bytes(g["config_json"]).decode())
    kw["cylinder_center"] = tuple(kw["cylinder_center"])
    if kw.get("prescribed_velocity") is not None:
        kw["prescribed_velocity"] = tuple(kw["prescribed_velocity"])
    cfg = SimConfig(**kw)
    eng = Engine(cfg, device_particles=True)
    assert eng.dev_particles
    res = run(cfg, verbose=False, engine=eng)
    st = res["state"]
    assert res["engine"].status() == 0
    got = np.array([*st.particle_pos, *st.particle_vel, *st.particle_force])
    rot = np.array([st.particle_omega, st.particle_angle, st.particle_torque])
    if not cfg.enable_rotation:
        np.testing.assert_array_equal(got, g["particle"])
        assert res["sedimentation_history"] == json.loads(bytes(g["history_json"]).decode())
    else:
        np.testing.assert_allclose(got, g["particle"], rtol=1e-12, atol=1e-12 * float(np.max(np.abs(g["particle"]))))
        np.testing.assert_allclose(rot, g["rotation"], rtol=1e-10, atol=0)
    assert res["final_step"] == int(g["final_step"][0])
