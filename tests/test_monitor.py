"""Sedimentation output files against the reference's own monitor callback on
the same synthetic sequence of states (fixtures: tests/golden/make_golden_monitor.py):
status.json (all keys but the wall-clock ``updated_at``), the history JSON,
the velocity snapshots and the final velocity field, equal."""
import json
import os

import numpy as np
import pytest

from tests.golden.make_golden_monitor import KINDS, PLOT_EVERY, SNAPSHOT_EVERY, config_kwargs, sequence

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _load(path):
    with open(path) as fh:
        return json.load(fh)


@pytest.mark.parametrize("kind", KINDS)
def test_sedimentation_outputs_match_reference(tmp_path, kind):
    from iblbm_b200.config import SimConfig
    from iblbm_b200.monitor import create_sedimentation_callback
    gold = os.path.join(HERE, f"monitor_{kind}")
    cfg = SimConfig(**config_kwargs(kind))
    out = str(tmp_path / kind)
    cb = create_sedimentation_callback(out, cfg, plot_every=PLOT_EVERY, snapshot_every=SNAPSHOT_EVERY)
    seq = sequence(kind)
    for step, st, elapsed in seq:
        cb(step=step, Cd=0.0, Cl=0.0, error=1.0, state=st, elapsed=elapsed, converged=False)
    cb.finalize(converged=False, final_state=seq[-1][1], final_step=seq[-1][0], termination_reason="max_steps")

    mine, ref = _load(os.path.join(out, "status.json")), _load(os.path.join(gold, "status.json"))
    mine.pop("updated_at")
    ref.pop("updated_at")
    assert mine == ref
    assert _load(os.path.join(out, "sedimentation_history.json")) == _load(
        os.path.join(gold, "sedimentation_history.json"))
    assert sorted(os.listdir(os.path.join(out, "snapshots"))) == sorted(os.listdir(os.path.join(gold, "snapshots")))
    files = [os.path.join("snapshots", f) for f in os.listdir(os.path.join(gold, "snapshots"))]
    for f in files + ["velocity_field.npz"]:
        a, b = np.load(os.path.join(out, f)), np.load(os.path.join(gold, f))
        assert sorted(a.files) == sorted(b.files), f
        for k in b.files:
            assert a[k].dtype == b[k].dtype, (f, k)
            np.testing.assert_array_equal(a[k], b[k], err_msg=f"{f}:{k}")


def test_history_written_on_schedule(tmp_path):
    """The history file exists after the first call (written at calls 1 and
    every PLOT_EVERY-th), before finalize."""
    from iblbm_b200.config import SimConfig
    from iblbm_b200.monitor import create_sedimentation_callback
    cfg = SimConfig(**config_kwargs("multi"))
    cb = create_sedimentation_callback(str(tmp_path), cfg, plot_every=PLOT_EVERY, snapshot_every=0)
    step, st, elapsed = sequence("multi")[0]
    cb(step=step, Cd=0.0, Cl=0.0, error=1.0, state=st, elapsed=elapsed, converged=False)
    assert len(_load(str(tmp_path / "sedimentation_history.json"))) == 1
    assert not (tmp_path / "snapshots").exists()


@pytest.mark.gpu
def test_monitor_on_a_sedimentation_run(tmp_path):
    """The callback on this package's run(): two settling discs (default form); one
    history record per check with both particles and the MDF statistics, and a
    completed status with the peak Reynolds numbers."""
    import torch
    assert torch.cuda.is_available()
    from iblbm_b200 import run
    from iblbm_b200.monitor import create_sedimentation_callback
    from tests.golden.make_golden import RUN_CASES
    from tests.test_gpu_f32 import _cfg
    cfg = _cfg(dict(RUN_CASES["c5_sed2_mdf_cmmrt_p4"]))
    cb = create_sedimentation_callback(str(tmp_path), cfg, snapshot_every=2)
    res = run(cfg, verbose=False, callback=cb)
    cb.finalize(converged=res["converged"], final_state=res["state"], final_step=res["final_step"],
                termination_reason=res["termination_reason"])
    hist = _load(str(tmp_path / "sedimentation_history.json"))
    status = _load(str(tmp_path / "status.json"))
    n_checks = res["final_step"] // cfg.check_interval
    assert len(hist) == n_checks == status["history_len"]
    assert all(len(r["particles"]) == 2 and "mdf_iter" in r for r in hist)
    assert status["completed"] and status["step"] == res["final_step"]
    assert status["mdf_iter_stats"]["n_steps"] == n_checks
    assert len(status["Re_standard_peaks"]) == 2
    for r, h in zip(hist, res["sedimentation_history"]):
        for p, q in zip(r["particles"], h["particles"]):
            assert (p["x"], p["y"]) == (q["x"], q["y"])
