"""Gradient-based calibration (numi_cloth.calibrate): Adam on the bag's six
compliance groups and its damping, every candidate's forward + adjoint run
as one batch, recovers hidden parameters of a synthetic target trajectory."""
import numpy as np
import pytest

import numi_cloth as nc
from numi_cloth import calibrate as cal
from test_adjoint import _bag_without_fruits, _configs

pytestmark = pytest.mark.gpu

SCHED = dict(iterations=1, strainSweeps=1, reconcilePasses=0, finalPasses=0, certificatePasses=0, earlyExit=0,
             aerodynamics=0, sweptGround=1, frictions=1, damping=0.0)
LOSS_EVERY = 12


def _base_values(scene):
    m = nc.material_defaults()
    return np.array([6e-4, 2e-4, 6e-4, 1e-3, 3e-4, m.gripComplianceMPerN], np.float32)


def _targets(scene, cfg, tracked, values, damping):
    sv = nc.ClothSolver(scene)
    base = _base_values(scene)
    for p, (fam, _) in enumerate(cal.BAG_PARAMS):
        sv.replace_compliance(fam, float(base[p]), float(np.float32(values[p])))
    sv.set_damping(damping)
    out = []
    for k in range(len(cfg) // LOSS_EVERY):
        sv.step(cfg[k * LOSS_EVERY:(k + 1) * LOSS_EVERY], nc.Schedule.make(**SCHED))
        out.append(sv.particles()["positionAndInverseMass"][tracked, :3].astype(np.float64))
    sv.close()
    return np.stack(out)


def test_adam_on_batched_adjoint_recovers_hidden_parameters():
    scene = _bag_without_fruits()
    cfg = _configs(scene)
    base = _base_values(scene)
    tracked = np.concatenate([scene.cuff[::5], np.argsort(scene.particles["positionAndInverseMass"][:, 2])[:20]])
    tracked = np.unique(tracked).astype(np.uint32)
    rng = np.random.default_rng(5)
    hidden = base.astype(np.float64) * 10.0 ** rng.uniform(-0.3, 0.3, size=base.shape)
    hidden_damping = 0.5
    targets = _targets(scene, cfg, tracked, hidden, hidden_damping)
    n = 6
    logc0 = np.log(base.astype(np.float64))[None, :] + rng.uniform(-0.5, 0.5, size=(n, len(base)))
    d0 = rng.uniform(0.0, 1.0, size=n)
    c = cal.Calibration([scene] * n, cfg, nc.Schedule.make(**SCHED), tracked, targets, LOSS_EVERY, base)
    out = c.fit(logc0, d0, steps=50, lr=0.05, lr_damping=0.05)
    c.close()
    h = out["history"]
    print("best loss per step:", h.min(axis=1))
    best = int(np.argmin(out["loss"]))
    err = np.abs(out["logc"][best] - np.log(hidden))
    print("log-parameter error of the best candidate:", err, "damping", out["damping"][best], "hidden", hidden_damping)
    assert np.all(out["nonsmooth"] == 0)
    assert h[-1].min() < 0.1 * h[0].min()
    assert np.all(h[-1] < h[0])
