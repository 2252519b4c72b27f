"""The differentiable rollout at its stated size: a 64 x 64 cloth (4,096
particles, 4 mm) with a 3 x 3 corner patch on a seeded 6-DoF grip trajectory
(translation at most 5 cm, rotation at most 15 degrees), ground and 4
spheres, 96 substeps at 1/2880 s, checkpoints every 8 substeps, the loss over
32 seeded tracked particles against a target trajectory made at
log-compliances shifted by N(0, 0.3) (tests/helpers.py config3_*).

The adjoint differentiates the FP32 trajectory the GPU ran.  That trajectory
is within about 1.3e-6 m of the FP64 one, and the loss residuals are about
1e-3 m; the gradient error that this alone causes, estimated on the CPU from
the FP32 and FP64 oracles and FP64 Jacobians, is about 1e-4 (material and
damping) and 3e-4 (grip pose) norm-wise, inside the 1e-3 bar.

The adjoint's gradients with respect to the compliance groups (stretch,
shear, bend, grip), the damping and the grip pose are compared with
central finite differences (eps = 1e-4 on log-compliances and damping,
1e-6 m and 1e-6 rad on grip poses) of the FP64 oracle in the reference's
serial order, and in the kernels' batched order; bar 1e-3 relative in norm
per group.  The spheres start above the cloth and meet nothing in these 96
substeps, and neither does the ground, so the rollout is smooth (no
non-smooth events counted) and the adjoint differentiates all of it.
"""
import numpy as np
import pytest

import numi_cloth as nc
import oracle_py as op
from helpers import (CONFIG3_LOSS_EVERY, CONFIG3_SCHED, CONFIG3_SUBSTEPS, config3_configs, config3_scene,
                     config3_targets)
from test_adjoint import _normwise, _qmul

pytestmark = pytest.mark.gpu
REL = 1.0e-3


def _loss(osc, subs, osched, tracked, targets):
    o = op.Oracle(osc, 64)
    loss = 0.0
    for k in range(CONFIG3_SUBSTEPS // CONFIG3_LOSS_EVERY):
        o.step(subs[k * CONFIG3_LOSS_EVERY:(k + 1) * CONFIG3_LOSS_EVERY], osched)
        x = o.read()["particles"]["x"][tracked]
        loss += float(((x - targets[k]) ** 2).sum())
    return loss, o.stats()


def _fd(scene, cfg, tracked, targets, groups, mode):
    subs0 = op.substeps_from_configs(cfg)
    sched = nc.Schedule.make(**CONFIG3_SCHED)

    def run(scale=None, damping=None, subs=None):
        osc = op.from_abi(scene)
        if scale is not None:
            fam, sel, f = scale
            getattr(osc, fam)["compliance"][sel] *= f
        osched = op.schedule_from_abi(sched, mode)
        if damping is not None:
            osched.damping = damping
        return _loss(osc, subs0 if subs is None else subs, osched, tracked, targets)[0]

    eps = 1.0e-4
    osc0 = op.from_abi(scene)
    fams = {"distance": "distances", "bend": "bends", "grip": "grips"}
    out = {}
    for g, (fam, value) in enumerate(groups):
        arr = fams[fam]
        sel = getattr(osc0, arr)["compliance"] == np.float64(np.float32(value))
        out[g] = (run((arr, sel, np.exp(eps))) - run((arr, sel, np.exp(-eps)))) / (2 * eps)
    c = CONFIG3_SCHED["damping"]
    out["damping"] = (run(damping=c + eps) - run(damping=c - eps)) / (2 * eps)
    grip = {}
    h = 1.0e-6
    for s in (20, 61):
        for axis in (0, 2):
            p, m = subs0.copy(), subs0.copy()
            p["grip_target"][s, axis] += h
            m["grip_target"][s, axis] -= h
            grip[(s, axis)] = (run(subs=p) - run(subs=m)) / (2 * h)
        p, m = subs0.copy(), subs0.copy()
        p["grip_q"][s] = _qmul(np.array([0.0, np.sin(h / 2), 0.0, np.cos(h / 2)]), subs0["grip_q"][s])
        m["grip_q"][s] = _qmul(np.array([0.0, -np.sin(h / 2), 0.0, np.cos(h / 2)]), subs0["grip_q"][s])
        grip[(s, 4)] = (run(subs=p) - run(subs=m)) / (2 * h)
    return out, grip


def test_config3_gradients_match_fp64_finite_differences():
    scene = config3_scene()
    cfg = config3_configs(scene)
    tracked, targets, stats = config3_targets(scene, cfg)
    assert stats["yarn_contacts"] == 0 and stats["self_contacts"] == 0
    sv = nc.ClothSolver(scene)
    r = sv.rollout_grad(cfg, nc.Schedule.make(**CONFIG3_SCHED), tracked, targets, CONFIG3_LOSS_EVERY,
                        checkpoint_every=8)
    sv.close()
    assert [f for f, _ in r["groups"]] == ["distance", "distance", "bend", "grip"]
    assert r["nonsmooth"] == 0
    adj = {g: r["grads"][g] for g in range(len(r["groups"]))}
    adj["damping"] = r["damping"]
    for mode, name in ((op.SERIAL, "reference order"), (op.BATCHED, "batched order")):
        fd, fd_grip = _fd(scene, cfg, tracked, targets, r["groups"], mode)
        e_mat = _normwise([(adj[k], v) for k, v in fd.items()])
        e_grip = _normwise([(r["grip"][k[0], k[1]], v) for k, v in fd_grip.items()])
        print(f"config 3, FP64 central differences in the {name}: material + damping {e_mat:.2e}, grip pose "
              f"{e_grip:.2e} relative;", {k: (adj[k], fd[k]) for k in fd})
        assert e_mat <= REL
        assert e_grip <= REL
