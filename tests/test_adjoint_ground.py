"""Reverse-mode gradients through ground contact (numi_cloth_rollout_grad)
against central finite differences of the FP64 oracle in the kernels'
batched order.

Scene: a 16 x 16 cloth (4 mm) lying on the ground (the ground clamp at the
yarn radius), one corner on a grip that drags it 1 cm sideways, lifts it
4 mm and turns it 0.05 rad over 48 substeps.  Most particles stay on the
ground and stick; those the grip pulls slide (cloth/ground Coulomb
friction, tools/cloth_bag.cpp:2076) or lift off; bends meet the ground
active set, the step fraction and the ground clamp (cloth_bag.cpp:1782-1863),
and predict meets the swept ground clamp (cloth_bag.cpp:2692-2721).  The
adjoint differentiates each along the branches the forward took, so the
non-smooth counter stays at zero.  Bar, as for the airborne cloth: each
group of gradients (material + damping, grip pose) within 1e-3 relative in
norm.  The FP64 loss is smooth at the finite-difference step (central
differences at 3e-5, 1e-4 and 3e-4 agree to 3e-5), and the FP32 trajectory
is within 1.5e-8 m of the FP64 one.
"""
import numpy as np
import pytest

import numi_cloth as nc
import oracle_py as op
from helpers import small_square
from test_adjoint import _normwise, _qmul

pytestmark = pytest.mark.gpu

SUBSTEPS, LOSS_EVERY = 48, 12
SCHED = dict(iterations=1, strainSweeps=1, reconcilePasses=0, finalPasses=0, certificatePasses=0, earlyExit=0,
             aerodynamics=0, sweptGround=1, frictions=1, damping=0.8)
REL = 1.0e-3
RADIUS = 0.001   # the square scene's yarn radius: the ground clamp height


def _scene():
    return small_square(side=16, fruits=0, gripCorners=1, stretchCompliance=1e-4, shearCompliance=2e-4,
                        bendCompliance=1e-3, height=RADIUS, groundEnabled=1, spacing=0.004)


def _configs(scene):
    cfg = nc.substep_configs(scene, SUBSTEPS)
    s = np.arange(1, SUBSTEPS + 1) / SUBSTEPS
    base = cfg["gripTargetAndActive"][:, :3].astype(np.float64)
    cfg["gripTargetAndActive"][:, 0] = (base[:, 0] - 0.010 * s).astype(np.float32)
    cfg["gripTargetAndActive"][:, 2] = (base[:, 2] + 0.004 * s).astype(np.float32)
    ang = 0.05 * s
    cfg["gripOrientation"][:, 1] = np.sin(ang / 2).astype(np.float32)
    cfg["gripOrientation"][:, 3] = np.cos(ang / 2).astype(np.float32)
    return cfg


def _oracle(osc, subs, osched, tracked, targets=None):
    o = op.Oracle(osc, 64)
    xs = []
    for k in range(SUBSTEPS // LOSS_EVERY):
        o.step(subs[k * LOSS_EVERY:(k + 1) * LOSS_EVERY], osched)
        xs.append(o.read()["particles"]["x"][tracked].copy())
    xs = np.stack(xs)
    if targets is None:
        return xs, o.read()["particles"]["x"]
    return float(((xs - targets) ** 2).sum())


def _targets(scene, cfg):
    rng = np.random.default_rng(7)
    tracked = np.sort(rng.choice(scene.n, 12, replace=False)).astype(np.uint32)
    osched = op.schedule_from_abi(nc.Schedule.make(**SCHED), op.BATCHED)
    xs, final = _oracle(op.from_abi(scene), op.substeps_from_configs(cfg), osched, tracked)
    return tracked, xs + rng.uniform(-1e-3, 1e-3, size=xs.shape), final


def _fd(scene, cfg, tracked, targets, groups):
    subs0 = op.substeps_from_configs(cfg)
    sched = nc.Schedule.make(**SCHED)

    def loss(scale=None, damping=None, subs=None):
        osc = op.from_abi(scene)
        if scale is not None:
            fam, sel, f = scale
            getattr(osc, fam)["compliance"][sel] *= f
        osched = op.schedule_from_abi(sched, op.BATCHED)
        if damping is not None:
            osched.damping = damping
        return _oracle(osc, subs0 if subs is None else subs, osched, tracked, targets)

    eps = 1.0e-4
    osc0 = op.from_abi(scene)
    fams = {"distance": "distances", "bend": "bends", "grip": "grips"}
    out = {}
    for g, (fam, value) in enumerate(groups):
        arr = fams[fam]
        sel = getattr(osc0, arr)["compliance"] == np.float64(np.float32(value))
        out[g] = (loss((arr, sel, np.exp(eps))) - loss((arr, sel, np.exp(-eps)))) / (2 * eps)
    c = SCHED["damping"]
    out["damping"] = (loss(damping=c + eps) - loss(damping=c - eps)) / (2 * eps)
    grip = {}
    h = 1.0e-6
    for s in (10, 37):
        for axis in (0, 2):
            p, m = subs0.copy(), subs0.copy()
            p["grip_target"][s, axis] += h
            m["grip_target"][s, axis] -= h
            grip[(s, axis)] = (loss(subs=p) - loss(subs=m)) / (2 * h)
        p, m = subs0.copy(), subs0.copy()
        p["grip_q"][s] = _qmul(np.array([0.0, np.sin(h / 2), 0.0, np.cos(h / 2)]), subs0["grip_q"][s])
        m["grip_q"][s] = _qmul(np.array([0.0, -np.sin(h / 2), 0.0, np.cos(h / 2)]), subs0["grip_q"][s])
        grip[(s, 4)] = (loss(subs=p) - loss(subs=m)) / (2 * h)
    return out, grip


def test_ground_contact_scene_touches_the_ground():
    """Most of the cloth ends on the ground and the grip has lifted its
    corner off it."""
    scene = _scene()
    _, _, final = _targets(scene, _configs(scene))
    on = final[:, 2] <= RADIUS + 1e-6
    assert on.sum() > scene.n // 2 and final[:, 2].max() > RADIUS + 2e-3


def test_ground_contact_gradients_match_fp64_finite_differences():
    scene = _scene()
    cfg = _configs(scene)
    tracked, targets, _ = _targets(scene, cfg)
    sv = nc.ClothSolver(scene)
    r = sv.rollout_grad(cfg, nc.Schedule.make(**SCHED), tracked, targets, LOSS_EVERY, checkpoint_every=8)
    sv.close()
    assert [f for f, _ in r["groups"]] == ["distance", "distance", "bend", "grip"]
    assert r["nonsmooth"] == 0
    adj = {g: r["grads"][g] for g in range(len(r["groups"]))}
    adj["damping"] = r["damping"]
    fd, fd_grip = _fd(scene, cfg, tracked, targets, r["groups"])
    e_mat = _normwise([(adj[k], v) for k, v in fd.items()])
    e_grip = _normwise([(r["grip"][k[0], k[1]], v) for k, v in fd_grip.items()])
    print(f"ground contact, FP64 central differences: material + damping {e_mat:.2e}, grip pose {e_grip:.2e} "
          f"relative;", {k: (adj[k], fd[k]) for k in fd})
    assert e_mat <= REL
    assert e_grip <= REL
