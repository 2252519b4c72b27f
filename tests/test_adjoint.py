"""Reverse-mode gradients of a rollout (numi_cloth_rollout_grad) against
central finite differences of the FP64 oracle in the kernels' batched order.

Scene: a small square cloth held by one corner on a moving, rotating grip,
no ground, no spheres (the smooth regime the adjoint differentiates
exactly).  Loss: squared distance of tracked particles to targets at two
frame ends.  Bar, against FP64 central differences (eps = 1e-4 on
log-compliances and on damping, 1e-6 m and 1e-6 rad on grip poses): each
group of gradients (material, grip pose) within 1e-3 relative in norm, and
every component within 1e-3 of its own size or, for components below 1 % of
the group's largest, within 1e-5 of the largest (the FP32 state resolves
sensitivities that small only to that level); the non-smooth counter at zero.
"""
import numpy as np
import pytest

import numi_cloth as nc
import oracle_py as op
from helpers import small_square

pytestmark = pytest.mark.gpu

SUBSTEPS, LOSS_EVERY = 24, 12
SCHED = dict(iterations=1, strainSweeps=1, reconcilePasses=0, finalPasses=0, certificatePasses=0, earlyExit=0,
             aerodynamics=0, sweptGround=1, frictions=1, damping=0.8)
REL = 1.0e-3


def _scene():
    # Centred on the origin with the ground off: positions of a few cm keep
    # the FP32 state's resolution (an ulp of 4e-9 m rather than 6e-8 m at
    # 0.5 m) well below the constraint violations the compliance gradients
    # are made of.
    return small_square(side=12, fruits=0, gripCorners=1, stretchCompliance=2e-5, shearCompliance=5e-5,
                        bendCompliance=2e-4, height=0.0, groundEnabled=0)


def _configs(scene):
    cfg = nc.substep_configs(scene, SUBSTEPS)
    s = np.arange(1, SUBSTEPS + 1) / SUBSTEPS
    base = cfg["gripTargetAndActive"][:, :3].astype(np.float64)
    cfg["gripTargetAndActive"][:, 0] = (base[:, 0] + 0.004 * np.sin(2.0 * np.pi * s)).astype(np.float32)
    cfg["gripTargetAndActive"][:, 2] = (base[:, 2] + 0.006 * s).astype(np.float32)
    ang = 0.08 * s
    cfg["gripOrientation"][:, 0] = 0.0
    cfg["gripOrientation"][:, 1] = np.sin(ang / 2).astype(np.float32)
    cfg["gripOrientation"][:, 2] = 0.0
    cfg["gripOrientation"][:, 3] = np.cos(ang / 2).astype(np.float32)
    return cfg


def _tracked_targets(scene, cfg):
    rng = np.random.default_rng(7)
    tracked = np.sort(rng.choice(scene.n, 8, replace=False)).astype(np.uint32)
    sv = nc.ClothSolver(scene)
    tg = []
    for k in range(SUBSTEPS // LOSS_EVERY):
        sv.step(cfg[k * LOSS_EVERY:(k + 1) * LOSS_EVERY], nc.Schedule.make(**SCHED))
        x = sv.particles()["positionAndInverseMass"][tracked, :3].astype(np.float64)
        tg.append(x + rng.uniform(-1e-3, 1e-3, size=x.shape))
    sv.close()
    return tracked, np.stack(tg)


def _oracle_loss(osc, subs, osched, tracked, targets):
    o = op.Oracle(osc, 64)
    loss = 0.0
    for k in range(SUBSTEPS // LOSS_EVERY):
        o.step(subs[k * LOSS_EVERY:(k + 1) * LOSS_EVERY], osched)
        x = o.read()["particles"]["x"][tracked]
        loss += float(((x - targets[k]) ** 2).sum())
    return loss


def _qmul(a, b):
    """xyzw quaternion product a * b."""
    ax, ay, az, aw = a
    bx, by, bz, bw = b
    return np.array([aw * bx + ax * bw + ay * bz - az * by, aw * by - ax * bz + ay * bw + az * bx,
                     aw * bz + ax * by - ay * bx + az * bw, aw * bw - ax * bx - ay * by - az * bz])


def _fd(scene, cfg, tracked, targets):
    """FP64 central differences of the oracle loss."""
    base_sched = nc.Schedule.make(**SCHED)
    subs0 = op.substeps_from_configs(cfg)

    def loss_with(scale=None, damping=None, subs=None):
        osc = op.from_abi(scene)
        if scale is not None:
            fam, sel, f = scale
            arr = getattr(osc, fam)
            arr["compliance"][sel] = arr["compliance"][sel] * f
        osched = op.schedule_from_abi(base_sched, op.BATCHED)
        if damping is not None:
            osched.damping = damping
        return _oracle_loss(osc, subs0 if subs is None else subs, osched, tracked, targets)

    eps = 1.0e-4
    kinds = scene.distances["particlesAndColor"][:, 3]
    out = {}
    for name, fam, sel in (("log_c_warp", "distances", kinds == 0), ("log_c_weft", "distances", kinds == 1),
                           ("log_c_shear", "distances", kinds == 3),
                           ("log_c_bend", "bends", slice(None)), ("log_c_grip", "grips", slice(None))):
        out[name] = (loss_with((fam, sel, np.exp(eps))) - loss_with((fam, sel, np.exp(-eps)))) / (2 * eps)
    c = SCHED["damping"]
    out["damping"] = (loss_with(damping=c + eps) - loss_with(damping=c - eps)) / (2 * eps)
    grip = {}
    h = 1.0e-6
    for s in (5, 17):
        for axis in (0, 2):
            p, m = subs0.copy(), subs0.copy()
            p["grip_target"][s, axis] += h
            m["grip_target"][s, axis] -= h
            grip[(s, axis)] = (loss_with(subs=p) - loss_with(subs=m)) / (2 * h)
        # small rotation about y applied before the grip orientation
        p, m = subs0.copy(), subs0.copy()
        p["grip_q"][s] = _qmul(np.array([0.0, np.sin(h / 2), 0.0, np.cos(h / 2)]), subs0["grip_q"][s])
        m["grip_q"][s] = _qmul(np.array([0.0, -np.sin(h / 2), 0.0, np.cos(h / 2)]), subs0["grip_q"][s])
        grip[(s, 4)] = (loss_with(subs=p) - loss_with(subs=m)) / (2 * h)
    return out, grip


def _close(a, b, scale):
    return abs(a - b) <= REL * max(abs(b), 1e-2 * scale)


def _normwise(pairs):
    a = np.array([p[0] for p in pairs], np.float64)
    b = np.array([p[1] for p in pairs], np.float64)
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def test_rollout_gradients_match_fp64_finite_differences():
    scene = _scene()
    cfg = _configs(scene)
    tracked, targets = _tracked_targets(scene, cfg)
    sv = nc.ClothSolver(scene)
    r = sv.rollout_grad(cfg, nc.Schedule.make(**SCHED), tracked, targets, LOSS_EVERY, checkpoint_every=8)
    sv.close()
    fd, fd_grip = _fd(scene, cfg, tracked, targets)
    print("adjoint vs FP64 central differences:", {k: (r["grads"][k], fd[k]) for k in fd})
    print("grip pose:", {k: (r["grip"][k[0], k[1]], v) for k, v in fd_grip.items()})
    assert r["nonsmooth"] == 0
    assert _normwise([(r["grads"][k], v) for k, v in fd.items()]) <= REL
    assert _normwise([(r["grip"][k[0], k[1]], v) for k, v in fd_grip.items()]) <= REL
    scale = max(abs(v) for v in fd.values())
    for k, v in fd.items():
        assert _close(r["grads"][k], v, scale), (k, r["grads"][k], v)
    assert r["grads"]["log_c_bottom"] == 0.0   # no bottom records in a square cloth
    gscale = max(abs(v) for v in fd_grip.values())
    for (s, comp), v in fd_grip.items():
        assert _close(r["grip"][s, comp], v, gscale), (s, comp, r["grip"][s, comp], v)


def test_rollout_leaves_the_forward_state():
    scene = _scene()
    cfg = _configs(scene)
    tracked, targets = _tracked_targets(scene, cfg)
    a = nc.ClothSolver(scene)
    a.rollout_grad(cfg, nc.Schedule.make(**SCHED), tracked, targets, LOSS_EVERY, checkpoint_every=8)
    b = nc.ClothSolver(scene)
    for k in range(0, SUBSTEPS, 8):
        b.step(cfg[k:k + 8], nc.Schedule.make(**SCHED))
    assert np.array_equal(a.particles(), b.particles())


def test_checkpoint_interval_does_not_change_gradients():
    scene = _scene()
    cfg = _configs(scene)
    tracked, targets = _tracked_targets(scene, cfg)
    out = []
    for every in (4, 24):
        sv = nc.ClothSolver(scene)
        out.append(sv.rollout_grad(cfg, nc.Schedule.make(**SCHED), tracked, targets, LOSS_EVERY,
                                   checkpoint_every=every))
        sv.close()
    assert out[0]["loss"] == pytest.approx(out[1]["loss"], rel=1e-12)
    for k in out[0]["grads"]:
        assert out[0]["grads"][k] == pytest.approx(out[1]["grads"][k], rel=1e-9, abs=1e-15)


def test_unsupported_schedule_rejected():
    scene = _scene()
    cfg = _configs(scene)
    sv = nc.ClothSolver(scene)
    with pytest.raises(nc.ClothError):
        sv.rollout_grad(cfg, nc.Schedule.make(**dict(SCHED, iterations=2)), np.array([0], np.uint32),
                        np.zeros((2, 1, 3)), LOSS_EVERY)
