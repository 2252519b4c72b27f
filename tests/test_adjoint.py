"""Reverse-mode gradients of a rollout (numi_cloth_rollout_grad) against
central finite differences of the FP64 oracle in the kernels' batched order.

Scene: a small square cloth held by one corner on a moving, rotating grip,
no ground, no spheres (the smooth regime the adjoint differentiates
exactly).  Loss: squared distance of tracked particles to targets at two
frame ends.  Bar, against FP64 central differences (eps = 1e-4 on
log-compliances and on damping, 1e-6 m and 1e-6 rad on grip poses): each
group of gradients (material, grip pose) within 1e-3 relative in norm, and
every component within 1e-2 of its own size (components below 1e-3 of the
group's largest: within 1e-5 of the largest), since the FP32 state resolves
the smaller sensitivities only to a few 1e-4; the non-smooth counter at zero.
A second scene, the produce bag with its fruits removed, adds knots
(differentiated in forward mode) and the bag's six compliance groups.
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


def _fd(scene, cfg, tracked, targets, groups, grip_poses=True):
    """FP64 central differences of the oracle loss: per compliance group (all
    records of a family with the group's compliance scaled together), damping
    and grip poses."""
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
    osc0 = op.from_abi(scene)
    fams = {"distance": "distances", "knot": "knots", "bend": "bends", "grip": "grips"}
    out = {}
    for g, (fam, value) in enumerate(groups):
        arr = fams[fam]
        sel = getattr(osc0, arr)["compliance"] == np.float64(np.float32(value))
        out[g] = (loss_with((arr, sel, np.exp(eps))) - loss_with((arr, sel, np.exp(-eps)))) / (2 * eps)
    c = SCHED["damping"]
    out["damping"] = (loss_with(damping=c + eps) - loss_with(damping=c - eps)) / (2 * eps)
    grip = {}
    h = 1.0e-6
    for s in ((5, 17) if grip_poses else ()):
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
    return abs(a - b) <= 10.0 * REL * max(abs(b), 1e-3 * scale)


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
    assert [f for f, _ in r["groups"]] == ["distance", "distance", "bend", "grip"]   # stretch, shear
    fd, fd_grip = _fd(scene, cfg, tracked, targets, r["groups"])
    adj = {g: r["grads"][g] for g in range(len(r["groups"]))}
    adj["damping"] = r["damping"]
    print("adjoint vs FP64 central differences:", {k: (adj[k], fd[k]) for k in fd})
    print("grip pose:", {k: (r["grip"][k[0], k[1]], v) for k, v in fd_grip.items()})
    assert r["nonsmooth"] == 0
    assert _normwise([(adj[k], v) for k, v in fd.items()]) <= REL
    assert _normwise([(r["grip"][k[0], k[1]], v) for k, v in fd_grip.items()]) <= REL
    scale = max(abs(v) for v in fd.values())
    for k, v in fd.items():
        assert _close(adj[k], v, scale), (k, adj[k], v)
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
    assert np.allclose(out[0]["grads"], out[1]["grads"], rtol=1e-9, atol=1e-15)
    assert out[0]["damping"] == pytest.approx(out[1]["damping"], rel=1e-9)


def test_unsupported_schedule_rejected():
    scene = _scene()
    cfg = _configs(scene)
    sv = nc.ClothSolver(scene)
    with pytest.raises(nc.ClothError):
        sv.rollout_grad(cfg, nc.Schedule.make(**dict(SCHED, iterations=2)), np.array([0], np.uint32),
                        np.zeros((2, 1, 3)), LOSS_EVERY)


def _bag_without_fruits():
    """The produce bag hanging from its ten grips with the fruits removed, the
    ground off and the cloth centred on the origin; compliances raised so the
    constraint violations stay well above the FP32 position resolution."""
    m = nc.material_defaults()
    # compliances near m / (w dt^2): every projection moves its particles by
    # a fraction of the violation, so each group's sensitivity is well
    # resolved in FP32
    m.axialBodyComplianceMPerN = 6e-4
    m.axialCuffComplianceMPerN = 2e-4
    m.knotCompliance = 6e-4
    m.bendBodyComplianceMPerN = 1e-3
    m.bendCuffComplianceMPerN = 3e-4
    s = nc.bag_scene(material=m, scenario="recorded", timestep=1.0 / 5760.0)
    s.fruits = s.fruits[:0].copy()
    s.pairs = s.pairs[:0].copy()
    c = s.config
    c["constraintCounts"][:, 2] = 0   # ground off
    c["constraintCounts"][:, 3] = 0   # no fruits
    c["contactCounts"][:, 0] = 0
    c["contactCounts"][:, 1] = 0
    centre = s.particles["positionAndInverseMass"][:, :3].astype(np.float64).mean(axis=0)
    shift = centre.astype(np.float32)
    s.particles["positionAndInverseMass"][:, :3] -= shift
    s.particles["previousAndMass"][:, :3] -= shift
    s.rest[:, :3] -= shift
    s.rest64 = s.rest64 - shift.astype(np.float64)
    c["gripTargetAndActive"][:, :3] -= shift
    return s


def test_bag_knot_gradients_match_fp64_finite_differences():
    """Six compliance groups of the bag (axial body and cuff, knots, bend body
    and cuff, grips) and damping, knots differentiated by forward mode."""
    scene = _bag_without_fruits()
    cfg = _configs(scene)   # the ten grips move and turn together
    tracked, targets = _tracked_targets(scene, cfg)
    sv = nc.ClothSolver(scene)
    r = sv.rollout_grad(cfg, nc.Schedule.make(**SCHED), tracked, targets, LOSS_EVERY, checkpoint_every=8)
    sv.close()
    assert [f for f, _ in r["groups"]] == ["distance", "distance", "knot", "bend", "bend", "grip"]
    fd, _ = _fd(scene, cfg, tracked, targets, r["groups"], grip_poses=False)
    adj = {g: r["grads"][g] for g in range(len(r["groups"]))}
    adj["damping"] = r["damping"]
    print("bag adjoint vs FP64 central differences:", {k: (adj[k], fd[k]) for k in fd})
    assert r["nonsmooth"] == 0
    assert _normwise([(adj[k], v) for k, v in fd.items()]) <= REL
    scale = max(abs(v) for v in fd.values())
    for k, v in fd.items():
        assert _close(adj[k], v, scale), (k, adj[k], v)


def test_batched_gradients_equal_single_cloth_gradients():
    """The batched forward + adjoint (one launch per segment for all cloths,
    one CTA per cloth for the adjoint) gives each cloth the gradients of its
    own rollout."""
    scenes = [_scene(), small_square(side=9, fruits=0, gripCorners=1, stretchCompliance=3e-5, shearCompliance=4e-5,
                                     bendCompliance=1e-4, height=0.0, groundEnabled=0, seed=3), _bag_without_fruits()]
    cfgs = [_configs(s) for s in scenes]
    tracked = np.array([0, 5, 17, 40, 77], np.uint32)
    rng = np.random.default_rng(11)
    targets, singles = [], []
    for s, c in zip(scenes, cfgs):
        sv = nc.ClothSolver(s)
        x = sv.particles()["positionAndInverseMass"][tracked, :3].astype(np.float64)
        tg = np.stack([x + rng.uniform(-2e-3, 2e-3, size=x.shape) for _ in range(SUBSTEPS // LOSS_EVERY)])
        targets.append(tg)
        singles.append(sv.rollout_grad(c, nc.Schedule.make(**SCHED), tracked, tg, LOSS_EVERY, checkpoint_every=8))
        sv.close()
    solvers = [nc.ClothSolver(s) for s in scenes]
    batch = nc.ClothBatch(solvers)
    r = batch.rollout_grad(np.stack(cfgs), nc.Schedule.make(**SCHED), tracked, np.stack(targets), LOSS_EVERY,
                           checkpoint_every=8)
    for k, one in enumerate(singles):
        assert int(r["groups"][k]) == len(one["groups"])
        assert r["loss"][k] == pytest.approx(one["loss"], rel=1e-12)
        assert np.allclose(r["grads"][k], one["grads"], rtol=1e-10, atol=0.0)
        assert np.allclose(r["damping"][k], one["damping"], rtol=1e-10, atol=0.0)
        assert r["nonsmooth"][k] == one["nonsmooth"] == 0
    # the state after the call is the rollout's end state
    for sv, s, c in zip(solvers, scenes, cfgs):
        ref = nc.ClothSolver(s)
        ref.step(c, nc.Schedule.make(**SCHED))
        assert np.array_equal(sv.particles(), ref.particles())
    batch.close()
