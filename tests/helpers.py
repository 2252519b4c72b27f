"""Shared scene/schedule builders and runners for the parity tests."""
from __future__ import annotations

import os

import numpy as np

import numi_cloth as nc
import oracle_py as op

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")

# Point self contact in the reference's Gauss-Seidel order (the frame
# kernels with the ordered pass), and its oracle order.
SELF_REFERENCE = {"NUMI_CLOTH_SELF_ORDER": "reference"}

# Schedules exercised by the parity tests.  "reference" is the reference
# CPU substep (tools/cloth_bag.cpp:4891-5185) with a reduced certificate cap.
FULL = dict(iterations=2, strainSweeps=3, reconcilePasses=3, finalPasses=2, certificatePasses=4, earlyExit=1,
            aerodynamics=1, sweptGround=1, frictions=1)
PLAIN = dict(iterations=1, strainSweeps=1, reconcilePasses=0, finalPasses=0, certificatePasses=0, earlyExit=0,
             aerodynamics=0, sweptGround=1, frictions=1)


def small_square(side=24, fruits=6, **kw) -> nc.SceneArrays:
    """A small square cloth with spheres resting just above it."""
    args = dict(side=side, fruitCount=fruits, fruitHeightMin=0.5012, fruitHeightMax=0.5030, fruitRadiusMin=0.01,
                fruitRadiusMax=0.02, timestep=1.0 / 2880.0)
    args.update(kw)
    return nc.square_scene(**args)


def lift_trajectory_path() -> str:
    return os.path.join(GOLDEN, "lift-v1.csv")


def bag_frame_configs(scene: nc.SceneArrays, first: int, count: int, dt: float) -> np.ndarray:
    traj = nc.GripTrajectory(lift_trajectory_path())
    return traj.configs(scene.config, scene.handle_base, first, count, dt)


def make_solver(scene, grid=None, env=None):
    """A solver created under temporary launch-policy environment variables."""
    env = dict(env or {})
    if grid is not None:
        env["NUMI_CLOTH_GRID"] = str(grid)
    old = {k: os.environ.get(k) for k in env}
    os.environ.update({k: str(v) for k, v in env.items()})
    try:
        return nc.ClothSolver(scene)
    finally:
        for k, v in old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v


def run_gpu(scene, configs, sched: nc.Schedule, frames=1, grid=None, env=None):
    s = make_solver(scene, grid, env)
    per = len(configs) // frames
    for f in range(frames):
        s.step(configs[f * per:(f + 1) * per], sched)
    fail = s.failure()
    out = {"particles": s.particles(), "fruits": s.fruits(), "distances": s.distances(), "grips": s.grips(),
           "failure": fail, "residuals": s.residuals(), "info": s.launch_info(), "self_contacts": s.self_contacts(),
           "release": s.release_masks()}
    s.close()
    return out


def run_oracle(scene, configs, sched: nc.Schedule, bits=32, mode=op.BATCHED, frames=1):
    o = op.Oracle(op.from_abi(scene), bits)
    subs = op.substeps_from_configs(configs)
    osched = op.schedule_from_abi(sched, mode)
    per = len(configs) // frames
    fail = 0
    for f in range(frames):
        fail |= o.step(subs[f * per:(f + 1) * per], osched)
    st = o.read()
    st["failure"] = fail
    st["residuals"] = o.residuals()
    st["stats"] = o.stats()
    return st


def gpu_positions(out) -> np.ndarray:
    return out["particles"]["positionAndInverseMass"][:, :3]


def gpu_fruit_positions(out) -> np.ndarray:
    return out["fruits"]["positionAndInverseMass"][:, :3]


def oracle_state_to_abi(scene, st):
    """GPU particle/fruit records (FP32) from an oracle state (FP64)."""
    P = scene.particles.copy()
    p = st["particles"]
    P["positionAndInverseMass"][:, :3] = p["x"]
    P["positionAndInverseMass"][:, 3] = p["w"]
    P["previousAndMass"][:, :3] = p["prev"]
    P["previousAndMass"][:, 3] = p["mass"]
    P["velocity"][:, :3] = p["v"]
    P["velocity"][:, 3] = p["vw"]
    F = scene.fruits.copy()
    f = st["fruits"]
    if len(F):
        F["positionAndInverseMass"][:, :3] = f["x"]
        F["previousAndRadius"][:, :3] = f["prev"]
        F["velocityAndGroundImpulse"][:, :3] = f["v"]
        F["velocityAndGroundImpulse"][:, 3] = f["ground_impulse"]
        F["angularVelocity"][:, :3] = f["omega"]
        F["orientation"] = f["q"]
    return P, F


def per_substep_errors(scene, configs, sched, mode=op.BATCHED, env=None):
    """Max particle / fruit position error of one GPU substep started from
    the FP64 trajectory's state (rounded to FP32), for every substep.  mode:
    the FP64 oracle's order, BATCHED (the kernels' order) or SERIAL (the
    reference's order); env: launch-policy variables of the GPU solver."""
    o = op.Oracle(op.from_abi(scene), 64)
    subs = op.substeps_from_configs(configs)
    osched = op.schedule_from_abi(sched, mode)
    s = make_solver(scene, env=env)
    errs, ferrs = [], []
    try:
        for k in range(len(configs)):
            st = o.read()
            P, F = oracle_state_to_abi(scene, st)
            s.write_particles(P)
            if len(F):
                s.write_fruits(F)
            s.step(configs[k:k + 1], sched)
            o.step(subs[k:k + 1], osched)
            nxt = o.read()
            errs.append(float(np.abs(s.particles()["positionAndInverseMass"][:, :3].astype(np.float64)
                                     - nxt["particles"]["x"]).max()))
            if len(F):
                ferrs.append(float(np.abs(s.fruits()["positionAndInverseMass"][:, :3].astype(np.float64)
                                          - nxt["fruits"]["x"]).max()))
        assert s.failure() == 0
    finally:
        s.close()
    return np.array(errs), np.array(ferrs) if ferrs else np.zeros(1)


# ---------------------------------------------------------------- config 3
# The differentiable rollout's scene and grip trajectory are the benchmark's
# (bench.py); the target trajectory here comes from the FP64 oracle.
from bench import (CONFIG3_LOSS_EVERY, CONFIG3_SCHED, CONFIG3_SUBSTEPS, CONFIG3_TRACKED,  # noqa: E402
                   config3_configs, config3_scene)


def config3_targets(scene: nc.SceneArrays, cfg: np.ndarray, seed: int = 3):
    """32 seeded tracked particles and their target trajectory: the FP64
    oracle (reference order) at log-compliances shifted by N(0, 0.3)."""
    rng = np.random.default_rng(seed)
    tracked = np.sort(rng.choice(scene.n, CONFIG3_TRACKED, replace=False)).astype(np.uint32)
    shift = np.exp(rng.normal(0.0, 0.3, size=3))
    osc = op.from_abi(scene)
    kinds = osc.distances["kind"]
    osc.distances["compliance"][kinds != 3] *= shift[0]
    osc.distances["compliance"][kinds == 3] *= shift[1]
    osc.bends["compliance"] *= shift[2]
    o = op.Oracle(osc, 64)
    subs = op.substeps_from_configs(cfg)
    osched = op.schedule_from_abi(nc.Schedule.make(**CONFIG3_SCHED), op.SERIAL)
    out = []
    for k in range(CONFIG3_SUBSTEPS // CONFIG3_LOSS_EVERY):
        o.step(subs[k * CONFIG3_LOSS_EVERY:(k + 1) * CONFIG3_LOSS_EVERY], osched)
        out.append(o.read()["particles"]["x"][tracked].copy())
    return tracked, np.stack(out), o.stats()
