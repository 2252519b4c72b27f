"""GPU parity: the sm_100a frame kernel against the CPU oracle.

Bar: on the same inputs and the same batched colour schedule the FP32 GPU
path equals the FP32 restatement bit for bit; every substep of the first
frame, started from the FP64 trajectory's state, lands within 1e-5 m of the
FP64 restatement (the error accumulated over a whole frame of contact is
stated and bounded by 1e-4 m); two GPU runs are bit-identical; one CTA and
many CTAs give the same bits.
"""
import numpy as np
import pytest

import numi_cloth as nc
import oracle_py as op
from helpers import (FULL, PLAIN, bag_frame_configs, gpu_fruit_positions, gpu_positions, per_substep_errors, run_gpu,
                     run_oracle, small_square)

pytestmark = pytest.mark.gpu

POS_TOL_FP64 = 1.0e-5   # m: one FP32 substep vs the FP64 substep from the same state
FRAME_TOL_FP64 = 1.0e-4  # m: accumulated over a whole frame of contact (stated, chaotic growth)


def _check_bitexact(g, o):
    gp = gpu_positions(g)
    opos = o["particles"]["x"]
    assert np.array_equal(gp.astype(np.float64), opos), f"max |dx| = {np.abs(gp - opos).max()}"
    gv = g["particles"]["velocity"][:, :3].astype(np.float64)
    assert np.array_equal(gv, o["particles"]["v"]), f"max |dv| = {np.abs(gv - o['particles']['v']).max()}"
    if len(g["fruits"]):
        gf = gpu_fruit_positions(g).astype(np.float64)
        assert np.array_equal(gf, o["fruits"]["x"]), f"fruit max |dx| = {np.abs(gf - o['fruits']['x']).max()}"
        assert np.array_equal(g["fruits"]["velocityAndGroundImpulse"][:, :3].astype(np.float64), o["fruits"]["v"])
        assert np.array_equal(g["fruits"]["angularVelocity"][:, :3].astype(np.float64), o["fruits"]["omega"])
    lam = g["distances"]["material"][:, 2].astype(np.float64)
    assert np.array_equal(lam, o["distances"]["lambda_"])


@pytest.mark.parametrize("sched", [PLAIN, FULL], ids=["plain", "full"])
def test_square_frame_bitexact_fp32(sched):
    scene = small_square()
    cfg = nc.substep_configs(scene, 48)
    s = nc.Schedule.make(**sched)
    g = run_gpu(scene, cfg, s)
    o = run_oracle(scene, cfg, s, bits=32)
    assert g["failure"] == 0, nc.failure_names(g["failure"])
    _check_bitexact(g, o)


def test_square_per_substep_fp64_tolerance():
    scene = small_square()
    cfg = nc.substep_configs(scene, 48)
    s = nc.Schedule.make(**FULL)
    errs, ferrs = per_substep_errors(scene, cfg, s)
    print(f"square 24x24, per substep over the first frame: max particle error vs FP64 = {errs.max():.3e} m, "
          f"fruit = {ferrs.max():.3e} m")
    assert errs.max() <= POS_TOL_FP64
    assert ferrs.max() <= POS_TOL_FP64


def test_square_frame_fp64_accumulated():
    scene = small_square()
    cfg = nc.substep_configs(scene, 48)
    s = nc.Schedule.make(**FULL)
    g = run_gpu(scene, cfg, s)
    o = run_oracle(scene, cfg, s, bits=64)
    err = np.abs(gpu_positions(g).astype(np.float64) - o["particles"]["x"]).max()
    ferr = np.abs(gpu_fruit_positions(g).astype(np.float64) - o["fruits"]["x"]).max()
    print(f"square 24x24, one frame accumulated: max particle error vs FP64 = {err:.3e} m, fruit = {ferr:.3e} m")
    assert err <= FRAME_TOL_FP64
    assert ferr <= FRAME_TOL_FP64


def test_bag_frame_bitexact_and_fp64():
    dt = 1.0 / 5760.0
    scene = nc.bag_scene(scenario="recorded", timestep=dt)
    cfg = bag_frame_configs(scene, 0, 48, dt)
    s = nc.Schedule.make(**FULL)
    g = run_gpu(scene, cfg, s)
    # resident cluster path: 256 particles in the shared memory of each CTA
    n = len(scene.particles)
    assert g["info"]["resident"] and g["info"]["grid"] == (n + 255) // 256 == g["info"]["cluster"]
    o32 = run_oracle(scene, cfg, s, bits=32)
    _check_bitexact(g, o32)
    o64 = run_oracle(scene, cfg, s, bits=64)
    err = np.abs(gpu_positions(g).astype(np.float64) - o64["particles"]["x"]).max()
    print(f"bag, 1 frame at 1/5760 s accumulated: max particle error vs FP64 = {err:.3e} m")
    assert err <= FRAME_TOL_FP64
    errs, _ = per_substep_errors(scene, cfg, s)
    print(f"bag, per substep over the first frame: max particle error vs FP64 = {errs.max():.3e} m")
    assert errs.max() <= POS_TOL_FP64


def test_multi_cta_equals_single_cta():
    scene = small_square(side=32, fruits=8)
    cfg = nc.substep_configs(scene, 12)
    s = nc.Schedule.make(**FULL)
    one = run_gpu(scene, cfg, s, grid=1)
    many = run_gpu(scene, cfg, s, grid=7)
    assert many["info"]["grid"] == 7
    assert np.array_equal(one["particles"], many["particles"])
    assert np.array_equal(one["fruits"], many["fruits"])


def test_cluster_equals_cooperative_grid():
    """One thread-block cluster (hardware cluster barrier) and the
    cooperative grid (global-memory barrier) give the same bits."""
    scene = small_square(side=96, fruits=16)
    cfg = nc.substep_configs(scene, 12)
    s = nc.Schedule.make(**FULL)
    grid = run_gpu(scene, cfg, s, env={"NUMI_CLOTH_CLUSTER": "0", "NUMI_CLOTH_RESIDENT": "0"})
    clus = run_gpu(scene, cfg, s, env={"NUMI_CLOTH_CLUSTER": "16", "NUMI_CLOTH_RESIDENT": "0"})
    assert grid["info"]["grid"] > 16 and not grid["info"]["resident"]
    assert clus["info"]["grid"] in (8, 16) and clus["info"]["cluster"] == clus["info"]["grid"]
    assert np.array_equal(grid["particles"], clus["particles"])
    assert np.array_equal(grid["fruits"], clus["fruits"])
    o = run_oracle(scene, cfg, s, bits=32)
    _check_bitexact(clus, o)


@pytest.mark.parametrize("side,ranks,chunk", [(40, 1, "4096"), (40, 7, None), (60, 15, "256"), (96, 3, None),
                                              (128, 4, None)])
def test_resident_equals_global(side, ranks, chunk):
    """Particles resident in the shared memory of one CTA or spread over a
    cluster's distributed shared memory give the same bits as particles in
    global memory, and as the oracle."""
    scene = small_square(side=side, fruits=12)
    cfg = nc.substep_configs(scene, 12)
    s = nc.Schedule.make(**FULL)
    env = {"NUMI_CLOTH_RESIDENT": "1" if side * side <= 4096 else "2"}
    if chunk:
        env["NUMI_CLOTH_RESIDENT_CHUNK"] = chunk
    res = run_gpu(scene, cfg, s, env=env)
    glob = run_gpu(scene, cfg, s, env={"NUMI_CLOTH_RESIDENT": "0"})
    assert res["info"]["resident"] and res["info"]["grid"] == ranks
    assert not glob["info"]["resident"]
    assert res["failure"] == 0
    assert np.array_equal(res["particles"], glob["particles"])
    assert np.array_equal(res["fruits"], glob["fruits"])
    assert np.array_equal(res["distances"], glob["distances"])
    o = run_oracle(scene, cfg, s, bits=32)
    _check_bitexact(res, o)


@pytest.mark.parametrize("side,grid", [(96, 0), (64, 37)])
def test_neighbour_syncs_equal_grid_barriers(side, grid):
    """Colours separated by neighbour syncs (each CTA waits only for the
    CTAs that share a particle with it) give the grid barrier's bits, and
    the oracle's."""
    scene = small_square(side=side, fruits=12)
    cfg = nc.substep_configs(scene, 24)
    s = nc.Schedule.make(**dict(FULL, strainSweeps=2, selfCollision=1))
    env = {"NUMI_CLOTH_RESIDENT": "0"}
    if grid:
        env["NUMI_CLOTH_GRID"] = str(grid)
    nbr = run_gpu(scene, cfg, s, env=env)
    bar = run_gpu(scene, cfg, s, env=dict(env, NUMI_CLOTH_NEIGHBOUR_SYNC="0"))
    assert nbr["info"]["grid"] > 1 and nbr["failure"] == 0 and bar["failure"] == 0
    assert nbr["info"]["neighbour_syncs"] and not bar["info"]["neighbour_syncs"]
    assert np.array_equal(nbr["particles"], bar["particles"])
    assert np.array_equal(nbr["fruits"], bar["fruits"])
    assert np.array_equal(nbr["distances"], bar["distances"])
    _check_bitexact(nbr, run_oracle(scene, cfg, s, bits=32))


def test_bag_neighbour_syncs_bitexact():
    """The produce bag (knots, bends, 12 fruits, grips, self contact) on a
    cooperative grid with neighbour syncs between its colours gives the
    one-CTA run's bits and the oracle's."""
    dt = 1.0 / 5760.0
    scene = nc.bag_scene(scenario="recorded", timestep=dt)
    cfg = bag_frame_configs(scene, 0, 24, dt)
    s = nc.Schedule.make(**dict(FULL, selfCollision=1))
    many = run_gpu(scene, cfg, s, env={"NUMI_CLOTH_GRID": "6", "NUMI_CLOTH_RESIDENT": "0"})
    one = run_gpu(scene, cfg, s)
    assert many["info"]["grid"] == 6 and many["info"]["neighbour_syncs"]
    assert many["failure"] == 0 and one["failure"] == 0
    assert np.array_equal(many["particles"], one["particles"])
    assert np.array_equal(many["fruits"], one["fruits"])
    _check_bitexact(many, run_oracle(scene, cfg, s, bits=32))


def test_patch_regrab_multi_cta_bitexact():
    """The reference's patch-regrab fixture (three grip generations, each
    re-attaching to the cuff particles nearest the grip target) on one CTA
    and on a cooperative grid: the attach reads the positions the previous
    substep left, on every launch shape, and the result is the oracle's."""
    import os

    traj = nc.GripTrajectory(os.path.join(os.path.dirname(__file__), "golden", "reference_fixtures",
                                          "synthetic-patch-regrab.csv"))
    assert traj.select_nearest
    dt = (1.0 / 120.0) / 24
    scene = nc.bag_scene(scenario="recorded", timestep=dt, select_nearest=True)
    cfg = traj.configs(scene.config, scene.handle_base, 0, 24, dt)
    s = nc.Schedule.make(**FULL)
    one = run_gpu(scene, cfg, s)
    many = run_gpu(scene, cfg, s, env={"NUMI_CLOTH_GRID": "6", "NUMI_CLOTH_RESIDENT": "0"})
    assert many["info"]["grid"] == 6 and one["failure"] == 0 and many["failure"] == 0
    assert np.array_equal(one["grips"], many["grips"])
    assert np.array_equal(one["particles"], many["particles"])
    o = run_oracle(scene, cfg, s, bits=32)
    _check_bitexact(many, o)
    _check_bitexact(one, o)


def test_two_runs_bit_identical():
    scene = small_square(side=40, fruits=10)
    cfg = nc.substep_configs(scene, 24)
    s = nc.Schedule.make(**FULL)
    a = run_gpu(scene, cfg, s, grid=16)
    b = run_gpu(scene, cfg, s, grid=16)
    assert np.array_equal(a["particles"], b["particles"])
    assert np.array_equal(a["fruits"], b["fruits"])


@pytest.mark.parametrize("resident", ["2", "0"], ids=["resident-cluster", "global-grid"])
def test_large_square_multi_cta_bitexact(resident):
    """65,536 particles, three substeps: a 16-CTA cluster holding the
    particles in distributed shared memory, and the full cooperative grid."""
    scene = nc.square_scene()
    cfg = nc.substep_configs(scene, 3)
    s = nc.Schedule.make(**PLAIN)
    g = run_gpu(scene, cfg, s, env={"NUMI_CLOTH_RESIDENT": resident})
    assert g["info"]["grid"] > 1
    assert g["info"]["resident"] == (resident == "2")
    o = run_oracle(scene, cfg, s, bits=32)
    assert g["failure"] == 0
    _check_bitexact(g, o)


def _fast_fruits(side=24, fruits=6):
    """Spheres a few mm above the cloth moving down at 6 m/s: 2 mm per substep,
    so the swept (continuous) fruit/yarn test finds the impacts."""
    scene = small_square(side=side, fruits=fruits)
    scene.fruits["velocityAndGroundImpulse"][:, 2] = -6.0
    return scene


@pytest.mark.parametrize("sched", [PLAIN, FULL], ids=["plain", "full"])
def test_swept_fruit_yarn_bitexact_fp32(sched):
    """The swept fruit/yarn phase (solveSweptBallYarn, batched order) gives the
    FP32 oracle's bits, and it changes the result (the impacts are found)."""
    scene = _fast_fruits()
    cfg = nc.substep_configs(scene, 12)
    s = nc.Schedule.make(**dict(sched, sweptFruitYarn=1))
    g = run_gpu(scene, cfg, s)
    o = run_oracle(scene, cfg, s, bits=32)
    assert g["failure"] == 0, nc.failure_names(g["failure"])
    _check_bitexact(g, o)
    plain = run_gpu(scene, cfg, nc.Schedule.make(**dict(sched, sweptFruitYarn=0)))
    assert not np.array_equal(plain["particles"], g["particles"])


def test_swept_fruit_yarn_launch_modes():
    scene = _fast_fruits(side=40, fruits=10)
    cfg = nc.substep_configs(scene, 8)
    s = nc.Schedule.make(**dict(FULL, sweptFruitYarn=1))
    a = run_gpu(scene, cfg, s, env={"NUMI_CLOTH_RESIDENT": "0"})
    b = run_gpu(scene, cfg, s, grid=6)
    c = run_gpu(scene, cfg, s)
    assert np.array_equal(a["particles"], b["particles"]) and np.array_equal(a["particles"], c["particles"])
    assert np.array_equal(a["fruits"], c["fruits"])
