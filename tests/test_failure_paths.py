"""Failure paths of the boundary: the failure word and return codes the
reference's callers test (include/numi/cloth_bag_gpu.h:10-17), made on the
host or by a bounded wait that runs out; nothing here faults a GPU.

Create-time rejections run without a GPU (numi_cloth_create checks before it
touches the device); the rest are -m gpu tests.
"""
import os

import numpy as np
import pytest

import numi_cloth as nc
import oracle_py as op
from helpers import PLAIN, ROOT, make_solver, small_square

FIX = os.path.join(ROOT, "tests", "golden", "reference_fixtures")


def _create_rc(scene) -> int:
    with pytest.raises(nc.ClothError) as e:
        nc.ClothSolver(scene)
    return int(str(e.value).rsplit(" ", 1)[-1])


# ------------------------------------------------------------ create time
def test_create_rejects_wrong_abi_version():
    s = small_square(side=8, fruits=1)
    s.config["control"][0, 0] = 12
    assert _create_rc(s) == -1   # NUMI_CLOTH_EINVAL


def test_create_rejects_out_of_range_particle():
    s = small_square(side=8, fruits=1)
    s.distances["particlesAndColor"][5, 1] = s.n + 3
    assert _create_rc(s) == -1


def test_create_rejects_bend_middle_out_of_range():
    s = small_square(side=8, fruits=1)
    s.bends["particlesAndColor"][0, 1] = s.n
    assert _create_rc(s) == -1


def test_create_rejects_colour_conflict():
    """Two distances of one colour that share a particle: EBATCH, the
    reference host's verifyColoring (tools/cloth_bag_metal.mm:1705-1819)."""
    s = small_square(side=8, fruits=1)
    d = s.distances["particlesAndColor"]
    first = np.flatnonzero(d[:, 2] == d[0, 2])
    a, b = first[0], first[1]
    d[b, 0] = d[a, 0] if d[a, 0] != d[b, 1] else d[a, 1]
    assert _create_rc(s) == -3   # NUMI_CLOTH_EBATCH


def test_create_rejects_degenerate_distance():
    s = small_square(side=8, fruits=1)
    s.distances["particlesAndColor"][3, 1] = s.distances["particlesAndColor"][3, 0]
    assert _create_rc(s) in (-1, -3)


def test_create_rejects_duplicate_grip_particle():
    s = small_square(side=8, fruits=1)
    if len(s.grips) < 2:
        pytest.skip("needs two grips")
    s.grips["particle"][1, 0] = s.grips["particle"][0, 0]
    assert _create_rc(s) == -3


def test_distant_regrab_trajectories_load():
    """The loader accepts them: the reference rejects them only when the
    re-grab happens (tools/cloth_bag.cpp:1584-1588)."""
    for name in ("invalid-distant-regrab.csv", "invalid-distant-patch-regrab.csv"):
        nc.GripTrajectory(os.path.join(FIX, name))


# ------------------------------------------------------------- on the GPU
def _cuda(torch=None):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.set_device(0)
    torch.zeros(1, device="cuda")
    return torch


@pytest.mark.gpu
@pytest.mark.parametrize("name,nearest", [("invalid-distant-regrab.csv", 0),
                                          ("invalid-distant-patch-regrab.csv", 1)])
def test_distant_regrab_sets_grip_capture(name, nearest):
    """A re-grab 1 m from the cuff: GRIP_CAPTURE on the GPU, as in both
    oracles (FP32 batched order and FP64 reference order)."""
    _cuda()
    dt = 1.0 / 120.0 / 24.0
    scene = nc.bag_scene(scenario="recorded", timestep=dt, select_nearest=bool(nearest))
    traj = nc.GripTrajectory(os.path.join(FIX, name))
    cfg = traj.configs(scene.config, scene.handle_base, 0, 24, dt)
    sched = nc.Schedule.make(**PLAIN)
    sv = nc.ClothSolver(scene)
    sv.step(cfg, sched)
    fail = sv.failure()
    sv.close()
    assert fail & nc.abi.FAILURE_GRIP_CAPTURE, nc.failure_names(fail)
    for bits, mode in ((32, op.BATCHED), (64, op.SERIAL)):
        o = op.Oracle(op.from_abi(scene), bits)
        ofail = o.step(op.substeps_from_configs(cfg), op.schedule_from_abi(sched, mode))
        assert ofail & nc.abi.FAILURE_GRIP_CAPTURE


@pytest.mark.gpu
def test_bounded_barrier_wait_runs_out():
    """Every grid barrier waits for one CTA that does not exist (a test hook,
    NUMI_CLOTH_TEST_MISSING_CTA): the bounded wait gives up, the launch ends
    with TIMEOUT instead of hanging, and the device stays usable."""
    torch = _cuda()
    scene = small_square(side=24, fruits=2)
    cfg = nc.substep_configs(scene, 4)
    sched = nc.Schedule.make(**PLAIN)
    sv = make_solver(scene, grid=2, env={"NUMI_CLOTH_TEST_MISSING_CTA": 1, "NUMI_CLOTH_WAIT_LIMIT": 20000})
    assert sv.launch_info()["grid"] == 2
    sv.step(cfg, sched)
    fail = sv.failure()
    sv.close()
    assert fail & nc.abi.FAILURE_TIMEOUT, nc.failure_names(fail)
    # the context still works: the same cloth without the hook steps cleanly
    ok = make_solver(scene, grid=2)
    ok.step(cfg, sched)
    assert ok.failure() == 0
    ok.close()
    torch.cuda.synchronize()


@pytest.mark.gpu
def test_nan_particle_sets_nonfinite():
    _cuda()
    scene = small_square(side=16, fruits=1)
    sv = nc.ClothSolver(scene)
    p = sv.particles()
    p["positionAndInverseMass"][37, 0] = np.nan
    sv.write_particles(p)
    sv.step(nc.substep_configs(scene, 2), nc.Schedule.make(**PLAIN))
    fail = sv.failure()
    sv.close()
    assert fail & nc.abi.FAILURE_NONFINITE, nc.failure_names(fail)


@pytest.mark.gpu
def test_invalid_config_reported_and_nothing_runs():
    """validConfig (ClothBag.metal:16-55): a non-finite timestep sets
    NONFINITE on the host and the state is not touched."""
    _cuda()
    scene = small_square(side=12, fruits=1)
    sv = nc.ClothSolver(scene)
    before = sv.particles().copy()
    cfg = nc.substep_configs(scene, 2)
    cfg["gravityAndTimestep"][1, 3] = np.inf
    sv.step(cfg, nc.Schedule.make(**PLAIN))
    fail = sv.failure()
    after = sv.particles()
    sv.close()
    assert fail & nc.abi.FAILURE_NONFINITE
    assert np.array_equal(before.view(np.uint8), after.view(np.uint8))
