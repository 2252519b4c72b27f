"""The allocation-free entry point, numi_cloth_step_noalloc.

Some callers cannot let a library allocate GPU memory: hosts that own every
device byte through their own pool or arena, sized once at start-up, and
real-time loops where a cudaMalloc (which may synchronise the whole device)
is not allowed once they run.  For them the library steps caller-owned device
buffers and keeps its own scratch in one statically allocated device array.
This test owns the buffers (allocated through torch), calls the entry point
twice in a row through the C ABI and requires the same bits as the ordinary
handle-based path after each call, with the schedule's damping off and on.
It runs alone or after the other tests: every call clears the shared scratch
it needs zeroed.
"""
import numpy as np
import pytest

import numi_cloth as nc
from helpers import FULL, bag_frame_configs

pytestmark = pytest.mark.gpu


def _device_state(torch, scene):
    dev = torch.device("cuda", torch.cuda.current_device())

    def put(a, dtype=None):
        a = np.ascontiguousarray(a if dtype is None else a.astype(dtype))
        return torch.from_numpy(a.view(np.uint8).reshape(-1).copy()).to(dev)

    p = scene.particles
    d = scene.distances
    dm = d["material"].copy()
    lam = dm[:, 2].copy()
    dm[:, 2] = 0.0
    k = scene.knots
    b = scene.bends
    bij = np.zeros((len(b), 4), np.uint32)
    bij[:, :3] = b["particlesAndColor"][:, :3]
    bufs = {
        "positions": put(p["positionAndInverseMass"]),
        "previous": put(p["previousAndMass"]),
        "velocities": put(p["velocity"]),
        "rest": put(scene.rest),
        "distanceIJ": put(d["particlesAndColor"][:, :2]),
        "distanceMaterial": put(dm),
        "distanceLambda": put(lam),
        "knotIJ": put(k["particles"]),
        "knotMaterial": put(k["material"][:, :2]),
        "knotLambda": put(k["material"][:, 2]),
        "bendIJ": put(bij),
        "bendMaterial": put(b["material"][:, [0, 2]]),
        "bendLambda": put(b["material"][:, 3]),
        "grips": put(scene.grips),
        "fruits": put(scene.fruits),
        "fruitPairs": put(scene.pairs),
        "cuffParticles": put(scene.cuff),
        "failure": torch.zeros(4, dtype=torch.uint8, device=dev),
    }
    st = nc.abi.DeviceState()
    for name, t in bufs.items():
        setattr(st, name, t.data_ptr())
    return st, bufs


def _host(t, dtype, shape):
    return t.cpu().numpy().view(dtype).reshape(shape)


@pytest.mark.parametrize("damping", [0.0, 0.8])
def test_noalloc_matches_handle_path_two_calls(damping):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.set_device(0)
    torch.zeros(1, device="cuda")
    dt = 1.0 / 5760.0
    scene = nc.bag_scene(scenario="recorded", timestep=dt)
    sched = nc.Schedule.make(**dict(FULL, damping=damping))
    frames = [bag_frame_configs(scene, 0, 48, dt), bag_frame_configs(scene, 48, 48, dt)]

    ref = nc.ClothSolver(scene)
    st, bufs = _device_state(torch, scene)
    batches, counts = nc.colour_runs(scene)
    stream = torch.cuda.current_stream()
    undamped = None
    if damping != 0.0:
        # the same call without damping ends elsewhere: the damping is used
        flat = nc.ClothSolver(scene)
        flat.step(frames[0], nc.Schedule.make(**FULL))
        undamped = flat.particles()["positionAndInverseMass"].copy()
        flat.close()
    try:
        for k, cfg in enumerate(frames):
            ref.step(cfg, sched)
            assert ref.failure() == 0
            rc = nc.step_noalloc(scene, st, batches, counts, cfg, sched, stream.cuda_stream)
            assert rc == 0, rc
            torch.cuda.synchronize()
            assert int(_host(bufs["failure"], np.uint32, (1,))[0]) == 0
            rp = ref.particles()
            rf = ref.fruits()
            n = scene.n
            got = _host(bufs["positions"], np.float32, (n, 4))
            assert np.array_equal(got, rp["positionAndInverseMass"])
            assert np.array_equal(_host(bufs["velocities"], np.float32, (n, 4)), rp["velocity"])
            assert np.array_equal(_host(bufs["previous"], np.float32, (n, 4)), rp["previousAndMass"])
            got_f = _host(bufs["fruits"], nc.abi.FRUIT, (len(scene.fruits),))
            assert np.array_equal(got_f.view(np.uint8), rf.view(np.uint8))
            lam = _host(bufs["distanceLambda"], np.float32, (len(scene.distances),))
            assert np.array_equal(lam, ref.distances()["material"][:, 2])
            if k == 0 and undamped is not None:
                assert not np.array_equal(got, undamped)
    finally:
        ref.close()


def test_noalloc_rejects_run_past_records():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.set_device(0)
    torch.zeros(1, device="cuda")
    scene = nc.square_scene(side=12, fruitCount=1)
    st, bufs = _device_state(torch, scene)
    batches, counts = nc.colour_runs(scene)
    bad = batches.copy()
    bad[0, 1] = len(scene.distances) + 1   # the first distance run (first, count, colour, prefixes) reaches past D
    rc = nc.step_noalloc(scene, st, bad, counts, nc.substep_configs(scene, 1), nc.Schedule.make())
    assert rc == -1
    bad = batches.copy()
    bad[0, 3] = (int(bad[0, 1]) + 1) << 16   # strain-limited prefix longer than the run
    rc = nc.step_noalloc(scene, st, bad, counts, nc.substep_configs(scene, 1), nc.Schedule.make())
    assert rc == -1


def test_noalloc_rejects_oversize():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    scene = nc.square_scene(side=80, fruitCount=2)   # 6,400 particles > 4,096
    st = nc.abi.DeviceState()
    batches, counts = nc.colour_runs(scene)
    rc = nc.step_noalloc(scene, st, batches, counts, nc.substep_configs(scene, 1), nc.Schedule.make())
    assert rc == -1
