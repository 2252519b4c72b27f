"""Batched stepping: many independent cloths in one persistent launch give
the same bits as stepping each cloth alone, under every launch shape, and as
a replayed CUDA graph."""
import numpy as np
import pytest

import numi_cloth as nc
from helpers import FULL, PLAIN, run_oracle, small_square

pytestmark = pytest.mark.gpu


def _scenes():
    """Cloths of uneven sizes, as the batched square-cloth workload has."""
    out = []
    for k, (side, fruits) in enumerate([(40, 3), (16, 1), (33, 8), (24, 2), (57, 4), (20, 0), (48, 6)]):
        out.append(small_square(side=side, fruits=fruits, seed=100 + k))
    return out


def _configs(scenes, substeps, first=0):
    cfg = [nc.substep_configs(s, first + substeps)[first:] for s in scenes]
    return np.stack(cfg)


def _alone(scenes, cfg, sched, frames=1):
    out = []
    for s, c in zip(scenes, cfg):
        sv = nc.ClothSolver(s)
        for _ in range(frames):
            sv.step(c, sched)
        out.append((sv.particles(), sv.fruits(), sv.failure()))
        sv.close()
    return out


def _batched(scenes, cfg, sched, frames=1, shape=None):
    solvers = [nc.ClothSolver(s) for s in scenes]
    batch = nc.ClothBatch(solvers)
    if shape is not None:
        batch.set_shape(*shape)
    for _ in range(frames):
        batch.step(cfg, sched)
    out = [(sv.particles(), sv.fruits(), sv.failure()) for sv in solvers]
    batch.close()
    for sv in solvers:
        sv.close()
    return out


@pytest.mark.parametrize("shape", [(0, 256), (1024, 256), (4096, 512)], ids=["global", "resident1k", "resident4k-512"])
def test_batch_equals_alone(shape):
    scenes = _scenes()
    cfg = _configs(scenes, 12)
    sched = nc.Schedule.make(**FULL)
    a = _alone(scenes, cfg, sched)
    b = _batched(scenes, cfg, sched, shape=shape)
    for (pa, fa, xa), (pb, fb, xb) in zip(a, b):
        assert xa == 0 and xb == 0
        assert np.array_equal(pa, pb)
        assert np.array_equal(fa, fb)


def test_batch_member_equals_oracle():
    scenes = _scenes()[:3]
    cfg = _configs(scenes, 8)
    sched = nc.Schedule.make(**PLAIN)
    b = _batched(scenes, cfg, sched)
    o = run_oracle(scenes[2], cfg[2], sched, bits=32)
    gp = b[2][0]["positionAndInverseMass"][:, :3].astype(np.float64)
    assert np.array_equal(gp, o["particles"]["x"])


def test_batch_tune_keeps_state_and_bits():
    scenes = _scenes()
    cfg = _configs(scenes, 6)
    sched = nc.Schedule.make(**FULL)
    a = _alone(scenes, cfg, sched)
    solvers = [nc.ClothSolver(s) for s in scenes]
    batch = nc.ClothBatch(solvers)
    shape = batch.tune(cfg, sched)
    assert shape["threads"] in (256, 512) and shape["ctas"] >= 1
    batch.step(cfg, sched)
    for sv, (pa, fa, _) in zip(solvers, a):
        assert np.array_equal(sv.particles(), pa)
        assert np.array_equal(sv.fruits(), fa)
    batch.close()


def test_batch_graph_replay_equals_steps():
    import torch
    scenes = _scenes()
    sched = nc.Schedule.make(**FULL)
    cfg0, cfg1 = _configs(scenes, 6, 0), _configs(scenes, 6, 6)
    a = _batched(scenes, np.concatenate([cfg0, cfg1], axis=1)[:, :6], sched)   # warm the comparison path
    solvers = [nc.ClothSolver(s) for s in scenes]
    ref = [nc.ClothSolver(s) for s in scenes]
    rb = nc.ClothBatch(ref)
    rb.step(cfg0, sched)
    rb.step(cfg1, sched)
    batch = nc.ClothBatch(solvers)
    pinned = torch.empty(cfg0.nbytes, dtype=torch.uint8, pin_memory=True)
    pinned.numpy()[:] = np.frombuffer(cfg0.tobytes(), np.uint8)
    batch.capture(pinned, 6, sched)
    batch.replay()
    torch.cuda.synchronize()
    pinned.numpy()[:] = np.frombuffer(cfg1.tobytes(), np.uint8)
    batch.replay()
    for sv, rv in zip(solvers, ref):
        assert np.array_equal(sv.particles(), rv.particles())
        assert np.array_equal(sv.fruits(), rv.fruits())
    assert a is not None
    batch.close()
    rb.close()


def test_per_cloth_damping_equals_schedule_damping():
    scene = small_square(side=24, fruits=2)
    cfg = nc.substep_configs(scene, 8)
    a = nc.ClothSolver(scene)
    a.step(cfg, nc.Schedule.make(**dict(PLAIN, damping=40.0)))
    b = nc.ClothSolver(scene)
    b.set_damping(40.0)
    b.step(cfg, nc.Schedule.make(**PLAIN))
    c = nc.ClothSolver(scene)
    c.step(cfg, nc.Schedule.make(**PLAIN))
    assert np.array_equal(a.particles(), b.particles())
    assert not np.array_equal(a.particles(), c.particles())
