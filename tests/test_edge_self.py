"""Edge/edge yarn self-collision and yarn/yarn self friction
(solvePrimitiveSelfCollision, applyClothSelfFriction and
measurePrimitiveSelfPenetration, tools/cloth_bag.cpp:3880-4247).

The oracle's serial order is pinned bit for bit to the compiled reference
(tests/test_oracle_pin.py).  The kernels run the same Gauss-Seidel sweep, a
segment's candidates in the reference's box-tree leaf order (the tree built
on the GPU from the pass-start boxes); the oracle's batched order is that
sweep, and the GPU must equal it bit for bit in FP32.
"""
import numpy as np
import pytest

import numi_cloth as nc
import oracle_py as op
from helpers import FULL, bag_frame_configs, gpu_positions, make_solver, per_substep_errors, run_oracle, small_square

POS_TOL_FP64 = 1.0e-5     # m: one FP32 substep vs the FP64 substep from the same state
ORDER_TOL_FP64 = 1.0e-5   # m: one FP64 substep, kernel order vs reference order
DT = 1.0 / 5760.0


def _bag(frames=1):
    scene = nc.bag_scene(scenario="recorded", timestep=DT)
    return scene, bag_frame_configs(scene, 0, 48 * frames, DT)


def _sched(**kw):
    args = dict(FULL)
    args.update(primitiveSelf=1)
    args.update(kw)
    return nc.Schedule.make(**args)


def crossing_square(side=20, lift=0.0009):
    """A square whose right half is folded over its left half and lowered
    onto it: the upper yarns cross the lower ones closer than the yarn
    diameter (2 mm), rows and columns far apart (not local)."""
    scene = small_square(side=side, fruits=0)
    pos = scene.particles["positionAndInverseMass"]
    half = side // 2
    for r in range(side):
        for c in range(half, side):
            i, j = r * side + c, r * side + (side - 1 - c)
            pos[i, 0] = pos[j, 0] + np.float32(0.0013)   # offset so yarns cross, not stack
            pos[i, 1] = pos[j, 1] + np.float32(0.0011)
            pos[i, 2] = pos[j, 2] + np.float32(lift)
    scene.particles["previousAndMass"][:, :3] = pos[:, :3]
    scene.particles["velocity"][:] = 0.0
    return scene


def _gpu(scene, cfg, sched, env=None, grid=None, frames=1):
    s = make_solver(scene, grid=grid, env=env)
    try:
        per = len(cfg) // frames
        for f in range(frames):
            s.step(cfg[f * per:(f + 1) * per], sched)
        return {"failure": s.failure(), "particles": s.particles(), "fruits": s.fruits(),
                "edge": s.edge_contacts(), "info": s.launch_info()}
    finally:
        s.close()


def _assert_same(g, o):
    gp = gpu_positions(g).astype(np.float64)
    assert np.array_equal(gp, o["particles"]["x"]), f"max |dx| = {np.abs(gp - o['particles']['x']).max():.3e}"
    gv = g["particles"]["velocity"][:, :3].astype(np.float64)
    assert np.array_equal(gv, o["particles"]["v"]), f"max |dv| = {np.abs(gv - o['particles']['v']).max():.3e}"
    if len(g["fruits"]):
        gf = g["fruits"]["positionAndInverseMass"][:, :3].astype(np.float64)
        assert np.array_equal(gf, o["fruits"]["x"])
    st = o["stats"]
    assert g["edge"] == (st["edge_contacts"], st["self_friction_contacts"]), (g["edge"], st)


# ----------------------------------------------------------------- CPU ----

def test_bag_family_is_active():
    """The authored bag starts with yarns closer than their diameter: the
    family acts from the first frame (the reference moves particles by
    millimetres with it, 2-16 mm over the golden runs)."""
    scene, cfg = _bag()
    o = run_oracle(scene, cfg, _sched(), bits=64)
    assert o["failure"] == 0
    assert o["stats"]["edge_contacts"] > 50 and o["stats"]["self_friction_contacts"] > 20


def test_kernel_order_against_reference_order_fp64():
    """Per substep from the reference-order trajectory: the kernels' order
    against the reference's.  The edge/edge pairs run in the reference's
    order (segment by segment, candidates in tree leaf order), so the two
    differ by the colour order of the constraint sweeps alone."""
    scene, cfg = _bag()
    subs = op.substeps_from_configs(cfg)
    ser = op.schedule_from_abi(_sched(), op.SERIAL)
    bat = op.schedule_from_abi(_sched(), op.BATCHED)
    ref = op.Oracle(op.from_abi(scene), 64)
    errs = []
    for k in range(len(cfg)):
        st = ref.read()
        probe = op.Oracle(op.from_abi(scene), 64)
        probe.write(st["particles"], st["fruits"], st["grips"])
        ref.step(subs[k:k + 1], ser)
        probe.step(subs[k:k + 1], bat)
        errs.append(np.abs(probe.read()["particles"]["x"] - ref.read()["particles"]["x"]).max())
    errs = np.array(errs)
    print(f"bag, kernel order vs reference order, per substep (FP64): max {errs.max():.3e} m")
    assert errs.max() <= ORDER_TOL_FP64


def test_crossing_layers_resolved_fp64():
    """Folded layers whose yarns cross closer than the yarn diameter make
    edge/edge contacts."""
    scene = crossing_square()
    cfg = nc.substep_configs(scene, 24)
    o = run_oracle(scene, cfg, _sched(), bits=64)
    assert o["failure"] == 0
    assert o["stats"]["edge_contacts"] > 0


# ----------------------------------------------------------------- GPU ----

@pytest.mark.gpu
def test_gpu_bag_bitexact_fp32():
    scene, cfg = _bag()
    s = _sched()
    g = _gpu(scene, cfg, s)
    assert g["failure"] == 0
    assert g["info"]["resident"] and g["info"]["cluster"] == (len(scene.particles) + 255) // 256
    _assert_same(g, run_oracle(scene, cfg, s, bits=32))
    print(f"bag, one frame with edge/edge self-collision: {g['edge'][0]} contacts, {g['edge'][1]} self-friction "
          f"contacts, bit-identical to the FP32 oracle")


@pytest.mark.gpu
def test_gpu_bag_two_frames_bitexact_fp32():
    scene, cfg = _bag(frames=2)
    s = _sched()
    g = _gpu(scene, cfg, s, frames=2)
    assert g["failure"] == 0
    _assert_same(g, run_oracle(scene, cfg, s, bits=32, frames=2))


@pytest.mark.gpu
def test_gpu_bag_per_substep_fp64():
    scene, cfg = _bag()
    errs, _ = per_substep_errors(scene, cfg, _sched())
    print(f"bag with edge/edge self-collision, per substep over the first frame: max particle error vs FP64 = "
          f"{errs.max():.3e} m")
    assert errs.max() <= POS_TOL_FP64


@pytest.mark.gpu
@pytest.mark.parametrize("cell", ["0.001", "10"])
def test_gpu_bag_list_paths(cell):
    """A tiny build cell makes every segment too long for the grid (all on
    the long-segment list); a huge one puts every segment in one cell.  The
    pair list, and so the result, is the same."""
    scene, cfg = _bag()
    s = _sched()
    g = _gpu(scene, cfg[:12], s, env={"NUMI_CLOTH_EDGE_CELL": cell})
    assert g["failure"] == 0
    _assert_same(g, run_oracle(scene, cfg[:12], s, bits=32))


@pytest.mark.gpu
@pytest.mark.parametrize("grid", [1, 5])
def test_gpu_crossing_layers_bitexact(grid):
    scene = crossing_square()
    cfg = nc.substep_configs(scene, 24)
    s = _sched()
    g = _gpu(scene, cfg, s, grid=grid)
    assert g["failure"] == 0
    assert g["edge"][0] > 0
    _assert_same(g, run_oracle(scene, cfg, s, bits=32))


@pytest.mark.gpu
def test_gpu_bag_cooperative_grid_equals_one_cta():
    """One CTA holding every particle, the default resident cluster and a
    cooperative grid over global memory give the same bits."""
    scene, cfg = _bag()
    s = _sched()
    a = _gpu(scene, cfg[:24], s, env={"NUMI_CLOTH_RESIDENT_CHUNK": "4096"})
    b = _gpu(scene, cfg[:24], s, grid=6)
    c = _gpu(scene, cfg[:24], s)
    assert a["failure"] == 0 and b["failure"] == 0 and c["failure"] == 0
    assert a["info"]["grid"] == 1 and b["info"]["grid"] == 6 and c["info"]["cluster"] > 1
    assert np.array_equal(gpu_positions(a), gpu_positions(c))
    assert a["edge"] == c["edge"]
    assert np.array_equal(gpu_positions(a), gpu_positions(b))
    assert a["edge"] == b["edge"]


@pytest.mark.gpu
def test_gpu_batch_equals_alone():
    scene, cfg = _bag()
    s = _sched()
    alone = _gpu(scene, cfg[:24], s)
    solvers = [nc.ClothSolver(scene) for _ in range(3)]
    batch = nc.ClothBatch(solvers)
    try:
        batch.step(np.stack([cfg[:24]] * 3), s)
        for sv in solvers:
            assert sv.failure() == 0
            assert np.array_equal(sv.particles()["positionAndInverseMass"], alone["particles"]["positionAndInverseMass"])
            assert sv.edge_contacts() == alone["edge"]
    finally:
        batch.close()
        for sv in solvers:
            sv.close()


@pytest.mark.gpu
def test_gpu_adjoint_rejects_edge_family():
    scene, cfg = _bag()
    sv = nc.ClothSolver(scene)
    try:
        with pytest.raises(Exception):
            sv.rollout_grad(cfg[:8], nc.Schedule.make(iterations=1, reconcilePasses=0, finalPasses=0,
                                                       certificatePasses=0, aerodynamics=0, primitiveSelf=1),
                            np.array([0], np.uint32), np.zeros((1, 1, 3)), 8)
    finally:
        sv.close()
