"""Point/point self contact (tools/cloth_bag.cpp:4249-4315): the oracle's
two pass orders, and the GPU hash grid against them.

The default kernels run the batched order: every non-local pair closer than
2r at the start of the pass, each particle's summed corrections applied
once.  Where every particle is in at most one pair the reference's
Gauss-Seidel pass and the batched pass make the same moves, bit for bit in
FP64; where particles have several partners they differ (stated below).
The kernels built with the ordered pass (NUMI_CLOTH_SELF_ORDER=reference)
keep the reference's Gauss-Seidel order everywhere: phase A resolves
isolated pairs in parallel, one CTA resolves the coupled particles'
listed pairs in the reference's order (wavefronts, else serially), and a
serial pass over the whole cloth backs both up; they are bit-identical to
the FP32 oracle in that order.
"""
import numpy as np
import pytest

import numi_cloth as nc
import oracle_py as op
from helpers import (FULL, SELF_REFERENCE, gpu_positions, make_solver, per_substep_errors, run_gpu, run_oracle,
                     small_square)


POS_TOL_FP64 = 1.0e-5   # m: one FP32 substep vs the FP64 reference-order substep from the same state
FIRST_DEEP_SUBSTEP_STATED = 2.0e-4   # m: the offset fold's first substep (1.05e-4 measured), stated

def folded_square(side=24, gap=0.0015, fruits=0):
    """A square folded in half over its middle row: the upper layer lies
    `gap` above the lower one, so every upper particle is within 2r = 2 mm of
    the lower particle under it (rows more than two apart: not local)."""
    scene = small_square(side=side, fruits=fruits)
    pos = scene.particles["positionAndInverseMass"]
    prev = scene.particles["previousAndMass"]
    half = side // 2
    for r in range(half, side):
        mirror = side - 1 - r
        for c in range(side):
            i, j = r * side + c, mirror * side + c
            pos[i, 0], pos[i, 1] = pos[j, 0], pos[j, 1]
            pos[i, 2] = pos[j, 2] + np.float32(gap)
    prev[:, :3] = pos[:, :3]
    scene.particles["velocity"][:] = 0.0
    return scene


def _oracle(scene, bits):
    return op.Oracle(op.from_abi(scene), bits)


def test_isolated_pairs_batched_equals_serial_fp64():
    """Isolated overlapping pairs: the batched pass moves every particle
    exactly as the reference's serial pass does."""
    scene = small_square(side=24, fruits=0)
    pos = scene.particles["positionAndInverseMass"]
    side = 24
    # five far-apart pairs, each particle 1.2-1.8 mm above another one
    for k, (src, dst) in enumerate([(30, 200), (60, 330), (100, 460), (140, 520), (170, 560)]):
        pos[dst, :3] = pos[src, :3] + np.array([0.0002 * k, -0.0001, 0.0012 + 0.00015 * k], np.float32)
        assert abs(src // side - dst // side) > 2
    a, b = _oracle(scene, 64), _oracle(scene, 64)
    pen_a = a.self_pass(serial=True)
    pen_b = b.self_pass(serial=False)
    assert pen_a == pen_b and pen_a > 0.0
    xa, xb = a.read()["particles"]["x"], b.read()["particles"]["x"]
    assert np.array_equal(xa, xb)
    moved = np.flatnonzero(np.any(xa != pos[:, :3].astype(np.float64), axis=1))
    assert len(moved) == 10
    assert a.stats()["self_contacts"] == b.stats()["self_contacts"] == 5


def test_batched_pass_separates_folded_layers():
    """On a folded cloth one batched pass resolves every overlapping pair
    (each particle has exactly one partner across the fold), and both orders
    find the same pairs."""
    scene = folded_square()
    o_ser, o_bat = _oracle(scene, 64), _oracle(scene, 64)
    pen_s = o_ser.self_pass(serial=True)
    pen_b = o_bat.self_pass(serial=False)
    assert pen_b == pytest.approx(0.0005, rel=1e-3) and pen_s == pen_b
    assert o_bat.stats()["self_contacts"] == o_ser.stats()["self_contacts"] > 0
    x = o_bat.read()["particles"]["x"]
    side, half = 24, 12
    up = np.array([r * side + c for r in range(half + 3, side) for c in range(side)])
    lo = np.array([(side - 1 - r) * side + c for r in range(half + 3, side) for c in range(side)])
    gaps = np.linalg.norm(x[up] - x[lo], axis=1)
    # pairs whose particles carry no other contact end exactly 2r apart
    assert np.all(gaps >= 0.002 - 1e-9)


def offset_folded_square(side=24, spacing=0.0015, gap=0.001, shift=0.5):
    """A dense square (1.5 mm spacing) folded over its middle row with the
    upper layer shifted half a spacing along both axes and lowered to `gap`
    above the lower one: every upper particle is within 2r of the four lower
    particles around it (up to four partners each)."""
    scene = small_square(side=side, fruits=0, spacing=spacing)
    pos = scene.particles["positionAndInverseMass"]
    half = side // 2
    for r in range(half, side):
        mirror = side - 1 - r
        for c in range(side):
            i, j = r * side + c, mirror * side + c
            pos[i, 0] = pos[j, 0] + np.float32(shift * spacing)
            pos[i, 1] = pos[j, 1] + np.float32(shift * spacing)
            pos[i, 2] = pos[j, 2] + np.float32(gap)
    scene.particles["previousAndMass"][:, :3] = pos[:, :3]
    scene.particles["velocity"][:] = 0.0
    return scene


MULTI_PARTNER_STATED = 5.0e-4   # m: the measured gap, stated (3.4e-4 on this fold)


def test_multi_partner_contacts_batched_vs_serial_fp64():
    """Where particles have several partners the batched (Jacobi) pass and
    the reference's Gauss-Seidel pass differ: one FP64 pass and one FP64
    substep from the same state on the offset fold (987 contacts, up to
    four partners per particle) differ by 3.4e-4 m.  Stated, not within the
    1e-5 m bar; on the benchmark scenes (the bag, the 256x256 cloth's first
    frame) every particle has at most one partner and the orders agree
    (tests/test_headline_parity.py, tests/test_gpu_parity.py), and the
    reference-order kernels remove the gap (tests below)."""
    scene = offset_folded_square()
    a, b = _oracle(scene, 64), _oracle(scene, 64)
    a.self_pass(serial=True)
    b.self_pass(serial=False)
    assert a.stats()["self_contacts"] == b.stats()["self_contacts"] > 900
    one_pass = np.abs(a.read()["particles"]["x"] - b.read()["particles"]["x"]).max()
    cfg = nc.substep_configs(scene, 1)
    sched = nc.Schedule.make(**dict(FULL, selfCollision=1))
    subs = op.substeps_from_configs(cfg)
    s_ser, s_bat = _oracle(scene, 64), _oracle(scene, 64)
    s_ser.step(subs, op.schedule_from_abi(sched, op.SERIAL))
    s_bat.step(subs, op.schedule_from_abi(sched, op.BATCHED))
    substep = np.abs(s_ser.read()["particles"]["x"] - s_bat.read()["particles"]["x"]).max()
    print(f"offset fold, batched vs reference order (FP64): one pass {one_pass:.3e} m, one substep {substep:.3e} m")
    assert 0.0 < one_pass <= MULTI_PARTNER_STATED and 0.0 < substep <= MULTI_PARTNER_STATED


@pytest.mark.gpu
def test_gpu_self_contact_bitexact_fp32():
    """The hash-grid kernel phases give the FP32 batched oracle's bits over
    a frame with the folded cloth, and the same contact count."""
    scene = folded_square(fruits=4)
    cfg = nc.substep_configs(scene, 12)
    s = nc.Schedule.make(**dict(FULL, selfCollision=1))
    solver_out = run_gpu(scene, cfg, s)
    o = run_oracle(scene, cfg, s, bits=32)
    assert solver_out["failure"] == 0, nc.failure_names(solver_out["failure"])
    gp = gpu_positions(solver_out).astype(np.float64)
    assert np.array_equal(gp, o["particles"]["x"]), f"max |dx| = {np.abs(gp - o['particles']['x']).max()}"
    assert np.array_equal(solver_out["particles"]["velocity"][:, :3].astype(np.float64), o["particles"]["v"])
    assert solver_out["self_contacts"][0] == o["stats"]["self_contacts"] > 0


@pytest.mark.gpu
@pytest.mark.parametrize("resident", ["0", "1"], ids=["global", "resident"])
def test_gpu_self_contact_launch_modes(resident):
    """Same bits with particles in global memory and resident in shared
    memory, and from a multi-CTA cooperative grid."""
    scene = folded_square(side=32)
    cfg = nc.substep_configs(scene, 6)
    s = nc.Schedule.make(**dict(FULL, selfCollision=1))
    a = run_gpu(scene, cfg, s, env={"NUMI_CLOTH_RESIDENT": resident})
    b = run_gpu(scene, cfg, s, grid=5)
    assert a["failure"] == 0 and b["failure"] == 0
    assert np.array_equal(a["particles"], b["particles"])


@pytest.mark.gpu
def test_gpu_self_contact_full_buckets_use_the_overflow_list():
    """A cloth squeezed into a couple of hash cells (far more particles per
    cell than a bucket holds): the overflow list keeps every particle, the
    pass stays bit-identical to the oracle and raises no failure."""
    scene = small_square(side=10, fruits=0)
    pos = scene.particles["positionAndInverseMass"]
    centre = pos[:, :3].mean(axis=0)
    pos[:, 0] = centre[0] + (pos[:, 0] - centre[0]) * np.float32(0.05)
    pos[:, 1] = centre[1] + (pos[:, 1] - centre[1]) * np.float32(0.05)
    scene.particles["previousAndMass"][:, :3] = pos[:, :3]
    cfg = nc.substep_configs(scene, 2)
    s = nc.Schedule.make(**dict(FULL, selfCollision=1))
    g = run_gpu(scene, cfg, s)
    o = run_oracle(scene, cfg, s, bits=32)
    assert g["failure"] == 0, nc.failure_names(g["failure"])
    assert np.array_equal(gpu_positions(g).astype(np.float64), o["particles"]["x"])
    assert g["self_contacts"][0] == o["stats"]["self_contacts"] > 100


def test_offset_fold_fp64_orders_agree():
    """One FP64 substep of the offset fold (every family on, point self
    contact in both iterations) in the reference-order kernels' order and in
    the reference's order: the same bits."""
    scene = offset_folded_square()
    cfg = nc.substep_configs(scene, 1)
    sched = nc.Schedule.make(**dict(FULL, selfCollision=1))
    subs = op.substeps_from_configs(cfg)
    ser, bat = _oracle(scene, 64), _oracle(scene, 64)
    ser.step(subs, op.schedule_from_abi(sched, op.SERIAL))
    bat.step(subs, op.schedule_from_abi(sched, op.BATCHED_SELF_REFERENCE))
    assert np.array_equal(ser.read()["particles"]["x"], bat.read()["particles"]["x"])
    assert ser.stats()["self_contacts"] == bat.stats()["self_contacts"] > 900


@pytest.mark.gpu
@pytest.mark.parametrize("launch", ["one-cta", "grid", "resident"])
def test_gpu_multi_partner_fold_bitexact_fp32(launch):
    """Reference-order kernels, up to four partners per particle: phase A
    lists the coupled particles and the ordered pass resolves them in the
    reference's order; the GPU gives the FP32 oracle's bits (the reference's
    Gauss-Seidel pass in FP32) and the same contact count, on one CTA, a
    cooperative grid and a resident cluster."""
    scene = offset_folded_square()
    cfg = nc.substep_configs(scene, 12)
    s = nc.Schedule.make(**dict(FULL, selfCollision=1))
    kw = {"one-cta": dict(grid=1, env=dict(SELF_REFERENCE, NUMI_CLOTH_RESIDENT="0")),
          "grid": dict(grid=6, env=SELF_REFERENCE),
          "resident": dict(env=dict(SELF_REFERENCE, NUMI_CLOTH_RESIDENT="1"))}[launch]
    g = run_gpu(scene, cfg, s, **kw)
    assert g["info"]["self_order_reference"]
    o = run_oracle(scene, cfg, s, bits=32, mode=op.BATCHED_SELF_REFERENCE)
    assert g["failure"] == 0, nc.failure_names(g["failure"])
    gp = gpu_positions(g).astype(np.float64)
    assert np.array_equal(gp, o["particles"]["x"]), f"max |dx| = {np.abs(gp - o['particles']['x']).max()}"
    assert np.array_equal(g["particles"]["velocity"][:, :3].astype(np.float64), o["particles"]["v"])
    assert g["self_contacts"][0] == o["stats"]["self_contacts"] > 900


@pytest.mark.gpu
def test_gpu_multi_partner_fold_per_substep_fp64():
    """Reference-order kernels: every substep of the offset fold's first 12,
    started from the FP64 reference-order state, against the FP64 reference.  The first substep
    resolves 1 mm interpenetrations of about a thousand four-partner pairs;
    there the FP32 substep (the GPU's, equal to the FP32 oracle's bit for
    bit) departs from FP64 by about 1e-4 m, which is precision, not order:
    the FP64 batched and reference orders agree bit for bit on it
    (test_offset_fold_fp64_orders_agree).  The later substeps are within
    1e-5 m (stated)."""
    scene = offset_folded_square()
    cfg = nc.substep_configs(scene, 12)
    s = nc.Schedule.make(**dict(FULL, selfCollision=1))
    errs, _ = per_substep_errors(scene, cfg, s, op.SERIAL, env=SELF_REFERENCE)
    print(f"offset fold, per substep against the FP64 reference order: first {errs[0]:.3e} m, "
          f"then max {errs[1:].max():.3e} m (median {np.median(errs[1:]):.3e})")
    assert errs[0] <= FIRST_DEEP_SUBSTEP_STATED
    assert errs[1:].max() <= POS_TOL_FP64

@pytest.mark.gpu
@pytest.mark.parametrize("case", ["folded", "squeezed"])
def test_gpu_reference_order_other_scenes(case):
    """Reference-order kernels on the folded cloth (isolated pairs: phase A
    alone) and on a cloth squeezed into a couple of cells (every particle
    coupled, the overflow list in use: the serial fallback), bit-identical
    to the FP32 oracle in that order, with its contact counts."""
    if case == "folded":
        scene = folded_square(fruits=4)
        cfg = nc.substep_configs(scene, 12)
    else:
        scene = small_square(side=10, fruits=0)
        pos = scene.particles["positionAndInverseMass"]
        centre = pos[:, :3].mean(axis=0)
        pos[:, 0] = centre[0] + (pos[:, 0] - centre[0]) * np.float32(0.05)
        pos[:, 1] = centre[1] + (pos[:, 1] - centre[1]) * np.float32(0.05)
        scene.particles["previousAndMass"][:, :3] = pos[:, :3]
        cfg = nc.substep_configs(scene, 2)
    s = nc.Schedule.make(**dict(FULL, selfCollision=1))
    solver = make_solver(scene, env=SELF_REFERENCE)
    solver.step(cfg, s)
    fail = solver.failure()
    gp = solver.particles()["positionAndInverseMass"][:, :3].astype(np.float64)
    contacts = solver.self_contacts()[0]
    order = solver.self_order_stats()
    solver.close()
    o = run_oracle(scene, cfg, s, bits=32, mode=op.BATCHED_SELF_REFERENCE)
    assert fail == 0, nc.failure_names(fail)
    assert np.array_equal(gp, o["particles"]["x"]), f"max |dx| = {np.abs(gp - o['particles']['x']).max()}"
    assert contacts == o["stats"]["self_contacts"] > 0
    print(f"{case}: {order}")
    if case == "squeezed":
        assert order["fallbacks"] > 0


@pytest.mark.gpu
@pytest.mark.parametrize("edge", [0, 1], ids=["points", "with-edge-edge"])
def test_gpu_reference_order_bag(edge):
    """Reference-order kernels on the produce bag under the reference's own
    schedule with the lift, one frame (with the edge/edge family: the
    reference-order edge kernel): bit-identical to the FP32 oracle in that
    order, with its contact counts."""
    import bench
    from helpers import bag_frame_configs
    from test_gpu_parity import _check_bitexact

    dt = 1.0 / 5760.0
    scene = nc.bag_scene(scenario="recorded", timestep=dt)
    cfg = bag_frame_configs(scene, 0, 48, dt)
    s = nc.Schedule.make(**dict(bench.BAG_SCHEDULE, primitiveSelf=edge))
    g = run_gpu(scene, cfg, s, env=SELF_REFERENCE)
    o = run_oracle(scene, cfg, s, bits=32, mode=op.BATCHED_SELF_REFERENCE)
    assert g["info"]["self_order_reference"]
    assert g["failure"] == 0, nc.failure_names(g["failure"])
    _check_bitexact(g, o)
    assert g["self_contacts"][0] == o["stats"]["self_contacts"]
