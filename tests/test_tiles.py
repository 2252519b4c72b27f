"""Tile mode of the cooperative grid: colour chains between grid barriers
on per-CTA closures in shared memory (cloth_tile.cuh).

A CTA recomputes, from the same inputs and in the same colour order, every
item whose result reaches its own particles, so tile mode must give the
bits of the colour-by-colour schedule (NUMI_CLOTH_TILES=0) and of the FP32
oracle on every schedule it covers.
"""
import numpy as np
import pytest

import numi_cloth as nc
import oracle_py as op
from helpers import SELF_REFERENCE, make_solver, run_gpu, run_oracle, small_square
from test_gpu_parity import _check_bitexact

pytestmark = pytest.mark.gpu

BENCH_LIKE = dict(iterations=1, strainSweeps=1, reconcilePasses=0, finalPasses=0, certificatePasses=0,
                  earlyExit=0, aerodynamics=0, sweptGround=1, frictions=1, selfCollision=1)


TILES = {"NUMI_CLOTH_TILES": "1"}
COLOURS = {"NUMI_CLOTH_TILES": "0"}


def _both(scene, cfg, sched, frames=1):
    tiled = run_gpu(scene, cfg, sched, frames=frames, env=TILES)
    plain = run_gpu(scene, cfg, sched, frames=frames, env=COLOURS)
    return tiled, plain


def _same(a, b):
    assert np.array_equal(a["particles"].view(np.uint8), b["particles"].view(np.uint8))
    assert np.array_equal(a["fruits"].view(np.uint8), b["fruits"].view(np.uint8))
    assert np.array_equal(a["distances"].view(np.uint8), b["distances"].view(np.uint8))
    assert np.array_equal(a["grips"].view(np.uint8), b["grips"].view(np.uint8))
    assert a["self_contacts"] == b["self_contacts"]


@pytest.mark.parametrize("variant", ["bench", "sweeps2-damped", "no-self", "no-strain", "no-fruits", "many-fruits",
                                     "folded", "folded-reference-order"])
def test_tiles_equal_colour_schedule_and_oracle(variant):
    """Tile mode against the colour-by-colour launch and the oracle; the
    folded variants lay the upper half of the cloth over the lower one,
    shifted half a spacing, so that point self contact has particles with
    several partners (in the reference order phase A lists them and CTA 0
    runs the ordered pass)."""
    sched = dict(BENCH_LIKE)
    kw = dict(side=96, fruits=12)
    env = TILES
    if variant == "sweeps2-damped":
        sched.update(strainSweeps=2, damping=0.3)
    elif variant == "no-self":
        sched.update(selfCollision=0)
    elif variant == "no-strain":
        sched.update(strainSweeps=0)
    elif variant == "no-fruits":
        kw.update(fruits=0)
    elif variant == "many-fruits":
        kw.update(fruits=48, fruitRadiusMin=0.005, fruitRadiusMax=0.02)
    plain_env = COLOURS
    mode = op.BATCHED
    if variant.startswith("folded"):
        # a 48 x 48 fold (1,152 particles over 1,152, four partners each) on
        # a forced cooperative grid of 16 CTAs
        from test_self_contact import offset_folded_square
        scene = offset_folded_square(side=48)
        forced = {"NUMI_CLOTH_GRID": "16", "NUMI_CLOTH_TILE_GRID": "16", "NUMI_CLOTH_RESIDENT": "0"}
        if variant.endswith("reference-order"):
            forced.update(SELF_REFERENCE)
            mode = op.BATCHED_SELF_REFERENCE
        env, plain_env = dict(TILES, **forced), dict(COLOURS, **forced)
    else:
        scene = small_square(**kw)
    cfg = nc.substep_configs(scene, 24)
    s = nc.Schedule.make(**sched)
    tiled = run_gpu(scene, cfg, s, env=env)
    plain = run_gpu(scene, cfg, s, env=plain_env)
    assert tiled["info"]["last_tiles"], tiled["info"]
    assert not plain["info"]["last_tiles"]
    assert tiled["failure"] == 0 and plain["failure"] == 0, nc.failure_names(tiled["failure"] | plain["failure"])
    _same(tiled, plain)
    _check_bitexact(tiled, run_oracle(scene, cfg, s, bits=32, mode=mode))


def test_tiles_across_launches_and_frames():
    """Launches that end on the alternate buffers copy them back: two frames
    of 12 substeps equal one of 24 and the colour schedule."""
    scene = small_square(side=128, fruits=16)
    cfg = nc.substep_configs(scene, 24)
    s = nc.Schedule.make(**BENCH_LIKE)
    one = run_gpu(scene, cfg, s, env=TILES)
    two = run_gpu(scene, cfg, s, frames=2, env=TILES)
    odd = run_gpu(scene, cfg, s, frames=3, env=TILES)
    assert one["info"]["last_tiles"]
    _same(one, two)
    _same(one, odd)
    _same(one, run_gpu(scene, cfg, s, env=COLOURS))


@pytest.mark.parametrize("grid", [40, 96])
def test_tiles_other_grid_sizes(grid):
    """Fewer tile CTAs (bigger tiles and closures) give the same bits."""
    scene = small_square(side=112, fruits=8)
    cfg = nc.substep_configs(scene, 12)
    s = nc.Schedule.make(**BENCH_LIKE)
    a = run_gpu(scene, cfg, s, env=dict(TILES, NUMI_CLOTH_TILE_GRID=str(grid)))
    assert a["info"]["last_tiles"] and a["info"]["grid"] == grid
    b = run_gpu(scene, cfg, s, env=COLOURS)
    _same(a, b)


def test_tiles_rebuilt_after_material_change():
    scene = small_square(side=96, fruits=6)
    cfg = nc.substep_configs(scene, 12)
    s = nc.Schedule.make(**BENCH_LIKE)
    out = []
    for env in (TILES, COLOURS):
        sv = make_solver(scene, env=env)
        sv.step(cfg, s)
        fam, val = sv.compliance_groups()[0]
        sv.replace_compliance(fam, val, val * 10.0)
        sv.step(cfg, s)
        out.append((sv.particles(), sv.distances(), sv.launch_info()))
        sv.close()
    assert out[0][2]["last_tiles"] and not out[1][2]["last_tiles"]
    assert np.array_equal(out[0][0].view(np.uint8), out[1][0].view(np.uint8))
    assert np.array_equal(out[0][1].view(np.uint8), out[1][1].view(np.uint8))


def test_non_tile_schedule_on_tiled_cloth():
    """Schedules tile mode does not cover run colour by colour on the same
    handle, and the two kinds of launch can follow each other."""
    scene = small_square(side=96, fruits=6)
    cfg = nc.substep_configs(scene, 12)
    full = nc.Schedule.make(iterations=2, strainSweeps=2, reconcilePasses=1, finalPasses=1, certificatePasses=2,
                            earlyExit=1, aerodynamics=1, sweptGround=1, frictions=1, selfCollision=1)
    bench = nc.Schedule.make(**BENCH_LIKE)
    outs = []
    for env in (TILES, COLOURS):
        sv = make_solver(scene, env=env)
        sv.step(cfg, bench)
        sv.step(cfg, full)
        info = sv.launch_info()
        sv.step(cfg, bench)
        outs.append((sv.particles(), info, sv.launch_info(), sv.failure()))
        sv.close()
    assert not outs[0][1]["last_tiles"] and outs[0][2]["last_tiles"]
    assert outs[0][3] == 0 and outs[1][3] == 0
    assert np.array_equal(outs[0][0].view(np.uint8), outs[1][0].view(np.uint8))


def test_tune_keeps_state_and_bits():
    """numi_cloth_tune times the colour-by-colour launch and tile mode at
    three CTA counts, keeps the fastest and leaves the state as it was: a
    tuned handle steps to the same bits as an untuned one."""
    scene = small_square(side=96, fruits=6)
    cfg = nc.substep_configs(scene, 12)
    s = nc.Schedule.make(**BENCH_LIKE)
    tuned = make_solver(scene)
    before = tuned.particles()
    r = tuned.tune(cfg, s)
    print("tune:", r)
    assert np.array_equal(tuned.particles().view(np.uint8), before.view(np.uint8))
    assert tuned.failure() == 0
    colours = r["colours_per_sync"]
    assert colours == 1 or colours > 1 and r["threads"] == 512
    tuned.step(cfg, s)
    plain = make_solver(scene)
    plain.step(cfg, s)
    assert np.array_equal(tuned.particles().view(np.uint8), plain.particles().view(np.uint8))
    assert tuned.launch_info()["last_tiles"] == (colours > 1)
    tuned.close()
    plain.close()
