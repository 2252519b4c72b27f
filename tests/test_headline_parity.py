"""Parity of the benchmarked configuration: the 256x256 cloth (65,536
particles, 4 mm, 64 spheres, two gripped corners, ground, hash-grid point
self contact) under the bench schedule, one full 48-substep frame at
dt = 1/2880 s, and the end-state invariants under a certifying schedule.

Bars: bit-identical to the FP32 oracle in the kernels' batched order; every
substep of the first frame, started from the FP64 trajectory's state,
within 1e-5 m of the FP64 oracle (both orders stated); end-state strain-limit
violation and ground / fruit / self penetration at most 1 um once the strain
limit is certified (3 sweeps, final passes, certificate passes on the last
substep, tools/cloth_bag.cpp:5059-5185), and the same residuals and release
masks as the oracles.
"""
import numpy as np
import pytest

import bench
import numi_cloth as nc
import oracle_py as op
from helpers import bag_frame_configs, per_substep_errors, run_gpu, run_oracle
from test_gpu_parity import _check_bitexact

pytestmark = pytest.mark.gpu

POS_TOL_FP64 = 1.0e-5   # m: one FP32 substep vs the FP64 substep from the same state
INVARIANT_TOL = 1.0e-6  # m: end-state strain-limit violation and penetrations
CERTIFIED = dict(bench.BENCH_SCHEDULE, strainSweeps=3, finalPasses=2, certificatePasses=8, earlyExit=1)


def _bench_scene():
    return nc.square_scene(side=bench.SIDE)


def test_bench_frame_bitexact_fp32():
    scene = _bench_scene()
    cfg = nc.substep_configs(scene, bench.SUBSTEPS)
    s = nc.Schedule.make(**bench.BENCH_SCHEDULE)
    g = run_gpu(scene, cfg, s)
    o = run_oracle(scene, cfg, s, bits=32)
    assert g["info"]["grid"] > 1
    assert g["failure"] == 0, nc.failure_names(g["failure"])
    _check_bitexact(g, o)
    assert np.allclose(g["residuals"], np.asarray(o["residuals"], np.float64), rtol=1e-12, atol=0.0)
    assert g["self_contacts"][0] == o["stats"]["self_contacts"]
    # stated: one strain sweep per substep leaves the corners over the limit
    print(f"bench schedule, end of frame 1: strain-limit violation {g['residuals'][0]:.3e} m, "
          f"ground {g['residuals'][1]:.3e} m, fruit {g['residuals'][2]:.3e} m, self {g['residuals'][3]:.3e} m")


@pytest.mark.parametrize("mode", [op.BATCHED, op.SERIAL], ids=["batched-order", "reference-order"])
def test_bench_per_substep_fp64(mode):
    scene = _bench_scene()
    cfg = nc.substep_configs(scene, bench.SUBSTEPS)
    s = nc.Schedule.make(**bench.BENCH_SCHEDULE)
    errs, ferrs = per_substep_errors(scene, cfg, s, mode)
    print(f"256x256 bench schedule, FP64 {'batched' if mode == op.BATCHED else 'reference'} order, per substep "
          f"over the first frame: max particle error {errs.max():.3e} m (median {np.median(errs):.3e}), "
          f"fruit {ferrs.max():.3e} m")
    assert errs.max() <= POS_TOL_FP64
    assert ferrs.max() <= POS_TOL_FP64


def test_bench_certified_invariants():
    scene = _bench_scene()
    cfg = nc.substep_configs(scene, bench.SUBSTEPS)
    s = nc.Schedule.make(**CERTIFIED)
    g = run_gpu(scene, cfg, s)
    o = run_oracle(scene, cfg, s, bits=32)
    assert g["failure"] == 0, nc.failure_names(g["failure"])
    _check_bitexact(g, o)
    r = g["residuals"]
    print(f"certified schedule, end of frame 1: strain-limit violation {r[0]:.3e} m, ground {r[1]:.3e} m, "
          f"fruit {r[2]:.3e} m, self {r[3]:.3e} m")
    assert np.allclose(r, np.asarray(o["residuals"], np.float64), rtol=1e-12, atol=0.0)
    assert r[0] <= INVARIANT_TOL and r[1] <= INVARIANT_TOL and r[2] <= INVARIANT_TOL and r[3] <= INVARIANT_TOL


def test_bag_reference_schedule_invariants():
    """The produce bag under the reference's own schedule (bench `bag`
    object) with the lift: zero residuals and the release masks of both
    oracles after one frame."""
    dt = 1.0 / 5760.0
    scene = nc.bag_scene(scenario="recorded", timestep=dt)
    cfg = bag_frame_configs(scene, 0, 48, dt)
    s = nc.Schedule.make(**bench.BAG_SCHEDULE)
    g = run_gpu(scene, cfg, s)
    o32 = run_oracle(scene, cfg, s, bits=32)
    o64 = run_oracle(scene, cfg, s, bits=64, mode=op.SERIAL)
    assert g["failure"] == 0, nc.failure_names(g["failure"])
    _check_bitexact(g, o32)
    r = g["residuals"]
    print(f"bag, reference schedule, end of frame 1: residuals {r}")
    assert np.all(np.asarray(r) <= INVARIANT_TOL)
    masks = (o32["stats"]["candidate_mask"], o32["stats"]["released_mask"])
    assert g["release"] == masks
    assert masks == (o64["stats"]["candidate_mask"], o64["stats"]["released_mask"])
