"""Released-fruit masks (updateReleasedFruit, tools/cloth_bag.cpp:4545-4597)
on the GPU against the oracle: the mask is an end-state invariant of the
reference runs, and the GPU must flag the same fruits."""
import numpy as np
import pytest

import numi_cloth as nc
from helpers import FULL, bag_frame_configs, run_gpu, run_oracle

DT = 1.0 / 5760.0


def bag_with_fruits_at_the_mouth():
    """The produce bag with fruit 0 lifted 0.2 m above the mouth (leaves
    through the mouth: released) and fruit 1 just above the mouth plane
    (a mouth candidate, not yet clear of it)."""
    scene = nc.bag_scene(scenario="recorded", timestep=DT)
    rim = scene.particles["positionAndInverseMass"][scene.rim, :3].astype(np.float64)
    centre = rim.mean(axis=0)
    f = scene.fruits
    f["positionAndInverseMass"][0, :3] = (centre + [0.0, 0.0, 0.2]).astype(np.float32)
    f["positionAndInverseMass"][1, :3] = (centre + [0.0, 0.0, 0.01]).astype(np.float32)
    f["previousAndRadius"][:2, :3] = f["positionAndInverseMass"][:2, :3]
    f["velocityAndGroundImpulse"][:2] = 0.0
    return scene


@pytest.mark.gpu
def test_release_masks_match_oracle():
    scene = bag_with_fruits_at_the_mouth()
    cfg = bag_frame_configs(scene, 0, 4, DT)
    s = nc.Schedule.make(**dict(FULL, release=1))
    g = run_gpu(scene, cfg, s)
    o32 = run_oracle(scene, cfg, s, bits=32)
    o64 = run_oracle(scene, cfg, s, bits=64)
    assert g["failure"] == 0
    cand, released = g["release"]
    assert (cand, released) == (o32["stats"]["candidate_mask"], o32["stats"]["released_mask"])
    assert (cand, released) == (o64["stats"]["candidate_mask"], o64["stats"]["released_mask"])
    assert released & 1 and cand & 2 and not released & 2


@pytest.mark.gpu
def test_release_off_leaves_masks_clear():
    scene = bag_with_fruits_at_the_mouth()
    cfg = bag_frame_configs(scene, 0, 2, DT)
    g = run_gpu(scene, cfg, nc.Schedule.make(**FULL))
    assert g["release"] == (0, 0)


def test_oracle_release_flags_lifted_fruit():
    """The oracle (FP64, reference order) releases the fruit lifted clear of
    the mouth and marks the one in the mouth plane as a candidate."""
    import oracle_py as op
    scene = bag_with_fruits_at_the_mouth()
    cfg = bag_frame_configs(scene, 0, 2, DT)
    o = op.Oracle(op.from_abi(scene), 64)
    o.step(op.substeps_from_configs(cfg), op.schedule_from_abi(nc.Schedule.make(**dict(FULL, release=1)), op.SERIAL))
    st = o.stats()
    assert st["released_mask"] & 1 and st["candidate_mask"] & 2 and not st["released_mask"] & 2
