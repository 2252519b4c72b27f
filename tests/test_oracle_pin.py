"""Pins of the CPU oracle against the reference (no GPU).

The golden vectors in tests/golden/ref_*.npz were produced by the reference
CPU cloth itself (tools/cloth_bag.cpp compiled by oracle/ref.mk, driven by
oracle/ref_shim.cpp; see tests/golden/make_golden.py).  The oracle's serial
order must reproduce them bit for bit.  Where the compiled reference is
present, the shim's substep loop is also checked against the reference
simulate() state hash.
"""
import json
import os
import re

import numpy as np
import pytest

import oracle_py as op

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = ["recorded_lift", "grounded", "spin", "patch_regrab_v3", "regrab_v2", "rotation_v1", "pickup"]


def load_case(name):
    z = np.load(os.path.join(GOLDEN, f"ref_{name}.npz"))
    prm = op.Params.from_buffer_copy(z["params"].tobytes())
    scene = op.OracleScene(z["particles"], z["distances"], z["knots"], z["bends"], z["grips"], z["fruits"],
                           z["pairs"], prm, z["cuff"], z["rim"], z["local_off"], z["local_idx"])
    return z, scene


def reference_schedule(iterations, release):
    """The reference substep (tools/cloth_bag.cpp:4891-5185) in serial order."""
    return op.schedule(op.SERIAL, iterations=iterations, strain_sweeps=3, reconcile_passes=8, final_passes=2,
                       certificate_passes=128, early_exit=1, self_collision=1, aerodynamics=1, swept_ground=1,
                       swept_fruit_yarn=1, frictions=1, release=release)


@pytest.mark.parametrize("name", CASES)
def test_oracle_serial_matches_reference(name):
    z, scene = load_case(name)
    steps, subs, its = (int(v) for v in z["meta"])
    grounded = name == "grounded"
    o = op.Oracle(scene, 64)
    sched = reference_schedule(its, 0 if grounded else 1)
    fail = 0
    for s in range(steps):
        fail |= o.step(z["substeps"][s * subs:(s + 1) * subs], sched)
    assert fail == 0
    st = o.read()
    ref_p, ref_f = z["final_particles"], z["final_fruits"]
    for field in ("x", "v", "prev"):
        assert np.array_equal(st["particles"][field], ref_p[field]), (
            field, np.abs(st["particles"][field] - ref_p[field]).max())
    for field in ("x", "v", "omega", "q"):
        assert np.array_equal(st["fruits"][field], ref_f[field]), (
            field, np.abs(st["fruits"][field] - ref_f[field]).max())
    stats = o.stats()
    if not grounded:
        assert stats["released_mask"] == int(z["masks"][0])
        assert stats["candidate_mask"] == int(z["masks"][1])


@pytest.mark.parametrize("name", CASES)
def test_oracle_serial_full_family_matches_reference(name):
    """With the edge/edge yarn self-collision family and its self friction
    switched on, the serial order reproduces the reference substep loop (as
    the reference simulate() runs it) bit for bit."""
    z, scene = load_case(name)
    steps, subs, its = (int(v) for v in z["meta"])
    grounded = name == "grounded"
    o = op.Oracle(scene, 64)
    sched = reference_schedule(its, 0 if grounded else 1)
    sched.primitive_self = 1
    fail = 0
    for s in range(steps):
        fail |= o.step(z["substeps"][s * subs:(s + 1) * subs], sched)
    assert fail == 0
    st = o.read()
    ref_p, ref_f = z["full_particles"], z["full_fruits"]
    for field in ("x", "v", "prev"):
        assert np.array_equal(st["particles"][field], ref_p[field]), (
            field, np.abs(st["particles"][field] - ref_p[field]).max())
    for field in ("x", "v", "omega", "q"):
        assert np.array_equal(st["fruits"][field], ref_f[field]), field
    stats = o.stats()
    assert stats["edge_contacts"] > 0 and stats["self_friction_contacts"] > 0
    if not grounded:
        assert stats["released_mask"] == int(z["full_masks"][0])
        assert stats["candidate_mask"] == int(z["full_masks"][1])


ORDER_TOL_FP64 = 1.0e-5   # m: one FP64 substep, batched (kernel) order vs reference order


@pytest.mark.parametrize("name", CASES)
def test_oracle_batched_close_to_serial(name):
    """Per substep, from the reference-order trajectory (particles, fruits
    and grips copied into a fresh oracle), the batched (kernel) order with
    every family on, the edge/edge family included, stays within
    ORDER_TOL_FP64 of the reference order: the two differ only by the
    colour order of the constraint sweeps."""
    z, scene = load_case(name)
    steps, subs, its = (int(v) for v in z["meta"])
    release = 0 if name == "grounded" else 1
    ser = reference_schedule(its, release)
    ser.primitive_self = 1
    bat = reference_schedule(its, release)
    bat.primitive_self = 1
    bat.mode = op.BATCHED
    ref = op.Oracle(scene, 64)
    errs = []
    for k in range(min(len(z["substeps"]), 12)):
        st = ref.read()
        probe = op.Oracle(scene, 64)
        probe.write(st["particles"], st["fruits"], st["grips"])
        ref.step(z["substeps"][k:k + 1], ser)
        probe.step(z["substeps"][k:k + 1], bat)
        errs.append(np.abs(probe.read()["particles"]["x"] - ref.read()["particles"]["x"]).max())
    assert max(errs) <= ORDER_TOL_FP64, (name, max(errs))


def test_restated_probes_known_answers():
    import ctypes

    L = op.lib()
    for name, n in (("oracle_probe_strain", 4), ("oracle_probe_cloth_ground_friction", 4),
                    ("oracle_probe_rolling", 4), ("oracle_probe_self_ccd", 4), ("oracle_probe_self_friction", 8)):
        out = (ctypes.c_double * n)()
        assert getattr(L, name)(out) == 1, name


def _ref_probe_values():
    text = open(os.path.join(GOLDEN, "ref_probes.txt")).read()
    vals = {}
    for line in text.splitlines():
        m = re.match(r"probe=(\S+) (.*)", line)
        if m:
            vals[m.group(1)] = dict(kv.split("=", 1) for kv in m.group(2).split() if "=" in kv)
    return vals, text


def test_probes_match_reference_printout():
    import ctypes

    vals, text = _ref_probe_values()
    assert text.count("result=PASS") == 10
    L = op.lib()
    out = (ctypes.c_double * 4)()
    L.oracle_probe_strain(out)
    ref = vals["unilateral_cloth_strain_limit"]
    assert f"{out[0]:.12f}" == ref["limited_extension"]
    assert f"{out[1]:.12f}" == ref["correction"]
    L.oracle_probe_cloth_ground_friction(out)
    ref = vals["cloth_ground_coulomb_friction"]
    assert f"{out[1]:.12f}" == ref["sliding_speed"]
    assert f"{out[2]:.12f}" == ref["sliding_energy"]
    L.oracle_probe_rolling(out)
    ref = vals["solid_sphere_slide_to_roll"]
    assert f"{out[0]:.12f}" == ref["final_speed"]
    assert f"{out[3]:.12f}" == ref["energy_ratio"]
    a = (ctypes.c_double * 8)()
    L.oracle_probe_aerodynamics(a)
    ref = vals["explicit_yarn_and_fruit_aerodynamics"]
    assert f"{-a[1]:.12f}" == ref["yarn_crossflow_force"]
    assert f"{-a[0]:.12f}" == ref["yarn_axial_force"]
    assert f"{a[4]:.12f}" == ref["fruit_speed"]
    assert f"{a[5]:.12f}" == ref["fruit_angular_speed"]
    assert abs(a[0] - a[2]) < 1e-12 and abs(a[1] - a[3]) < 1e-12   # refinement invariance
    L.oracle_probe_self_ccd(out)
    ref = vals["continuous_yarn_capsule_self_contact"]
    assert f"{out[0]:.12f}" == ref["edge_contact_height"]
    assert f"{out[1]:.12f}" == ref["edge_removed_advance"]
    assert int(out[2]) == int(ref["edge_contacts"])
    L.oracle_probe_self_friction(a)
    ref = vals["cloth_self_coulomb_friction"]
    for k, key in enumerate(("sticking_slip", "sticking_momentum", "sticking_energy", "sliding_slip",
                             "sliding_momentum", "sliding_cone_ratio")):
        assert f"{a[k]:.12f}" == ref[key], key


def test_shim_loop_equals_reference_simulate():
    """The shim's substep loop is the reference simulate() (live, when the
    compiled reference is present)."""
    import ref_py as rp

    if not rp.available():
        pytest.skip("compiled reference not present")
    hashes = json.load(open(os.path.join(GOLDEN, "ref_hashes.json")))
    h = hashes["grounded"]
    a = h["args"]
    assert h["simulate"] == h["shim_full"]
    live = rp.simulate_hash("grounded", a["steps"], a["frame_dt"], 2, 1)
    run = rp.run("grounded", a["steps"], a["frame_dt"], 2, 1, primitive=1)
    assert live == run["hash"]


def test_golden_hashes_self_consistent():
    hashes = json.load(open(os.path.join(GOLDEN, "ref_hashes.json")))
    for name, h in hashes.items():
        assert h["simulate"] == h["shim_full"], name
