#!/usr/bin/env python3
"""Generate the golden vectors of the cloth oracle from the compiled reference.

Run in a checkout next to the reference sources (default /root/reference):

    python tests/golden/make_golden.py [--reference /root/reference]

It builds oracle/_ref (oracle/ref.mk), then writes into tests/golden/:
  reference_fixtures/   the reference's own calibration fixtures (grip
                        trajectories v1-v3, material artifacts), copied as data
  ref_<case>.npz        reference scene (construction order, FP64), its render
                        triangles, the grip
                        pose of every substep, and the reference's final
                        particle/fruit state after the reference substep loop,
                        without (final_*) and with (full_*) the primitive
                        (edge/edge) self-collision family
  ref_spin.obj          the reference executable's OBJ of the spin case's final state
  ref_probes.txt        stdout of the reference executable's analytic probes
  ref_hashes.json       reference simulate() state hashes (full substep) and
                        the shim loop's hash of the same runs
The committed fixtures let the oracle be checked where the reference is absent.
"""
from __future__ import annotations

import argparse
import json
import os
import shutil
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

CASES = {
    # name: (scenario, trajectory file, steps, frame dt, substeps, iterations)
    "recorded_lift": ("recorded", "lift-v1.csv", 2, 1.0 / 120.0, 8, 2),
    "grounded": ("grounded", None, 1, 1.0 / 120.0, 6, 3),
    "spin": ("spin", None, 1, 1.0 / 120.0, 6, 2),
    "patch_regrab_v3": ("recorded", "reference_fixtures/synthetic-patch-regrab.csv", 1, 1.0 / 120.0, 24, 2),
    "regrab_v2": ("recorded", "reference_fixtures/synthetic-regrab.csv", 1, 1.0 / 120.0, 24, 2),
    "rotation_v1": ("recorded", "reference_fixtures/synthetic-rotation.csv", 1, 1.0 / 120.0, 12, 2),
    "pickup": ("pickup", None, 1, 1.0 / 120.0, 6, 2),
}

PROBES = ["--strain-probe", "--cloth-ground-friction-probe", "--rolling-probe", "--aerodynamics-probe",
          "--rolling-resistance-probe", "--deformable-response-probe", "--self-ccd-probe",
          "--yarn-mechanics-probe", "--self-friction-probe", "--mouth-release-probe"]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("NUMI_CLOTH_REFERENCE", "/root/reference"))
    args = ap.parse_args()
    subprocess.run(["make", "-s", "-f", "ref.mk", f"REFERENCE={args.reference}"], cwd=os.path.join(ROOT, "oracle"),
                   check=True)
    import ref_py as rp

    fx = os.path.join(HERE, "reference_fixtures")
    os.makedirs(fx, exist_ok=True)
    for sub in ("trajectories", "synthetic"):
        src = os.path.join(args.reference, "calibration", sub)
        for name in sorted(os.listdir(src)):
            if name.endswith(".csv") and sub == "trajectories" or name.endswith("material.txt"):
                shutil.copyfile(os.path.join(src, name), os.path.join(fx, name))

    hashes = {}
    for name, (scenario, traj, steps, fdt, subs, its) in CASES.items():
        tpath = os.path.join(HERE, traj) if traj else None
        scene = rp.scene(scenario)
        run = rp.run(scenario, steps, fdt, subs, its, tpath, primitive=0, point_self=1)
        full = rp.run(scenario, steps, fdt, subs, its, tpath, primitive=1, point_self=1)
        ref_hash = rp.simulate_hash(scenario, steps, fdt, subs, its, tpath)
        hashes[name] = {"simulate": hex(ref_hash), "shim_full": hex(full["hash"]),
                        "shim_restricted": hex(run["hash"]),
                        "args": {"scenario": scenario, "trajectory": traj, "steps": steps, "frame_dt": fdt,
                                 "substeps": subs, "iterations": its}}
        prm = scene.params
        params = np.frombuffer(bytes(prm), dtype=np.uint8)
        np.savez_compressed(
            os.path.join(HERE, f"ref_{name}.npz"),
            particles=scene.particles, distances=scene.distances, knots=scene.knots, bends=scene.bends,
            grips=scene.grips, fruits=scene.fruits, pairs=scene.pairs, cuff=scene.cuff, rim=scene.rim,
            local_off=scene.local_off, local_idx=scene.local_idx, params=params, substeps=run["substeps"],
            final_particles=run["particles"], final_fruits=run["fruits"],
            masks=np.array([run["released_mask"], run["candidate_mask"]], np.uint64),
            full_particles=full["particles"], full_fruits=full["fruits"],
            full_masks=np.array([full["released_mask"], full["candidate_mask"]], np.uint64),
            meta=np.array([steps, subs, its], np.uint32), triangles=rp.render_triangles(scenario))
        print(name, hashes[name])
    # one OBJ frame written by the reference executable (dumpOBJ) after the
    # spin case's run
    a = CASES["spin"]
    subprocess.run([rp.BINARY, "--scenario", "spin", "--steps", str(a[2]), "--timestep", repr(a[3]), "--substeps",
                    str(a[4]), "--iterations", str(a[5]), "--dump-obj", os.path.join(HERE, "ref_spin.obj")],
                   check=True, capture_output=True)
    with open(os.path.join(HERE, "ref_hashes.json"), "w") as f:
        json.dump(hashes, f, indent=1, sort_keys=True)
    lines = []
    for p in PROBES:
        out = subprocess.run([rp.BINARY, p], capture_output=True, text=True, check=True).stdout
        lines.append(out.strip())
    with open(os.path.join(HERE, "ref_probes.txt"), "w") as f:
        f.write("\n".join(lines) + "\n")


if __name__ == "__main__":
    main()
