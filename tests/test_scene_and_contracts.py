"""Host logic without a GPU: scene builders, colouring, the material and
grip-trajectory file contracts, and the C ABI surface."""
import ctypes
import os
import re

import numpy as np
import pytest

import numi_cloth as nc

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
FIX = os.path.join(GOLDEN, "reference_fixtures")


# ------------------------------------------------------------------ scenes
def _ref_scene(name="recorded_lift"):
    return np.load(os.path.join(GOLDEN, f"ref_{name}.npz"))


def test_bag_matches_reference_scene():
    """The product bag builder reproduces the reference makeCloth/makeBalls
    (tools/cloth_bag.cpp:610-973), rounded once to FP32."""
    z = _ref_scene()
    s = nc.bag_scene(scenario="recorded")
    assert s.n == len(z["particles"]) == 1465
    pos = s.particles["positionAndInverseMass"]
    assert np.array_equal(pos[:, :3], z["particles"]["x"].astype(np.float32))
    assert np.array_equal(pos[:, 3], z["particles"]["w"].astype(np.float32))
    assert np.array_equal(s.rest64, z["particles"]["rest"])
    # distances: same (i, j) set; rest lengths are the FP64 values rounded
    ref = {(int(d["i"]), int(d["j"])): d for d in z["distances"]}
    assert len(ref) == len(s.distances) == 2904
    for rec in s.distances:
        i, j = int(rec["particlesAndColor"][0]), int(rec["particlesAndColor"][1])
        d = ref[(i, j)]
        assert rec["material"][0] == np.float32(d["rest"])
        assert rec["material"][1] == np.float32(d["compliance"])
        assert rec["material"][3] == np.float32(d["maxext"])
        assert rec["particlesAndColor"][3] == d["kind"]
    refk = {tuple(int(v) for v in k["p"]): k for k in z["knots"]}
    assert len(s.knots) == len(refk) == 1369
    for rec in s.knots:
        k = refk[tuple(int(v) for v in rec["particles"])]
        assert rec["material"][0] == np.float32(k["restcos"])
    refb = {tuple(int(v) for v in b["p"]): b for b in z["bends"]}
    assert len(s.bends) == len(refb) == 2834
    for rec in s.bends:
        b = refb[tuple(int(v) for v in rec["particlesAndColor"][:3])]
        assert rec["material"][0] == np.float32(b["restchord"])
        assert rec["material"][1] == np.float32(b["restarc"])
    assert np.array_equal(s.grips["particle"][:, 0], z["grips"]["particle"])
    assert np.array_equal(s.grips["targetOffsetAndCompliance"][:, :3], z["grips"]["offset"].astype(np.float32))
    assert np.array_equal(s.fruits["positionAndInverseMass"][:, :3], z["fruits"]["x"].astype(np.float32))
    assert np.array_equal(s.fruits["previousAndRadius"][:, 3], z["fruits"]["radius"].astype(np.float32))
    assert np.array_equal(s.local_off, z["local_off"]) and np.array_equal(s.local_idx, z["local_idx"])
    assert np.array_equal(s.cuff, z["cuff"]) and np.array_equal(s.rim, z["rim"])


def test_bag_colouring_counts():
    """First-fit colouring gives the reference Metal host's 5/6/5/15 colours
    (tools/cloth_bag_metal.mm:627-676)."""
    s = nc.bag_scene()
    assert (s.extra["distance_colours"], s.extra["knot_colours"], s.extra["bend_colours"],
            s.extra["pair_colours"]) == (5, 6, 5, 15)


def _conflict_free(colours, writers):
    for c in np.unique(colours):
        w = writers[colours == c].ravel()
        if len(np.unique(w)) != len(w):
            return False
    return True


@pytest.mark.parametrize("builder", ["bag", "square"])
def test_batches_conflict_free_and_contiguous(builder):
    s = nc.bag_scene() if builder == "bag" else nc.square_scene(side=48)
    d = s.distances["particlesAndColor"]
    assert np.all(np.diff(d[:, 2].astype(np.int64)) >= 0)
    assert _conflict_free(d[:, 2], d[:, :2])
    b = s.bends["particlesAndColor"]
    assert _conflict_free(b[:, 3], b[:, [0, 2]])
    if len(s.knots):
        assert _conflict_free(s.knots["control"][:, 0], s.knots["particles"])
    p = s.pairs["fruitsAndColor"]
    assert _conflict_free(p[:, 2], p[:, :2])
    # yarn segments lead every colour run
    for c in np.unique(d[:, 2]):
        kinds = d[d[:, 2] == c, 3]
        yarn = kinds != 3
        assert not np.any(yarn[1:] & ~yarn[:-1])


def test_square_counts():
    s = nc.square_scene()
    assert s.n == 65536
    assert len(s.distances) + len(s.bends) == 390658
    assert len(s.bends) == 130048
    assert s.extra["yarn_segments"] == 130560
    assert s.extra["distance_colours"] == 8 and s.extra["bend_colours"] == 4
    f = s.fruits
    assert len(f) == 64
    r = f["previousAndRadius"][:, 3]
    assert r.min() >= 0.02 and r.max() <= 0.05
    assert np.all(f["positionAndInverseMass"][:, 2] - r >= 0.55 - 1e-6)


# --------------------------------------------------------------- contracts
def test_material_defaults_artifact_parity():
    m = nc.load_material(os.path.join(FIX, "default-material.txt"))
    d = nc.material_defaults()
    for name, _ in nc.Material._fields_:
        assert getattr(m, name) == getattr(d, name), name


def test_material_rejects_invalid():
    with pytest.raises(nc.ClothError, match="artifact is missing: fruit_rotational_drag"):
        nc.load_material(os.path.join(FIX, "invalid-material.txt"))


def test_material_rejects_unknown_and_duplicate(tmp_path):
    base = open(os.path.join(FIX, "default-material.txt")).read()
    p = tmp_path / "unknown.txt"
    p.write_text(base + "mystery=1\n")
    with pytest.raises(nc.ClothError, match="unknown cloth material field"):
        nc.load_material(str(p))
    p = tmp_path / "dup.txt"
    p.write_text(base + "yarn_radius_m=0.004\n")
    with pytest.raises(nc.ClothError, match="nonempty and unique"):
        nc.load_material(str(p))
    p = tmp_path / "bounds.txt"
    p.write_text(base.replace("yarn_radius_m=0.004", "yarn_radius_m=0.5"))
    with pytest.raises(nc.ClothError, match="outside contract bounds: yarn_radius_m"):
        nc.load_material(str(p))


def test_material_changes_bag_scene():
    m = nc.material_defaults()
    m.axialBodyComplianceMPerN = 2.0e-8
    s = nc.bag_scene(material=m)
    assert np.any(s.distances["material"][:, 1] == np.float32(2.0e-8))


@pytest.mark.parametrize("name,schema_select,generations", [
    ("synthetic-identity.csv", False, 1),
    ("synthetic-rotation.csv", False, 1),
    ("synthetic-regrab.csv", False, 3),
    ("synthetic-patch-regrab.csv", True, 3),
])
def test_trajectory_loads(name, schema_select, generations):
    t = nc.GripTrajectory(os.path.join(FIX, name))
    assert t.select_nearest == schema_select
    assert abs(t.duration - 1.0 / 120.0) < 1e-9
    gens = max(t.sample(k * t.duration / 50.0).generation for k in range(51))
    assert gens == generations


def test_trajectory_rejects_reactivation():
    with pytest.raises(nc.ClothError, match="cannot reactivate after release"):
        nc.GripTrajectory(os.path.join(FIX, "invalid-reactivation.csv"))


def test_trajectory_sampling_slerp():
    t = nc.GripTrajectory(os.path.join(FIX, "synthetic-rotation.csv"))
    p = t.sample(t.duration * 0.5)
    q = np.array(p.orientation[:])
    assert abs(np.linalg.norm(q) - 1.0) < 1e-12
    assert q[1] > 0.0 and abs(p.translation[2] - 0.001) < 1e-9


def test_trajectory_configs_sample_substep_end():
    s = nc.bag_scene()
    t = nc.GripTrajectory(os.path.join(GOLDEN, "lift-v1.csv"))
    dt = 1.0 / 2880.0
    cfg = t.configs(s.config, s.handle_base, 0, 48, dt)
    z = cfg["gripTargetAndActive"][:, 2].astype(np.float64)
    expected = s.handle_base[2] + 0.3 * (np.arange(1, 49) * dt)
    assert np.allclose(z, expected, atol=1e-6)


def test_trajectory_rejects_uncovered_time():
    t = nc.GripTrajectory(os.path.join(FIX, "synthetic-identity.csv"))
    with pytest.raises(nc.ClothError):
        t.sample(1.0)


# --------------------------------------------------------------------- ABI
def _declared_functions():
    names = set()
    for h in ("numi_cloth.h", "numi_cloth_scene.h"):
        text = open(os.path.join(ROOT, "include", h)).read()
        names |= set(re.findall(r"\b(numi_cloth_[a-z0-9_]+)\s*\(", text))
    return names


def test_library_exports_every_declared_symbol():
    lib = nc.load_library()
    missing = [n for n in sorted(_declared_functions()) if not hasattr(lib, n)]
    assert not missing, missing
    assert b"sm_100a" in lib.numi_cloth_version()


def test_record_sizes_match_reference_abi():
    sizes = {"CONFIG": 224, "PARTICLE": 48, "DISTANCE": 32, "GRIP": 48, "KNOT": 48, "BEND": 32, "FRUIT": 96,
             "FRUIT_PAIR": 32}
    for name, size in sizes.items():
        assert getattr(nc.abi, name).itemsize == size


def test_reference_header_offsets(tmp_path):
    """Byte layout identical to the reference ABI header (compiled check,
    where the reference sources are present)."""
    ref = os.path.join(os.environ.get("NUMI_CLOTH_REFERENCE", "/root/reference"), "include")
    if not os.path.isdir(ref):
        pytest.skip("reference headers not present")
    src = tmp_path / "abi_check.cpp"
    fields = {
        "Config": ["control", "constraintCounts", "contactCounts", "gravityAndTimestep", "gripTargetAndActive",
                   "gripOrientation", "gripControl", "gripMaterial", "clothMaterial", "fruitMaterial",
                   "airVelocityAndDensity", "aerodynamicCoefficients", "mouthControl", "mouthMaterial"],
        "Particle": ["positionAndInverseMass", "previousAndMass", "velocity"],
        "Distance": ["particlesAndColor", "material"],
        "Grip": ["particle", "targetOffsetAndCompliance", "lambda"],
        "Knot": ["particles", "control", "material"],
        "Bend": ["particlesAndColor", "material"],
        "Fruit": ["positionAndInverseMass", "previousAndRadius", "velocityAndGroundImpulse", "angularVelocity",
                  "orientation", "identity"],
        "FruitPair": ["fruitsAndColor", "contact"],
    }
    lines = ['#include <cstddef>', '#include "numi/cloth_bag_gpu.h"', '#include "numi_cloth.h"']
    for t, fs in fields.items():
        lines.append(f"static_assert(sizeof(NumiClothBagGPU{t}) == sizeof(NumiCloth{t}));")
        for f in fs:
            lines.append(f"static_assert(offsetof(NumiClothBagGPU{t}, {f}) == offsetof(NumiCloth{t}, {f}));")
    lines.append("int main() { return 0; }")
    src.write_text("\n".join(lines) + "\n")
    import subprocess

    r = subprocess.run(["g++", "-std=c++20", f"-I{ref}", f"-I{os.path.join(ROOT, 'include')}", str(src), "-o",
                        str(tmp_path / "abi_check")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
