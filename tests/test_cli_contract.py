"""The command-line contract of the reference cloth executable, on the GPU
path: the key=value lines and exit codes that the reference's cmake checks
consume (cmake/CheckGripTrajectory.cmake:11-104,
cmake/ExpectGripTrajectoryFailure.cmake:5-27,
cmake/CheckClothMaterialParity.cmake:5-60), run with the same arguments and
matched with the same regular expressions.
"""
import os
import re
import subprocess

import pytest

from helpers import ROOT

FIX = os.path.join(ROOT, "tests", "golden", "reference_fixtures")
EXE = os.path.join(ROOT, "numi-solver_b200", "numi_cloth", "numi-cloth-replay")
CPU_ARGS = ["--scenario", "recorded", "--steps", "1", "--substeps", "24", "--iterations", "32", "--replays", "2"]


def _run(args, timeout=600):
    return subprocess.run([EXE] + args, capture_output=True, text=True, timeout=timeout)


def test_cli_rejects_bad_option_with_exit_2():
    """Argument errors leave with exit code 2 and a message, as the
    reference's exception handler (tools/cloth_bag.cpp:5924-5927)."""
    out = _run(["--scenario", "sideways"])
    assert out.returncode == 2
    assert "unknown scenario: sideways" in out.stderr
    out = _run(["--steps"])
    assert out.returncode == 2 and "missing value for --steps" in out.stderr


def test_cli_rejects_reactivation_with_exit_2():
    out = _run(["--scenario", "recorded", "--grip-trajectory", os.path.join(FIX, "invalid-reactivation.csv"),
                "--steps", "1", "--substeps", "1", "--iterations", "1", "--replays", "2"])
    assert out.returncode == 2
    assert re.search("cannot.reactivate.after.release", out.stdout + out.stderr)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["invalid-distant-regrab.csv", "invalid-distant-patch-regrab.csv"])
def test_cli_rejects_distant_regrab(name):
    """ExpectGripTrajectoryFailure.cmake: exit code 2 and the capture-radius
    message (the GPU grip attach sets GRIP_CAPTURE)."""
    out = _run(["--scenario", "recorded", "--grip-trajectory", os.path.join(FIX, name), "--steps", "1",
                "--substeps", "1", "--iterations", "1", "--replays", "2"])
    assert out.returncode == 2, out.stdout + out.stderr
    assert re.search("reattachment.exceeds.capture.radius", out.stdout + out.stderr)


@pytest.mark.gpu
def test_cli_patch_regrab_keys():
    out = _run(CPU_ARGS + ["--grip-trajectory", os.path.join(FIX, "synthetic-patch-regrab.csv")])
    text = out.stdout
    assert out.returncode == 0, text + out.stderr
    for pattern in ["grip_trajectory_schema=numi.grip.trajectory.v3",
                    "attachment_generations=3 selection_mode=nearest_cuff_patch", "regrab_count=2",
                    "patch_selection_count=2", "maximum_patch_ring_shift=12", "selected_patch_center_ring=24",
                    "patch_particles_unique=true patch_topology_exact=true", "deterministic=true", "result=PASS"]:
        assert re.search(pattern, text), pattern


@pytest.mark.gpu
def test_cli_regrab_keys():
    out = _run(CPU_ARGS + ["--grip-trajectory", os.path.join(FIX, "synthetic-regrab.csv")])
    text = out.stdout
    assert out.returncode == 0, text + out.stderr
    for pattern in ["grip_trajectory_schema=numi.grip.trajectory.v2", "attachment_generations=3",
                    "regrab_count=2", "inactive_grip_substeps=[1-9][0-9]*", "deterministic=true", "result=PASS"]:
        assert re.search(pattern, text), pattern


@pytest.mark.gpu
def test_cli_rotation_changes_state():
    ident = _run(CPU_ARGS + ["--grip-trajectory", os.path.join(FIX, "synthetic-identity.csv")])
    rot = _run(CPU_ARGS + ["--grip-trajectory", os.path.join(FIX, "synthetic-rotation.csv")])
    assert ident.returncode == 0 and rot.returncode == 0, ident.stdout + rot.stdout
    assert re.search("deterministic=true", ident.stdout) and re.search("result=PASS", ident.stdout)
    assert re.search("maximum_rotation_radians=0.0349", rot.stdout) and re.search("result=PASS", rot.stdout)
    h1 = re.search("state_hash=0x[0-9a-f]+", ident.stdout).group(0)
    h2 = re.search("state_hash=0x[0-9a-f]+", rot.stdout).group(0)
    assert h1 != h2


@pytest.mark.gpu
def test_cli_material_defaults_parity():
    """CheckClothMaterialParity.cmake (cpu kind): the authored defaults and
    the explicit default artifact give the same state hashes."""
    args = ["--steps", "1", "--substeps", "1", "--iterations", "1", "--replays", "2"]
    a = _run(args)
    b = _run(args + ["--material", os.path.join(FIX, "default-material.txt")])
    assert a.returncode == 0 and b.returncode == 0, a.stdout + a.stderr + b.stdout + b.stderr
    ha = re.findall("state_hash=0x[0-9a-f]+", a.stdout)
    hb = re.findall("state_hash=0x[0-9a-f]+", b.stdout)
    assert ha and ha == hb
    assert "material_artifact_loaded=true" in b.stdout
