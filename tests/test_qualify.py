"""Calibration qualification and the numi.cloth.material.v1 artifact
(tools/cloth_calibration.cpp), restated in numi_cloth.qualify: report text,
material text, error messages and exit codes equal the compiled reference
tool's on its own synthetic fixtures and on its 19-parameter runtime
contract (tests/golden/calibration, made by make_calibration_golden.py).
"""
import io
import json
import os

import pytest

from numi_cloth import qualify as q

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "calibration")
CASES = json.load(open(os.path.join(GOLDEN, "cases.json")))


@pytest.mark.parametrize("case", sorted(CASES))
def test_equals_reference_tool(case, tmp_path, monkeypatch):
    want = CASES[case]
    monkeypatch.chdir(GOLDEN)
    material = tmp_path / "material.txt"
    argv = []
    for a in want["args"]:
        argv += ["--material-output", str(material)] if a == "MATERIAL" else [a]
    out, err = io.StringIO(), io.StringIO()
    rc = q.main(argv, stdout=out, stderr=err)
    assert rc == want["rc"]
    assert out.getvalue() == want["stdout"]
    assert err.getvalue() == want["stderr"]
    assert (material.read_text() if material.exists() else None) == want["material"]


def test_jacobi_eigenvalues_known_answer():
    # [[2, 1], [1, 2]] has eigenvalues 1 and 3
    ev = q.jacobi_eigenvalues([[2.0, 1.0], [1.0, 2.0]])
    assert abs(ev[0] - 1.0) < 1e-14 and abs(ev[1] - 3.0) < 1e-14


def test_fnv1a_uses_the_reference_offset_basis():
    """The tool hashes with offset basis 1469598103934665603, one digit
    short of the published FNV-1a basis 14695981039346656037; the
    restatement keeps the tool's (the golden hashes pin it)."""
    assert q.fnv1a64(b"") == 1469598103934665603
    h = (1469598103934665603 ^ ord("a")) * 1099511628211 & 0xFFFFFFFFFFFFFFFF
    assert q.fnv1a64(b"a") == h


def test_material_refused_when_unqualified():
    p = open(os.path.join(GOLDEN, "parameters.csv"), "rb").read()
    o = open(os.path.join(GOLDEN, "heldout-failure-observations.csv"), "rb").read()
    r = q.fit(p, o)
    assert not r.qualified
    with pytest.raises(q.QualifyError, match="refusing material output"):
        q.material(r)


# ----------------------------------------------------------------- GPU ----

@pytest.mark.gpu
def test_adjoint_fed_qualification(tmp_path):
    """The qualifier fed by the adjoint (numi_cloth.calibrate.adjoint_observations):
    the dlog_ sensitivities of end-of-rollout particle coordinates to the
    material compliance groups equal FP64 central differences of the oracle
    (eps = 1e-4, within 1e-3 relative in norm, the adjoint tests' bar), and
    measurements synthesised on those sensitivities are fitted back, the fit
    qualifies on held-out trials and the material artifact is written."""
    import numpy as np

    import numi_cloth as nc
    import oracle_py as op
    from numi_cloth.calibrate import adjoint_observations
    from test_adjoint import REL, SCHED, SUBSTEPS, _configs, _scene

    scene = _scene()
    cfg = _configs(scene)
    sched = nc.Schedule.make(**SCHED)
    sv = nc.ClothSolver(scene)
    try:
        groups = sv.compliance_groups()
        params = [(f"{fam}_{k}", [k]) for k, (fam, _) in enumerate(groups) if fam != "grip"]
        cal = [(f"p{p}_{'xyz'[a]}", p, a) for p, a in ((20, 2), (45, 0), (70, 2), (95, 1), (120, 2), (140, 0))]
        held = [(f"p{p}_{'xyz'[a]}", p, a) for p, a in ((33, 2), (110, 2))]
        names, cal_csv = adjoint_observations(sv, cfg, sched, cal, params, "calibration", "cal")
        _, held_csv = adjoint_observations(sv, cfg, sched, held, params, "heldout", "held")
    finally:
        sv.close()

    # sensitivities against FP64 central differences of the oracle
    subs = op.substeps_from_configs(cfg)
    osched = op.schedule_from_abi(sched, op.BATCHED)
    fams = {"distance": "distances", "bend": "bends", "knot": "knots"}

    def coords(g, f):
        osc = op.from_abi(scene)
        fam, value = groups[g]
        arr = getattr(osc, fams[fam])
        sel = arr["compliance"] == np.float64(np.float32(value))
        arr["compliance"][sel] = arr["compliance"][sel] * f
        o = op.Oracle(osc, 64)
        assert o.step(subs[:SUBSTEPS], osched) == 0
        return o.read()["particles"]["x"]

    eps = 1.0e-4
    rows = [l.split(",") for l in cal_csv.strip().split("\n")[1:]]
    adj = np.array([[float(v) for v in r[6:]] for r in rows])
    fd = np.zeros_like(adj)
    for c, (_, gs) in enumerate(params):
        xp, xm = coords(gs[0], np.exp(eps)), coords(gs[0], np.exp(-eps))
        for r, (_, p, a) in enumerate(cal):
            fd[r, c] = (xp[p, a] - xm[p, a]) / (2 * eps)
    print("adjoint dlog_ sensitivities:\n", adj, "\nFP64 central differences:\n", fd)
    assert np.linalg.norm(adj - fd) / np.linalg.norm(fd) <= REL

    # measurements made on the sensitivities from known log changes
    truth = np.array([0.2, -0.15, 0.1][:len(params)])

    def with_measured(csv):
        lines = csv.strip().split("\n")
        out = [lines[0]]
        for line in lines[1:]:
            f = line.split(",")
            s = np.array([float(v) for v in f[6:]])
            f[3] = repr(float(f[5]) + float(s @ truth))
            f[4] = repr(1.0e-6)
            out.append(",".join(f))
        return "\n".join(out) + "\n"

    obs = with_measured(cal_csv) + "\n".join(with_measured(held_csv).split("\n")[1:])
    base = [float(groups[gs[0]][1]) for _, gs in params]
    ptext = "name,base,minimum,maximum\n" + "".join(f"{n},{repr(b)},{repr(b / 10)},{repr(b * 10)}\n"
                                                    for n, b in zip(names, base))
    (tmp_path / "p.csv").write_text(ptext)
    (tmp_path / "o.csv").write_text(obs)
    out, err = io.StringIO(), io.StringIO()
    rc = q.main(["--parameters", str(tmp_path / "p.csv"), "--observations", str(tmp_path / "o.csv"),
                 "--max-condition", "1e6", "--material-output", str(tmp_path / "m.txt")], stdout=out, stderr=err)
    print(out.getvalue(), err.getvalue())
    assert rc == 0 and "qualified=true" in out.getvalue()
    r = q.fit(ptext.encode(), obs.encode(), q.Options(maximum_condition=1e6))
    assert np.allclose(r.deltas, truth, rtol=1e-5, atol=1e-7)
    text = (tmp_path / "m.txt").read_text()
    assert text.startswith("schema=numi.cloth.material.v1\n")
    for n, b, d in zip(names, base, truth):
        assert f"{n}=" in text


def test_material_artifact_loads(tmp_path):
    """The qualified full-contract artifact (19 parameters, the reference
    runtime check's case) loads through the library's material reader, as
    the reference feeds it back to its simulator."""
    import numi_cloth as nc

    text = CASES["full_contract"]["material"]
    path = tmp_path / "material.txt"
    path.write_text(text)
    m = nc.load_material(str(path))
    values = dict(l.split("=", 1) for l in text.strip().split("\n")[3:])
    assert len(values) == 19
    for name, v in values.items():
        head, *rest = name.split("_")
        field = head + "".join(w[:1].upper() + w[1:] for w in rest)   # the record's field name
        assert abs(getattr(m, field) - float(v)) <= 1e-12 * max(1.0, abs(float(v))), name
