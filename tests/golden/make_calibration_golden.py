"""Golden outputs of the reference calibration qualifier.

Copies the reference's synthetic calibration fixtures (data files) and its
19-parameter contract into tests/golden/calibration/, writes the
full-contract unit observations its runtime check builds
(cmake/CheckClothCalibrationRuntime.cmake), runs the compiled reference
tool (oracle/_ref/cloth_calibration, built by oracle/ref.mk from
tools/cloth_calibration.cpp) on every case and records stdout, stderr, the
exit code and the material file in cases.json.

    make -f oracle/ref.mk all && python tests/golden/make_calibration_golden.py
"""
import json
import os
import shutil
import subprocess
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = os.environ.get("NUMI_CLOTH_REFERENCE", "/root/reference")
OUT = os.path.join(HERE, "calibration")
TOOL = os.path.join(ROOT, "oracle", "_ref", "cloth_calibration")

INPUTS = ["parameters.csv", "qualified-observations.csv", "heldout-failure-observations.csv",
          "rank-deficient-parameters.csv", "rank-deficient-observations.csv", "trial-leakage-observations.csv"]


def full_contract():
    """The runtime check's observations: one calibration and one heldout
    unit row per parameter of the 19-parameter contract."""
    names = [l.split(",")[0] for l in open(os.path.join(OUT, "cloth-parameters-v1.csv")).read().splitlines()[1:] if l]
    text = "trial_id,split,observable,measured,sigma,baseline" + "".join(f",dlog_{n}" for n in names) + "\n"
    for r, n in enumerate(names):
        sens = "".join(",1.0" if c == r else ",0.0" for c in range(len(names)))
        text += f"cal_{n},calibration,unit_{n},0.0,1.0,0.0{sens}\nheldout_{n},heldout,unit_{n},0.0,1.0,0.0{sens}\n"
    open(os.path.join(OUT, "full-contract-observations.csv"), "w").write(text)


CASES = {
    "qualified": ["--parameters", "parameters.csv", "--observations", "qualified-observations.csv", "MATERIAL"],
    "qualified_options": ["--parameters", "parameters.csv", "--observations", "qualified-observations.csv",
                          "--ridge", "0.001", "--max-condition", "100", "--max-calibration-rmse-z", "3"],
    "heldout_failure": ["--parameters", "parameters.csv", "--observations", "heldout-failure-observations.csv"],
    "heldout_failure_material": ["--parameters", "parameters.csv", "--observations",
                                 "heldout-failure-observations.csv", "MATERIAL"],
    "heldout_failure_allowed": ["--parameters", "parameters.csv", "--observations",
                                "heldout-failure-observations.csv", "--allow-no-heldout-improvement"],
    "rank_deficient": ["--parameters", "rank-deficient-parameters.csv", "--observations",
                       "rank-deficient-observations.csv"],
    "trial_leakage": ["--parameters", "parameters.csv", "--observations", "trial-leakage-observations.csv"],
    "full_contract": ["--parameters", "cloth-parameters-v1.csv", "--observations", "full-contract-observations.csv",
                      "--allow-no-heldout-improvement", "MATERIAL"],
    "bad_threshold": ["--parameters", "parameters.csv", "--observations", "qualified-observations.csv",
                      "--max-condition", "1"],
    "missing_flag": ["--parameters", "parameters.csv"],
}


def main():
    os.makedirs(OUT, exist_ok=True)
    for name in INPUTS:
        shutil.copyfile(os.path.join(REF, "calibration", "synthetic", name), os.path.join(OUT, name))
    shutil.copyfile(os.path.join(REF, "calibration", "cloth-parameters-v1.csv"),
                    os.path.join(OUT, "cloth-parameters-v1.csv"))
    full_contract()
    cases = {}
    with tempfile.TemporaryDirectory() as tmp:
        for case, args in CASES.items():
            material = os.path.join(tmp, case + ".material")
            argv = []
            for a in args:
                argv += ["--material-output", material] if a == "MATERIAL" else [a]
            p = subprocess.run([TOOL] + argv, cwd=OUT, capture_output=True, text=True)
            cases[case] = {"args": args, "rc": p.returncode, "stdout": p.stdout, "stderr": p.stderr,
                           "material": open(material).read() if os.path.exists(material) else None}
    json.dump(cases, open(os.path.join(OUT, "cases.json"), "w"), indent=1)
    print({k: v["rc"] for k, v in cases.items()})


if __name__ == "__main__":
    main()
