"""Calibration qualification and the material artifact
(tools/cloth_calibration.cpp, `numi-solver-cloth-calibration`).

The reference fits log-scale parameter changes to observations by weighted
linear least squares on their sensitivities (`dlog_<name>` columns, there
made by central finite differences outside the tool), qualifies the fit
against held-out observations and bounds, and only then writes the
`numi.cloth.material.v1` artifact.  This module restates that tool: the
same CSV contracts and errors, the same column-normalised normal equations
with a ridge, Jacobi eigenvalues for rank and condition, Gauss-Jordan
elimination, the same gates and the same report and material text (fixed,
12 decimals), and the same exit codes (0 qualified, 1 not qualified, 2
error).  `numi_cloth.calibrate.adjoint_observations` fills the sensitivity
columns from the adjoint instead of finite differences.

Command line: python -m numi_cloth.qualify --parameters FILE
--observations FILE [--report FILE] [--material-output FILE] [--ridge L]
[--max-condition K] [--max-calibration-rmse-z Z] [--max-heldout-rmse-z Z]
[--max-heldout-max-z Z] [--allow-no-heldout-improvement]
"""
from __future__ import annotations

import math
import sys
from dataclasses import dataclass, field

RESULT_SCHEMA = "numi.cloth.calibration.result.v1"   # tools/cloth_calibration.cpp:21
MATERIAL_SCHEMA = "numi.cloth.material.v1"          # tools/cloth_calibration.cpp:22


class QualifyError(RuntimeError):
    """An input the reference tool rejects (it exits 2 with `error: <msg>`)."""


@dataclass
class Parameter:
    name: str
    base: float
    minimum: float
    maximum: float


@dataclass
class Observation:
    trial: str
    heldout: bool
    observable: str
    measured: float
    sigma: float
    baseline: float
    sensitivities: list = field(default_factory=list)


@dataclass
class Options:
    """Thresholds and paths (defaults: tools/cloth_calibration.cpp:51-62)."""
    parameters_path: str = ""
    observations_path: str = ""
    report_path: str = ""
    material_path: str = ""
    ridge: float = 1.0e-10
    maximum_condition: float = 1.0e4
    maximum_calibration_rmse_z: float = 2.0
    maximum_heldout_rmse_z: float = 2.0
    maximum_heldout_absolute_z: float = 4.0
    require_heldout_improvement: bool = True


# ------------------------------------------------------------------ CSV ----

def _trim(s: str) -> str:
    return s.strip(" \t\r\n")


def _parse_row(line: str, number: int) -> list[str]:
    """One CSV row: double-quote quoting with "" escapes, fields trimmed
    (parseCSVRow, tools/cloth_calibration.cpp:78-115)."""
    fields, cur, quoted, i = [], [], False, 0
    while i < len(line):
        ch = line[i]
        if quoted:
            if ch == '"':
                if i + 1 < len(line) and line[i + 1] == '"':
                    cur.append('"')
                    i += 1
                else:
                    quoted = False
            else:
                cur.append(ch)
        elif ch == '"':
            if cur:
                raise QualifyError(f"CSV quote must begin a field at line {number}")
            quoted = True
        elif ch == ",":
            fields.append(_trim("".join(cur)))
            cur = []
        else:
            cur.append(ch)
        i += 1
    if quoted:
        raise QualifyError(f"unterminated CSV quote at line {number}")
    fields.append(_trim("".join(cur)))
    return fields


def read_csv(text: str, path: str = "") -> list[list[str]]:
    """Rows of a CSV text; blank and '#' lines skipped (readCSV :131-150)."""
    rows = []
    for number, line in enumerate(text.split("\n"), start=1):
        if number == len(text.split("\n")) and line == "":
            break
        stripped = _trim(line)
        if not stripped or stripped.startswith("#"):
            continue
        rows.append(_parse_row(line, number))
    if not rows:
        raise QualifyError(f"CSV has no rows: {path}")
    return rows


def _finite(text: str, what: str) -> float:
    try:
        v = float(text)
    except ValueError:
        raise QualifyError(f"invalid number for {what}: {text}") from None
    if not math.isfinite(v):
        raise QualifyError(f"non-finite or trailing data for {what}: {text}")
    return v


def parse_parameters(text: str, path: str = "") -> list[Parameter]:
    """The parameter contract name,base,minimum,maximum (loadParameters :177-211)."""
    rows = read_csv(text, path)
    if rows[0] != ["name", "base", "minimum", "maximum"]:
        raise QualifyError("parameter CSV header must be name,base,minimum,maximum")
    out, names = [], set()
    for row in rows[1:]:
        if len(row) != 4:
            raise QualifyError("parameter CSV row has wrong field count")
        p = Parameter(row[0], _finite(row[1], "base"), _finite(row[2], "minimum"), _finite(row[3], "maximum"))
        if not p.name or p.name in names:
            raise QualifyError("parameter names must be nonempty and unique")
        names.add(p.name)
        if not (p.minimum > 0.0 and p.minimum < p.base < p.maximum):
            raise QualifyError(f"parameter bounds must satisfy 0 < minimum < base < maximum for {p.name}")
        out.append(p)
    if not out:
        raise QualifyError("parameter CSV has no parameters")
    return out


def parse_observations(text: str, params: list[Parameter], path: str = "") -> list[Observation]:
    """Observations with one dlog_ sensitivity per parameter; a trial stays in
    one split; trial and observable pairs are unique (loadObservations
    :213-297)."""
    rows = read_csv(text, path)
    head = rows[0]
    if len(head) != 6 + len(params):
        raise QualifyError("observation CSV must have six fixed fields and one dlog_ sensitivity per parameter")
    for k, name in enumerate(("trial_id", "split", "observable", "measured", "sigma", "baseline")):
        if head[k] != name:
            raise QualifyError(f"observation CSV fixed header mismatch at {name}")
    column = {}
    for c in range(6, len(head)):
        if not head[c].startswith("dlog_"):
            raise QualifyError("sensitivity columns must start with dlog_")
        if head[c][5:] in column:
            raise QualifyError(f"duplicate sensitivity column: {head[c]}")
        column[head[c][5:]] = c
    for p in params:
        if p.name not in column:
            raise QualifyError(f"missing dlog_ sensitivity for {p.name}")
    out, pairs, splits = [], set(), {}
    for row in rows[1:]:
        if len(row) != len(head):
            raise QualifyError("observation CSV row has wrong field count")
        if row[1] not in ("calibration", "heldout"):
            raise QualifyError("split must be calibration or heldout")
        o = Observation(row[0], row[1] == "heldout", row[2], _finite(row[3], "measured"), _finite(row[4], "sigma"),
                        _finite(row[5], "baseline"))
        if not o.trial or not o.observable or not (o.sigma > 0.0):
            raise QualifyError("trial, observable, and positive sigma are required")
        if splits.setdefault(o.trial, o.heldout) != o.heldout:
            raise QualifyError(f"trial IDs may not cross calibration and heldout splits: {o.trial}")
        if (o.trial, o.observable) in pairs:
            raise QualifyError(f"duplicate trial and observable pair: {o.trial}")
        pairs.add((o.trial, o.observable))
        o.sensitivities = [_finite(row[column[p.name]], "sensitivity") for p in params]
        out.append(o)
    return out


# -------------------------------------------------------------- algebra ----

def jacobi_eigenvalues(m: list[list[float]]) -> list[float]:
    """Eigenvalues of a symmetric matrix by cyclic-free Jacobi rotations on
    the largest off-diagonal entry until it is at most 1e-14, ascending
    (symmetricEigenvalues :299-350; Jacobi 1846)."""
    a = [list(r) for r in m]
    n = len(a)
    if n == 0:
        return []
    for _ in range(100 * n * n):
        p = q = 0
        big = 0.0
        for r in range(n):
            for c in range(r + 1, n):
                if abs(a[r][c]) > big:
                    big, p, q = abs(a[r][c]), r, c
        if big <= 1.0e-14:
            break
        ang = 0.5 * math.atan2(2.0 * a[p][q], a[q][q] - a[p][p])
        co, si = math.cos(ang), math.sin(ang)
        for k in range(n):
            if k in (p, q):
                continue
            fp, fq = a[k][p], a[k][q]
            a[k][p] = a[p][k] = co * fp - si * fq
            a[k][q] = a[q][k] = si * fp + co * fq
        dp, dq, off = a[p][p], a[q][q], a[p][q]
        a[p][p] = co * co * dp - 2.0 * si * co * off + si * si * dq
        a[q][q] = si * si * dp + 2.0 * si * co * off + co * co * dq
        a[p][q] = a[q][p] = 0.0
    return sorted(a[k][k] for k in range(n))


def gauss_jordan(m: list[list[float]], rhs: list[float]) -> list[float]:
    """Gauss-Jordan elimination with partial pivoting (solveLinearSystem
    :352-384)."""
    a = [list(r) for r in m]
    b = list(rhs)
    n = len(a)
    for col in range(n):
        piv = col
        for r in range(col + 1, n):
            if abs(a[r][col]) > abs(a[piv][col]):
                piv = r
        if abs(a[piv][col]) <= 1.0e-14:
            raise QualifyError("calibration normal matrix is singular")
        a[piv], a[col] = a[col], a[piv]
        b[piv], b[col] = b[col], b[piv]
        div = a[col][col]
        for e in range(col, n):
            a[col][e] /= div
        b[col] /= div
        for r in range(n):
            if r == col:
                continue
            f = a[r][col]
            for e in range(col, n):
                a[r][e] -= f * a[col][e]
            b[r] -= f * b[col]
    return b


def evaluate(obs: list[Observation], heldout: bool, deltas: list[float]) -> tuple[float, float]:
    """(RMS z, max |z|) of the linear prediction baseline + S delta over one
    split (evaluate :386-411)."""
    sq, mx, count = 0.0, 0.0, 0
    for o in obs:
        if o.heldout != heldout:
            continue
        pred = o.baseline
        for k, d in enumerate(deltas):
            pred += o.sensitivities[k] * d
        z = (pred - o.measured) / o.sigma
        sq += z * z
        mx = max(mx, abs(z))
        count += 1
    if count == 0:
        return math.inf, math.inf
    return math.sqrt(sq / count), mx


def fnv1a64(data: bytes) -> int:
    """FNV-1a over 64 bits with the tool's offset basis 1469598103934665603
    (fnv1a64 :168-175; the published basis is 14695981039346656037)."""
    h = 1469598103934665603
    for byte in data:
        h ^= byte
        h = (h * 1099511628211) & 0xFFFFFFFFFFFFFFFF
    return h


# ----------------------------------------------------------------- fit ----

@dataclass
class Result:
    parameters: list
    deltas: list
    calibration_rows: int
    heldout_rows: int
    rank: int
    condition: float
    baseline_calibration: tuple
    fitted_calibration: tuple
    baseline_heldout: tuple
    fitted_heldout: tuple
    bounds_qualified: bool
    heldout_improved: bool
    qualified: bool
    parameters_hash: int
    observations_hash: int

    def fitted(self) -> dict:
        return {p.name: p.base * math.exp(d) for p, d in zip(self.parameters, self.deltas)}


def fit(parameters_text: bytes, observations_text: bytes, options: Options = Options()) -> Result:
    """The reference run (tools/cloth_calibration.cpp:542-678) on the two
    files' bytes."""
    params = parse_parameters(parameters_text.decode(), options.parameters_path)
    obs = parse_observations(observations_text.decode(), params, options.observations_path)
    cal = [o for o in obs if not o.heldout]
    held = len(obs) - len(cal)
    if len(cal) < len(params):
        raise QualifyError("calibration rows must be at least the parameter count")
    if held < 2:
        raise QualifyError("at least two heldout rows are required")
    n = len(params)
    design = [[o.sensitivities[c] / o.sigma for c in range(n)] for o in cal]
    target = [(o.measured - o.baseline) / o.sigma for o in cal]
    norms = [0.0] * n
    for row in design:
        for c in range(n):
            norms[c] += row[c] * row[c]
    norms = [math.sqrt(v) for v in norms]
    if any(not (v > 0.0) for v in norms):
        raise QualifyError("each parameter needs nonzero calibration sensitivity")
    gram = [[0.0] * n for _ in range(n)]
    rhs = [0.0] * n
    for r, row in enumerate(design):
        for i in range(n):
            vi = row[i] / norms[i]
            rhs[i] += vi * target[r]
            for j in range(n):
                gram[i][j] += vi * row[j] / norms[j]
    eig = jacobi_eigenvalues(gram)
    top = eig[-1]
    tol = top / (options.maximum_condition * options.maximum_condition)
    rank = sum(1 for v in eig if v > tol)
    cond = math.sqrt(top / eig[0]) if eig[0] > 0.0 else math.inf
    deltas = [0.0] * n
    if rank == n and cond <= options.maximum_condition:
        reg = [list(r) for r in gram]
        for i in range(n):
            reg[i][i] += options.ridge
        sol = gauss_jordan(reg, rhs)
        deltas = [sol[i] / norms[i] for i in range(n)]
    zero = [0.0] * n
    bc, fc = evaluate(obs, False, zero), evaluate(obs, False, deltas)
    bh, fh = evaluate(obs, True, zero), evaluate(obs, True, deltas)
    bounds = all(p.minimum <= p.base * math.exp(d) <= p.maximum for p, d in zip(params, deltas))
    improved = fh[0] + 1.0e-12 < bh[0]
    qualified = (rank == n and cond <= options.maximum_condition and bounds and
                 fc[0] <= options.maximum_calibration_rmse_z and fh[0] <= options.maximum_heldout_rmse_z and
                 fh[1] <= options.maximum_heldout_absolute_z and
                 (not options.require_heldout_improvement or improved))
    return Result(params, deltas, len(cal), held, rank, cond, bc, fc, bh, fh, bounds, improved, qualified,
                  fnv1a64(parameters_text), fnv1a64(observations_text))


def _f(v: float) -> str:
    """A double as std::fixed with 12 decimals."""
    if math.isinf(v):
        return "inf" if v > 0 else "-inf"
    if math.isnan(v):
        return "nan" if math.copysign(1.0, v) > 0 else "-nan"
    return f"{v:.12f}"


def _b(v: bool) -> str:
    return "true" if v else "false"


def report(r: Result, options: Options = Options()) -> str:
    """The result text (formatReport :487-528)."""
    lines = [
        f"schema={RESULT_SCHEMA}",
        f"parameters_hash=0x{r.parameters_hash:x}",
        f"observations_hash=0x{r.observations_hash:x}",
        f"parameter_count={len(r.parameters)} calibration_rows={r.calibration_rows} heldout_rows={r.heldout_rows}",
        f"rank={r.rank} condition_number={_f(r.condition)} maximum_condition={_f(options.maximum_condition)}",
        f"baseline_calibration_rmse_z={_f(r.baseline_calibration[0])} "
        f"fitted_calibration_rmse_z={_f(r.fitted_calibration[0])} "
        f"maximum_calibration_rmse_z={_f(options.maximum_calibration_rmse_z)}",
        f"baseline_heldout_rmse_z={_f(r.baseline_heldout[0])} fitted_heldout_rmse_z={_f(r.fitted_heldout[0])} "
        f"fitted_heldout_max_z={_f(r.fitted_heldout[1])} maximum_heldout_rmse_z={_f(options.maximum_heldout_rmse_z)} "
        f"maximum_heldout_max_z={_f(options.maximum_heldout_absolute_z)}",
        f"heldout_improved={_b(r.heldout_improved)} improvement_required={_b(options.require_heldout_improvement)} "
        f"bounds_qualified={_b(r.bounds_qualified)}",
    ]
    for p, d in zip(r.parameters, r.deltas):
        lines.append(f"parameter={p.name} base={_f(p.base)} fitted={_f(p.base * math.exp(d))} "
                     f"minimum={_f(p.minimum)} maximum={_f(p.maximum)} log_delta={_f(d)}")
    lines.append(f"qualified={_b(r.qualified)}")
    lines.append(f"result={'PASS' if r.qualified else 'FAIL'}")
    return "\n".join(lines) + "\n"


def material(r: Result) -> str:
    """The numi.cloth.material.v1 artifact of a qualified fit (:665-677);
    refused for an unqualified one."""
    if not r.qualified:
        raise QualifyError("refusing material output from unqualified calibration")
    lines = [f"schema={MATERIAL_SCHEMA}", f"parameters_hash=0x{r.parameters_hash:x}",
             f"observations_hash=0x{r.observations_hash:x}"]
    lines += [f"{p.name}={_f(p.base * math.exp(d))}" for p, d in zip(r.parameters, r.deltas)]
    return "\n".join(lines) + "\n"


# ----------------------------------------------------------------- CLI ----

def parse_options(argv: list[str]) -> Options:
    """The tool's flags (parseOptions :413-484)."""
    o = Options()
    paths = {"--parameters": "parameters_path", "--observations": "observations_path", "--report": "report_path",
             "--material-output": "material_path"}
    numbers = {"--ridge": ("ridge", "ridge"), "--max-condition": ("maximum_condition", "max-condition"),
               "--max-calibration-rmse-z": ("maximum_calibration_rmse_z", "max-calibration-rmse-z"),
               "--max-heldout-rmse-z": ("maximum_heldout_rmse_z", "max-heldout-rmse-z"),
               "--max-heldout-max-z": ("maximum_heldout_absolute_z", "max-heldout-max-z")}
    i = 0
    while i < len(argv):
        a = argv[i]
        if a in paths or a in numbers:
            if i + 1 >= len(argv):
                raise QualifyError(f"{a} requires a value")
            i += 1
            if a in paths:
                setattr(o, paths[a], argv[i])
            else:
                setattr(o, numbers[a][0], _finite(argv[i], numbers[a][1]))
        elif a == "--allow-no-heldout-improvement":
            o.require_heldout_improvement = False
        else:
            raise QualifyError(f"unknown argument: {a}")
        i += 1
    if not o.parameters_path or not o.observations_path:
        raise QualifyError("--parameters and --observations are required")
    if (o.ridge < 0.0 or o.maximum_condition <= 1.0 or o.maximum_calibration_rmse_z <= 0.0 or
            o.maximum_heldout_rmse_z <= 0.0 or o.maximum_heldout_absolute_z <= 0.0):
        raise QualifyError("qualification thresholds are invalid")
    return o


def _read(path: str) -> bytes:
    try:
        with open(path, "rb") as f:
            return f.read()
    except OSError:
        raise QualifyError(f"cannot open {path}") from None


def _write(path: str, text: str):
    try:
        with open(path, "w") as f:
            f.write(text)
    except OSError:
        raise QualifyError(f"cannot create {path}") from None


def main(argv: list[str] | None = None, stdout=None, stderr=None) -> int:
    """Run as the reference tool: the report on stdout (and --report), the
    material with --material-output when qualified; 0 qualified, 1 not, 2
    error."""
    stdout = stdout or sys.stdout
    stderr = stderr or sys.stderr
    try:
        o = parse_options(list(sys.argv[1:] if argv is None else argv))
        r = fit(_read(o.parameters_path), _read(o.observations_path), o)
        text = report(r, o)
        stdout.write(text)
        if o.report_path:
            _write(o.report_path, text)
        if o.material_path:
            _write(o.material_path, material(r))
        return 0 if r.qualified else 1
    except QualifyError as e:
        stderr.write(f"error: {e}\n")
        return 2


if __name__ == "__main__":
    sys.exit(main())
