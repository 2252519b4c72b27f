"""Gradient-based calibration of cloth compliances and damping.

The reference fits its material artifact by a linearised least-squares step
on sensitivities measured outside the simulator by central finite
differences (tools/cloth_calibration.cpp:542-683,
docs/CLOTH_SPECIMEN_CALIBRATION.md:52-82).  Here the sensitivities come from
the adjoint: every candidate parameter set is a cloth of one batch, the
batch runs its forward and adjoint together (numi_cloth_batch_rollout_grad),
and Adam descends on the log-compliances and the damping of every
candidate at once.
"""
from __future__ import annotations

import time

import numpy as np

from . import ClothBatch, ClothSolver, Schedule

# Calibrated parameters of the produce bag: (constraint family, material
# field); the bag's records of a family carry one of these compliances.
BAG_PARAMS = (
    ("distance", "axialBodyComplianceMPerN"),
    ("distance", "axialCuffComplianceMPerN"),
    ("knot", "knotCompliance"),
    ("bend", "bendBodyComplianceMPerN"),
    ("bend", "bendCuffComplianceMPerN"),
    ("grip", "gripComplianceMPerN"),
)
FAMILIES = ("distance", "knot", "bend", "grip")


def group_index(values: np.ndarray, params=BAG_PARAMS) -> list[int]:
    """Gradient slot of each parameter: groups are the distinct compliance
    values of each family, ascending, family by family (the order of
    numi_cloth_compliance_groups)."""
    slots, base = [], 0
    order = {}
    for fam in FAMILIES:
        vals = sorted({float(values[p]) for p, (f, _) in enumerate(params) if f == fam})
        for k, v in enumerate(vals):
            order[(fam, v)] = base + k
        base += len(vals)
    for p, (fam, _) in enumerate(params):
        slots.append(order[(fam, float(values[p]))])
    return slots


class Adam:
    """Adam (Kingma and Ba 2015) on an array of parameters."""

    def __init__(self, shape, lr: float, beta1: float = 0.9, beta2: float = 0.999, eps: float = 1e-12):
        self.lr, self.b1, self.b2, self.eps = lr, beta1, beta2, eps
        self.m = np.zeros(shape)
        self.v = np.zeros(shape)
        self.t = 0

    def step(self, x: np.ndarray, g: np.ndarray) -> np.ndarray:
        self.t += 1
        self.m = self.b1 * self.m + (1 - self.b1) * g
        self.v = self.b2 * self.v + (1 - self.b2) * g * g
        mh = self.m / (1 - self.b1 ** self.t)
        vh = self.v / (1 - self.b2 ** self.t)
        return x - self.lr * mh / (np.sqrt(vh) + self.eps)


class Calibration:
    """Candidates of one scene as a batch; every evaluation restores the
    initial state, applies each candidate's parameters and runs the batched
    forward + adjoint."""

    def __init__(self, scenes, configs: np.ndarray, schedule: Schedule, tracked, targets, loss_every: int,
                 base_values: np.ndarray, params=BAG_PARAMS, checkpoint_every: int = 8, stream: int | None = None):
        self.params = params
        self.solvers = [ClothSolver(s) for s in scenes]
        for sv in self.solvers:
            if stream is not None:
                sv.set_stream(stream)
            sv.snapshot(0)
        self.batch = ClothBatch(self.solvers)
        if stream is not None:
            self.batch.set_stream(stream)
        n = len(self.solvers)
        self.configs = np.ascontiguousarray(np.broadcast_to(configs, (n,) + configs.shape))
        self.schedule = schedule
        self.tracked = np.ascontiguousarray(tracked, np.uint32)
        self.targets = np.ascontiguousarray(np.broadcast_to(targets, (n,) + targets.shape))
        self.loss_every = loss_every
        self.checkpoint_every = checkpoint_every
        self.values = np.tile(np.asarray(base_values, np.float32), (n, 1))   # current float32 compliances
        self.rollout_seconds = 0.0
        self.rollouts = 0

    def close(self):
        self.batch.close()
        for sv in self.solvers:
            sv.close()

    def _apply(self, logc: np.ndarray, damping: np.ndarray):
        for k, sv in enumerate(self.solvers):
            new = np.exp(logc[k]).astype(np.float32)
            for p, (fam, _) in enumerate(self.params):
                if new[p] == self.values[k, p]:
                    continue
                # a value shared with another parameter of the family would
                # merge their records: step one ulp away
                others = [self.values[k, q] for q, (f, _) in enumerate(self.params) if f == fam and q != p]
                while new[p] in others:
                    new[p] = np.nextafter(new[p], np.float32(np.inf))
                sv.replace_compliance(fam, float(self.values[k, p]), float(new[p]))
                self.values[k, p] = new[p]
            sv.set_damping(float(damping[k]))

    def evaluate(self, logc: np.ndarray, damping: np.ndarray) -> tuple[np.ndarray, np.ndarray, np.ndarray, np.ndarray]:
        """Loss, d loss / d log-compliance [n, params], d loss / d damping, and
        the non-smooth event counts of every candidate."""
        for sv in self.solvers:
            sv.restore(0)
        self._apply(logc, damping)
        t0 = time.perf_counter()
        r = self.batch.rollout_grad(self.configs, self.schedule, self.tracked, self.targets, self.loss_every,
                                    self.checkpoint_every)
        self.rollout_seconds += time.perf_counter() - t0
        self.rollouts += 1
        g = np.zeros_like(logc)
        for k in range(len(self.solvers)):
            slots = group_index(self.values[k], self.params)
            g[k] = [r["grads"][k][s] for s in slots]
        return r["loss"], g, r["damping"], r["nonsmooth"]

    def fit(self, logc0: np.ndarray, damping0: np.ndarray, steps: int, lr: float = 0.1, lr_damping: float = 0.005,
            damping_max: float = 1.0, frozen=None) -> dict:
        """Adam on every candidate's log-compliances and damping; `frozen`
        (one flag per parameter, damping last) keeps those at their start."""
        logc, damp = logc0.astype(np.float64).copy(), damping0.astype(np.float64).copy()
        opt_c, opt_d = Adam(logc.shape, lr), Adam(damp.shape, lr_damping)
        hold = np.zeros(logc.shape[1] + 1, bool) if frozen is None else np.asarray(frozen, bool)
        history = []
        loss = None
        for _ in range(steps):
            loss, g, gd, rough = self.evaluate(logc, damp)
            history.append(loss.copy())
            g = np.where(hold[None, :-1], 0.0, g)
            logc = opt_c.step(logc, g)
            if not hold[-1]:
                damp = np.clip(opt_d.step(damp, gd), 0.0, damping_max)
        final, _, _, rough = self.evaluate(logc, damp)
        history.append(final.copy())
        return {"logc": logc, "damping": damp, "loss": final, "history": np.array(history), "nonsmooth": rough}


def adjoint_observations(solver: ClothSolver, configs: np.ndarray, schedule: Schedule, observables,
                         parameters=None, split: str = "calibration", trial: str = "trial", measured=None,
                         sigma: float = 1.0, checkpoint_every: int = 8) -> tuple[list[str], str]:
    """Rows of the calibration qualifier's observation CSV
    (numi_cloth.qualify; tools/cloth_calibration.cpp:213-297) for one trial,
    with the `dlog_` sensitivity columns made by the adjoint instead of
    central finite differences.

    observables: (name, particle, axis) triples, each the particle's axis
    coordinate at the end of the rollout; parameters: (name, [compliance
    group indices]) pairs, default one per compliance group, each the log
    scale of the groups' compliances.  baseline is the forward value, measured
    the given values (default: the baseline), sigma the given one.  The
    solver state is left as it was.  Returns (parameter names, CSV text).

    One reverse sweep per observable: the rollout loss is the squared
    distance of the tracked particle to a target, and with the target half a
    unit below the forward position along the axis, d loss / d theta is
    exactly d coordinate / d theta."""
    configs = np.ascontiguousarray(configs)
    groups = solver.compliance_groups()
    if parameters is None:
        parameters = [(f"{fam}_{value:.6g}", [g]) for g, (fam, value) in enumerate(groups)]
    n = len(configs)
    slot = 1
    solver.snapshot(slot)
    solver.step(configs, schedule)
    x = solver.particles()["positionAndInverseMass"][:, :3].astype(np.float64)
    solver.restore(slot)
    rows = []
    for k, (name, particle, axis) in enumerate(observables):
        target = x[particle].copy()
        target[axis] -= 0.5
        r = solver.rollout_grad(configs, schedule, np.array([particle], np.uint32), target.reshape(1, 1, 3), n,
                                checkpoint_every)
        solver.restore(slot)
        sens = [float(sum(r["grads"][g] for g in gs)) for _, gs in parameters]
        base = float(x[particle, axis])
        meas = base if measured is None else float(measured[k])
        rows.append(",".join([trial, split, name, repr(meas), repr(float(sigma)), repr(base)] +
                             [repr(v) for v in sens]))
    names = [p for p, _ in parameters]
    header = "trial_id,split,observable,measured,sigma,baseline" + "".join(f",dlog_{p}" for p in names)
    return names, header + "\n" + "\n".join(rows) + "\n"


def tracked_trajectory(scene, configs: np.ndarray, schedule: Schedule, tracked, loss_every: int, values,
                       damping: float, base_values, params=BAG_PARAMS, stream: int | None = None) -> np.ndarray:
    """Positions of the tracked particles after every loss_every substeps
    (the observations of the fit), forward only, for compliances `values`
    (one per parameter) and `damping`."""
    sv = ClothSolver(scene)
    try:
        if stream is not None:
            sv.set_stream(stream)
        current = np.asarray(base_values, np.float32).copy()
        for p, (fam, _) in enumerate(params):
            new = np.float32(values[p])
            if new == current[p]:
                continue
            # never step onto another parameter's value of the family (their
            # records would merge)
            others = [current[q] for q, (f, _) in enumerate(params) if f == fam and q != p]
            while new in others:
                new = np.nextafter(new, np.float32(np.inf))
            sv.replace_compliance(fam, float(current[p]), float(new))
            current[p] = new
        sv.set_damping(float(damping))
        out = []
        for k in range(len(configs) // loss_every):
            sv.step(configs[k * loss_every:(k + 1) * loss_every], schedule)
            out.append(sv.particles()["positionAndInverseMass"][np.asarray(tracked), :3].astype(np.float64))
        return np.stack(out)
    finally:
        sv.close()


def sensitivities(scene, configs: np.ndarray, schedule: Schedule, tracked, loss_every: int, log_values,
                  damping: float, base_values, params=BAG_PARAMS, step: float = 0.1, damping_step: float = 0.002,
                  stream: int | None = None) -> np.ndarray:
    """Central-difference Jacobian of the flattened observations with
    respect to each log-compliance (step in log) and the damping (last
    column), at the given parameters, from forward runs."""
    cols = []
    for p in range(len(params) + 1):
        run = []
        for sign in (1.0, -1.0):
            lv = np.array(log_values, np.float64)
            dmp = damping
            if p < len(params):
                lv[p] += sign * step
            else:
                dmp = max(0.0, damping + sign * damping_step)
            run.append(tracked_trajectory(scene, configs, schedule, tracked, loss_every, np.exp(lv), dmp,
                                          base_values, params, stream).ravel())
        h = 2.0 * step if p < len(params) else (max(0.0, damping + damping_step) - max(0.0, damping - damping_step))
        cols.append((run[0] - run[1]) / h)
    return np.stack(cols, axis=1)


def identifiable(jacobian: np.ndarray, sigma: float, max_condition: float = 1.0e4, min_norm: float = 1.0):
    """Which parameters the observations can determine, by the calibration
    qualifier's tests (tools/cloth_calibration.cpp:301-393, numi_cloth.qualify):
    each kept parameter moves the observations by at least `min_norm` noise
    units (sigma, metres) per unit of its parameter, and the Gram matrix of
    the kept column-normalised sensitivities has full rank and a condition
    number (square root of the eigenvalue ratio, Jacobi eigenvalues) at most
    `max_condition`; of several sets that pass, the largest with the lowest
    condition.  Returns (keep flags, condition number of the kept set)."""
    from itertools import combinations

    from .qualify import jacobi_eigenvalues

    design = np.asarray(jacobian, np.float64) / sigma
    norms = np.sqrt((design * design).sum(axis=0))
    able = [j for j in range(design.shape[1]) if norms[j] >= min_norm]
    for size in range(len(able), 0, -1):
        best = None
        for keep in combinations(able, size):
            cols = design[:, list(keep)] / norms[list(keep)]
            eig = jacobi_eigenvalues((cols.T @ cols).tolist())
            if eig[0] <= 0.0:
                continue
            cond = float(np.sqrt(eig[-1] / eig[0]))
            if cond <= max_condition and (best is None or cond < best[1]):
                best = (keep, cond)
        if best is not None:
            flags = np.zeros(design.shape[1], bool)
            flags[list(best[0])] = True
            return flags, best[1]
    return np.zeros(design.shape[1], bool), float("inf")
