"""ctypes binding of the CPU oracle (liboracle.so) - TEST INFRASTRUCTURE.

Imported only by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
leg, as the checker of the B200 path.  Converts the ABI-record scene arrays
of numi_cloth into the oracle's FP64 records.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

PARTICLE = np.dtype(
    [("x", "<f8", 3), ("w", "<f8"), ("prev", "<f8", 3), ("mass", "<f8"), ("v", "<f8", 3), ("vw", "<f8"),
     ("rest", "<f8", 3), ("pad", "<f8")]
)
DISTANCE = np.dtype(
    [("i", "<u4"), ("j", "<u4"), ("colour", "<u4"), ("kind", "<u4"), ("rest", "<f8"), ("compliance", "<f8"),
     ("lambda_", "<f8"), ("maxext", "<f8")]
)
KNOT = np.dtype(
    [("p", "<u4", 4), ("colour", "<u4"), ("pad", "<u4", 3), ("restcos", "<f8"), ("compliance", "<f8"),
     ("lambda_", "<f8"), ("pad2", "<f8")]
)
BEND = np.dtype(
    [("p", "<u4", 3), ("colour", "<u4"), ("restchord", "<f8"), ("restarc", "<f8"), ("compliance", "<f8"),
     ("lambda_", "<f8")]
)
GRIP = np.dtype(
    [("particle", "<u4"), ("gen", "<u4"), ("ring", "<u4"), ("pad", "<u4"), ("offset", "<f8", 3),
     ("compliance", "<f8"), ("lambda_", "<f8", 3), ("capture", "<f8"), ("error", "<f8"), ("pad2", "<f8", 3)]
)
FRUIT = np.dtype(
    [("x", "<f8", 3), ("w", "<f8"), ("prev", "<f8", 3), ("radius", "<f8"), ("v", "<f8", 3),
     ("ground_impulse", "<f8"), ("omega", "<f8", 3), ("pad", "<f8"), ("q", "<f8", 4), ("appearance", "<u4"),
     ("pad2", "<u4", 3)]
)
PAIR = np.dtype([("a", "<u4"), ("b", "<u4"), ("colour", "<u4"), ("stable", "<u4"), ("wn", "<f8", 3), ("ni", "<f8")])
for _dt, _size in ((PARTICLE, 128), (DISTANCE, 48), (KNOT, 64), (BEND, 48), (GRIP, 112), (FRUIT, 176), (PAIR, 48)):
    assert _dt.itemsize == _size, (_dt, _size)


class Params(ctypes.Structure):
    _fields_ = [
        ("radius", ctypes.c_double),
        ("mu_cloth_ground", ctypes.c_double),
        ("mu_self", ctypes.c_double),
        ("mu_pair", ctypes.c_double),
        ("mu_fruit_ground", ctypes.c_double),
        ("rolling", ctypes.c_double),
        ("mu_fruit_yarn", ctypes.c_double),
        ("air", ctypes.c_double * 3),
        ("air_density", ctypes.c_double),
        ("aero", ctypes.c_double * 4),
        ("capture_radius", ctypes.c_double),
        ("hysteresis", ctypes.c_double),
        ("ground", ctypes.c_uint32),
        ("ring_count", ctypes.c_uint32),
        ("patch_half", ctypes.c_uint32),
        ("grid_width", ctypes.c_uint32),
        ("rim_count", ctypes.c_uint32),
        ("bottom_center", ctypes.c_uint32),
        ("pad", ctypes.c_uint32 * 2),
    ]


SUBSTEP = np.dtype(
    [("dt", "<f8"), ("gravity", "<f8", 3), ("grip_target", "<f8", 3), ("grip_q", "<f8", 4), ("grip_active", "<u4"),
     ("grip_gen", "<u4"), ("grip_select", "<u4"), ("pad", "<u4")]
)


class OSchedule(ctypes.Structure):
    _fields_ = [
        (n, ctypes.c_uint32)
        for n in (
            "iterations", "strain_sweeps", "reconcile_passes", "final_passes", "certificate_passes", "early_exit",
            "self_collision", "aerodynamics", "swept_ground", "swept_fruit_yarn", "frictions", "release",
        )
    ] + [("damping", ctypes.c_double), ("mode", ctypes.c_uint32), ("primitive_self", ctypes.c_uint32)]


class OScene(ctypes.Structure):
    _fields_ = [
        ("particles", ctypes.c_void_p), ("n", ctypes.c_uint32),
        ("distances", ctypes.c_void_p), ("d", ctypes.c_uint32),
        ("knots", ctypes.c_void_p), ("k", ctypes.c_uint32),
        ("bends", ctypes.c_void_p), ("b", ctypes.c_uint32),
        ("grips", ctypes.c_void_p), ("g", ctypes.c_uint32),
        ("fruits", ctypes.c_void_p), ("f", ctypes.c_uint32),
        ("pairs", ctypes.c_void_p), ("p", ctypes.c_uint32),
        ("cuff", ctypes.c_void_p), ("rim", ctypes.c_void_p),
        ("local_off", ctypes.c_void_p), ("local_idx", ctypes.c_void_p),
        ("params", ctypes.POINTER(Params)),
    ]


BATCHED, SERIAL, BATCHED_SELF_REFERENCE = 0, 1, 2
_LIB = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib() -> ctypes.CDLL:
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        vp = ctypes.c_void_p
        L.oracle_create.restype = vp
        L.oracle_create.argtypes = [ctypes.c_int, ctypes.POINTER(OScene)]
        L.oracle_destroy.argtypes = [vp]
        L.oracle_step.restype = ctypes.c_uint32
        L.oracle_step.argtypes = [vp, vp, ctypes.c_uint32, ctypes.POINTER(OSchedule)]
        L.oracle_read.argtypes = [vp, vp, vp, vp, vp, vp]
        L.oracle_write.argtypes = [vp, vp, vp]
        L.oracle_write_grips.argtypes = [vp, vp]
        L.oracle_residuals.argtypes = [vp, ctypes.POINTER(ctypes.c_double)]
        L.oracle_stats.argtypes = [vp, ctypes.POINTER(ctypes.c_uint64)]
        L.oracle_self_pass.restype = ctypes.c_double
        L.oracle_self_pass.argtypes = [vp, ctypes.c_int]
        for name, n in (("oracle_probe_strain", 4), ("oracle_probe_cloth_ground_friction", 4),
                        ("oracle_probe_rolling", 4), ("oracle_probe_aerodynamics", 8),
                        ("oracle_probe_self_ccd", 4), ("oracle_probe_self_friction", 8)):
            fn = getattr(L, name)
            fn.restype = ctypes.c_int
            fn.argtypes = [ctypes.POINTER(ctypes.c_double)]
        _LIB = L
    return _LIB


def _p(a):
    return None if a is None or len(a) == 0 else ctypes.c_void_p(a.ctypes.data)


class OracleScene:
    """FP64 oracle records of a scene (kept alive while an Oracle uses them)."""

    def __init__(self, particles, distances, knots, bends, grips, fruits, pairs, params: Params, cuff=None, rim=None,
                 local_off=None, local_idx=None):
        self.particles = np.ascontiguousarray(particles, PARTICLE)
        self.distances = np.ascontiguousarray(distances, DISTANCE)
        self.knots = np.ascontiguousarray(knots, KNOT)
        self.bends = np.ascontiguousarray(bends, BEND)
        self.grips = np.ascontiguousarray(grips, GRIP)
        self.fruits = np.ascontiguousarray(fruits, FRUIT)
        self.pairs = np.ascontiguousarray(pairs, PAIR)
        self.params = params
        self.cuff = None if cuff is None else np.ascontiguousarray(cuff, np.uint32)
        self.rim = None if rim is None else np.ascontiguousarray(rim, np.uint32)
        self.local_off = None if local_off is None else np.ascontiguousarray(local_off, np.uint32)
        self.local_idx = None if local_idx is None else np.ascontiguousarray(local_idx, np.uint32)

    def struct(self) -> OScene:
        s = OScene()
        s.particles, s.n = _p(self.particles), len(self.particles)
        s.distances, s.d = _p(self.distances), len(self.distances)
        s.knots, s.k = _p(self.knots), len(self.knots)
        s.bends, s.b = _p(self.bends), len(self.bends)
        s.grips, s.g = _p(self.grips), len(self.grips)
        s.fruits, s.f = _p(self.fruits), len(self.fruits)
        s.pairs, s.p = _p(self.pairs), len(self.pairs)
        s.cuff, s.rim = _p(self.cuff), _p(self.rim)
        s.local_off, s.local_idx = _p(self.local_off), _p(self.local_idx)
        s.params = ctypes.pointer(self.params)
        return s


def from_abi(scene) -> OracleScene:
    """Oracle records from a numi_cloth.SceneArrays (FP32 values widened exactly)."""
    n = scene.n
    cfg = scene.config[0]
    P = np.zeros(n, PARTICLE)
    pw = scene.particles["positionAndInverseMass"].astype(np.float64)
    P["x"] = pw[:, :3]
    P["w"] = pw[:, 3]
    pm = scene.particles["previousAndMass"].astype(np.float64)
    P["prev"] = pm[:, :3]
    P["mass"] = pm[:, 3]
    vv = scene.particles["velocity"].astype(np.float64)
    P["v"] = vv[:, :3]
    P["vw"] = vv[:, 3]
    P["rest"] = scene.rest.astype(np.float64)[:, :3]
    D = np.zeros(len(scene.distances), DISTANCE)
    pc = scene.distances["particlesAndColor"]
    D["i"], D["j"], D["colour"], D["kind"] = pc[:, 0], pc[:, 1], pc[:, 2], pc[:, 3]
    m = scene.distances["material"].astype(np.float64)
    D["rest"], D["compliance"], D["lambda_"], D["maxext"] = m[:, 0], m[:, 1], m[:, 2], m[:, 3]
    K = np.zeros(len(scene.knots), KNOT)
    if len(K):
        K["p"] = scene.knots["particles"]
        K["colour"] = scene.knots["control"][:, 0]
        km = scene.knots["material"].astype(np.float64)
        K["restcos"], K["compliance"], K["lambda_"] = km[:, 0], km[:, 1], km[:, 2]
    B = np.zeros(len(scene.bends), BEND)
    if len(B):
        bp = scene.bends["particlesAndColor"]
        B["p"] = bp[:, :3]
        B["colour"] = bp[:, 3]
        bm = scene.bends["material"].astype(np.float64)
        B["restchord"], B["restarc"], B["compliance"], B["lambda_"] = bm[:, 0], bm[:, 1], bm[:, 2], bm[:, 3]
    G = np.zeros(len(scene.grips), GRIP)
    if len(G):
        G["particle"] = scene.grips["particle"][:, 0]
        G["gen"] = scene.grips["particle"][:, 1]
        G["ring"] = scene.grips["particle"][:, 3]
        go = scene.grips["targetOffsetAndCompliance"].astype(np.float64)
        G["offset"], G["compliance"] = go[:, :3], go[:, 3]
        G["lambda_"] = scene.grips["lambda"].astype(np.float64)[:, :3]
    F = np.zeros(len(scene.fruits), FRUIT)
    if len(F):
        fr = scene.fruits
        a = fr["positionAndInverseMass"].astype(np.float64)
        F["x"], F["w"] = a[:, :3], a[:, 3]
        a = fr["previousAndRadius"].astype(np.float64)
        F["prev"], F["radius"] = a[:, :3], a[:, 3]
        a = fr["velocityAndGroundImpulse"].astype(np.float64)
        F["v"], F["ground_impulse"] = a[:, :3], a[:, 3]
        F["omega"] = fr["angularVelocity"].astype(np.float64)[:, :3]
        F["q"] = fr["orientation"].astype(np.float64)
        F["appearance"] = fr["identity"][:, 0]
    PR = np.zeros(len(scene.pairs), PAIR)
    if len(PR):
        fc = scene.pairs["fruitsAndColor"]
        PR["a"], PR["b"], PR["colour"], PR["stable"] = fc[:, 0], fc[:, 1], fc[:, 2], fc[:, 3]
    prm = Params()
    cm = cfg["clothMaterial"].astype(np.float64)
    fm = cfg["fruitMaterial"].astype(np.float64)
    prm.radius = cm[0]
    prm.mu_cloth_ground, prm.mu_self = cm[2], cm[3]
    prm.mu_pair, prm.mu_fruit_ground, prm.rolling, prm.mu_fruit_yarn = fm
    av = cfg["airVelocityAndDensity"].astype(np.float64)
    prm.air[:] = av[:3]
    prm.air_density = av[3]
    prm.aero[:] = cfg["aerodynamicCoefficients"].astype(np.float64)
    prm.capture_radius = float(cfg["gripMaterial"][0])
    prm.hysteresis = float(cfg["mouthMaterial"][0])
    prm.ground = int(cfg["constraintCounts"][2] != 0)
    prm.ring_count = int(cfg["gripControl"][2])
    prm.patch_half = int(cfg["gripControl"][3])
    prm.grid_width = int(scene.grid_width)
    prm.rim_count = int(len(scene.rim))
    prm.bottom_center = int(cfg["mouthControl"][1])
    return OracleScene(P, D, K, B, G, F, PR, prm, scene.cuff if len(scene.cuff) else None,
                       scene.rim if len(scene.rim) else None, scene.local_off, scene.local_idx)


def substeps_from_configs(configs) -> np.ndarray:
    """Oracle substep records from per-substep ABI Configs (FP32 widened)."""
    out = np.zeros(len(configs), SUBSTEP)
    g = configs["gravityAndTimestep"].astype(np.float64)
    out["dt"] = g[:, 3]
    out["gravity"] = g[:, :3]
    t = configs["gripTargetAndActive"].astype(np.float64)
    out["grip_target"] = t[:, :3]
    out["grip_active"] = (t[:, 3] > 0).astype(np.uint32)
    out["grip_q"] = configs["gripOrientation"].astype(np.float64)
    out["grip_gen"] = configs["gripControl"][:, 0]
    out["grip_select"] = configs["gripControl"][:, 1]
    return out


def schedule(mode=BATCHED, **kw) -> OSchedule:
    s = OSchedule()
    d = dict(iterations=1, strain_sweeps=3, reconcile_passes=8, final_passes=2, certificate_passes=128,
             early_exit=1, self_collision=0, aerodynamics=1, swept_ground=1, swept_fruit_yarn=0, frictions=1,
             release=0, damping=0.0, primitive_self=0)
    d.update(kw)
    for k, v in d.items():
        setattr(s, k, v)
    s.mode = mode
    return s


def schedule_from_abi(sched, mode=BATCHED) -> OSchedule:
    return schedule(
        mode,
        iterations=sched.iterations, strain_sweeps=sched.strainSweeps, reconcile_passes=sched.reconcilePasses,
        final_passes=sched.finalPasses, certificate_passes=sched.certificatePasses, early_exit=sched.earlyExit,
        self_collision=sched.selfCollision, aerodynamics=sched.aerodynamics, swept_ground=sched.sweptGround,
        swept_fruit_yarn=sched.sweptFruitYarn, frictions=sched.frictions, release=sched.release,
        damping=float(sched.damping), primitive_self=getattr(sched, "primitiveSelf", 0),
    )


class Oracle:
    def __init__(self, scene: OracleScene, bits: int = 64):
        self.scene = scene
        self._s = scene.struct()
        self._h = lib().oracle_create(bits, ctypes.byref(self._s))
        if not self._h:
            raise ValueError("oracle rejected the scene")
        self.bits = bits

    def __del__(self):
        if getattr(self, "_h", None):
            lib().oracle_destroy(self._h)
            self._h = None

    def step(self, substeps: np.ndarray, sched: OSchedule) -> int:
        substeps = np.ascontiguousarray(substeps, SUBSTEP)
        return int(lib().oracle_step(self._h, _p(substeps), len(substeps), ctypes.byref(sched)))

    def read(self):
        sc = self.scene
        P = np.zeros(len(sc.particles), PARTICLE)
        D = np.zeros(len(sc.distances), DISTANCE)
        G = np.zeros(len(sc.grips), GRIP)
        F = np.zeros(len(sc.fruits), FRUIT)
        PR = np.zeros(len(sc.pairs), PAIR)
        lib().oracle_read(self._h, _p(P), _p(D), _p(G), _p(F), _p(PR))
        return {"particles": P, "distances": D, "grips": G, "fruits": F, "pairs": PR}

    def write(self, particles=None, fruits=None, grips=None):
        lib().oracle_write(self._h, _p(particles), _p(fruits))
        if grips is not None and len(grips):
            lib().oracle_write_grips(self._h, _p(np.ascontiguousarray(grips, GRIP)))

    def residuals(self) -> np.ndarray:
        out = (ctypes.c_double * 4)()
        lib().oracle_residuals(self._h, out)
        return np.array(out[:])

    def self_pass(self, serial: bool = True) -> float:
        """One point self-contact pass on the current state: the reference's
        Gauss-Seidel order, or the kernels' batched order; its deepest
        penetration."""
        return float(lib().oracle_self_pass(self._h, 1 if serial else 0))

    def stats(self) -> dict:
        out = (ctypes.c_uint64 * 8)()
        lib().oracle_stats(self._h, out)
        keys = ("candidate_mask", "released_mask", "reconcile_max", "certificate_max", "yarn_contacts",
                "self_contacts", "edge_contacts", "self_friction_contacts")
        return dict(zip(keys, (int(v) for v in out)))
