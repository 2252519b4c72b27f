"""ctypes binding of oracle/_ref/libref_shim.so - TEST INFRASTRUCTURE.

The shim is the reference CPU cloth compiled from the reference sources (see
ref.mk); it exists only where those sources were present at build time.
Used to pin the oracle and to generate tests/golden/ fixtures.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

import oracle_py as op

HERE = os.path.dirname(os.path.abspath(__file__))
SHIM = os.path.join(HERE, "_ref", "libref_shim.so")
BINARY = os.path.join(HERE, "_ref", "cloth_bag")
SCENARIOS = {"grounded": 0, "spin": 1, "pickup": 2, "recorded": 3}
_LIB = None


def available() -> bool:
    return os.path.exists(SHIM)


def lib():
    global _LIB
    if _LIB is None:
        L = ctypes.CDLL(SHIM)
        vp, u32 = ctypes.c_void_p, ctypes.c_uint32
        L.ref_scene_counts.argtypes = [ctypes.c_int, ctypes.POINTER(u32)]
        L.ref_scene_export.argtypes = [ctypes.c_int] + [vp] * 11 + [ctypes.POINTER(op.Params)]
        L.ref_simulate_hash.restype = ctypes.c_uint64
        L.ref_simulate_hash.argtypes = [ctypes.c_int, u32, ctypes.c_double, u32, u32, ctypes.c_char_p]
        L.ref_run.restype = ctypes.c_int
        L.ref_run.argtypes = [ctypes.c_int, u32, ctypes.c_double, u32, u32, ctypes.c_char_p, u32, u32, vp, vp, vp,
                              ctypes.POINTER(ctypes.c_uint64)]
        L.ref_apply_material.restype = ctypes.c_int
        L.ref_apply_material.argtypes = [ctypes.c_char_p]
        L.ref_reset_material.argtypes = []
        L.ref_render_triangles.restype = u32
        L.ref_render_triangles.argtypes = [ctypes.c_int, vp]
        _LIB = L
    return _LIB


def _p(a):
    return None if a is None or len(a) == 0 else ctypes.c_void_p(a.ctypes.data)


def scene(scenario: str) -> op.OracleScene:
    """The reference scene in construction order, as oracle records."""
    c = (ctypes.c_uint32 * 8)()
    lib().ref_scene_counts(SCENARIOS[scenario], c)
    n, d, k, b, g, f, nl, bottom = list(c)
    P = np.zeros(n, op.PARTICLE)
    D = np.zeros(d, op.DISTANCE)
    K = np.zeros(k, op.KNOT)
    B = np.zeros(b, op.BEND)
    G = np.zeros(g, op.GRIP)
    F = np.zeros(f, op.FRUIT)
    PR = np.zeros(f * (f - 1) // 2, op.PAIR)
    lo = np.zeros(n + 1, np.uint32)
    li = np.zeros(nl, np.uint32)
    cuff = np.zeros(96, np.uint32)
    rim = np.zeros(48, np.uint32)
    prm = op.Params()
    lib().ref_scene_export(SCENARIOS[scenario], _p(P), _p(D), _p(K), _p(B), _p(G), _p(F), _p(PR), _p(lo), _p(li),
                           _p(cuff), _p(rim), ctypes.byref(prm))
    return op.OracleScene(P, D, K, B, G, F, PR, prm, cuff, rim, lo, li)


def render_triangles(scenario) -> np.ndarray:
    n = lib().ref_render_triangles(SCENARIOS[scenario], None)
    out = np.zeros((n, 3), np.uint32)
    lib().ref_render_triangles(SCENARIOS[scenario], _p(out))
    return out


def simulate_hash(scenario, steps, frame_dt, substeps, iterations, trajectory=None) -> int:
    return int(lib().ref_simulate_hash(SCENARIOS[scenario], steps, frame_dt, substeps, iterations,
                                       trajectory.encode() if trajectory else None))


def run(scenario, steps, frame_dt, substeps, iterations, trajectory=None, primitive=0, point_self=1, n=1465):
    subs = np.zeros(steps * substeps, op.SUBSTEP)
    P = np.zeros(n, op.PARTICLE)
    F = np.zeros(12, op.FRUIT)
    out = (ctypes.c_uint64 * 3)()
    rc = lib().ref_run(SCENARIOS[scenario], steps, frame_dt, substeps, iterations,
                       trajectory.encode() if trajectory else None, primitive, point_self, _p(subs), _p(P), _p(F), out)
    if rc != 0:
        raise RuntimeError(f"reference run failed: {rc}")
    return {"substeps": subs, "particles": P, "fruits": F, "hash": int(out[0]), "released_mask": int(out[1]),
            "candidate_mask": int(out[2])}
