"""The square cloth scene of the benchmark, built for the oracle without the
product library (test infrastructure: the CPU baseline and the reference arm
of bench.py build their inputs here).

A restatement, in numpy, of the square-cloth builder of the C ABI
(numi_cloth_scene_square): a side x side grid at `spacing` in the plane
z = height, warp / weft distances with the strain limit, both shear
diagonals, skip-one bends, first-fit colouring (64-bit masks, record order)
with the yarn and shear colour spaces apart and each colour's yarn segments
first, two gripped corners, seeded spheres (SplitMix64; Steele, Lea and
Flood 2014) redrawn until each overlaps no earlier one, every value rounded once to FP32 as the ABI records are and
widened back, so the oracle runs the same workload as the GPU.  The
authored material values are the reference's defaults
(include/numi/cloth_material.h:15-60).
"""
from __future__ import annotations

import numpy as np

import oracle_py as op

# reference material defaults used by the square scene
CLOTH_GROUND_FRICTION = 0.45
CLOTH_SELF_FRICTION = 0.34
FRUIT_YARN_FRICTION = 0.36
FRUIT_GROUND_FRICTION = 0.42
FRUIT_PAIR_FRICTION = 0.30
ROLLING_RESISTANCE = 0.015
AERO = (1.10, 0.010, 0.47, 0.010)   # yarn crossflow, yarn skin, fruit drag, fruit rotational drag
MASK64 = (1 << 64) - 1
SPHERE_DRAWS = 4096   # draws per sphere before the builder gives up


def _f32(v):
    return np.asarray(v, np.float64).astype(np.float32).astype(np.float64)


def _splitmix64(state: int) -> tuple[int, int]:
    state = (state + 0x9E3779B97F4A7C15) & MASK64
    z = state
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK64
    return state, z ^ (z >> 31)


def _uniform01(state: int) -> tuple[int, float]:
    state, z = _splitmix64(state)
    return state, float(z >> 11) * 2.0 ** -53


def _first_fit(pairs: np.ndarray, n: int) -> tuple[np.ndarray, int]:
    """First free colour of every record in record order (writers: its two
    particles), a 64-bit used-colour mask per particle."""
    used = [0] * n
    colour = np.zeros(len(pairs), np.uint32)
    top = 0
    for k, (a, b) in enumerate(pairs.tolist()):
        busy = used[a] | used[b]
        c = ((~busy) & -(~busy)).bit_length() - 1
        if c >= 64:
            raise ValueError("colouring exceeds 64 colours")
        colour[k] = c
        top = max(top, c + 1)
        used[a] |= 1 << c
        used[b] |= 1 << c
    return colour, top


def build(side: int = 256, spacing: float = 0.004, height: float = 0.5, particle_mass: float = 0.0005,
          stretch_compliance: float = 1.0e-8, shear_compliance: float = 1.0e-8, bend_compliance: float = 1.0e-5,
          strain_limit: float = 0.10, grip_compliance: float = 2.0e-4, grip_corners: int = 2, fruit_count: int = 64,
          fruit_radius=(0.02, 0.05), fruit_mass: float = 0.1, fruit_height=(0.55, 1.0), thickness: float = 0.001,
          seed: int = 20260815, ground: bool = True) -> op.OracleScene:
    n = side * side
    half = 0.5 * (side - 1) * spacing
    jj, ii = np.meshgrid(np.arange(side), np.arange(side))
    pos = np.stack([jj.ravel() * spacing - half, ii.ravel() * spacing - half, np.full(n, height)], axis=1)
    ids = np.arange(n, dtype=np.uint32).reshape(side, side)
    P = np.zeros(n, op.PARTICLE)
    P["x"] = _f32(pos)
    P["w"] = _f32(np.full(n, 1.0 / particle_mass))
    P["prev"] = P["x"]
    P["mass"] = _f32(np.full(n, particle_mass))
    P["rest"] = P["x"]
    # distances: warp, weft (kind 0, 1, strain-limited), shear (kind 3)
    specs = [
        (ids[:, :-1].ravel(), ids[:, 1:].ravel(), 0, stretch_compliance, strain_limit),
        (ids[:-1, :].ravel(), ids[1:, :].ravel(), 1, stretch_compliance, strain_limit),
        (ids[:-1, :-1].ravel(), ids[1:, 1:].ravel(), 3, shear_compliance, 0.0),
        (ids[:-1, 1:].ravel(), ids[1:, :-1].ravel(), 3, shear_compliance, 0.0),
    ]
    first = np.concatenate([s[0] for s in specs])
    second = np.concatenate([s[1] for s in specs])
    kind = np.concatenate([np.full(len(s[0]), s[2], np.uint32) for s in specs])
    comp = np.concatenate([np.full(len(s[0]), s[3]) for s in specs])
    limit = np.concatenate([np.full(len(s[0]), s[4]) for s in specs])
    colour = np.zeros(len(first), np.uint32)
    offset = 0
    for shear in (False, True):
        members = np.flatnonzero((kind == 3) == shear)
        c, top = _first_fit(np.stack([first[members], second[members]], axis=1), n)
        colour[members] = c + offset
        offset += top
    order = np.lexsort((np.where(kind == 3, 1, 0), colour))   # stable by (colour, yarn before shear)
    D = np.zeros(len(first), op.DISTANCE)
    D["i"], D["j"], D["colour"], D["kind"] = first[order], second[order], colour[order], kind[order]
    D["rest"] = _f32(np.linalg.norm(pos[second[order]] - pos[first[order]], axis=1))
    D["compliance"] = _f32(comp[order])
    D["maxext"] = _f32(limit[order])
    # skip-one bends, horizontal then vertical
    b0 = np.concatenate([ids[:, :-2].ravel(), ids[:-2, :].ravel()])
    b1 = np.concatenate([ids[:, 1:-1].ravel(), ids[1:-1, :].ravel()])
    b2 = np.concatenate([ids[:, 2:].ravel(), ids[2:, :].ravel()])
    bc, _ = _first_fit(np.stack([b0, b2], axis=1), n)
    border = np.argsort(bc, kind="stable")
    B = np.zeros(len(b0), op.BEND)
    B["p"] = np.stack([b0[border], b1[border], b2[border]], axis=1)
    B["colour"] = bc[border]
    B["restchord"] = _f32(np.linalg.norm(pos[b2[border]] - pos[b0[border]], axis=1))
    B["restarc"] = _f32(np.linalg.norm(pos[b1[border]] - pos[b0[border]], axis=1) +
                        np.linalg.norm(pos[b2[border]] - pos[b1[border]], axis=1))
    B["compliance"] = _f32(np.full(len(b0), bend_compliance))
    # gripped corners
    corners = [int(ids[0, 0])] + ([int(ids[0, side - 1])] if grip_corners >= 2 else [])
    corners = corners[:grip_corners]
    G = np.zeros(len(corners), op.GRIP)
    for g, i in enumerate(corners):
        G[g]["particle"] = i
        G[g]["gen"] = 1
        G[g]["offset"] = _f32(pos[i] - pos[0])
        G[g]["compliance"] = _f32(grip_compliance)
    # seeded spheres, each redrawn until it overlaps no earlier sphere
    F = np.zeros(fruit_count, op.FRUIT)
    state = seed
    placed = []
    for k in range(fruit_count):
        for _ in range(SPHERE_DRAWS):
            state, u = _uniform01(state)
            x = -half + 2.0 * half * u
            state, u = _uniform01(state)
            y = -half + 2.0 * half * u
            state, u = _uniform01(state)
            bottom = fruit_height[0] + (fruit_height[1] - fruit_height[0]) * u
            state, u = _uniform01(state)
            r = fruit_radius[0] + (fruit_radius[1] - fruit_radius[0]) * u
            z = bottom + r
            if all((x - a) * (x - a) + (y - b) * (y - b) + (z - c) * (z - c) >= (r + q) * (r + q)
                   for a, b, c, q in placed):
                break
        else:
            raise ValueError("no room for the requested spheres")
        placed.append((x, y, z, r))
        F[k]["x"] = _f32([x, y, z])
        F[k]["prev"] = F[k]["x"]
        F[k]["w"] = _f32(1.0 / fruit_mass)
        F[k]["radius"] = _f32(r)
        F[k]["q"] = [0.0, 0.0, 0.0, 1.0]
        F[k]["appearance"] = k & 3
    pa = np.array([(a, b) for a in range(fruit_count) for b in range(a + 1, fruit_count)], np.uint32).reshape(-1, 2)
    PR = np.zeros(len(pa), op.PAIR)
    if len(pa):
        pc, _ = _first_fit(pa, max(fruit_count, 1))
        porder = np.argsort(pc, kind="stable")
        PR["a"], PR["b"], PR["colour"], PR["stable"] = pa[porder, 0], pa[porder, 1], pc[porder], porder
    prm = op.Params()
    prm.radius = float(_f32(thickness))
    prm.mu_cloth_ground = float(_f32(CLOTH_GROUND_FRICTION))
    prm.mu_self = float(_f32(CLOTH_SELF_FRICTION))
    prm.mu_pair = float(_f32(FRUIT_PAIR_FRICTION))
    prm.mu_fruit_ground = float(_f32(FRUIT_GROUND_FRICTION))
    prm.rolling = float(_f32(ROLLING_RESISTANCE))
    prm.mu_fruit_yarn = float(_f32(FRUIT_YARN_FRICTION))
    prm.air_density = float(_f32(1.225))
    prm.aero[:] = _f32(AERO)
    prm.capture_radius = 1.0e9
    prm.hysteresis = float(_f32(0.025))
    prm.ground = 1 if ground else 0
    prm.grid_width = side
    return op.OracleScene(P, D, np.zeros(0, op.KNOT), B, G, F, PR, prm)


def substeps(scene: op.OracleScene, count: int, dt: float = 1.0 / 2880.0) -> np.ndarray:
    """count substeps with the static grip at the first corner (the base
    Config's grip target, active while the scene has grips)."""
    out = np.zeros(count, op.SUBSTEP)
    out["dt"] = float(_f32(dt))
    out["gravity"] = [0.0, 0.0, float(_f32(-9.81))]
    out["grip_target"] = scene.particles["x"][0]
    out["grip_q"] = [0.0, 0.0, 0.0, 1.0]
    out["grip_active"] = 1 if len(scene.grips) else 0
    out["grip_gen"] = 1
    return out
