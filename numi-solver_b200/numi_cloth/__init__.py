"""Python binding of the B200 XPBD cloth substep library (libnumi_cloth.so).

The product is the C ABI in include/numi_cloth.h and include/numi_cloth_scene.h;
this module is a thin ctypes mirror of it for tests, the benchmark and
calibration scripts.  It mirrors the reference host's roles: scene
construction (tools/cloth_bag.cpp:610-973 / tools/cloth_bag_metal.mm:524-1274),
the per-frame substep launch (runGPU, tools/cloth_bag_metal.mm:4010) and the
--material / --grip-trajectory contracts.  There is no CPU fallback: without
the built library every entry point raises.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field

import numpy as np

from . import abi
from .abi import (
    BEND,
    CONFIG,
    DISTANCE,
    FLOAT4,
    FRUIT,
    FRUIT_PAIR,
    GRIP,
    KNOT,
    PARTICLE,
    Material,
    Schedule,
    SquareSpec,
    failure_names,
)

__all__ = [
    "abi",
    "Schedule",
    "Material",
    "SquareSpec",
    "SceneArrays",
    "ClothSolver",
    "ClothError",
    "library_path",
    "load_library",
    "bag_scene",
    "square_scene",
    "material_defaults",
    "load_material",
    "GripTrajectory",
    "failure_names",
]

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


class ClothError(RuntimeError):
    pass


def library_path() -> str:
    return os.path.join(_HERE, "libnumi_cloth.so")


def load_library() -> ctypes.CDLL:
    """Load the in-tree library; raise loudly when it is not built."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = library_path()
    if not os.path.exists(path):
        raise ClothError(f"libnumi_cloth.so is not built ({path}); run `make -C numi-solver_b200`")
    lib = ctypes.CDLL(path)
    vp, u32, i32 = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int
    sigs = {
        "numi_cloth_version": (ctypes.c_char_p, []),
        "numi_cloth_create": (i32, [vp, ctypes.POINTER(vp)]),
        "numi_cloth_destroy": (None, [vp]),
        "numi_cloth_set_stream": (i32, [vp, vp]),
        "numi_cloth_step": (i32, [vp, vp, u32, ctypes.POINTER(Schedule)]),
        "numi_cloth_failure": (u32, [vp]),
        "numi_cloth_read_particles": (i32, [vp, vp, u32]),
        "numi_cloth_write_particles": (i32, [vp, vp, u32]),
        "numi_cloth_read_fruits": (i32, [vp, vp, u32]),
        "numi_cloth_write_fruits": (i32, [vp, vp, u32]),
        "numi_cloth_read_distances": (i32, [vp, vp, u32]),
        "numi_cloth_read_grips": (i32, [vp, vp, u32]),
        "numi_cloth_residuals": (i32, [vp, ctypes.POINTER(ctypes.c_double)]),
        "numi_cloth_release_masks": (i32, [vp, ctypes.POINTER(u32)]),
        "numi_cloth_snapshot": (i32, [vp, u32]),
        "numi_cloth_restore": (i32, [vp, u32]),
        "numi_cloth_launch_info": (i32, [vp, ctypes.POINTER(u32)]),
        "numi_cloth_tune": (i32, [vp, vp, u32, vp, ctypes.POINTER(u32)]),
        "numi_cloth_self_contacts": (i32, [vp, ctypes.POINTER(ctypes.c_ulonglong), ctypes.POINTER(ctypes.c_double)]),
        "numi_cloth_self_order_stats": (i32, [vp, ctypes.POINTER(ctypes.c_ulonglong)]),
        "numi_cloth_edge_contacts": (i32, [vp, ctypes.POINTER(ctypes.c_ulonglong)]),
        "numi_cloth_set_damping": (i32, [vp, ctypes.c_float]),
        "numi_cloth_rollout_grad": (i32, [vp, vp, u32, ctypes.POINTER(Schedule), u32, vp, u32, vp, u32,
                                          ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double), vp,
                                          ctypes.POINTER(u32)]),
        "numi_cloth_compliance_groups": (i32, [vp, ctypes.POINTER(u32), ctypes.POINTER(ctypes.c_float),
                                               ctypes.POINTER(u32)]),
        "numi_cloth_replace_compliance": (i32, [vp, u32, ctypes.c_float, ctypes.c_float]),
        "numi_cloth_batch_create": (i32, [ctypes.POINTER(vp), u32, ctypes.POINTER(vp)]),
        "numi_cloth_batch_destroy": (None, [vp]),
        "numi_cloth_batch_set_stream": (i32, [vp, vp]),
        "numi_cloth_batch_step": (i32, [vp, vp, u32, ctypes.POINTER(Schedule)]),
        "numi_cloth_batch_shape": (i32, [vp, ctypes.POINTER(u32)]),
        "numi_cloth_batch_set_shape": (i32, [vp, u32, u32]),
        "numi_cloth_batch_tune": (i32, [vp, vp, u32, ctypes.POINTER(Schedule), ctypes.POINTER(u32)]),
        "numi_cloth_batch_capture": (i32, [vp, vp, u32, ctypes.POINTER(Schedule)]),
        "numi_cloth_batch_replay": (i32, [vp]),
        "numi_cloth_batch_rollout_grad": (i32, [vp, vp, u32, ctypes.POINTER(Schedule), u32, vp, u32, vp, u32, vp, vp,
                                                vp, vp]),
        "numi_cloth_trace": (i32, [vp, ctypes.POINTER(ctypes.c_ulonglong), u32, u32]),
        "numi_cloth_trace_cta": (i32, [vp, ctypes.POINTER(ctypes.c_ulonglong), u32]),
        "numi_cloth_step_noalloc": (
            i32, [vp, ctypes.POINTER(abi.DeviceState), vp, ctypes.POINTER(u32), vp, u32, ctypes.POINTER(Schedule), vp],
        ),
        "numi_cloth_material_defaults": (None, [ctypes.POINTER(Material)]),
        "numi_cloth_material_load": (i32, [ctypes.c_char_p, ctypes.POINTER(Material), ctypes.c_char_p, ctypes.c_size_t]),
        "numi_cloth_scene_bag": (vp, [ctypes.POINTER(Material), i32, ctypes.c_double, i32]),
        "numi_cloth_square_defaults": (None, [ctypes.POINTER(SquareSpec)]),
        "numi_cloth_scene_square": (vp, [ctypes.POINTER(SquareSpec), ctypes.POINTER(Material)]),
        "numi_cloth_scene_destroy": (None, [vp]),
        "numi_cloth_scene_view": (i32, [vp, ctypes.POINTER(abi.SceneStruct)]),
        "numi_cloth_scene_counts": (i32, [vp, ctypes.POINTER(u32)]),
        "numi_cloth_scene_rest_fp64": (i32, [vp, ctypes.POINTER(ctypes.c_double)]),
        "numi_cloth_trajectory_load": (vp, [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_size_t]),
        "numi_cloth_trajectory_destroy": (None, [vp]),
        "numi_cloth_trajectory_sample": (i32, [vp, ctypes.c_double, ctypes.POINTER(abi.GripPose)]),
        "numi_cloth_trajectory_info": (
            i32,
            [vp, ctypes.POINTER(u32), ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_uint64)],
        ),
        "numi_cloth_trajectory_configs": (
            i32,
            [vp, vp, ctypes.POINTER(ctypes.c_double), ctypes.c_uint64, u32, ctypes.c_double, vp],
        ),
        "numi_cloth_scene_triangles": (u32, [vp, vp, u32]),
        "numi_cloth_bag_handle_base": (i32, [ctypes.c_int, ctypes.POINTER(ctypes.c_double)]),
        "numi_cloth_bag_grip_target": (i32, [ctypes.c_int, ctypes.c_double, ctypes.POINTER(ctypes.c_double)]),
        "numi_cloth_bag_scenario_configs": (
            i32, [ctypes.c_int, vp, ctypes.c_uint64, u32, ctypes.c_double, vp, vp]),
        "numi_cloth_state_hash": (ctypes.c_uint64, [ctypes.POINTER(abi.HashState)]),
        "numi_cloth_write_obj": (i32, [ctypes.c_char_p, ctypes.POINTER(abi.ObjState)]),
        "numi_cloth_replay": (i32, [ctypes.POINTER(abi.ReplayOptions), ctypes.POINTER(abi.ReplayResult),
                                    ctypes.c_char_p, ctypes.c_size_t]),
    }
    for name, (res, args) in sigs.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _LIB = lib
    return lib


def _ptr(a: np.ndarray | None):
    return None if a is None or a.size == 0 else ctypes.c_void_p(a.ctypes.data)


def material_defaults() -> Material:
    m = Material()
    load_library().numi_cloth_material_defaults(ctypes.byref(m))
    return m


def load_material(path: str) -> Material:
    """Parse a numi.cloth.material.v1 artifact (rejections raise ClothError)."""
    m = Material()
    err = ctypes.create_string_buffer(512)
    if load_library().numi_cloth_material_load(path.encode(), ctypes.byref(m), err, 512) != 0:
        raise ClothError(err.value.decode())
    return m


@dataclass
class SceneArrays:
    """The arrays numi_cloth_create takes, as ABI-record NumPy arrays."""

    config: np.ndarray                       # CONFIG[1]
    particles: np.ndarray                    # PARTICLE[N]
    rest: np.ndarray                         # float4[N]
    distances: np.ndarray                    # DISTANCE[D]
    knots: np.ndarray                        # KNOT[K]
    bends: np.ndarray                        # BEND[B]
    grips: np.ndarray                        # GRIP[G]
    fruits: np.ndarray                       # FRUIT[F]
    pairs: np.ndarray                        # FRUIT_PAIR[P]
    cuff: np.ndarray                         # uint32[2 * rings]
    rim: np.ndarray                          # uint32[rim]
    local_off: np.ndarray | None = None      # uint32[N+1]
    local_idx: np.ndarray | None = None
    grid_width: int = 0
    rest64: np.ndarray | None = None         # float64[N, 3]
    bottom_center: int = 0
    handle_base: tuple = (0.0, 0.0, 0.0)     # grip handle origin in FP64
    extra: dict = field(default_factory=dict)

    @property
    def n(self) -> int:
        return len(self.particles)

    def copy(self) -> "SceneArrays":
        out = SceneArrays(**{k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in self.__dict__.items()})
        out.extra = dict(self.extra)
        return out

    def struct(self) -> abi.SceneStruct:
        s = abi.SceneStruct()
        s.config = _ptr(self.config)
        s.particles = _ptr(self.particles)
        s.restPositions = _ptr(self.rest)
        s.distances = _ptr(self.distances)
        s.knots = _ptr(self.knots)
        s.bends = _ptr(self.bends)
        s.grips = _ptr(self.grips)
        s.fruits = _ptr(self.fruits)
        s.fruitPairs = _ptr(self.pairs)
        s.cuffParticles = _ptr(self.cuff)
        s.mouthRim = _ptr(self.rim)
        s.localOffsets = _ptr(self.local_off)
        s.localIndices = _ptr(self.local_idx)
        s.gridWidth = self.grid_width
        return s


def _scene_from_handle(h) -> SceneArrays:
    lib = load_library()
    if not h:
        raise ClothError("scene construction failed")
    try:
        view = abi.SceneStruct()
        lib.numi_cloth_scene_view(h, ctypes.byref(view))
        counts = (ctypes.c_uint32 * 15)()
        lib.numi_cloth_scene_counts(h, counts)
        n, d, k, b, g, f, p, rings, rim = counts[:9]

        def grab(ptr, dtype, count):
            if count == 0 or not ptr:
                return np.zeros(0, dtype)
            buf = (ctypes.c_char * (count * dtype.itemsize)).from_address(ptr)
            return np.frombuffer(bytes(buf), dtype=dtype).copy()

        rest64 = np.zeros(3 * n, np.float64)
        lib.numi_cloth_scene_rest_fp64(h, rest64.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        ntri = lib.numi_cloth_scene_triangles(h, None, 0)
        triangles = np.zeros((ntri, 3), np.uint32)
        lib.numi_cloth_scene_triangles(h, triangles.ctypes.data, ntri)
        local_off = grab(view.localOffsets, np.dtype("<u4"), n + 1) if view.localOffsets else None
        local_idx = (
            grab(view.localIndices, np.dtype("<u4"), int(local_off[-1])) if local_off is not None else None
        )
        cfg = grab(view.config, CONFIG, 1)
        arrays = SceneArrays(
            config=cfg,
            particles=grab(view.particles, PARTICLE, n),
            rest=grab(view.restPositions, np.dtype("<f4"), 4 * n).reshape(n, 4),
            distances=grab(view.distances, DISTANCE, d),
            knots=grab(view.knots, KNOT, k),
            bends=grab(view.bends, BEND, b),
            grips=grab(view.grips, GRIP, g),
            fruits=grab(view.fruits, FRUIT, f),
            pairs=grab(view.fruitPairs, FRUIT_PAIR, p),
            cuff=grab(view.cuffParticles, np.dtype("<u4"), 2 * rings),
            rim=grab(view.mouthRim, np.dtype("<u4"), rim),
            local_off=local_off,
            local_idx=local_idx,
            grid_width=view.gridWidth,
            rest64=rest64.reshape(n, 3),
            bottom_center=int(counts[14]),
            extra={
                "distance_colours": int(counts[9]),
                "knot_colours": int(counts[10]),
                "bend_colours": int(counts[11]),
                "pair_colours": int(counts[12]),
                "yarn_segments": int(counts[13]),
            },
        )
        arrays.extra["triangles"] = triangles
        return arrays
    finally:
        lib.numi_cloth_scene_destroy(h)


SCENARIOS = {"grounded": 0, "spin": 1, "pickup": 2, "recorded": 3}


def bag_scene(
    material: Material | None = None,
    scenario: str = "recorded",
    timestep: float = 1.0 / 5760.0,
    select_nearest: bool = False,
) -> SceneArrays:
    """The reference produce bag (1,465 particles, 12 fruits, 10 grips)."""
    lib = load_library()
    m = material if material is not None else material_defaults()
    h = lib.numi_cloth_scene_bag(ctypes.byref(m), SCENARIOS[scenario], timestep, 1 if select_nearest else 0)
    s = _scene_from_handle(h)
    c = s.config[0]
    s.handle_base = tuple(float(v) for v in _bag_handle_base(scenario))
    s.extra["scenario"] = scenario
    s.extra["material"] = m
    del c
    return s


def bag_scenario_configs(scene: SceneArrays, first_substep: int, count: int, dt: float):
    """Configs of the grounded, spin and pickup scenarios for substeps
    first..first+count-1, and their FP64 grip targets [count, 3]."""
    out = np.zeros(count, CONFIG)
    targets = np.zeros((count, 3), np.float64)
    rc = load_library().numi_cloth_bag_scenario_configs(
        SCENARIOS[scene.extra["scenario"]], _ptr(scene.config), first_substep, count, dt, _ptr(out), _ptr(targets))
    if rc != 0:
        raise ClothError("scenario has no scripted grip (recorded runs use GripTrajectory.configs)")
    return out, targets


def state_hash(particle_state: np.ndarray, fruit_state: np.ndarray, grip_target, grip_active: bool,
               generation: int = 1, grip_particles=None, grip_offsets=None, patch_selections: int = 0) -> int:
    """The reference's hashResult over an FP64 state: particle_state [n, 6]
    (position, velocity), fruit_state [f, 13] (position, velocity, angular
    velocity, orientation w x y z)."""
    ps = np.ascontiguousarray(particle_state, np.float64)
    fs = np.ascontiguousarray(fruit_state, np.float64)
    hs = abi.HashState()
    hs.particles, hs.fruits = len(ps), len(fs)
    hs.particleState = ps.ctypes.data
    hs.fruitState = fs.ctypes.data if len(fs) else None
    hs.gripTarget = (ctypes.c_double * 3)(*grip_target)
    hs.gripActive = 1 if grip_active else 0
    hs.generation = generation
    hs.patchSelections = patch_selections
    gp = np.ascontiguousarray(grip_particles if grip_particles is not None else np.zeros(0), np.uint32)
    go = np.ascontiguousarray(grip_offsets if grip_offsets is not None else np.zeros((0, 3)), np.float64)
    hs.grips = len(gp)
    hs.gripParticle = gp.ctypes.data if len(gp) else None
    hs.gripOffset = go.ctypes.data if len(go) else None
    return int(load_library().numi_cloth_state_hash(ctypes.byref(hs)))


def replay(scenario: str, steps: int, substeps: int = 48, frame_dt: float = 1.0 / 60.0, schedule: Schedule | None = None,
           replays: int = 1, material: str | None = None, trajectory: str | None = None,
           dump_frames: str | None = None, dump_every: int = 0, dump_obj: str | None = None) -> dict:
    """numi_cloth_replay: a produce-bag scenario frame after frame on the GPU."""
    o = abi.ReplayOptions()
    o.scenario = SCENARIOS[scenario]
    o.steps, o.substeps, o.replays, o.frameTimestep = steps, substeps, replays, frame_dt
    o.material = material.encode() if material else None
    o.gripTrajectory = trajectory.encode() if trajectory else None
    o.dumpObj = dump_obj.encode() if dump_obj else None
    o.dumpFrames = dump_frames.encode() if dump_frames else None
    o.dumpEvery = dump_every
    o.schedule = schedule if schedule is not None else Schedule.make()
    r = abi.ReplayResult()
    err = ctypes.create_string_buffer(512)
    rc = load_library().numi_cloth_replay(ctypes.byref(o), ctypes.byref(r), err, 512)
    if rc != 0:
        raise ClothError(err.value.decode() or f"replay failed ({rc})")
    return {"hash": int(r.hash), "replay_hash": int(r.replayHash), "deterministic": bool(r.deterministic),
            "failure": int(r.failure), "particles": r.particles, "fruits": r.fruits,
            "render_triangles": r.renderTriangles, "generation": r.generation,
            "residuals": list(r.residuals), "self_contacts": int(r.selfContacts),
            "edge_contacts": (int(r.edgeContacts[0]), int(r.edgeContacts[1])),
            "masks": (int(r.masks[0]), int(r.masks[1])), "reconcile_max": int(r.reconcileMax),
            "certificate_max": int(r.certificateMax), "seconds": r.seconds,
            "regrab_count": int(r.regrabCount), "patch_selections": int(r.patchSelections),
            "max_patch_ring_shift": int(r.maxPatchRingShift), "patch_center": int(r.patchCenter),
            "patch_particles_unique": bool(r.patchParticlesUnique),
            "patch_topology_exact": bool(r.patchTopologyExact),
            "inactive_grip_substeps": int(r.inactiveGripSubsteps)}


def _bag_handle_base(scenario: str):
    # authoredPosition(kLevels - 1, 0) in FP64 (tools/cloth_bag.cpp:475-527)
    import math

    level, ring, levels, around = 27, 0, 28, 48
    vertical = level / (levels - 1)

    def smooth(v):
        x = min(max(v, 0.0), 1.0)
        return x * x * (3.0 - 2.0 * x)

    body = smooth(vertical / 0.55)
    fold = min(max((vertical - 0.72) / 0.28, 0.0), 1.0)
    skirt = 1.0 - smooth(vertical / 0.18)
    angle0 = 2.0 * math.pi * ring / around
    base_radius = 0.266 + 0.030 * body - 0.116 * fold + 0.045 * skirt
    angle = angle0 + 0.08 * vertical
    wrinkle = 1.0 + 0.035 * math.sin(5.0 * angle + 5.0 * math.pi * vertical) + 0.018 * math.sin(
        9.0 * angle - 3.0 * math.pi * vertical
    )
    loose_rim = fold * (0.007 * math.sin(3.0 * angle + 0.35) + 0.004 * math.sin(7.0 * angle - 0.80))
    loose_skirt = skirt * (0.020 * math.sin(3.0 * angle - 0.40) + 0.012 * math.sin(7.0 * angle + 0.70))
    rim_sag = fold * (
        0.016 * math.sin(angle + 0.55) + 0.008 * math.sin(3.0 * angle - 0.30) + 0.004 * math.sin(6.0 * angle + 0.90)
    )
    radius = base_radius * wrinkle + loose_rim + loose_skirt
    skirt_sag = skirt * (0.012 * math.sin(4.0 * angle + 0.20) + 0.006 * math.sin(9.0 * angle - 0.50))
    folded = 0.167 + 0.038 * (fold / 0.35) if fold < 0.35 else 0.205 - 0.025 * ((fold - 0.35) / 0.65)
    lift = 0.52 if scenario == "spin" else 0.0
    return (radius * math.cos(angle), radius * math.sin(angle), folded + rim_sag + skirt_sag + 0.009 + lift)


def square_scene(spec: SquareSpec | None = None, material: Material | None = None, **overrides) -> SceneArrays:
    """Square s x s weave with shear diagonals and skip-one bends."""
    lib = load_library()
    if spec is None:
        spec = SquareSpec()
        lib.numi_cloth_square_defaults(ctypes.byref(spec))
    for k, v in overrides.items():
        setattr(spec, k, v)
    m = material if material is not None else material_defaults()
    h = lib.numi_cloth_scene_square(ctypes.byref(spec), ctypes.byref(m))
    s = _scene_from_handle(h)
    p0 = s.rest64[0]
    s.handle_base = (float(p0[0]), float(p0[1]), float(p0[2]))
    s.extra["spec"] = {name: getattr(spec, name) for name, _ in SquareSpec._fields_}
    return s


class GripTrajectory:
    """numi.grip.trajectory.v1..v3; the loader rejects what the reference rejects."""

    def __init__(self, path: str):
        lib = load_library()
        err = ctypes.create_string_buffer(512)
        self._h = lib.numi_cloth_trajectory_load(path.encode(), err, 512)
        if not self._h:
            raise ClothError(err.value.decode())
        sel = ctypes.c_uint32()
        dur = ctypes.c_double()
        fp = ctypes.c_uint64()
        lib.numi_cloth_trajectory_info(self._h, ctypes.byref(sel), ctypes.byref(dur), ctypes.byref(fp))
        self.select_nearest = bool(sel.value)
        self.duration = dur.value
        self.fingerprint = fp.value

    def __del__(self):
        if getattr(self, "_h", None) and _LIB is not None:
            _LIB.numi_cloth_trajectory_destroy(self._h)
            self._h = None

    def sample(self, t: float) -> abi.GripPose:
        p = abi.GripPose()
        if load_library().numi_cloth_trajectory_sample(self._h, t, ctypes.byref(p)) != 0:
            raise ClothError(f"grip trajectory sample outside its duration: {t}")
        return p

    def configs(self, base: np.ndarray, handle_base, first_substep: int, count: int, dt: float) -> np.ndarray:
        out = np.zeros(count, CONFIG)
        hb = (ctypes.c_double * 3)(*handle_base)
        rc = load_library().numi_cloth_trajectory_configs(
            self._h, _ptr(base), hb, first_substep, count, dt, _ptr(out)
        )
        if rc != 0:
            raise ClothError("grip trajectory does not cover the requested substeps")
        return out


class ClothSolver:
    """One solver handle on the current CUDA device (numi_cloth_create)."""

    def __init__(self, scene: SceneArrays):
        self.lib = load_library()
        self.scene = scene
        self._keep = scene.struct()
        h = ctypes.c_void_p()
        rc = self.lib.numi_cloth_create(ctypes.byref(self._keep), ctypes.byref(h))
        if rc != 0:
            raise ClothError(f"numi_cloth_create failed: {rc}")
        self._h = h
        self.n = scene.n

    def close(self):
        if getattr(self, "_h", None):
            self.lib.numi_cloth_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    FAMILIES = ("distance", "knot", "bend", "grip")

    def compliance_groups(self) -> list[tuple[str, float]]:
        """(family, compliance) of every compliance group, in gradient order."""
        fam = (ctypes.c_uint32 * 16)()
        val = (ctypes.c_float * 16)()
        count = ctypes.c_uint32()
        self._check(self.lib.numi_cloth_compliance_groups(self._h, fam, val, ctypes.byref(count)))
        return [(self.FAMILIES[fam[k]], float(val[k])) for k in range(count.value)]

    def replace_compliance(self, family: str, old: float, new: float):
        """Set every record of `family` whose compliance is `old` to `new`."""
        self._check(self.lib.numi_cloth_replace_compliance(self._h, self.FAMILIES.index(family), old, new))

    def rollout_grad(self, configs: np.ndarray, schedule: Schedule, tracked, targets, loss_every: int,
                     checkpoint_every: int = 8) -> dict:
        """Advance len(configs) substeps and return the tracked-particle
        loss and its reverse-mode gradients (numi_cloth_rollout_grad):
        `grads[g]` per compliance group (see compliance_groups), `damping`,
        and per-substep grip pose gradients `grip` [substeps, 6]."""
        configs = np.ascontiguousarray(configs, CONFIG)
        tracked = np.ascontiguousarray(tracked, np.uint32)
        targets = np.ascontiguousarray(targets, np.float64)
        n = len(configs)
        if targets.shape != (n // loss_every, len(tracked), 3):
            raise ClothError("targets must be [substeps // loss_every, tracked, 3]")
        groups = self.compliance_groups()
        loss = ctypes.c_double()
        grads = (ctypes.c_double * (len(groups) + 1))()
        grip = np.zeros((n, 6), np.float64)
        rough = ctypes.c_uint32()
        self._check(self.lib.numi_cloth_rollout_grad(
            self._h, configs.ctypes.data, n, ctypes.byref(schedule), checkpoint_every, tracked.ctypes.data,
            len(tracked), targets.ctypes.data, loss_every, ctypes.byref(loss), grads, grip.ctypes.data,
            ctypes.byref(rough)))
        return {"loss": loss.value, "groups": groups, "grads": np.array(grads[:len(groups)]),
                "damping": grads[len(groups)], "grip": grip, "nonsmooth": int(rough.value)}

    def set_damping(self, damping: float):
        """Per-cloth velocity damping c (v <- v / (1 + c dt)); < 0: the schedule's."""
        self._check(self.lib.numi_cloth_set_damping(self._h, damping))

    def set_stream(self, stream_ptr: int | None):
        self.lib.numi_cloth_set_stream(self._h, ctypes.c_void_p(stream_ptr) if stream_ptr else None)

    def step(self, configs: np.ndarray, schedule: Schedule):
        configs = np.ascontiguousarray(configs, CONFIG)
        rc = self.lib.numi_cloth_step(self._h, _ptr(configs), len(configs), ctypes.byref(schedule))
        if rc != 0:
            raise ClothError(f"numi_cloth_step failed: {rc}")

    def failure(self) -> int:
        return int(self.lib.numi_cloth_failure(self._h))

    def particles(self, out: np.ndarray | None = None) -> np.ndarray:
        """The particle records; `out` (PARTICLE[n], contiguous, e.g. over
        pinned host memory) receives them when given."""
        if out is None:
            out = np.zeros(self.n, PARTICLE)
        elif out.dtype != PARTICLE or len(out) != self.n or not out.flags["C_CONTIGUOUS"]:
            raise ClothError("particles(out=): a contiguous PARTICLE array of the cloth's size")
        self._check(self.lib.numi_cloth_read_particles(self._h, _ptr(out), self.n))
        return out

    def write_particles(self, p: np.ndarray):
        p = np.ascontiguousarray(p, PARTICLE)
        self._check(self.lib.numi_cloth_write_particles(self._h, _ptr(p), len(p)))

    def fruits(self, out: np.ndarray | None = None) -> np.ndarray:
        """The fruit records; `out` (FRUIT[f], contiguous) receives them when given."""
        if out is None:
            out = np.zeros(len(self.scene.fruits), FRUIT)
        elif out.dtype != FRUIT or len(out) != len(self.scene.fruits) or not out.flags["C_CONTIGUOUS"]:
            raise ClothError("fruits(out=): a contiguous FRUIT array of the cloth's fruit count")
        self._check(self.lib.numi_cloth_read_fruits(self._h, _ptr(out), len(out)))
        return out

    def write_fruits(self, f: np.ndarray):
        f = np.ascontiguousarray(f, FRUIT)
        self._check(self.lib.numi_cloth_write_fruits(self._h, _ptr(f), len(f)))

    def distances(self) -> np.ndarray:
        out = np.zeros(len(self.scene.distances), DISTANCE)
        self._check(self.lib.numi_cloth_read_distances(self._h, _ptr(out), len(out)))
        return out

    def grips(self) -> np.ndarray:
        out = np.zeros(len(self.scene.grips), GRIP)
        self._check(self.lib.numi_cloth_read_grips(self._h, _ptr(out), len(out)))
        return out

    def residuals(self) -> np.ndarray:
        out = (ctypes.c_double * 4)()
        self._check(self.lib.numi_cloth_residuals(self._h, out))
        return np.array(out[:])

    def snapshot(self, slot: int = 0):
        self._check(self.lib.numi_cloth_snapshot(self._h, slot))

    def restore(self, slot: int = 0):
        self._check(self.lib.numi_cloth_restore(self._h, slot))

    def release_masks(self) -> tuple[int, int]:
        """(mouth candidates, released) fruit bit masks, sticky since create."""
        out = (ctypes.c_uint32 * 2)()
        self._check(self.lib.numi_cloth_release_masks(self._h, out))
        return int(out[0]), int(out[1])

    def self_contacts(self) -> tuple[int, float]:
        """(pairs resolved, largest penetration resolved in m) since create."""
        n = ctypes.c_ulonglong()
        pen = ctypes.c_double()
        self._check(self.lib.numi_cloth_self_contacts(self._h, ctypes.byref(n), ctypes.byref(pen)))
        return int(n.value), float(pen.value)

    def self_order_stats(self) -> dict:
        """How the point self-contact passes kept the reference's order since
        create: passes that ran the ordered pass, pairs listed, ordered-pass
        rounds, passes resolved by the serial fallback."""
        out = (ctypes.c_ulonglong * 4)()
        self._check(self.lib.numi_cloth_self_order_stats(self._h, out))
        return {"ordered_passes": int(out[0]), "listed_pairs": int(out[1]), "rounds": int(out[2]),
                "fallbacks": int(out[3])}

    def edge_contacts(self) -> tuple[int, int]:
        """(edge/edge solves that moved particles, yarn/yarn self-friction
        contacts) since create."""
        out = (ctypes.c_ulonglong * 2)()
        self._check(self.lib.numi_cloth_edge_contacts(self._h, out))
        return int(out[0]), int(out[1])

    def tune(self, configs: np.ndarray, schedule: Schedule) -> dict:
        """numi_cloth_tune: time the colours-per-sync choices (the
        colour-by-colour launch, tile mode at three CTA counts) on these
        substeps, keep the fastest; the state is left as it was."""
        configs = np.ascontiguousarray(configs, CONFIG)
        out = (ctypes.c_uint32 * 4)()
        self._check(self.lib.numi_cloth_tune(self._h, configs.ctypes.data, len(configs), ctypes.byref(schedule), out))
        return {"colours_per_sync": out[0], "ctas": out[1], "threads": out[2], "us": out[3]}

    def launch_info(self) -> dict:
        out = (ctypes.c_uint32 * 6)()
        self._check(self.lib.numi_cloth_launch_info(self._h, out))
        return {"grid": out[0], "block": out[1], "barriers_per_substep": out[2], "launches": out[3],
                "cluster": out[4], "resident": bool(out[5] & 1), "neighbour_syncs": bool(out[5] & 2),
                "tiles": bool(out[5] & 4), "last_tiles": bool(out[5] & 8), "self_order_reference": bool(out[5] & 16)}

    def trace(self, substeps: int) -> np.ndarray:
        """Per-barrier globaltimer stamps (ns) of the last step, [substeps, 128]."""
        out = np.zeros((substeps, 128), np.uint64)
        self._check(self.lib.numi_cloth_trace(
            self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_ulonglong)), substeps, 128))
        return out

    def trace_cta(self, substeps: int) -> np.ndarray:
        """Per-CTA barrier arrival stamps (ns), [substeps, 128, grid]."""
        grid = self.launch_info()["grid"]
        out = np.zeros((substeps, 128, grid), np.uint64)
        self._check(self.lib.numi_cloth_trace_cta(
            self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_ulonglong)), substeps))
        return out

    @staticmethod
    def _check(rc: int):
        if rc != 0:
            raise ClothError(f"numi_cloth call failed: {rc}")


def substep_configs(scene: SceneArrays, count: int, dt: float | None = None) -> np.ndarray:
    """count copies of the scene's base Config (static grip target)."""
    cfg = np.repeat(scene.config, count)
    if dt is not None:
        cfg["gravityAndTimestep"][:, 3] = dt
    return cfg


def colour_runs(scene: SceneArrays):
    """NumiClothBatch records of the scene's colour runs (distance, knot,
    bend, fruit pair) and the count of each family; distance runs carry the
    yarn-prefix | strain-limited-prefix << 16 word."""
    from .abi import KIND_SHEAR

    def runs(colours, extra=None):
        out = []
        k = 0
        while k < len(colours):
            first = k
            while k < len(colours) and colours[k] == colours[first]:
                k += 1
            w = extra(first, k) if extra else 0
            out.append((first, k - first, int(colours[first]), w))
        return out

    d = scene.distances

    def dist_extra(first, end):
        yarn = limited = 0
        for i in range(first, end):
            if d["particlesAndColor"][i, 3] != KIND_SHEAR:
                yarn = i - first + 1
            if d["material"][i, 3] > 0:
                limited = i - first + 1
        return yarn | (limited << 16)

    fams = [
        runs(d["particlesAndColor"][:, 2], dist_extra),
        runs(scene.knots["control"][:, 0]) if len(scene.knots) else [],
        runs(scene.bends["particlesAndColor"][:, 3]) if len(scene.bends) else [],
        runs(scene.pairs["fruitsAndColor"][:, 2]) if len(scene.pairs) else [],
    ]
    flat = [r for f in fams for r in f]
    recs = np.zeros((max(len(flat), 1), 4), np.uint32)
    for i, r in enumerate(flat):
        recs[i] = r
    return recs, np.array([len(f) for f in fams], np.uint32)


def step_noalloc(scene: SceneArrays, state: abi.DeviceState, batches: np.ndarray, counts: np.ndarray,
                 configs: np.ndarray, schedule: Schedule, stream_ptr: int | None = None) -> int:
    """numi_cloth_step_noalloc: step device buffers the caller owns; returns
    the ABI return code (0 ok, <0 error, >0 a rejected Config's failure bit)."""
    configs = np.ascontiguousarray(configs, CONFIG)
    batches = np.ascontiguousarray(batches, np.uint32)
    counts = np.ascontiguousarray(counts, np.uint32)
    return int(load_library().numi_cloth_step_noalloc(
        _ptr(scene.config), ctypes.byref(state), _ptr(batches),
        counts.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), _ptr(configs), len(configs),
        ctypes.byref(schedule), ctypes.c_void_p(stream_ptr) if stream_ptr else None))


class ClothBatch:
    """Many ClothSolvers stepped by one persistent launch (numi_cloth_batch_*).

    The batch borrows the solvers; close it before them.  Configs are given
    as one array of shape [cloths, substeps] (CONFIG records)."""

    def __init__(self, solvers: list):
        self.lib = load_library()
        self.solvers = list(solvers)
        handles = (ctypes.c_void_p * len(self.solvers))(*[sv._h for sv in self.solvers])
        h = ctypes.c_void_p()
        rc = self.lib.numi_cloth_batch_create(handles, len(self.solvers), ctypes.byref(h))
        if rc != 0:
            raise ClothError(f"numi_cloth_batch_create failed ({rc})")
        self._h = h
        self._graph_cfg = None

    def close(self):
        if getattr(self, "_h", None):
            self.lib.numi_cloth_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def _check(self, rc: int):
        if rc != 0:
            raise ClothError(f"cloth batch call failed ({rc})")

    def _configs(self, configs: np.ndarray) -> tuple[np.ndarray, int]:
        configs = np.ascontiguousarray(configs, abi.CONFIG)
        if configs.ndim != 2 or configs.shape[0] != len(self.solvers):
            raise ClothError("configs must be [cloths, substeps]")
        return configs, configs.shape[1]

    def set_stream(self, stream_ptr: int | None):
        self._check(self.lib.numi_cloth_batch_set_stream(self._h, ctypes.c_void_p(stream_ptr or 0)))

    def step(self, configs: np.ndarray, schedule: Schedule):
        configs, n = self._configs(configs)
        self._check(self.lib.numi_cloth_batch_step(self._h, configs.ctypes.data, n, ctypes.byref(schedule)))

    def shape(self) -> dict:
        out = (ctypes.c_uint32 * 3)()
        self._check(self.lib.numi_cloth_batch_shape(self._h, out))
        return {"resident_chunk": out[0], "threads": out[1], "ctas": out[2]}

    def set_shape(self, resident_chunk: int, threads: int):
        self._check(self.lib.numi_cloth_batch_set_shape(self._h, resident_chunk, threads))

    def tune(self, configs: np.ndarray, schedule: Schedule) -> dict:
        configs, n = self._configs(configs)
        out = (ctypes.c_uint32 * 3)()
        self._check(self.lib.numi_cloth_batch_tune(self._h, configs.ctypes.data, n, ctypes.byref(schedule), out))
        return {"resident_chunk": out[0], "threads": out[1], "ctas": out[2]}

    def capture(self, pinned_configs, substeps: int, schedule: Schedule):
        """Capture one step as a CUDA graph reading `pinned_configs` (a pinned
        host buffer, e.g. a pinned torch uint8 tensor, holding [cloths,
        substeps] CONFIG records) at every replay."""
        self._graph_cfg = pinned_configs
        self._check(self.lib.numi_cloth_batch_capture(self._h, ctypes.c_void_p(pinned_configs.data_ptr()), substeps,
                                                      ctypes.byref(schedule)))

    def replay(self):
        self._check(self.lib.numi_cloth_batch_replay(self._h))

    def rollout_grad(self, configs: np.ndarray, schedule: Schedule, tracked, targets, loss_every: int,
                     checkpoint_every: int = 8) -> dict:
        """numi_cloth_batch_rollout_grad: loss [cloths], group gradients
        [cloths, groups], damping gradient [cloths], non-smooth counts."""
        configs, n = self._configs(configs)
        count = len(self.solvers)
        tracked = np.ascontiguousarray(tracked, np.uint32)
        targets = np.ascontiguousarray(targets, np.float64)
        if targets.shape != (count, n // loss_every, len(tracked), 3):
            raise ClothError("targets must be [cloths, substeps // loss_every, tracked, 3]")
        loss = np.zeros(count, np.float64)
        grads = np.zeros((count, 17), np.float64)
        groups = np.zeros(count, np.uint32)
        rough = np.zeros(count, np.uint32)
        self._check(self.lib.numi_cloth_batch_rollout_grad(
            self._h, configs.ctypes.data, n, ctypes.byref(schedule), checkpoint_every, tracked.ctypes.data,
            len(tracked), targets.ctypes.data, loss_every, loss.ctypes.data, grads.ctypes.data, groups.ctypes.data,
            rough.ctypes.data))
        return {"loss": loss, "grads": [grads[k, :int(groups[k])] for k in range(count)],
                "damping": grads[np.arange(count), groups.astype(np.int64)], "groups": groups, "nonsmooth": rough}
