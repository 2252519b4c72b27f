"""NumPy/ctypes views of the pointer-free cloth ABI (include/numi_cloth.h).

The record dtypes are byte-identical to the reference GPU ABI v13
(include/numi/cloth_bag_gpu.h:19-190 in the reference tree); the sizes are
asserted at import time.
"""
from __future__ import annotations

import ctypes

import numpy as np

ABI_VERSION = 13

FAILURE_ABI = 1 << 0
FAILURE_RANGE = 1 << 1
FAILURE_BATCH = 1 << 2
FAILURE_NONFINITE = 1 << 3
FAILURE_GRIP_CAPTURE = 1 << 4
FAILURE_TIMEOUT = 1 << 5

FAILURE_NAMES = {
    FAILURE_ABI: "abi",
    FAILURE_RANGE: "range",
    FAILURE_BATCH: "batch",
    FAILURE_NONFINITE: "nonfinite",
    FAILURE_GRIP_CAPTURE: "grip_capture",
    FAILURE_TIMEOUT: "timeout",
}

_f4 = ("<f4", (4,))
_u4 = ("<u4", (4,))

CONFIG = np.dtype(
    [
        ("control", *_u4),
        ("constraintCounts", *_u4),
        ("contactCounts", *_u4),
        ("gravityAndTimestep", *_f4),
        ("gripTargetAndActive", *_f4),
        ("gripOrientation", *_f4),
        ("gripControl", *_u4),
        ("gripMaterial", *_f4),
        ("clothMaterial", *_f4),
        ("fruitMaterial", *_f4),
        ("airVelocityAndDensity", *_f4),
        ("aerodynamicCoefficients", *_f4),
        ("mouthControl", *_u4),
        ("mouthMaterial", *_f4),
    ]
)
PARTICLE = np.dtype([("positionAndInverseMass", *_f4), ("previousAndMass", *_f4), ("velocity", *_f4)])
DISTANCE = np.dtype([("particlesAndColor", *_u4), ("material", *_f4)])
GRIP = np.dtype([("particle", *_u4), ("targetOffsetAndCompliance", *_f4), ("lambda", *_f4)])
KNOT = np.dtype([("particles", *_u4), ("control", *_u4), ("material", *_f4)])
BEND = np.dtype([("particlesAndColor", *_u4), ("material", *_f4)])
FRUIT = np.dtype(
    [
        ("positionAndInverseMass", *_f4),
        ("previousAndRadius", *_f4),
        ("velocityAndGroundImpulse", *_f4),
        ("angularVelocity", *_f4),
        ("orientation", *_f4),
        ("identity", *_u4),
    ]
)
FRUIT_PAIR = np.dtype([("fruitsAndColor", *_u4), ("contact", *_f4)])
FLOAT4 = np.dtype("<f4", (4,))

for _dt, _size in (
    (CONFIG, 224),
    (PARTICLE, 48),
    (DISTANCE, 32),
    (GRIP, 48),
    (KNOT, 48),
    (BEND, 32),
    (FRUIT, 96),
    (FRUIT_PAIR, 32),
):
    assert _dt.itemsize == _size, (_dt, _dt.itemsize, _size)

KIND_WARP, KIND_WEFT, KIND_BOTTOM, KIND_SHEAR = 0, 1, 2, 3


class Schedule(ctypes.Structure):
    """NumiClothSchedule (include/numi_cloth.h)."""

    _fields_ = [
        ("iterations", ctypes.c_uint32),
        ("strainSweeps", ctypes.c_uint32),
        ("reconcilePasses", ctypes.c_uint32),
        ("finalPasses", ctypes.c_uint32),
        ("certificatePasses", ctypes.c_uint32),
        ("earlyExit", ctypes.c_uint32),
        ("selfCollision", ctypes.c_uint32),
        ("aerodynamics", ctypes.c_uint32),
        ("sweptGround", ctypes.c_uint32),
        ("sweptFruitYarn", ctypes.c_uint32),
        ("frictions", ctypes.c_uint32),
        ("release", ctypes.c_uint32),
        ("damping", ctypes.c_float),
        ("primitiveSelf", ctypes.c_uint32),
        ("reserved", ctypes.c_uint32 * 2),
    ]

    @classmethod
    def make(cls, **kw) -> "Schedule":
        s = cls()
        defaults = dict(
            iterations=1,
            strainSweeps=3,
            reconcilePasses=8,
            finalPasses=2,
            certificatePasses=128,
            earlyExit=1,
            selfCollision=0,
            aerodynamics=1,
            sweptGround=1,
            sweptFruitYarn=0,
            frictions=1,
            release=0,
            damping=0.0,
            primitiveSelf=0,
        )
        defaults.update(kw)
        for k, v in defaults.items():
            setattr(s, k, v)
        return s

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_ if name != "reserved"}


class SceneStruct(ctypes.Structure):
    """NumiClothScene (include/numi_cloth.h)."""

    _fields_ = [
        ("config", ctypes.c_void_p),
        ("particles", ctypes.c_void_p),
        ("restPositions", ctypes.c_void_p),
        ("distances", ctypes.c_void_p),
        ("knots", ctypes.c_void_p),
        ("bends", ctypes.c_void_p),
        ("grips", ctypes.c_void_p),
        ("fruits", ctypes.c_void_p),
        ("fruitPairs", ctypes.c_void_p),
        ("cuffParticles", ctypes.c_void_p),
        ("mouthRim", ctypes.c_void_p),
        ("localOffsets", ctypes.c_void_p),
        ("localIndices", ctypes.c_void_p),
        ("gridWidth", ctypes.c_uint32),
        ("reserved", ctypes.c_uint32 * 3),
    ]


class Material(ctypes.Structure):
    """NumiClothMaterial: the 19 numi.cloth.material.v1 parameters."""

    _fields_ = [
        (name, ctypes.c_double)
        for name in (
            "ordinaryNodeMassKg",
            "hemNodeMassKg",
            "yarnRadiusM",
            "axialBodyComplianceMPerN",
            "axialCuffComplianceMPerN",
            "knotCompliance",
            "bendBodyComplianceMPerN",
            "bendCuffComplianceMPerN",
            "gripComplianceMPerN",
            "clothGroundFriction",
            "clothSelfFriction",
            "fruitYarnFriction",
            "fruitGroundFriction",
            "fruitPairFriction",
            "fruitRollingResistance",
            "yarnCrossflowDrag",
            "yarnSkinFriction",
            "fruitDrag",
            "fruitRotationalDrag",
        )
    ]


class SquareSpec(ctypes.Structure):
    """NumiClothSquareSpec (include/numi_cloth_scene.h)."""

    _fields_ = [
        ("side", ctypes.c_uint32),
        ("spacing", ctypes.c_double),
        ("height", ctypes.c_double),
        ("particleMass", ctypes.c_double),
        ("stretchCompliance", ctypes.c_double),
        ("shearCompliance", ctypes.c_double),
        ("bendCompliance", ctypes.c_double),
        ("strainLimit", ctypes.c_double),
        ("gripCompliance", ctypes.c_double),
        ("gripCorners", ctypes.c_uint32),
        ("fruitCount", ctypes.c_uint32),
        ("fruitRadiusMin", ctypes.c_double),
        ("fruitRadiusMax", ctypes.c_double),
        ("fruitMass", ctypes.c_double),
        ("fruitHeightMin", ctypes.c_double),
        ("fruitHeightMax", ctypes.c_double),
        ("thickness", ctypes.c_double),
        ("seed", ctypes.c_uint64),
        ("timestep", ctypes.c_double),
        ("groundEnabled", ctypes.c_uint32),
    ]


class GripPose(ctypes.Structure):
    _fields_ = [
        ("time", ctypes.c_double),
        ("translation", ctypes.c_double * 3),
        ("orientation", ctypes.c_double * 4),
        ("active", ctypes.c_uint32),
        ("generation", ctypes.c_uint32),
    ]


def failure_names(word: int) -> list[str]:
    return [name for bit, name in FAILURE_NAMES.items() if word & bit]


class DeviceState(ctypes.Structure):
    """NumiClothDeviceState: device buffers of one cloth, library layout."""

    _fields_ = [
        (name, ctypes.c_void_p)
        for name in (
            "positions", "previous", "velocities", "rest", "distanceIJ", "distanceMaterial", "distanceLambda",
            "knotIJ", "knotMaterial", "knotLambda", "bendIJ", "bendMaterial", "bendLambda", "grips", "fruits",
            "fruitPairs", "cuffParticles", "failure",
        )
    ]


NOALLOC_MAX_PARTICLES = 4096
NOALLOC_MAX_DISTANCES = 8192
NOALLOC_MAX_SUBSTEPS = 256


class HashState(ctypes.Structure):
    """NumiClothHashState (include/numi_cloth_replay.h)."""

    _fields_ = [
        ("particles", ctypes.c_uint32), ("fruits", ctypes.c_uint32), ("grips", ctypes.c_uint32),
        ("gripActive", ctypes.c_uint32),
        ("particleState", ctypes.c_void_p), ("fruitState", ctypes.c_void_p),
        ("gripTarget", ctypes.c_double * 3),
        ("generation", ctypes.c_uint32), ("patchSelections", ctypes.c_uint32),
        ("gripParticle", ctypes.c_void_p), ("gripOffset", ctypes.c_void_p),
    ]


class ObjState(ctypes.Structure):
    """NumiClothObjState (include/numi_cloth_replay.h)."""

    _fields_ = [
        ("particles", ctypes.c_uint32), ("triangles", ctypes.c_uint32),
        ("positions", ctypes.c_void_p), ("triangleIndices", ctypes.c_void_p),
        ("scenario", ctypes.c_int), ("gripActive", ctypes.c_uint32),
        ("gripTarget", ctypes.c_double * 3), ("gripOrientationWxyz", ctypes.c_double * 4),
        ("patchCenter", ctypes.c_uint32), ("fruits", ctypes.c_uint32),
        ("fruitState", ctypes.c_void_p), ("fruitAppearance", ctypes.c_void_p),
    ]


class ReplayOptions(ctypes.Structure):
    """NumiClothReplayOptions (include/numi_cloth_replay.h)."""

    _fields_ = [
        ("scenario", ctypes.c_int), ("steps", ctypes.c_uint32), ("substeps", ctypes.c_uint32),
        ("replays", ctypes.c_uint32), ("frameTimestep", ctypes.c_double),
        ("material", ctypes.c_char_p), ("gripTrajectory", ctypes.c_char_p),
        ("dumpObj", ctypes.c_char_p), ("dumpFrames", ctypes.c_char_p),
        ("dumpEvery", ctypes.c_uint32), ("pad", ctypes.c_uint32),
        ("schedule", Schedule),
    ]


class ReplayResult(ctypes.Structure):
    """NumiClothReplayResult (include/numi_cloth_replay.h)."""

    _fields_ = [
        ("hash", ctypes.c_uint64), ("replayHash", ctypes.c_uint64),
        ("deterministic", ctypes.c_uint32), ("failure", ctypes.c_uint32),
        ("particles", ctypes.c_uint32), ("fruits", ctypes.c_uint32),
        ("renderTriangles", ctypes.c_uint32), ("generation", ctypes.c_uint32),
        ("residuals", ctypes.c_double * 4),
        ("selfContacts", ctypes.c_ulonglong), ("edgeContacts", ctypes.c_ulonglong * 2),
        ("masks", ctypes.c_uint32 * 2), ("reconcileMax", ctypes.c_uint32), ("certificateMax", ctypes.c_uint32),
        ("seconds", ctypes.c_double),
        ("regrabCount", ctypes.c_uint32), ("patchSelections", ctypes.c_uint32),
        ("maxPatchRingShift", ctypes.c_uint32), ("patchCenter", ctypes.c_uint32),
        ("patchParticlesUnique", ctypes.c_uint32), ("patchTopologyExact", ctypes.c_uint32),
        ("inactiveGripSubsteps", ctypes.c_uint64),
    ]
