/*
 * numi_cloth_replay.h - replay harness of the produce-bag scenarios on the
 * GPU path (host side, above numi_cloth.h).
 *
 * The reference CLI (tools/cloth_bag.cpp:5504-5760) runs a scenario
 * (grounded, spin, pickup, recorded with a grip trajectory) frame after
 * frame, optionally twice, hashes the final state (hashResult, :5312-5360),
 * and writes OBJ frames (dumpOBJ, :5362-5400).  numi_cloth_replay does the
 * same on one numi_cloth handle through the public C API; the state hash
 * and OBJ writer are the reference's, applied to the FP32 state widened to
 * FP64.  numi-cloth-replay (replay_main.cpp) is the command line.
 */
#ifndef NUMI_CLOTH_REPLAY_H
#define NUMI_CLOTH_REPLAY_H

#include <stddef.h>
#include <stdint.h>

#include "numi_cloth.h"

#ifdef __cplusplus
extern "C" {
#endif

/* The state hashResult covers, in FP64.  particleState: particles x 6
 * (position xyz, velocity xyz); fruitState: fruits x 13 (position xyz,
 * velocity xyz, angular velocity xyz, orientation w x y z); the grip target
 * and activity; for an attachment generation above 1 the grips' offsets and,
 * after a nearest-patch selection, their particles. */
typedef struct NumiClothHashState {
    uint32_t particles, fruits, grips;
    uint32_t gripActive;
    const double* particleState;
    const double* fruitState;
    double gripTarget[3];
    uint32_t generation;
    uint32_t patchSelections;
    const uint32_t* gripParticle;   /* grips */
    const double* gripOffset;       /* grips x 3 */
} NumiClothHashState;

/* FNV-1a over the bytes of every value, the reference's hashResult. */
uint64_t numi_cloth_state_hash(const NumiClothHashState* state);

/* One OBJ frame in the reference's dumpOBJ format.  fruitState: fruits x 11
 * (centre xyz, radius, orientation w x y z, angular velocity xyz). */
typedef struct NumiClothObjState {
    uint32_t particles;
    uint32_t triangles;
    const double* positions;          /* particles x 3 */
    const uint32_t* triangleIndices;  /* triangles x 3, 0-based */
    int scenario;                     /* NUMI_CLOTH_SCENARIO_* */
    uint32_t gripActive;
    double gripTarget[3];
    double gripOrientationWxyz[4];
    uint32_t patchCenter;
    uint32_t fruits;
    const double* fruitState;
    const uint32_t* fruitAppearance;
} NumiClothObjState;

int numi_cloth_write_obj(const char* path, const NumiClothObjState* state);

typedef struct NumiClothReplayOptions {
    int scenario;                 /* NUMI_CLOTH_SCENARIO_* */
    uint32_t steps;               /* frames */
    uint32_t substeps;            /* per frame */
    uint32_t replays;             /* 1, or 2 to check the hash of a second run */
    double frameTimestep;         /* s */
    const char* material;         /* numi.cloth.material.v1 artifact or NULL */
    const char* gripTrajectory;   /* numi.grip.trajectory.v1..v3 (recorded) or NULL */
    const char* dumpObj;          /* OBJ of the final state or NULL */
    const char* dumpFrames;       /* OBJ frame prefix or NULL */
    uint32_t dumpEvery;           /* 0: the quarters */
    uint32_t pad;
    NumiClothSchedule schedule;
} NumiClothReplayOptions;

typedef struct NumiClothReplayResult {
    uint64_t hash;
    uint64_t replayHash;
    uint32_t deterministic;       /* replays = 2 and equal hashes */
    uint32_t failure;             /* NUMI_CLOTH_FAILURE_* bits */
    uint32_t particles, fruits, renderTriangles, generation;
    double residuals[4];          /* numi_cloth_residuals */
    unsigned long long selfContacts;
    unsigned long long edgeContacts[2];
    uint32_t masks[2];            /* mouth candidates, released fruits (numi_cloth_release_masks) */
    uint32_t reconcileMax;        /* most reconciliation passes of a substep */
    uint32_t certificateMax;      /* most certificate passes of a substep */
    double seconds;               /* wall time of the first run's frames */
    /* grip metrics of the first run (tools/cloth_bag.cpp:1563-1620, 5409-5437) */
    uint32_t regrabCount;         /* attachments of a new generation */
    uint32_t patchSelections;     /* nearest-cuff-patch selections (v3) */
    uint32_t maxPatchRingShift;   /* largest cyclic ring shift between selections */
    uint32_t patchCenter;         /* centre ring of the last selected patch */
    uint32_t patchParticlesUnique;/* 1: no two grips hold one particle */
    uint32_t patchTopologyExact;  /* 1: the grips are the 2 x 5 patch around patchCenter */
    uint64_t inactiveGripSubsteps;/* substeps with the grip released */
} NumiClothReplayResult;

/* Run the scenario; err receives a message on a rejected input. */
int numi_cloth_replay(const NumiClothReplayOptions* options, NumiClothReplayResult* result, char* err,
                      size_t err_size);

#ifdef __cplusplus
}
#endif

#endif
