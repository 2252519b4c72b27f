/*
 * numi_cloth_scene.h - host-side scene builders and input contracts.
 *
 * These replace the reference host's scene construction and file contracts:
 *   - produce bag:   makeCloth / makeBalls (tools/cloth_bag.cpp:610-973) and
 *                    the Metal twin makeInitialState with greedy colouring
 *                    (tools/cloth_bag_metal.mm:524-1274);
 *   - square cloth:  not in the reference; a row-major s x s weave with
 *                    warp/weft, both shear diagonals and skip-one bends;
 *   - material:      numi.cloth.material.v1 (include/numi/cloth_material.h:112-192);
 *   - trajectory:    numi.grip.trajectory.v1..v3 (include/numi/grip_trajectory.h:189-362).
 * A built scene owns its arrays; numi_cloth_scene_view exposes them as the
 * NumiClothScene that numi_cloth_create takes.
 */
#ifndef NUMI_CLOTH_SCENE_H
#define NUMI_CLOTH_SCENE_H

#include "numi_cloth.h"

#ifdef __cplusplus
extern "C" {
#endif

/* The 19 calibrated parameters of numi.cloth.material.v1
 * (include/numi/cloth_material.h:18-38), in artifact order. */
typedef struct NumiClothMaterial {
    double ordinaryNodeMassKg;
    double hemNodeMassKg;
    double yarnRadiusM;
    double axialBodyComplianceMPerN;
    double axialCuffComplianceMPerN;
    double knotCompliance;
    double bendBodyComplianceMPerN;
    double bendCuffComplianceMPerN;
    double gripComplianceMPerN;
    double clothGroundFriction;
    double clothSelfFriction;
    double fruitYarnFriction;
    double fruitGroundFriction;
    double fruitPairFriction;
    double fruitRollingResistance;
    double yarnCrossflowDrag;
    double yarnSkinFriction;
    double fruitDrag;
    double fruitRotationalDrag;
} NumiClothMaterial;

/* Authored defaults (cloth_material.h:18-38). */
void numi_cloth_material_defaults(NumiClothMaterial* out);

/* Parse a numi.cloth.material.v1 artifact.  Returns 0, or -1 with a
 * message in err (same rejections as loadClothMaterialArtifact). */
int numi_cloth_material_load(const char* path, NumiClothMaterial* out,
                             char* err, size_t err_size);

/* Reference scenarios of the produce bag (tools/cloth_bag.cpp:66-71). */
enum {
    NUMI_CLOTH_SCENARIO_GROUNDED = 0,
    NUMI_CLOTH_SCENARIO_SPIN = 1,
    NUMI_CLOTH_SCENARIO_PICKUP = 2,
    NUMI_CLOTH_SCENARIO_RECORDED = 3
};

typedef struct numi_cloth_scene numi_cloth_scene_t;

/* The produce bag: 1,465 particles, 12 fruits, 10 seam grips (no grips in
 * the grounded scenario).  timestep is the substep dt written to Config. */
numi_cloth_scene_t* numi_cloth_scene_bag(const NumiClothMaterial* material,
                                         int scenario, double timestep,
                                         int select_nearest_cuff_patch);

/* Square cloth spec (no reference counterpart). */
typedef struct NumiClothSquareSpec {
    uint32_t side;             /* particles per row */
    double spacing;            /* m */
    double height;             /* initial z of the cloth plane, m */
    double particleMass;       /* kg */
    double stretchCompliance;  /* warp/weft, m/N */
    double shearCompliance;    /* both diagonals, m/N */
    double bendCompliance;     /* skip-one chords, m/N */
    double strainLimit;        /* max relative extension of warp/weft */
    double gripCompliance;     /* m/N; corner attachments */
    uint32_t gripCorners;      /* 0, 1 (corner 0) or 2 (corners 0 and side-1) */
    uint32_t fruitCount;       /* spheres (<= 64), seeded, none overlapping another;
                                  the builder returns NULL when 4096 draws find no room */
    double fruitRadiusMin, fruitRadiusMax, fruitMass;
    double fruitHeightMin, fruitHeightMax;   /* height of the sphere bottom */
    double thickness;          /* yarn radius r; self contact distance 2r */
    uint64_t seed;
    double timestep;
    uint32_t groundEnabled;
} NumiClothSquareSpec;

void numi_cloth_square_defaults(NumiClothSquareSpec* out);
numi_cloth_scene_t* numi_cloth_scene_square(const NumiClothSquareSpec* spec,
                                            const NumiClothMaterial* material);

void numi_cloth_scene_destroy(numi_cloth_scene_t* scene);

/* Borrowed view of the scene arrays (valid until destroy). */
int numi_cloth_scene_view(const numi_cloth_scene_t* scene, NumiClothScene* out);

/* Counts: particles, distances, knots, bends, grips, fruits, fruit pairs,
 * cuff ring count, mouth rim count, distance colours, knot colours,
 * bend colours, pair colours, yarn segments, bottom centre. */
int numi_cloth_scene_counts(const numi_cloth_scene_t* scene, uint32_t out[15]);

/* Render triangles (3 indices each; the bag's are the reference's
 * renderTriangles, tools/cloth_bag.cpp:812-839; the square's two per quad).
 * Copies at most capacity triangles into out (may be NULL); returns the
 * triangle count. */
uint32_t numi_cloth_scene_triangles(const numi_cloth_scene_t* scene, uint32_t* out, uint32_t capacity);

/* The bag's grip handle: the authored top-ring particle 0 in FP64, lifted
 * for the spin scenario (tools/cloth_bag.cpp:475-527, :1476-1480). */
int numi_cloth_bag_handle_base(int scenario, double out[3]);

/* Scripted grip target of the spin and pickup scenarios at time t (s)
 * (spinGripTarget, pickupGripTarget, tools/cloth_bag.cpp:1476-1502). */
int numi_cloth_bag_grip_target(int scenario, double time, double out[3]);

/* Per-substep Configs of the grounded, spin and pickup scenarios for
 * substeps first..first+count-1 (recorded runs use
 * numi_cloth_trajectory_configs): the grip target of the end of each
 * substep with identity orientation (updateGrip, tools/cloth_bag.cpp:1621-1627);
 * grounded copies base.  targets (count x 3, may be NULL) receives the FP64
 * grip targets. */
int numi_cloth_bag_scenario_configs(int scenario, const NumiClothConfig* base, uint64_t first_substep,
                                    uint32_t count, double timestep, NumiClothConfig* out, double* targets);

/* Rest positions in FP64 (the values the FP32 records were rounded from). */
int numi_cloth_scene_rest_fp64(const numi_cloth_scene_t* scene, double* out_xyz);

/* Grip trajectory (v1..v3).  Loading rejects exactly what the reference
 * loader rejects; the message lands in err. */
typedef struct numi_cloth_trajectory numi_cloth_trajectory_t;
numi_cloth_trajectory_t* numi_cloth_trajectory_load(const char* path, char* err,
                                                    size_t err_size);
void numi_cloth_trajectory_destroy(numi_cloth_trajectory_t* trajectory);

typedef struct NumiClothGripPose {
    double time;
    double translation[3];
    double orientation[4];     /* xyzw */
    uint32_t active;
    uint32_t generation;
} NumiClothGripPose;

int numi_cloth_trajectory_sample(const numi_cloth_trajectory_t* trajectory,
                                 double time, NumiClothGripPose* out);
/* 1 for v3 (nearest-cuff-patch re-grab), else 0; duration in seconds. */
int numi_cloth_trajectory_info(const numi_cloth_trajectory_t* trajectory,
                               uint32_t* select_nearest, double* duration,
                               uint64_t* fingerprint);

/* Schema version (1..3), pose count, the largest pose rotation angle
 * 2 acos|w| (radians) and the highest attachment generation: the summary
 * the reference CLI prints (maximumGripTrajectoryRotation,
 * gripTrajectoryAttachmentGenerations, include/numi/grip_trajectory.h:371-389). */
int numi_cloth_trajectory_summary(const numi_cloth_trajectory_t* trajectory, uint32_t* version,
                                  uint32_t* poses, double* max_rotation, uint32_t* generations);

/* Fill count per-substep Configs from base for substeps first..first+count-1:
 * the grip pose is sampled at the end of each substep, (k+1)*dt
 * (tools/cloth_bag.cpp:4776-4779), relative to handle_base. */
int numi_cloth_trajectory_configs(const numi_cloth_trajectory_t* trajectory,
                                  const NumiClothConfig* base,
                                  const double handle_base[3],
                                  uint64_t first_substep, uint32_t count,
                                  double timestep, NumiClothConfig* out);

#ifdef __cplusplus
}
#endif

#endif /* NUMI_CLOTH_SCENE_H */
