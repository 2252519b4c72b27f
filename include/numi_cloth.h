/*
 * numi_cloth.h - C ABI of the B200 XPBD cloth substep.
 *
 * Record layouts are byte-identical to the pointer-free GPU ABI v13 of the
 * reference cloth path (include/numi/cloth_bag_gpu.h:19-190, sizes asserted
 * at :192-209), so a caller that already fills those buffers for the Metal
 * encoder (tools/cloth_bag_metal.mm:4091-4202) can hand the same bytes to
 * this library.  The functions replace the reference's Metal host entry
 * runGPU (tools/cloth_bag_metal.mm:4010) and its per-substep command
 * encoding (tools/cloth_bag_metal.mm:4211-4709).
 *
 * Conventions
 *   - Caller owns host arrays; they are copied in and out.  The library owns
 *     all device buffers of a handle.
 *   - No exceptions cross the ABI.  Functions return NUMI_CLOTH_OK (0) or a
 *     negative NUMI_CLOTH_E* code; stepping returns the reference failure
 *     word (bits below) and a TIMEOUT bit for a bounded barrier wait.
 *   - One handle = one GPU (the current device at create time) and one
 *     CUDA stream.  A handle is not thread-safe; distinct handles are.
 *   - Deterministic: no floating-point atomics touch simulated state, so two
 *     runs from the same inputs are bit-identical.
 */
#ifndef NUMI_CLOTH_H
#define NUMI_CLOTH_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#define NUMI_CLOTH_ALIGN16 alignas(16)
#else
#define NUMI_CLOTH_ALIGN16 _Alignas(16)
#endif

/* ABI version of the record layouts (reference cloth_bag_gpu.h:5). */
#define NUMI_CLOTH_ABI_VERSION 13u
#define NUMI_CLOTH_INVALID_PARTICLE 0xffffffffu
#define NUMI_CLOTH_MOUTH_RIM_CAPACITY 64u

/* Failure word (reference cloth_bag_gpu.h:10-17) plus TIMEOUT. */
enum {
    NUMI_CLOTH_FAILURE_NONE = 0u,
    NUMI_CLOTH_FAILURE_ABI = 1u << 0,
    NUMI_CLOTH_FAILURE_RANGE = 1u << 1,
    NUMI_CLOTH_FAILURE_BATCH = 1u << 2,
    NUMI_CLOTH_FAILURE_NONFINITE = 1u << 3,
    NUMI_CLOTH_FAILURE_GRIP_CAPTURE = 1u << 4,
    /* A grid barrier wait ran past its iteration limit; the kernel stopped
     * at a phase boundary and the state is that of the last full phase. */
    NUMI_CLOTH_FAILURE_TIMEOUT = 1u << 5
};

/* Return codes of the non-stepping functions. */
enum {
    NUMI_CLOTH_OK = 0,
    NUMI_CLOTH_EINVAL = -1,   /* bad argument, size or layout */
    NUMI_CLOTH_ECUDA = -2,    /* a CUDA runtime call failed */
    NUMI_CLOTH_EBATCH = -3,   /* colour batches are not conflict free */
    NUMI_CLOTH_ENOMEM = -4,
    NUMI_CLOTH_ESTATE = -5    /* handle is poisoned by an earlier failure */
};

typedef struct NUMI_CLOTH_ALIGN16 numi_float4 { float x, y, z, w; } numi_float4;
typedef struct NUMI_CLOTH_ALIGN16 numi_uint4 { uint32_t x, y, z, w; } numi_uint4;

/* 224 B.  Field meaning follows cloth_bag_gpu.h:19-57. */
typedef struct NUMI_CLOTH_ALIGN16 NumiClothConfig {
    numi_uint4 control;             /* x ABI, y particles, z distances, w grips */
    numi_uint4 constraintCounts;    /* x knots, y bends, z ground on/off, w fruits */
    numi_uint4 contactCounts;       /* x fruit pairs, y fruit*segments, z,w unused here */
    numi_float4 gravityAndTimestep; /* xyz gravity, w substep dt */
    numi_float4 gripTargetAndActive;/* xyz handle position, w >0 active */
    numi_float4 gripOrientation;    /* unit quaternion xyzw */
    numi_uint4 gripControl;         /* x generation, y 1 = nearest cuff patch,
                                       z knots per cuff row, w patch half width */
    numi_float4 gripMaterial;       /* x capture radius */
    numi_float4 clothMaterial;      /* x yarn radius, y self cell, z ground mu, w self mu */
    numi_float4 fruitMaterial;      /* x pair mu, y ground mu, z rolling, w fruit/yarn mu */
    numi_float4 airVelocityAndDensity;
    numi_float4 aerodynamicCoefficients; /* yarn crossflow, yarn skin, fruit, fruit rot */
    numi_uint4 mouthControl;        /* x rim count, y bottom centre */
    numi_float4 mouthMaterial;      /* x release hysteresis */
} NumiClothConfig;

/* 48 B (cloth_bag_gpu.h:59-66). */
typedef struct NUMI_CLOTH_ALIGN16 NumiClothParticle {
    numi_float4 positionAndInverseMass;
    numi_float4 previousAndMass;
    numi_float4 velocity;           /* w: cloth/ground normal impulse */
} NumiClothParticle;

/* 32 B (cloth_bag_gpu.h:66-72).  particlesAndColor.w is the yarn kind:
 * 0 warp, 1 weft, 2 bottom, 3 shear (shear is not a yarn segment: it takes
 * no fruit contact and no air load).  material.w <= 0 disables the strain
 * limiter for that constraint. */
typedef struct NUMI_CLOTH_ALIGN16 NumiClothDistance {
    numi_uint4 particlesAndColor;
    numi_float4 material;           /* rest, compliance, lambda, max extension */
} NumiClothDistance;

/* 48 B (cloth_bag_gpu.h:74-82). */
typedef struct NUMI_CLOTH_ALIGN16 NumiClothGrip {
    numi_uint4 particle;            /* particle, generation, capture bits, ring */
    numi_float4 targetOffsetAndCompliance;
    numi_float4 lambda;
} NumiClothGrip;

/* 48 B (cloth_bag_gpu.h:84-91). */
typedef struct NUMI_CLOTH_ALIGN16 NumiClothKnot {
    numi_uint4 particles;           /* warp first, warp second, weft first, weft second */
    numi_uint4 control;             /* x colour */
    numi_float4 material;           /* rest cosine, compliance, lambda */
} NumiClothKnot;

/* 32 B (cloth_bag_gpu.h:93-98). */
typedef struct NUMI_CLOTH_ALIGN16 NumiClothBend {
    numi_uint4 particlesAndColor;   /* first, middle, third, colour */
    numi_float4 material;           /* rest chord, rest arc, compliance, lambda */
} NumiClothBend;

/* 96 B (cloth_bag_gpu.h:100-113). */
typedef struct NUMI_CLOTH_ALIGN16 NumiClothFruit {
    numi_float4 positionAndInverseMass;
    numi_float4 previousAndRadius;
    numi_float4 velocityAndGroundImpulse;
    numi_float4 angularVelocity;
    numi_float4 orientation;
    numi_uint4 identity;
} NumiClothFruit;

/* 32 B (cloth_bag_gpu.h:115-120). */
typedef struct NUMI_CLOTH_ALIGN16 NumiClothFruitPair {
    numi_uint4 fruitsAndColor;
    numi_float4 contact;
} NumiClothFruitPair;

/* 16 B (cloth_bag_gpu.h:184-188). */
typedef struct NUMI_CLOTH_ALIGN16 NumiClothBatch {
    numi_uint4 control;             /* first, count, colour, reserved */
} NumiClothBatch;

/* Per-substep schedule.  The reference CPU oracle fixes these at
 * iterations=CLI, strain sweeps=3, reconciliation<=8 with early exit,
 * final passes=2, certificate<=128 on the last substep of a frame
 * (tools/cloth_bag.cpp:4891-5185). */
typedef struct NumiClothSchedule {
    uint32_t iterations;
    uint32_t strainSweeps;          /* sweeps per strain-limiter call */
    uint32_t reconcilePasses;       /* maximum reconciliation passes */
    uint32_t finalPasses;           /* final contact passes */
    uint32_t certificatePasses;     /* maximum, last substep of a call only */
    uint32_t earlyExit;             /* 1: stop reconcile/certificate on residuals */
    uint32_t selfCollision;         /* 1: point/point hash-grid self contact */
    uint32_t aerodynamics;          /* 1: yarn and fruit air loads */
    uint32_t sweptGround;           /* 1: swept ground prediction after advance */
    uint32_t sweptFruitYarn;        /* 1: swept fruit/yarn contact before iterations */
    uint32_t frictions;             /* 1: apply the Coulomb/rolling frictions */
    uint32_t release;               /* 1: update the mouth release masks */
    float damping;                  /* v <- v/(1+c dt) after gravity; 0 = reference */
    uint32_t primitiveSelf;         /* 1: edge/edge yarn self-collision (swept before
                                       the iterations, present at every endpoint),
                                       its certificate test and yarn/yarn self
                                       friction (tools/cloth_bag.cpp:3880-4247) */
    uint32_t reserved[2];
} NumiClothSchedule;

/* Scene handed to numi_cloth_create.  Constraint arrays must be grouped in
 * contiguous colour runs (one batch per run); the library checks that no
 * two records of a batch write the same particle or fruit. */
typedef struct NumiClothScene {
    const NumiClothConfig* config;
    const NumiClothParticle* particles;
    const numi_float4* restPositions;    /* xyz rest, used for inverse mass 0; may be NULL */
    const NumiClothDistance* distances;
    const NumiClothKnot* knots;
    const NumiClothBend* bends;
    const NumiClothGrip* grips;
    const NumiClothFruit* fruits;
    const NumiClothFruitPair* fruitPairs;
    const uint32_t* cuffParticles;       /* 2 rows x gripControl.z ring particles */
    const uint32_t* mouthRim;            /* mouthControl.x ordered rim particles */
    /* 2-hop local topology excluded from self contact (tools/cloth_bag.cpp:842-861):
     * CSR over particles, each row sorted ascending.  When localOffsets is
     * NULL and gridWidth > 0, particles are a gridWidth-wide row-major grid
     * and the local set is the Chebyshev ball of radius 2. */
    const uint32_t* localOffsets;
    const uint32_t* localIndices;
    uint32_t gridWidth;
    uint32_t reserved[3];
} NumiClothScene;

typedef struct numi_cloth numi_cloth_t;

/* Create a solver on the current CUDA device.  Returns NUMI_CLOTH_OK and a
 * handle, or a negative code (NUMI_CLOTH_EBATCH for a colouring conflict). */
int numi_cloth_create(const NumiClothScene* scene, numi_cloth_t** out);
void numi_cloth_destroy(numi_cloth_t* handle);

/* Velocity damping of this cloth, v <- v / (1 + c dt) after gravity, in
 * place of the schedule's `damping` (c < 0 restores the schedule's).  Set it
 * before adding the cloth to a batch.  No reference counterpart: the
 * reference has no damping term (c = 0 is the reference). */
int numi_cloth_set_damping(numi_cloth_t* handle, float damping);

/* Launch on this CUDA stream (cudaStream_t passed as void*; NULL = default). */
int numi_cloth_set_stream(numi_cloth_t* handle, void* stream);

/* Advance count substeps.  configs[i] is the live Config of substep i (the
 * reference's trajectoryConfigs, ClothBag.metal:466-489); only grip pose,
 * grip generation, timestep and gravity may change between substeps.  The
 * last substep of the call runs the certificate loop.  Asynchronous on the
 * handle's stream; returns NUMI_CLOTH_OK or a negative code.  Read the
 * failure word with numi_cloth_failure.  The Configs are copied on the
 * stream: pageable ones may be reused on return, pinned ones only after the
 * stream has passed the step. */
int numi_cloth_step(numi_cloth_t* handle, const NumiClothConfig* configs,
                    uint32_t count, const NumiClothSchedule* schedule);

/* Synchronise the stream and return the accumulated failure word. */
uint32_t numi_cloth_failure(numi_cloth_t* handle);

/* Host copies of the state (synchronous).  Particle records travel as one
 * copy through a device staging buffer, transposed to and from the state
 * arrays on the device; pinned host buffers copy fastest. */
int numi_cloth_read_particles(numi_cloth_t* handle, NumiClothParticle* out, uint32_t count);
int numi_cloth_write_particles(numi_cloth_t* handle, const NumiClothParticle* in, uint32_t count);
int numi_cloth_read_fruits(numi_cloth_t* handle, NumiClothFruit* out, uint32_t count);
int numi_cloth_write_fruits(numi_cloth_t* handle, const NumiClothFruit* in, uint32_t count);
int numi_cloth_read_distances(numi_cloth_t* handle, NumiClothDistance* out, uint32_t count);
int numi_cloth_read_grips(numi_cloth_t* handle, NumiClothGrip* out, uint32_t count);

/* Residuals of the current state, reduced in FP64 on the device:
 * out[0] max strain-limit violation (m), out[1] max ground penetration (m),
 * out[2] max fruit/yarn penetration (m), out[3] max self penetration (m). */
int numi_cloth_residuals(numi_cloth_t* handle, double out[4]);

/* Point self-contact counters since create: pairs resolved and the largest
 * penetration resolved (m), the reference's metrics.selfContacts and
 * maximumSelfPenetration (tools/cloth_bag.cpp:4949-4958).  Zero until a
 * step ran with selfCollision. */
int numi_cloth_self_contacts(numi_cloth_t* handle, unsigned long long* contacts, double* max_penetration);

/* How the point self-contact passes since create kept the reference's
 * Gauss-Seidel order: out[0] passes whose phase A listed coupled pairs (the
 * ordered pass ran), out[1] pairs listed over those passes, out[2]
 * ordered-pass rounds, out[3] passes resolved by the serial fallback.  No
 * counterpart in the reference, whose pass is serial.  Zero until a step ran
 * with selfCollision. */
int numi_cloth_self_order_stats(numi_cloth_t* handle, unsigned long long out[4]);

/* Edge/edge yarn self-collision counters since create: out[0] edge/edge
 * solves that moved particles (the reference's edgeEdgeSelfContacts plus
 * sweptEdgeEdgeSelfContacts), out[1] yarn/yarn self-friction contacts
 * (clothSelfFrictionContacts), tools/cloth_bag.cpp:3986-3992, 4085.  Zero
 * until a step ran with primitiveSelf. */
int numi_cloth_edge_contacts(numi_cloth_t* handle, unsigned long long out[2]);

/* Release masks after the last step: out[0] fruits that entered the mouth
 * (candidates), out[1] fruits released, one bit per fruit, sticky since
 * create (updateReleasedFruit, tools/cloth_bag.cpp:4545-4597).  Updated
 * every substep of a step whose schedule has release = 1. */
int numi_cloth_release_masks(numi_cloth_t* handle, uint32_t out[2]);

/* Launch-shape tuner of one cloth on the cooperative grid: times `count`
 * substeps of `configs` under `schedule` for each colours-per-sync choice
 * the cloth and schedule allow (one constraint colour between
 * synchronisations, the colour-by-colour launch; or tile mode, whose CTAs
 * run every constraint colour of a substep on their closures between two
 * grid barriers, at the SM count, three quarters and half of it, in CTAs),
 * keeps the fastest, and leaves the cloth's state as it was.  out: [0]
 * constraint colours per synchronisation of the kept shape, [1] CTAs, [2]
 * threads per CTA, [3] its time for the configs in us (0: nothing to
 * choose).  ESTATE on a cloth whose failure word is set. */
int numi_cloth_tune(numi_cloth_t* handle, const NumiClothConfig* configs, uint32_t count,
                    const NumiClothSchedule* schedule, uint32_t out[4]);

/* Device-side snapshot of the full dynamic state into slot (0..7), and back. */
int numi_cloth_snapshot(numi_cloth_t* handle, uint32_t slot);
int numi_cloth_restore(numi_cloth_t* handle, uint32_t slot);

/* Launch geometry of the last step: grid CTAs, threads per CTA, barriers
 * per substep, kernel launches, cluster size (0: no cluster), and flags:
 * bit 0 when the particles are resident in (distributed) shared memory,
 * bit 1 when constraint colours are separated by neighbour syncs instead of
 * the grid barrier, bit 2 when the cloth has tile plans (colour chains run
 * on per-CTA closures in shared memory between grid barriers), bit 3 when
 * the last step ran in that tile mode, bit 4 when point self contact keeps
 * the reference's Gauss-Seidel order (NUMI_CLOTH_SELF_ORDER=reference at
 * create; else the batched order). */
int numi_cloth_launch_info(numi_cloth_t* handle, uint32_t out[6]);

/* Pass counters: out[0] barriers of the last substep, out[1] the most
 * reconciliation passes and out[2] the most certificate passes one substep
 * took since create (the reference's max_contact_reconciliation_passes and
 * max_primitive_certificate_passes, tools/cloth_bag.cpp:5838-5841). */
int numi_cloth_pass_counts(numi_cloth_t* handle, uint32_t out[3]);

/* Per-phase device timestamps of the last step (profiling aid).  Enabled
 * when the handle was created with NUMI_CLOTH_TRACE=<substeps> in the
 * environment; out receives substeps x slots (slots must be 128) globaltimer
 * values in ns, one per grid barrier in program order, 0 where unused.
 * Returns NUMI_CLOTH_ESTATE when tracing is off.  No reference counterpart:
 * the reference records only command-buffer GPU start/end times
 * (tools/cloth_bag_metal.mm:4758-4760). */
int numi_cloth_trace(numi_cloth_t* handle, unsigned long long* out,
                     uint32_t substeps, uint32_t slots);

/* Per-CTA barrier arrival stamps of the last step, [substeps][128][CTAs of
 * that launch] (ns; numi_cloth_launch_info's grid), when the handle was also
 * created with NUMI_CLOTH_TRACE_CTA=1. */
int numi_cloth_trace_cta(numi_cloth_t* handle, unsigned long long* out, uint32_t substeps);

/* ---------------------------------------------------------------------------
 * Allocation-free stepping.  No counterpart in the reference: its Metal host
 * always allocates its own buffers (tools/cloth_bag_metal.mm:4091-4202).
 *
 * For callers that cannot let the library allocate GPU memory: hosts that
 * own every device byte through their own pool or arena (a simulator that
 * sizes its device heap once at start-up, a game or robot controller that
 * forbids allocation once its real-time loop runs), and hosts for which a
 * cudaMalloc is too costly mid-run because it may synchronise the whole
 * device.  The caller passes every input and output as device buffers in the
 * library's structure-of-arrays layout; the library's own scratch (contact
 * records, air forces, fixed-point fruit sums, reduction partials, the
 * substep Configs) lives in one statically allocated device array of about
 * 1.2 MB that every GPU that loads the library keeps until the process
 * exits.  No call allocates device memory: no cudaMalloc, no cudaFree and no
 * allocating library routine.
 *
 * Limits: at most NUMI_CLOTH_NOALLOC_MAX_PARTICLES particles,
 * NUMI_CLOTH_NOALLOC_MAX_DISTANCES distances, 64 fruits, 32 grips, 2,016
 * fruit pairs, 64 colour runs per family and NUMI_CLOTH_NOALLOC_MAX_SUBSTEPS
 * substeps per call; larger inputs are rejected with NUMI_CLOTH_EINVAL, and
 * so is a colour run that reaches past its family's record count (or whose
 * yarn or strain-limited prefix is longer than the run), and a schedule with
 * selfCollision (the point self-contact hash grid is not part of the static
 * scratch), primitiveSelf (nor are the edge/edge pass buffers) or release
 * (the state carries no mouth rim).  The colouring itself is the caller's
 * contract: the kernel checks every particle index it reads against the
 * particle count (an index out of range sets NUMI_CLOTH_FAILURE_RANGE and the
 * item is skipped), but two items of one run that share a particle are not
 * detected.  The cloth runs on one CTA (the resident small-cloth path).
 *
 * The first call on a device looks up the scratch array's device address
 * (once per device, with that device current) and keeps it for the life of
 * the process; after a cudaDeviceReset of that device the kept address is
 * stale, so do not use this entry point after a reset.  All calls share the
 * one scratch array and every call clears the parts that must start at zero
 * and keeps nothing from the call before, so calls whose kernels overlap on
 * the GPU (different streams, no ordering between them) race on it: order
 * them on one stream or with events.
 * ------------------------------------------------------------------------ */
#define NUMI_CLOTH_NOALLOC_MAX_PARTICLES 4096u
#define NUMI_CLOTH_NOALLOC_MAX_DISTANCES 8192u
#define NUMI_CLOTH_NOALLOC_MAX_SUBSTEPS 256u

/* Device buffers of one cloth, library layout (float4 = 4 floats). */
typedef struct NumiClothDeviceState {
    float* positions;              /* float4[N] xyz, inverse mass        (in/out) */
    float* previous;               /* float4[N] xyz, mass                (in/out) */
    float* velocities;             /* float4[N] xyz, ground impulse      (in/out) */
    const float* rest;             /* float4[N] rest positions           (in) */
    const uint32_t* distanceIJ;    /* uint2[D] particle pair, colour-run order (in) */
    const float* distanceMaterial; /* float4[D] rest, compliance, 0, max extension (in) */
    float* distanceLambda;         /* float[D]                           (out) */
    const uint32_t* knotIJ;        /* uint4[K]                           (in) */
    const float* knotMaterial;     /* float2[K] rest cosine, compliance  (in) */
    float* knotLambda;             /* float[K]                           (out) */
    const uint32_t* bendIJ;        /* uint4[B] first, middle, third, 0   (in) */
    const float* bendMaterial;     /* float2[B] rest chord, compliance   (in) */
    float* bendLambda;             /* float[B]                           (out) */
    NumiClothGrip* grips;          /* [G]                                (in/out) */
    NumiClothFruit* fruits;        /* [F]                                (in/out) */
    NumiClothFruitPair* fruitPairs;/* [P]                                (in/out) */
    const uint32_t* cuffParticles; /* 2 x ring count, or NULL            (in) */
    uint32_t* failure;             /* one word: zeroed, then failure bits (out) */
} NumiClothDeviceState;

/* Advance count substeps of the cloth described by base (counts, material)
 * and state, on stream (cudaStream_t as void*), without allocating.
 * batches holds the distance, knot, bend and fruit-pair colour runs, in that
 * order, batchCounts[4] of each; control = (first, count, colour, x) where for
 * distance runs x = yarn-prefix count | strain-limited-prefix count << 16.
 * configs (host) are validated as by numi_cloth_step; an invalid one sets
 * its failure bit in the host-visible return value and nothing runs.
 * Returns NUMI_CLOTH_OK, NUMI_CLOTH_EINVAL (size over a limit, bad
 * argument, with a message on stderr) or NUMI_CLOTH_ECUDA; a rejected Config
 * returns its failure bit as a positive value. */
int numi_cloth_step_noalloc(const NumiClothConfig* base, const NumiClothDeviceState* state,
                            const NumiClothBatch* batches, const uint32_t batchCounts[4],
                            const NumiClothConfig* configs, uint32_t count,
                            const NumiClothSchedule* schedule, void* stream);

/* ------------------------------------------------------------------------
 * Reverse-mode gradients of a rollout.  No reference counterpart: the
 * reference calibrates with finite-difference sensitivities computed
 * outside the simulator (docs/CLOTH_SPECIMEN_CALIBRATION.md:52-82); this
 * feeds a gradient-based fitter.
 *
 * Compliance groups are the distinct compliance values of each constraint
 * family (family 0 distance, 1 knot, 2 bend, 3 grip), ascending, family by
 * family: on the produce bag the axial body and cuff distances, the knots,
 * the bend body and cuff, and the grips; on a square cloth the stretch and
 * shear distances, the bends and the grips.  numi_cloth_compliance_groups
 * lists them (at most NUMI_CLOTH_MAX_GROUPS); numi_cloth_replace_compliance
 * sets every record of `family` whose compliance equals `from` to `to`
 * (how a fitter applies a new group value).
 *
 * numi_cloth_rollout_grad advances the cloth by `substeps` substeps
 * (configs as numi_cloth_step), checkpointing the state every
 * `checkpoint_every` substeps, and returns the loss L = sum over the
 * substeps s with (s + 1) % loss_every == 0 of
 * sum_t |x_tracked[t](s) - target(s, t)|^2 (targets: [substeps / loss_every]
 * [n_tracked][3], m) and its gradients, reduced in FP64:
 *   grads[g]      dL / d log-scale of compliance group g (count + 1 entries);
 *   grads[count]  dL / d damping c (v <- v / (1 + c dt));
 *   grip_grads    (optional, [substeps][6]) dL / d grip target position xyz
 *                 and dL / d a small rotation (axis-angle, applied before
 *                 the grip orientation) of each substep's Config.
 * The state after the call is the state after the rollout.
 *
 * Supported schedules: iterations = 1, no reconciliation, final or
 * certificate passes, aerodynamics = 0, selfCollision = 0.  Fruit contacts,
 * cloth/ground friction, the swept ground and bend ground active sets are
 * not differentiated: the number of such events met is returned in
 * *nonsmooth (0 = the gradient is exact for the discrete forward).  Returns
 * NUMI_CLOTH_EINVAL for unsupported schedules. */
#define NUMI_CLOTH_MAX_GROUPS 16u
int numi_cloth_compliance_groups(numi_cloth_t* handle, uint32_t family[NUMI_CLOTH_MAX_GROUPS],
                                 float compliance[NUMI_CLOTH_MAX_GROUPS], uint32_t* count);
int numi_cloth_replace_compliance(numi_cloth_t* handle, uint32_t family, float from, float to);
int numi_cloth_rollout_grad(numi_cloth_t* handle, const NumiClothConfig* configs, uint32_t substeps,
                            const NumiClothSchedule* schedule, uint32_t checkpoint_every,
                            const uint32_t* tracked, uint32_t n_tracked, const double* targets,
                            uint32_t loss_every, double* loss, double* grads, double* grip_grads,
                            uint32_t* nonsmooth);

/* ------------------------------------------------------------------------
 * Batched stepping: many independent cloths (same device) advanced by one
 * persistent kernel launch per step.  Every CTA takes the next cloth from a
 * device work queue, largest first, and runs its whole frame alone.  No
 * reference counterpart: the reference runs one cloth per process
 * (tools/cloth_bag_metal.mm:4010-4760); this is the batched forward of the
 * square-cloth instances and of calibration candidates.
 *
 * The batch borrows the handles: destroy it before them.  Each cloth's
 * state stays in its handle, so numi_cloth_read_* / numi_cloth_failure /
 * snapshot / restore work on batch members as on single cloths.
 * ------------------------------------------------------------------------ */
typedef struct numi_cloth_batch numi_cloth_batch_t;

int numi_cloth_batch_create(numi_cloth_t* const* cloths, uint32_t count, numi_cloth_batch_t** out);
void numi_cloth_batch_destroy(numi_cloth_batch_t* batch);
int numi_cloth_batch_set_stream(numi_cloth_batch_t* batch, void* stream);

/* Advance every cloth by `substeps` substeps.  configs holds count x
 * substeps Configs, cloth-major in the order the cloths were given (cloth
 * k's substeps start at k * substeps); each is validated against its
 * cloth's creation Config as numi_cloth_step does. */
int numi_cloth_batch_step(numi_cloth_batch_t* batch, const NumiClothConfig* configs, uint32_t substeps,
                          const NumiClothSchedule* schedule);

/* Launch shape: out[0] resident particle chunk (cloths with at most that
 * many particles keep them in shared memory; 0 = none), out[1] threads per
 * CTA, out[2] CTAs of the persistent launch. */
int numi_cloth_batch_shape(numi_cloth_batch_t* batch, uint32_t out[3]);
/* A shape whose resident chunk leaves no shared memory for the edge/edge
 * family's box-tree sort keys (32 KB) serves only schedules with
 * primitiveSelf = 0: a step or capture with primitiveSelf on returns EINVAL
 * on it, and the tuner skips it for such schedules. */
int numi_cloth_batch_set_shape(numi_cloth_batch_t* batch, uint32_t resident_chunk, uint32_t threads);

/* Autotuner: times one step of every candidate shape (resident chunk 0,
 * 256 ... 4096; 256 or 512 threads) on the current state, restores the
 * state after each, and keeps the fastest; out (optional) receives it. */
int numi_cloth_batch_tune(numi_cloth_batch_t* batch, const NumiClothConfig* configs, uint32_t substeps,
                          const NumiClothSchedule* schedule, uint32_t out[3]);

/* CUDA graph of one step: the copy of `configs` (PINNED host memory the
 * caller keeps and may rewrite between replays; same layout as
 * numi_cloth_batch_step), the work-queue reset, the frame launch and the
 * substep-counter advance.  numi_cloth_batch_replay validates the current
 * contents of configs on the host and launches the graph. */
int numi_cloth_batch_capture(numi_cloth_batch_t* batch, const NumiClothConfig* configs, uint32_t substeps,
                             const NumiClothSchedule* schedule);
int numi_cloth_batch_replay(numi_cloth_batch_t* batch);

/* Gradients of every cloth of a batch: numi_cloth_rollout_grad for all
 * cloths at once, the forward of every cloth in one persistent launch per
 * checkpoint segment, the taped replays likewise, and the adjoint of every
 * cloth's segment in one grid (a CTA per cloth).  configs: count x substeps
 * cloth-major; tracked: shared by the cloths; targets: [count][substeps /
 * loss_every][n_tracked][3]; loss[count]; grads: [count][NUMI_CLOTH_MAX_GROUPS
 * + 1], cloth k's group gradients first (groups_out[k] of them, in the order
 * of numi_cloth_compliance_groups) then dL / d damping at index
 * groups_out[k]; nonsmooth[count] (optional).  Same schedule limits as
 * numi_cloth_rollout_grad. */
int numi_cloth_batch_rollout_grad(numi_cloth_batch_t* batch, const NumiClothConfig* configs, uint32_t substeps,
                                  const NumiClothSchedule* schedule, uint32_t checkpoint_every,
                                  const uint32_t* tracked, uint32_t n_tracked, const double* targets,
                                  uint32_t loss_every, double* loss, double* grads, uint32_t* groups_out,
                                  uint32_t* nonsmooth);

/* Library version string. */
const char* numi_cloth_version(void);

#ifdef __cplusplus
}
#endif

#endif /* NUMI_CLOTH_H */
