/*
 * oracle.h - C API of the CPU restatement of the reference XPBD cloth
 * substep (TEST INFRASTRUCTURE ONLY).
 *
 * This is the parity oracle.  Only tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py load it, as the checker; the product never
 * links it.  It restates tools/cloth_bag.cpp (the reference FP64 CPU
 * cloth) in two orders:
 *   ORACLE_SERIAL  - the reference CPU order: every constraint family in
 *                    array order, fruit-major fruit/yarn Gauss-Seidel,
 *                    hash-grid point self contact (tools/cloth_bag.cpp:4712-5310);
 *   ORACLE_BATCHED - the colour-batch schedule of the B200 kernels (colour
 *                    runs of the arrays; fruit/yarn with fruit positions
 *                    frozen over a sweep and summed; batched point self
 *                    contact: every pair at the start of the pass, sums
 *                    applied once);
 *   ORACLE_BATCHED_SELF_REFERENCE - the same with point self contact in the
 *                    reference's Gauss-Seidel order (the kernels built with
 *                    the ordered pass, NUMI_CLOTH_SELF_ORDER=reference).
 * and in two scalar types: 64 (the FP64 oracle) and 32 (float with the
 * kernels' exact evaluation order, fixed-point fruit sums and FP64 fixed-tree
 * air reductions, used to prove bit-identity of the GPU path).
 * Pinned to the compiled reference through oracle/_ref (ref_shim.cpp) and
 * the golden vectors under tests/golden/.
 */
#ifndef NUMI_CLOTH_ORACLE_H
#define NUMI_CLOTH_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct OracleParticle {
    double x[3];
    double w;
    double prev[3];
    double mass;
    double v[3];
    double vw;          /* predicted vertical velocity during a substep, ground impulse after */
    double rest[3];
    double pad;
} OracleParticle;       /* 128 B */

typedef struct OracleDistance {
    uint32_t i, j, colour, kind;   /* kind 3 = shear (not a yarn segment) */
    double rest, compliance, lambda, maxext;
} OracleDistance;       /* 48 B */

typedef struct OracleKnot {
    uint32_t p[4];
    uint32_t colour, pad[3];
    double restcos, compliance, lambda, pad2;
} OracleKnot;           /* 64 B */

typedef struct OracleBend {
    uint32_t p[3];
    uint32_t colour;
    double restchord, restarc, compliance, lambda;
} OracleBend;           /* 48 B */

typedef struct OracleGrip {
    uint32_t particle, gen, ring, pad;
    double offset[3];
    double compliance;
    double lambda[3];
    double capture;
    double error;
    double pad2[3];
} OracleGrip;           /* 112 B */

typedef struct OracleFruit {
    double x[3], w;
    double prev[3], radius;
    double v[3], ground_impulse;
    double omega[3], pad;
    double q[4];        /* xyzw */
    uint32_t appearance, pad2[3];
} OracleFruit;          /* 176 B */

typedef struct OraclePair {
    uint32_t a, b, colour, stable;
    double wn[3], ni;
} OraclePair;           /* 48 B */

typedef struct OracleParams {
    double radius;
    double mu_cloth_ground, mu_self, mu_pair, mu_fruit_ground, rolling, mu_fruit_yarn;
    double air[3], air_density;
    double aero[4];
    double capture_radius;
    double hysteresis;
    uint32_t ground, ring_count, patch_half, grid_width;
    uint32_t rim_count, bottom_center, pad[2];
} OracleParams;

typedef struct OracleSubstep {
    double dt;
    double gravity[3];
    double grip_target[3];
    double grip_q[4];   /* xyzw */
    uint32_t grip_active, grip_gen, grip_select, pad;
} OracleSubstep;

typedef struct OracleSchedule {
    uint32_t iterations, strain_sweeps, reconcile_passes, final_passes, certificate_passes, early_exit;
    uint32_t self_collision, aerodynamics, swept_ground, swept_fruit_yarn, frictions, release;
    double damping;
    uint32_t mode;      /* 0 batched, 1 serial */
    uint32_t primitive_self;   /* edge/edge yarn self-collision and self friction */
} OracleSchedule;

typedef struct OracleScene {
    const OracleParticle* particles; uint32_t n;
    const OracleDistance* distances; uint32_t d;
    const OracleKnot* knots; uint32_t k;
    const OracleBend* bends; uint32_t b;
    const OracleGrip* grips; uint32_t g;
    const OracleFruit* fruits; uint32_t f;
    const OraclePair* pairs; uint32_t p;
    const uint32_t* cuff;            /* 2 x ring_count */
    const uint32_t* rim;             /* rim_count */
    const uint32_t* local_off;       /* n+1, or NULL with params.grid_width */
    const uint32_t* local_idx;
    const OracleParams* params;
} OracleScene;

enum { ORACLE_BATCHED = 0, ORACLE_SERIAL = 1, ORACLE_BATCHED_SELF_REFERENCE = 2 };

/* bits: 32 or 64.  Returns NULL on a malformed scene. */
void* oracle_create(int bits, const OracleScene* scene);
void oracle_destroy(void* h);
/* Advance count substeps.  Returns the failure word (reference bits). */
uint32_t oracle_step(void* h, const OracleSubstep* subs, uint32_t count, const OracleSchedule* schedule);
/* State out (double); any pointer may be NULL. */
void oracle_read(void* h, OracleParticle* particles, OracleDistance* distances, OracleGrip* grips,
                 OracleFruit* fruits, OraclePair* pairs);
/* Overwrite particle and fruit state. */
void oracle_write(void* h, const OracleParticle* particles, const OracleFruit* fruits);
void oracle_write_grips(void* h, const OracleGrip* grips);
/* FP64 residuals of the current state: strain, ground, fruit/yarn, self. */
void oracle_residuals(void* h, double out[4]);
/* Release masks (mouth candidates, released) and counters:
 * out[0..1] masks, out[2] max reconcile passes, out[3] max certificate passes,
 * out[4] fruit/yarn contacts, out[5] self contacts, out[6] edge/edge
 * contacts, out[7] self-friction contacts. */
void oracle_stats(void* h, uint64_t out[8]);
/* One point self-contact pass on the current state (serial = the
 * reference's Gauss-Seidel order, else the batched order); returns the
 * largest penetration it resolved. */
double oracle_self_pass(void* h, int serial);
/* Restated probes with known answers; returns 1 on pass and fills values. */
int oracle_probe_strain(double out[4]);
int oracle_probe_cloth_ground_friction(double out[4]);
int oracle_probe_rolling(double out[4]);
int oracle_probe_aerodynamics(double out[8]);
int oracle_probe_self_ccd(double out[4]);
int oracle_probe_self_friction(double out[8]);

#ifdef __cplusplus
}
#endif

#endif
