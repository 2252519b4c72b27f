// Reference shim - TEST INFRASTRUCTURE, never part of the product.
//
// Compiles the reference CPU cloth (tools/cloth_bag.cpp of the reference
// tree) from where it lies, by including it into this translation unit, and
// exposes its scene and its substep functions through a C API.  It is the
// generator of the golden vectors under tests/golden/ and the pin of the
// CPU oracle: the oracle's serial order must reproduce the reference's
// results bit for bit on the reference's own scene.
//
// ref_run drives the reference's functions in the reference substep order
// (tools/cloth_bag.cpp:4759-5287).  With primitive = 1 it is the reference
// simulate() (checked by its state hash against simulate() itself); with
// primitive = 0 it omits the edge/edge primitive self-collision family
// (solvePrimitiveSelfCollision, applyClothSelfFriction and the primitive
// certificate residual), which the oracle and the B200 path do not restate
// yet.
#include <cstdint>
#include <cstring>

#define main numi_reference_cloth_bag_main
#include "tools/cloth_bag.cpp"
#undef main

#include "oracle.h"

namespace {

Scenario scenario_of(int s) {
    switch (s) {
        case 1: return Scenario::spin;
        case 2: return Scenario::pickup;
        case 3: return Scenario::recorded;
        default: return Scenario::grounded;
    }
}

void put3(double* dst, const Vec3& v) {
    dst[0] = v.x;
    dst[1] = v.y;
    dst[2] = v.z;
}

void export_particles(const ClothModel& c, OracleParticle* out) {
    for (size_t i = 0; i < c.particles.size(); ++i) {
        const Particle& p = c.particles[i];
        OracleParticle& o = out[i];
        std::memset(&o, 0, sizeof(o));
        put3(o.x, p.position);
        put3(o.prev, p.previous);
        put3(o.v, p.velocity);
        put3(o.rest, p.rest);
        o.w = p.inverseMass;
        o.mass = p.mass;
    }
}

void export_fruits(const std::array<Ball, kFruitCount>& balls, OracleFruit* out) {
    for (size_t k = 0; k < balls.size(); ++k) {
        const Ball& b = balls[k];
        OracleFruit& o = out[k];
        std::memset(&o, 0, sizeof(o));
        put3(o.x, b.position);
        put3(o.prev, b.previous);
        put3(o.v, b.velocity);
        put3(o.omega, b.angularVelocity);
        o.q[0] = b.orientation.x;
        o.q[1] = b.orientation.y;
        o.q[2] = b.orientation.z;
        o.q[3] = b.orientation.w;
        o.w = b.inverseMass;
        o.radius = b.radius;
        o.appearance = b.appearance;
    }
}

struct Loaded {
    numi::GripTrajectory trajectory;
    bool has = false;
};

bool load_trajectory(const char* path, Loaded& out) {
    if (path == nullptr || path[0] == 0) return true;
    try {
        out.trajectory = numi::loadGripTrajectory(path);
        out.has = true;
        return true;
    } catch (...) {
        return false;
    }
}

}  // namespace

extern "C" {

// Counts of the reference scene: particles, distances, knots, bends, grips,
// fruits, local-topology entries, bottom centre.
int ref_scene_counts(int scenario, uint32_t out[8]) {
    const ClothModel c = makeCloth(scenario_of(scenario));
    uint32_t local = 0;
    for (const auto& l : c.localTopology) local += static_cast<uint32_t>(l.size());
    out[0] = static_cast<uint32_t>(c.particles.size());
    out[1] = static_cast<uint32_t>(c.distances.size());
    out[2] = static_cast<uint32_t>(c.knots.size());
    out[3] = static_cast<uint32_t>(c.bends.size());
    out[4] = static_cast<uint32_t>(c.grips.size());
    out[5] = static_cast<uint32_t>(kFruitCount);
    out[6] = local;
    out[7] = c.bottomCenter;
    return 0;
}

// The reference's render triangles (3 indices each) into out when not
// NULL; returns their count.
uint32_t ref_render_triangles(int scenario, uint32_t* out) {
    const ClothModel c = makeCloth(scenario_of(scenario));
    if (out)
        for (size_t t = 0; t < c.renderTriangles.size(); ++t) {
            out[3 * t] = c.renderTriangles[t].first;
            out[3 * t + 1] = c.renderTriangles[t].second;
            out[3 * t + 2] = c.renderTriangles[t].third;
        }
    return static_cast<uint32_t>(c.renderTriangles.size());
}

// The reference scene in construction order (makeCloth / makeBalls).
int ref_scene_export(int scenario, OracleParticle* P, OracleDistance* D, OracleKnot* K, OracleBend* B,
                     OracleGrip* G, OracleFruit* F, OraclePair* PR, uint32_t* local_off, uint32_t* local_idx,
                     uint32_t* cuff, uint32_t* rim, OracleParams* prm) {
    const Scenario sc = scenario_of(scenario);
    const ClothModel c = makeCloth(sc);
    const auto balls = makeBalls(sc);
    export_particles(c, P);
    for (size_t k = 0; k < c.distances.size(); ++k) {
        const DistanceConstraint& d = c.distances[k];
        D[k] = OracleDistance{d.first, d.second, 0u, static_cast<uint32_t>(d.kind), d.restLength, d.compliance,
                              d.lambda, strainExtensionLimit(d.kind)};
    }
    for (size_t k = 0; k < c.knots.size(); ++k) {
        const KnotConstraint& q = c.knots[k];
        OracleKnot o{};
        o.p[0] = q.warpFirst;
        o.p[1] = q.warpSecond;
        o.p[2] = q.weftFirst;
        o.p[3] = q.weftSecond;
        o.restcos = q.restCosine;
        o.compliance = q.compliance;
        K[k] = o;
    }
    for (size_t k = 0; k < c.bends.size(); ++k) {
        const YarnBendConstraint& b = c.bends[k];
        OracleBend o{};
        o.p[0] = b.first;
        o.p[1] = b.middle;
        o.p[2] = b.third;
        o.restchord = b.restChord;
        o.restarc = b.restArc;
        o.compliance = b.compliance;
        B[k] = o;
    }
    for (size_t k = 0; k < c.grips.size(); ++k) {
        const GripConstraint& g = c.grips[k];
        OracleGrip o{};
        o.particle = g.particle;
        o.gen = c.gripAttachmentGeneration;
        put3(o.offset, g.targetOffset);
        o.compliance = g.compliance;
        G[k] = o;
    }
    export_fruits(balls, F);
    uint32_t pk = 0;
    for (uint32_t a = 0; a < kFruitCount; ++a)
        for (uint32_t b = a + 1u; b < kFruitCount; ++b) {
            OraclePair o{};
            o.a = a;
            o.b = b;
            o.stable = pk;
            PR[pk++] = o;
        }
    uint32_t off = 0;
    for (size_t i = 0; i < c.localTopology.size(); ++i) {
        local_off[i] = off;
        for (uint32_t j : c.localTopology[i]) local_idx[off++] = j;
    }
    local_off[c.localTopology.size()] = off;
    for (uint32_t level = kLevels - 2u; level < kLevels; ++level)
        for (uint32_t ring = 0; ring < kAround; ++ring) cuff[(level - (kLevels - 2u)) * kAround + ring] = nodeIndex(level, ring);
    for (uint32_t ring = 0; ring < kAround; ++ring) rim[ring] = nodeIndex(kLevels - 1u, ring);
    std::memset(prm, 0, sizeof(*prm));
    prm->radius = kClothRadius;
    prm->mu_cloth_ground = kClothGroundFriction;
    prm->mu_self = kClothSelfFriction;
    prm->mu_pair = kFruitPairFriction;
    prm->mu_fruit_ground = kFruitGroundFriction;
    prm->rolling = kFruitRollingResistanceCoefficient;
    prm->mu_fruit_yarn = kFruitClothFriction;
    prm->air_density = kAirDensity;
    prm->aero[0] = kYarnCrossflowDragCoefficient;
    prm->aero[1] = kYarnSkinFrictionCoefficient;
    prm->aero[2] = kFruitDragCoefficient;
    prm->aero[3] = kFruitRotationalDragCoefficient;
    prm->capture_radius = kGripCaptureRadius;
    prm->hysteresis = kMouthReleaseHysteresis;
    prm->ground = sc != Scenario::spin ? 1u : 0u;
    prm->ring_count = kAround;
    prm->patch_half = 2u;
    prm->rim_count = kAround;
    prm->bottom_center = c.bottomCenter;
    return 0;
}

// Load a numi.cloth.material.v1 artifact into the reference globals
// (applyClothMaterial, tools/cloth_bag.cpp:76-102).  Returns 0 or -1.
int ref_apply_material(const char* path) {
    try {
        applyClothMaterial(numi::loadClothMaterialArtifact(path));
        return 0;
    } catch (...) {
        return -1;
    }
}

void ref_reset_material(void) { applyClothMaterial(numi::ClothMaterialArtifact{}); }

// The reference's own simulate() and hashResult().
uint64_t ref_simulate_hash(int scenario, uint32_t steps, double frame_dt, uint32_t substeps, uint32_t iterations,
                           const char* trajectory) {
    Loaded t;
    if (!load_trajectory(trajectory, t)) return 0;
    try {
        const SimulationResult r =
            simulate(steps, frame_dt, substeps, iterations, scenario_of(scenario), nullptr, nullptr,
                     t.has ? &t.trajectory : nullptr);
        return hashResult(r);
    } catch (...) {
        return 0;
    }
}

// The reference substep loop driven through the reference's functions.
// subs (steps * substeps entries, may be NULL) receives the grip pose each
// substep used; the final state lands in P/F; out_u[0] = state hash,
// out_u[1] = released mask, out_u[2] = candidate mask.
int ref_run(int scenario, uint32_t steps, double frame_dt, uint32_t substeps, uint32_t iterations,
            const char* trajectory, uint32_t primitive, uint32_t point_self, OracleSubstep* subs,
            OracleParticle* P, OracleFruit* F, uint64_t* out_u) {
    Loaded t;
    if (!load_trajectory(trajectory, t)) return -1;
    const numi::GripTrajectory* traj = t.has ? &t.trajectory : nullptr;
    try {
        const Scenario sc = scenario_of(scenario);
        if ((sc == Scenario::recorded) != (traj != nullptr)) return -1;
        SimulationResult R;
        R.scenario = sc;
        R.cloth = makeCloth(sc);
        R.balls = makeBalls(sc);
        ClothModel& cloth = R.cloth;
        auto& balls = R.balls;
        Metrics& m = R.metrics;
        const double dt = frame_dt / static_cast<double>(substeps);
        const Vec3 g{0.0, 0.0, -9.81};
        const bool ground = sc != Scenario::spin;
        std::vector<Vec3> predicted(cloth.particles.size());
        std::vector<double> cloth_ground_impulse(cloth.particles.size());
        for (uint32_t step = 0; step < steps; ++step) {
            for (uint32_t sub = 0; sub < substeps; ++sub) {
                std::fill(cloth_ground_impulse.begin(), cloth_ground_impulse.end(), 0.0);
                std::array<BallPairContactImpulse, kBallPairCount> pairs{};
                std::vector<BallYarnContactImpulse> yarn(balls.size() * cloth.yarnSegments.size());
                std::array<double, kFruitCount> fruit_ground{};
                SelfContactImpulses self_impulses;
                if (sc != Scenario::grounded)
                    updateGrip(cloth, m, sc, static_cast<double>(step * substeps + sub + 1u) * dt, traj);
                if (subs != nullptr) {
                    OracleSubstep& o = subs[step * substeps + sub];
                    std::memset(&o, 0, sizeof(o));
                    o.dt = dt;
                    put3(o.gravity, g);
                    put3(o.grip_target, cloth.gripTarget);
                    o.grip_q[0] = cloth.gripOrientation.x;
                    o.grip_q[1] = cloth.gripOrientation.y;
                    o.grip_q[2] = cloth.gripOrientation.z;
                    o.grip_q[3] = cloth.gripOrientation.w;
                    o.grip_active = (sc != Scenario::grounded && cloth.gripActive) ? 1u : 0u;
                    o.grip_gen = cloth.gripAttachmentGeneration;
                    o.grip_select = (traj != nullptr && traj->selectNearestCuffPatch) ? 1u : 0u;
                }
                // predict
                for (Particle& p : cloth.particles) {
                    p.previous = p.position;
                    if (p.inverseMass == 0.0) {
                        p.position = p.rest;
                        p.velocity = (p.position - p.previous) / dt;
                        continue;
                    }
                    p.velocity += g * dt;
                }
                applyYarnAerodynamics(cloth, {}, dt, &m);
                for (size_t i = 0; i < cloth.particles.size(); ++i) {
                    Particle& p = cloth.particles[i];
                    predicted[i] = p.velocity;
                    if (p.inverseMass == 0.0) continue;
                    p.position += p.velocity * dt;
                }
                for (Ball& b : balls) {
                    b.previous = b.position;
                    b.velocity += g * dt;
                }
                applyFruitAerodynamics(balls, {}, dt, &m);
                for (Ball& b : balls) b.position += b.velocity * dt;
                if (sc != Scenario::spin) sweepGroundPrediction(cloth.particles, balls, dt, fruit_ground);
                for (auto& d : cloth.distances) d.lambda = 0.0;
                for (auto& b : cloth.bends) b.lambda = 0.0;
                for (auto& k : cloth.knots) k.lambda = 0.0;
                for (auto& gr : cloth.grips) gr.lambda = {};
                if (primitive) solvePrimitiveSelfCollision(cloth, true, m, dt, &self_impulses);
                for (size_t b = 0; b < balls.size(); ++b)
                    for (size_t s = 0; s < cloth.yarnSegments.size(); ++s)
                        solveSweptBallYarn(cloth.particles, cloth.yarnSegments[s], balls[b], dt, ground,
                                           yarn[b * cloth.yarnSegments.size() + s], m.sweptBallYarnContacts);
                const auto pair_sweep = [&] {
                    size_t k = 0;
                    for (size_t a = 0; a < balls.size(); ++a)
                        for (size_t b = a + 1u; b < balls.size(); ++b, ++k) solveBallPair(balls[a], balls[b], dt, pairs[k]);
                };
                const auto ground_pass = [&] {
                    if (ground)
                        solveGround(cloth.particles, balls, dt, fruit_ground, m.maximumClothGroundCorrection,
                                    m.maximumBallGroundCorrection);
                };
                for (uint32_t it = 0; it < iterations; ++it) {
                    for (auto& d : cloth.distances) solveDistance(cloth.particles, d, dt);
                    for (auto& k : cloth.knots) solveKnot(cloth.particles, k, dt);
                    if (it % 2u == 0u)
                        for (auto& b : cloth.bends) solveBend(cloth.particles, b, dt, ground);
                    if (cloth.gripActive)
                        for (auto& gr : cloth.grips)
                            solveGrip(cloth.particles, gr,
                                      cloth.gripTarget + rotateVector(cloth.gripOrientation, gr.targetOffset), dt);
                    pair_sweep();
                    solveBallYarnContactSweep(cloth, balls, dt, ground, yarn, m);
                    if (point_self) solveSelfCollision(cloth, m.selfContacts);
                    ground_pass();
                }
                const auto strain3 = [&] {
                    for (int s = 0; s < 3; ++s) solveStrainLimits(cloth.particles, cloth.distances);
                };
                for (uint32_t pass = 0; pass < 8u; ++pass) {
                    pair_sweep();
                    solveBallYarnContactSweep(cloth, balls, dt, ground, yarn, m);
                    strain3();
                    ground_pass();
                    const double br = measureBallYarnPenetration(cloth, balls);
                    const double gr = ground ? measureGroundPenetration(cloth.particles, balls) : 0.0;
                    if (br < 1.0e-6 && gr < 1.0e-9 && measureStrainLimitViolation(cloth) < 1.0e-6) break;
                }
                const auto endpoint = [&] {
                    if (primitive) solvePrimitiveSelfCollision(cloth, false, m, dt, &self_impulses);
                    strain3();
                };
                const auto finals = [&] {
                    for (int pass = 0; pass < 2; ++pass) {
                        pair_sweep();
                        solveBallYarnContactSweep(cloth, balls, dt, ground, yarn, m);
                        ground_pass();
                    }
                };
                endpoint();
                finals();
                if (sub + 1u == substeps) {
                    for (uint32_t pass = 0; pass < 128u; ++pass) {
                        endpoint();
                        finals();
                        const double pr = primitive ? measurePrimitiveSelfPenetration(cloth) : 0.0;
                        const double br = measureBallYarnPenetration(cloth, balls);
                        const double gr = ground ? measureGroundPenetration(cloth.particles, balls) : 0.0;
                        if (pr < 1.0e-6 && br < 1.0e-6 && gr < 1.0e-9 && measureStrainLimitViolation(cloth) < 1.0e-6)
                            break;
                    }
                }
                for (size_t i = 0; i < cloth.particles.size(); ++i) {
                    Particle& p = cloth.particles[i];
                    if (p.inverseMass == 0.0) {
                        p.position = p.rest;
                        p.velocity = (p.position - p.previous) / dt;
                    } else {
                        p.velocity = (p.position - p.previous) / dt;
                        if (ground && p.position.z <= kClothRadius + 1.0e-6)
                            cloth_ground_impulse[i] = std::max(0.0, (p.velocity.z - predicted[i].z) / p.inverseMass);
                    }
                }
                for (Ball& b : balls) b.velocity = (b.position - b.previous) / dt;
                applyClothGroundFriction(cloth.particles, cloth_ground_impulse, m);
                if (primitive) applyClothSelfFriction(cloth, self_impulses, m);
                applyBallYarnFriction(cloth, balls, yarn, m, ground);
                applyBallPairFriction(balls, pairs, m);
                applyBallGroundFriction(balls, fruit_ground, dt, m, kFruitRollingResistanceCoefficient);
                if (sc != Scenario::grounded) updateReleasedFruit(cloth, balls, m);
                for (Ball& b : balls) integrateOrientation(b, dt);
            }
        }
        if (P) export_particles(cloth, P);
        if (F) export_fruits(balls, F);
        if (out_u) {
            out_u[0] = hashResult(R);
            out_u[1] = m.releasedMask;
            out_u[2] = m.mouthCandidateMask;
        }
        return 0;
    } catch (...) {
        return -2;
    }
}

}  // extern "C"
