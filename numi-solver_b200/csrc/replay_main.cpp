// numi-cloth-replay: the reference cloth CLI's simulation run
// (tools/cloth_bag.cpp:5504-5760) on the B200 path.  Same options as the
// reference for the run itself (--steps --substeps --iterations --replays
// --timestep --scenario --material --grip-trajectory --dump-obj
// --dump-frames --dump-every); the schedule is the reference's substep
// (iterations, 3 strain sweeps, reconciliation up to 8 with early exit, 2
// final passes, certificate up to 128) with every contact family on.
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>

#include "numi_cloth_replay.h"
#include "numi_cloth_scene.h"

int main(int argc, char** argv) {
    NumiClothReplayOptions o{};
    // the reference CLI's defaults (tools/cloth_bag.cpp:5502-5522)
    o.scenario = NUMI_CLOTH_SCENARIO_GROUNDED;
    o.steps = 120;
    o.substeps = 24;
    o.replays = 2;
    o.frameTimestep = 1.0 / 120.0;
    uint32_t iterations = 32;
    try {
        for (int a = 1; a < argc; ++a) {
            const std::string v = argv[a];
            auto next = [&]() -> const char* {
                if (a + 1 >= argc) throw std::invalid_argument("missing value for " + v);
                return argv[++a];
            };
            if (v == "--steps") o.steps = static_cast<uint32_t>(std::stoul(next()));
            else if (v == "--substeps") o.substeps = static_cast<uint32_t>(std::stoul(next()));
            else if (v == "--iterations") iterations = static_cast<uint32_t>(std::stoul(next()));
            else if (v == "--replays") o.replays = static_cast<uint32_t>(std::stoul(next()));
            else if (v == "--timestep") o.frameTimestep = std::stod(next());
            else if (v == "--material") o.material = next();
            else if (v == "--grip-trajectory") o.gripTrajectory = next();
            else if (v == "--dump-obj") o.dumpObj = next();
            else if (v == "--dump-frames") o.dumpFrames = next();
            else if (v == "--dump-every") o.dumpEvery = static_cast<uint32_t>(std::stoul(next()));
            else if (v == "--scenario") {
                const std::string s = next();
                if (s == "grounded") o.scenario = NUMI_CLOTH_SCENARIO_GROUNDED;
                else if (s == "spin") o.scenario = NUMI_CLOTH_SCENARIO_SPIN;
                else if (s == "pickup") o.scenario = NUMI_CLOTH_SCENARIO_PICKUP;
                else if (s == "recorded") o.scenario = NUMI_CLOTH_SCENARIO_RECORDED;
                else throw std::invalid_argument("unknown scenario: " + s);
            } else if (v == "--help") {
                std::printf("usage: numi-cloth-replay [--steps N] [--substeps N] [--iterations N] [--replays 1|2] "
                            "[--timestep DT] [--scenario grounded|spin|pickup|recorded] [--material FILE] "
                            "[--grip-trajectory FILE] [--dump-obj PATH] [--dump-frames PREFIX] [--dump-every N]\n");
                return 0;
            } else {
                throw std::invalid_argument("unknown option: " + v);
            }
        }
    } catch (const std::exception& e) {
        std::fprintf(stderr, "numi-cloth-replay: %s\n", e.what());
        return 2;
    }
    if (iterations == 0u) {
        std::fprintf(stderr, "numi-cloth-replay: simulation controls must be positive\n");
        return 2;
    }
    NumiClothSchedule& s = o.schedule;
    s.iterations = iterations;
    s.strainSweeps = 3;
    s.reconcilePasses = 8;
    s.finalPasses = 2;
    s.certificatePasses = 128;
    s.earlyExit = 1;
    s.selfCollision = 1;
    s.aerodynamics = 1;
    s.sweptGround = 1;
    s.sweptFruitYarn = 1;
    s.frictions = 1;
    s.release = o.scenario == NUMI_CLOTH_SCENARIO_GROUNDED ? 0u : 1u;
    s.primitiveSelf = 1;
    char err[512] = {0};
    // the trajectory summary the reference prints before the run
    // (tools/cloth_bag.cpp:5734-5751)
    uint32_t schema = 0, poses = 0, generations = 0, select_nearest = 0;
    double max_rotation = 0.0, duration = 0.0;
    uint64_t fingerprint = 0;
    if (o.gripTrajectory != nullptr) {
        numi_cloth_trajectory_t* t = numi_cloth_trajectory_load(o.gripTrajectory, err, sizeof(err));
        if (t == nullptr) {
            std::fprintf(stderr, "numi-cloth-replay: %s\n", err[0] ? err : "grip trajectory rejected");
            return 2;
        }
        numi_cloth_trajectory_summary(t, &schema, &poses, &max_rotation, &generations);
        numi_cloth_trajectory_info(t, &select_nearest, &duration, &fingerprint);
        numi_cloth_trajectory_destroy(t);
    }
    NumiClothReplayResult r{};
    const int rc = numi_cloth_replay(&o, &r, err, sizeof(err));
    if (rc != NUMI_CLOTH_OK) {
        std::fprintf(stderr, "numi-cloth-replay: %s\n", err[0] ? err : "replay failed");
        return 2;
    }
    // failures the reference raises as exceptions (exit code 2, message on
    // stderr): a re-grab beyond the capture radius (cloth_bag.cpp:1584-1588)
    if (r.failure & NUMI_CLOTH_FAILURE_GRIP_CAPTURE) {
        std::fprintf(stderr, "numi-cloth-replay: grip reattachment exceeds capture radius\n");
        return 2;
    }
    const char* names[] = {"grounded", "spin", "pickup", "recorded"};
    std::printf("material_schema=numi.cloth.material.v1 material_artifact_loaded=%s\n",
                o.material != nullptr ? "true" : "false");
    if (o.gripTrajectory != nullptr)
        std::printf("grip_trajectory_schema=numi.grip.trajectory.v%u content_fingerprint=0x%llx poses=%u "
                    "duration_seconds=%.9f maximum_rotation_radians=%.9f attachment_generations=%u "
                    "selection_mode=%s\n",
                    schema, static_cast<unsigned long long>(fingerprint), poses, duration, max_rotation,
                    generations, select_nearest ? "nearest_cuff_patch" : "fixed_patch");
    std::printf("model=explicit_yarn_cloth_b200 scenario=%s nodes=%u render_triangles=%u balls=%u steps=%u "
                "substeps=%u iterations=%u replays=%u simulated_seconds=%.9f\n",
                names[o.scenario], r.particles, r.renderTriangles, r.fruits, o.steps, o.substeps, iterations,
                o.replays, o.steps * o.frameTimestep);
    const bool deterministic = o.replays == 2u && r.deterministic != 0u;
    std::printf("final_strain_limit_violation=%.9f max_published_ground_penetration=%.9f "
                "max_published_ball_penetration=%.9f max_self_penetration=%.9f self_contacts=%llu "
                "edge_edge_self_contacts=%llu cloth_self_friction_contacts=%llu released_mask=%u "
                "mouth_candidate_mask=%u max_contact_reconciliation_passes=%u max_primitive_certificate_passes=%u "
                "regrab_count=%u inactive_grip_substeps=%llu patch_selection_count=%u maximum_patch_ring_shift=%u "
                "selected_patch_center_ring=%u patch_particles_unique=%s patch_topology_exact=%s "
                "attachment_generation=%u failure=%u deterministic=%s state_hash=0x%llx replay_hash=0x%llx\n",
                r.residuals[0], r.residuals[1], r.residuals[2], r.residuals[3], r.selfContacts, r.edgeContacts[0],
                r.edgeContacts[1], r.masks[1], r.masks[0], r.reconcileMax, r.certificateMax, r.regrabCount,
                static_cast<unsigned long long>(r.inactiveGripSubsteps), r.patchSelections, r.maxPatchRingShift,
                r.patchCenter, r.patchParticlesUnique ? "true" : "false", r.patchTopologyExact ? "true" : "false",
                r.generation, r.failure, deterministic ? "true" : "false", static_cast<unsigned long long>(r.hash),
                static_cast<unsigned long long>(r.replayHash));
    std::printf("seconds=%.6f\n", r.seconds);
    // the reference's acceptance (acceptable, cloth_bag.cpp:5441-5497) on
    // what this harness measures: no failure bit (finite state, captures
    // within radius), a deterministic replay, the end-state residual gates,
    // the pickup outcome and the spatial patch checks
    const bool patch_ok = r.patchSelections == 0u ||
                          (r.patchSelections == r.regrabCount && r.patchParticlesUnique && r.patchTopologyExact);
    const bool pickup_ok = o.scenario != NUMI_CLOTH_SCENARIO_PICKUP || __builtin_popcount(r.masks[1]) >= 2;
    const bool pass = r.failure == 0u && deterministic && patch_ok && pickup_ok && r.residuals[0] < 2.0e-6 &&
                      r.residuals[1] < 2.0e-6 && r.residuals[2] < 2.0e-6;
    std::printf("result=%s\n", pass ? "PASS" : "FAIL");
    return pass ? 0 : 1;
}
