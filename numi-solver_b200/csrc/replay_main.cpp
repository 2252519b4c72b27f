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
    o.scenario = NUMI_CLOTH_SCENARIO_GROUNDED;
    o.steps = 180;
    o.substeps = 48;
    o.replays = 1;
    o.frameTimestep = 1.0 / 60.0;
    uint32_t iterations = 1;
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
        std::fprintf(stderr, "error: %s\n", e.what());
        return 2;
    }
    if (iterations == 0u) {
        std::fprintf(stderr, "error: simulation controls must be positive\n");
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
    NumiClothReplayResult r{};
    const int rc = numi_cloth_replay(&o, &r, err, sizeof(err));
    if (rc != NUMI_CLOTH_OK) {
        std::fprintf(stderr, "error: %s\n", err[0] ? err : "replay failed");
        return 1;
    }
    const char* names[] = {"grounded", "spin", "pickup", "recorded"};
    std::printf("model=explicit_yarn_cloth_b200 scenario=%s nodes=%u render_triangles=%u fruits=%u steps=%u "
                "substeps=%u iterations=%u\n",
                names[o.scenario], r.particles, r.renderTriangles, r.fruits, o.steps, o.substeps, iterations);
    std::printf("hash=0x%016llx replay_hash=0x%016llx deterministic=%s failure=%u seconds=%.6f\n",
                static_cast<unsigned long long>(r.hash), static_cast<unsigned long long>(r.replayHash),
                r.deterministic ? "true" : "false", r.failure, r.seconds);
    std::printf("strain_violation=%.9e ground_penetration=%.9e fruit_yarn_penetration=%.9e self_penetration=%.9e "
                "self_contacts=%llu edge_edge_contacts=%llu self_friction_contacts=%llu released_mask=%u "
                "mouth_candidate_mask=%u attachment_generation=%u max_contact_reconciliation_passes=%u "
                "max_primitive_certificate_passes=%u\n",
                r.residuals[0], r.residuals[1], r.residuals[2], r.residuals[3], r.selfContacts, r.edgeContacts[0],
                r.edgeContacts[1], r.masks[0], r.masks[1], r.generation, r.reconcileMax, r.certificateMax);
    return r.failure == 0u ? 0 : 1;
}
