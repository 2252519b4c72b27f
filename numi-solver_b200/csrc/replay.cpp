// Replay harness of the produce-bag scenarios on the GPU path: the
// reference CLI's run (tools/cloth_bag.cpp:5504-5760, simulate :4712) driven
// through the library's own C API.  Scenarios grounded / spin / pickup /
// recorded, frame after frame on one handle (continuation), OBJ frames in
// the reference's format (dumpOBJ, :5362-5400), the reference's state hash
// (hashResult, :5312-5360) and an optional second run that must give the
// same hash.
#include <algorithm>
#include <bit>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <string>
#include <vector>

#include "numi_cloth.h"
#include "numi_cloth_replay.h"
#include "numi_cloth_scene.h"

namespace {

struct Fnv {
    uint64_t h = 1469598103934665603ull;
    void add(double v) {
        const uint64_t bits = std::bit_cast<uint64_t>(v);
        for (int b = 0; b < 8; ++b) {
            h ^= static_cast<uint8_t>(bits >> (8 * b));
            h *= 1099511628211ull;
        }
    }
};

void set_err(char* err, size_t n, const std::string& m) {
    if (err && n) {
        std::strncpy(err, m.c_str(), n - 1);
        err[n - 1] = '\0';
    }
}

}  // namespace

extern "C" uint64_t numi_cloth_state_hash(const NumiClothHashState* s) {
    if (s == nullptr) return 0;
    Fnv f;
    for (uint32_t i = 0; i < s->particles; ++i)
        for (int k = 0; k < 6; ++k) f.add(s->particleState[6u * i + k]);
    for (uint32_t b = 0; b < s->fruits; ++b)
        for (int k = 0; k < 13; ++k) f.add(s->fruitState[13u * b + k]);
    for (int k = 0; k < 3; ++k) f.add(s->gripTarget[k]);
    f.add(s->gripActive ? 1.0 : 0.0);
    if (s->generation > 1u) {
        f.add(static_cast<double>(s->generation));
        for (uint32_t g = 0; g < s->grips; ++g) {
            if (s->patchSelections > 0u) f.add(static_cast<double>(s->gripParticle[g]));
            for (int k = 0; k < 3; ++k) f.add(s->gripOffset[3u * g + k]);
        }
    }
    return f.h;
}

extern "C" int numi_cloth_write_obj(const char* path, const NumiClothObjState* s) {
    if (path == nullptr || s == nullptr) return NUMI_CLOTH_EINVAL;
    std::ofstream out(path);
    if (!out) return NUMI_CLOTH_EINVAL;
    out << std::setprecision(9);
    out << "# Numi Solver explicit-yarn cloth bag reference\n";
    out << "# vertices " << s->particles << " render_triangles " << s->triangles << '\n';
    for (uint32_t i = 0; i < s->particles; ++i)
        out << "v " << s->positions[3u * i] << ' ' << s->positions[3u * i + 1u] << ' ' << s->positions[3u * i + 2u]
            << '\n';
    for (uint32_t t = 0; t < s->triangles; ++t)
        out << "f " << s->triangleIndices[3u * t] + 1u << ' ' << s->triangleIndices[3u * t + 1u] + 1u << ' '
            << s->triangleIndices[3u * t + 2u] + 1u << '\n';
    if (s->scenario != NUMI_CLOTH_SCENARIO_GROUNDED)
        out << "# grip center " << s->gripTarget[0] << ' ' << s->gripTarget[1] << ' ' << s->gripTarget[2]
            << " active " << (s->gripActive ? 1 : 0) << " orientation " << s->gripOrientationWxyz[0] << ' '
            << s->gripOrientationWxyz[1] << ' ' << s->gripOrientationWxyz[2] << ' ' << s->gripOrientationWxyz[3]
            << " patch_center " << s->patchCenter << '\n';
    for (uint32_t b = 0; b < s->fruits; ++b) {
        const double* q = s->fruitState + 11u * b;
        out << "# ball " << b << " center " << q[0] << ' ' << q[1] << ' ' << q[2] << " radius " << q[3]
            << " appearance " << s->fruitAppearance[b] << " orientation " << q[4] << ' ' << q[5] << ' ' << q[6]
            << ' ' << q[7] << " angular_velocity " << q[8] << ' ' << q[9] << ' ' << q[10] << '\n';
    }
    return out ? NUMI_CLOTH_OK : NUMI_CLOTH_EINVAL;
}

namespace {

// One run of a scenario; fills the hash and the result fields it owns.
struct Run {
    const NumiClothReplayOptions& o;
    const NumiClothMaterial& material;
    numi_cloth_trajectory_t* traj;
    bool select_nearest;
    std::vector<uint32_t> capture;   // completed steps to write as OBJ frames
    char* err;
    size_t err_size;

    int go(bool write, NumiClothReplayResult* r, uint64_t* hash) {
        const double dt = o.frameTimestep / static_cast<double>(o.substeps);
        numi_cloth_scene_t* scene = numi_cloth_scene_bag(&material, o.scenario, dt, select_nearest ? 1 : 0);
        if (scene == nullptr) {
            set_err(err, err_size, "scene build failed");
            return NUMI_CLOTH_EINVAL;
        }
        NumiClothScene view;
        numi_cloth_scene_view(scene, &view);
        uint32_t counts[15];
        numi_cloth_scene_counts(scene, counts);
        const uint32_t n = counts[0], g = counts[4], f = counts[5];
        std::vector<uint32_t> tris(3u * numi_cloth_scene_triangles(scene, nullptr, 0));
        numi_cloth_scene_triangles(scene, tris.data(), static_cast<uint32_t>(tris.size() / 3u));
        double handle[3];
        numi_cloth_bag_handle_base(o.scenario, handle);
        numi_cloth_t* h = nullptr;
        int rc = numi_cloth_create(&view, &h);
        if (rc != NUMI_CLOTH_OK) {
            numi_cloth_scene_destroy(scene);
            set_err(err, err_size, "numi_cloth_create failed");
            return rc;
        }
        // host view of the grip (the reference's ClothModel fields)
        double grip[3] = {0.0, 0.0, 0.0};
        bool grip_active = false;
        double grip_q[4] = {1.0, 0.0, 0.0, 0.0};   // wxyz
        uint32_t generation = 1u, selections = 0u, patch_center = 0u;
        // the reference's grip metrics (tools/cloth_bag.cpp:1563-1620)
        uint32_t regrabs = 0u, ring_shift = 0u;
        uint64_t inactive = 0u;
        if (o.scenario != NUMI_CLOTH_SCENARIO_GROUNDED) {
            std::copy(handle, handle + 3, grip);
            grip_active = true;
        }
        std::vector<NumiClothParticle> P(n);
        std::vector<NumiClothFruit> F(f);
        std::vector<NumiClothGrip> G(g);
        auto read = [&]() {
            numi_cloth_read_particles(h, P.data(), n);
            if (f) numi_cloth_read_fruits(h, F.data(), f);
            if (g) numi_cloth_read_grips(h, G.data(), g);
        };
        auto write_frame = [&](const std::string& path) {
            read();
            std::vector<double> xyz(3u * n), fr(11u * f);
            std::vector<uint32_t> app(f);
            for (uint32_t i = 0; i < n; ++i) {
                xyz[3u * i] = P[i].positionAndInverseMass.x;
                xyz[3u * i + 1u] = P[i].positionAndInverseMass.y;
                xyz[3u * i + 2u] = P[i].positionAndInverseMass.z;
            }
            for (uint32_t b = 0; b < f; ++b) {
                const NumiClothFruit& q = F[b];
                const double v[11] = {q.positionAndInverseMass.x, q.positionAndInverseMass.y, q.positionAndInverseMass.z,
                                      q.previousAndRadius.w,      q.orientation.w,           q.orientation.x,
                                      q.orientation.y,            q.orientation.z,           q.angularVelocity.x,
                                      q.angularVelocity.y,        q.angularVelocity.z};
                std::copy(v, v + 11, fr.begin() + 11u * b);
                app[b] = q.identity.x;
            }
            NumiClothObjState st{};
            st.particles = n;
            st.positions = xyz.data();
            st.triangles = static_cast<uint32_t>(tris.size() / 3u);
            st.triangleIndices = tris.data();
            st.scenario = o.scenario;
            std::copy(grip, grip + 3, st.gripTarget);
            st.gripActive = grip_active ? 1u : 0u;
            std::copy(grip_q, grip_q + 4, st.gripOrientationWxyz);
            st.patchCenter = patch_center;
            st.fruits = f;
            st.fruitState = fr.data();
            st.fruitAppearance = app.data();
            numi_cloth_write_obj(path.c_str(), &st);
        };
        auto dump = [&](uint32_t completed) {
            if (!write || std::find(capture.begin(), capture.end(), completed) == capture.end()) return;
            write_frame(std::string(o.dumpFrames) + "-" + std::to_string(completed) + ".obj");
        };
        dump(0u);
        std::vector<NumiClothConfig> cfg(o.substeps);
        std::vector<double> targets(3u * o.substeps);
        const auto t0 = std::chrono::steady_clock::now();
        uint32_t failure = 0;
        for (uint32_t step = 0; step < o.steps && failure == 0u; ++step) {
            const uint64_t first = static_cast<uint64_t>(step) * o.substeps;
            // substeps of this frame that attach a new grip generation: the
            // frame is stepped in launches that end after each of them, so
            // the selected patch centre of every re-grab can be read
            std::vector<uint32_t> cuts;
            if (o.scenario == NUMI_CLOTH_SCENARIO_RECORDED) {
                rc = numi_cloth_trajectory_configs(traj, view.config, handle, first, o.substeps, dt, cfg.data());
                // the grip state updateGrip keeps, substep by substep
                // (tools/cloth_bag.cpp:1504-1620)
                for (uint32_t k = 0; k < o.substeps; ++k) {
                    NumiClothGripPose pose;
                    numi_cloth_trajectory_sample(traj, static_cast<double>(first + k + 1u) * dt, &pose);
                    for (int e = 0; e < 3; ++e) grip[e] = handle[e] + pose.translation[e];
                    grip_active = pose.active != 0u;
                    grip_q[0] = pose.orientation[3];
                    grip_q[1] = pose.orientation[0];
                    grip_q[2] = pose.orientation[1];
                    grip_q[3] = pose.orientation[2];
                    if (pose.active && pose.generation != generation) {
                        if (select_nearest) {
                            ++selections;
                            cuts.push_back(k + 1u);
                        }
                        ++regrabs;
                        generation = pose.generation;
                    }
                    if (!pose.active) ++inactive;
                }
            } else {
                rc = numi_cloth_bag_scenario_configs(o.scenario, view.config, first, o.substeps, dt, cfg.data(),
                                                     targets.data());
                if (o.scenario != NUMI_CLOTH_SCENARIO_GROUNDED)
                    std::copy(targets.end() - 3, targets.end(), grip);
            }
            // the attach substeps end launches of their own (at most one
            // attach per launch), then the frame's remainder
            const size_t attaches = cuts.size();
            if (cuts.empty() || cuts.back() != o.substeps) cuts.push_back(o.substeps);
            uint32_t done = 0;
            for (size_t c = 0; c < cuts.size() && rc == NUMI_CLOTH_OK && failure == 0u; ++c) {
                const uint32_t end = cuts[c];
                rc = numi_cloth_step(h, cfg.data() + done, end - done, &o.schedule);
                if (rc != NUMI_CLOTH_OK) break;
                failure = numi_cloth_failure(h);
                if (c < attaches && g > 0u && failure == 0u) {
                    // the nearest-patch centre this re-grab selected
                    // (cyclicRingDistance, tools/cloth_bag.cpp:462-468)
                    numi_cloth_read_grips(h, G.data(), g);
                    const uint32_t centre = G[0].particle.w;
                    const uint32_t direct = centre > patch_center ? centre - patch_center : patch_center - centre;
                    const uint32_t around = view.config->gripControl.z;
                    ring_shift = std::max(ring_shift, std::min(direct, around - direct));
                    patch_center = centre;
                }
                done = end;
            }
            if (rc != NUMI_CLOTH_OK) break;
            dump(step + 1u);
        }
        const double seconds =
            std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (write && o.dumpObj != nullptr) write_frame(o.dumpObj);
        read();

        std::vector<double> xv(6u * n), fs(13u * f), off(3u * g);
        std::vector<uint32_t> gp(g);
        for (uint32_t i = 0; i < n; ++i) {
            const double v[6] = {P[i].positionAndInverseMass.x, P[i].positionAndInverseMass.y,
                                 P[i].positionAndInverseMass.z, P[i].velocity.x,
                                 P[i].velocity.y,              P[i].velocity.z};
            std::copy(v, v + 6, xv.begin() + 6u * i);
        }
        for (uint32_t b = 0; b < f; ++b) {
            const NumiClothFruit& q = F[b];
            const double v[13] = {q.positionAndInverseMass.x, q.positionAndInverseMass.y, q.positionAndInverseMass.z,
                                  q.velocityAndGroundImpulse.x, q.velocityAndGroundImpulse.y,
                                  q.velocityAndGroundImpulse.z, q.angularVelocity.x, q.angularVelocity.y,
                                  q.angularVelocity.z, q.orientation.w, q.orientation.x, q.orientation.y,
                                  q.orientation.z};
            std::copy(v, v + 13, fs.begin() + 13u * b);
        }
        for (uint32_t k = 0; k < g; ++k) {
            gp[k] = G[k].particle.x;
            off[3u * k] = G[k].targetOffsetAndCompliance.x;
            off[3u * k + 1u] = G[k].targetOffsetAndCompliance.y;
            off[3u * k + 2u] = G[k].targetOffsetAndCompliance.z;
        }
        NumiClothHashState hs{};
        hs.particles = n;
        hs.fruits = f;
        hs.grips = g;
        hs.particleState = xv.data();
        hs.fruitState = fs.data();
        std::copy(grip, grip + 3, hs.gripTarget);
        hs.gripActive = grip_active ? 1u : 0u;
        hs.generation = generation;
        hs.patchSelections = selections;
        hs.gripParticle = gp.data();
        hs.gripOffset = off.data();
        *hash = numi_cloth_state_hash(&hs);
        if (r != nullptr) {
            r->failure = failure;
            r->seconds = seconds;
            r->particles = n;
            r->fruits = f;
            r->renderTriangles = static_cast<uint32_t>(tris.size() / 3u);
            numi_cloth_residuals(h, r->residuals);
            double pen = 0.0;
            numi_cloth_self_contacts(h, &r->selfContacts, &pen);
            numi_cloth_edge_contacts(h, r->edgeContacts);
            numi_cloth_release_masks(h, r->masks);
            uint32_t passes[3] = {0, 0, 0};
            numi_cloth_pass_counts(h, passes);
            r->reconcileMax = passes[1];
            r->certificateMax = passes[2];
            r->generation = generation;
            r->regrabCount = regrabs;
            r->inactiveGripSubsteps = inactive;
            r->patchSelections = selections;
            r->maxPatchRingShift = ring_shift;
            r->patchCenter = patch_center;
            // gripParticlesUnique and gripPatchTopologyExact
            // (tools/cloth_bag.cpp:5409-5437) on the final grips
            bool unique = true;
            for (uint32_t a = 0; a < g; ++a)
                for (uint32_t b = a + 1u; b < g; ++b) unique = unique && G[a].particle.x != G[b].particle.x;
            const uint32_t rings = view.config->gripControl.z;
            bool exact = g == 10u && view.cuffParticles != nullptr && rings >= 5u;
            for (uint32_t row = 0; exact && row < 2u; ++row)
                for (uint32_t slot = 0; slot < 5u; ++slot) {
                    const uint32_t ring = (patch_center + rings + slot - 2u) % rings;
                    exact = exact && G[row * 5u + slot].particle.x == view.cuffParticles[row * rings + ring];
                }
            r->patchParticlesUnique = unique ? 1u : 0u;
            r->patchTopologyExact = exact ? 1u : 0u;
        }
        numi_cloth_destroy(h);
        numi_cloth_scene_destroy(scene);
        return rc;
    }
};

}  // namespace

extern "C" int numi_cloth_replay(const NumiClothReplayOptions* o, NumiClothReplayResult* r, char* err,
                                 size_t err_size) {
    if (o == nullptr || r == nullptr) return NUMI_CLOTH_EINVAL;
    *r = NumiClothReplayResult{};
    if (o->steps == 0u || o->substeps == 0u || (o->replays != 1u && o->replays != 2u) ||
        !std::isfinite(o->frameTimestep) || o->frameTimestep <= 0.0 || o->scenario < NUMI_CLOTH_SCENARIO_GROUNDED ||
        o->scenario > NUMI_CLOTH_SCENARIO_RECORDED) {
        set_err(err, err_size, "simulation controls must be positive");
        return NUMI_CLOTH_EINVAL;
    }
    if (o->dumpEvery != 0u && o->dumpFrames == nullptr) {
        set_err(err, err_size, "--dump-every requires --dump-frames");
        return NUMI_CLOTH_EINVAL;
    }
    if ((o->scenario == NUMI_CLOTH_SCENARIO_RECORDED) != (o->gripTrajectory != nullptr)) {
        set_err(err, err_size, "recorded scenario requires exactly one grip trajectory");
        return NUMI_CLOTH_EINVAL;
    }
    NumiClothMaterial material;
    numi_cloth_material_defaults(&material);
    if (o->material != nullptr && numi_cloth_material_load(o->material, &material, err, err_size) != 0)
        return NUMI_CLOTH_EINVAL;
    numi_cloth_trajectory_t* traj = nullptr;
    bool select_nearest = false;
    if (o->gripTrajectory != nullptr) {
        traj = numi_cloth_trajectory_load(o->gripTrajectory, err, err_size);
        if (traj == nullptr) return NUMI_CLOTH_EINVAL;
        uint32_t sel = 0;
        double duration = 0.0;
        uint64_t fp = 0;
        numi_cloth_trajectory_info(traj, &sel, &duration, &fp);
        select_nearest = sel != 0u;
        if (duration + 1.0e-12 < static_cast<double>(o->steps) * o->frameTimestep) {
            numi_cloth_trajectory_destroy(traj);
            set_err(err, err_size, "grip trajectory does not cover the requested simulation");
            return NUMI_CLOTH_EINVAL;
        }
    }
    Run run{*o, material, traj, select_nearest, {}, err, err_size};
    // frames to write (tools/cloth_bag.cpp:5611-5633): the quarters, or every N
    if (o->dumpFrames != nullptr) {
        if (o->dumpEvery == 0u) {
            for (uint32_t quarter = 0; quarter <= 4u; ++quarter) {
                const uint32_t completed = (o->steps * quarter + 2u) / 4u;
                if (run.capture.empty() || run.capture.back() != completed) run.capture.push_back(completed);
            }
        } else {
            for (uint32_t completed = 0; completed < o->steps; completed += o->dumpEvery)
                run.capture.push_back(completed);
            run.capture.push_back(o->steps);
        }
    }
    int rc = run.go(true, r, &r->hash);
    if (rc == NUMI_CLOTH_OK && o->replays == 2u) {
        rc = run.go(false, nullptr, &r->replayHash);
        r->deterministic = r->hash == r->replayHash ? 1u : 0u;
    }
    if (traj != nullptr) numi_cloth_trajectory_destroy(traj);
    return rc;
}
