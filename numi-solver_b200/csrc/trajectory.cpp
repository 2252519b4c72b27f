// numi.grip.trajectory.v1..v3 (include/numi/grip_trajectory.h:189-362):
// a schema line, the fixed 9-column header, then rows of time, translation,
// quaternion xyzw and the active flag.  Times strictly increase; quaternions
// are unit within 1e-3 (normalised, sign-continuous); v1 forbids
// re-activation, v2/v3 bump the attachment generation on every 0 -> 1, v3
// also re-selects the nearest cuff patch; the first pose is t=0, identity,
// active.  Sampling lerps translation and slerps orientation (normalised
// lerp above cos 0.9995); the active flag and generation are the left
// neighbour's.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <fstream>
#include <limits>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "numi_cloth_scene.h"

namespace {

struct Pose {
    double t;
    double tr[3];
    double q[4];   // xyzw
    bool active;
    uint32_t generation;
};

std::string trim(std::string v) {
    const auto sp = [](unsigned char c) { return c == ' ' || c == '\t' || c == '\r' || c == '\n'; };
    while (!v.empty() && sp(v.front())) v.erase(v.begin());
    while (!v.empty() && sp(v.back())) v.pop_back();
    return v;
}

double number(const std::string& text, const char* field) {
    size_t used = 0;
    double v = 0;
    try {
        v = std::stod(text, &used);
    } catch (const std::exception&) {
        throw std::runtime_error(std::string("invalid grip trajectory number for ") + field);
    }
    if (used != text.size() || !std::isfinite(v))
        throw std::runtime_error(std::string("non-finite grip trajectory number for ") + field);
    return v;
}

double qdot(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2] + a[3] * b[3]; }

void qnormalize(double* q) {
    const double m = std::sqrt(qdot(q, q));
    if (!(m > 1.0e-14)) throw std::runtime_error("grip trajectory quaternion has zero length");
    for (int k = 0; k < 4; ++k) q[k] /= m;
}

void interpolate(const double* a, const double* b_in, double f, double* out) {
    double b[4] = {b_in[0], b_in[1], b_in[2], b_in[3]};
    double c = qdot(a, b);
    if (c < 0.0) {
        for (double& v : b) v = -v;
        c = -c;
    }
    c = std::clamp(c, -1.0, 1.0);
    if (c > 0.9995) {
        for (int k = 0; k < 4; ++k) out[k] = a[k] + f * (b[k] - a[k]);
    } else {
        const double angle = std::acos(c);
        const double s = std::sin(angle);
        const double wa = std::sin((1.0 - f) * angle) / s;
        const double wb = std::sin(f * angle) / s;
        for (int k = 0; k < 4; ++k) out[k] = wa * a[k] + wb * b[k];
    }
    qnormalize(out);
}

void set_err(char* err, size_t size, const std::string& msg) {
    if (err && size) {
        std::strncpy(err, msg.c_str(), size - 1);
        err[size - 1] = 0;
    }
}

}  // namespace

struct numi_cloth_trajectory {
    std::vector<Pose> poses;
    bool select_nearest = false;
    uint32_t version = 0;   // schema v1..v3
    uint64_t fingerprint = 0;
};

extern "C" {

numi_cloth_trajectory_t* numi_cloth_trajectory_load(const char* path, char* err, size_t err_size) {
    try {
        if (!path) throw std::runtime_error("null path");
        std::ifstream in(path, std::ios::binary);
        if (!in) throw std::runtime_error(std::string("cannot open grip trajectory: ") + path);
        std::ostringstream buf;
        buf << in.rdbuf();
        const std::string source = buf.str();
        auto* t = new numi_cloth_trajectory();
        uint64_t hash = 1469598103934665603ull;   // FNV-1a 64 of the file bytes
        for (unsigned char c : source) {
            hash ^= c;
            hash *= 1099511628211ull;
        }
        t->fingerprint = hash;
        std::istringstream lines(source);
        std::string line;
        bool schema = false, header = false, reactivate = false, prev_active = true;
        uint32_t generation = 1u;
        size_t line_no = 0;
        const char* expected[9] = {"time_s",       "translation_x_m", "translation_y_m",
                                   "translation_z_m", "quaternion_x", "quaternion_y",
                                   "quaternion_z", "quaternion_w",    "active"};
        try {
            while (std::getline(lines, line)) {
                ++line_no;
                line = trim(line);
                if (line.empty() || line[0] == '#') continue;
                if (!schema) {
                    if (line != "schema=numi.grip.trajectory.v1" && line != "schema=numi.grip.trajectory.v2" &&
                        line != "schema=numi.grip.trajectory.v3")
                        throw std::runtime_error("grip trajectory schema mismatch");
                    reactivate = line != "schema=numi.grip.trajectory.v1";
                    t->select_nearest = line == "schema=numi.grip.trajectory.v3";
                    t->version = static_cast<uint32_t>(line.back() - '0');
                    schema = true;
                    continue;
                }
                std::vector<std::string> fields;
                size_t begin = 0;
                while (true) {
                    const size_t comma = line.find(',', begin);
                    fields.push_back(trim(line.substr(begin, comma == std::string::npos ? std::string::npos : comma - begin)));
                    if (comma == std::string::npos) break;
                    begin = comma + 1;
                }
                if (!header) {
                    bool same = fields.size() == 9;
                    for (size_t k = 0; same && k < 9; ++k) same = fields[k] == expected[k];
                    if (!same) throw std::runtime_error("grip trajectory CSV header mismatch");
                    header = true;
                    continue;
                }
                if (fields.size() != 9)
                    throw std::runtime_error("grip trajectory row has wrong field count at " + std::to_string(line_no));
                Pose p{};
                p.t = number(fields[0], "time_s");
                for (int k = 0; k < 3; ++k) p.tr[k] = number(fields[1 + k], expected[1 + k]);
                for (int k = 0; k < 4; ++k) p.q[k] = number(fields[4 + k], expected[4 + k]);
                if (fields[8] == "1")
                    p.active = true;
                else if (fields[8] == "0")
                    p.active = false;
                else
                    throw std::runtime_error("grip trajectory active must be 0 or 1");
                if (p.t < 0.0 || (!t->poses.empty() && !(p.t > t->poses.back().t)))
                    throw std::runtime_error("grip trajectory times must be nonnegative and strictly increasing");
                if (std::abs(std::sqrt(qdot(p.q, p.q)) - 1.0) > 1.0e-3)
                    throw std::runtime_error("grip trajectory quaternion must be unit length within 1e-3");
                qnormalize(p.q);
                if (!t->poses.empty() && qdot(t->poses.back().q, p.q) < 0.0)
                    for (double& v : p.q) v = -v;
                if (!prev_active && p.active) {
                    if (!reactivate) throw std::runtime_error("grip trajectory v1 cannot reactivate after release");
                    if (generation == std::numeric_limits<uint32_t>::max())
                        throw std::runtime_error("grip trajectory has too many attachment generations");
                    ++generation;
                }
                p.generation = generation;
                prev_active = p.active;
                t->poses.push_back(p);
            }
            if (!schema || !header || t->poses.size() < 2u)
                throw std::runtime_error("grip trajectory requires schema, header, and at least two poses");
            const Pose& f = t->poses.front();
            const double tr = std::sqrt(f.tr[0] * f.tr[0] + f.tr[1] * f.tr[1] + f.tr[2] * f.tr[2]);
            const double rot = 2.0 * std::acos(std::clamp(std::abs(f.q[3]), 0.0, 1.0));
            if (std::abs(f.t) > 1.0e-12 || tr > 1.0e-9 || rot > 1.0e-9 || !f.active)
                throw std::runtime_error(
                    "grip trajectory must start at t=0 with zero translation, identity orientation, and an active "
                    "seam grip");
        } catch (...) {
            delete t;
            throw;
        }
        return t;
    } catch (const std::exception& e) {
        set_err(err, err_size, e.what());
        return nullptr;
    }
}

void numi_cloth_trajectory_destroy(numi_cloth_trajectory_t* t) { delete t; }

int numi_cloth_trajectory_sample(const numi_cloth_trajectory_t* t, double time, NumiClothGripPose* out) {
    if (!t || !out || t->poses.empty()) return NUMI_CLOTH_EINVAL;
    if (!std::isfinite(time) || time < 0.0 || time > t->poses.back().t + 1.0e-9) return NUMI_CLOTH_EINVAL;
    const Pose* a = &t->poses.front();
    const Pose* b = a;
    double f = 0.0;
    if (time <= t->poses.front().t) {
        a = b = &t->poses.front();
    } else if (time >= t->poses.back().t) {
        a = b = &t->poses.back();
    } else {
        const auto up = std::lower_bound(t->poses.begin(), t->poses.end(), time,
                                         [](const Pose& p, double v) { return p.t < v; });
        b = &*up;
        a = &*(up - 1);
        f = (time - a->t) / (b->t - a->t);
    }
    out->time = time;
    if (a == b) {
        for (int k = 0; k < 3; ++k) out->translation[k] = a->tr[k];
        for (int k = 0; k < 4; ++k) out->orientation[k] = a->q[k];
        out->active = a->active ? 1u : 0u;
        out->generation = a->generation;
        return NUMI_CLOTH_OK;
    }
    for (int k = 0; k < 3; ++k) out->translation[k] = a->tr[k] + f * (b->tr[k] - a->tr[k]);
    interpolate(a->q, b->q, f, out->orientation);
    out->active = (f >= 1.0 ? b->active : a->active) ? 1u : 0u;
    out->generation = f >= 1.0 ? b->generation : a->generation;
    return NUMI_CLOTH_OK;
}

int numi_cloth_trajectory_info(const numi_cloth_trajectory_t* t, uint32_t* select_nearest, double* duration,
                               uint64_t* fingerprint) {
    if (!t) return NUMI_CLOTH_EINVAL;
    if (select_nearest) *select_nearest = t->select_nearest ? 1u : 0u;
    if (duration) *duration = t->poses.back().t;
    if (fingerprint) *fingerprint = t->fingerprint;
    return NUMI_CLOTH_OK;
}

// maximumGripTrajectoryRotation and gripTrajectoryAttachmentGenerations
// (include/numi/grip_trajectory.h:371-389): the largest rotation angle
// 2 acos|w| of any pose, and the highest attachment generation.
int numi_cloth_trajectory_summary(const numi_cloth_trajectory_t* t, uint32_t* version, uint32_t* poses,
                                  double* max_rotation, uint32_t* generations) {
    if (!t) return NUMI_CLOTH_EINVAL;
    double rot = 0.0;
    uint32_t gen = 0u;
    for (const Pose& p : t->poses) {
        rot = std::max(rot, 2.0 * std::acos(std::clamp(std::abs(p.q[3]), 0.0, 1.0)));
        gen = std::max(gen, p.generation);
    }
    if (version) *version = t->version;
    if (poses) *poses = static_cast<uint32_t>(t->poses.size());
    if (max_rotation) *max_rotation = rot;
    if (generations) *generations = gen;
    return NUMI_CLOTH_OK;
}

int numi_cloth_trajectory_configs(const numi_cloth_trajectory_t* t, const NumiClothConfig* base,
                                  const double handle_base[3], uint64_t first, uint32_t count, double dt,
                                  NumiClothConfig* out) {
    if (!t || !base || !handle_base || !out || !(dt > 0.0)) return NUMI_CLOTH_EINVAL;
    for (uint32_t k = 0; k < count; ++k) {
        NumiClothGripPose pose;
        const double time = static_cast<double>(first + k + 1u) * dt;
        if (numi_cloth_trajectory_sample(t, time, &pose) != NUMI_CLOTH_OK) return NUMI_CLOTH_EINVAL;
        NumiClothConfig c = *base;
        c.gripTargetAndActive = {static_cast<float>(handle_base[0] + pose.translation[0]),
                                 static_cast<float>(handle_base[1] + pose.translation[1]),
                                 static_cast<float>(handle_base[2] + pose.translation[2]),
                                 pose.active ? 1.0f : 0.0f};
        c.gripOrientation = {static_cast<float>(pose.orientation[0]), static_cast<float>(pose.orientation[1]),
                             static_cast<float>(pose.orientation[2]), static_cast<float>(pose.orientation[3])};
        c.gripControl.x = pose.generation;
        c.gripControl.y = t->select_nearest ? 1u : 0u;
        out[k] = c;
    }
    return NUMI_CLOTH_OK;
}

}  // extern "C"
