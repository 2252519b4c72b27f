// Host-side scene builders and file contracts of the cloth solver.
//
// Produce bag: the reference scene of tools/cloth_bag.cpp:475-973 (authored
// wall and bottom weave, masses, warp/weft/bottom distances, crossing-angle
// knots, skip-one bends, ten seam grips, twelve fruits) with the first-fit
// 64-bit-mask colouring of tools/cloth_bag_metal.mm:627-676 (and its knot,
// bend and fruit-pair twins).  Geometry is evaluated in FP64 and rounded
// once to the FP32 records.
// Square cloth: no reference counterpart (see numi_cloth_scene.h).
#include <algorithm>
#include <array>
#include <bit>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <fstream>
#include <limits>
#include <numbers>
#include <sstream>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include "numi_cloth_scene.h"

namespace {

struct D3 {
    double x = 0, y = 0, z = 0;
};
D3 operator+(D3 a, D3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
D3 operator-(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
D3 operator*(D3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
double dot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
double norm(D3 a) { return std::sqrt(dot(a, a)); }
D3 unit(D3 a) {
    const double m = norm(a);
    return m > 1.0e-14 ? a * (1.0 / m) : D3{1.0, 0.0, 0.0};
}

numi_float4 f4(double x, double y, double z, double w) {
    return {static_cast<float>(x), static_cast<float>(y), static_cast<float>(z), static_cast<float>(w)};
}
numi_uint4 u4(uint32_t x, uint32_t y, uint32_t z, uint32_t w) { return {x, y, z, w}; }

// ----------------------------------------------------------- bag geometry
constexpr uint32_t kAround = 48;
constexpr uint32_t kLevels = 28;
constexpr uint32_t kBottomGrid = 13;
constexpr uint32_t kBottomInterior = kBottomGrid - 2u;
constexpr double kAirborneLift = 0.52;
constexpr double kGroundLift = 0.009;
constexpr double kPi = std::numbers::pi;

uint32_t node(uint32_t level, uint32_t ring) { return level * kAround + ring % kAround; }

double smooth(double v) {
    const double x = std::clamp(v, 0.0, 1.0);
    return x * x * (3.0 - 2.0 * x);
}

// Authored wall position (tools/cloth_bag.cpp:475-527).
D3 wall_position(uint32_t level, uint32_t ring) {
    const double vertical = static_cast<double>(level) / static_cast<double>(kLevels - 1);
    const double body = smooth(vertical / 0.55);
    const double fold = std::clamp((vertical - 0.72) / 0.28, 0.0, 1.0);
    const double skirt = 1.0 - smooth(vertical / 0.18);
    const double angle0 = 2.0 * kPi * static_cast<double>(ring) / static_cast<double>(kAround);
    const double base_radius = 0.266 + 0.030 * body - 0.116 * fold + 0.045 * skirt;
    const double angle = angle0 + 0.08 * vertical;
    const double wrinkle = 1.0 + 0.035 * std::sin(5.0 * angle + 5.0 * kPi * vertical) +
                           0.018 * std::sin(9.0 * angle - 3.0 * kPi * vertical);
    const double loose_rim = fold * (0.007 * std::sin(3.0 * angle + 0.35) + 0.004 * std::sin(7.0 * angle - 0.80));
    const double loose_skirt =
        skirt * (0.020 * std::sin(3.0 * angle - 0.40) + 0.012 * std::sin(7.0 * angle + 0.70));
    const double rim_sag = fold * (0.016 * std::sin(angle + 0.55) + 0.008 * std::sin(3.0 * angle - 0.30) +
                                   0.004 * std::sin(6.0 * angle + 0.90));
    const double radius = base_radius * wrinkle + loose_rim + loose_skirt;
    const double body_sag = body * (0.018 * std::sin(2.0 * angle + 0.30) + 0.009 * std::sin(5.0 * angle - 0.70));
    const double skirt_sag = skirt * (0.012 * std::sin(4.0 * angle + 0.20) + 0.006 * std::sin(9.0 * angle - 0.50));
    const double body_height = 0.012 + 0.155 * std::min(vertical / 0.72, 1.0) + body_sag;
    const double folded_height = fold < 0.35 ? 0.167 + 0.038 * (fold / 0.35) : 0.205 - 0.025 * ((fold - 0.35) / 0.65);
    return {radius * std::cos(angle), radius * std::sin(angle),
            (vertical < 0.72 ? body_height : folded_height) + rim_sag + skirt_sag + kGroundLift};
}

// Concentric square-to-disc map of the bottom weave (tools/cloth_bag.cpp:529-550).
std::pair<double, double> bottom_coordinate(uint32_t row, uint32_t column) {
    const double half = 0.5 * static_cast<double>(kBottomGrid - 1u);
    const double u = (static_cast<double>(column) - half) / half;
    const double v = (static_cast<double>(row) - half) / half;
    if (std::abs(u) < 1.0e-12 && std::abs(v) < 1.0e-12) return {0.0, 0.0};
    double radius, angle;
    if (std::abs(u) >= std::abs(v)) {
        radius = u;
        angle = (kPi / 4.0) * (v / u);
    } else {
        radius = v;
        angle = kPi / 2.0 - (kPi / 4.0) * (u / v);
    }
    return {radius * std::cos(angle), radius * std::sin(angle)};
}

bool bottom_boundary(uint32_t row, uint32_t column) {
    return row == 0u || column == 0u || row + 1u == kBottomGrid || column + 1u == kBottomGrid;
}

uint32_t bottom_index(uint32_t row, uint32_t column) {
    if (bottom_boundary(row, column)) {
        const auto [x, y] = bottom_coordinate(row, column);
        double angle = std::atan2(y, x);
        if (angle < 0.0) angle += 2.0 * kPi;
        return node(0u, static_cast<uint32_t>(std::llround(angle * static_cast<double>(kAround) / (2.0 * kPi))) %
                            kAround);
    }
    return kAround * kLevels + (row - 1u) * kBottomInterior + column - 1u;
}

D3 bottom_position(uint32_t row, uint32_t column) {
    const auto [x, y] = bottom_coordinate(row, column);
    const double radial = std::hypot(x, y);
    if (radial < 1.0e-12) return {0.0, 0.0, 0.012 + kGroundLift};
    double angle = std::atan2(y, x);
    if (angle < 0.0) angle += 2.0 * kPi;
    const double ring_coord = angle * static_cast<double>(kAround) / (2.0 * kPi);
    const uint32_t first = static_cast<uint32_t>(std::floor(ring_coord)) % kAround;
    const uint32_t second = (first + 1u) % kAround;
    const double fraction = ring_coord - std::floor(ring_coord);
    const D3 outer = wall_position(0u, first) * (1.0 - fraction) + wall_position(0u, second) * fraction;
    return {outer.x * radial, outer.y * radial, 0.012 + kGroundLift + radial * (outer.z - 0.012 - kGroundLift)};
}

// ------------------------------------------------------------- colouring
// First-fit colouring with a 64-bit colour mask per particle, in record
// order; returns the colour of each record (throws past 64 colours).
template <class Writers>
std::vector<uint32_t> first_fit(size_t count, size_t targets, Writers writers, uint32_t& colours) {
    std::vector<uint64_t> used(targets, 0u);
    std::vector<uint32_t> colour(count);
    colours = 0u;
    for (size_t k = 0; k < count; ++k) {
        uint32_t w[4];
        const uint32_t nw = writers(k, w);
        uint64_t busy = 0u;
        for (uint32_t e = 0; e < nw; ++e) busy |= used[w[e]];
        const uint64_t free = ~busy;
        if (free == 0u) throw std::logic_error("colouring exceeds 64 colours");
        const uint32_t c = static_cast<uint32_t>(std::countr_zero(free));
        colour[k] = c;
        colours = std::max(colours, c + 1u);
        for (uint32_t e = 0; e < nw; ++e) used[w[e]] |= uint64_t{1} << c;
    }
    return colour;
}

// Stable order by (colour, key); key sorts yarn segments ahead of shear.
std::vector<size_t> colour_order(const std::vector<uint32_t>& colour, const std::vector<uint32_t>& key) {
    std::vector<size_t> order(colour.size());
    for (size_t k = 0; k < order.size(); ++k) order[k] = k;
    std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) {
        if (colour[a] != colour[b]) return colour[a] < colour[b];
        return key[a] < key[b];
    });
    return order;
}

struct DistanceSpec {
    uint32_t first, second, kind;
    double compliance, limit;
};
struct KnotSpec {
    std::array<uint32_t, 4> p;
};
struct BendSpec {
    uint32_t first, middle, third;
    double compliance;
};

}  // namespace

struct numi_cloth_scene {
    NumiClothConfig config{};
    std::vector<NumiClothParticle> particles;
    std::vector<numi_float4> rest;
    std::vector<double> rest64;
    std::vector<NumiClothDistance> distances;
    std::vector<NumiClothKnot> knots;
    std::vector<NumiClothBend> bends;
    std::vector<NumiClothGrip> grips;
    std::vector<NumiClothFruit> fruits;
    std::vector<NumiClothFruitPair> pairs;
    std::vector<uint32_t> cuff;
    std::vector<uint32_t> rim;
    std::vector<uint32_t> local_off;
    std::vector<uint32_t> local_idx;
    uint32_t grid_width = 0;
    uint32_t dist_colours = 0, knot_colours = 0, bend_colours = 0, pair_colours = 0;
    uint32_t yarn_segments = 0;
    uint32_t bottom_center = 0;
    std::vector<uint32_t> triangles;   // render triangles, 3 indices each
};

namespace {

void add_particles(numi_cloth_scene* s, const std::vector<D3>& pos, const std::vector<double>& mass) {
    s->particles.resize(pos.size());
    s->rest.resize(pos.size());
    s->rest64.resize(3 * pos.size());
    for (size_t i = 0; i < pos.size(); ++i) {
        const double w = mass[i] > 0.0 ? 1.0 / mass[i] : 0.0;
        s->particles[i].positionAndInverseMass = f4(pos[i].x, pos[i].y, pos[i].z, w);
        s->particles[i].previousAndMass = f4(pos[i].x, pos[i].y, pos[i].z, mass[i]);
        s->particles[i].velocity = f4(0, 0, 0, 0);
        s->rest[i] = f4(pos[i].x, pos[i].y, pos[i].z, 0.0);
        s->rest64[3 * i] = pos[i].x;
        s->rest64[3 * i + 1] = pos[i].y;
        s->rest64[3 * i + 2] = pos[i].z;
    }
}

// Distances coloured as one class per colour group: group_of(kind) selects
// which kinds share a colour space (the bag has one group; the square
// cloth colours yarn and shear separately so a yarn colour holds no shear).
void add_distances(numi_cloth_scene* s, const std::vector<D3>& pos, const std::vector<DistanceSpec>& specs,
                   bool separate_shear) {
    const size_t n = pos.size();
    std::vector<uint32_t> colour(specs.size());
    uint32_t offset = 0;
    for (int group = 0; group < (separate_shear ? 2 : 1); ++group) {
        std::vector<size_t> members;
        for (size_t k = 0; k < specs.size(); ++k) {
            const bool shear = specs[k].kind == 3u;
            if (!separate_shear || (group == 1) == shear) members.push_back(k);
        }
        uint32_t colours = 0;
        const auto c = first_fit(members.size(), n,
                                 [&](size_t m, uint32_t* w) {
                                     w[0] = specs[members[m]].first;
                                     w[1] = specs[members[m]].second;
                                     return 2u;
                                 },
                                 colours);
        for (size_t m = 0; m < members.size(); ++m) colour[members[m]] = c[m] + offset;
        offset += colours;
    }
    s->dist_colours = offset;
    std::vector<uint32_t> key(specs.size());
    for (size_t k = 0; k < specs.size(); ++k) key[k] = specs[k].kind == 3u ? 1u : 0u;
    const auto order = colour_order(colour, key);
    s->distances.clear();
    s->yarn_segments = 0;
    for (size_t k : order) {
        const DistanceSpec& d = specs[k];
        NumiClothDistance r{};
        r.particlesAndColor = u4(d.first, d.second, colour[k], d.kind);
        r.material = f4(norm(pos[d.second] - pos[d.first]), d.compliance, 0.0, d.limit);
        s->distances.push_back(r);
        if (d.kind != 3u) ++s->yarn_segments;
    }
}

void add_knots(numi_cloth_scene* s, const std::vector<D3>& pos, const std::vector<KnotSpec>& specs,
               double compliance) {
    uint32_t colours = 0;
    const auto colour = first_fit(specs.size(), pos.size(),
                                  [&](size_t k, uint32_t* w) {
                                      for (int e = 0; e < 4; ++e) w[e] = specs[k].p[e];
                                      return 4u;
                                  },
                                  colours);
    s->knot_colours = colours;
    const auto order = colour_order(colour, std::vector<uint32_t>(specs.size(), 0u));
    for (size_t k : order) {
        const auto& p = specs[k].p;
        const D3 warp = unit(pos[p[1]] - pos[p[0]]);
        const D3 weft = unit(pos[p[3]] - pos[p[2]]);
        NumiClothKnot r{};
        r.particles = u4(p[0], p[1], p[2], p[3]);
        r.control = u4(colour[k], 0, 0, 0);
        r.material = f4(dot(warp, weft), compliance, 0.0, 0.0);
        s->knots.push_back(r);
    }
}

void add_bends(numi_cloth_scene* s, const std::vector<D3>& pos, const std::vector<BendSpec>& specs) {
    uint32_t colours = 0;
    const auto colour = first_fit(specs.size(), pos.size(),
                                  [&](size_t k, uint32_t* w) {
                                      w[0] = specs[k].first;
                                      w[1] = specs[k].third;
                                      return 2u;
                                  },
                                  colours);
    s->bend_colours = colours;
    const auto order = colour_order(colour, std::vector<uint32_t>(specs.size(), 0u));
    for (size_t k : order) {
        const BendSpec& b = specs[k];
        NumiClothBend r{};
        r.particlesAndColor = u4(b.first, b.middle, b.third, colour[k]);
        r.material = f4(norm(pos[b.third] - pos[b.first]),
                        norm(pos[b.middle] - pos[b.first]) + norm(pos[b.third] - pos[b.middle]), b.compliance, 0.0);
        s->bends.push_back(r);
    }
}

void add_pairs(numi_cloth_scene* s) {
    const uint32_t F = static_cast<uint32_t>(s->fruits.size());
    std::vector<std::array<uint32_t, 2>> specs;
    for (uint32_t a = 0; a < F; ++a)
        for (uint32_t b = a + 1u; b < F; ++b) specs.push_back({a, b});
    uint32_t colours = 0;
    const auto colour = first_fit(specs.size(), F,
                                  [&](size_t k, uint32_t* w) {
                                      w[0] = specs[k][0];
                                      w[1] = specs[k][1];
                                      return 2u;
                                  },
                                  colours);
    s->pair_colours = colours;
    const auto order = colour_order(colour, std::vector<uint32_t>(specs.size(), 0u));
    for (size_t k : order) {
        NumiClothFruitPair r{};
        r.fruitsAndColor = u4(specs[k][0], specs[k][1], colour[k], static_cast<uint32_t>(k));
        r.contact = f4(0, 0, 0, 0);
        s->pairs.push_back(r);
    }
}

// 2-hop neighbourhood over the distance graph (tools/cloth_bag.cpp:842-861).
void add_local_topology(numi_cloth_scene* s, size_t n) {
    std::vector<std::vector<uint32_t>> direct(n);
    for (const auto& d : s->distances) {
        direct[d.particlesAndColor.x].push_back(d.particlesAndColor.y);
        direct[d.particlesAndColor.y].push_back(d.particlesAndColor.x);
    }
    s->local_off.assign(n + 1, 0u);
    s->local_idx.clear();
    for (uint32_t i = 0; i < n; ++i) {
        std::vector<uint32_t> local{i};
        for (uint32_t a : direct[i]) {
            local.push_back(a);
            for (uint32_t b : direct[a]) local.push_back(b);
        }
        std::sort(local.begin(), local.end());
        local.erase(std::unique(local.begin(), local.end()), local.end());
        s->local_off[i] = static_cast<uint32_t>(s->local_idx.size());
        s->local_idx.insert(s->local_idx.end(), local.begin(), local.end());
    }
    s->local_off[n] = static_cast<uint32_t>(s->local_idx.size());
}

void base_config(numi_cloth_scene* s, const NumiClothMaterial& m, double dt, bool ground) {
    NumiClothConfig& c = s->config;
    c.control = u4(NUMI_CLOTH_ABI_VERSION, static_cast<uint32_t>(s->particles.size()),
                   static_cast<uint32_t>(s->distances.size()), static_cast<uint32_t>(s->grips.size()));
    c.constraintCounts = u4(static_cast<uint32_t>(s->knots.size()), static_cast<uint32_t>(s->bends.size()),
                            ground ? 1u : 0u, static_cast<uint32_t>(s->fruits.size()));
    c.contactCounts =
        u4(static_cast<uint32_t>(s->pairs.size()), static_cast<uint32_t>(s->fruits.size()) * s->yarn_segments, 0, 0);
    c.gravityAndTimestep = f4(0.0, 0.0, -9.81, dt);
    c.gripOrientation = f4(0, 0, 0, 1);
    c.gripMaterial = f4(0.12, 0, 0, 0);
    float max_limited = 0.0f;
    for (const auto& d : s->distances)
        if (d.material.w > 0.0f) max_limited = std::max(max_limited, d.material.x * (1.0f + d.material.w));
    c.clothMaterial = f4(m.yarnRadiusM, std::max(0.1f, max_limited + 0.008001f), m.clothGroundFriction,
                         m.clothSelfFriction);
    c.fruitMaterial = f4(m.fruitPairFriction, m.fruitGroundFriction, m.fruitRollingResistance, m.fruitYarnFriction);
    c.airVelocityAndDensity = f4(0, 0, 0, 1.225);
    c.aerodynamicCoefficients = f4(m.yarnCrossflowDrag, m.yarnSkinFriction, m.fruitDrag, m.fruitRotationalDrag);
    c.mouthMaterial = f4(0.025, 0, 0, 0);
}

NumiClothFruit make_fruit(D3 p, double radius, double mass, uint32_t appearance) {
    NumiClothFruit f{};
    f.positionAndInverseMass = f4(p.x, p.y, p.z, 1.0 / mass);
    f.previousAndRadius = f4(p.x, p.y, p.z, radius);
    f.velocityAndGroundImpulse = f4(0, 0, 0, 0);
    f.angularVelocity = f4(0, 0, 0, 0);
    f.orientation = f4(0, 0, 0, 1);
    f.identity = u4(appearance, 0, 0, 0);
    return f;
}

uint64_t splitmix64(uint64_t& state) {
    uint64_t z = (state += 0x9e3779b97f4a7c15ull);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}
double uniform01(uint64_t& state) { return static_cast<double>(splitmix64(state) >> 11) * 0x1.0p-53; }

void set_err(char* err, size_t size, const std::string& msg) {
    if (err && size) {
        std::strncpy(err, msg.c_str(), size - 1);
        err[size - 1] = 0;
    }
}

std::string trim(std::string v) {
    const auto sp = [](unsigned char c) { return c == ' ' || c == '\t' || c == '\r' || c == '\n'; };
    while (!v.empty() && sp(v.front())) v.erase(v.begin());
    while (!v.empty() && sp(v.back())) v.pop_back();
    return v;
}

}  // namespace

extern "C" {

void numi_cloth_material_defaults(NumiClothMaterial* m) {
    if (!m) return;
    *m = NumiClothMaterial{0.000050, 0.000100, 0.004, 1.0e-8, 1.0e-9, 2.0e-6, 8.0e-2, 1.0e-8, 2.0e-4, 0.45,
                           0.34,     0.36,     0.42,  0.30,   0.015,  1.10,   0.010,  0.47,   0.010};
}

// numi.cloth.material.v1 (include/numi/cloth_material.h:112-192): name=value
// lines, '#' comments, unique keys, schema and both provenance hashes
// required, all 19 parameters required and inside the contract bounds.
int numi_cloth_material_load(const char* path, NumiClothMaterial* out, char* err, size_t err_size) {
    try {
        if (!path || !out) throw std::runtime_error("null argument");
        std::ifstream in(path);
        if (!in) throw std::runtime_error(std::string("cannot open cloth material artifact: ") + path);
        NumiClothMaterial m;
        numi_cloth_material_defaults(&m);
        struct Field {
            const char* name;
            double* value;
            double lo, hi;
        };
        const Field fields[] = {
            {"ordinary_node_mass_kg", &m.ordinaryNodeMassKg, 0.000010, 0.000200},
            {"hem_node_mass_kg", &m.hemNodeMassKg, 0.000020, 0.000400},
            {"yarn_radius_m", &m.yarnRadiusM, 0.0005, 0.010},
            {"axial_body_compliance_m_per_n", &m.axialBodyComplianceMPerN, 1.0e-11, 1.0e-4},
            {"axial_cuff_compliance_m_per_n", &m.axialCuffComplianceMPerN, 1.0e-12, 1.0e-5},
            {"knot_compliance", &m.knotCompliance, 1.0e-10, 1.0e-2},
            {"bend_body_compliance_m_per_n", &m.bendBodyComplianceMPerN, 1.0e-5, 100.0},
            {"bend_cuff_compliance_m_per_n", &m.bendCuffComplianceMPerN, 1.0e-12, 1.0e-3},
            {"grip_compliance_m_per_n", &m.gripComplianceMPerN, 1.0e-8, 1.0},
            {"cloth_ground_friction", &m.clothGroundFriction, 0.01, 2.0},
            {"cloth_self_friction", &m.clothSelfFriction, 0.01, 2.0},
            {"fruit_yarn_friction", &m.fruitYarnFriction, 0.01, 2.0},
            {"fruit_ground_friction", &m.fruitGroundFriction, 0.01, 2.0},
            {"fruit_pair_friction", &m.fruitPairFriction, 0.01, 2.0},
            {"fruit_rolling_resistance", &m.fruitRollingResistance, 0.0001, 0.20},
            {"yarn_crossflow_drag", &m.yarnCrossflowDrag, 0.10, 3.0},
            {"yarn_skin_friction", &m.yarnSkinFriction, 0.0001, 0.20},
            {"fruit_drag", &m.fruitDrag, 0.05, 2.0},
            {"fruit_rotational_drag", &m.fruitRotationalDrag, 0.0001, 0.20},
        };
        std::unordered_set<std::string> seen;
        std::string schema, line;
        while (std::getline(in, line)) {
            line = trim(line);
            if (line.empty() || line[0] == '#') continue;
            const size_t eq = line.find('=');
            if (eq == std::string::npos) throw std::runtime_error("cloth material line must contain '='");
            const std::string name = trim(line.substr(0, eq));
            const std::string text = trim(line.substr(eq + 1));
            if (name.empty() || text.empty() || !seen.insert(name).second)
                throw std::runtime_error("cloth material fields must be nonempty and unique");
            if (name == "schema") {
                schema = text;
                continue;
            }
            if (name == "parameters_hash" || name == "observations_hash") continue;
            const Field* f = nullptr;
            for (const auto& cand : fields)
                if (name == cand.name) f = &cand;
            if (!f) throw std::runtime_error("unknown cloth material field: " + name);
            size_t used = 0;
            double v = 0;
            try {
                v = std::stod(text, &used);
            } catch (const std::exception&) {
                throw std::runtime_error("invalid cloth material value for " + name);
            }
            if (used != text.size() || !std::isfinite(v))
                throw std::runtime_error("non-finite cloth material value for " + name);
            *f->value = v;
        }
        if (schema != "numi.cloth.material.v1") throw std::runtime_error("cloth material schema mismatch");
        if (!seen.count("parameters_hash") || !seen.count("observations_hash"))
            throw std::runtime_error("cloth material provenance hashes are required");
        for (const auto& f : fields)
            if (!seen.count(f.name)) throw std::runtime_error(std::string("cloth material artifact is missing: ") + f.name);
        for (const auto& f : fields)
            if (!(*f.value >= f.lo && *f.value <= f.hi))
                throw std::runtime_error(std::string("cloth material parameter outside contract bounds: ") + f.name);
        *out = m;
        return 0;
    } catch (const std::exception& e) {
        set_err(err, err_size, e.what());
        return -1;
    }
}

numi_cloth_scene_t* numi_cloth_scene_bag(const NumiClothMaterial* material, int scenario, double timestep,
                                         int select_nearest) {
    try {
        NumiClothMaterial m;
        if (material)
            m = *material;
        else
            numi_cloth_material_defaults(&m);
        auto* s = new numi_cloth_scene();
        const double lift = scenario == NUMI_CLOTH_SCENARIO_SPIN ? kAirborneLift : 0.0;
        std::vector<D3> pos;
        std::vector<double> mass;
        for (uint32_t level = 0; level < kLevels; ++level)
            for (uint32_t ring = 0; ring < kAround; ++ring) {
                D3 p = wall_position(level, ring);
                p.z += lift;
                pos.push_back(p);
                mass.push_back(level + 2u >= kLevels ? m.hemNodeMassKg : m.ordinaryNodeMassKg);
            }
        for (uint32_t row = 1; row + 1u < kBottomGrid; ++row)
            for (uint32_t col = 1; col + 1u < kBottomGrid; ++col) {
                D3 p = bottom_position(row, col);
                p.z += lift;
                pos.push_back(p);
                mass.push_back(m.ordinaryNodeMassKg);
            }
        add_particles(s, pos, mass);
        // distances: weft rings, warp columns, bottom rows, bottom columns
        std::vector<DistanceSpec> ds;
        const double limit = 0.285;
        for (uint32_t level = 0; level < kLevels; ++level)
            for (uint32_t ring = 0; ring < kAround; ++ring)
                ds.push_back({node(level, ring), node(level, ring + 1u), 1u,
                              level + 2u >= kLevels ? m.axialCuffComplianceMPerN : m.axialBodyComplianceMPerN, limit});
        for (uint32_t level = 0; level + 1u < kLevels; ++level)
            for (uint32_t ring = 0; ring < kAround; ++ring)
                ds.push_back({node(level, ring), node(level + 1u, ring), 0u, m.axialBodyComplianceMPerN, limit});
        for (uint32_t row = 0; row < kBottomGrid; ++row)
            for (uint32_t col = 0; col + 1u < kBottomGrid; ++col)
                if (!(bottom_boundary(row, col) && bottom_boundary(row, col + 1u)))
                    ds.push_back({bottom_index(row, col), bottom_index(row, col + 1u), 2u, m.axialBodyComplianceMPerN,
                                  limit});
        for (uint32_t col = 0; col < kBottomGrid; ++col)
            for (uint32_t row = 0; row + 1u < kBottomGrid; ++row)
                if (!(bottom_boundary(row, col) && bottom_boundary(row + 1u, col)))
                    ds.push_back({bottom_index(row, col), bottom_index(row + 1u, col), 2u, m.axialBodyComplianceMPerN,
                                  limit});
        add_distances(s, pos, ds, false);
        std::vector<KnotSpec> ks;
        for (uint32_t level = 1; level + 1u < kLevels; ++level)
            for (uint32_t ring = 0; ring < kAround; ++ring)
                ks.push_back({{node(level - 1u, ring), node(level + 1u, ring), node(level, ring + kAround - 1u),
                               node(level, ring + 1u)}});
        for (uint32_t row = 1; row + 1u < kBottomGrid; ++row)
            for (uint32_t col = 1; col + 1u < kBottomGrid; ++col)
                ks.push_back({{bottom_index(row - 1u, col), bottom_index(row + 1u, col), bottom_index(row, col - 1u),
                               bottom_index(row, col + 1u)}});
        add_knots(s, pos, ks, m.knotCompliance);
        std::vector<BendSpec> bs;
        for (uint32_t level = 0; level < kLevels; ++level)
            for (uint32_t ring = 0; ring < kAround; ++ring)
                bs.push_back({node(level, ring + kAround - 1u), node(level, ring), node(level, ring + 1u),
                              level + 2u >= kLevels ? m.bendCuffComplianceMPerN : m.bendBodyComplianceMPerN});
        for (uint32_t level = 1; level + 1u < kLevels; ++level)
            for (uint32_t ring = 0; ring < kAround; ++ring)
                bs.push_back({node(level - 1u, ring), node(level, ring), node(level + 1u, ring),
                              m.bendBodyComplianceMPerN});
        for (uint32_t row = 1; row + 1u < kBottomGrid; ++row)
            for (uint32_t col = 1; col + 1u < kBottomGrid; ++col) {
                bs.push_back({bottom_index(row, col - 1u), bottom_index(row, col), bottom_index(row, col + 1u),
                              m.bendBodyComplianceMPerN});
                bs.push_back({bottom_index(col - 1u, row), bottom_index(col, row), bottom_index(col + 1u, row),
                              m.bendBodyComplianceMPerN});
            }
        add_bends(s, pos, bs);
        // seam grips (tools/cloth_bag.cpp:673-693)
        const D3 base = wall_position(kLevels - 1u, 0u) + D3{0.0, 0.0, lift};
        if (scenario != NUMI_CLOTH_SCENARIO_GROUNDED) {
            for (uint32_t level = kLevels - 2u; level < kLevels; ++level)
                for (int off : {-2, -1, 0, 1, 2}) {
                    const uint32_t ring = static_cast<uint32_t>((static_cast<int>(kAround) + off) % static_cast<int>(kAround));
                    const uint32_t i = node(level, ring);
                    NumiClothGrip g{};
                    g.particle = u4(i, 1u, 0u, 0u);
                    g.targetOffsetAndCompliance =
                        f4(pos[i].x - base.x, pos[i].y - base.y, pos[i].z - base.z, m.gripComplianceMPerN);
                    s->grips.push_back(g);
                }
        }
        // fruits (tools/cloth_bag.cpp:931-973)
        const double fp[12][3] = {{0.190, 0.000, 0.088},  {0.118, 0.149, 0.083},  {-0.042, 0.185, 0.093},
                                  {-0.171, 0.082, 0.078}, {-0.171, -0.082, 0.086}, {-0.042, -0.185, 0.090},
                                  {0.118, -0.149, 0.081}, {0.000, 0.000, 0.084},  {0.105, 0.000, 0.210},
                                  {0.000, 0.105, 0.210},  {-0.105, 0.000, 0.215}, {0.000, -0.105, 0.210}};
        const double fr[12] = {0.070, 0.065, 0.075, 0.060, 0.068, 0.072, 0.063, 0.066, 0.072, 0.064, 0.070, 0.067};
        const double fm[12] = {0.21, 0.17, 0.26, 0.14, 0.19, 0.23, 0.16, 0.18, 0.23, 0.17, 0.21, 0.18};
        const uint32_t fa[12] = {0, 1, 2, 1, 3, 0, 2, 3, 0, 1, 2, 3};
        for (int k = 0; k < 12; ++k)
            s->fruits.push_back(
                make_fruit(D3{fp[k][0], fp[k][1], fp[k][2] + kGroundLift + lift}, fr[k], fm[k], fa[k]));
        add_pairs(s);
        for (uint32_t level = kLevels - 2u; level < kLevels; ++level)
            for (uint32_t ring = 0; ring < kAround; ++ring) s->cuff.push_back(node(level, ring));
        for (uint32_t ring = 0; ring < kAround; ++ring) s->rim.push_back(node(kLevels - 1u, ring));
        add_local_topology(s, pos.size());
        s->bottom_center = bottom_index((kBottomGrid - 1u) / 2u, (kBottomGrid - 1u) / 2u);
        // render triangles (tools/cloth_bag.cpp:812-839): the wall quads, then
        // the bottom grid with alternating diagonals
        for (uint32_t level = 0; level + 1u < kLevels; ++level)
            for (uint32_t ring = 0; ring < kAround; ++ring) {
                const uint32_t next = (ring + 1u) % kAround;
                const uint32_t a = node(level, ring), b = node(level, next), c = node(level + 1u, ring),
                               d = node(level + 1u, next);
                s->triangles.insert(s->triangles.end(), {a, b, c, b, d, c});
            }
        for (uint32_t row = 0; row + 1u < kBottomGrid; ++row)
            for (uint32_t col = 0; col + 1u < kBottomGrid; ++col) {
                const uint32_t a = bottom_index(row, col), b = bottom_index(row, col + 1u),
                               c = bottom_index(row + 1u, col), d = bottom_index(row + 1u, col + 1u);
                if ((row + col) % 2u == 0u)
                    s->triangles.insert(s->triangles.end(), {a, c, b, b, c, d});
                else
                    s->triangles.insert(s->triangles.end(), {a, d, b, a, c, d});
            }
        base_config(s, m, timestep, scenario != NUMI_CLOTH_SCENARIO_SPIN);
        NumiClothConfig& c = s->config;
        c.gripTargetAndActive = f4(base.x, base.y, base.z, s->grips.empty() ? 0.0 : 1.0);
        c.gripControl = u4(1u, select_nearest ? 1u : 0u, kAround, 2u);
        c.mouthControl = u4(kAround, s->bottom_center, 0, 0);
        return s;
    } catch (...) {
        return nullptr;
    }
}

void numi_cloth_square_defaults(NumiClothSquareSpec* s) {
    if (!s) return;
    *s = NumiClothSquareSpec{};
    s->side = 256;
    s->spacing = 0.004;
    s->height = 0.5;
    s->particleMass = 0.0005;
    s->stretchCompliance = 1.0e-8;
    s->shearCompliance = 1.0e-8;
    s->bendCompliance = 1.0e-5;
    s->strainLimit = 0.10;
    s->gripCompliance = 2.0e-4;
    s->gripCorners = 2;
    s->fruitCount = 64;
    s->fruitRadiusMin = 0.02;
    s->fruitRadiusMax = 0.05;
    s->fruitMass = 0.1;
    s->fruitHeightMin = 0.55;
    s->fruitHeightMax = 1.0;
    s->thickness = 0.001;
    s->seed = 20260815ull;
    s->timestep = 1.0 / 2880.0;
    s->groundEnabled = 1;
}

numi_cloth_scene_t* numi_cloth_scene_square(const NumiClothSquareSpec* spec, const NumiClothMaterial* material) {
    try {
        if (!spec || spec->side < 3u || spec->fruitCount > 64u) return nullptr;
        NumiClothMaterial m;
        if (material)
            m = *material;
        else
            numi_cloth_material_defaults(&m);
        m.yarnRadiusM = spec->thickness;
        auto* s = new numi_cloth_scene();
        const uint32_t side = spec->side;
        const double h = spec->spacing;
        const double half = 0.5 * static_cast<double>(side - 1u) * h;
        std::vector<D3> pos(static_cast<size_t>(side) * side);
        std::vector<double> mass(pos.size(), spec->particleMass);
        auto id = [side](uint32_t i, uint32_t j) { return i * side + j; };
        for (uint32_t i = 0; i < side; ++i)
            for (uint32_t j = 0; j < side; ++j) pos[id(i, j)] = D3{j * h - half, i * h - half, spec->height};
        add_particles(s, pos, mass);
        std::vector<DistanceSpec> ds;
        for (uint32_t i = 0; i < side; ++i)
            for (uint32_t j = 0; j + 1u < side; ++j)
                ds.push_back({id(i, j), id(i, j + 1u), 0u, spec->stretchCompliance, spec->strainLimit});
        for (uint32_t i = 0; i + 1u < side; ++i)
            for (uint32_t j = 0; j < side; ++j)
                ds.push_back({id(i, j), id(i + 1u, j), 1u, spec->stretchCompliance, spec->strainLimit});
        for (uint32_t i = 0; i + 1u < side; ++i)
            for (uint32_t j = 0; j + 1u < side; ++j) ds.push_back({id(i, j), id(i + 1u, j + 1u), 3u, spec->shearCompliance, 0.0});
        for (uint32_t i = 0; i + 1u < side; ++i)
            for (uint32_t j = 0; j + 1u < side; ++j) ds.push_back({id(i, j + 1u), id(i + 1u, j), 3u, spec->shearCompliance, 0.0});
        add_distances(s, pos, ds, true);
        std::vector<BendSpec> bs;
        for (uint32_t i = 0; i < side; ++i)
            for (uint32_t j = 0; j + 2u < side; ++j) bs.push_back({id(i, j), id(i, j + 1u), id(i, j + 2u), spec->bendCompliance});
        for (uint32_t i = 0; i + 2u < side; ++i)
            for (uint32_t j = 0; j < side; ++j) bs.push_back({id(i, j), id(i + 1u, j), id(i + 2u, j), spec->bendCompliance});
        add_bends(s, pos, bs);
        const D3 base = pos[id(0, 0)];
        if (spec->gripCorners >= 1u) {
            std::vector<uint32_t> corners{id(0, 0)};
            if (spec->gripCorners >= 2u) corners.push_back(id(0, side - 1u));
            for (uint32_t i : corners) {
                NumiClothGrip g{};
                g.particle = u4(i, 1u, 0u, 0u);
                g.targetOffsetAndCompliance =
                    f4(pos[i].x - base.x, pos[i].y - base.y, pos[i].z - base.z, spec->gripCompliance);
                s->grips.push_back(g);
            }
        }
        // Seeded spheres, each redrawn (up to kSphereDraws times) until it
        // overlaps no earlier sphere, so the scene starts without fruit/fruit
        // penetration.
        constexpr uint32_t kSphereDraws = 4096;
        uint64_t rng = spec->seed;
        std::vector<D3> centres;
        std::vector<double> radii;
        for (uint32_t k = 0; k < spec->fruitCount; ++k) {
            D3 c{};
            double r = 0.0;
            bool clear = false;
            for (uint32_t draw = 0; draw < kSphereDraws && !clear; ++draw) {
                const double x = -half + 2.0 * half * uniform01(rng);
                const double y = -half + 2.0 * half * uniform01(rng);
                const double bottom =
                    spec->fruitHeightMin + (spec->fruitHeightMax - spec->fruitHeightMin) * uniform01(rng);
                r = spec->fruitRadiusMin + (spec->fruitRadiusMax - spec->fruitRadiusMin) * uniform01(rng);
                c = D3{x, y, bottom + r};
                clear = true;
                for (size_t j = 0; j < centres.size() && clear; ++j) {
                    const double dx = c.x - centres[j].x, dy = c.y - centres[j].y, dz = c.z - centres[j].z;
                    clear = dx * dx + dy * dy + dz * dz >= (r + radii[j]) * (r + radii[j]);
                }
            }
            if (!clear) {
                delete s;
                return nullptr;   // no room for the requested spheres
            }
            centres.push_back(c);
            radii.push_back(r);
            s->fruits.push_back(make_fruit(c, r, spec->fruitMass, k & 3u));
        }
        add_pairs(s);
        s->grid_width = side;
        for (uint32_t i = 0; i + 1u < side; ++i)
            for (uint32_t j = 0; j + 1u < side; ++j) {
                const uint32_t a = id(i, j), b = id(i, j + 1u), c = id(i + 1u, j), d = id(i + 1u, j + 1u);
                s->triangles.insert(s->triangles.end(), {a, b, c, b, d, c});
            }
        base_config(s, m, spec->timestep, spec->groundEnabled != 0u);
        NumiClothConfig& c = s->config;
        c.gripTargetAndActive = f4(base.x, base.y, base.z, s->grips.empty() ? 0.0 : 1.0);
        c.gripControl = u4(1u, 0u, 0u, 0u);
        c.gripMaterial = f4(1.0e9, 0, 0, 0);
        c.clothMaterial.y = static_cast<float>(2.0 * spec->thickness);
        return s;
    } catch (...) {
        return nullptr;
    }
}

void numi_cloth_scene_destroy(numi_cloth_scene_t* s) { delete s; }

int numi_cloth_scene_view(const numi_cloth_scene_t* s, NumiClothScene* out) {
    if (!s || !out) return NUMI_CLOTH_EINVAL;
    *out = NumiClothScene{};
    out->config = &s->config;
    out->particles = s->particles.data();
    out->restPositions = s->rest.data();
    out->distances = s->distances.empty() ? nullptr : s->distances.data();
    out->knots = s->knots.empty() ? nullptr : s->knots.data();
    out->bends = s->bends.empty() ? nullptr : s->bends.data();
    out->grips = s->grips.empty() ? nullptr : s->grips.data();
    out->fruits = s->fruits.empty() ? nullptr : s->fruits.data();
    out->fruitPairs = s->pairs.empty() ? nullptr : s->pairs.data();
    out->cuffParticles = s->cuff.empty() ? nullptr : s->cuff.data();
    out->mouthRim = s->rim.empty() ? nullptr : s->rim.data();
    out->localOffsets = s->local_off.empty() ? nullptr : s->local_off.data();
    out->localIndices = s->local_idx.empty() ? nullptr : s->local_idx.data();
    out->gridWidth = s->grid_width;
    return NUMI_CLOTH_OK;
}

int numi_cloth_scene_counts(const numi_cloth_scene_t* s, uint32_t out[15]) {
    if (!s || !out) return NUMI_CLOTH_EINVAL;
    const uint32_t v[15] = {static_cast<uint32_t>(s->particles.size()),
                            static_cast<uint32_t>(s->distances.size()),
                            static_cast<uint32_t>(s->knots.size()),
                            static_cast<uint32_t>(s->bends.size()),
                            static_cast<uint32_t>(s->grips.size()),
                            static_cast<uint32_t>(s->fruits.size()),
                            static_cast<uint32_t>(s->pairs.size()),
                            static_cast<uint32_t>(s->cuff.size() / 2u),
                            static_cast<uint32_t>(s->rim.size()),
                            s->dist_colours,
                            s->knot_colours,
                            s->bend_colours,
                            s->pair_colours,
                            s->yarn_segments,
                            s->bottom_center};
    std::memcpy(out, v, sizeof(v));
    return NUMI_CLOTH_OK;
}

uint32_t numi_cloth_scene_triangles(const numi_cloth_scene_t* s, uint32_t* out, uint32_t capacity) {
    if (!s) return 0;
    const uint32_t count = static_cast<uint32_t>(s->triangles.size() / 3u);
    if (out) std::memcpy(out, s->triangles.data(), 3u * std::min(count, capacity) * sizeof(uint32_t));
    return count;
}

int numi_cloth_bag_handle_base(int scenario, double out[3]) {
    if (!out || scenario < NUMI_CLOTH_SCENARIO_GROUNDED || scenario > NUMI_CLOTH_SCENARIO_RECORDED)
        return NUMI_CLOTH_EINVAL;
    D3 p = wall_position(kLevels - 1u, 0u);
    if (scenario == NUMI_CLOTH_SCENARIO_SPIN) p.z += kAirborneLift;
    out[0] = p.x;
    out[1] = p.y;
    out[2] = p.z;
    return NUMI_CLOTH_OK;
}

// The scripted grip motions of the spin and pickup scenarios
// (spinGripTarget, pickupGripTarget, tools/cloth_bag.cpp:1476-1502).
int numi_cloth_bag_grip_target(int scenario, double time, double out[3]) {
    if (!out) return NUMI_CLOTH_EINVAL;
    D3 base = wall_position(kLevels - 1u, 0u);
    if (scenario == NUMI_CLOTH_SCENARIO_SPIN) {
        base.z += kAirborneLift;
        const double radius = 0.28, angular_speed = 4.8, ramp = 0.18;
        const double angle = angular_speed * (time - ramp * (1.0 - std::exp(-time / ramp)));
        out[0] = base.x + radius * (std::cos(angle) - 1.0);
        out[1] = base.y + radius * std::sin(angle);
        out[2] = base.z + 0.035 * std::sin(0.5 * angle);
        return NUMI_CLOTH_OK;
    }
    if (scenario == NUMI_CLOTH_SCENARIO_PICKUP) {
        const double lift = smooth(time / 0.80);
        const double snap = smooth((time - 1.00) / 0.23);
        const double recovery = smooth((time - 1.45) / 0.50);
        out[0] = base.x + -0.10 * snap;
        out[1] = base.y + 0.04 * std::sin(kPi * snap);
        out[2] = base.z + (1.25 * lift - 0.85 * snap + 0.75 * recovery);
        return NUMI_CLOTH_OK;
    }
    return NUMI_CLOTH_EINVAL;
}

int numi_cloth_bag_scenario_configs(int scenario, const NumiClothConfig* base, uint64_t first_substep,
                                    uint32_t count, double timestep, NumiClothConfig* out, double* targets) {
    if (!base || !out || !(timestep > 0.0)) return NUMI_CLOTH_EINVAL;
    if (scenario != NUMI_CLOTH_SCENARIO_GROUNDED && scenario != NUMI_CLOTH_SCENARIO_SPIN &&
        scenario != NUMI_CLOTH_SCENARIO_PICKUP)
        return NUMI_CLOTH_EINVAL;
    for (uint32_t k = 0; k < count; ++k) {
        out[k] = *base;
        double g[3] = {0.0, 0.0, 0.0};
        if (scenario != NUMI_CLOTH_SCENARIO_GROUNDED) {
            // the grip moves to its pose at the end of the substep
            // (tools/cloth_bag.cpp:4776-4786)
            const double time = static_cast<double>(first_substep + k + 1u) * timestep;
            numi_cloth_bag_grip_target(scenario, time, g);
            out[k].gripTargetAndActive = f4(g[0], g[1], g[2], 1.0);
            out[k].gripOrientation = f4(0.0, 0.0, 0.0, 1.0);
        }
        if (targets) {
            targets[3u * k + 0u] = g[0];
            targets[3u * k + 1u] = g[1];
            targets[3u * k + 2u] = g[2];
        }
    }
    return NUMI_CLOTH_OK;
}

int numi_cloth_scene_rest_fp64(const numi_cloth_scene_t* s, double* out) {
    if (!s || !out) return NUMI_CLOTH_EINVAL;
    std::memcpy(out, s->rest64.data(), s->rest64.size() * sizeof(double));
    return NUMI_CLOTH_OK;
}

}  // extern "C"
