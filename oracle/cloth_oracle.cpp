// CPU restatement of the reference XPBD cloth substep - TEST INFRASTRUCTURE.
//
// Used only as the checker by tests/, __graft_entry__.smoke() and bench.py's
// CPU-baseline leg; never linked into the product.  Every function cites the
// reference function it restates (file:line in the reference tree).  The
// float instantiation mirrors the B200 kernels' evaluation order term by
// term so that, on the same inputs and the same batched schedule, the GPU
// path and this oracle agree bit for bit; the double instantiation is the
// FP64 oracle the FP32 path is measured against.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <map>
#include <numbers>
#include <type_traits>
#include <unordered_map>
#include <utility>
#include <vector>

#include "oracle.h"

namespace {

template <class R>
struct V {
    R x{}, y{}, z{};
};
template <class R> V<R> operator+(V<R> a, V<R> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class R> V<R> operator-(V<R> a, V<R> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class R> V<R> operator*(V<R> a, R s) { return {a.x * s, a.y * s, a.z * s}; }
// tools/cloth_bag.cpp:122-124: a / s is a * (1 / s).
template <class R> V<R> vdiv(V<R> a, R s) { return a * (R(1) / s); }
template <class R> R dot(V<R> a, V<R> b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
template <class R> R lsq(V<R> a) { return dot(a, a); }
template <class R> R len(V<R> a) { return std::sqrt(lsq(a)); }
template <class R> V<R> cross(V<R> a, V<R> b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
// tools/cloth_bag.cpp:156-159.
template <class R> V<R> normalized(V<R> a) {
    const R m = len(a);
    return m > R(1.0e-14) ? vdiv(a, m) : V<R>{R(1), R(0), R(0)};
}
template <class R> struct Q {   // xyzw
    R x{}, y{}, z{}, w{1};
};
// tools/cloth_bag.cpp:206-214.
template <class R> V<R> rotate(Q<R> q, V<R> v) {
    const V<R> u{q.x, q.y, q.z};
    const V<R> twice = cross(u, v) * R(2);
    return (v + twice * q.w) + cross(u, twice);
}
template <class R> V<R> inverse_rotate(Q<R> q, V<R> v) { return rotate(Q<R>{-q.x, -q.y, -q.z, q.w}, v); }
template <class R> R rmin(R a, R b) { return b < a ? b : a; }
template <class R> R rmax(R a, R b) { return a < b ? b : a; }
template <class R> R clamp01(R v) { return rmin(rmax(v, R(0)), R(1)); }

constexpr double kFixedScale = 1099511627776.0;   // 2^40

struct BatchInfo {
    uint32_t first, count, limited, yarn;
};

// Colour runs of an array (the schedule the kernels run).
template <class Rec, class Colour, class Yarn, class Limited>
std::vector<BatchInfo> colour_runs(const std::vector<Rec>& recs, Colour colour, Yarn yarn, Limited limited) {
    std::vector<BatchInfo> out;
    uint32_t k = 0;
    const uint32_t n = static_cast<uint32_t>(recs.size());
    while (k < n) {
        BatchInfo b{k, 0, 0, 0};
        const uint32_t c = colour(recs[k]);
        while (k < n && colour(recs[k]) == c) {
            if (yarn(recs[k])) b.yarn = k - b.first + 1u;
            if (limited(recs[k])) b.limited = k - b.first + 1u;
            ++k;
        }
        b.count = k - b.first;
        out.push_back(b);
    }
    return out;
}

template <class R>
struct Sim {
    static constexpr bool kF32 = std::is_same_v<R, float>;
    // particles
    std::vector<V<R>> x, xp, v, rest, force;
    std::vector<R> w, mass, vw;
    // distances
    std::vector<uint32_t> di, dj, dcol, dkind;
    std::vector<R> drest, dcomp, dlam, dmax;
    // knots
    std::vector<uint32_t> kp0, kp1, kp2, kp3, kcol;
    std::vector<R> kcos, kcomp, klam;
    // bends
    std::vector<uint32_t> bp0, bp1, bp2, bcol;
    std::vector<R> bchord, bcomp, blam;
    // grips
    struct Grip {
        uint32_t particle, gen, ring;
        V<R> offset;
        R compliance;
        V<R> lambda;
        R capture, error;
    };
    std::vector<Grip> grips;
    // fruits
    struct Fruit {
        V<R> x, prev, v, omega;
        R w, radius, ground;
        Q<R> q;
        uint32_t appearance;
    };
    std::vector<Fruit> fruits;
    struct Pair {
        uint32_t a, b, colour;
        V<R> wn;
        R ni;
    };
    std::vector<Pair> pairs;
    std::vector<uint32_t> serial_pairs;   // pair indices in (a, b) order
    std::vector<uint32_t> cuff, rim, local_off, local_idx;
    OracleParams prm{};
    R radius{};
    std::vector<BatchInfo> dist_b, knot_b, bend_b, pair_b;
    // fruit/yarn contact records of the current substep: (segment, fruit)
    struct YarnRecord {
        V<R> wn;
        R ni{}, ws0{}, ws1{};
    };
    std::map<std::pair<uint32_t, uint32_t>, YarnRecord> yarn;
    // fruit sums of a batched sweep
    std::vector<long long> fix;     // float mode: 9 per fruit
    std::vector<double> acc;        // double mode: 9 per fruit
    uint32_t failure = 0;
    uint64_t reconcile_max = 0, cert_max = 0, yarn_contacts = 0, self_contacts = 0;
    uint64_t edge_contacts = 0, self_friction_contacts = 0;
    R self_cone = R(0);   // largest tangential / limit ratio of self friction
    uint32_t candidate_mask = 0, released_mask = 0;
    // yarn segments: the distances that are not shear diagonals, in array
    // order (the reference's yarnSegments, tools/cloth_bag.cpp:695-713)
    std::vector<uint32_t> ya, yb;
    // edge/edge contact impulses of the current substep, keyed
    // (first segment << 32) | second segment (SelfEdgeEdgeContactImpulse,
    // tools/cloth_bag.cpp:3962-3985)
    struct EdgeRecord {
        uint32_t a0{}, a1{}, b0{}, b1{};
        V<R> wn;
        R wf[2]{}, ws[2]{};
        R ni{};
    };
    std::map<uint64_t, EdgeRecord> edge_rec;

    // ------------------------------------------------------------- set-up
    bool init(const OracleScene& s) {
        if (!s.particles || !s.params || s.n == 0) return false;
        prm = *s.params;
        radius = static_cast<R>(prm.radius);
        const uint32_t n = s.n;
        x.resize(n); xp.resize(n); v.resize(n); rest.resize(n); force.resize(n);
        w.resize(n); mass.resize(n); vw.resize(n);
        for (uint32_t i = 0; i < n; ++i) {
            const OracleParticle& p = s.particles[i];
            x[i] = {R(p.x[0]), R(p.x[1]), R(p.x[2])};
            xp[i] = {R(p.prev[0]), R(p.prev[1]), R(p.prev[2])};
            v[i] = {R(p.v[0]), R(p.v[1]), R(p.v[2])};
            rest[i] = {R(p.rest[0]), R(p.rest[1]), R(p.rest[2])};
            w[i] = R(p.w);
            mass[i] = R(p.mass);
            vw[i] = R(p.vw);
        }
        for (uint32_t k = 0; k < s.d; ++k) {
            const OracleDistance& d = s.distances[k];
            if (d.i >= n || d.j >= n || d.i == d.j) return false;
            di.push_back(d.i); dj.push_back(d.j); dcol.push_back(d.colour); dkind.push_back(d.kind);
            drest.push_back(R(d.rest)); dcomp.push_back(R(d.compliance)); dlam.push_back(R(d.lambda));
            dmax.push_back(R(d.maxext));
            if (d.kind != 3u) {
                ya.push_back(d.i);
                yb.push_back(d.j);
            }
        }
        for (uint32_t k = 0; k < s.k; ++k) {
            const OracleKnot& q = s.knots[k];
            for (uint32_t e = 0; e < 4; ++e) if (q.p[e] >= n) return false;
            kp0.push_back(q.p[0]); kp1.push_back(q.p[1]); kp2.push_back(q.p[2]); kp3.push_back(q.p[3]);
            kcol.push_back(q.colour); kcos.push_back(R(q.restcos)); kcomp.push_back(R(q.compliance));
            klam.push_back(R(q.lambda));
        }
        for (uint32_t k = 0; k < s.b; ++k) {
            const OracleBend& b = s.bends[k];
            for (uint32_t e = 0; e < 3; ++e) if (b.p[e] >= n) return false;
            bp0.push_back(b.p[0]); bp1.push_back(b.p[1]); bp2.push_back(b.p[2]); bcol.push_back(b.colour);
            bchord.push_back(R(b.restchord)); bcomp.push_back(R(b.compliance)); blam.push_back(R(b.lambda));
        }
        for (uint32_t k = 0; k < s.g; ++k) {
            const OracleGrip& g = s.grips[k];
            if (g.particle >= n) return false;
            grips.push_back({g.particle, g.gen, g.ring, {R(g.offset[0]), R(g.offset[1]), R(g.offset[2])},
                             R(g.compliance), {R(g.lambda[0]), R(g.lambda[1]), R(g.lambda[2])}, R(g.capture),
                             R(g.error)});
        }
        for (uint32_t k = 0; k < s.f; ++k) {
            const OracleFruit& f = s.fruits[k];
            Fruit o;
            o.x = {R(f.x[0]), R(f.x[1]), R(f.x[2])};
            o.prev = {R(f.prev[0]), R(f.prev[1]), R(f.prev[2])};
            o.v = {R(f.v[0]), R(f.v[1]), R(f.v[2])};
            o.omega = {R(f.omega[0]), R(f.omega[1]), R(f.omega[2])};
            o.w = R(f.w);
            o.radius = R(f.radius);
            o.ground = R(f.ground_impulse);
            o.q = {R(f.q[0]), R(f.q[1]), R(f.q[2]), R(f.q[3])};
            o.appearance = f.appearance;
            fruits.push_back(o);
        }
        if (fruits.size() > 64u) return false;
        for (uint32_t k = 0; k < s.p; ++k) {
            const OraclePair& p = s.pairs[k];
            if (p.a >= s.f || p.b >= s.f || p.a == p.b) return false;
            pairs.push_back({p.a, p.b, p.colour, {R(p.wn[0]), R(p.wn[1]), R(p.wn[2])}, R(p.ni)});
        }
        serial_pairs.resize(pairs.size());
        for (uint32_t k = 0; k < pairs.size(); ++k) serial_pairs[k] = k;
        std::stable_sort(serial_pairs.begin(), serial_pairs.end(), [&](uint32_t a, uint32_t b) {
            return std::make_pair(pairs[a].a, pairs[a].b) < std::make_pair(pairs[b].a, pairs[b].b);
        });
        if (s.cuff) cuff.assign(s.cuff, s.cuff + 2u * prm.ring_count);
        if (s.rim) rim.assign(s.rim, s.rim + prm.rim_count);
        if (s.local_off) {
            local_off.assign(s.local_off, s.local_off + n + 1u);
            local_idx.assign(s.local_idx, s.local_idx + local_off[n]);
        }
        std::vector<uint32_t> ids(s.d);
        for (uint32_t k = 0; k < s.d; ++k) ids[k] = k;
        dist_b = colour_runs(ids, [&](uint32_t k) { return dcol[k]; }, [&](uint32_t k) { return dkind[k] != 3u; },
                             [&](uint32_t k) { return dmax[k] > R(0); });
        ids.resize(s.k);
        for (uint32_t k = 0; k < s.k; ++k) ids[k] = k;
        knot_b = colour_runs(ids, [&](uint32_t k) { return kcol[k]; }, [](uint32_t) { return false; },
                             [](uint32_t) { return false; });
        ids.resize(s.b);
        for (uint32_t k = 0; k < s.b; ++k) ids[k] = k;
        bend_b = colour_runs(ids, [&](uint32_t k) { return bcol[k]; }, [](uint32_t) { return false; },
                             [](uint32_t) { return false; });
        ids.resize(s.p);
        for (uint32_t k = 0; k < s.p; ++k) ids[k] = k;
        pair_b = colour_runs(ids, [&](uint32_t k) { return pairs[k].colour; }, [](uint32_t) { return false; },
                             [](uint32_t) { return false; });
        fix.assign(9u * 64u, 0);
        acc.assign(9u * 64u, 0.0);
        return true;
    }

    // ------------------------------------------------------ constraints
    // XPBD distance (tools/cloth_bag.cpp:1649-1673).
    void solve_distance(uint32_t k, R dt2) {
        const uint32_t a = di[k], b = dj[k];
        const V<R> diff = x[b] - x[a];
        const R L = len(diff);
        if (L < R(1.0e-12)) return;
        const R alpha = dcomp[k] / dt2;
        const R den = (w[a] + w[b]) + alpha;
        if (den <= R(0)) return;
        const R value = L - drest[k];
        const R dl = (-value - alpha * dlam[k]) / den;
        const V<R> corr = diff * (dl / L);
        x[a] = x[a] - corr * w[a];
        x[b] = x[b] + corr * w[b];
        dlam[k] = dlam[k] + dl;
    }

    // Crossing-angle knot (tools/cloth_bag.cpp:1675-1725).
    void solve_knot(uint32_t k, R dt2) {
        const uint32_t i0 = kp0[k], i1 = kp1[k], i2 = kp2[k], i3 = kp3[k];
        const V<R> warpv = x[i1] - x[i0];
        const V<R> weftv = x[i3] - x[i2];
        const R wl = len(warpv), fl = len(weftv);
        if (wl < R(1.0e-12) || fl < R(1.0e-12)) return;
        const V<R> warp = vdiv(warpv, wl);
        const V<R> weft = vdiv(weftv, fl);
        const R cosine = rmin(rmax(dot(warp, weft), R(-1)), R(1));
        const R value = cosine - kcos[k];
        const V<R> gw = vdiv(weft - warp * cosine, wl);
        const V<R> gf = vdiv(warp - weft * cosine, fl);
        const V<R> g0 = gw * R(-1);
        const V<R> g2 = gf * R(-1);
        const R alpha = kcomp[k] / dt2;
        R den = alpha;
        den = den + w[i0] * lsq(g0);
        den = den + w[i1] * lsq(gw);
        den = den + w[i2] * lsq(g2);
        den = den + w[i3] * lsq(gf);
        if (den <= R(0)) return;
        const R dl = (-value - alpha * klam[k]) / den;
        klam[k] = klam[k] + dl;
        x[i0] = x[i0] + g0 * (w[i0] * dl);
        x[i1] = x[i1] + gw * (w[i1] * dl);
        x[i2] = x[i2] + g2 * (w[i2] * dl);
        x[i3] = x[i3] + gf * (w[i3] * dl);
    }

    // Skip-one chord with the ground active set (tools/cloth_bag.cpp:1782-1863).
    void solve_bend(uint32_t k, R dt2, bool ground) {
        const uint32_t idx[2] = {bp0[k], bp2[k]};
        const V<R> diff = x[idx[1]] - x[idx[0]];
        const R chord = len(diff);
        if (chord < R(1.0e-12)) return;
        const R value = chord - bchord[k];
        const V<R> dir = vdiv(diff, chord);
        const V<R> g[2] = {dir * R(-1), dir};
        const R alpha = bcomp[k] / dt2;
        R free_den = alpha;
        free_den = free_den + w[idx[0]] * lsq(g[0]);
        free_den = free_den + w[idx[1]] * lsq(g[1]);
        if (free_den < R(1.0e-16)) return;
        const R numerator = -value - alpha * blam[k];
        const R free_dl = numerator / free_den;
        bool active[2];
        R den = alpha;
        for (int s = 0; s < 2; ++s) {
            active[s] = ground && x[idx[s]].z <= radius + R(1.0e-9) && g[s].z * free_dl < R(0);
            den = den + w[idx[s]] * (lsq(g[s]) - (active[s] ? g[s].z * g[s].z : R(0)));
        }
        if (den < R(1.0e-16)) return;
        const R dl = numerator / den;
        R fraction = R(1);
        if (ground) {
            for (int s = 0; s < 2; ++s) {
                if (active[s]) continue;
                const R vc = g[s].z * w[idx[s]] * dl;
                if (vc >= R(0)) continue;
                fraction = rmin(fraction, rmax(R(0), x[idx[s]].z - radius) / -vc);
            }
        }
        const R applied = dl * fraction;
        blam[k] = blam[k] + applied;
        for (int s = 0; s < 2; ++s) {
            V<R> corr = g[s] * (w[idx[s]] * applied);
            if (active[s]) corr.z = R(0);
            V<R> np = x[idx[s]] + corr;
            if (ground && np.z < radius) np.z = radius;
            x[idx[s]] = np;
        }
    }

    // Unilateral strain limit (tools/cloth_bag.cpp:1732-1763).
    R limit_strain(uint32_t k) {
        if (!(dmax[k] > R(0))) return R(0);
        const uint32_t a = di[k], b = dj[k];
        const V<R> diff = x[b] - x[a];
        const R L = len(diff);
        const R maxL = drest[k] * (R(1) + dmax[k]);
        if (L <= maxL || L < R(1.0e-12)) return R(0);
        const R den = w[a] + w[b];
        if (den <= R(0)) return R(0);
        const R cm = L - maxL;
        const V<R> dir = vdiv(diff, L);
        x[a] = x[a] + dir * (w[a] * cm / den);
        x[b] = x[b] - dir * (w[b] * cm / den);
        return cm;
    }

    // ------------------------------------------------------------- grips
    // Re-grab on a generation change (tools/cloth_bag.cpp:1520-1611).
    void grip_attach(const OracleSubstep& sub, bool serial) {
        if (!sub.grip_active || grips.empty()) return;
        const V<R> target{R(sub.grip_target[0]), R(sub.grip_target[1]), R(sub.grip_target[2])};
        const Q<R> q{R(sub.grip_q[0]), R(sub.grip_q[1]), R(sub.grip_q[2]), R(sub.grip_q[3])};
        if (serial) {
            // The reference re-grabs all ten grips together and rejects the
            // whole re-grab when any particle is beyond the capture radius.
            if (grips[0].gen == sub.grip_gen) return;
            if (grips[0].gen == 0xffffffffu || grips[0].gen + 1u != sub.grip_gen) {
                failure |= 1u << 4;
                return;
            }
            uint32_t center = 0;
            if (sub.grip_select == 1u) {
                R nearest = std::numeric_limits<R>::infinity();
                for (uint32_t ring = 0; ring < prm.ring_count; ++ring) {
                    const R dsq = lsq(x[cuff[prm.ring_count + ring]] - target);
                    if (dsq < nearest) {
                        nearest = dsq;
                        center = ring;
                    }
                }
                const uint32_t width = 2u * prm.patch_half + 1u;
                for (uint32_t g = 0; g < grips.size(); ++g) {
                    const uint32_t row = g / width, slot = g % width;
                    const uint32_t ring = (center + prm.ring_count + slot - prm.patch_half) % prm.ring_count;
                    grips[g].particle = cuff[row * prm.ring_count + ring];
                    grips[g].ring = center;
                }
            }
            R maxcap = R(0);
            for (const Grip& g : grips) maxcap = rmax(maxcap, len(x[g.particle] - target));
            if (maxcap > R(prm.capture_radius)) {
                failure |= 1u << 4;
                return;
            }
            for (Grip& g : grips) {
                const V<R> pos = x[g.particle];
                g.offset = inverse_rotate(q, pos - target);
                g.lambda = {};
                g.error = rmax(g.error, len(pos - (target + rotate(q, g.offset))));
                g.capture = rmax(g.capture, len(pos - target));
                g.gen = sub.grip_gen;
            }
            return;
        }
        // Batched: per grip, as the kernel (ClothBag.metal:577-673 semantics).
        for (uint32_t g = 0; g < grips.size(); ++g) {
            Grip& gr = grips[g];
            if (gr.gen == sub.grip_gen) continue;
            if (gr.gen == 0xffffffffu || gr.gen + 1u != sub.grip_gen) {
                failure |= 1u << 4;
                continue;
            }
            uint32_t particle = gr.particle;
            if (sub.grip_select == 1u) {
                uint32_t center = 0;
                R nearest = std::numeric_limits<R>::infinity();
                for (uint32_t ring = 0; ring < prm.ring_count; ++ring) {
                    const R dsq = lsq(x[cuff[prm.ring_count + ring]] - target);
                    if (dsq < nearest) {
                        nearest = dsq;
                        center = ring;
                    }
                }
                const uint32_t width = 2u * prm.patch_half + 1u;
                const uint32_t row = g / width, slot = g % width;
                const uint32_t ring = (center + prm.ring_count + slot - prm.patch_half) % prm.ring_count;
                particle = cuff[row * prm.ring_count + ring];
                gr.particle = particle;
                gr.ring = center;
            }
            const V<R> pos = x[particle];
            const V<R> sep = pos - target;
            const R cap = len(sep);
            if (cap > R(prm.capture_radius)) {
                failure |= 1u << 4;
                continue;
            }
            const V<R> off = inverse_rotate(q, sep);
            const R err = len(pos - (target + rotate(q, off)));
            gr.offset = off;
            gr.gen = sub.grip_gen;
            gr.capture = rmax(gr.capture, cap);
            gr.lambda = {};
            gr.error = rmax(gr.error, err);
        }
    }

    // Compliant vector attachment (tools/cloth_bag.cpp:1630-1647).
    void solve_grips(const OracleSubstep& sub, R dt) {
        if (!sub.grip_active) return;
        const V<R> target0{R(sub.grip_target[0]), R(sub.grip_target[1]), R(sub.grip_target[2])};
        const Q<R> q{R(sub.grip_q[0]), R(sub.grip_q[1]), R(sub.grip_q[2]), R(sub.grip_q[3])};
        for (Grip& g : grips) {
            if (g.gen != sub.grip_gen) continue;
            const uint32_t i = g.particle;
            const R alpha = g.compliance / (dt * dt);
            const R den = w[i] + alpha;
            if (den <= R(0)) continue;
            const V<R> target = target0 + rotate(q, g.offset);
            const V<R> value = x[i] - target;
            const V<R> dl = vdiv(value * R(-1) - g.lambda * alpha, den);
            g.lambda = g.lambda + dl;
            x[i] = x[i] + dl * w[i];
        }
    }

    // -------------------------------------------------------------- fruits
    R inverse_inertia(const Fruit& f) const { return R(2.5) * f.w / (f.radius * f.radius); }

    // tools/cloth_bag.cpp:1897-1919.
    void solve_pair(uint32_t k, R dt) {
        Pair& p = pairs[k];
        Fruit& a = fruits[p.a];
        Fruit& b = fruits[p.b];
        const V<R> diff = b.x - a.x;
        const R L = len(diff);
        const R target = a.radius + b.radius;
        if (L >= target || L < R(1.0e-12)) return;
        const R den = a.w + b.w;
        const R lambda = (target - L) / den;
        const V<R> normal = vdiv(diff, L);
        const V<R> corr = normal * lambda;
        a.x = a.x - corr * a.w;
        b.x = b.x + corr * b.w;
        const R imp = lambda / dt;
        p.wn = p.wn + normal * imp;
        p.ni = p.ni + imp;
    }

    void pair_sweep(R dt, bool serial) {
        if (serial) {
            for (uint32_t k : serial_pairs) solve_pair(k, dt);
        } else {
            for (const BatchInfo& b : pair_b)
                for (uint32_t k = b.first; k < b.first + b.count; ++k) solve_pair(k, dt);
        }
    }

    void apply_fruit_impulse(Fruit& f, V<R> imp, V<R> offset) {
        f.v = f.v + imp * f.w;
        f.omega = f.omega + cross(offset, imp) * inverse_inertia(f);
    }

    // tools/cloth_bag.cpp:1921-1983.
    void pair_friction(uint32_t k, R mu) {
        const Pair& p = pairs[k];
        if (p.ni <= R(0) || lsq(p.wn) < R(1.0e-20)) return;
        Fruit& a = fruits[p.a];
        Fruit& b = fruits[p.b];
        const V<R> normal = normalized(p.wn);
        const V<R> oa = normal * a.radius;
        const V<R> ob = normal * -b.radius;
        const V<R> ca = a.v + cross(a.omega, oa);
        const V<R> cb = b.v + cross(b.omega, ob);
        const V<R> rel = cb - ca;
        const V<R> tv = rel - normal * dot(rel, normal);
        const R slip = len(tv);
        if (slip < R(1.0e-10)) return;
        const V<R> t = vdiv(tv, slip);
        const R den = ((a.w + b.w) + inverse_inertia(a) * lsq(cross(oa, t))) + inverse_inertia(b) * lsq(cross(ob, t));
        if (den <= R(0)) return;
        const R limit = mu * p.ni;
        const R ti = rmin(slip / den, limit);
        if (ti <= R(0)) return;
        const V<R> imp_b = t * -ti;
        apply_fruit_impulse(b, imp_b, ob);
        apply_fruit_impulse(a, imp_b * R(-1), oa);
    }

    // tools/cloth_bag.cpp:1985-2074.
    void ground_friction(Fruit& f, R mu, R rolling) {
        const R ni = f.ground;
        if (ni <= R(0)) return;
        const V<R> offset{R(0), R(0), -f.radius};
        const V<R> n{R(0), R(0), R(1)};
        const V<R> cv = f.v + cross(f.omega, offset);
        const V<R> tv = cv - n * dot(cv, n);
        const R slip = len(tv);
        const R inv_i = inverse_inertia(f);
        if (slip > R(1.0e-10)) {
            const V<R> t = vdiv(tv, slip);
            const R den = f.w + inv_i * lsq(cross(offset, t));
            const R limit = mu * ni;
            const R ti = rmin(slip / den, limit);
            if (ti > R(0)) apply_fruit_impulse(f, t * -ti, offset);
        }
        const V<R> roll{f.omega.x, f.omega.y, R(0)};
        const R rs = len(roll);
        if (ni <= R(0) || rs <= R(1.0e-12) || rolling <= R(0)) return;
        const R required = rs / inv_i;
        const R limit = rolling * f.radius * ni;
        const R ai = rmin(required, limit);
        f.omega = f.omega - roll * (ai * inv_i / rs);
    }

    // tools/cloth_bag.cpp:979-989.
    void integrate_orientation(Fruit& f, R dt) {
        const R aw = R(0), ax = f.omega.x, ay = f.omega.y, az = f.omega.z;
        const R bw = f.q.w, bx = f.q.x, by = f.q.y, bz = f.q.z;
        const R pw = ((aw * bw - ax * bx) - ay * by) - az * bz;
        const R px = ((aw * bx + ax * bw) + ay * bz) - az * by;
        const R py = ((aw * by - ax * bz) + ay * bw) + az * bx;
        const R pz = ((aw * bz + ax * by) - ay * bx) + az * bw;
        const R h = R(0.5) * dt;
        const R qw = bw + pw * h, qx = bx + px * h, qy = by + py * h, qz = bz + pz * h;
        const R m = std::sqrt(((qw * qw + qx * qx) + qy * qy) + qz * qz);
        if (m > R(1.0e-14)) {
            const R s = R(1) / m;
            f.q = {qx * s, qy * s, qz * s, qw * s};
        } else {
            f.q = {R(0), R(0), R(0), R(1)};
        }
    }

    // tools/cloth_bag.cpp:991-1011, 1109-1181.
    void fruit_air(Fruit& f, R dt) {
        const R pi = R(std::numbers::pi);
        const V<R> airv{R(prm.air[0]), R(prm.air[1]), R(prm.air[2])};
        const R rho = R(prm.air_density);
        const V<R> rel = f.v - airv;
        const R frontal = pi * f.radius * f.radius;
        const R tcoef = R(0.5) * rho * R(prm.aero[2]) * frontal;
        const R tatt = R(1) / (R(1) + f.w * tcoef * len(rel) * dt);
        f.v = airv + rel * tatt;
        R r5;
        if constexpr (kF32) {
            const R r2 = f.radius * f.radius;
            r5 = r2 * r2 * f.radius;
        } else {
            r5 = std::pow(f.radius, 5.0);
        }
        const R rcoef = (R(3) * pi * pi / R(8)) * rho * R(prm.aero[3]) * r5;
        const R ratt = R(1) / (R(1) + inverse_inertia(f) * rcoef * len(f.omega) * dt);
        f.omega = f.omega * ratt;
    }

    // ---------------------------------------------------------- fruit/yarn
    // closestPointsOnSegments(p, p, a, b) (tools/cloth_bag.cpp:2751-2824).
    static void point_segment(V<R> p, V<R> a, V<R> b, V<R>& closest, R& weight) {
        const V<R> dir = b - a;
        const R lb = lsq(dir);
        if (lb <= R(1.0e-20)) {
            closest = a;
            weight = R(0);
            return;
        }
        const R proj = dot(dir, p - a);
        weight = rmin(rmax(proj / lb, R(0)), R(1));
        closest = a + dir * weight;
    }

    // applyBallYarnCorrection (tools/cloth_bag.cpp:2863-2953); the fruit
    // displacement is returned in delta rather than applied.
    // direct != nullptr: move that fruit position after every step, as the
    // reference does (serial order); else sum the steps into delta.
    R yarn_correction(V<R>& pa, V<R>& pb, R wa, R wb, R w0, R w1, R wf, V<R> n, R correction, bool ground,
                      V<R>& delta, V<R>* direct = nullptr) {
        const R wt[2] = {w0, w1};
        V<R>* p[2] = {&pa, &pb};
        const R pw[2] = {wa, wb};
        bool active[2] = {false, false};
        if (ground && n.z < R(0)) {
            for (int s = 0; s < 2; ++s) {
                active[s] = wt[s] > R(0) && p[s]->z <= radius + R(1.0e-9);
                if (active[s]) p[s]->z = radius;
            }
        }
        R remaining = correction;
        R total = R(0);
        for (int it = 0; it < 3 && remaining > R(1.0e-14); ++it) {
            V<R> resp[2];
            R den = wf;
            for (int s = 0; s < 2; ++s) {
                resp[s] = n * pw[s];
                if (active[s]) resp[s].z = R(0);
                den = den + dot(n, resp[s]) * wt[s] * wt[s];
            }
            if (den <= R(0)) break;
            const R unconstrained = remaining / den;
            R step = unconstrained;
            if (ground && n.z < R(0)) {
                for (int s = 0; s < 2; ++s) {
                    const R vr = resp[s].z * wt[s];
                    if (active[s] || vr >= R(0)) continue;
                    const R dg = rmax(R(0), p[s]->z - radius);
                    step = rmin(step, dg / -vr);
                }
            }
            if (direct)
                *direct = *direct - n * (wf * step);
            else
                delta = delta - n * (wf * step);
            for (int s = 0; s < 2; ++s) *p[s] = *p[s] + resp[s] * (wt[s] * step);
            total = total + step;
            remaining = rmax(R(0), remaining - den * step);
            if (step >= unconstrained - R(1.0e-14)) break;
            bool activated = false;
            for (int s = 0; s < 2; ++s) {
                if (!active[s] && wt[s] > R(0) && p[s]->z <= radius + R(1.0e-9)) {
                    p[s]->z = radius;
                    active[s] = true;
                    activated = true;
                }
            }
            if (!activated) break;
        }
        return total;
    }

    // solveBallYarn (tools/cloth_bag.cpp:2955-3020) against fruit position X.
    // Returns the multiplier; pa/pb/delta updated.
    R yarn_contact(uint32_t seg, uint32_t f, V<R> X, V<R>& pa, V<R>& pb, bool ground, R dt, V<R>& delta,
                   bool& touched, V<R>* direct = nullptr) {
        const Fruit& fr = fruits[f];
        const R target = fr.radius + radius;
        if (X.x < rmin(pa.x, pb.x) - target || X.x > rmax(pa.x, pb.x) + target || X.y < rmin(pa.y, pb.y) - target ||
            X.y > rmax(pa.y, pb.y) + target || X.z < rmin(pa.z, pb.z) - target || X.z > rmax(pa.z, pb.z) + target)
            return R(0);
        V<R> closest;
        R t;
        point_segment(X, pa, pb, closest, t);
        V<R> sep = closest - X;
        R dist = len(sep);
        if (dist >= target) return R(0);
        if (dist < R(1.0e-12)) {
            const V<R> sd = normalized(pb - pa);
            sep = normalized(cross(sd, std::abs(sd.z) < R(0.9) ? V<R>{R(0), R(0), R(1)} : V<R>{R(1), R(0), R(0)}));
            dist = R(0);
        }
        const V<R> n = normalized(sep);
        const R w0 = R(1) - t;
        const R w1 = t;
        const R corr = target - dist;
        const R lam = yarn_correction(pa, pb, w[di[seg]], w[dj[seg]], w0, w1, fr.w, n, corr, ground, delta, direct);
        touched = true;
        if (lam > R(0)) {
            const R imp = lam / dt;
            YarnRecord& r = yarn[{seg, f}];
            r.wn = r.wn - n * imp;
            r.ni = r.ni + imp;
            r.ws0 = r.ws0 + w0 * imp;
            r.ws1 = r.ws1 + w1 * imp;
            ++yarn_contacts;
        }
        return lam;
    }

    void add_fruit_sum(uint32_t slot, R value) {
        if constexpr (kF32) {
            if (value != R(0)) fix[slot] += std::llrint(static_cast<double>(value) * kFixedScale);
        } else {
            acc[slot] += value;
        }
    }
    R take_fruit_sum(uint32_t slot) {
        if constexpr (kF32) {
            const long long v = fix[slot];
            fix[slot] = 0;
            return static_cast<R>(static_cast<double>(v) * (1.0 / kFixedScale));
        } else {
            const double v = acc[slot];
            acc[slot] = 0.0;
            return v;
        }
    }

    // One present fruit/yarn sweep.
    void yarn_sweep(bool serial, bool ground, R dt) {
        if (fruits.empty()) return;
        if (serial) {
            // tools/cloth_bag.cpp:3141-3176: fruit-major, the fruit moves
            // after every segment.
            for (uint32_t f = 0; f < fruits.size(); ++f)
                for (uint32_t seg = 0; seg < di.size(); ++seg) {
                    if (dkind[seg] == 3u) continue;
                    V<R> pa = x[di[seg]], pb = x[dj[seg]];
                    V<R> delta{};
                    bool touched = false;
                    yarn_contact(seg, f, fruits[f].x, pa, pb, ground, dt, delta, touched, &fruits[f].x);
                    if (touched) {
                        x[di[seg]] = pa;
                        x[dj[seg]] = pb;
                    }
                }
            return;
        }
        std::vector<V<R>> frozen(fruits.size());
        for (uint32_t f = 0; f < fruits.size(); ++f) frozen[f] = fruits[f].x;
        for (const BatchInfo& b : dist_b) {
            for (uint32_t seg = b.first; seg < b.first + b.yarn; ++seg) {
                V<R> pa = x[di[seg]], pb = x[dj[seg]];
                bool changed = false;
                for (uint32_t f = 0; f < fruits.size(); ++f) {
                    V<R> delta{};
                    bool touched = false;
                    yarn_contact(seg, f, frozen[f], pa, pb, ground, dt, delta, touched);
                    changed = changed || touched;
                    if (touched && (delta.x != R(0) || delta.y != R(0) || delta.z != R(0))) {
                        add_fruit_sum(3u * f + 0u, delta.x);
                        add_fruit_sum(3u * f + 1u, delta.y);
                        add_fruit_sum(3u * f + 2u, delta.z);
                    }
                }
                if (changed) {
                    x[di[seg]] = pa;
                    x[dj[seg]] = pb;
                }
            }
        }
        for (uint32_t f = 0; f < fruits.size(); ++f) {
            const R dx = take_fruit_sum(3u * f + 0u);
            const R dy = take_fruit_sum(3u * f + 1u);
            const R dz = take_fruit_sum(3u * f + 2u);
            fruits[f].x = V<R>{fruits[f].x.x + dx, fruits[f].x.y + dy, fruits[f].x.z + dz};
        }
    }

    // solveSweptBallYarn (tools/cloth_bag.cpp:3022-3109), serial order.
    void swept_yarn_serial(bool ground, R dt) {
        for (uint32_t f = 0; f < fruits.size(); ++f) {
            Fruit& fr = fruits[f];
            for (uint32_t seg = 0; seg < di.size(); ++seg) {
                if (dkind[seg] == 3u) continue;
                const uint32_t ia = di[seg], ib = dj[seg];
                const R target = fr.radius + radius;
                R bound = len(fr.x - fr.prev) + len(x[ia] - xp[ia]);
                bound = bound + len(x[ib] - xp[ib]);
                if (bound < R(1.0e-14)) continue;
                auto sample = [&](R time, V<R>& bp, V<R>& sa, V<R>& sb, V<R>& closest, R& weight, R& dist) {
                    bp = fr.prev + (fr.x - fr.prev) * time;
                    sa = xp[ia] + (x[ia] - xp[ia]) * time;
                    sb = xp[ib] + (x[ib] - xp[ib]) * time;
                    point_segment(bp, sa, sb, closest, weight);
                    dist = len(closest - bp);
                };
                R time = R(0);
                V<R> bp, sa, sb, closest;
                R weight, dist;
                sample(R(0), bp, sa, sb, closest, weight, dist);
                bool found = dist <= target + R(1.0e-9);
                if (!found) {
                    for (int it = 0; it < 80; ++it) {
                        sample(time, bp, sa, sb, closest, weight, dist);
                        const R gap = dist - target;
                        if (gap <= R(1.0e-9)) {
                            found = true;
                            break;
                        }
                        const R advance = R(0.9) * gap / bound;
                        if (!std::isfinite(advance) || advance <= R(0) || time + advance >= R(1)) break;
                        time = time + rmax(advance, R(1.0e-10));
                    }
                }
                if (!found || dist < R(1.0e-12)) continue;
                const V<R> n = vdiv(closest - bp, dist);
                const R w0 = R(1) - weight, w1 = weight;
                const V<R> seg_rem = (x[ia] - sa) * w0 + (x[ib] - sb) * w1;
                const V<R> ball_rem = fr.x - bp;
                const R removed = dot(ball_rem - seg_rem, n);
                if (removed <= R(0)) continue;
                V<R> pa = x[ia], pb = x[ib];
                V<R> delta{};
                const R lam = yarn_correction(pa, pb, w[ia], w[ib], w0, w1, fr.w, n, removed, ground, delta, &fr.x);
                x[ia] = pa;
                x[ib] = pb;
                if (lam <= R(0)) continue;
                const R imp = lam / dt;
                YarnRecord& r = yarn[{seg, f}];
                r.wn = r.wn - n * imp;
                r.ni = r.ni + imp;
                r.ws0 = r.ws0 + w0 * imp;
                r.ws1 = r.ws1 + w1 * imp;
                ++yarn_contacts;
            }
        }
    }

    // solveSweptBallYarn in the kernels' batched order: segments of a yarn
    // colour in parallel, fruits (positions and previous positions) frozen
    // over the sweep, each segment visiting the fruits in ascending order,
    // the fruits' displacements summed and applied after the sweep.
    void swept_yarn_batched(bool ground, R dt) {
        if (fruits.empty()) return;
        const uint32_t nf = static_cast<uint32_t>(fruits.size());
        std::vector<V<R>> fx(nf), fp(nf);
        for (uint32_t f = 0; f < nf; ++f) {
            fx[f] = fruits[f].x;
            fp[f] = fruits[f].prev;
        }
        for (const BatchInfo& b : dist_b) {
            for (uint32_t seg = b.first; seg < b.first + b.yarn; ++seg) {
                const uint32_t ia = di[seg], ib = dj[seg];
                V<R> pa = x[ia], pb = x[ib];
                bool changed = false;
                for (uint32_t f = 0; f < nf; ++f) {
                    const Fruit& fr = fruits[f];
                    const R target = fr.radius + radius;
                    R bound = len(fx[f] - fp[f]) + len(pa - xp[ia]);
                    bound = bound + len(pb - xp[ib]);
                    if (bound < R(1.0e-14)) continue;
                    V<R> bp, sa, sb, closest;
                    R weight, dist;
                    auto sample = [&](R time) {
                        bp = fp[f] + (fx[f] - fp[f]) * time;
                        sa = xp[ia] + (pa - xp[ia]) * time;
                        sb = xp[ib] + (pb - xp[ib]) * time;
                        point_segment(bp, sa, sb, closest, weight);
                        dist = len(closest - bp);
                    };
                    R time = R(0);
                    sample(R(0));
                    bool found = dist <= target + R(1.0e-9);
                    if (!found) {
                        for (int it = 0; it < 80; ++it) {
                            sample(time);
                            const R gap = dist - target;
                            if (gap <= R(1.0e-9)) {
                                found = true;
                                break;
                            }
                            const R advance = R(0.9) * gap / bound;
                            if (!std::isfinite(advance) || advance <= R(0) || time + advance >= R(1)) break;
                            time = time + rmax(advance, R(1.0e-10));
                        }
                    }
                    if (!found || dist < R(1.0e-12)) continue;
                    const V<R> n = vdiv(closest - bp, dist);
                    const R w0 = R(1) - weight, w1 = weight;
                    const V<R> seg_rem = (pa - sa) * w0 + (pb - sb) * w1;
                    const V<R> ball_rem = fx[f] - bp;
                    const R removed = dot(ball_rem - seg_rem, n);
                    if (removed <= R(0)) continue;
                    V<R> delta{};
                    const R lam = yarn_correction(pa, pb, w[ia], w[ib], w0, w1, fr.w, n, removed, ground, delta);
                    changed = true;
                    add_fruit_sum(3u * f + 0u, delta.x);
                    add_fruit_sum(3u * f + 1u, delta.y);
                    add_fruit_sum(3u * f + 2u, delta.z);
                    if (lam <= R(0)) continue;
                    const R imp = lam / dt;
                    YarnRecord& r = yarn[{seg, f}];
                    r.wn = r.wn - n * imp;
                    r.ni = r.ni + imp;
                    r.ws0 = r.ws0 + w0 * imp;
                    r.ws1 = r.ws1 + w1 * imp;
                    ++yarn_contacts;
                }
                if (changed) {
                    x[ia] = pa;
                    x[ib] = pb;
                }
            }
        }
        for (uint32_t f = 0; f < nf; ++f) {
            const R dx = take_fruit_sum(3u * f + 0u);
            const R dy = take_fruit_sum(3u * f + 1u);
            const R dz = take_fruit_sum(3u * f + 2u);
            fruits[f].x = V<R>{fruits[f].x.x + dx, fruits[f].x.y + dy, fruits[f].x.z + dz};
        }
    }

    // applyBallYarnFriction (tools/cloth_bag.cpp:3178-3270) for one record.
    void yarn_friction_one(uint32_t seg, uint32_t f, const YarnRecord& r, const Fruit& fr, V<R>& va, V<R>& vb,
                           bool ground, R mu, V<R>& dv, V<R>& dw) {
        const R ni = r.ni;
        if (ni <= R(0) || lsq(r.wn) < R(1.0e-20)) return;
        const V<R> normal = normalized(r.wn);
        R wt[2] = {r.ws0 / ni, r.ws1 / ni};
        const R sum = wt[0] + wt[1];
        if (sum <= R(1.0e-12)) return;
        wt[0] = wt[0] / sum;
        wt[1] = wt[1] / sum;
        const V<R> yv = (V<R>{} + va * wt[0]) + vb * wt[1];
        const V<R> off = normal * -fr.radius;
        const V<R> bcv = fr.v + cross(fr.omega, off);
        const V<R> rel = bcv - yv;
        const V<R> tv = rel - normal * dot(rel, normal);
        const R slip = len(tv);
        if (slip < R(1.0e-10)) return;
        const V<R> t = vdiv(tv, slip);
        const R inv_i = inverse_inertia(fr);
        R den = fr.w + inv_i * lsq(cross(off, t));
        V<R> resp[2];
        const uint32_t idx[2] = {di[seg], dj[seg]};
        for (int s = 0; s < 2; ++s) {
            resp[s] = t * w[idx[s]];
            if (ground && x[idx[s]].z <= radius + R(1.0e-6) && resp[s].z < R(0)) resp[s].z = R(0);
            den = den + dot(t, resp[s]) * wt[s] * wt[s];
        }
        if (den <= R(0)) return;
        const R limit = mu * ni;
        const R ti = rmin(slip / den, limit);
        if (ti <= R(0)) return;
        const V<R> imp = t * -ti;
        dv = imp * fr.w;
        dw = cross(off, imp) * inv_i;
        va = va + resp[0] * (ti * wt[0]);
        vb = vb + resp[1] * (ti * wt[1]);
        (void)f;
    }

    void yarn_friction(bool serial, bool ground, R mu) {
        if (fruits.empty() || yarn.empty()) return;
        if (serial) {
            for (uint32_t f = 0; f < fruits.size(); ++f)
                for (uint32_t seg = 0; seg < di.size(); ++seg) {
                    const auto it = yarn.find({seg, f});
                    if (it == yarn.end()) continue;
                    Fruit& fr = fruits[f];
                    V<R> va = v[di[seg]], vb = v[dj[seg]];
                    V<R> dv{}, dw{};
                    yarn_friction_one(seg, f, it->second, fr, va, vb, ground, mu, dv, dw);
                    fr.v = fr.v + dv;
                    fr.omega = fr.omega + dw;
                    v[di[seg]] = va;
                    v[dj[seg]] = vb;
                }
            return;
        }
        for (const BatchInfo& b : dist_b)
            for (uint32_t seg = b.first; seg < b.first + b.yarn; ++seg) {
                V<R> va = v[di[seg]], vb = v[dj[seg]];
                bool any = false;
                for (uint32_t f = 0; f < fruits.size(); ++f) {
                    const auto it = yarn.find({seg, f});
                    if (it == yarn.end()) continue;
                    any = true;
                    V<R> dv{}, dw{};
                    yarn_friction_one(seg, f, it->second, fruits[f], va, vb, ground, mu, dv, dw);
                    if (dv.x != R(0) || dv.y != R(0) || dv.z != R(0) || dw.x != R(0) || dw.y != R(0) ||
                        dw.z != R(0)) {
                        add_fruit_sum(3u * 64u + 6u * f + 0u, dv.x);
                        add_fruit_sum(3u * 64u + 6u * f + 1u, dv.y);
                        add_fruit_sum(3u * 64u + 6u * f + 2u, dv.z);
                        add_fruit_sum(3u * 64u + 6u * f + 3u, dw.x);
                        add_fruit_sum(3u * 64u + 6u * f + 4u, dw.y);
                        add_fruit_sum(3u * 64u + 6u * f + 5u, dw.z);
                    }
                }
                if (any) {
                    v[di[seg]] = va;
                    v[dj[seg]] = vb;
                }
            }
        for (uint32_t f = 0; f < fruits.size(); ++f) {
            Fruit& fr = fruits[f];
            const R a = take_fruit_sum(3u * 64u + 6u * f + 0u), b2 = take_fruit_sum(3u * 64u + 6u * f + 1u),
                    c = take_fruit_sum(3u * 64u + 6u * f + 2u);
            fr.v = V<R>{fr.v.x + a, fr.v.y + b2, fr.v.z + c};
            const R d = take_fruit_sum(3u * 64u + 6u * f + 3u), e = take_fruit_sum(3u * 64u + 6u * f + 4u),
                    g = take_fruit_sum(3u * 64u + 6u * f + 5u);
            fr.omega = V<R>{fr.omega.x + d, fr.omega.y + e, fr.omega.z + g};
        }
    }

    // ------------------------------------------------------------ self
    bool local_pair(uint32_t a, uint32_t b) const {
        if (!local_off.empty())
            return std::binary_search(local_idx.begin() + local_off[a], local_idx.begin() + local_off[a + 1u], b);
        const uint32_t gw = prm.grid_width;
        if (gw == 0) return a == b;
        const int ra = static_cast<int>(a / gw), ca = static_cast<int>(a % gw);
        const int rb = static_cast<int>(b / gw), cb = static_cast<int>(b % gw);
        return std::abs(ra - rb) <= 2 && std::abs(ca - cb) <= 2;
    }

    static uint64_t spatial_key(int x_, int y_, int z_) {
        constexpr int bias = 1 << 20;
        auto enc = [](int v) { return static_cast<uint64_t>(v + bias) & 0x1fffffu; };
        return enc(x_) | (enc(y_) << 21u) | (enc(z_) << 42u);
    }

    // solveSelfCollision (tools/cloth_bag.cpp:4249-4315), serial order.
    R self_serial() {
        const R target = R(2) * radius;
        const R inv_cell = R(1) / target;
        std::unordered_map<uint64_t, std::vector<uint32_t>> cells;
        const uint32_t n = static_cast<uint32_t>(x.size());
        for (uint32_t i = 0; i < n; ++i)
            cells[spatial_key(static_cast<int>(std::floor(x[i].x * inv_cell)),
                              static_cast<int>(std::floor(x[i].y * inv_cell)),
                              static_cast<int>(std::floor(x[i].z * inv_cell)))]
                .push_back(i);
        R maxpen = R(0);
        for (uint32_t a = 0; a < n; ++a) {
            const int bx = static_cast<int>(std::floor(x[a].x * inv_cell));
            const int by = static_cast<int>(std::floor(x[a].y * inv_cell));
            const int bz = static_cast<int>(std::floor(x[a].z * inv_cell));
            for (int dz = -1; dz <= 1; ++dz)
                for (int dy = -1; dy <= 1; ++dy)
                    for (int dx = -1; dx <= 1; ++dx) {
                        const auto it = cells.find(spatial_key(bx + dx, by + dy, bz + dz));
                        if (it == cells.end()) continue;
                        for (uint32_t b : it->second) {
                            if (b <= a || local_pair(a, b)) continue;
                            const V<R> diff = x[b] - x[a];
                            const R L = len(diff);
                            if (L >= target || L < R(1.0e-12)) continue;
                            const R den = w[a] + w[b];
                            if (den <= R(0)) continue;
                            const V<R> corr = diff * ((target - L) / (L * den));
                            x[a] = x[a] - corr * w[a];
                            x[b] = x[b] + corr * w[b];
                            maxpen = rmax(maxpen, target - L);
                            ++self_contacts;
                        }
                    }
        }
        return maxpen;
    }

    // Point self contact in the kernel's batched order (restates
    // solveSelfCollision, tools/cloth_bag.cpp:4249-4315): every non-local
    // pair closer than 2r at the start of the pass, each particle's
    // corrections summed (2^-40 fixed point in FP32, FP64 sums in FP64) and
    // applied once.
    R self_batched() {
        const R target = R(2) * radius;
        const R inv_cell = R(1) / target;
        const uint32_t n = static_cast<uint32_t>(x.size());
        const std::vector<V<R>> x0 = x;
        std::unordered_map<uint64_t, std::vector<uint32_t>> cells;
        auto cell = [&](const V<R>& p, int k[3]) {
            k[0] = static_cast<int>(std::floor(p.x * inv_cell));
            k[1] = static_cast<int>(std::floor(p.y * inv_cell));
            k[2] = static_cast<int>(std::floor(p.z * inv_cell));
        };
        for (uint32_t i = 0; i < n; ++i) {
            int k[3];
            cell(x0[i], k);
            cells[spatial_key(k[0], k[1], k[2])].push_back(i);
        }
        R maxpen = R(0);
        for (uint32_t a = 0; a < n; ++a) {
            int k[3];
            cell(x0[a], k);
            long long fs[3] = {0, 0, 0};
            double ds[3] = {0.0, 0.0, 0.0};
            std::vector<uint32_t> near;
            for (int dz = -1; dz <= 1; ++dz)
                for (int dy = -1; dy <= 1; ++dy)
                    for (int dx = -1; dx <= 1; ++dx) {
                        const auto it = cells.find(spatial_key(k[0] + dx, k[1] + dy, k[2] + dz));
                        if (it != cells.end()) near.insert(near.end(), it->second.begin(), it->second.end());
                    }
            std::sort(near.begin(), near.end());
            bool touched = false;
            for (uint32_t b : near) {
                if (b == a) continue;
                const V<R> diff = x0[b] - x0[a];
                const R L = len(diff);
                if (L >= target || L < R(1.0e-12)) continue;
                const R den = w[a] + w[b];
                if (den <= R(0)) continue;
                if (local_pair(a, b)) continue;
                const V<R> corr = diff * ((target - L) / (L * den));
                const R c3[3] = {-(corr.x * w[a]), -(corr.y * w[a]), -(corr.z * w[a])};
                for (int e = 0; e < 3; ++e) {
                    if constexpr (kF32)
                        fs[e] += std::llrint(static_cast<double>(c3[e]) * kFixedScale);
                    else
                        ds[e] += static_cast<double>(c3[e]);
                }
                touched = true;
                if (a < b) {
                    ++self_contacts;
                    maxpen = rmax(maxpen, target - L);
                }
            }
            if (!touched) continue;
            if constexpr (kF32) {
                x[a] = V<R>{x[a].x + static_cast<R>(static_cast<double>(fs[0]) * (1.0 / kFixedScale)),
                            x[a].y + static_cast<R>(static_cast<double>(fs[1]) * (1.0 / kFixedScale)),
                            x[a].z + static_cast<R>(static_cast<double>(fs[2]) * (1.0 / kFixedScale))};
            } else {
                x[a] = V<R>{x[a].x + static_cast<R>(ds[0]), x[a].y + static_cast<R>(ds[1]),
                            x[a].z + static_cast<R>(ds[2])};
            }
        }
        return maxpen;
    }

    // ------------------------------------------------------ edge/edge self
    // closestPointsOnSegments (tools/cloth_bag.cpp:2751-2824): closest points
    // cp = p0 + (p1 - p0) s and cq = q0 + (q1 - q0) t.
    static void segment_closest(V<R> p0, V<R> p1, V<R> q0, V<R> q1, V<R>& cp, V<R>& cq, R& s, R& t) {
        const V<R> d1 = p1 - p0, d2 = q1 - q0, off = p0 - q0;
        const R l1 = lsq(d1), l2 = lsq(d2), sp = dot(d2, off);
        const R eps = R(1.0e-20);
        s = R(0);
        t = R(0);
        if (l1 <= eps && l2 <= eps) {
            cp = p0;
            cq = q0;
            return;
        }
        if (l1 <= eps) {
            t = clamp01(sp / l2);
        } else {
            const R fp = dot(d1, off);
            if (l2 <= eps) {
                s = clamp01(-fp / l1);
            } else {
                const R c = dot(d1, d2);
                const R den = l1 * l2 - c * c;
                if (den > eps) s = clamp01((c * sp - fp * l2) / den);
                t = (c * s + sp) / l2;
                if (t < R(0)) {
                    t = R(0);
                    s = clamp01(-fp / l1);
                } else if (t > R(1)) {
                    t = R(1);
                    s = clamp01((c - fp) / l1);
                }
            }
        }
        cp = p0 + d1 * s;
        cq = q0 + d2 * t;
    }

    // selfContactNormal (tools/cloth_bag.cpp:3400-3414).
    static V<R> contact_normal(V<R> sep, V<R> fa, V<R> fb, V<R> prev_off) {
        const R L = len(sep);
        if (L > R(1.0e-12)) return vdiv(sep, L);
        V<R> nrm = normalized(cross(fa, fb));
        if (dot(prev_off, nrm) > R(0)) nrm = nrm * R(-1);
        return nrm;
    }

    struct Box {
        V<R> lo{std::numeric_limits<R>::infinity(), std::numeric_limits<R>::infinity(),
                std::numeric_limits<R>::infinity()};
        V<R> hi{-std::numeric_limits<R>::infinity(), -std::numeric_limits<R>::infinity(),
                -std::numeric_limits<R>::infinity()};
        void add(V<R> p) {   // includePoint (tools/cloth_bag.cpp:3651-3658)
            lo = {rmin(lo.x, p.x), rmin(lo.y, p.y), rmin(lo.z, p.z)};
            hi = {rmax(hi.x, p.x), rmax(hi.y, p.y), rmax(hi.z, p.z)};
        }
        bool overlaps(const Box& o) const {   // overlapBounds (tools/cloth_bag.cpp:3758-3768)
            return lo.x <= o.hi.x && hi.x >= o.lo.x && lo.y <= o.hi.y && hi.y >= o.lo.y && lo.z <= o.hi.z &&
                   hi.z >= o.lo.z;
        }
        R centre(uint32_t axis) const {   // boundsCenterAxis (tools/cloth_bag.cpp:3770-3779)
            return axis == 0u ? R(0.5) * (lo.x + hi.x) : axis == 1u ? R(0.5) * (lo.y + hi.y) : R(0.5) * (lo.z + hi.z);
        }
    };
    struct Sphere {
        V<R> c;
        R r{};
    };

    // edgeBounds (tools/cloth_bag.cpp:3675-3691): the segment (and its
    // substep-start copy when swept) grown by the expansion.
    Box edge_box(uint32_t k, bool swept, R ex) const {
        Box b;
        b.add(x[ya[k]]);
        if (swept) b.add(xp[ya[k]]);
        b.add(x[yb[k]]);
        if (swept) b.add(xp[yb[k]]);
        b.lo = b.lo - V<R>{ex, ex, ex};
        b.hi = b.hi + V<R>{ex, ex, ex};
        return b;
    }

    // edgeCollisionSphere (tools/cloth_bag.cpp:3697-3720).
    Sphere edge_sphere(uint32_t k, bool swept, R ex) const {
        const V<R> pts[4] = {x[ya[k]], x[yb[k]], xp[ya[k]], xp[yb[k]]};
        const uint32_t count = swept ? 4u : 2u;
        V<R> c{};
        for (uint32_t e = 0; e < count; ++e) c = c + pts[e];
        c = vdiv(c, static_cast<R>(count));
        R r = R(0);
        for (uint32_t e = 0; e < count; ++e) r = rmax(r, len(pts[e] - c));
        return {c, r + ex};
    }

    static bool spheres_overlap(const Sphere& a, const Sphere& b) {   // tools/cloth_bag.cpp:3722-3728
        const R r = a.r + b.r;
        return lsq(a.c - b.c) <= r * r;
    }

    bool edge_local(uint32_t i, uint32_t j) const {   // edgePairLocal (tools/cloth_bag.cpp:2740-2749)
        return local_pair(ya[i], ya[j]) || local_pair(ya[i], yb[j]) || local_pair(yb[i], ya[j]) ||
               local_pair(yb[i], yb[j]);
    }

    // Bounding-volume tree over segment boxes (makeCollisionBVH,
    // buildCollisionBVHNode, gatherCollisionCandidates,
    // tools/cloth_bag.cpp:3781-3878): leaves of at most 8 primitives; an
    // inner node orders its primitives by box centre along the longest axis
    // of the centres (ties by index) and splits them at the middle.  A query
    // returns the primitives whose boxes overlap, left subtree first, which
    // is the order of the reference's depth-first stack.
    struct Tree {
        struct Node {
            Box b;
            uint32_t begin, end, left, right;
        };
        std::vector<uint32_t> order;
        std::vector<Node> nodes;
        const std::vector<Box>* boxes = nullptr;

        void build(const std::vector<Box>& bx) {
            boxes = &bx;
            order.resize(bx.size());
            for (uint32_t k = 0; k < bx.size(); ++k) order[k] = k;
            nodes.clear();
            if (!bx.empty()) node(0u, static_cast<uint32_t>(bx.size()));
        }
        uint32_t node(uint32_t begin, uint32_t end) {
            const uint32_t id = static_cast<uint32_t>(nodes.size());
            nodes.push_back({});
            Box all, centres;
            for (uint32_t k = begin; k < end; ++k) {
                const Box& b = (*boxes)[order[k]];
                all.add(b.lo);
                all.add(b.hi);
                centres.add({b.centre(0), b.centre(1), b.centre(2)});
            }
            nodes[id] = {all, begin, end, ~0u, ~0u};
            if (end - begin <= 8u) return id;
            const V<R> e = centres.hi - centres.lo;
            const uint32_t axis = e.y > e.x ? (e.z > e.y ? 2u : 1u) : (e.z > e.x ? 2u : 0u);
            std::sort(order.begin() + begin, order.begin() + end, [&](uint32_t a, uint32_t b) {
                const R ca = (*boxes)[a].centre(axis), cb = (*boxes)[b].centre(axis);
                return ca < cb || (ca == cb && a < b);
            });
            const uint32_t mid = begin + (end - begin) / 2u;
            const uint32_t l = node(begin, mid);
            const uint32_t r = node(mid, end);
            nodes[id].left = l;
            nodes[id].right = r;
            return id;
        }
        void query(const Box& q, std::vector<uint32_t>& out, uint32_t id = 0u) const {
            if (id == 0u) out.clear();
            if (nodes.empty()) return;
            const Node& nd = nodes[id];
            if (!nd.b.overlaps(q)) return;
            if (nd.left == ~0u) {
                for (uint32_t k = nd.begin; k < nd.end; ++k)
                    if ((*boxes)[order[k]].overlaps(q)) out.push_back(order[k]);
                return;
            }
            query(q, out, nd.left);
            query(q, out, nd.right);
        }
    };

    // Add one solve's impulse into the pair's record (tools/cloth_bag.cpp:3962-3985).
    void edge_record(uint32_t i, uint32_t j, const EdgeRecord& local) {
        const uint64_t key = (static_cast<uint64_t>(i) << 32) | j;
        auto [it, inserted] = edge_rec.try_emplace(key);
        EdgeRecord& r = it->second;
        if (inserted) {
            r.a0 = ya[i];
            r.a1 = yb[i];
            r.b0 = ya[j];
            r.b1 = yb[j];
        }
        r.wn = r.wn + local.wn;
        for (int e = 0; e < 2; ++e) {
            r.wf[e] = r.wf[e] + local.wf[e];
            r.ws[e] = r.ws[e] + local.ws[e];
        }
        r.ni = r.ni + local.ni;
    }

    // The impulse of one solve, as the reference's per-solve record
    // (tools/cloth_bag.cpp:3545-3557, 3651-3663).
    static void edge_impulse(EdgeRecord& rec, V<R> nrm, const R fw[2], const R sw[2], R lam, R dt) {
        const R imp = lam / dt;
        rec.wn = rec.wn - nrm * imp;
        for (int e = 0; e < 2; ++e) {
            rec.wf[e] = rec.wf[e] + fw[e] * imp;
            rec.ws[e] = rec.ws[e] + sw[e] * imp;
        }
        rec.ni = rec.ni + imp;
    }

    // solveSweptEdgeEdge (tools/cloth_bag.cpp:3452-3567): conservative
    // advancement of the closest distance from the substep start, then one
    // position correction that takes back the approach after the impact.
    R edge_swept(uint32_t i, uint32_t j, R dt, EdgeRecord* rec) {
        const R target = R(2) * radius;
        const R tol = R(1.0e-9);
        const uint32_t id[4] = {ya[i], yb[i], ya[j], yb[j]};
        R bound = R(0);
        for (uint32_t e = 0; e < 4u; ++e) bound = bound + len(x[id[e]] - xp[id[e]]);
        if (bound < R(1.0e-14)) return R(0);
        V<R> P[4], cp, cq;
        R s = R(0), t = R(0), dist = R(0);
        auto sample = [&](R time) {
            for (uint32_t e = 0; e < 4u; ++e) P[e] = xp[id[e]] + (x[id[e]] - xp[id[e]]) * time;
            segment_closest(P[0], P[1], P[2], P[3], cp, cq, s, t);
            dist = len(cq - cp);
        };
        R time = R(0);
        sample(R(0));
        bool found = dist <= target + tol;
        if (!found) {
            for (uint32_t k = 0; k < 80u; ++k) {
                sample(time);
                const R gap = dist - target;
                if (gap <= tol) {
                    found = true;
                    break;
                }
                const R adv = R(0.9) * gap / bound;
                if (!std::isfinite(adv) || adv <= R(0) || time + adv >= R(1)) break;
                time = time + rmax(adv, R(1.0e-10));
            }
        }
        if (!found) return R(0);
        const R fw[2] = {R(1) - s, s}, sw[2] = {R(1) - t, t};
        const V<R> fprev = xp[id[0]] * fw[0] + xp[id[1]] * fw[1];
        const V<R> sprev = xp[id[2]] * sw[0] + xp[id[3]] * sw[1];
        const V<R> nrm = contact_normal(cq - cp, P[1] - P[0], P[3] - P[2], fprev - sprev);
        V<R> frem{}, srem{};
        for (uint32_t e = 0; e < 2u; ++e) {
            frem = frem + (x[id[e]] - P[e]) * fw[e];
            srem = srem + (x[id[e + 2u]] - P[e + 2u]) * sw[e];
        }
        const R removed = dot(frem - srem, nrm);
        if (removed <= R(0)) return R(0);
        R den = R(0);
        for (uint32_t e = 0; e < 2u; ++e) {
            den = den + w[id[e]] * fw[e] * fw[e];
            den = den + w[id[e + 2u]] * sw[e] * sw[e];
        }
        if (den <= R(0)) return R(0);
        const R lam = removed / den;
        for (uint32_t e = 0; e < 2u; ++e) {
            x[id[e]] = x[id[e]] - nrm * (w[id[e]] * fw[e] * lam);
            x[id[e + 2u]] = x[id[e + 2u]] + nrm * (w[id[e + 2u]] * sw[e] * lam);
        }
        if (rec) edge_impulse(*rec, nrm, fw, sw, lam, dt);
        ++edge_contacts;
        return removed;
    }

    // solveEdgeEdge (tools/cloth_bag.cpp:3569-3640): push two segments
    // closer than the yarn diameter apart at their closest points.
    R edge_present(uint32_t i, uint32_t j, R dt, EdgeRecord* rec) {
        const R target = R(2) * radius;
        const uint32_t id[4] = {ya[i], yb[i], ya[j], yb[j]};
        V<R> cp, cq;
        R s, t;
        segment_closest(x[id[0]], x[id[1]], x[id[2]], x[id[3]], cp, cq, s, t);
        const V<R> sep = cq - cp;
        const R dist = len(sep);
        if (dist >= target) return R(0);
        const R fw[2] = {R(1) - s, s}, sw[2] = {R(1) - t, t};
        const V<R> fprev = xp[id[0]] * fw[0] + xp[id[1]] * fw[1];
        const V<R> sprev = xp[id[2]] * sw[0] + xp[id[3]] * sw[1];
        const V<R> nrm = contact_normal(sep, x[id[1]] - x[id[0]], x[id[3]] - x[id[2]], fprev - sprev);
        R den = R(0);
        for (uint32_t e = 0; e < 2u; ++e) {
            den = den + w[id[e]] * fw[e] * fw[e];
            den = den + w[id[e + 2u]] * sw[e] * sw[e];
        }
        if (den <= R(0)) return target - dist;
        const R lam = (target - dist) / den;
        for (uint32_t e = 0; e < 2u; ++e) {
            x[id[e]] = x[id[e]] - nrm * (w[id[e]] * fw[e] * lam);
            x[id[e + 2u]] = x[id[e + 2u]] + nrm * (w[id[e + 2u]] * sw[e] * lam);
        }
        if (rec) edge_impulse(*rec, nrm, fw, sw, lam, dt);
        ++edge_contacts;
        return target - dist;
    }

    // solvePrimitiveSelfCollision (tools/cloth_bag.cpp:3880-3993), serial
    // order: segment by segment, its candidates in tree order, boxes and
    // spheres of the tree taken at the start of the pass and the query box
    // at the segment's turn.
    R edge_serial(bool swept, R dt, bool ascending = false) {
        const R ex = R(0.5) * (R(2) * radius);
        const uint32_t m = static_cast<uint32_t>(ya.size());
        std::vector<Box> boxes(m);
        std::vector<Sphere> sph(m);
        for (uint32_t k = 0; k < m; ++k) {
            boxes[k] = edge_box(k, swept, ex);
            sph[k] = edge_sphere(k, swept, ex);
        }
        Tree tree;
        tree.build(boxes);
        std::vector<uint32_t> cand;
        R maxc = R(0);
        for (uint32_t i = 0; i < m; ++i) {
            tree.query(edge_box(i, swept, ex), cand);
            if (ascending) std::sort(cand.begin(), cand.end());
            for (uint32_t j : cand) {
                if (j <= i || !spheres_overlap(sph[i], sph[j]) || edge_local(i, j)) continue;
                EdgeRecord local{};
                const R c = swept ? edge_swept(i, j, dt, &local) : edge_present(i, j, dt, &local);
                maxc = rmax(maxc, c);
                if (local.ni > R(0)) edge_record(i, j, local);
            }
        }
        return maxc;
    }

    // measurePrimitiveSelfPenetration (tools/cloth_bag.cpp:4182-4247): the
    // deepest non-local segment pair.  Every pair closer than the yarn
    // diameter passes the box and sphere filters, so the value is the
    // maximum over all non-local pairs (and 0).
    R edge_penetration() const {
        const R target = R(2) * radius;
        const R ex = R(0.5) * target;
        const uint32_t m = static_cast<uint32_t>(ya.size());
        std::vector<Box> boxes(m);
        std::vector<Sphere> sph(m);
        for (uint32_t k = 0; k < m; ++k) {
            boxes[k] = edge_box(k, false, ex);
            sph[k] = edge_sphere(k, false, ex);
        }
        Tree tree;
        tree.build(boxes);
        std::vector<uint32_t> cand;
        R pen = R(0);
        for (uint32_t i = 0; i < m; ++i) {
            tree.query(boxes[i], cand);
            for (uint32_t j : cand) {
                if (j <= i || !spheres_overlap(sph[i], sph[j]) || edge_local(i, j)) continue;
                V<R> cp, cq;
                R s, t;
                segment_closest(x[ya[i]], x[yb[i]], x[ya[j]], x[yb[j]], cp, cq, s, t);
                pen = rmax(pen, target - len(cq - cp));
            }
        }
        return pen;
    }

    // applyClothSelfFriction (tools/cloth_bag.cpp:3995-4090): Coulomb
    // friction on every pair record in key order, at the record's
    // impulse-weighted normal and barycentric weights.
    void edge_friction_serial(R mu) {
        for (const auto& [key, r] : edge_rec) {
            if (r.ni <= R(0) || lsq(r.wn) < R(1.0e-20)) continue;
            const V<R> nrm = normalized(r.wn);
            R fw[2], sw[2];
            R fsum = R(0), ssum = R(0);
            for (int e = 0; e < 2; ++e) {
                fw[e] = r.wf[e] / r.ni;
                sw[e] = r.ws[e] / r.ni;
                fsum = fsum + fw[e];
                ssum = ssum + sw[e];
            }
            if (fsum <= R(1.0e-12) || ssum <= R(1.0e-12)) continue;
            const uint32_t fi[2] = {r.a0, r.a1}, si[2] = {r.b0, r.b1};
            V<R> fv{}, sv{};
            for (int e = 0; e < 2; ++e) {
                fw[e] = fw[e] / fsum;
                sw[e] = sw[e] / ssum;
                fv = fv + v[fi[e]] * fw[e];
                sv = sv + v[si[e]] * sw[e];
            }
            const V<R> rel = fv - sv;
            const V<R> tv = rel - nrm * dot(rel, nrm);
            const R slip = len(tv);
            if (slip < R(1.0e-10)) continue;
            const V<R> tn = vdiv(tv, slip);
            R den = R(0);
            for (int e = 0; e < 2; ++e) {
                den = den + w[fi[e]] * fw[e] * fw[e];
                den = den + w[si[e]] * sw[e] * sw[e];
            }
            if (den <= R(0)) continue;
            const R limit = mu * r.ni;
            const R imp = rmin(slip / den, limit);
            if (imp <= R(0)) continue;
            const V<R> on_first = tn * (-imp);
            for (int e = 0; e < 2; ++e) {
                v[fi[e]] = v[fi[e]] + on_first * (w[fi[e]] * fw[e]);
                v[si[e]] = v[si[e]] - on_first * (w[si[e]] * sw[e]);
            }
            if (limit > R(0)) self_cone = rmax(self_cone, imp / limit);   // tools/cloth_bag.cpp:1462-1474
            ++self_friction_contacts;
        }
    }

    // The kernels' order (restates solvePrimitiveSelfCollision,
    // tools/cloth_bag.cpp:3880-3993): the same Gauss-Seidel sweep with the
    // same pass-start spheres, current query boxes and tree leaf order; a
    // cloth of more than 4,096 yarn segments (the kernels' tree limit) takes
    // a segment's candidates in ascending index order instead.
    R edge_batched(bool swept, R dt) { return edge_serial(swept, dt, ya.size() > 4096u); }
    // applyClothSelfFriction is already in key order, which the kernels keep.
    void edge_friction_batched(R mu) { edge_friction_serial(mu); }

    R edge_pass(bool serial, bool swept, R dt) { return serial ? edge_serial(swept, dt) : edge_batched(swept, dt); }
    void edge_friction(bool serial, R mu) {
        if (serial)
            edge_friction_serial(mu);
        else
            edge_friction_batched(mu);
    }

    // applyClothGroundFriction for one particle (tools/cloth_bag.cpp:2076-2115).
    static void cloth_ground_friction(V<R>& vel, R wi, R gi, R mu) {
        if (gi <= R(0) || wi <= R(0)) return;
        const V<R> tv{vel.x, vel.y, R(0)};
        const R slip = len(tv);
        if (slip < R(1.0e-10)) return;
        const R limit = mu * gi;
        const R ti = rmin(slip / wi, limit);
        if (ti <= R(0)) return;
        vel = vel - tv * (ti * wi / slip);
    }

    // ---------------------------------------------------------- ground
    // tools/cloth_bag.cpp:2655-2690.
    void ground(R dt) {
        for (auto& p : x)
            if (radius - p.z > R(0)) p.z = radius;
        for (Fruit& f : fruits) {
            const R pen = f.radius - f.x.z;
            if (pen > R(0)) {
                f.ground = f.ground + pen / (f.w * dt);
                f.x.z = f.radius;
            }
        }
    }

    // ------------------------------------------------------- residuals
    // FP64 measures (tools/cloth_bag.cpp:1765-1780, 1880-1895, 3111-3139).
    void residuals(bool ground_on, double out[3]) const {
        double strain = 0.0, gpen = 0.0, fpen = 0.0;
        for (uint32_t k = 0; k < di.size(); ++k) {
            if (!(dmax[k] > R(0))) continue;
            const V<R>& a = x[di[k]];
            const V<R>& b = x[dj[k]];
            const double dx = static_cast<double>(b.x) - static_cast<double>(a.x);
            const double dy = static_cast<double>(b.y) - static_cast<double>(a.y);
            const double dz = static_cast<double>(b.z) - static_cast<double>(a.z);
            const double L = std::sqrt((dx * dx + dy * dy) + dz * dz);
            const double maxL = static_cast<double>(drest[k]) * (1.0 + static_cast<double>(dmax[k]));
            strain = std::max(strain, L - maxL);
        }
        if (ground_on) {
            for (const auto& p : x) gpen = std::max(gpen, static_cast<double>(radius) - static_cast<double>(p.z));
            for (const Fruit& f : fruits)
                gpen = std::max(gpen, static_cast<double>(f.radius) - static_cast<double>(f.x.z));
        }
        for (const Fruit& f : fruits) {
            const double X[3] = {static_cast<double>(f.x.x), static_cast<double>(f.x.y), static_cast<double>(f.x.z)};
            const double target = static_cast<double>(f.radius) + static_cast<double>(radius);
            for (uint32_t k = 0; k < di.size(); ++k) {
                if (dkind[k] == 3u) continue;
                const V<R>& pa = x[di[k]];
                const V<R>& pb = x[dj[k]];
                const double A[3] = {static_cast<double>(pa.x), static_cast<double>(pa.y), static_cast<double>(pa.z)};
                const double B[3] = {static_cast<double>(pb.x), static_cast<double>(pb.y), static_cast<double>(pb.z)};
                bool outside = false;
                for (int e = 0; e < 3; ++e)
                    outside = outside || X[e] < std::min(A[e], B[e]) - target || X[e] > std::max(A[e], B[e]) + target;
                if (outside) continue;
                const double dir[3] = {B[0] - A[0], B[1] - A[1], B[2] - A[2]};
                const double lb = (dir[0] * dir[0] + dir[1] * dir[1]) + dir[2] * dir[2];
                double t = 0.0;
                if (lb > 1.0e-20) {
                    const double proj = (dir[0] * (X[0] - A[0]) + dir[1] * (X[1] - A[1])) + dir[2] * (X[2] - A[2]);
                    t = std::clamp(proj / lb, 0.0, 1.0);
                }
                const double cx = A[0] + dir[0] * t - X[0];
                const double cy = A[1] + dir[1] * t - X[1];
                const double cz = A[2] + dir[2] * t - X[2];
                fpen = std::max(fpen, target - std::sqrt((cx * cx + cy * cy) + cz * cz));
            }
        }
        out[0] = strain;
        out[1] = gpen;
        out[2] = fpen;
    }

    bool converged(bool ground_on) const {
        double r[3];
        residuals(ground_on, r);
        return r[2] < 1.0e-6 && r[1] < 1.0e-9 && r[0] < 1.0e-6;
    }

    // ----------------------------------------------------------- air
    // applyYarnAerodynamics (tools/cloth_bag.cpp:1013-1107).
    void yarn_air(bool serial, R dt) {
        const R pi = R(std::numbers::pi);
        const V<R> airv{R(prm.air[0]), R(prm.air[1]), R(prm.air[2])};
        const R rho = R(prm.air_density);
        const uint32_t n = static_cast<uint32_t>(x.size());
        std::fill(force.begin(), force.end(), V<R>{});
        auto segment = [&](uint32_t s) {
            const uint32_t a = di[s], b = dj[s];
            const V<R> span = x[b] - x[a];
            const R L = len(span);
            if (L < R(1.0e-12)) return;
            const V<R> axis = vdiv(span, L);
            const V<R> rel = (v[a] + v[b]) * R(0.5) - airv;
            const V<R> axial = axis * dot(rel, axis);
            const V<R> crossv = rel - axial;
            const R cross_area = R(2) * radius * L;
            const R wet_area = R(2) * pi * radius * L;
            const R ccoef = R(0.5) * rho * R(prm.aero[0]) * cross_area;
            const R scoef = R(0.5) * rho * R(prm.aero[1]) * wet_area;
            V<R> f1{}, f2{};
            const R cs = len(crossv);
            if (!(cs < R(1.0e-14) || ccoef <= R(0))) f1 = crossv * (-ccoef * cs);
            const R as = len(axial);
            if (!(as < R(1.0e-14) || scoef <= R(0))) f2 = axial * (-scoef * as);
            const V<R> f = f1 + f2;
            force[a] = force[a] + f * R(0.5);
            force[b] = force[b] + f * R(0.5);
        };
        if (serial) {
            for (uint32_t s = 0; s < di.size(); ++s)
                if (dkind[s] != 3u) segment(s);
        } else {
            for (const BatchInfo& b : dist_b)
                for (uint32_t s = b.first; s < b.first + b.yarn; ++s) segment(s);
        }
        R att = R(1);
        if constexpr (kF32) {
            // FP64 fixed tree over 256-particle chunks, as the kernel.
            const uint32_t chunks = (n + 255u) / 256u;
            std::vector<double> cp(chunks), cq(chunks);
            for (uint32_t ch = 0; ch < chunks; ++ch) {
                double sp[256], sq[256];
                for (uint32_t t = 0; t < 256u; ++t) {
                    const uint32_t i = ch * 256u + t;
                    double pw = 0.0, q = 0.0;
                    if (i < n && w[i] > R(0)) {
                        const V<R> f = force[i];
                        const V<R> rv = v[i] - airv;
                        pw = static_cast<double>(f.x) * rv.x + static_cast<double>(f.y) * rv.y +
                             static_cast<double>(f.z) * rv.z;
                        q = static_cast<double>(w[i]) * (static_cast<double>(f.x) * f.x +
                                                         static_cast<double>(f.y) * f.y +
                                                         static_cast<double>(f.z) * f.z);
                    }
                    sp[t] = pw;
                    sq[t] = q;
                }
                for (uint32_t st = 128u; st > 0u; st >>= 1u)
                    for (uint32_t t = 0; t < st; ++t) {
                        sp[t] += sp[t + st];
                        sq[t] += sq[t + st];
                    }
                cp[ch] = sp[0];
                cq[ch] = sq[0];
            }
            double sp[256], sq[256];
            for (uint32_t t = 0; t < 256u; ++t) {
                double pw = 0.0, q = 0.0;
                for (uint32_t ch = t; ch < chunks; ch += 256u) {
                    pw += cp[ch];
                    q += cq[ch];
                }
                sp[t] = pw;
                sq[t] = q;
            }
            for (uint32_t st = 128u; st > 0u; st >>= 1u)
                for (uint32_t t = 0; t < st; ++t) {
                    sp[t] += sp[t + st];
                    sq[t] += sq[t + st];
                }
            double a = 1.0;
            if (sq[0] > 0.0) a = sp[0] < 0.0 ? 1.0 / (1.0 + static_cast<double>(dt) * sq[0] / -sp[0]) : 0.0;
            att = static_cast<R>(a);
        } else {
            double power = 0.0, wsq = 0.0;
            for (uint32_t i = 0; i < n; ++i) {
                if (w[i] <= R(0)) continue;
                power += dot(force[i], v[i] - airv);
                wsq += w[i] * lsq(force[i]);
            }
            if (wsq > 0.0) att = power < 0.0 ? 1.0 / (1.0 + dt * wsq / -power) : 0.0;
        }
        for (uint32_t i = 0; i < n; ++i)
            if (w[i] > R(0)) v[i] = v[i] + force[i] * (att * w[i] * dt);
    }

    // ----------------------------------------------------------- release
    // updateReleasedFruit (tools/cloth_bag.cpp:4419-4597).
    void release() {
        const uint32_t m = static_cast<uint32_t>(rim.size());
        if (m < 3u) return;
        std::vector<V<double>> ring(m);
        V<double> center{};
        for (uint32_t k = 0; k < m; ++k) {
            const V<R>& p = x[rim[k]];
            ring[k] = {double(p.x), double(p.y), double(p.z)};
            center = center + ring[k];
        }
        center = vdiv(center, static_cast<double>(m));
        V<double> area{};
        for (uint32_t k = 0; k < m; ++k) area = area + cross(ring[k] - center, ring[(k + 1u) % m] - center);
        if (lsq(area) < 1.0e-16) return;
        V<double> normal = normalized(area);
        const V<R>& bc = x[prm.bottom_center];
        if (dot(normal, center - V<double>{double(bc.x), double(bc.y), double(bc.z)}) < 0.0) normal = normal * -1.0;
        V<double> tangent = ring[0] - center;
        tangent = tangent - normal * dot(tangent, normal);
        if (lsq(tangent) < 1.0e-16)
            tangent = cross(normal, std::abs(normal.z) < 0.9 ? V<double>{0, 0, 1} : V<double>{1, 0, 0});
        tangent = normalized(tangent);
        const V<double> bitangent = normalized(cross(normal, tangent));
        auto inside = [&](V<double> point, double clearance) {
            const V<double> rel = point - center;
            const double px = dot(rel, tangent), py = dot(rel, bitangent);
            bool in = false;
            double best = std::numeric_limits<double>::infinity();
            for (uint32_t a = 0, b = m - 1u; a < m; b = a++) {
                const V<double> ra = ring[a] - center, rb = ring[b] - center;
                const double ax = dot(ra, tangent), ay = dot(ra, bitangent);
                const double bx = dot(rb, tangent), by = dot(rb, bitangent);
                const double ex = bx - ax, ey = by - ay;
                const double el = ex * ex + ey * ey;
                const double fr = el > 1.0e-20 ? std::clamp(((px - ax) * ex + (py - ay) * ey) / el, 0.0, 1.0) : 0.0;
                const double sx = px - (ax + fr * ex), sy = py - (ay + fr * ey);
                best = std::min(best, sx * sx + sy * sy);
                if ((ay > py) != (by > py)) {
                    const double cx = ax + (bx - ax) * (py - ay) / (by - ay);
                    if (px < cx) in = !in;
                }
            }
            return in || best <= clearance * clearance;
        };
        auto rim_distance = [&](V<double> point) {
            double best = std::numeric_limits<double>::infinity();
            for (uint32_t a = 0; a < m; ++a) {
                const V<double> st = ring[a];
                const V<double> e = ring[(a + 1u) % m] - st;
                const double el = lsq(e);
                const double fr = el > 1.0e-20 ? std::clamp(dot(point - st, e) / el, 0.0, 1.0) : 0.0;
                best = std::min(best, lsq(point - (st + e * fr)));
            }
            return std::sqrt(best);
        };
        for (uint32_t f = 0; f < fruits.size(); ++f) {
            const V<double> p{double(fruits[f].x.x), double(fruits[f].x.y), double(fruits[f].x.z)};
            const double need = double(fruits[f].radius) + double(radius);
            const bool in_proj = inside(p, 0.0);
            const bool near_proj = inside(p, need);
            const double out = dot(p - center, normal);
            const uint32_t bit = 1u << f;
            if (in_proj && out > 0.0) candidate_mask |= bit;
            const double axial = out - need;
            const double rim_clear = rim_distance(p) - need;
            const bool cap = near_proj && axial > prm.hysteresis;
            const bool around = (candidate_mask & bit) != 0u && !in_proj && out > 0.0 && rim_clear > prm.hysteresis;
            if (cap || around) released_mask |= bit;
        }
    }

    // ------------------------------------------------------------ substep
    void substep(const OracleSubstep& sub, const OracleSchedule& s, bool last) {
        const bool serial = s.mode == ORACLE_SERIAL;
        const R dt = R(sub.dt);
        const R dt2 = dt * dt;
        const R inv_dt = R(1) / dt;
        const bool ground_on = prm.ground != 0u;
        const V<R> g{R(sub.gravity[0]), R(sub.gravity[1]), R(sub.gravity[2])};
        yarn.clear();
        edge_rec.clear();
        const bool prim = s.primitive_self != 0u;
        grip_attach(sub, serial);
        for (Grip& gr : grips) gr.lambda = {};
        const uint32_t n = static_cast<uint32_t>(x.size());
        const bool air = s.aerodynamics != 0u;
        const R damp = R(s.damping);
        // begin (tools/cloth_bag.cpp:4788-4813)
        for (uint32_t i = 0; i < n; ++i) {
            const V<R> prev = x[i];
            xp[i] = prev;
            if (w[i] == R(0)) {
                x[i] = rest[i];
                v[i] = (x[i] - prev) * inv_dt;
            } else {
                v[i] = v[i] + g * dt;
                if (damp != R(0)) v[i] = v[i] * (R(1) / (R(1) + damp * dt));
            }
        }
        if (air) yarn_air(serial, dt);
        for (uint32_t i = 0; i < n; ++i) {
            vw[i] = v[i].z;
            if (w[i] != R(0)) x[i] = x[i] + v[i] * dt;
        }
        for (Fruit& f : fruits) {
            f.prev = f.x;
            f.v = f.v + g * dt;
            f.ground = R(0);
            if (air) fruit_air(f, dt);
            f.x = f.x + f.v * dt;
        }
        for (Pair& p : pairs) {
            p.wn = {};
            p.ni = R(0);
        }
        if (s.swept_ground && ground_on) {   // sweepGroundPrediction (tools/cloth_bag.cpp:2692-2721)
            for (uint32_t i = 0; i < n; ++i)
                if (xp[i].z >= radius && x[i].z < radius) x[i].z = radius;
            for (Fruit& f : fruits)
                if (f.prev.z >= f.radius && f.x.z < f.radius) {
                    const R adv = f.radius - f.x.z;
                    f.ground = f.ground + adv / (f.w * dt);
                    f.x.z = f.radius;
                }
        }
        std::fill(dlam.begin(), dlam.end(), R(0));
        std::fill(klam.begin(), klam.end(), R(0));
        std::fill(blam.begin(), blam.end(), R(0));
        if (prim) edge_pass(serial, true, dt);
        if (s.swept_fruit_yarn) {
            if (serial)
                swept_yarn_serial(ground_on, dt);
            else
                swept_yarn_batched(ground_on, dt);
        }
        auto sweep_distance = [&] {
            if (serial)
                for (uint32_t k = 0; k < di.size(); ++k) solve_distance(k, dt2);
            else
                for (const BatchInfo& b : dist_b)
                    for (uint32_t k = b.first; k < b.first + b.count; ++k) solve_distance(k, dt2);
        };
        auto sweep_strain = [&] {
            for (uint32_t sw = 0; sw < s.strain_sweeps; ++sw) {
                if (serial)
                    for (uint32_t k = 0; k < di.size(); ++k) limit_strain(k);
                else
                    for (const BatchInfo& b : dist_b)
                        for (uint32_t k = b.first; k < b.first + b.limited; ++k) limit_strain(k);
            }
        };
        for (uint32_t it = 0; it < s.iterations; ++it) {
            sweep_distance();
            if (serial)
                for (uint32_t k = 0; k < kp0.size(); ++k) solve_knot(k, dt2);
            else
                for (const BatchInfo& b : knot_b)
                    for (uint32_t k = b.first; k < b.first + b.count; ++k) solve_knot(k, dt2);
            if ((it & 1u) == 0u) {
                if (serial)
                    for (uint32_t k = 0; k < bp0.size(); ++k) solve_bend(k, dt2, ground_on);
                else
                    for (const BatchInfo& b : bend_b)
                        for (uint32_t k = b.first; k < b.first + b.count; ++k) solve_bend(k, dt2, ground_on);
            }
            solve_grips(sub, dt);
            pair_sweep(dt, serial);
            yarn_sweep(serial, ground_on, dt);
            // point self contact: the kernels' batched pass, or (the
            // reference-order kernels, and the serial order) the reference's
            // Gauss-Seidel pass
            if (s.self_collision) {
                if (serial || s.mode == ORACLE_BATCHED_SELF_REFERENCE)
                    self_serial();
                else
                    self_batched();
            }
            if (ground_on) ground(dt);
        }
        auto contacts = [&](bool with_strain) {
            pair_sweep(dt, serial);
            yarn_sweep(serial, ground_on, dt);
            if (with_strain) sweep_strain();
            if (ground_on) ground(dt);
        };
        uint32_t passes = 0;
        for (uint32_t p = 0; p < s.reconcile_passes; ++p) {
            contacts(true);
            passes = p + 1u;
            if (s.early_exit && converged(ground_on)) break;
        }
        reconcile_max = std::max<uint64_t>(reconcile_max, passes);
        // the endpoint: present edge/edge contacts, then the strain limit
        // (tools/cloth_bag.cpp:5097-5110)
        if (prim) edge_pass(serial, false, dt);
        sweep_strain();
        for (uint32_t p = 0; p < s.final_passes; ++p) contacts(false);
        if (last) {
            uint32_t cert = 0;
            for (uint32_t p = 0; p < s.certificate_passes; ++p) {
                if (prim) edge_pass(serial, false, dt);
                sweep_strain();
                for (uint32_t q = 0; q < s.final_passes; ++q) contacts(false);
                cert = p + 1u;
                if (converged(ground_on) && (!prim || edge_penetration() < R(1.0e-6))) break;
            }
            cert_max = std::max<uint64_t>(cert_max, cert);
        }
        // finalize + cloth/ground friction (tools/cloth_bag.cpp:5186-5211, 2076-2115)
        for (uint32_t i = 0; i < n; ++i) {
            R gi = R(0);
            if (w[i] == R(0)) {
                x[i] = rest[i];
                v[i] = (x[i] - xp[i]) * inv_dt;
            } else {
                v[i] = (x[i] - xp[i]) * inv_dt;
                if (ground_on && x[i].z <= radius + R(1.0e-6)) {
                    const R nvc = v[i].z - vw[i];
                    gi = rmax(R(0), nvc / w[i]);
                }
                if (s.frictions) cloth_ground_friction(v[i], w[i], gi, R(prm.mu_cloth_ground));
            }
            vw[i] = gi;
        }
        for (Fruit& f : fruits) f.v = (f.x - f.prev) * inv_dt;
        if (s.frictions) {
            if (prim) edge_friction(serial, R(prm.mu_self));
            yarn_friction(serial, ground_on, R(prm.mu_fruit_yarn));
            if (serial) {
                for (uint32_t k : serial_pairs) pair_friction(k, R(prm.mu_pair));
            } else {
                for (const BatchInfo& b : pair_b)
                    for (uint32_t k = b.first; k < b.first + b.count; ++k) pair_friction(k, R(prm.mu_pair));
            }
            for (Fruit& f : fruits) ground_friction(f, R(prm.mu_fruit_ground), R(prm.rolling));
        }
        if (s.release) release();
        for (Fruit& f : fruits) integrate_orientation(f, dt);
    }
};

struct Handle {
    int bits;
    Sim<float>* f = nullptr;
    Sim<double>* d = nullptr;
};

template <class R>
void read_state(const Sim<R>& s, OracleParticle* ps, OracleDistance* ds, OracleGrip* gs, OracleFruit* fs,
                OraclePair* prs) {
    if (ps)
        for (size_t i = 0; i < s.x.size(); ++i) {
            OracleParticle& p = ps[i];
            p.x[0] = s.x[i].x; p.x[1] = s.x[i].y; p.x[2] = s.x[i].z;
            p.prev[0] = s.xp[i].x; p.prev[1] = s.xp[i].y; p.prev[2] = s.xp[i].z;
            p.v[0] = s.v[i].x; p.v[1] = s.v[i].y; p.v[2] = s.v[i].z;
            p.rest[0] = s.rest[i].x; p.rest[1] = s.rest[i].y; p.rest[2] = s.rest[i].z;
            p.w = s.w[i]; p.mass = s.mass[i]; p.vw = s.vw[i]; p.pad = 0;
        }
    if (ds)
        for (size_t k = 0; k < s.di.size(); ++k) {
            ds[k] = OracleDistance{s.di[k], s.dj[k], s.dcol[k], s.dkind[k], double(s.drest[k]), double(s.dcomp[k]),
                                   double(s.dlam[k]), double(s.dmax[k])};
        }
    if (gs)
        for (size_t k = 0; k < s.grips.size(); ++k) {
            const auto& g = s.grips[k];
            OracleGrip& o = gs[k];
            o = OracleGrip{};
            o.particle = g.particle; o.gen = g.gen; o.ring = g.ring;
            o.offset[0] = g.offset.x; o.offset[1] = g.offset.y; o.offset[2] = g.offset.z;
            o.compliance = g.compliance;
            o.lambda[0] = g.lambda.x; o.lambda[1] = g.lambda.y; o.lambda[2] = g.lambda.z;
            o.capture = g.capture; o.error = g.error;
        }
    if (fs)
        for (size_t k = 0; k < s.fruits.size(); ++k) {
            const auto& f = s.fruits[k];
            OracleFruit& o = fs[k];
            o = OracleFruit{};
            o.x[0] = f.x.x; o.x[1] = f.x.y; o.x[2] = f.x.z; o.w = f.w;
            o.prev[0] = f.prev.x; o.prev[1] = f.prev.y; o.prev[2] = f.prev.z; o.radius = f.radius;
            o.v[0] = f.v.x; o.v[1] = f.v.y; o.v[2] = f.v.z; o.ground_impulse = f.ground;
            o.omega[0] = f.omega.x; o.omega[1] = f.omega.y; o.omega[2] = f.omega.z;
            o.q[0] = f.q.x; o.q[1] = f.q.y; o.q[2] = f.q.z; o.q[3] = f.q.w;
            o.appearance = f.appearance;
        }
    if (prs)
        for (size_t k = 0; k < s.pairs.size(); ++k) {
            const auto& p = s.pairs[k];
            prs[k] = OraclePair{p.a, p.b, p.colour, 0u, {double(p.wn.x), double(p.wn.y), double(p.wn.z)}, double(p.ni)};
        }
}

template <class R>
void write_state(Sim<R>& s, const OracleParticle* ps, const OracleFruit* fs) {
    if (ps)
        for (size_t i = 0; i < s.x.size(); ++i) {
            const OracleParticle& p = ps[i];
            s.x[i] = {R(p.x[0]), R(p.x[1]), R(p.x[2])};
            s.xp[i] = {R(p.prev[0]), R(p.prev[1]), R(p.prev[2])};
            s.v[i] = {R(p.v[0]), R(p.v[1]), R(p.v[2])};
            s.vw[i] = R(p.vw);
        }
    if (fs)
        for (size_t k = 0; k < s.fruits.size(); ++k) {
            const OracleFruit& f = fs[k];
            auto& o = s.fruits[k];
            o.x = {R(f.x[0]), R(f.x[1]), R(f.x[2])};
            o.prev = {R(f.prev[0]), R(f.prev[1]), R(f.prev[2])};
            o.v = {R(f.v[0]), R(f.v[1]), R(f.v[2])};
            o.omega = {R(f.omega[0]), R(f.omega[1]), R(f.omega[2])};
            o.q = {R(f.q[0]), R(f.q[1]), R(f.q[2]), R(f.q[3])};
            o.ground = R(f.ground_impulse);
        }
}

// The grips' attachment state (particle, generation, patch ring, offset,
// multiplier, capture distance and error), as a reference run left it.
template <class R>
void write_grips(Sim<R>& s, const OracleGrip* gs) {
    for (size_t k = 0; k < s.grips.size(); ++k) {
        const OracleGrip& o = gs[k];
        auto& g = s.grips[k];
        g.particle = o.particle;
        g.gen = o.gen;
        g.ring = o.ring;
        g.offset = {R(o.offset[0]), R(o.offset[1]), R(o.offset[2])};
        g.compliance = R(o.compliance);
        g.lambda = {R(o.lambda[0]), R(o.lambda[1]), R(o.lambda[2])};
        g.capture = R(o.capture);
        g.error = R(o.error);
    }
}

}  // namespace

extern "C" {

void* oracle_create(int bits, const OracleScene* scene) {
    if (!scene || (bits != 32 && bits != 64)) return nullptr;
    auto* h = new Handle{bits};
    bool ok;
    if (bits == 32) {
        h->f = new Sim<float>();
        ok = h->f->init(*scene);
    } else {
        h->d = new Sim<double>();
        ok = h->d->init(*scene);
    }
    if (!ok) {
        delete h->f;
        delete h->d;
        delete h;
        return nullptr;
    }
    return h;
}

void oracle_destroy(void* p) {
    auto* h = static_cast<Handle*>(p);
    if (!h) return;
    delete h->f;
    delete h->d;
    delete h;
}

uint32_t oracle_step(void* p, const OracleSubstep* subs, uint32_t count, const OracleSchedule* schedule) {
    auto* h = static_cast<Handle*>(p);
    if (!h || !subs || !schedule) return 1u << 1;
    for (uint32_t k = 0; k < count; ++k) {
        if (h->f)
            h->f->substep(subs[k], *schedule, k + 1u == count);
        else
            h->d->substep(subs[k], *schedule, k + 1u == count);
    }
    return h->f ? h->f->failure : h->d->failure;
}

void oracle_read(void* p, OracleParticle* ps, OracleDistance* ds, OracleGrip* gs, OracleFruit* fs, OraclePair* prs) {
    auto* h = static_cast<Handle*>(p);
    if (!h) return;
    if (h->f)
        read_state(*h->f, ps, ds, gs, fs, prs);
    else
        read_state(*h->d, ps, ds, gs, fs, prs);
}

void oracle_write(void* p, const OracleParticle* ps, const OracleFruit* fs) {
    auto* h = static_cast<Handle*>(p);
    if (!h) return;
    if (h->f)
        write_state(*h->f, ps, fs);
    else
        write_state(*h->d, ps, fs);
}

void oracle_write_grips(void* p, const OracleGrip* gs) {
    auto* h = static_cast<Handle*>(p);
    if (!h || !gs) return;
    if (h->f)
        write_grips(*h->f, gs);
    else
        write_grips(*h->d, gs);
}

void oracle_residuals(void* p, double out[4]) {
    auto* h = static_cast<Handle*>(p);
    out[3] = 0.0;
    if (h->f)
        h->f->residuals(h->f->prm.ground != 0u, out);
    else
        h->d->residuals(h->d->prm.ground != 0u, out);
}

double oracle_self_pass(void* p, int serial) {
    auto* h = static_cast<Handle*>(p);
    if (h->f) return static_cast<double>(serial ? h->f->self_serial() : h->f->self_batched());
    return serial ? h->d->self_serial() : h->d->self_batched();
}

void oracle_stats(void* p, uint64_t out[8]) {
    auto* h = static_cast<Handle*>(p);
    auto fill = [&](const auto& s) {
        out[0] = s.candidate_mask;
        out[1] = s.released_mask;
        out[2] = s.reconcile_max;
        out[3] = s.cert_max;
        out[4] = s.yarn_contacts;
        out[5] = s.self_contacts;
        out[6] = s.edge_contacts;
        out[7] = s.self_friction_contacts;
    };
    if (h->f)
        fill(*h->f);
    else
        fill(*h->d);
}


// ---------------------------------------------------------------- probes
// Restated known-answer probes of tools/cloth_bag.cpp, driven through the
// oracle's own functions.

// --strain-probe (tools/cloth_bag.cpp:2609-2653): extension 0.285,
// correction 0.215, centre fixed.
int oracle_probe_strain(double out[4]) {
    Sim<double> s;
    s.x = {{-0.75, 0.0, 0.0}, {0.75, 0.0, 0.0}};
    s.w = {1.0, 1.0};
    s.di = {0u}; s.dj = {1u}; s.drest = {1.0}; s.dmax = {0.285};
    const double corr = s.limit_strain(0);
    out[0] = len(s.x[1] - s.x[0]) - 1.0;
    out[1] = corr;
    out[2] = 0.5 * (s.x[0].x + s.x[1].x);
    out[3] = 0.0;
    return std::abs(out[0] - 0.285) < 1e-12 && std::abs(out[1] - 0.215) < 1e-12 && std::abs(out[2]) < 1e-12;
}

// --self-ccd-probe (tools/cloth_bag.cpp:2547-2603): a free segment falls
// through a fixed crossing one in a single step; the swept solve stops it at
// the yarn diameter above (yarn radius 4 mm, the authored material).
int oracle_probe_self_ccd(double out[4]) {
    Sim<double> s;
    s.radius = 0.004;
    s.x = {{-1.0, 0.0, 0.0}, {1.0, 0.0, 0.0}, {0.0, -1.0, -0.02}, {0.0, 1.0, -0.02}};
    s.xp = {{-1.0, 0.0, 0.0}, {1.0, 0.0, 0.0}, {0.0, -1.0, 0.02}, {0.0, 1.0, 0.02}};
    s.w = {0.0, 0.0, 1.0, 1.0};
    s.ya = {0u, 2u};
    s.yb = {1u, 3u};
    const double removed = s.edge_swept(0u, 1u, 1.0, nullptr);
    out[0] = 0.5 * (s.x[2].z + s.x[3].z);
    out[1] = removed;
    out[2] = static_cast<double>(s.edge_contacts);
    out[3] = 0.0;
    return s.edge_contacts == 1u && std::abs(out[0] - 0.008) < 2.0e-9 && out[1] > 0.027;
}

// --self-friction-probe (tools/cloth_bag.cpp:4102-4180): one edge/edge record
// between a segment sliding at 1 m/s and a resting one, normal impulse 10
// (sticks) and 1 (slides), friction 0.34 (the authored material).
int oracle_probe_self_friction(double out[8]) {
    auto run = [](double normal_impulse, double res[4]) {
        Sim<double> s;
        s.v = {{1.0, 0.0, 0.0}, {1.0, 0.0, 0.0}, {}, {}};
        s.w = {1.0, 1.0, 1.0, 1.0};
        Sim<double>::EdgeRecord r{};
        r.a0 = 0u; r.a1 = 1u; r.b0 = 2u; r.b1 = 3u;
        r.wn = {0.0, 0.0, normal_impulse};
        r.wf[0] = r.wf[1] = r.ws[0] = r.ws[1] = normal_impulse / 2.0;
        r.ni = normal_impulse;
        s.edge_rec.emplace(0u, r);
        s.edge_friction_serial(0.34);
        const V<double> fv = vdiv(s.v[0] + s.v[1], 2.0), sv = vdiv(s.v[2] + s.v[3], 2.0);
        double momentum = 0.0, energy = 0.0;
        for (const V<double>& q : s.v) {
            momentum += q.x;
            energy += 0.5 * lsq(q);
        }
        res[0] = len(fv - sv);
        res[1] = momentum;
        res[2] = energy;
        res[3] = s.self_cone;
        return s.self_friction_contacts;
    };
    double stick[4], slide[4];
    const uint64_t c0 = run(10.0, stick), c1 = run(1.0, slide);
    out[0] = stick[0]; out[1] = stick[1]; out[2] = stick[2];
    out[3] = slide[0]; out[4] = slide[1]; out[5] = slide[3];
    out[6] = out[7] = 0.0;
    return stick[0] < 1e-12 && std::abs(stick[1] - 2.0) < 1e-12 && std::abs(stick[2] - 0.5) < 1e-12 &&
           slide[0] > 0.5 && std::abs(slide[1] - 2.0) < 1e-12 && std::abs(slide[3] - 1.0) < 1e-12 && c0 == 1u &&
           c1 == 1u;
}

// --cloth-ground-friction-probe (tools/cloth_bag.cpp:2302-2368): unit
// mass sliding at 1 m/s, mu 0.45; impulses 10 (sticks), 1 (slides to 0.55),
// 0 (unloaded).
int oracle_probe_cloth_ground_friction(double out[4]) {
    const double mu = 0.45;
    V<double> stick{1.0, 0.0, 0.0}, slide{1.0, 0.0, 0.0}, free_{1.0, 0.0, 0.0};
    Sim<double>::cloth_ground_friction(stick, 1.0, 10.0, mu);
    Sim<double>::cloth_ground_friction(slide, 1.0, 1.0, mu);
    Sim<double>::cloth_ground_friction(free_, 1.0, 0.0, mu);
    out[0] = len(stick);
    out[1] = len(slide);
    out[2] = 0.5 * lsq(slide);
    out[3] = len(free_);
    return out[0] < 1e-12 && std::abs(out[1] - 0.55) < 1e-12 && std::abs(out[2] - 0.15125) < 1e-12 &&
           std::abs(out[3] - 1.0) < 1e-12;
}

// --rolling-probe (tools/cloth_bag.cpp:2126-2202): a solid sphere sliding at
// 1 m/s on mu 0.42 ends rolling at 5/7 m/s with energy ratio 5/7.
int oracle_probe_rolling(double out[4]) {
    Sim<double> s;
    Sim<double>::Fruit f{};
    f.radius = 0.07;
    f.w = 1.0 / 0.21;
    f.x = {0.0, 0.0, 0.07};
    f.v = {1.0, 0.0, 0.0};
    f.q = {0.0, 0.0, 0.0, 1.0};
    const double dt = 1.0 / 480.0;
    const double e0 = 0.5 * 0.21 * lsq(f.v);
    for (int k = 0; k < 240; ++k) {
        f.ground = 0.21 * 9.81 * dt;
        s.ground_friction(f, 0.42, 0.0);
        s.integrate_orientation(f, dt);
        f.x = f.x + f.v * dt;
    }
    const V<double> cv = f.v + cross(f.omega, V<double>{0.0, 0.0, -f.radius});
    const double e1 = 0.5 * 0.21 * lsq(f.v) + 0.5 * lsq(f.omega) / s.inverse_inertia(f);
    out[0] = len(f.v);
    out[1] = len(f.omega) * 0.07;
    out[2] = std::hypot(cv.x, cv.y);
    out[3] = e1 / e0;
    const double e = 5.0 / 7.0;
    return std::abs(out[0] - e) < 1e-9 && std::abs(out[1] - e) < 1e-9 && out[2] < 1e-9 && std::abs(out[3] - e) < 1e-9;
}

// --aerodynamics-probe (tools/cloth_bag.cpp:1198-1451), yarn and fruit
// parts: out = coarse force (x, y), refined force (x, y), fruit speed,
// fruit angular speed, yarn energy before, after.
int oracle_probe_aerodynamics(double out[8]) {
    auto yarn = [](std::vector<V<double>> pos, std::vector<double> masses, double dt, V<double>& force) {
        Sim<double> s;
        const size_t n = pos.size();
        s.x = pos; s.v.assign(n, V<double>{3.0, 4.0, 0.0}); s.force.assign(n, V<double>{});
        s.w.resize(n); s.mass = masses;
        for (size_t i = 0; i < n; ++i) s.w[i] = 1.0 / masses[i];
        for (size_t i = 0; i + 1 < n; ++i) {
            s.di.push_back(uint32_t(i)); s.dj.push_back(uint32_t(i + 1)); s.dkind.push_back(0u);
        }
        s.prm = OracleParams{};
        s.prm.air_density = 1.225;
        s.prm.aero[0] = 1.10; s.prm.aero[1] = 0.010;
        s.radius = 0.004;
        V<double> m0{};
        for (size_t i = 0; i < n; ++i) m0 = m0 + s.v[i] * masses[i];
        s.yarn_air(true, dt);
        V<double> m1{};
        double e = 0.0;
        for (size_t i = 0; i < n; ++i) {
            m1 = m1 + s.v[i] * masses[i];
            e += 0.5 * masses[i] * lsq(s.v[i]);
        }
        force = vdiv(m1 - m0, dt);
        return e;
    };
    V<double> coarse, refined;
    const double e1 = yarn({{-0.5, 0, 0}, {0.5, 0, 0}}, {0.5, 0.5}, 0.01, coarse);
    yarn({{-0.5, 0, 0}, {0, 0, 0}, {0.5, 0, 0}}, {0.25, 0.5, 0.25}, 0.01, refined);
    Sim<double> s;
    s.prm = OracleParams{};
    s.prm.air_density = 1.225;
    s.prm.aero[2] = 0.47; s.prm.aero[3] = 0.010;
    Sim<double>::Fruit f{};
    f.radius = 0.10; f.w = 1.0; f.v = {5.0, 0.0, 0.0}; f.omega = {0.0, 0.0, 10.0};
    s.fruit_air(f, 0.01);
    out[0] = coarse.x; out[1] = coarse.y; out[2] = refined.x; out[3] = refined.y;
    out[4] = len(f.v); out[5] = len(f.omega);
    out[6] = 0.5 * 1.0 * 25.0; out[7] = e1;
    return 1;
}

}  // extern "C"
