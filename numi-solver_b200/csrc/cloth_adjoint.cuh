// Reverse-mode adjoint of the cloth substep (no reference counterpart: the
// reference calibrates with external finite-difference sensitivities,
// docs/CLOTH_SPECIMEN_CALIBRATION.md:52-82).
//
// The forward runs a segment of substeps on one CTA and records a tape: the
// positions at the start of every substep and after every phase barrier,
// and the velocities at the start of every substep.  This kernel walks the
// segment's substeps and each substep's phases in reverse and applies the
// vector-Jacobian product of every projection.  Branch decisions are
// recomputed in FP32 from the tape exactly as the forward made them; the
// derivatives are evaluated in FP64 at the FP32 state, and adjoints and
// parameter gradients are accumulated in FP64.
//
// Differentiated: predict with gravity and damping, the swept ground clamp,
// XPBD distance / shear / knot / bend projections (one iteration, so lambda
// starts at zero), the bend's ground active set, step fraction and ground
// clamp, compliant grips, the ground clamp, unilateral strain limits,
// finalize with cloth/ground Coulomb friction (sticking and sliding).  Each
// is piecewise smooth: the pieces the forward took are recomputed in FP32
// and differentiated exactly.  Fruit/yarn contact and its friction move
// the cloth through the fruits' rigid-body state, which the adjoint does not
// carry; where they change the cloth the event is counted in `nonsmooth` and
// passed through as the identity.
#pragma once

#include "cloth_kernels.cuh"

enum AdjointPhase : uint32_t {
    ADJ_KNOT = 10,
    ADJ_BEGIN = 0,
    ADJ_DIST = 1,
    ADJ_BEND = 2,
    ADJ_GRIP = 3,
    ADJ_YARN = 4,
    ADJ_GROUND = 5,
    ADJ_STRAIN = 6,
    ADJ_FINAL = 7,
    ADJ_TAIL = 9,
};

// Gradients: d loss / d log-scale of each compliance group (the distinct
// compliance values of each constraint family, numbered by the host), then
// d loss / d damping.
#define ADJ_MAX_GROUPS 16u

struct AdjointArgs {
    const DeviceCloth* cloth;        // device copy of the handle's descriptor
    const NumiClothConfig* cfg;      // the segment's Configs
    const float4* tape;              // [substeps][slots][n]
    const float4* tape_v;            // [substeps][n]
    const uint2* phases;             // [slots - 1] (type, batch) per barrier
    uint32_t slots;
    uint32_t substeps;               // substeps of the segment
    uint32_t first_substep;          // rollout index of the segment's first substep
    float damping;                   // the schedule's (or the cloth's) damping
    uint32_t frictions;              // the schedule's frictions switch
    const uint32_t* tracked;         // [n_tracked]
    uint32_t n_tracked;
    const double* targets;           // [losses][n_tracked][3]
    uint32_t loss_every;             // loss after substeps s with (s + 1) % loss_every == 0
    double4* gx;                     // [n] adjoint of positions (xyz; w unused)
    double4* gv;                     // [n] adjoint of velocities
    double4* gprev;                  // [n] scratch: adjoint of the substep's start positions via finalize
    const uint8_t* d_group;          // [distances] compliance group
    const uint8_t* k_group;          // [knots]
    const uint8_t* b_group;          // [bends]
    const uint8_t* g_group;          // [grips]
    uint32_t groups;
    double* grads;                   // [groups + 1] accumulated (groups, then damping)
    double* grip_grads;              // [rollout substeps][6] or null
    double* loss;                    // [1] accumulated
    unsigned int* nonsmooth;         // [1] count of non-smooth events met
};

namespace adj {

struct D3v {
    double x, y, z;
};
__device__ __forceinline__ D3v d3(const double4& a) { return D3v{a.x, a.y, a.z}; }
__device__ __forceinline__ D3v d3f(const V3& a) { return D3v{a.x, a.y, a.z}; }
__device__ __forceinline__ D3v d4f(const float4& a) { return D3v{a.x, a.y, a.z}; }
__device__ __forceinline__ double dotd(D3v a, D3v b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ D3v addd(D3v a, D3v b) { return D3v{a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ D3v subd(D3v a, D3v b) { return D3v{a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ D3v muld(D3v a, double s) { return D3v{a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ D3v crossd(D3v a, D3v b) {
    return D3v{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ void put(double4* g, uint32_t i, D3v v) { g[i] = make_double4(v.x, v.y, v.z, 0.0); }

// VJP of x_a' = x_a - w_a dl n, x_b' = x_b + w_b dl n with
// dl = -(L - rest) / (w_a + w_b + alpha) (lambda from zero), n = (x_b - x_a)/L,
// at the FP32 state a, b (derivatives in FP64).  Returns d loss / d alpha.
__device__ __forceinline__ double distance_vjp(double4* gx, uint32_t ia, uint32_t ib, const float4& a, const float4& b,
                                               double rest, double alpha) {
    const D3v dd = subd(d4f(b), d4f(a));
    const double L = sqrt(dotd(dd, dd));
    const D3v n = muld(dd, 1.0 / L);
    const double den = (static_cast<double>(a.w) + b.w) + alpha;
    const double dl = -(L - rest) / den;
    const D3v ga = d3(gx[ia]), gb = d3(gx[ib]);
    const D3v u = subd(muld(gb, b.w), muld(ga, a.w));
    const double un = dotd(u, n);
    const D3v gd = addd(muld(n, -un / den), muld(subd(u, muld(n, un)), dl / L));
    put(gx, ia, subd(ga, gd));
    put(gx, ib, addd(gb, gd));
    return -un * dl / den;
}

// Forward-mode dual number (value, one tangent) for the knot projection,
// whose Jacobian involves the derivatives of its own gradients.
struct Dual {
    double v, d;
};
__device__ __forceinline__ Dual operator+(Dual a, Dual b) { return Dual{a.v + b.v, a.d + b.d}; }
__device__ __forceinline__ Dual operator-(Dual a, Dual b) { return Dual{a.v - b.v, a.d - b.d}; }
__device__ __forceinline__ Dual operator*(Dual a, Dual b) { return Dual{a.v * b.v, a.d * b.v + a.v * b.d}; }
__device__ __forceinline__ Dual operator/(Dual a, Dual b) {
    return Dual{a.v / b.v, (a.d * b.v - a.v * b.d) / (b.v * b.v)};
}
__device__ __forceinline__ Dual dsqrt(Dual a) {
    const double r = sqrt(a.v);
    return Dual{r, a.d / (2.0 * r)};
}
struct DV {
    Dual x, y, z;
};
__device__ __forceinline__ DV operator-(DV a, DV b) { return DV{a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ DV operator*(DV a, Dual s) { return DV{a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ Dual ddot(DV a, DV b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }

// Knot projection (nc::solve_knot with lambda from zero) on dual numbers:
// positions p[4], inverse masses w[4], compliance alpha; writes out[4].
__device__ __forceinline__ void knot_dual(const DV p[4], const double w[4], Dual alpha, double rest, DV out[4]) {
    const DV warpv = p[1] - p[0];
    const DV weftv = p[3] - p[2];
    const Dual wl = dsqrt(ddot(warpv, warpv));
    const Dual fl = dsqrt(ddot(weftv, weftv));
    const Dual one{1.0, 0.0};
    const DV warp = warpv * (one / wl);
    const DV weft = weftv * (one / fl);
    Dual cosine = ddot(warp, weft);
    if (cosine.v > 1.0) cosine = Dual{1.0, 0.0};
    if (cosine.v < -1.0) cosine = Dual{-1.0, 0.0};
    const Dual value = cosine - Dual{rest, 0.0};
    const DV gw = (weft - warp * cosine) * (one / wl);
    const DV gf = (warp - weft * cosine) * (one / fl);
    const Dual W[4] = {{w[0], 0.0}, {w[1], 0.0}, {w[2], 0.0}, {w[3], 0.0}};
    const Dual den = alpha + W[0] * ddot(gw, gw) + W[1] * ddot(gw, gw) + W[2] * ddot(gf, gf) + W[3] * ddot(gf, gf);
    const Dual dl = Dual{0.0, 0.0} - value / den;
    const Dual zero{0.0, 0.0};
    const DV g[4] = {DV{zero, zero, zero} - gw, gw, DV{zero, zero, zero} - gf, gf};
    for (int q = 0; q < 4; ++q) {
        const Dual s = W[q] * dl;
        out[q] = DV{p[q].x + g[q].x * s, p[q].y + g[q].y * s, p[q].z + g[q].z * s};
    }
}

// Branches the forward bend projection took (nc::bend_core): active[s]
// when the ground holds particle s's normal motion; frac_src the particle
// whose ground distance limits the step (-1: none, fraction 1), frac_zero
// when that distance is zero; clamp[s] when the new position is lifted back
// to the ground.
struct BendBranches {
    bool active[2];
    int frac_src;
    bool frac_zero;
    bool clamp[2];
};

// The forward's FP32 decisions for one bend with lambda from zero; false
// when the forward leaves the pair unchanged.
__device__ __forceinline__ bool bend_branches(const float4& p0, const float4& p2, const float2& m, float dt2,
                                              float radius, bool ground, BendBranches& b) {
    const float4 p[2] = {p0, p2};
    const V3 diff = xyz(p2) - xyz(p0);
    const float chord = len3(diff);
    if (chord < 1.0e-12f) return false;
    const float value = chord - m.x;
    const V3 dir = vdiv(diff, chord);
    const V3 g[2] = {dir * -1.0f, dir};
    const float alpha = m.y / dt2;
    float free_den = alpha;
    free_den = free_den + p[0].w * lsq(g[0]);
    free_den = free_den + p[1].w * lsq(g[1]);
    if (free_den < 1.0e-16f) return false;
    const float lam = 0.0f;
    const float numerator = -value - alpha * lam;
    const float free_dl = numerator / free_den;
    float den = alpha;
    for (int s = 0; s < 2; ++s) {
        b.active[s] = ground && p[s].z <= radius + 1.0e-9f && g[s].z * free_dl < 0.0f;
        den = den + p[s].w * (lsq(g[s]) - (b.active[s] ? g[s].z * g[s].z : 0.0f));
    }
    if (den < 1.0e-16f) return false;
    const float dl = numerator / den;
    float fraction = 1.0f;
    b.frac_src = -1;
    b.frac_zero = false;
    if (ground) {
        for (int s = 0; s < 2; ++s) {
            if (b.active[s]) continue;
            const float vc = g[s].z * p[s].w * dl;
            if (vc >= 0.0f) continue;
            const float cand = fmaxf(0.0f, p[s].z - radius) / -vc;
            if (cand < fraction) {
                fraction = cand;
                b.frac_src = s;
                b.frac_zero = !(p[s].z - radius > 0.0f);
            }
        }
    }
    const float applied = dl * fraction;
    for (int s = 0; s < 2; ++s) {
        V3 corr = g[s] * (p[s].w * applied);
        if (b.active[s]) corr.z = 0.0f;
        const V3 np = xyz(p[s]) + corr;
        b.clamp[s] = ground && np.z < radius;
    }
    return true;
}

// The bend projection on dual numbers along the forward's branches:
// positions p[2] (the pair's ends), inverse masses w[2], compliance alpha
// (over dt^2); writes out[2].
__device__ __forceinline__ void bend_dual(const DV p[2], const double w[2], Dual alpha, double rest, double radius,
                                          const BendBranches& b, DV out[2]) {
    const Dual zero{0.0, 0.0};
    const Dual one{1.0, 0.0};
    const DV diff = p[1] - p[0];
    const Dual chord = dsqrt(ddot(diff, diff));
    const Dual value = chord - Dual{rest, 0.0};
    const DV dir = diff * (one / chord);
    const DV g[2] = {DV{zero, zero, zero} - dir, dir};
    const Dual numerator = zero - value;
    Dual den = alpha;
    for (int s = 0; s < 2; ++s)
        den = den + Dual{w[s], 0.0} * (ddot(g[s], g[s]) - (b.active[s] ? g[s].z * g[s].z : zero));
    const Dual dl = numerator / den;
    Dual fraction = one;
    if (b.frac_src >= 0) {
        const int s = b.frac_src;
        if (b.frac_zero) {
            fraction = zero;
        } else {
            const Dual vc = g[s].z * Dual{w[s], 0.0} * dl;
            fraction = (p[s].z - Dual{radius, 0.0}) / (zero - vc);
        }
    }
    const Dual applied = dl * fraction;
    for (int s = 0; s < 2; ++s) {
        const Dual k = Dual{w[s], 0.0} * applied;
        DV np{p[s].x + g[s].x * k, p[s].y + g[s].y * k, p[s].z + (b.active[s] ? zero : g[s].z * k)};
        if (b.clamp[s]) np.z = Dual{radius, 0.0};
        out[s] = np;
    }
}

}  // namespace adj

__device__ __forceinline__ void adjoint_segment(const AdjointArgs& A) {
    using namespace adj;
    const DeviceCloth& d = *A.cloth;
    const uint32_t n = d.n;
    double acc[ADJ_MAX_GROUPS + 1u];
    for (uint32_t e = 0; e <= ADJ_MAX_GROUPS; ++e) acc[e] = 0.0;
    const uint32_t damp_slot = A.groups;
    double loss = 0.0;
    unsigned int rough = 0u;
    __shared__ double s_grip[NC_MAX_GRIPS][6];
    for (uint32_t si = A.substeps; si-- > 0u;) {
        const NumiClothConfig& cf = A.cfg[si];
        const float dt = cf.gravityAndTimestep.w;
        const float dt2 = dt * dt;
        const double dtd = dt;
        const float radius = cf.clothMaterial.x;
        const bool ground = cf.constraintCounts.z != 0u;
        const float4* T = A.tape + static_cast<size_t>(si) * A.slots * n;
        const uint32_t step = A.first_substep + si;
        // loss seed at the end of the substep
        if (A.loss_every != 0u && (step + 1u) % A.loss_every == 0u) {
            const uint32_t li = (step + 1u) / A.loss_every - 1u;
            const float4* xe = T + static_cast<size_t>(A.slots - 1u) * n;
            for (uint32_t t = threadIdx.x; t < A.n_tracked; t += blockDim.x) {
                const uint32_t i = A.tracked[t];
                const double* tg = A.targets + (static_cast<size_t>(li) * A.n_tracked + t) * 3u;
                const D3v diff{static_cast<double>(xe[i].x) - tg[0], static_cast<double>(xe[i].y) - tg[1],
                               static_cast<double>(xe[i].z) - tg[2]};
                loss += dotd(diff, diff);
                put(A.gx, i, addd(d3(A.gx[i]), muld(diff, 2.0)));
            }
            __syncthreads();
        }
        for (uint32_t b = A.slots - 1u; b-- > 0u;) {
            const uint2 ph = A.phases[b];
            const float4* pre = T + static_cast<size_t>(b) * n;     // positions before the phase
            const float4* post = pre + n;                            // after its barrier
            switch (ph.x) {
            case ADJ_TAIL:
                break;
            case ADJ_YARN:
                // fruit/yarn contact moved the cloth: not differentiated
                for (uint32_t i = threadIdx.x; i < n; i += blockDim.x)
                    if (pre[i].x != post[i].x || pre[i].y != post[i].y || pre[i].z != post[i].z) ++rough;
                break;
            case ADJ_FINAL: {
                // v_end = (x - x_start) / dt, then the cloth/ground Coulomb
                // friction of a grounded particle (nc::finalize_particle):
                // with normal impulse gi = (v_end.z - v_pred.z) / w, sticking
                // (|v_t| / w <= mu gi) zeroes the tangential velocity and
                // sliding removes mu (v_end.z - v_pred.z) along the slip.
                // The adjoint of the predicted normal velocity goes to
                // gprev.w for the predict step.
                const float4* xs = T;
                const float4* vs = A.tape_v + static_cast<size_t>(si) * n;
                const float inv_dt = 1.0f / dt;
                const float mu = cf.clothMaterial.z;
                for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
                    if (pre[i].w == 0.0f) {
                        A.gx[i] = make_double4(0, 0, 0, 0);
                        A.gv[i] = make_double4(0, 0, 0, 0);
                        A.gprev[i] = make_double4(0, 0, 0, 0);
                        continue;
                    }
                    D3v gvv = d3(A.gv[i]);
                    double gvpz = 0.0;
                    if (ground && A.frictions != 0u && pre[i].z <= radius + 1.0e-6f) {
                        // the forward's decisions, in FP32
                        const float w = pre[i].w;
                        const V3 vel = (xyz(pre[i]) - xyz(xs[i])) * inv_dt;
                        float vpz = vs[i].z + cf.gravityAndTimestep.z * dt;
                        if (A.damping != 0.0f) vpz = vpz * (1.0f / (1.0f + A.damping * dt));
                        const float gi = fmaxf(0.0f, (vel.z - vpz) / w);
                        const V3 tv{vel.x, vel.y, 0.0f};
                        const float slip = len3(tv);
                        if (gi > 0.0f && !(slip < 1.0e-10f) && fminf(slip / w, mu * gi) > 0.0f) {
                            if (slip / w <= mu * gi) {
                                gvv.x = 0.0;   // sticking
                                gvv.y = 0.0;
                            } else {
                                // sliding: v_t' = v_t - phi v_t / |v_t|, phi = mu (v.z - v_pred.z)
                                const D3v vd = muld(subd(d4f(pre[i]), d4f(xs[i])), 1.0 / dtd);
                                double vpd = static_cast<double>(vs[i].z) + static_cast<double>(cf.gravityAndTimestep.z) * dtd;
                                if (A.damping != 0.0f) vpd /= 1.0 + static_cast<double>(A.damping) * dtd;
                                const double sl = sqrt(vd.x * vd.x + vd.y * vd.y);
                                const double nx = vd.x / sl, ny = vd.y / sl;
                                const double phi = static_cast<double>(mu) * (vd.z - vpd);
                                const double gn = gvv.x * nx + gvv.y * ny;
                                const double gtx = gvv.x - phi / sl * (gvv.x - nx * gn);
                                const double gty = gvv.y - phi / sl * (gvv.y - ny * gn);
                                const double gphi = -gn;
                                gvv = D3v{gtx, gty, gvv.z + static_cast<double>(mu) * gphi};
                                gvpz = -static_cast<double>(mu) * gphi;
                            }
                        }
                    }
                    put(A.gx, i, addd(d3(A.gx[i]), muld(gvv, 1.0 / dtd)));
                    const D3v gp = muld(gvv, -1.0 / dtd);
                    A.gprev[i] = make_double4(gp.x, gp.y, gp.z, gvpz);
                    A.gv[i] = make_double4(0, 0, 0, 0);
                }
                break;
            }
            case ADJ_STRAIN:
            case ADJ_DIST: {
                const Batch bt = d.dist_batches[ph.y];
                const uint32_t count = ph.x == ADJ_STRAIN ? bt.limited : bt.count;
                for (uint32_t r = threadIdx.x; r < count; r += blockDim.x) {
                    const uint32_t k = bt.first + r;
                    const uint2 ij = d.d_ij[k];
                    const float4 m = d.d_mat[k];
                    const float4 a = pre[ij.x], bb = pre[ij.y];
                    const V3 diff = xyz(bb) - xyz(a);
                    const float L = len3(diff);
                    if (ph.x == ADJ_STRAIN) {
                        if (!(m.w > 0.0f)) continue;
                        const float maxL = m.x * (1.0f + m.w);
                        if (L <= maxL || L < 1.0e-12f) continue;
                        if (a.w + bb.w <= 0.0f) continue;
                        // x_a += dir w_a (L - maxL)/den: the distance form with rest maxL, alpha 0
                        distance_vjp(A.gx, ij.x, ij.y, a, bb, static_cast<double>(maxL), 0.0);
                    } else {
                        if (L < 1.0e-12f) continue;
                        const float alpha = m.y / dt2;
                        if ((a.w + bb.w) + alpha <= 0.0f) continue;
                        const double alphad = static_cast<double>(m.y) / (dtd * dtd);
                        const double galpha =
                            distance_vjp(A.gx, ij.x, ij.y, a, bb, static_cast<double>(m.x), alphad);
                        acc[A.d_group[k]] += galpha * alphad;
                    }
                }
                break;
            }
            case ADJ_KNOT: {
                const Batch bt = d.knot_batches[ph.y];
                for (uint32_t r = threadIdx.x; r < bt.count; r += blockDim.x) {
                    const uint32_t k = bt.first + r;
                    const uint4 q = d.k_ij[k];
                    const float2 m = d.k_mat[k];
                    const uint32_t idx[4] = {q.x, q.y, q.z, q.w};
                    float4 p[4];
                    for (int e = 0; e < 4; ++e) p[e] = pre[idx[e]];
                    // the forward's own skip tests, in FP32
                    const float wl = len3(xyz(p[1]) - xyz(p[0]));
                    const float fl = len3(xyz(p[3]) - xyz(p[2]));
                    if (wl < 1.0e-12f || fl < 1.0e-12f) continue;
                    const V3 warp = vdiv(xyz(p[1]) - xyz(p[0]), wl);
                    const V3 weft = vdiv(xyz(p[3]) - xyz(p[2]), fl);
                    const float cosine = fminf(fmaxf(dot3(warp, weft), -1.0f), 1.0f);
                    const V3 gw = vdiv(weft - warp * cosine, wl);
                    const V3 gf = vdiv(warp - weft * cosine, fl);
                    const float alpha = m.y / dt2;
                    float den = alpha;
                    den = den + p[0].w * lsq(gw * -1.0f);
                    den = den + p[1].w * lsq(gw);
                    den = den + p[2].w * lsq(gf * -1.0f);
                    den = den + p[3].w * lsq(gf);
                    if (den <= 0.0f) continue;
                    // VJP by forward mode: one tangent per input (12 coordinates, alpha)
                    double u[12];
                    for (int e = 0; e < 4; ++e) {
                        const double4 ge = A.gx[idx[e]];
                        u[3 * e] = ge.x;
                        u[3 * e + 1] = ge.y;
                        u[3 * e + 2] = ge.z;
                    }
                    const double w[4] = {p[0].w, p[1].w, p[2].w, p[3].w};
                    const double alphad = static_cast<double>(m.y) / (dtd * dtd);
                    double gin[13];
                    for (int dir = 0; dir < 13; ++dir) {
                        DV pd[4];
                        for (int e = 0; e < 4; ++e) {
                            pd[e] = DV{Dual{p[e].x, dir == 3 * e ? 1.0 : 0.0}, Dual{p[e].y, dir == 3 * e + 1 ? 1.0 : 0.0},
                                       Dual{p[e].z, dir == 3 * e + 2 ? 1.0 : 0.0}};
                        }
                        DV out[4];
                        knot_dual(pd, w, Dual{alphad, dir == 12 ? 1.0 : 0.0}, static_cast<double>(m.x), out);
                        double acc_dir = 0.0;
                        for (int e = 0; e < 4; ++e)
                            acc_dir += u[3 * e] * out[e].x.d + u[3 * e + 1] * out[e].y.d + u[3 * e + 2] * out[e].z.d;
                        gin[dir] = acc_dir;
                    }
                    for (int e = 0; e < 4; ++e)
                        A.gx[idx[e]] = make_double4(gin[3 * e], gin[3 * e + 1], gin[3 * e + 2], 0.0);
                    acc[A.k_group[k]] += gin[12] * alphad;
                }
                break;
            }
            case ADJ_BEND: {
                const Batch bt = d.bend_batches[ph.y];
                for (uint32_t r = threadIdx.x; r < bt.count; r += blockDim.x) {
                    const uint32_t k = bt.first + r;
                    const uint4 q = d.b_ij[k];
                    const float2 m = d.b_mat[k];
                    const float4 p0 = pre[q.x], p2 = pre[q.z];
                    BendBranches br;
                    if (!bend_branches(p0, p2, m, dt2, radius, ground, br)) continue;
                    const double alphad = static_cast<double>(m.y) / (dtd * dtd);
                    if (!br.active[0] && !br.active[1] && br.frac_src < 0 && !br.clamp[0] && !br.clamp[1]) {
                        // clear of the ground: the distance form
                        const double galpha =
                            distance_vjp(A.gx, q.x, q.z, p0, p2, static_cast<double>(m.x), alphad);
                        acc[A.b_group[k]] += galpha * alphad;
                        continue;
                    }
                    // on the ground: VJP by forward mode along the forward's
                    // branches, one tangent per input (6 coordinates, alpha)
                    const uint32_t idx[2] = {q.x, q.z};
                    const float4 pp[2] = {p0, p2};
                    double u[6];
                    for (int e = 0; e < 2; ++e) {
                        const double4 ge = A.gx[idx[e]];
                        u[3 * e] = ge.x;
                        u[3 * e + 1] = ge.y;
                        u[3 * e + 2] = ge.z;
                    }
                    const double w[2] = {p0.w, p2.w};
                    double gin[7];
                    for (int dir = 0; dir < 7; ++dir) {
                        DV pd[2];
                        for (int e = 0; e < 2; ++e)
                            pd[e] = DV{Dual{pp[e].x, dir == 3 * e ? 1.0 : 0.0}, Dual{pp[e].y, dir == 3 * e + 1 ? 1.0 : 0.0},
                                       Dual{pp[e].z, dir == 3 * e + 2 ? 1.0 : 0.0}};
                        DV out[2];
                        bend_dual(pd, w, Dual{alphad, dir == 6 ? 1.0 : 0.0}, static_cast<double>(m.x),
                                  static_cast<double>(radius), br, out);
                        double acc_dir = 0.0;
                        for (int e = 0; e < 2; ++e)
                            acc_dir += u[3 * e] * out[e].x.d + u[3 * e + 1] * out[e].y.d + u[3 * e + 2] * out[e].z.d;
                        gin[dir] = acc_dir;
                    }
                    for (int e = 0; e < 2; ++e)
                        A.gx[idx[e]] = make_double4(gin[3 * e], gin[3 * e + 1], gin[3 * e + 2], 0.0);
                    acc[A.b_group[k]] += gin[6] * alphad;
                }
                break;
            }
            case ADJ_GRIP: {
                const bool active = cf.gripTargetAndActive.w > 0.0f;
                const uint32_t g = threadIdx.x;
                double gg[6] = {0, 0, 0, 0, 0, 0};
                if (active && g < d.g_count) {
                    const NumiClothGrip grip = d.grips[g];
                    if (grip.particle.y == cf.gripControl.x) {
                        const uint32_t i = grip.particle.x;
                        const float4 p = pre[i];
                        const float alpha = grip.targetOffsetAndCompliance.w / dt2;
                        if (p.w + alpha > 0.0f) {
                            const float4 qr = make_float4(cf.gripOrientation.x, cf.gripOrientation.y,
                                                          cf.gripOrientation.z, cf.gripOrientation.w);
                            const V3 ro = rotate_q(qr, V3{grip.targetOffsetAndCompliance.x,
                                                          grip.targetOffsetAndCompliance.y,
                                                          grip.targetOffsetAndCompliance.z});
                            const D3v target = addd(D3v{cf.gripTargetAndActive.x, cf.gripTargetAndActive.y,
                                                        cf.gripTargetAndActive.z},
                                                    d3f(ro));
                            const D3v gout = d3(A.gx[i]);
                            const double w = p.w;
                            const double al = static_cast<double>(grip.targetOffsetAndCompliance.w) / (dtd * dtd);
                            const double dn = w + al;
                            // x' = (alpha x + w T) / (w + alpha)
                            put(A.gx, i, muld(gout, al / dn));
                            const D3v gT = muld(gout, w / dn);
                            const D3v xm = subd(d4f(p), target);
                            acc[A.g_group[g]] += dotd(gout, muld(xm, w / (dn * dn))) * al;
                            const D3v rot = crossd(d3f(ro), gT);
                            gg[0] = gT.x;
                            gg[1] = gT.y;
                            gg[2] = gT.z;
                            gg[3] = rot.x;
                            gg[4] = rot.y;
                            gg[5] = rot.z;
                        }
                    }
                }
                if (g < NC_MAX_GRIPS)
                    for (int e = 0; e < 6; ++e) s_grip[g][e] = gg[e];
                __syncthreads();
                if (threadIdx.x == 0 && A.grip_grads != nullptr) {
                    double* out = A.grip_grads + static_cast<size_t>(step) * 6u;
                    for (uint32_t k = 0; k < min(d.g_count, NC_MAX_GRIPS); ++k)
                        for (int e = 0; e < 6; ++e) out[e] += s_grip[k][e];
                }
                break;
            }
            case ADJ_GROUND:
                if (ground)
                    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x)
                        if (radius - pre[i].z > 0.0f) A.gx[i].z = 0.0;
                break;
            case ADJ_BEGIN: {
                // x' = x_s + v' dt, v' = (v_s + g dt) / (1 + c dt)
                const float4* vs = A.tape_v + static_cast<size_t>(si) * n;
                const double c = A.damping;
                const double kf = c != 0.0 ? 1.0 / (1.0 + c * dtd) : 1.0;
                const double dk = -dtd / ((1.0 + c * dtd) * (1.0 + c * dtd));
                const D3v grav{cf.gravityAndTimestep.x, cf.gravityAndTimestep.y, cf.gravityAndTimestep.z};
                for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
                    if (pre[i].w == 0.0f) {
                        A.gx[i] = make_double4(0, 0, 0, 0);
                        A.gv[i] = make_double4(0, 0, 0, 0);
                        continue;
                    }
                    D3v gpos = d3(A.gx[i]);
                    // swept ground clamp: the predicted z is set to the radius
                    if (ground && pre[i].z >= radius && post[i].z == radius) gpos.z = 0.0;
                    // v' feeds x' and, through friction, the finalize step
                    D3v gvp = muld(gpos, dtd);
                    gvp.z += A.gprev[i].w;
                    const D3v v0 = addd(D3v{vs[i].x, vs[i].y, vs[i].z}, muld(grav, dtd));
                    acc[damp_slot] += dotd(gvp, v0) * dk;
                    put(A.gv, i, muld(gvp, kf));
                    put(A.gx, i, addd(gpos, d3(A.gprev[i])));
                    A.gprev[i] = make_double4(0, 0, 0, 0);
                }
                break;
            }
            default:
                break;
            }
            __syncthreads();
        }
    }
    // fixed-order block reductions
    __shared__ double s_red[NC_THREADS];
    __shared__ unsigned int s_rough;
    if (threadIdx.x == 0) s_rough = 0u;
    __syncthreads();
    if (rough) atomicAdd(&s_rough, rough);
    for (uint32_t e = 0; e <= A.groups + 1u; ++e) {
        s_red[threadIdx.x] = e <= A.groups ? acc[e] : loss;
        __syncthreads();
        for (uint32_t st = blockDim.x / 2u; st > 0u; st >>= 1u) {
            if (threadIdx.x < st) s_red[threadIdx.x] += s_red[threadIdx.x + st];
            __syncthreads();
        }
        if (threadIdx.x == 0) {
            if (e <= A.groups)
                A.grads[e] += s_red[0];
            else
                *A.loss += s_red[0];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) *A.nonsmooth += s_rough;
}

// One cloth's segment on one CTA.
__global__ void __launch_bounds__(NC_THREADS) numi_cloth_adjoint_kernel(AdjointArgs A) { adjoint_segment(A); }

// Many cloths' segments, one CTA each.
__global__ void __launch_bounds__(NC_THREADS) numi_cloth_adjoint_batch_kernel(const AdjointArgs* args) {
    adjoint_segment(args[blockIdx.x]);
}

// Device-to-device copies of many regions in one launch, one CTA per
// region (cloth state checkpoints of a batch).
struct CopyOp {
    const void* src;
    void* dst;
    unsigned long long bytes;
};

__global__ void numi_cloth_copy_kernel(const CopyOp* ops) {
    const CopyOp op = ops[blockIdx.x];
    if ((reinterpret_cast<uintptr_t>(op.src) | reinterpret_cast<uintptr_t>(op.dst) | op.bytes) % 16u == 0u) {
        const float4* s = static_cast<const float4*>(op.src);
        float4* d = static_cast<float4*>(op.dst);
        for (unsigned long long k = threadIdx.x; k < op.bytes / 16u; k += blockDim.x) d[k] = s[k];
    } else {
        const unsigned char* s = static_cast<const unsigned char*>(op.src);
        unsigned char* d = static_cast<unsigned char*>(op.dst);
        for (unsigned long long k = threadIdx.x; k < op.bytes; k += blockDim.x) d[k] = s[k];
    }
}
