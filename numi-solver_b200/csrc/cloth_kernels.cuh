// Persistent cooperative frame kernel of the XPBD cloth substep (sm_100a).
//
// One launch advances `substeps` substeps.  Every phase is a grid-stride
// loop over independent items (a colour batch, the particles, the fruits);
// phases are separated by a bounded grid barrier.  With a single CTA the
// barrier is __syncthreads, so a small cloth (the produce bag) runs as one
// resident CTA with no global synchronisation at all.
//
// Phase order per substep follows the reference CPU substep
// (tools/cloth_bag.cpp:4762-5262) with the reference Metal colour schedule
// for the constraint sweeps (tools/cloth_bag_metal.mm:4211-4709):
//   grip attach + begin + (air) + advance + swept ground
//   swept fruit/yarn
//   iterations: distance colours, knot colours, bend colours (even
//     iterations), grip + fruit pairs, fruit/yarn, self contact, ground
//   reconciliation passes (early exit on FP64 residuals)
//   endpoint strain + final contact passes, certificate (last substep)
//   finalize + frictions + orientation + release
//
// Fruits are few (<= 64): every fruit-only step runs in the last CTA and
// is ordered by __syncthreads.  Fruit displacements produced by the
// segment-parallel fruit/yarn sweep are summed in 2^-40 m fixed point
// with integer atomics, so the sum is exact and independent of the order
// in which segments run.
#pragma once

#include "cloth_device.cuh"
#include "vec.cuh"

#include <cooperative_groups.h>

#define NC_THREADS 256      /* threads of a CTA in the cooperative-grid launch; width of the fixed reduction trees */
#define NC_BLOCK_MAX 512    /* largest CTA (cluster launch) */
#define NC_FIXED_SCALE 1099511627776.0   /* 2^40 */
#define NC_BARRIER_SPIN_LIMIT (1u << 22)

namespace nc {
namespace {   // internal linkage: the edge kernels' unit includes these too

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(unsigned* p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ float4 ld(const float4* p) { return __ldcg(p); }
__device__ __forceinline__ float ldf(const float* p) { return __ldcg(p); }
__device__ __forceinline__ void fail(const DeviceCloth& d, unsigned bit) { atomicOr(d.failure, bit); }
__device__ __forceinline__ long long to_fixed(float v) {
    return __double2ll_rn(static_cast<double>(v) * NC_FIXED_SCALE);
}
__device__ __forceinline__ float from_fixed(unsigned long long v) {
    return static_cast<float>(static_cast<double>(static_cast<long long>(v)) * (1.0 / NC_FIXED_SCALE));
}

__device__ __forceinline__ unsigned ld_relaxed(const unsigned* p) {
    unsigned v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void red_release_add_u64(unsigned long long* p, unsigned long long v) {
    asm volatile("red.release.gpu.global.add.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ unsigned long long globaltimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

struct SubCfg {
    float dt;
    V3 gravity;
    float radius;        // yarn radius r (ground height of cloth particles)
    bool ground;
    bool grip_active;
    uint32_t grip_gen;
    uint32_t grip_select;
    uint32_t ring_count;
    uint32_t patch_half;
    float capture_radius;
    V3 grip_target;
    float4 grip_q;
    float mu_cloth_ground;
    float mu_pair, mu_fruit_ground, rolling, mu_fruit_yarn;
    float mu_self;       // yarn/yarn self friction
    V3 air;
    float air_density;
    float4 aero;         // crossflow, skin, fruit drag, fruit rotational drag
};

__device__ __forceinline__ SubCfg load_cfg(const NumiClothConfig* c) {
    SubCfg s;
    s.dt = c->gravityAndTimestep.w;
    s.gravity = V3{c->gravityAndTimestep.x, c->gravityAndTimestep.y, c->gravityAndTimestep.z};
    s.radius = c->clothMaterial.x;
    s.ground = c->constraintCounts.z != 0u;
    s.grip_active = c->gripTargetAndActive.w > 0.0f;
    s.grip_gen = c->gripControl.x;
    s.grip_select = c->gripControl.y;
    s.ring_count = c->gripControl.z;
    s.patch_half = c->gripControl.w;
    s.capture_radius = c->gripMaterial.x;
    s.grip_target = V3{c->gripTargetAndActive.x, c->gripTargetAndActive.y, c->gripTargetAndActive.z};
    s.grip_q = make_float4(c->gripOrientation.x, c->gripOrientation.y, c->gripOrientation.z,
                           c->gripOrientation.w);
    s.mu_cloth_ground = c->clothMaterial.z;
    s.mu_pair = c->fruitMaterial.x;
    s.mu_fruit_ground = c->fruitMaterial.y;
    s.rolling = c->fruitMaterial.z;
    s.mu_fruit_yarn = c->fruitMaterial.w;
    s.mu_self = c->clothMaterial.w;
    s.air = V3{c->airVelocityAndDensity.x, c->airVelocityAndDensity.y, c->airVelocityAndDensity.z};
    s.air_density = c->airVelocityAndDensity.w;
    s.aero = make_float4(c->aerodynamicCoefficients.x, c->aerodynamicCoefficients.y,
                         c->aerodynamicCoefficients.z, c->aerodynamicCoefficients.w);
    return s;
}

__device__ __forceinline__ float inverse_inertia(float w, float radius) {
    return 2.5f * w / (radius * radius);
}

// Per-thread view of a launch.  In resident mode (one thread-block cluster,
// particles kept in distributed shared memory for the whole launch) particle
// i lives in the shared memory of cluster rank i >> shift at offset
// i & (chunk - 1); otherwise it lives in global memory.
struct Ctx {
    const DeviceCloth& d;
    const Schedule& s;
    SubCfg c;
    uint32_t tid;
    uint32_t nthreads;
    bool fruit_cta;
    bool grip_cta;
    uint32_t barriers;
    bool fruit_pending;       // fixed-point fruit sums waiting to be applied
    uint32_t epoch;
    uint32_t sub;
    unsigned long long seq;   // barriers passed in this launch
    unsigned nseq;            // colour syncs passed in this launch
    FruitShared* fs;          // fruit-CTA shared state (valid in the fruit CTA)
    bool resident;
    uint32_t rank;            // cluster rank (resident) or 0
    uint32_t ranks;           // CTAs that own particles (resident) or 1
    uint32_t shift;           // log2 of the particles each CTA owns
    float4* xs;               // this CTA's positions in shared memory
    float4* vs;               // this CTA's velocities in shared memory
    // global position and velocity buffers the phases read and write:
    // DeviceCloth::x and ::v, or in tile mode (cloth_tile.cuh) whichever of
    // them and their alternates holds the current values
    float4* gx;
    float4* gv;
    // tile mode: this CTA's plan and its local particle positions, both in
    // shared memory
    const uint32_t* tp;
    float4* tx;
    FrictionStage* fst;       // tile mode, fruit CTA: the staged friction sweep
    bool hold_tail;           // tile mode: a grid barrier follows the fruit-CTA tail
    bool fruit_wait;          // tile mode: the next predict waits for the fruit-CTA friction
    uint4 tile_box;           // tile mode: rows and columns (grid cloth) or index range of chain 0's closure
};

__device__ __forceinline__ float4* resident_ptr(const Ctx& c, float4* local_base, uint32_t i) {
    const uint32_t r = i >> c.shift;
    float4* p = local_base + (i & ((1u << c.shift) - 1u));
    return r == c.rank ? p : static_cast<float4*>(__cluster_map_shared_rank(p, r));
}
// Particle position (xyz, inverse mass) and velocity accessors.
__device__ __forceinline__ float4 px(const Ctx& c, uint32_t i) {
    return c.resident ? *resident_ptr(c, c.xs, i) : __ldcg(c.gx + i);
}
__device__ __forceinline__ void px_set(const Ctx& c, uint32_t i, float4 v) {
    if (c.resident)
        *resident_ptr(c, c.xs, i) = v;
    else
        c.gx[i] = v;
}
__device__ __forceinline__ float4 pv(const Ctx& c, uint32_t i) {
    return c.resident ? *resident_ptr(c, c.vs, i) : __ldcg(c.gv + i);
}
__device__ __forceinline__ void pv_set(const Ctx& c, uint32_t i, float4 v) {
    if (c.resident)
        *resident_ptr(c, c.vs, i) = v;
    else
        c.gv[i] = v;
}

// Loop range of this thread over count items: grid-stride in the global
// modes; in resident mode each CTA takes one contiguous slice (constraint
// arrays follow particle order, so a slice touches mostly its own particles).
struct Range {
    uint32_t i, end, stride;
};
__device__ __forceinline__ Range item_range(const Ctx& c, uint32_t count) {
    if (c.resident) {
        const uint32_t lo = static_cast<uint32_t>(static_cast<unsigned long long>(count) * c.rank / c.ranks);
        const uint32_t hi = static_cast<uint32_t>(static_cast<unsigned long long>(count) * (c.rank + 1u) / c.ranks);
        return Range{lo + threadIdx.x, hi, blockDim.x};
    }
    return Range{c.tid, count, c.nthreads};
}
// Particles: resident mode walks the CTA's own particles.
__device__ __forceinline__ Range particle_range(const Ctx& c) {
    if (c.resident) {
        const uint32_t first = c.rank << c.shift;
        const uint32_t end = min(first + (1u << c.shift), c.d.n);
        return Range{first + threadIdx.x, end, blockDim.x};
    }
    return Range{c.tid, c.d.n, c.nthreads};
}

// ---------------------------------------------------------------- grip ----
// Re-attachment on a generation change (tools/cloth_bag.cpp:1520-1611;
// ClothBag.metal:577-673).  Block 0, one thread per grip.
__device__ void grip_attach(const Ctx& ctx) {
    const DeviceCloth& d = ctx.d;
    const SubCfg& c = ctx.c;
    const uint32_t g = threadIdx.x;
    if (g >= d.g_count || !c.grip_active) return;
    NumiClothGrip grip = d.grips[g];
    if (grip.particle.y == c.grip_gen) return;
    if (grip.particle.y == 0xffffffffu || grip.particle.y + 1u != c.grip_gen) {
        fail(d, NUMI_CLOTH_FAILURE_GRIP_CAPTURE);
        return;
    }
    uint32_t particle = grip.particle.x;
    if (c.grip_select == 1u) {
        uint32_t center = 0u;
        float nearest = INFINITY;
        for (uint32_t ring = 0u; ring < c.ring_count; ++ring) {
            const uint32_t cand = d.cuff[c.ring_count + ring];
            const V3 sep = xyz(px(ctx, cand)) - c.grip_target;
            const float dsq = lsq(sep);
            if (dsq < nearest) {
                nearest = dsq;
                center = ring;
            }
        }
        const uint32_t width = 2u * c.patch_half + 1u;
        const uint32_t row = g / width;
        const uint32_t slot = g % width;
        const uint32_t ring = (center + c.ring_count + slot - c.patch_half) % c.ring_count;
        particle = d.cuff[row * c.ring_count + ring];
        grip.particle.x = particle;
        grip.particle.w = center;
    }
    const V3 position = xyz(px(ctx, particle));
    const V3 sep = position - c.grip_target;
    const float capture = len3(sep);
    if (!finite3(position) || !isfinite(capture)) {
        fail(d, NUMI_CLOTH_FAILURE_NONFINITE);
        return;
    }
    if (capture > c.capture_radius) {
        fail(d, NUMI_CLOTH_FAILURE_GRIP_CAPTURE);
        return;
    }
    const V3 offset = inverse_rotate_q(c.grip_q, sep);
    const V3 rebuilt = c.grip_target + rotate_q(c.grip_q, offset);
    const float err = len3(position - rebuilt);
    grip.targetOffsetAndCompliance.x = offset.x;
    grip.targetOffsetAndCompliance.y = offset.y;
    grip.targetOffsetAndCompliance.z = offset.z;
    grip.particle.y = c.grip_gen;
    grip.particle.z = __float_as_uint(fmaxf(__uint_as_float(grip.particle.z), capture));
    grip.lambda.x = 0.0f;
    grip.lambda.y = 0.0f;
    grip.lambda.z = 0.0f;
    grip.lambda.w = fmaxf(grip.lambda.w, err);
    d.grips[g] = grip;
}

// Compliant vector attachment (tools/cloth_bag.cpp:1630-1647) on a loaded
// particle and grip record; false when it changes nothing.
__device__ __forceinline__ bool grip_core(const DeviceCloth& d, const SubCfg& c, NumiClothGrip& grip, float4& p) {
    const float alpha = grip.targetOffsetAndCompliance.w / (c.dt * c.dt);
    const float den = p.w + alpha;
    if (den <= 0.0f) return false;
    const V3 offset{grip.targetOffsetAndCompliance.x, grip.targetOffsetAndCompliance.y,
                    grip.targetOffsetAndCompliance.z};
    const V3 target = c.grip_target + rotate_q(c.grip_q, offset);
    const V3 value = xyz(p) - target;
    const V3 lambda{grip.lambda.x, grip.lambda.y, grip.lambda.z};
    const V3 dl = vdiv(value * -1.0f - lambda * alpha, den);
    const V3 nl = lambda + dl;
    const V3 np = xyz(p) + dl * p.w;
    if (!finite3(np)) fail(d, NUMI_CLOTH_FAILURE_NONFINITE);
    p = with_xyz(p, np);
    grip.lambda.x = nl.x;
    grip.lambda.y = nl.y;
    grip.lambda.z = nl.z;
    return true;
}

__device__ void solve_grips(const Ctx& ctx) {
    const DeviceCloth& d = ctx.d;
    const SubCfg& c = ctx.c;
    const uint32_t g = threadIdx.x;
    if (g >= d.g_count || !c.grip_active) return;
    NumiClothGrip grip = d.grips[g];
    if (grip.particle.y != c.grip_gen) return;
    const uint32_t i = grip.particle.x;
    float4 p = px(ctx, i);
    if (!grip_core(d, c, grip, p)) return;
    px_set(ctx, i, p);
    d.grips[g] = grip;
}

// ---------------------------------------------------------- constraints ---
// XPBD distance (tools/cloth_bag.cpp:1649-1673) on loaded values: updates
// the two particles and the multiplier; false when it changes nothing.
__device__ __forceinline__ bool distance_core(float4& a, float4& b, const float4& m, float& lam, float dt2) {
    const V3 diff = xyz(b) - xyz(a);
    const float L = len3(diff);
    if (L < 1.0e-12f) return false;
    const float alpha = m.y / dt2;
    const float den = (a.w + b.w) + alpha;
    if (den <= 0.0f) return false;
    const float value = L - m.x;
    const float dl = (-value - alpha * lam) / den;
    const V3 corr = diff * (dl / L);
    const V3 na = xyz(a) - corr * a.w;
    const V3 nb = xyz(b) + corr * b.w;
    a = with_xyz(a, na);
    b = with_xyz(b, nb);
    lam = lam + dl;
    return true;
}

__device__ __forceinline__ void solve_distance(const Ctx& ctx, uint32_t k, float dt2) {
    const DeviceCloth& d = ctx.d;
    const uint2 ij = __ldg(d.d_ij + k);
    const float4 m = __ldg(d.d_mat + k);
    float4 a = px(ctx, ij.x);
    float4 b = px(ctx, ij.y);
    float lam = ldf(d.d_lambda + k);
    if (!distance_core(a, b, m, lam, dt2)) return;
    px_set(ctx, ij.x, a);
    px_set(ctx, ij.y, b);
    d.d_lambda[k] = lam;
}

// Items a thread gathers before it computes any of them.  The items of one
// colour share no particle, so a thread may load all of its next NC_ILP
// items first and overlap their latencies; every item's arithmetic is the
// same as item by item.
#define NC_ILP 4

// Item j of a gathered group: its index within the batch (a dead slot
// repeats the group's first item, loads it and stores nothing).
struct IlpSlots {
    uint32_t i[NC_ILP];
    bool live[NC_ILP];
};
__device__ __forceinline__ IlpSlots ilp_slots(const Range& r) {
    IlpSlots s;
#pragma unroll
    for (int j = 0; j < NC_ILP; ++j) {
        const uint32_t i = r.i + static_cast<uint32_t>(j) * r.stride;
        s.live[j] = i < r.end;
        s.i[j] = s.live[j] ? i : r.i;
    }
    return s;
}

// One colour of distance constraints.
__device__ __forceinline__ void distance_colour(const Ctx& ctx, uint32_t first, uint32_t count, float dt2) {
    const DeviceCloth& d = ctx.d;
    for (Range r = item_range(ctx, count); r.i < r.end; r.i += NC_ILP * r.stride) {
        const IlpSlots sl = ilp_slots(r);
        uint2 ij[NC_ILP];
        float4 m[NC_ILP], a[NC_ILP], b[NC_ILP];
        float lam[NC_ILP];
#pragma unroll
        for (int j = 0; j < NC_ILP; ++j) {
            ij[j] = __ldg(d.d_ij + first + sl.i[j]);
            m[j] = __ldg(d.d_mat + first + sl.i[j]);
            lam[j] = ldf(d.d_lambda + first + sl.i[j]);
        }
#pragma unroll
        for (int j = 0; j < NC_ILP; ++j) {
            a[j] = px(ctx, ij[j].x);
            b[j] = px(ctx, ij[j].y);
        }
#pragma unroll
        for (int j = 0; j < NC_ILP; ++j) {
            if (!sl.live[j] || !distance_core(a[j], b[j], m[j], lam[j], dt2)) continue;
            px_set(ctx, ij[j].x, a[j]);
            px_set(ctx, ij[j].y, b[j]);
            d.d_lambda[first + sl.i[j]] = lam[j];
        }
    }
}

// Crossing-angle knot (tools/cloth_bag.cpp:1675-1725).
__device__ __forceinline__ void solve_knot(const Ctx& ctx, uint32_t k, float dt2) {
    const DeviceCloth& d = ctx.d;
    const uint4 q = __ldg(d.k_ij + k);
    const float2 m = __ldg(d.k_mat + k);
    const float4 p0 = px(ctx, q.x);
    const float4 p1 = px(ctx, q.y);
    const float4 p2 = px(ctx, q.z);
    const float4 p3 = px(ctx, q.w);
    const V3 warpv = xyz(p1) - xyz(p0);
    const V3 weftv = xyz(p3) - xyz(p2);
    const float wl = len3(warpv);
    const float fl = len3(weftv);
    if (wl < 1.0e-12f || fl < 1.0e-12f) return;
    const V3 warp = vdiv(warpv, wl);
    const V3 weft = vdiv(weftv, fl);
    const float cosine = fminf(fmaxf(dot3(warp, weft), -1.0f), 1.0f);
    const float value = cosine - m.x;
    const V3 gw = vdiv(weft - warp * cosine, wl);
    const V3 gf = vdiv(warp - weft * cosine, fl);
    const V3 g0 = gw * -1.0f;
    const V3 g2 = gf * -1.0f;
    const float alpha = m.y / dt2;
    float den = alpha;
    den = den + p0.w * lsq(g0);
    den = den + p1.w * lsq(gw);
    den = den + p2.w * lsq(g2);
    den = den + p3.w * lsq(gf);
    if (den <= 0.0f) return;
    const float lam = ldf(d.k_lambda + k);
    const float dl = (-value - alpha * lam) / den;
    d.k_lambda[k] = lam + dl;
    px_set(ctx, q.x, with_xyz(p0, xyz(p0) + g0 * (p0.w * dl)));
    px_set(ctx, q.y, with_xyz(p1, xyz(p1) + gw * (p1.w * dl)));
    px_set(ctx, q.z, with_xyz(p2, xyz(p2) + g2 * (p2.w * dl)));
    px_set(ctx, q.w, with_xyz(p3, xyz(p3) + gf * (p3.w * dl)));
}

// Skip-one chord bend with the ground active set (tools/cloth_bag.cpp:1782-1863)
// on loaded values: updates the two chord ends and the multiplier; false
// when it changes nothing.
__device__ __forceinline__ bool bend_core(float4 p[2], const float2& m, float& lam, float dt2, float radius,
                                          bool ground) {
    const V3 diff = xyz(p[1]) - xyz(p[0]);
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
    const float numerator = -value - alpha * lam;
    const float free_dl = numerator / free_den;
    bool active[2];
    float den = alpha;
    for (int s = 0; s < 2; ++s) {
        active[s] = ground && p[s].z <= radius + 1.0e-9f && g[s].z * free_dl < 0.0f;
        den = den + p[s].w * (lsq(g[s]) - (active[s] ? g[s].z * g[s].z : 0.0f));
    }
    if (den < 1.0e-16f) return false;
    const float dl = numerator / den;
    float fraction = 1.0f;
    if (ground) {
        for (int s = 0; s < 2; ++s) {
            if (active[s]) continue;
            const float vc = g[s].z * p[s].w * dl;
            if (vc >= 0.0f) continue;
            fraction = fminf(fraction, fmaxf(0.0f, p[s].z - radius) / -vc);
        }
    }
    const float applied = dl * fraction;
    lam = lam + applied;
    for (int s = 0; s < 2; ++s) {
        V3 corr = g[s] * (p[s].w * applied);
        if (active[s]) corr.z = 0.0f;
        V3 np = xyz(p[s]) + corr;
        if (ground && np.z < radius) np.z = radius;
        p[s] = with_xyz(p[s], np);
    }
    return true;
}

__device__ __forceinline__ void solve_bend(const Ctx& ctx, uint32_t k, float dt2, float radius, bool ground) {
    const DeviceCloth& d = ctx.d;
    const uint4 q = __ldg(d.b_ij + k);
    const float2 m = __ldg(d.b_mat + k);
    float4 p[2] = {px(ctx, q.x), px(ctx, q.z)};
    float lam = ldf(d.b_lambda + k);
    if (!bend_core(p, m, lam, dt2, radius, ground)) return;
    d.b_lambda[k] = lam;
    px_set(ctx, q.x, p[0]);
    px_set(ctx, q.z, p[1]);
}

// One colour of bends.
__device__ __forceinline__ void bend_colour(const Ctx& ctx, uint32_t first, uint32_t count, float dt2, float radius,
                                            bool ground) {
    const DeviceCloth& d = ctx.d;
    for (Range r = item_range(ctx, count); r.i < r.end; r.i += NC_ILP * r.stride) {
        const IlpSlots sl = ilp_slots(r);
        uint4 q[NC_ILP];
        float2 m[NC_ILP];
        float lam[NC_ILP];
        float4 p[NC_ILP][2];
#pragma unroll
        for (int j = 0; j < NC_ILP; ++j) {
            q[j] = __ldg(d.b_ij + first + sl.i[j]);
            m[j] = __ldg(d.b_mat + first + sl.i[j]);
            lam[j] = ldf(d.b_lambda + first + sl.i[j]);
        }
#pragma unroll
        for (int j = 0; j < NC_ILP; ++j) {
            p[j][0] = px(ctx, q[j].x);
            p[j][1] = px(ctx, q[j].z);
        }
#pragma unroll
        for (int j = 0; j < NC_ILP; ++j) {
            if (!sl.live[j] || !bend_core(p[j], m[j], lam[j], dt2, radius, ground)) continue;
            d.b_lambda[first + sl.i[j]] = lam[j];
            px_set(ctx, q[j].x, p[j][0]);
            px_set(ctx, q[j].z, p[j][1]);
        }
    }
}

// Unilateral strain limit (tools/cloth_bag.cpp:1732-1763) on loaded values;
// false when it changes nothing.  The correction is not published.
__device__ __forceinline__ bool strain_core(float4& a, float4& b, const float4& m) {
    if (!(m.w > 0.0f)) return false;
    const V3 diff = xyz(b) - xyz(a);
    const float L = len3(diff);
    const float maxL = m.x * (1.0f + m.w);
    if (L <= maxL || L < 1.0e-12f) return false;
    const float den = a.w + b.w;
    if (den <= 0.0f) return false;
    const float cm = L - maxL;
    const V3 dir = vdiv(diff, L);
    a = with_xyz(a, xyz(a) + dir * (a.w * cm / den));
    b = with_xyz(b, xyz(b) - dir * (b.w * cm / den));
    return true;
}

__device__ __forceinline__ void limit_strain(const Ctx& ctx, uint32_t k) {
    const DeviceCloth& d = ctx.d;
    const float4 m = __ldg(d.d_mat + k);
    if (!(m.w > 0.0f)) return;
    const uint2 ij = __ldg(d.d_ij + k);
    float4 a = px(ctx, ij.x);
    float4 b = px(ctx, ij.y);
    if (!strain_core(a, b, m)) return;
    px_set(ctx, ij.x, a);
    px_set(ctx, ij.y, b);
}

// One colour's strain-limited prefix.
__device__ __forceinline__ void strain_colour(const Ctx& ctx, uint32_t first, uint32_t count) {
    const DeviceCloth& d = ctx.d;
    for (Range r = item_range(ctx, count); r.i < r.end; r.i += NC_ILP * r.stride) {
        const IlpSlots sl = ilp_slots(r);
        uint2 ij[NC_ILP];
        float4 m[NC_ILP], a[NC_ILP], b[NC_ILP];
#pragma unroll
        for (int j = 0; j < NC_ILP; ++j) {
            ij[j] = __ldg(d.d_ij + first + sl.i[j]);
            m[j] = __ldg(d.d_mat + first + sl.i[j]);
        }
#pragma unroll
        for (int j = 0; j < NC_ILP; ++j) {
            a[j] = px(ctx, ij[j].x);
            b[j] = px(ctx, ij[j].y);
        }
#pragma unroll
        for (int j = 0; j < NC_ILP; ++j) {
            if (!sl.live[j] || !strain_core(a[j], b[j], m[j])) continue;
            px_set(ctx, ij[j].x, a[j]);
            px_set(ctx, ij[j].y, b[j]);
        }
    }
}

// ------------------------------------------------------------- fruits -----
struct FruitState {
    V3 x;
    float w;
    V3 prev;
    float radius;
    V3 v;
    float ground_impulse;
    V3 omega;
    float4 q;   // xyzw
};

__device__ __forceinline__ FruitState load_fruit(const NumiClothFruit& f) {
    FruitState s;
    s.x = V3{f.positionAndInverseMass.x, f.positionAndInverseMass.y, f.positionAndInverseMass.z};
    s.w = f.positionAndInverseMass.w;
    s.prev = V3{f.previousAndRadius.x, f.previousAndRadius.y, f.previousAndRadius.z};
    s.radius = f.previousAndRadius.w;
    s.v = V3{f.velocityAndGroundImpulse.x, f.velocityAndGroundImpulse.y, f.velocityAndGroundImpulse.z};
    s.ground_impulse = f.velocityAndGroundImpulse.w;
    s.omega = V3{f.angularVelocity.x, f.angularVelocity.y, f.angularVelocity.z};
    s.q = make_float4(f.orientation.x, f.orientation.y, f.orientation.z, f.orientation.w);
    return s;
}

__device__ __forceinline__ void store_fruit(NumiClothFruit& f, const FruitState& s) {
    f.positionAndInverseMass.x = s.x.x;
    f.positionAndInverseMass.y = s.x.y;
    f.positionAndInverseMass.z = s.x.z;
    f.previousAndRadius.x = s.prev.x;
    f.previousAndRadius.y = s.prev.y;
    f.previousAndRadius.z = s.prev.z;
    f.velocityAndGroundImpulse.x = s.v.x;
    f.velocityAndGroundImpulse.y = s.v.y;
    f.velocityAndGroundImpulse.z = s.v.z;
    f.velocityAndGroundImpulse.w = s.ground_impulse;
    f.angularVelocity.x = s.omega.x;
    f.angularVelocity.y = s.omega.y;
    f.angularVelocity.z = s.omega.z;
    f.orientation.x = s.q.x;
    f.orientation.y = s.q.y;
    f.orientation.z = s.q.z;
    f.orientation.w = s.q.w;
}

// Implicit quadratic drag (tools/cloth_bag.cpp:991-1011, 1109-1181).
__device__ __forceinline__ float drag_attenuation(float speed, float coefficient, float w, float dt) {
    return 1.0f / (1.0f + w * coefficient * speed * dt);
}

__device__ void fruit_air(FruitState& f, const SubCfg& c) {
    const float pi = 3.14159265358979323846f;
    const V3 rel = f.v - c.air;
    const float frontal = pi * f.radius * f.radius;
    const float tcoef = 0.5f * c.air_density * c.aero.z * frontal;
    const float tatt = drag_attenuation(len3(rel), tcoef, f.w, c.dt);
    f.v = c.air + rel * tatt;
    const float r2 = f.radius * f.radius;
    const float r5 = r2 * r2 * f.radius;
    const float rcoef = (3.0f * pi * pi / 8.0f) * c.air_density * c.aero.w * r5;
    const float ratt = drag_attenuation(len3(f.omega), rcoef, inverse_inertia(f.w, f.radius), c.dt);
    f.omega = f.omega * ratt;
}

// Sphere/sphere separation (tools/cloth_bag.cpp:1897-1919).
// All fruit-pair colours, in the fruit CTA: fruit positions staged in
// shared memory, one warp walks the colours (a colour's pairs are disjoint,
// so its lanes never touch the same fruit); pair impulses accumulate in
// shared memory.
__device__ void fruit_pair_sweep(const DeviceCloth& d, FruitShared& fs, float dt) {
    for (uint32_t f = threadIdx.x; f < d.f_count; f += blockDim.x) {
        const NumiClothFruit& fr = d.fruits[f];
        fs.fx[f] = make_float4(fr.positionAndInverseMass.x, fr.positionAndInverseMass.y,
                               fr.positionAndInverseMass.z, fr.positionAndInverseMass.w);
        fs.fr[f] = fr.previousAndRadius.w;
    }
    __syncthreads();
    // Fruits move only through pair contacts, so when no pair touches at the
    // start of the sweep none touches at any point of it: skip the walk.
    bool touching = false;
    for (uint32_t k = threadIdx.x; k < d.p_count; k += blockDim.x) {
        const uint32_t ia = fs.ab[k] & 0xffu;
        const uint32_t ib = fs.ab[k] >> 8;
        const float L = len3(xyz(fs.fx[ib]) - xyz(fs.fx[ia]));
        touching = touching || !(L >= fs.fr[ia] + fs.fr[ib] || L < 1.0e-12f);
    }
    if (!__syncthreads_or(touching)) return;
    if (threadIdx.x < 32u) {
        for (uint32_t b = 0; b < d.n_pair_batches; ++b) {
            const Batch bt = d.pair_batches[b];
            bool loaded = false;
            for (uint32_t k = bt.first + threadIdx.x; k < bt.first + bt.count; k += 32u) {
                const uint32_t ia = fs.ab[k] & 0xffu;
                const uint32_t ib = fs.ab[k] >> 8;
                const float4 A = fs.fx[ia];
                const float4 B = fs.fx[ib];
                const V3 diff = xyz(B) - xyz(A);
                const float L = len3(diff);
                const float target = fs.fr[ia] + fs.fr[ib];
                if (L >= target || L < 1.0e-12f) continue;
                const float den = A.w + B.w;
                const float lambda = (target - L) / den;
                const V3 normal = vdiv(diff, L);
                const V3 corr = normal * lambda;
                fs.fx[ia] = with_xyz(A, xyz(A) - corr * A.w);
                fs.fx[ib] = with_xyz(B, xyz(B) + corr * B.w);
                const float imp = lambda / dt;
                const float4 c = fs.contact[k];
                const V3 wn = xyz(c) + normal * imp;
                fs.contact[k] = make_float4(wn.x, wn.y, wn.z, c.w + imp);
                loaded = loaded || c.w + imp > 0.0f;
            }
            if (__any_sync(0xffffffffu, loaded) && threadIdx.x == 0) fs.loaded |= 1ull << b;
            __syncwarp();
        }
    }
    __syncthreads();
    for (uint32_t f = threadIdx.x; f < d.f_count; f += blockDim.x) {
        NumiClothFruit& fr = d.fruits[f];
        fr.positionAndInverseMass.x = fs.fx[f].x;
        fr.positionAndInverseMass.y = fs.fx[f].y;
        fr.positionAndInverseMass.z = fs.fx[f].z;
    }
    __syncthreads();
}

// Coulomb pair friction (tools/cloth_bag.cpp:1921-1983) on fruit states
// staged in shared memory (v.xyz + inverse mass, omega.xyz + radius).
__device__ __forceinline__ void pair_friction_smem(float4* sv, float4* so, uint32_t ia, uint32_t ib, V3 wn,
                                                   float ni, float mu) {
    if (ni <= 0.0f || lsq(wn) < 1.0e-20f) return;
    const float4 va = sv[ia], vb = sv[ib], oa4 = so[ia], ob4 = so[ib];
    const V3 normal = normalized3(wn);
    const V3 oa = normal * oa4.w;
    const V3 ob = normal * -ob4.w;
    const V3 ca = xyz(va) + cross3(xyz(oa4), oa);
    const V3 cb = xyz(vb) + cross3(xyz(ob4), ob);
    const V3 rel = cb - ca;
    const V3 tv = rel - normal * dot3(rel, normal);
    const float slip = len3(tv);
    if (slip < 1.0e-10f) return;
    const V3 t = vdiv(tv, slip);
    const float ia_inv = inverse_inertia(va.w, oa4.w);
    const float ib_inv = inverse_inertia(vb.w, ob4.w);
    const float den = ((va.w + vb.w) + ia_inv * lsq(cross3(oa, t))) + ib_inv * lsq(cross3(ob, t));
    if (den <= 0.0f) return;
    const float limit = mu * ni;
    const float ti = fminf(slip / den, limit);
    if (ti <= 0.0f) return;
    const V3 imp_b = t * -ti;
    const V3 imp_a = imp_b * -1.0f;
    sv[ib] = with_xyz(vb, xyz(vb) + imp_b * vb.w);
    so[ib] = with_xyz(ob4, xyz(ob4) + cross3(ob, imp_b) * ib_inv);
    sv[ia] = with_xyz(va, xyz(va) + imp_a * va.w);
    so[ia] = with_xyz(oa4, xyz(oa4) + cross3(oa, imp_a) * ia_inv);
}

__device__ __forceinline__ void apply_fruit_impulse(FruitState& f, V3 impulse, V3 offset) {
    f.v = f.v + impulse * f.w;
    f.omega = f.omega + cross3(offset, impulse) * inverse_inertia(f.w, f.radius);
}

// Fruit/ground Coulomb friction and rolling resistance
// (tools/cloth_bag.cpp:1985-2074).
__device__ void fruit_ground_friction(FruitState& f, const SubCfg& c) {
    const float ni = f.ground_impulse;
    if (ni <= 0.0f) return;
    const V3 offset{0.0f, 0.0f, -f.radius};
    const V3 n{0.0f, 0.0f, 1.0f};
    const V3 cv = f.v + cross3(f.omega, offset);
    const V3 tv = cv - n * dot3(cv, n);
    const float slip = len3(tv);
    const float inv_i = inverse_inertia(f.w, f.radius);
    if (slip > 1.0e-10f) {
        const V3 t = vdiv(tv, slip);
        const float den = f.w + inv_i * lsq(cross3(offset, t));
        const float limit = c.mu_fruit_ground * ni;
        const float ti = fminf(slip / den, limit);
        if (ti > 0.0f) apply_fruit_impulse(f, t * -ti, offset);
    }
    const V3 roll{f.omega.x, f.omega.y, 0.0f};
    const float rs = len3(roll);
    if (ni <= 0.0f || rs <= 1.0e-12f || c.rolling <= 0.0f) return;
    const float required = rs / inv_i;
    const float limit = c.rolling * f.radius * ni;
    const float ai = fminf(required, limit);
    f.omega = f.omega - roll * (ai * inv_i / rs);
}

// q <- normalize(q + (omega (x) q) dt/2) (tools/cloth_bag.cpp:979-989).
__device__ void integrate_orientation(FruitState& f, float dt) {
    const float aw = 0.0f, ax = f.omega.x, ay = f.omega.y, az = f.omega.z;
    const float bw = f.q.w, bx = f.q.x, by = f.q.y, bz = f.q.z;
    const float pw = ((aw * bw - ax * bx) - ay * by) - az * bz;
    const float px = ((aw * bx + ax * bw) + ay * bz) - az * by;
    const float py = ((aw * by - ax * bz) + ay * bw) + az * bx;
    const float pz = ((aw * bz + ax * by) - ay * bx) + az * bw;
    const float h = 0.5f * dt;
    const float qw = bw + pw * h, qx = bx + px * h, qy = by + py * h, qz = bz + pz * h;
    const float m = sqrtf(((qw * qw + qx * qx) + qy * qy) + qz * qz);
    if (m > 1.0e-14f) {
        const float s = 1.0f / m;
        f.q = make_float4(qx * s, qy * s, qz * s, qw * s);
    } else {
        f.q = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
    }
}

// -------------------------------------------------------- fruit / yarn ----
// Closest point of p on segment [a, b] (the point/segment case of
// closestPointsOnSegments, tools/cloth_bag.cpp:2751-2824).
__device__ __forceinline__ void point_segment(V3 p, V3 a, V3 b, V3& closest, float& weight) {
    const V3 dir = b - a;
    const float lb = lsq(dir);
    if (lb <= 1.0e-20f) {
        closest = a;
        weight = 0.0f;
        return;
    }
    const float proj = dot3(dir, p - a);
    weight = fminf(fmaxf(proj / lb, 0.0f), 1.0f);
    closest = a + dir * weight;
}

// Ground-aware yarn response (tools/cloth_bag.cpp:2863-2953).  Moves the
// two segment particles; returns the accumulated multiplier and the fruit
// displacement (to be summed, not applied here).
__device__ float yarn_correction(float4& pa, float4& pb, float wa_seg, float wb_seg, float wf, V3 n,
                                 float correction, bool ground, float radius, V3& fruit_delta) {
    const float wt[2] = {wa_seg, wb_seg};
    float4* p[2] = {&pa, &pb};
    bool active[2] = {false, false};
    if (ground && n.z < 0.0f) {
        for (int s = 0; s < 2; ++s) {
            active[s] = wt[s] > 0.0f && p[s]->z <= radius + 1.0e-9f;
            if (active[s]) p[s]->z = radius;
        }
    }
    float remaining = correction;
    float acc = 0.0f;
    for (int it = 0; it < 3 && remaining > 1.0e-14f; ++it) {
        V3 resp[2];
        float den = wf;
        for (int s = 0; s < 2; ++s) {
            resp[s] = n * p[s]->w;
            if (active[s]) resp[s].z = 0.0f;
            den = den + dot3(n, resp[s]) * wt[s] * wt[s];
        }
        if (den <= 0.0f) break;
        const float unconstrained = remaining / den;
        float step = unconstrained;
        if (ground && n.z < 0.0f) {
            for (int s = 0; s < 2; ++s) {
                const float vr = resp[s].z * wt[s];
                if (active[s] || vr >= 0.0f) continue;
                const float dg = fmaxf(0.0f, p[s]->z - radius);
                step = fminf(step, dg / -vr);
            }
        }
        fruit_delta = fruit_delta - n * (wf * step);
        for (int s = 0; s < 2; ++s) {
            const V3 np = xyz(*p[s]) + resp[s] * (wt[s] * step);
            p[s]->x = np.x;
            p[s]->y = np.y;
            p[s]->z = np.z;
        }
        acc = acc + step;
        remaining = fmaxf(0.0f, remaining - den * step);
        if (step >= unconstrained - 1.0e-14f) break;
        bool activated = false;
        for (int s = 0; s < 2; ++s) {
            if (!active[s] && wt[s] > 0.0f && p[s]->z <= radius + 1.0e-9f) {
                p[s]->z = radius;
                active[s] = true;
                activated = true;
            }
        }
        if (!activated) break;
    }
    return acc;
}

}  // namespace
}  // namespace nc
