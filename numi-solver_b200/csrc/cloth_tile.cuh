// Tile mode of the cooperative grid: colour chains between grid barriers.
//
// On the cooperative grid every constraint colour ends with a barrier,
// because the next colour reads particles the last one wrote; a substep of
// the 256x256 cloth passes 26 of them, and the substep time is their
// latency.  In tile mode each CTA (the fruit CTA excepted) owns a tile of
// particles (a 2-D block of a grid cloth, or an index strip) and, for a
// chain of colours, the closure of its tile: the items of every colour of
// the chain whose results reach an owned particle through the later
// colours, and the particles those items read.  It loads the closure's
// particles into shared memory, runs the chain there with CTA barriers
// between the colours, and stores only its own particles.  An item that
// several CTAs need is computed by each of them from the same inputs in the
// same colour order, with the same float operations, so every copy holds
// the bits the grid-barrier schedule gives; side effects (multipliers,
// friction records, fruit sums, contact statistics) are left to the item's
// owner, the CTA owning its first particle.
//
// A chain reads the positions the previous phase left and its CTAs store
// their results while others may still be loading, so positions alternate
// between two global buffers from phase to phase (Ctx::gx), and
// velocities, which the substep start reads as it predicts the closure,
// alternate from substep to substep (Ctx::gv).  A launch that ends on the
// second buffer copies it back.
//
// The substep (one XPBD iteration; no air load, swept fruit contact,
// edge/edge family or reconciliation, final or certificate passes) runs as
//   1. predict of the closure, distance and bend colours, grips (owner of
//      the gripped particle); fruit CTA: fruit predict and fruit pairs;
//   2. fruit/yarn colours, self-contact insert of the owned particles;
//   3. self-contact solve and ground clamp of the closure, strain colours,
//      finalize and cloth/ground friction of the owned particles; fruit
//      CTA: fruit sums, ground and finalize (more strain sweeps: one phase
//      each);
//   4. fruit CTA: fruit/yarn friction, fruit frictions, orientation,
//      release; CTA 0: the next substep's grip attach;
// with one grid barrier after each, instead of one per colour; the one
// after phase 4 only where the next substep needs it (friction on listed
// segments, a grip re-attach, the launch's last substep).
//
// Plan of one CTA (host-built, 16-byte aligned words, staged into shared
// memory once per launch with a bulk copy):
//   [0] local particles, [1] owned particles (the first ones),
//   [2] word offset of the particle list, [3] word offset of the items,
//   [4 + k] local particles chain k reads (a prefix of the list),
//   [8 + 2k], [9 + 2k] word offset and count of chain k's colour table
//   (k = 0 distance and bend colours, 1 fruit/yarn colours, 2 strain
//   colours); a colour is (first item, count | family << 28), an item
//   (first | second local particle << 16, record | owner << 31, two
//   material words).
#pragma once

namespace nc {
namespace {

#define NC_TILE_HEADER 16u
#define NC_TILE_CHAINS 3u
#define NC_TILE_CONSTRAINTS 0u
#define NC_TILE_YARN 1u
#define NC_TILE_STRAIN 2u
#define NC_TILE_DISTANCE 0u
#define NC_TILE_BEND 1u
#define NC_TILE_LIMIT 2u
#define NC_TILE_SEGMENT 3u
// Stage this CTA's plan into shared memory: one bulk load (nc::bulk_load,
// bounded wait).
__device__ bool tile_stage(const Ctx& ctx, uint32_t* plan) {
    const DeviceCloth& d = ctx.d;
    const uint32_t w0 = d.tile_off[ctx.rank], w1 = d.tile_off[ctx.rank + 1u];
    const BulkJob job{plan, d.tile_words + w0, (w1 - w0) * 4u};
    return bulk_load(d, &job, 1u);
}

__device__ __forceinline__ const uint32_t* tile_list(const Ctx& ctx) { return ctx.tp + ctx.tp[2]; }
__device__ __forceinline__ const uint4* tile_items(const Ctx& ctx) {
    return reinterpret_cast<const uint4*>(ctx.tp + ctx.tp[3]);
}
__device__ __forceinline__ float4* other_x(const Ctx& ctx) { return ctx.gx == ctx.d.x ? ctx.d.x_alt : ctx.d.x; }
__device__ __forceinline__ float4* other_v(const Ctx& ctx) { return ctx.gv == ctx.d.v ? ctx.d.v_alt : ctx.d.v; }

// Local particles of chain k from the current position buffer.
__device__ __forceinline__ void tile_load(const Ctx& ctx, uint32_t chain) {
    const uint32_t nl = ctx.tp[4u + chain];
    const uint32_t* gi = tile_list(ctx);
    for (uint32_t l = threadIdx.x; l < nl; l += blockDim.x) ctx.tx[l] = __ldcg(ctx.gx + gi[l]);
    __syncthreads();
}

// Owned particles to the other position buffer.
__device__ __forceinline__ void tile_store(const Ctx& ctx, float4* out) {
    const uint32_t own = ctx.tp[1];
    const uint32_t* gi = tile_list(ctx);
    for (uint32_t l = threadIdx.x; l < own; l += blockDim.x) out[gi[l]] = ctx.tx[l];
}

// Substep start of chain 0's particles (predict_particle from the current
// buffers); the owners keep the substep-start position and publish the
// predicted velocity (w = predicted vertical velocity) to v_next.
__device__ void tile_predict(const Ctx& ctx, float4* v_next) {
    const DeviceCloth& d = ctx.d;
    const uint32_t nl = ctx.tp[4u + NC_TILE_CONSTRAINTS];
    const uint32_t own = ctx.tp[1];
    const uint32_t* gi = tile_list(ctx);
    for (uint32_t l = threadIdx.x; l < nl; l += blockDim.x) {
        const uint32_t i = gi[l];
        const float4 p = __ldcg(ctx.gx + i);
        V3 pos, vel;
        predict_particle(ctx, i, p, __ldcg(ctx.gv + i), false, pos, vel);
        ctx.tx[l] = with_xyz(p, pos);
        if (l < own) {
            const float4 pp = ld(d.xp + i);
            d.xp[i] = make_float4(p.x, p.y, p.z, pp.w);
            v_next[i] = make_float4(vel.x, vel.y, vel.z, vel.z);
        }
    }
    __syncthreads();
}

// A chain's colours in order, CTA barriers between them.  Distances and
// bends start from zero multipliers (one iteration per substep), and the
// owner publishes every multiplier it computes (zero when the projection
// changes nothing, as after the reset of the substep start).
__device__ void tile_chain(const Ctx& ctx, uint32_t chain, float dt2) {
    const DeviceCloth& d = ctx.d;
    const uint32_t* table = ctx.tp + ctx.tp[8u + 2u * chain];
    const uint32_t colours = ctx.tp[9u + 2u * chain];
    const uint4* items = tile_items(ctx);
    float4* tx = ctx.tx;
    for (uint32_t c = 0; c < colours; ++c) {
        const uint32_t first = table[2u * c];
        const uint32_t count = table[2u * c + 1u] & 0x0fffffffu;
        const uint32_t family = table[2u * c + 1u] >> 28;
        for (uint32_t k = threadIdx.x; k < count; k += blockDim.x) {
            const uint4 it = items[first + k];
            const uint32_t al = it.x & 0xffffu, bl = it.x >> 16;
            const uint32_t rec = it.y & 0x7fffffffu;
            const bool owner = (it.y >> 31) != 0u;
            if (family == NC_TILE_DISTANCE) {
                float4 a = tx[al], b = tx[bl];
                const float4 m = make_float4(__uint_as_float(it.z), __uint_as_float(it.w), 0.0f, 0.0f);
                float lam = 0.0f;
                if (distance_core(a, b, m, lam, dt2)) {
                    tx[al] = a;
                    tx[bl] = b;
                }
                if (owner) d.d_lambda[rec] = lam;
            } else if (family == NC_TILE_BEND) {
                float4 p[2] = {tx[al], tx[bl]};
                const float2 m = make_float2(__uint_as_float(it.z), __uint_as_float(it.w));
                float lam = 0.0f;
                if (bend_core(p, m, lam, dt2, ctx.c.radius, ctx.c.ground)) {
                    tx[al] = p[0];
                    tx[bl] = p[1];
                }
                if (owner) d.b_lambda[rec] = lam;
            } else {
                float4 a = tx[al], b = tx[bl];
                const float4 m = make_float4(__uint_as_float(it.z), 0.0f, 0.0f, __uint_as_float(it.w));
                if (strain_core(a, b, m)) {
                    tx[al] = a;
                    tx[bl] = b;
                }
            }
        }
        __syncthreads();
    }
}

// Grips after the constraint colours (tools/cloth_bag.cpp:1630-1647), each
// by the CTA owning its particle; the multipliers start the substep at zero.
__device__ void tile_grips(const Ctx& ctx) {
    const DeviceCloth& d = ctx.d;
    const SubCfg& c = ctx.c;
    for (uint32_t g = threadIdx.x; g < d.g_count; g += blockDim.x) {
        NumiClothGrip grip = d.grips[g];
        const uint32_t own = d.tile_owner[grip.particle.x];
        if ((own >> 16) != ctx.rank) continue;
        grip.lambda.x = 0.0f;
        grip.lambda.y = 0.0f;
        grip.lambda.z = 0.0f;
        if (c.grip_active && grip.particle.y == c.grip_gen) {
            float4 p = ctx.tx[own & 0xffffu];
            if (grip_core(d, c, grip, p)) ctx.tx[own & 0xffffu] = p;
        }
        d.grips[g] = grip;
    }
    __syncthreads();
}

// The fruit/yarn colours on the closure: a warp takes 32 items of a colour
// at a time (yarn_warp_contacts); fruits are frozen over the sweep and the
// owners' displacement sums go to the global sums once.
__device__ void tile_yarn(const Ctx& ctx) {
    const DeviceCloth& d = ctx.d;
    __shared__ float4 s_fruit[NC_MAX_FRUITS];
    __shared__ float s_fw[NC_MAX_FRUITS];
    __shared__ unsigned long long s_sum[3u * NC_MAX_FRUITS];
    cta_sums_clear(s_sum, 3u * d.f_count);
    for (uint32_t f = threadIdx.x; f < d.f_count; f += blockDim.x) {
        const NumiClothFruit& fr = d.fruits[f];
        const float4 xw = __ldcg(reinterpret_cast<const float4*>(&fr.positionAndInverseMass));
        s_fruit[f] = make_float4(xw.x, xw.y, xw.z, __ldcg(&fr.previousAndRadius.w));
        s_fw[f] = xw.w;
    }
    __syncthreads();
    const uint32_t* table = ctx.tp + ctx.tp[8u + 2u * NC_TILE_YARN];
    const uint32_t colours = ctx.tp[9u + 2u * NC_TILE_YARN];
    const uint4* items = tile_items(ctx);
    const uint32_t lane = threadIdx.x & 31u;
    for (uint32_t c = 0; c < colours; ++c) {
        const uint32_t first = table[2u * c];
        const uint32_t count = table[2u * c + 1u] & 0x0fffffffu;
        for (uint32_t base = threadIdx.x - lane; base < count; base += blockDim.x) {
            const uint32_t k = base + lane;
            const bool valid = k < count;
            uint4 it = make_uint4(0u, 0u, 0u, 0u);
            float4 pa = make_float4(0, 0, 0, 0), pb = pa;
            if (valid) {
                it = items[first + k];
                pa = ctx.tx[it.x & 0xffffu];
                pb = ctx.tx[it.x >> 16];
            }
            if (yarn_warp_contacts(ctx, valid, (it.y >> 31) != 0u, it.y & 0x7fffffffu, pa, pb, s_fruit, s_fw,
                                   s_sum)) {
                ctx.tx[it.x & 0xffffu] = pa;
                ctx.tx[it.x >> 16] = pb;
            }
        }
        __syncthreads();
    }
    cta_sums_flush(s_sum, reinterpret_cast<unsigned long long*>(d.fruit_partial), 3u * d.f_count);
}

// Self-contact insert of the owned particles at their start-of-pass
// positions (the first pass of the substep).
__device__ __forceinline__ void tile_insert(const Ctx& ctx) {
    const unsigned long long tag = self_pass_tag(ctx, 0u);
    const uint32_t own = ctx.tp[1];
    const uint32_t* gi = tile_list(ctx);
    for (uint32_t l = threadIdx.x; l < own; l += blockDim.x) self_insert_one(ctx, tag, gi[l], ctx.tx[l]);
}

// Self-contact solve and ground clamp of the strain chain's particles
// (each a function of its start-of-pass position and the grid), counted
// for the owned ones.
__device__ void tile_self_ground(const Ctx& ctx, bool self) {
    const SubCfg& c = ctx.c;
    const uint32_t nl = ctx.tp[4u + NC_TILE_STRAIN];
    const uint32_t own = ctx.tp[1];
    const uint32_t* gi = tile_list(ctx);
    const uint32_t tag = self_pass_tag(ctx, 0u);
    unsigned long long contacts = 0ull, ghost_contacts = 0ull;
    float max_pen = 0.0f, ghost_pen = 0.0f;
    for (uint32_t l = threadIdx.x; l < nl; l += blockDim.x) {
        float4 p = ctx.tx[l];
        if (self) {
            float4 q;
            const bool mine = l < own;
            if (self_solve_one(ctx, tag, gi[l], p, q, mine ? contacts : ghost_contacts, mine ? max_pen : ghost_pen))
                p = q;
        }
        if (c.ground && c.radius - p.z > 0.0f) p = make_float4(p.x, p.y, c.radius, p.w);
        ctx.tx[l] = p;
    }
    if (self) self_stats_flush(ctx.d, contacts, max_pen);
    __syncthreads();
}

// Finalize and cloth/ground friction of the owned particles; the
// velocities are updated in place in the current velocity buffer.
__device__ void tile_finalize(const Ctx& ctx) {
    const uint32_t own = ctx.tp[1];
    const uint32_t* gi = tile_list(ctx);
    for (uint32_t l = threadIdx.x; l < own; l += blockDim.x) {
        const uint32_t i = gi[l];
        float4 p = ctx.tx[l];
        float4 v;
        if (finalize_particle(ctx, i, p, __ldcg(ctx.gv + i), v)) ctx.tx[l] = p;
        ctx.gv[i] = v;
    }
}

// One substep in tile mode (see the top of this file).
__device__ bool substep_tiles(Ctx& ctx, bool last) {
    const DeviceCloth& d = ctx.d;
    const Schedule& s = ctx.s;
    const float dt2 = ctx.c.dt * ctx.c.dt;
    const bool self = s.self_collision && d.hash_head != nullptr;
    const bool fruits = d.f_count > 0u;
    // 1. predict, distance and bend colours, grips
    {
        float4* x_next = other_x(ctx);
        float4* v_next = other_v(ctx);
        if (ctx.fruit_cta) {
            fruit_begin(ctx);
            if (d.p_count > 0u) {
                __syncthreads();
                fruit_pair_sweep(d, *ctx.fs, ctx.c.dt);
            }
        } else {
            tile_predict(ctx, v_next);
            tile_chain(ctx, NC_TILE_CONSTRAINTS, dt2);
            tile_grips(ctx);
            if (self && !fruits) tile_insert(ctx);
            tile_store(ctx, x_next);
        }
        if (ctx.tid == 0u) *d.yarn_list_n = 0u;
        ctx.gx = x_next;
        ctx.gv = v_next;
        NC_SYNC(ctx);
    }
    // 2. fruit/yarn colours, self-contact insert
    if (fruits) {
        float4* x_next = other_x(ctx);
        if (!ctx.fruit_cta) {
            tile_load(ctx, NC_TILE_YARN);
            tile_yarn(ctx);
            if (self) tile_insert(ctx);
            tile_store(ctx, x_next);
        }
        ctx.gx = x_next;
        ctx.fruit_pending = true;
        NC_SYNC(ctx);
    }
    // 3. self-contact solve + ground, strain sweeps, finalize
    const uint32_t sweeps = max(s.strain_sweeps, 1u);
    for (uint32_t sw = 0; sw < sweeps; ++sw) {
        float4* x_next = other_x(ctx);
        const bool final_sweep = sw + 1u == sweeps;
        if (ctx.fruit_cta) {
            if (sw == 0u) {
                fruit_flush(ctx);
                if (ctx.c.ground) fruit_ground(ctx);
                fruit_finalize(ctx);
                // the friction sweep's recorded segments, while the tiles
                // run the strain colours
                if (s.frictions && fruits) friction_stage(ctx);
            }
        } else {
            tile_load(ctx, NC_TILE_STRAIN);
            if (sw == 0u) tile_self_ground(ctx, self);
            if (s.strain_sweeps > 0u) tile_chain(ctx, NC_TILE_STRAIN, dt2);
            if (final_sweep) tile_finalize(ctx);
            tile_store(ctx, x_next);
        }
        ctx.gx = x_next;
        NC_SYNC(ctx);
    }
    // 4. frictions on the fruit CTA, the next substep's grip attach.  The
    // next substep's first phase reads nothing this phase writes unless the
    // friction sweep has listed segments (it changes their particles'
    // velocities) or the grips re-attach: otherwise no CTA waits here, and
    // the fruit CTA's tail overlaps the tiles' next predict and constraint
    // chain (the fruit CTA's own next phase follows its tail; the barrier
    // after that phase joins every CTA).  Every CTA takes the decision from
    // the configs and the list count, which no CTA changes before every CTA
    // has read it (the next substep's reset of the count runs only past
    // this barrier when the count is not zero).
    const bool friction_sweep = s.frictions && d.f_count > 0u;
    bool hold = last;
    if (!last) {
        const SubCfg next = nc::load_cfg(d.cfg + s.cfg_offset + ctx.sub + 1u);
        const bool attach = next.grip_active && (!ctx.c.grip_active || next.grip_gen != ctx.c.grip_gen);
        hold = attach || (friction_sweep && __ldcg(d.yarn_list_n) != 0u);
    }
    if (friction_sweep) yarn_friction_sweep(ctx);
    fruit_tail(ctx, last, friction_sweep);
    if (ctx.grip_cta && !last) {
        Ctx next = ctx;
        next.c = nc::load_cfg(d.cfg + s.cfg_offset + ctx.sub + 1u);
        grip_attach(next);
    }
    if (hold) NC_SYNC(ctx);
    return true;
}

}  // namespace
}  // namespace nc
