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
//   3. with self contact: its phase A and the ground clamp of the owned
//      particles, then (after the barrier, and only where phase A listed
//      pairs) its ordered pass on CTA 0 and one more barrier; strain
//      colours (without self contact the closure's ground clamp first),
//      finalize and cloth/ground friction of the owned particles; fruit
//      CTA: fruit sums, ground and finalize (more strain sweeps: one phase
//      each);
//   4. fruit CTA: fruit/yarn friction, fruit frictions, orientation,
//      release; CTA 0: the next substep's grip attach;
// with one grid barrier after each, instead of one per colour; after
// phase 4 only where the next substep needs one (a grip re-attach, the
// launch's last substep, a friction list too long to stage): otherwise a
// tile CTA whose next predict reads velocities the friction sweep rewrote
// waits for the fruit CTA's flag, and the others go on.
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

// The owned particles (the list's first) from the current position buffer.
__device__ __forceinline__ void tile_load_owned(const Ctx& ctx) {
    const uint32_t own = ctx.tp[1];
    const uint32_t* gi = tile_list(ctx);
    for (uint32_t l = threadIdx.x; l < own; l += blockDim.x) ctx.tx[l] = __ldcg(ctx.gx + gi[l]);
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

// Self-contact phase A (the ordered pass follows the barrier) and the
// ground clamp of the first nl local particles (the owned ones, or the
// strain chain's closure where the ground clamp alone runs there).
__device__ void tile_self_ground(const Ctx& ctx, bool self, uint32_t nl) {
    const SubCfg& c = ctx.c;
    const uint32_t* gi = tile_list(ctx);
    const uint32_t tag = self_pass_tag(ctx, 0u);
    unsigned long long contacts = 0ull;
    float max_pen = 0.0f;
    for (uint32_t l = threadIdx.x; l < nl; l += blockDim.x) {
        float4 p = ctx.tx[l];
        if (self) {
            float4 q;
#ifdef NC_SELF_ORDER_KERNELS
            if (self_exact_one(ctx, tag, gi[l], p, q, contacts, max_pen)) p = q;
#else
            if (self_solve_one(ctx, tag, gi[l], p, q, contacts, max_pen)) p = q;
#endif
        }
        if (c.ground && c.radius - p.z > 0.0f) p = make_float4(p.x, p.y, c.radius, p.w);
        ctx.tx[l] = p;
    }
#ifdef NC_SELF_ORDER_KERNELS
    if (self) self_pass_flush(ctx.d, contacts, max_pen);
#else
    if (self) self_stats_flush(ctx.d, contacts, max_pen);
#endif
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

// With the per-barrier trace on, a middle tile CTA stamps the end of each
// step inside the phases into trace slots 64 and up (a CTA barrier first,
// so the stamp follows the step's last thread).
#define NC_TILE_MARK_SLOT 64u
__device__ __forceinline__ void tile_mark(const Ctx& ctx, uint32_t k) {
    const DeviceCloth& d = ctx.d;
    if (d.trace == nullptr || ctx.rank != ctx.ranks / 2u) return;
    __syncthreads();
    if (threadIdx.x == 0 && NC_TILE_MARK_SLOT + k < NC_TRACE_SLOTS)
        d.trace[static_cast<size_t>(ctx.sub) * NC_TRACE_SLOTS + NC_TILE_MARK_SLOT + k] = globaltimer();
}

// The fruit CTA's own stamps (trace slots NC_FRUIT_MARK_SLOT and up).
#define NC_FRUIT_MARK_SLOT 100u
__device__ __forceinline__ void fruit_mark(const Ctx& ctx, uint32_t k) {
    const DeviceCloth& d = ctx.d;
    if (d.trace == nullptr || !ctx.fruit_cta) return;
    __syncthreads();
    if (threadIdx.x == 0 && NC_FRUIT_MARK_SLOT + k < NC_TRACE_SLOTS)
        d.trace[static_cast<size_t>(ctx.sub) * NC_TRACE_SLOTS + NC_FRUIT_MARK_SLOT + k] = globaltimer();
}

// Row and column of a particle of a grid cloth (row-major), else (0, index).
__device__ __forceinline__ uint2 tile_cell(const DeviceCloth& d, uint32_t i) {
    return d.grid_width != 0u ? make_uint2(i / d.grid_width, i % d.grid_width) : make_uint2(0u, i);
}

// The bounding box, in rows and columns (or indices), of the particles this
// CTA predicts in a substep's first phase (chain 0's closure); once per
// launch.
__device__ uint4 tile_closure_box(const Ctx& ctx) {
    __shared__ uint32_t s_box[4];
    if (threadIdx.x == 0) {
        s_box[0] = s_box[2] = 0xffffffffu;
        s_box[1] = s_box[3] = 0u;
    }
    __syncthreads();
    const uint32_t nl = ctx.tp[4u + NC_TILE_CONSTRAINTS];
    const uint32_t* gi = tile_list(ctx);
    uint32_t r0 = 0xffffffffu, r1 = 0u, c0 = 0xffffffffu, c1 = 0u;
    for (uint32_t l = threadIdx.x; l < nl; l += blockDim.x) {
        const uint2 rc = tile_cell(ctx.d, gi[l]);
        r0 = min(r0, rc.x);
        r1 = max(r1, rc.x);
        c0 = min(c0, rc.y);
        c1 = max(c1, rc.y);
    }
    atomicMin(&s_box[0], r0);
    atomicMax(&s_box[1], r1);
    atomicMin(&s_box[2], c0);
    atomicMax(&s_box[3], c1);
    __syncthreads();
    const uint4 box = make_uint4(s_box[0], s_box[1], s_box[2], s_box[3]);
    __syncthreads();
    return box;
}

// Whether a friction-listed segment may touch a particle this CTA predicts
// in the next substep's first phase (its closure box: a superset), whose
// velocity the friction sweep rewrites.  Tile CTAs.
__device__ bool tile_touches_listed(const Ctx& ctx, uint32_t listed) {
    const DeviceCloth& d = ctx.d;
    const uint4 b = ctx.tile_box;
    bool hit = false;
    for (uint32_t k = threadIdx.x; k < listed; k += blockDim.x) {
        const uint2 ij = __ldg(d.d_ij + __ldcg(d.yarn_list + k));
        const uint2 p = tile_cell(d, ij.x), q = tile_cell(d, ij.y);
        hit = hit || (p.x >= b.x && p.x <= b.y && p.y >= b.z && p.y <= b.w) ||
              (q.x >= b.x && q.x <= b.y && q.y >= b.z && q.y <= b.w);
    }
    return __syncthreads_or(hit) != 0;
}

// Wait (bounded) until the fruit CTA has finished the friction sweep of
// substep `done` - 1 of this launch; false when the wait gave up or another
// CTA aborted.
__device__ bool tile_wait_fruit(const Ctx& ctx, unsigned long long done) {
    const DeviceCloth& d = ctx.d;
    __shared__ unsigned s_fruit_abort;
    if (threadIdx.x == 0) {
        const unsigned limit = d.spin_limit != 0u ? d.spin_limit : NC_BARRIER_SPIN_LIMIT;
        unsigned ab = 0u;
        unsigned spins = 0u;
        while (ld_relaxed_u64(d.fruit_flag) < done) {
            ++spins;
            if ((spins & 63u) == 0u && ld_acquire(d.abort_flag) != 0u) {
                ab = 1u;
                break;
            }
            if (spins > limit) {
                atomicOr(d.failure, NUMI_CLOTH_FAILURE_TIMEOUT);
                atomicExch(d.abort_flag, 1u);
                ab = 1u;
                break;
            }
        }
        if (!ab) (void)ld_acquire_u64(d.fruit_flag);
        s_fruit_abort = ab;
    }
    __syncthreads();
    return s_fruit_abort == 0u;
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
            fruit_mark(ctx, 0u);
            fruit_begin(ctx);
            fruit_mark(ctx, 1u);
            if (d.p_count > 0u) {
                __syncthreads();
                fruit_pair_sweep(d, *ctx.fs, ctx.c.dt);
            }
            fruit_mark(ctx, 2u);
        } else {
            // the previous substep's friction rewrote velocities this CTA
            // predicts: wait for the fruit CTA's tail
            if (ctx.fruit_wait && !tile_wait_fruit(ctx, ctx.sub)) return false;
            ctx.fruit_wait = false;
            tile_mark(ctx, 0u);
            tile_predict(ctx, v_next);
            tile_mark(ctx, 1u);
            tile_chain(ctx, NC_TILE_CONSTRAINTS, dt2);
            tile_mark(ctx, 2u);
            tile_grips(ctx);
            if (self && !fruits) tile_insert(ctx);
            tile_store(ctx, x_next);
            tile_mark(ctx, 3u);
        }
        // the friction list restarts empty: here on a launch's first
        // substep, at the end of the fruit CTA's tail on the others
        if (ctx.tid == 0u && ctx.sub == 0u) *d.yarn_list_n = 0u;
        ctx.gx = x_next;
        ctx.gv = v_next;
        NC_SYNC(ctx);
    }
    // 2. fruit/yarn colours, self-contact insert
    if (fruits) {
        float4* x_next = other_x(ctx);
        if (!ctx.fruit_cta) {
            tile_mark(ctx, 4u);
            tile_load(ctx, NC_TILE_YARN);
            tile_mark(ctx, 5u);
            tile_yarn(ctx);
            tile_mark(ctx, 6u);
            if (self) tile_insert(ctx);
            tile_mark(ctx, 7u);
            tile_store(ctx, x_next);
            tile_mark(ctx, 8u);
        }
        ctx.gx = x_next;
        ctx.fruit_pending = true;
        NC_SYNC(ctx);
    }
    // 3. self-contact solve + ground, strain sweeps, finalize.  Every CTA
    // decides here, alike, whether a grid barrier must follow the fruit
    // CTA's tail (phase 4): the next substep's first phase reads nothing
    // the tail writes except the velocities the friction sweep rewrites and
    // the grips a re-attach rewrites.  Without a re-attach (or the launch's
    // end, or a list too long to stage) there is no barrier: a tile CTA
    // whose predict closure holds a listed segment's particle waits for the
    // fruit CTA's flag before its next predict, the others go on.  The
    // list and its count stay unchanged until the fruit CTA's tail resets
    // them, after this phase's barrier.
    const bool friction_sweep = s.frictions && d.f_count > 0u;
    {
        const uint32_t listed = friction_sweep ? min(__ldcg(d.yarn_list_n), d.d_count) : 0u;
        bool attach = false;
        if (!last) {
            const SubCfg next = nc::load_cfg(d.cfg + s.cfg_offset + ctx.sub + 1u);
            attach = next.grip_active && (!ctx.c.grip_active || next.grip_gen != ctx.c.grip_gen);
        }
        ctx.hold_tail = last || attach || listed > NC_FRICTION_STAGE;
        if (!ctx.hold_tail && listed > 0u && !ctx.fruit_cta) ctx.fruit_wait = tile_touches_listed(ctx, listed);
    }
    // With self contact the owners first resolve their own particles' self
    // contact (phase A) and ground clamp and publish them (one more grid
    // barrier), the ordered pass follows where phase A listed pairs, and the
    // strain chains then load resolved positions.
    const bool split = self;
    if (split) {
        float4* x_next = other_x(ctx);
        if (ctx.fruit_cta) {
            fruit_mark(ctx, 3u);
            fruit_flush(ctx);
            fruit_mark(ctx, 4u);
            if (ctx.c.ground) fruit_ground(ctx);
            fruit_finalize(ctx);
            fruit_mark(ctx, 5u);
            if (s.frictions && fruits) friction_stage(ctx);
            fruit_mark(ctx, 6u);
        } else {
            tile_mark(ctx, 9u);
            tile_load_owned(ctx);
            tile_mark(ctx, 10u);
            tile_self_ground(ctx, true, ctx.tp[1]);
            tile_mark(ctx, 11u);
            tile_store(ctx, x_next);
        }
        ctx.gx = x_next;
        NC_SYNC(ctx);
#ifdef NC_SELF_ORDER_KERNELS
        if (!self_settle(ctx, 0u)) return false;
#endif
    }
    const uint32_t sweeps = max(s.strain_sweeps, 1u);
    for (uint32_t sw = 0; sw < sweeps; ++sw) {
        float4* x_next = other_x(ctx);
        const bool final_sweep = sw + 1u == sweeps;
        if (ctx.fruit_cta) {
            if (sw == 0u && !split) {
                fruit_flush(ctx);
                if (ctx.c.ground) fruit_ground(ctx);
                fruit_finalize(ctx);
                // the friction sweep's recorded segments, while the tiles
                // run the strain colours
                if (s.frictions && fruits) friction_stage(ctx);
            }
        } else {
            if (!split) tile_mark(ctx, 9u);
            tile_load(ctx, NC_TILE_STRAIN);
            if (!split) tile_mark(ctx, 10u);
            if (sw == 0u && !split) tile_self_ground(ctx, false, ctx.tp[4u + NC_TILE_STRAIN]);
            tile_mark(ctx, 11u);
            if (s.strain_sweeps > 0u) tile_chain(ctx, NC_TILE_STRAIN, dt2);
            tile_mark(ctx, 12u);
            if (final_sweep) tile_finalize(ctx);
            tile_mark(ctx, 13u);
            tile_store(ctx, x_next);
            tile_mark(ctx, 14u);
        }
        ctx.gx = x_next;
        NC_SYNC(ctx);
    }
    // 4. frictions on the fruit CTA, the next substep's grip attach (the
    // barrier after it only where phase 3 decided so).  The fruit CTA
    // releases its flag as soon as the friction sweep has written the
    // velocities back: the rest of its tail touches only fruit state.
    fruit_mark(ctx, 7u);
    if (friction_sweep) yarn_friction_sweep(ctx);
    fruit_mark(ctx, 8u);
    if (ctx.fruit_cta) {
        __syncthreads();   // the sweep's velocity stores and list reads are done
        if (threadIdx.x == 0) {
            *d.yarn_list_n = 0u;
            asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(d.fruit_flag),
                         "l"(static_cast<unsigned long long>(ctx.sub) + 1ull)
                         : "memory");
        }
    }
    fruit_tail(ctx, last, friction_sweep);
    fruit_mark(ctx, 9u);
    if (ctx.grip_cta && !last) {
        Ctx next = ctx;
        next.c = nc::load_cfg(d.cfg + s.cfg_offset + ctx.sub + 1u);
        grip_attach(next);
    }
    if (ctx.hold_tail) {
        ctx.fruit_wait = false;
        NC_SYNC(ctx);
    }
    return true;
}

}  // namespace
}  // namespace nc
