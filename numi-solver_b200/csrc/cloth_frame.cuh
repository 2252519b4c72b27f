// The frame kernel: all phases of `substeps` substeps in one cooperative
// launch.  See cloth_kernels.cuh for the phase order and the per-phase
// equations.
#pragma once

#include "cloth_kernels.cuh"

// Dynamic shared memory of a frame: the cloth descriptor, the fruit CTA's
// state, then either (resident mode) the CTA's particle positions and
// velocities or (neighbour syncs) the CTA's colour item lists.
__host__ __device__ constexpr size_t nc_round256(size_t b) { return (b + 255u) & ~size_t(255u); }
__host__ __device__ constexpr size_t nc_fruit_offset() { return nc_round256(sizeof(DeviceCloth)); }
__host__ __device__ constexpr size_t nc_resident_offset() { return nc_round256(nc_fruit_offset() + sizeof(FruitShared)); }

namespace nc {
namespace {   // internal linkage: the edge kernels' unit includes these too

// FP64 scratch of the CTA-wide reductions (air-load chunk sums, the air
// attenuation, the residual maxima).  They run in different phases and each
// ends with a CTA barrier, so they share one array.
__shared__ __align__(16) double nc_red_smem[3][NC_BLOCK_MAX];

// Grid-wide barrier with a bounded wait.  Arrival is a release-add of 1 to
// a counter the host zeroes before each launch; barrier number s of the
// launch completes when an acquire load sees s times the number of CTAs on
// the cloth.  A CTA that waits past the limit
// raises TIMEOUT and the abort flag, and every CTA leaves at its next
// barrier (or as soon as it sees the flag while waiting).
__device__ bool grid_sync(Ctx& ctx) {
    const DeviceCloth& d = ctx.d;
    ++ctx.barriers;
    ++ctx.seq;
    if (d.trace_cta && ctx.barriers <= NC_TRACE_SLOTS) {
        __syncthreads();
        if (threadIdx.x == 0)
            d.trace_cta[(static_cast<size_t>(ctx.sub) * NC_TRACE_SLOTS + ctx.barriers - 1u) * ctx.ranks + ctx.rank] =
                globaltimer();
    }
    if (d.cluster_barrier) {
        cooperative_groups::this_cluster().sync();
        if (d.trace && ctx.rank == 0 && threadIdx.x == 0 && ctx.barriers <= NC_TRACE_SLOTS)
            d.trace[static_cast<size_t>(ctx.sub) * NC_TRACE_SLOTS + ctx.barriers - 1u] = globaltimer();
        return true;
    }
    if (ctx.ranks == 1) {
        __syncthreads();
        if (d.tape != nullptr && ctx.barriers < d.tape_slots) {
            // adjoint tape: positions after this barrier
            float4* slot = d.tape + (static_cast<size_t>(ctx.sub) * d.tape_slots + ctx.barriers) * d.n;
            for (uint32_t i = threadIdx.x; i < d.n; i += blockDim.x) slot[i] = px(ctx, i);
            __syncthreads();
        }
        if (d.trace && threadIdx.x == 0 && ctx.barriers <= NC_TRACE_SLOTS)
            d.trace[static_cast<size_t>(ctx.sub) * NC_TRACE_SLOTS + ctx.barriers - 1u] = globaltimer();
        return true;
    }
    __shared__ unsigned s_abort;
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned long long target = ctx.seq * (ctx.ranks + d.bar_phantom);
        const unsigned limit = d.spin_limit != 0u ? d.spin_limit : NC_BARRIER_SPIN_LIMIT;
        red_release_add_u64(d.bar_count, 1ull);
        unsigned ab = 0u;
        unsigned spins = 0u;
        // poll relaxed; one acquire load once the count is reached (the
        // count only grows)
        while (ld_relaxed_u64(d.bar_count) < target) {
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
        // no fence besides: the acquire load that sees the count orders this
        // thread after every arrival's release, and the CTA barrier below
        // orders the CTA's other threads after this thread
        if (!ab) (void)ld_acquire_u64(d.bar_count);
        s_abort = ab;
        if (d.trace && ctx.rank == 0 && ctx.barriers <= NC_TRACE_SLOTS)
            d.trace[static_cast<size_t>(ctx.sub) * NC_TRACE_SLOTS + ctx.barriers - 1u] = globaltimer();
    }
    __syncthreads();
    return s_abort == 0u;
}

#define NC_SYNC(ctx) \
    do { if (!grid_sync(ctx)) return false; } while (0)

// Neighbour syncs: this CTA's neighbour CTAs (static shared memory) and its
// colour item lists (dynamic shared memory after the fruit state: the
// colour_slots + 1 list offsets, then the batch-relative item indices),
// staged at the start of a launch.  Each CTA's finished-colour count has
// its own 128-byte line.
#define NC_NBR_MAX 64u
#define NC_NBR_FLAG_STRIDE 32u
__shared__ uint32_t nc_nbr[NC_NBR_MAX];
__shared__ uint32_t nc_nbr_count;
extern __shared__ __align__(16) unsigned char nc_frame_smem[];

__device__ __forceinline__ uint32_t* colour_lists() {
    return reinterpret_cast<uint32_t*>(nc_frame_smem + nc_resident_offset());
}

__device__ __forceinline__ void neighbour_stage(const Ctx& ctx) {
    const DeviceCloth& d = ctx.d;
    if (!d.nbr_on) return;
    const uint32_t lo = d.nbr_off[ctx.rank], hi = d.nbr_off[ctx.rank + 1u];
    for (uint32_t k = threadIdx.x; k < hi - lo; k += blockDim.x) nc_nbr[k] = d.nbr_idx[lo + k];
    if (threadIdx.x == 0) nc_nbr_count = hi - lo;
    const uint32_t w0 = d.nbr_block[ctx.rank], w1 = d.nbr_block[ctx.rank + 1u];
    uint32_t* lists = colour_lists();
    for (uint32_t k = threadIdx.x; k < w1 - w0; k += blockDim.x) lists[k] = d.nbr_items[w0 + k];
    __syncthreads();
}

// Positions of colour batch `slot` that this thread takes: in the CTA's
// list when neighbour syncs run, else the grid-stride range of the batch
// (count items).  colour_item maps a position to the batch-relative item.
__device__ __forceinline__ Range colour_items(const Ctx& ctx, uint32_t slot, uint32_t count) {
    if (ctx.d.nbr_on) {
        const uint32_t* lists = colour_lists();
        return Range{lists[slot] + threadIdx.x, lists[slot + 1u], blockDim.x};
    }
    return item_range(ctx, count);
}
__device__ __forceinline__ uint32_t colour_item(const Ctx& ctx, uint32_t pos) {
    return ctx.d.nbr_on ? colour_lists()[ctx.d.colour_slots + 1u + pos] : pos;
}

// Barrier between two constraint colours.  With neighbour syncs the CTA
// publishes the colours it has finished (a release store after the CTA
// barrier) and waits until each neighbour has finished as many (acquire):
// every CTA that touches one of its particles in any colour is then done
// with the previous colour, and none can be more than one colour ahead, so
// the colour order of every particle is the grid barrier's.  Bounded as the
// grid barrier.
__device__ bool colour_sync(Ctx& ctx) {
    const DeviceCloth& d = ctx.d;
    if (!d.nbr_on) return grid_sync(ctx);
    ++ctx.barriers;
    const unsigned target = ++ctx.nseq;
    __syncthreads();
    if (threadIdx.x == 0) st_release(d.nbr_flag + NC_NBR_FLAG_STRIDE * ctx.rank, target);
    int ab = 0;
    if (threadIdx.x < nc_nbr_count) {
        const unsigned* f = d.nbr_flag + NC_NBR_FLAG_STRIDE * nc_nbr[threadIdx.x];
        const unsigned limit = d.spin_limit != 0u ? d.spin_limit : NC_BARRIER_SPIN_LIMIT;
        unsigned spins = 0u;
        while (ld_relaxed(f) < target) {
            ++spins;
            if ((spins & 63u) == 0u && ld_acquire(d.abort_flag) != 0u) {
                ab = 1;
                break;
            }
            if (spins > limit) {
                atomicOr(d.failure, NUMI_CLOTH_FAILURE_TIMEOUT);
                atomicExch(d.abort_flag, 1u);
                ab = 1;
                break;
            }
        }
        if (!ab) (void)ld_acquire(f);
    }
    const int any = __syncthreads_or(ab);
    if (d.trace && ctx.rank == 0 && threadIdx.x == 0 && ctx.barriers <= NC_TRACE_SLOTS)
        d.trace[static_cast<size_t>(ctx.sub) * NC_TRACE_SLOTS + ctx.barriers - 1u] = globaltimer();
    return any == 0;
}

#define NC_CSYNC(ctx, colour_next) \
    do { if (!((colour_next) ? colour_sync(ctx) : grid_sync(ctx))) return false; } while (0)

// Apply (and clear) the fixed-point fruit displacement sums.  Fruit CTA.
__device__ void fruit_flush(Ctx& ctx) {
    if (!ctx.fruit_pending) return;
    ctx.fruit_pending = false;
    if (!ctx.fruit_cta) return;
    const DeviceCloth& d = ctx.d;
    // the barrier before this phase completed every add: plain loads, and
    // stores of zero for the next sweep
    unsigned long long* acc = reinterpret_cast<unsigned long long*>(d.fruit_partial);
    for (uint32_t f = threadIdx.x; f < d.f_count; f += blockDim.x) {
        NumiClothFruit& fr = d.fruits[f];
        const unsigned long long ax = __ldcg(acc + 3u * f + 0u);
        const unsigned long long ay = __ldcg(acc + 3u * f + 1u);
        const unsigned long long az = __ldcg(acc + 3u * f + 2u);
        const numi_float4 p = fr.positionAndInverseMass;
        acc[3u * f + 0u] = 0ull;
        acc[3u * f + 1u] = 0ull;
        acc[3u * f + 2u] = 0ull;
        fr.positionAndInverseMass = nf4<numi_float4>(p.x + from_fixed(ax), p.y + from_fixed(ay), p.z + from_fixed(az), p.w);
    }
    __syncthreads();
}

// ------------------------------------------------------------ phases -----

// Predict of one particle (tools/cloth_bag.cpp:4788-4826): gravity,
// damping and (air load off) the advance with the swept ground clamp, from
// position p and velocity vv; a particle of zero inverse mass follows its
// rest position.  prev is xyz(p).
__device__ __forceinline__ void predict_particle(const Ctx& ctx, uint32_t i, const float4& p, const float4& vv,
                                                 bool air, V3& pos, V3& vel) {
    const DeviceCloth& d = ctx.d;
    const SubCfg& c = ctx.c;
    const float dt = c.dt;
    const float inv_dt = 1.0f / dt;
    const float damp = d.damping >= 0.0f ? d.damping : ctx.s.damping;
    pos = xyz(p);
    const V3 prev = pos;
    vel = xyz(vv);
    if (p.w == 0.0f) {
        pos = xyz(__ldg(d.rest + i));
        vel = (pos - prev) * inv_dt;
    } else {
        vel = vel + c.gravity * dt;
        if (damp != 0.0f) vel = vel * (1.0f / (1.0f + damp * dt));
        if (!air) {
            pos = pos + vel * dt;
        }
    }
    if (!air && ctx.s.swept_ground && c.ground && prev.z >= c.radius && pos.z < c.radius) pos.z = c.radius;
}

__device__ void fruit_begin(Ctx& ctx);

// Grip attach + begin + advance (+ swept ground), aero off.
__device__ void phase_begin(Ctx& ctx) {
    const DeviceCloth& d = ctx.d;
    if (ctx.grip_cta) {
        // on one CTA the attach reads the positions before this CTA
        // predicts them; on more it ran at the end of the previous substep
        // (or before the launch's first), where every position is final
        if (ctx.ranks == 1u) grip_attach(ctx);
        __syncthreads();
        for (uint32_t g = threadIdx.x; g < d.g_count; g += blockDim.x) {
            d.grips[g].lambda.x = 0.0f;
            d.grips[g].lambda.y = 0.0f;
            d.grips[g].lambda.z = 0.0f;
        }
    }
    const bool air = ctx.s.aerodynamics != 0u;
    for (Range r = particle_range(ctx); r.i < r.end; r.i += r.stride) {
        const uint32_t i = r.i;
        float4 p = px(ctx, i);
        const float4 pp = ld(d.xp + i);
        V3 pos, vel;
        predict_particle(ctx, i, p, pv(ctx, i), air, pos, vel);
        d.xp[i] = make_float4(p.x, p.y, p.z, pp.w);
        px_set(ctx, i, with_xyz(p, pos));
        pv_set(ctx, i, make_float4(vel.x, vel.y, vel.z, vel.z));
    }
    if (ctx.tid == 0u) *d.yarn_list_n = 0u;
    for (uint32_t k = ctx.tid; k < d.d_count; k += ctx.nthreads) d.d_lambda[k] = 0.0f;
    for (uint32_t k = ctx.tid; k < d.k_count; k += ctx.nthreads) d.k_lambda[k] = 0.0f;
    for (uint32_t k = ctx.tid; k < d.b_count; k += ctx.nthreads) d.b_lambda[k] = 0.0f;
    fruit_begin(ctx);
}

// The fruits' part of the substep start (fruit CTA): predict with the
// swept ground, and the pair contact records cleared.
__device__ void fruit_begin(Ctx& ctx) {
    const DeviceCloth& d = ctx.d;
    const SubCfg& c = ctx.c;
    const float dt = c.dt;
    const bool air = ctx.s.aerodynamics != 0u;
    if (ctx.fruit_cta) {
        for (uint32_t f = threadIdx.x; f < d.f_count; f += blockDim.x) {
            FruitState s = load_fruit(d.fruits[f]);
            s.prev = s.x;
            s.v = s.v + c.gravity * dt;
            s.ground_impulse = 0.0f;
            if (air) fruit_air(s, c);
            s.x = s.x + s.v * dt;
            if (ctx.s.swept_ground && c.ground && s.prev.z >= s.radius && s.x.z < s.radius) {
                const float adv = s.radius - s.x.z;
                s.ground_impulse = s.ground_impulse + adv / (s.w * dt);
                s.x.z = s.radius;
            }
            store_fruit(d.fruits[f], s);
        }
        for (uint32_t k = threadIdx.x; k < d.p_count; k += blockDim.x) ctx.fs->contact[k] = make_float4(0, 0, 0, 0);
        if (threadIdx.x == 0) ctx.fs->loaded = 0ull;
    }
}

// Yarn air load (tools/cloth_bag.cpp:1013-1107): forces per yarn colour
// (conflict-free), FP64 fixed-tree reductions of drag power and
// inverse-mass-weighted force squared, then v += f * att * w * dt and the
// deferred advance + swept ground.
__device__ void air_force_batch(Ctx& ctx, const Batch& bt, float4* force) {
    const DeviceCloth& d = ctx.d;
    const SubCfg& c = ctx.c;
    const float pi = 3.14159265358979323846f;
    for (Range r = item_range(ctx, bt.yarn); r.i < r.end; r.i += r.stride) {
        const uint32_t s = bt.first + r.i;
        const uint2 ij = __ldg(d.d_ij + s);
        const V3 a = xyz(px(ctx, ij.x));
        const V3 b = xyz(px(ctx, ij.y));
        const V3 span = b - a;
        const float L = len3(span);
        if (L < 1.0e-12f) continue;
        const V3 axis = vdiv(span, L);
        const V3 rel = (xyz(pv(ctx, ij.x)) + xyz(pv(ctx, ij.y))) * 0.5f - c.air;
        const V3 axial = axis * dot3(rel, axis);
        const V3 cross_v = rel - axial;
        const float cross_area = 2.0f * c.radius * L;
        const float wet_area = 2.0f * pi * c.radius * L;
        const float ccoef = 0.5f * c.air_density * c.aero.x * cross_area;
        const float scoef = 0.5f * c.air_density * c.aero.y * wet_area;
        V3 f1{0.0f, 0.0f, 0.0f};
        const float cs = len3(cross_v);
        if (!(cs < 1.0e-14f || ccoef <= 0.0f)) f1 = cross_v * (-ccoef * cs);
        V3 f2{0.0f, 0.0f, 0.0f};
        const float as = len3(axial);
        if (!(as < 1.0e-14f || scoef <= 0.0f)) f2 = axial * (-scoef * as);
        const V3 f = f1 + f2;
        const V3 half = f * 0.5f;
        float4 fa = ld(force + ij.x);
        float4 fb = ld(force + ij.y);
        force[ij.x] = make_float4(fa.x + half.x, fa.y + half.y, fa.z + half.z, 0.0f);
        force[ij.y] = make_float4(fb.x + half.x, fb.y + half.y, fb.z + half.z, 0.0f);
    }
}

// Deterministic FP64 sum of two per-particle terms over 256-particle chunks
// with a fixed 256-wide tree (a 512-thread CTA reduces two chunks at once,
// each with the same tree); chunk partials land in red[2*chunk].
__device__ void air_reduce_chunks(Ctx& ctx, const float4* force) {
    const DeviceCloth& d = ctx.d;
    double* s_p = nc_red_smem[0];
    double* s_q = nc_red_smem[1];
    const uint32_t chunks = (d.n + NC_THREADS - 1u) / NC_THREADS;
    const uint32_t groups = blockDim.x / NC_THREADS;
    const uint32_t t = threadIdx.x % NC_THREADS;
    const uint32_t base = threadIdx.x - t;
    for (uint32_t first = ctx.rank * groups; first < chunks; first += ctx.ranks * groups) {
        const uint32_t ch = first + threadIdx.x / NC_THREADS;
        const uint32_t i = ch * NC_THREADS + t;
        double pw = 0.0, q = 0.0;
        if (ch < chunks && i < d.n) {
            const float4 p = px(ctx, i);
            if (p.w > 0.0f) {
                const V3 f = xyz(ld(force + i));
                const V3 rv = xyz(pv(ctx, i)) - ctx.c.air;
                pw = static_cast<double>(f.x) * rv.x + static_cast<double>(f.y) * rv.y +
                     static_cast<double>(f.z) * rv.z;
                q = static_cast<double>(p.w) * (static_cast<double>(f.x) * f.x +
                                                static_cast<double>(f.y) * f.y +
                                                static_cast<double>(f.z) * f.z);
            }
        }
        s_p[threadIdx.x] = pw;
        s_q[threadIdx.x] = q;
        __syncthreads();
        for (uint32_t st = NC_THREADS / 2u; st > 0u; st >>= 1u) {
            if (t < st) {
                s_p[base + t] += s_p[base + t + st];
                s_q[base + t] += s_q[base + t + st];
            }
            __syncthreads();
        }
        if (t == 0 && ch < chunks) {
            d.red[2u * ch] = s_p[base];
            d.red[2u * ch + 1u] = s_q[base];
        }
        __syncthreads();
    }
}

// Every CTA reduces the chunk partials with the same fixed tree (the first
// 256 threads; the tree shape does not depend on the launch).
__device__ float air_attenuation(Ctx& ctx) {
    const DeviceCloth& d = ctx.d;
    double* s_p = nc_red_smem[0];
    double* s_q = nc_red_smem[1];
    const uint32_t chunks = (d.n + NC_THREADS - 1u) / NC_THREADS;
    if (threadIdx.x < NC_THREADS) {
        double pw = 0.0, q = 0.0;
        for (uint32_t ch = threadIdx.x; ch < chunks; ch += NC_THREADS) {
            pw += __ldcg(d.red + 2u * ch);
            q += __ldcg(d.red + 2u * ch + 1u);
        }
        s_p[threadIdx.x] = pw;
        s_q[threadIdx.x] = q;
    }
    __syncthreads();
    for (uint32_t st = NC_THREADS / 2u; st > 0u; st >>= 1u) {
        if (threadIdx.x < st) {
            s_p[threadIdx.x] += s_p[threadIdx.x + st];
            s_q[threadIdx.x] += s_q[threadIdx.x + st];
        }
        __syncthreads();
    }
    const double power = s_p[0];
    const double wsq = s_q[0];
    __syncthreads();
    double att = 1.0;
    if (wsq > 0.0) att = power < 0.0 ? 1.0 / (1.0 + static_cast<double>(ctx.c.dt) * wsq / -power) : 0.0;
    return static_cast<float>(att);
}

__device__ void air_apply_advance(Ctx& ctx, const float4* force, float att) {
    const DeviceCloth& d = ctx.d;
    const SubCfg& c = ctx.c;
    const float dt = c.dt;
    for (Range r = particle_range(ctx); r.i < r.end; r.i += r.stride) {
        const uint32_t i = r.i;
        float4 p = px(ctx, i);
        const V3 prev = xyz(ld(d.xp + i));
        V3 vel = xyz(pv(ctx, i));
        V3 pos = xyz(p);
        if (p.w > 0.0f) {
            vel = vel + xyz(ld(force + i)) * (att * p.w * dt);
            pos = pos + vel * dt;
        }
        if (ctx.s.swept_ground && c.ground && prev.z >= c.radius && pos.z < c.radius) pos.z = c.radius;
        px_set(ctx, i, with_xyz(p, pos));
        pv_set(ctx, i, make_float4(vel.x, vel.y, vel.z, vel.z));
    }
}

// One yarn colour of the present fruit/yarn sweep
// (tools/cloth_bag.cpp:2955-3020, 3141-3176).  Fruit positions are the
// ones at the start of the sweep; each fruit's displacement is summed in
// fixed point and applied by fruit_flush.
//
// Warp broadphase: a warp bounds its 32 segments and keeps only the fruits
// whose centre lies inside that box grown by the contact distance.  Float
// subtraction is monotone, so a fruit outside the warp box also fails every
// per-segment box test; once a contact moves a segment its thread tests all
// remaining fruits again.  The result is identical to testing every fruit.
// CTA-level fixed-point fruit sums.  Integer addition is exact and
// associative, so adding a CTA's contributions in shared memory first and
// then its total once to the global sum gives the same bits as one global
// atomic per contribution, without hundreds of segments queueing on the
// same few addresses when a fruit rests on the cloth.
__device__ __forceinline__ void cta_sums_clear(unsigned long long* s, uint32_t count) {
    for (uint32_t k = threadIdx.x; k < count; k += blockDim.x) s[k] = 0ull;
}

__device__ __forceinline__ void cta_sums_add(unsigned long long* s, float v) {
    if (v != 0.0f) atomicAdd(s, static_cast<unsigned long long>(to_fixed(v)));
}

__device__ __forceinline__ void cta_sums_flush(unsigned long long* s, unsigned long long* g, uint32_t count) {
    __syncthreads();
    for (uint32_t k = threadIdx.x; k < count; k += blockDim.x) {
        const unsigned long long v = s[k];
        if (v != 0ull) atomicAdd(g + k, v);
    }
}

// Box test of a fruit against a yarn segment (the broadphase of the
// reference's per-fruit segment loop).
__device__ __forceinline__ bool fruit_near_segment(const float4& fs, const float4& pa, const float4& pb,
                                                   float radius) {
    const float target = fs.w + radius;
    return !(fs.x < fminf(pa.x, pb.x) - target || fs.x > fmaxf(pa.x, pb.x) + target ||
             fs.y < fminf(pa.y, pb.y) - target || fs.y > fmaxf(pa.y, pb.y) + target ||
             fs.z < fminf(pa.z, pb.z) - target || fs.z > fmaxf(pa.z, pb.z) + target);
}

// Friction contact records of one yarn segment during a sweep (see
// DeviceCloth::yarn_slot_a/b): the slot tags are loaded at the segment's
// first contact and kept in registers; the first record of a substep takes
// slot 0 without a search and retires the older ones.
struct SegRecords {
    uint32_t seg;
    bool loaded, live, was_live, recorded;
    uint32_t rtag[NC_YARN_SLOTS];

    __device__ explicit SegRecords(uint32_t s)
        : seg(s), loaded(false), live(false), was_live(false), recorded(false) {
#pragma unroll
        for (uint32_t q = 0; q < NC_YARN_SLOTS; ++q) rtag[q] = 0u;
    }

    // Add impulse imp along -n on fruit f with segment weights w0, w1.
    __device__ void add(const Ctx& ctx, uint32_t f, V3 n, float imp, float w0, float w1) {
        const DeviceCloth& d = ctx.d;
        if (!loaded) {
            loaded = true;
            live = __ldcg(d.yarn_live + seg) == ctx.epoch;
            was_live = live;
            if (live) {
#pragma unroll
                for (uint32_t q = 0; q < NC_YARN_SLOTS; ++q)
                    rtag[q] = __float_as_uint(__ldcg(&d.yarn_slot_b[seg * NC_YARN_SLOTS + q].z));
            }
        }
        const uint32_t tag = (ctx.epoch << 6) | f;
        int slot = -1;
        bool fresh = true;
        if (!live) {
            slot = 0;
        } else {
#pragma unroll
            for (uint32_t q = 0; q < NC_YARN_SLOTS; ++q) {
                if (rtag[q] == tag && fresh) {
                    slot = static_cast<int>(q);
                    fresh = false;
                }
            }
            if (fresh)
#pragma unroll
                for (uint32_t q = 0; q < NC_YARN_SLOTS; ++q)
                    if (slot < 0 && (rtag[q] >> 6) != (ctx.epoch & 0x3ffffffu)) slot = static_cast<int>(q);
        }
        if (slot < 0) {
            fail(d, NUMI_CLOTH_FAILURE_RANGE);
            return;
        }
        const uint32_t q = static_cast<uint32_t>(slot);
        float4 sa = make_float4(0, 0, 0, 0);
        float4 sb = make_float4(0, 0, __uint_as_float(tag), 0);
        if (!fresh) {
            sa = __ldcg(&d.yarn_slot_a[seg * NC_YARN_SLOTS + q]);
            sb = __ldcg(&d.yarn_slot_b[seg * NC_YARN_SLOTS + q]);
        }
        const V3 wn = V3{sa.x, sa.y, sa.z} - n * imp;
        sa = make_float4(wn.x, wn.y, wn.z, sa.w + imp);
        sb.x = sb.x + w0 * imp;
        sb.y = sb.y + w1 * imp;
        d.yarn_slot_a[seg * NC_YARN_SLOTS + q] = sa;
        d.yarn_slot_b[seg * NC_YARN_SLOTS + q] = sb;
#pragma unroll
        for (uint32_t r = 0; r < NC_YARN_SLOTS; ++r)
            if (r == q) rtag[r] = tag;
        if (q == 0u && fresh) {
#pragma unroll
            for (uint32_t r = 1; r < NC_YARN_SLOTS; ++r) {
                d.yarn_slot_b[seg * NC_YARN_SLOTS + r].z = __uint_as_float(0u);
                rtag[r] = 0u;
            }
        }
        live = true;
        recorded = true;
    }

    __device__ void finish(const Ctx& ctx) const {
        if (!recorded) return;
        ctx.d.yarn_live[seg] = ctx.epoch;
        // first record of the substep: the segment joins the friction list
        if (!was_live) ctx.d.yarn_list[atomicAdd(ctx.d.yarn_list_n, 1u)] = seg;
    }
};

// One warp's segments of a fruit/yarn colour (tools/cloth_bag.cpp:2955-3020,
// 3141-3176), each lane one segment (`valid` where it has one) on its loaded
// endpoints pa, pb; every lane of the warp takes part.
//
// Warp broadphase: a warp bounds its 32 segments and keeps only the fruits
// whose centre lies inside that box grown by the contact distance.  Float
// subtraction is monotone, so a fruit outside the warp box also fails every
// per-segment box test; once a contact moves a segment its thread tests all
// remaining fruits again.  The result is identical to testing every fruit,
// whichever segments share the warp.  The fruit displacement sums and the
// friction records are left to the segment's `owner`; another CTA that
// computes the same segment (a tile's ghost zone) only moves its copies of
// the endpoints.  Returns whether the lane's endpoints moved.
__device__ __forceinline__ bool yarn_warp_contacts(const Ctx& ctx, bool valid, bool owner, uint32_t seg, float4& pa,
                                                   float4& pb, const float4* s_fruit, const float* s_fw,
                                                   unsigned long long* s_sum) {
    const SubCfg& c = ctx.c;
    const uint32_t nf = ctx.d.f_count;
    const uint32_t lane = threadIdx.x & 31u;
    V3 lo{INFINITY, INFINITY, INFINITY}, hi{-INFINITY, -INFINITY, -INFINITY};
    if (valid) {
        lo = V3{fminf(pa.x, pb.x), fminf(pa.y, pb.y), fminf(pa.z, pb.z)};
        hi = V3{fmaxf(pa.x, pb.x), fmaxf(pa.y, pb.y), fmaxf(pa.z, pb.z)};
    }
    V3 wlo = lo, whi = hi;
    for (int o = 16; o > 0; o >>= 1) {
        wlo.x = fminf(wlo.x, __shfl_xor_sync(0xffffffffu, wlo.x, o));
        wlo.y = fminf(wlo.y, __shfl_xor_sync(0xffffffffu, wlo.y, o));
        wlo.z = fminf(wlo.z, __shfl_xor_sync(0xffffffffu, wlo.z, o));
        whi.x = fmaxf(whi.x, __shfl_xor_sync(0xffffffffu, whi.x, o));
        whi.y = fmaxf(whi.y, __shfl_xor_sync(0xffffffffu, whi.y, o));
        whi.z = fmaxf(whi.z, __shfl_xor_sync(0xffffffffu, whi.z, o));
    }
    // fruits near the warp's box, and (wide) near it grown by a margin:
    // while a segment's box stays within half the margin of the warp's
    // box, every fruit near it is on the wide mask
    const float margin = 8.0f * c.radius;
    unsigned long long mask = 0ull, wide = 0ull;
    for (uint32_t f0 = 0; f0 < nf; f0 += 32u) {
        const uint32_t f = f0 + lane;
        bool near = false, near_wide = false;
        if (f < nf) {
            const float4 fs = s_fruit[f];
            const float target = fs.w + c.radius;
            near = !(fs.x < wlo.x - target || fs.x > whi.x + target || fs.y < wlo.y - target ||
                     fs.y > whi.y + target || fs.z < wlo.z - target || fs.z > whi.z + target);
            const float reach = target + margin;
            near_wide = !(fs.x < wlo.x - reach || fs.x > whi.x + reach || fs.y < wlo.y - reach ||
                          fs.y > whi.y + reach || fs.z < wlo.z - reach || fs.z > whi.z + reach);
        }
        mask |= static_cast<unsigned long long>(__ballot_sync(0xffffffffu, near)) << f0;
        wide |= static_cast<unsigned long long>(__ballot_sync(0xffffffffu, near_wide)) << f0;
    }
    if (!valid || mask == 0ull) return false;
    // this segment's own candidates among the warp's: the box test the
    // loop applies, so the loop visits only fruits it would not skip
    {
        unsigned long long own = 0ull;
        for (unsigned long long m = mask; m != 0ull; m &= m - 1ull) {
            const uint32_t f = static_cast<uint32_t>(__ffsll(static_cast<long long>(m)) - 1);
            if (fruit_near_segment(s_fruit[f], pa, pb, c.radius)) own |= 1ull << f;
        }
        mask = own;
    }
    bool changed = false;
    SegRecords rec(seg);
    while (mask != 0ull) {
        const uint32_t f = static_cast<uint32_t>(__ffsll(static_cast<long long>(mask)) - 1);
        mask &= mask - 1ull;
        const float4 fs = s_fruit[f];
        const V3 X{fs.x, fs.y, fs.z};
        const float target = fs.w + c.radius;
        if (!fruit_near_segment(fs, pa, pb, c.radius)) continue;
        V3 closest;
        float t;
        point_segment(X, xyz(pa), xyz(pb), closest, t);
        V3 sep = closest - X;
        float dist = len3(sep);
        if (dist >= target) continue;
        if (dist < 1.0e-12f) {
            const V3 sd = normalized3(xyz(pb) - xyz(pa));
            sep = normalized3(cross3(sd, fabsf(sd.z) < 0.9f ? V3{0.0f, 0.0f, 1.0f} : V3{1.0f, 0.0f, 0.0f}));
            dist = 0.0f;
        }
        const V3 n = normalized3(sep);
        const float w0 = 1.0f - t;
        const float w1 = t;
        const float corr = target - dist;
        V3 delta{0.0f, 0.0f, 0.0f};
        const float lam = yarn_correction(pa, pb, w0, w1, s_fw[f], n, corr, c.ground, c.radius, delta);
        // the segment moved: its candidates are the later fruits near its
        // new box (those on the wide mask while the box stays within half
        // the margin of the warp's box, else any fruit)
        changed = true;
        mask = 0ull;
        const float half = 0.5f * margin;
        const bool inside = fminf(pa.x, pb.x) >= wlo.x - half && fmaxf(pa.x, pb.x) <= whi.x + half &&
                            fminf(pa.y, pb.y) >= wlo.y - half && fmaxf(pa.y, pb.y) <= whi.y + half &&
                            fminf(pa.z, pb.z) >= wlo.z - half && fmaxf(pa.z, pb.z) <= whi.z + half;
        unsigned long long pool = inside ? wide : (nf >= 64u ? ~0ull : (1ull << nf) - 1ull);
        pool &= f + 1u < 64u ? (~0ull << (f + 1u)) : 0ull;
        for (; pool != 0ull; pool &= pool - 1ull) {
            const uint32_t g = static_cast<uint32_t>(__ffsll(static_cast<long long>(pool)) - 1);
            if (fruit_near_segment(s_fruit[g], pa, pb, c.radius)) mask |= 1ull << g;
        }
        if (!owner) continue;
        cta_sums_add(s_sum + 3u * f + 0u, delta.x);
        cta_sums_add(s_sum + 3u * f + 1u, delta.y);
        cta_sums_add(s_sum + 3u * f + 2u, delta.z);
        if (lam <= 0.0f) continue;
        rec.add(ctx, f, n, lam / c.dt, w0, w1);
    }
    if (owner) rec.finish(ctx);
    return changed;
}

// One yarn colour of the fruit/yarn sweep.  Fruits do not move during a
// sweep (their summed displacements are applied after it), so the first
// colour stages them in shared memory for all colours, the CTA's
// displacement sums accumulate over the sweep, and the last colour adds
// them to the global sums.
__device__ void yarn_contact_batch(Ctx& ctx, uint32_t slot, const Batch& bt, bool first, bool last) {
    const DeviceCloth& d = ctx.d;
    __shared__ float4 s_fruit[NC_MAX_FRUITS];   // xyz position, w radius
    __shared__ float s_fw[NC_MAX_FRUITS];
    __shared__ unsigned long long s_sum[3u * NC_MAX_FRUITS];
    if (first) {
        cta_sums_clear(s_sum, 3u * d.f_count);
        for (uint32_t f = threadIdx.x; f < d.f_count; f += blockDim.x) {
            const NumiClothFruit& fr = d.fruits[f];
            const float4 xw = __ldcg(reinterpret_cast<const float4*>(&fr.positionAndInverseMass));
            s_fruit[f] = make_float4(xw.x, xw.y, xw.z, __ldcg(&fr.previousAndRadius.w));
            s_fw[f] = xw.w;
        }
        __syncthreads();
    }
    unsigned long long* acc = reinterpret_cast<unsigned long long*>(d.fruit_partial);
    const uint32_t nf = d.f_count;
    const uint32_t lane = threadIdx.x & 31u;
    // the colour's items of this CTA (its yarn segments lead its list) or
    // the grid-stride range, a warp at a time
    const Range rg = colour_items(ctx, slot, bt.yarn);
    for (uint32_t base = rg.i - lane; base < rg.end; base += rg.stride) {
        const uint32_t pos = base + lane;
        const uint32_t k = pos < rg.end ? colour_item(ctx, pos) : bt.yarn;
        const bool valid = k < bt.yarn;
        if (!__any_sync(0xffffffffu, valid)) break;
        const uint32_t seg = bt.first + (valid ? k : 0u);
        uint2 ij = make_uint2(0u, 0u);
        float4 pa = make_float4(0, 0, 0, 0), pb = pa;
        if (valid) {
            ij = __ldg(d.d_ij + seg);
            pa = px(ctx, ij.x);
            pb = px(ctx, ij.y);
        }
        if (yarn_warp_contacts(ctx, valid, true, seg, pa, pb, s_fruit, s_fw, s_sum)) {
            px_set(ctx, ij.x, pa);
            px_set(ctx, ij.y, pb);
        }
    }
    if (last) cta_sums_flush(s_sum, acc, 3u * nf);
}

// One yarn colour of the swept fruit/yarn sweep (solveSweptBallYarn,
// tools/cloth_bag.cpp:3022-3109): conservative advancement of every fruit
// against every segment over the substep's motion, at most 80 steps, then
// the ground-aware correction of the approach left after the impact.  The
// batched order is the present sweep's: segments of a colour in parallel,
// fruits (positions and previous positions) frozen over the sweep, each
// segment visiting the fruits in ascending order, fruit displacements summed.
// A fruit whose swept box is farther than the contact distance from the
// segment's swept box cannot be found by the advancement and is skipped.
__device__ void swept_contact_batch(Ctx& ctx, const Batch& bt, bool first, bool last) {
    const DeviceCloth& d = ctx.d;
    const SubCfg& c = ctx.c;
    __shared__ float4 s_fx[NC_MAX_FRUITS];   // position xyz, radius
    __shared__ float4 s_fp[NC_MAX_FRUITS];   // previous position xyz, inverse mass
    __shared__ unsigned long long s_sum[3u * NC_MAX_FRUITS];
    const uint32_t nf = d.f_count;
    if (first) {
        cta_sums_clear(s_sum, 3u * nf);
        for (uint32_t f = threadIdx.x; f < nf; f += blockDim.x) {
            const NumiClothFruit& fr = d.fruits[f];
            const float4 xw = __ldcg(reinterpret_cast<const float4*>(&fr.positionAndInverseMass));
            const float4 pr = __ldcg(reinterpret_cast<const float4*>(&fr.previousAndRadius));
            s_fx[f] = make_float4(xw.x, xw.y, xw.z, pr.w);
            s_fp[f] = make_float4(pr.x, pr.y, pr.z, xw.w);
        }
        __syncthreads();
    }
    unsigned long long* acc = reinterpret_cast<unsigned long long*>(d.fruit_partial);
    for (Range rg = item_range(ctx, bt.yarn); rg.i < rg.end; rg.i += rg.stride) {
        const uint32_t seg = bt.first + rg.i;
        const uint2 ij = __ldg(d.d_ij + seg);
        float4 pa = px(ctx, ij.x), pb = px(ctx, ij.y);
        const V3 qa = xyz(ld(d.xp + ij.x)), qb = xyz(ld(d.xp + ij.y));
        bool changed = false;
        SegRecords rec(seg);
        for (uint32_t f = 0; f < nf; ++f) {
            const float4 fx = s_fx[f], fp = s_fp[f];
            const float target = fx.w + c.radius;
            // swept boxes
            const float slack = target + 1.0e-6f;
            const V3 slo{fminf(fminf(pa.x, pb.x), fminf(qa.x, qb.x)), fminf(fminf(pa.y, pb.y), fminf(qa.y, qb.y)),
                         fminf(fminf(pa.z, pb.z), fminf(qa.z, qb.z))};
            const V3 shi{fmaxf(fmaxf(pa.x, pb.x), fmaxf(qa.x, qb.x)), fmaxf(fmaxf(pa.y, pb.y), fmaxf(qa.y, qb.y)),
                         fmaxf(fmaxf(pa.z, pb.z), fmaxf(qa.z, qb.z))};
            if (fmaxf(fx.x, fp.x) < slo.x - slack || fminf(fx.x, fp.x) > shi.x + slack ||
                fmaxf(fx.y, fp.y) < slo.y - slack || fminf(fx.y, fp.y) > shi.y + slack ||
                fmaxf(fx.z, fp.z) < slo.z - slack || fminf(fx.z, fp.z) > shi.z + slack)
                continue;
            const V3 X = xyz(fx), P = xyz(fp);
            float bound = len3(X - P) + len3(xyz(pa) - qa);
            bound = bound + len3(xyz(pb) - qb);
            if (bound < 1.0e-14f) continue;
            V3 bp, sa, sb, closest;
            float weight, dist;
            auto sample = [&](float time) {
                bp = P + (X - P) * time;
                sa = qa + (xyz(pa) - qa) * time;
                sb = qb + (xyz(pb) - qb) * time;
                point_segment(bp, sa, sb, closest, weight);
                dist = len3(closest - bp);
            };
            float time = 0.0f;
            sample(0.0f);
            bool found = dist <= target + 1.0e-9f;
            if (!found) {
                for (int it = 0; it < 80; ++it) {
                    sample(time);
                    const float gap = dist - target;
                    if (gap <= 1.0e-9f) {
                        found = true;
                        break;
                    }
                    const float advance = 0.9f * gap / bound;
                    if (!isfinite(advance) || advance <= 0.0f || time + advance >= 1.0f) break;
                    time = time + fmaxf(advance, 1.0e-10f);
                }
            }
            if (!found || dist < 1.0e-12f) continue;
            const V3 n = vdiv(closest - bp, dist);
            const float w0 = 1.0f - weight, w1 = weight;
            const V3 seg_rem = (xyz(pa) - sa) * w0 + (xyz(pb) - sb) * w1;
            const V3 ball_rem = X - bp;
            const float removed = dot3(ball_rem - seg_rem, n);
            if (removed <= 0.0f) continue;
            V3 delta{0.0f, 0.0f, 0.0f};
            const float lam = yarn_correction(pa, pb, w0, w1, fp.w, n, removed, c.ground, c.radius, delta);
            changed = true;
            cta_sums_add(s_sum + 3u * f + 0u, delta.x);
            cta_sums_add(s_sum + 3u * f + 1u, delta.y);
            cta_sums_add(s_sum + 3u * f + 2u, delta.z);
            if (lam <= 0.0f) continue;
            rec.add(ctx, f, n, lam / c.dt, w0, w1);
        }
        if (changed) {
            px_set(ctx, ij.x, pa);
            px_set(ctx, ij.y, pb);
        }
        rec.finish(ctx);
    }
    if (last) cta_sums_flush(s_sum, acc, 3u * nf);
}

__device__ bool yarn_sweep(Ctx& ctx) {
    if (ctx.d.f_count == 0u) return true;
    fruit_flush(ctx);
    uint32_t first = NC_MAX_BATCHES, last = 0;
    for (uint32_t b = 0; b < ctx.d.n_dist_batches; ++b)
        if (ctx.d.dist_batches[b].yarn != 0u) {
            first = min(first, b);
            last = b;
        }
    for (uint32_t b = first; b <= last && b < ctx.d.n_dist_batches; ++b) {
        const Batch bt = ctx.d.dist_batches[b];
        if (bt.yarn == 0u) continue;
        yarn_contact_batch(ctx, b, bt, b == first, b == last);
        NC_CSYNC(ctx, b != last);   // colour to colour: neighbour sync
    }
    ctx.fruit_pending = true;
    return true;
}

// ------------------------------------------------------- self contact ---
// Point/point self contact (tools/cloth_bag.cpp:4249-4315), batched: every
// particle resolves all its pairs closer than 2r against the positions at
// the start of the pass and applies the sum of its corrections once.  The
// reference pushes each pair apart in particle order (Gauss-Seidel); here
// the pair set and the per-pair correction are the reference's, the sums
// are 2^-40 fixed point so their order does not matter, and the two sides
// of a pair compute exactly opposite corrections.

// Not-a-neighbour test of the reference's localTopologyPair
// (tools/cloth_bag.cpp:2723-2730): the 2-hop topology list, or for a
// row-major grid cloth the 5 x 5 block around the particle.
__device__ __forceinline__ bool local_pair(const DeviceCloth& d, uint32_t a, uint32_t b) {
    if (d.local_off != nullptr) {
        uint32_t lo = __ldg(d.local_off + a), hi = __ldg(d.local_off + a + 1u);
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            const uint32_t v = __ldg(d.local_idx + mid);
            if (v == b) return true;
            if (v < b) lo = mid + 1u;
            else hi = mid;
        }
        return false;
    }
    if (d.grid_width == 0u) return a == b;
    const int ra = static_cast<int>(a / d.grid_width), ca = static_cast<int>(a % d.grid_width);
    const int rb = static_cast<int>(b / d.grid_width), cb = static_cast<int>(b % d.grid_width);
    return abs(ra - rb) <= 2 && abs(ca - cb) <= 2;
}

// Bucket of a hash cell: the cell key with 21 biased bits per axis (as the
// reference's spatialKey, tools/cloth_bag.cpp:2732-2738) through the
// SplitMix64 finalizer (Steele, Lea and Flood 2014), so that neighbouring
// cells of a flat cloth spread over the buckets.
__device__ __forceinline__ uint32_t cell_bucket(int x, int y, int z, uint32_t mask) {
    unsigned long long k = (static_cast<unsigned long long>(x + (1 << 20)) & 0x1fffffull) |
                           ((static_cast<unsigned long long>(y + (1 << 20)) & 0x1fffffull) << 21) |
                           ((static_cast<unsigned long long>(z + (1 << 20)) & 0x1fffffull) << 42);
    k = (k ^ (k >> 30)) * 0xbf58476d1ce4e5b9ull;
    k = (k ^ (k >> 27)) * 0x94d049bb133111ebull;
    return static_cast<uint32_t>(k ^ (k >> 31)) & mask;
}

__device__ __forceinline__ uint32_t self_pass_tag(const Ctx& ctx, uint32_t it) { return (ctx.epoch << 6) | (it & 63u); }

// Insert every particle at its start-of-pass position.  Tags only grow (the
// host clears the heads when the substep counter wraps), so a max with
// (tag, 0) resets a bucket of an older pass and leaves a current one alone;
// the add after it, in the same thread's order on the same address, takes
// the next slots.  The slots are claimed warp by warp: the lanes that hash
// to one bucket (neighbouring particles mostly share cells) form a group
// (match), its first lane claims as many slots as the group has lanes with
// one atomic, and each lane takes the claimed base plus its rank in the
// group (a segmented prefix count over the warp); lanes whose slots fall
// past the bucket's capacity claim overflow entries the same way (ballot
// and prefix count).  The slot order does not change any result: a query
// sums its corrections in fixed point.
__device__ __forceinline__ void self_insert_one(const Ctx& ctx, unsigned long long tag, uint32_t i, const float4& p) {
    const DeviceCloth& d = ctx.d;
    const float inv_cell = 1.0f / (4.0f * ctx.c.radius);
    const uint32_t bucket = cell_bucket(static_cast<int>(floorf(p.x * inv_cell)),
                                        static_cast<int>(floorf(p.y * inv_cell)),
                                        static_cast<int>(floorf(p.z * inv_cell)), d.hash_mask);
    const unsigned active = __activemask();
    const uint32_t lane = threadIdx.x & 31u;
    const unsigned below = (1u << lane) - 1u;
    const unsigned peers = __match_any_sync(active, bucket);
    const int leader = __ffs(static_cast<int>(peers)) - 1;
    unsigned long long base = 0ull;
    if (static_cast<int>(lane) == leader) {
        unsigned long long* head = d.hash_head + bucket;
        atomicMax(head, tag << 32);
        base = atomicAdd(head, static_cast<unsigned long long>(__popc(peers)));
    }
    base = __shfl_sync(peers, base, leader);
    const uint32_t slot = static_cast<uint32_t>(base) + static_cast<uint32_t>(__popc(peers & below));
    const bool over = slot >= NC_HASH_CAP;
    const unsigned overs = __ballot_sync(active, over);
    HashSlot* e;
    if (!over) {
        e = d.hash + bucket * NC_HASH_CAP + slot;
    } else {
        // a full bucket (a crumpled cloth packs many particles into a
        // cell): the particle goes to the overflow list every query scans
        const int first = __ffs(static_cast<int>(overs)) - 1;
        unsigned long long obase = 0ull;
        if (static_cast<int>(lane) == first) {
            atomicMax(d.hash_over_head, tag << 32);
            obase = atomicAdd(d.hash_over_head, static_cast<unsigned long long>(__popc(overs)));
        }
        obase = __shfl_sync(overs, obase, first);
        const uint32_t o = static_cast<uint32_t>(obase) + static_cast<uint32_t>(__popc(overs & below));
        if (o >= d.n) {
            fail(d, NUMI_CLOTH_FAILURE_RANGE);
            return;
        }
        e = d.hash_over + o;
    }
    e->pos = make_float4(p.x, p.y, p.z, __uint_as_float(i));
}

__device__ void self_insert(Ctx& ctx, uint32_t it) {
    const unsigned long long tag = self_pass_tag(ctx, it);
    for (Range r = particle_range(ctx); r.i < r.end; r.i += r.stride) self_insert_one(ctx, tag, r.i, px(ctx, r.i));
}

// Resolve every particle's pairs.  A cell is twice the contact distance,
// so the 2 x 2 x 2 cells on the particle's side of its own cell's centre
// hold every particle closer than the contact distance.  The eight bucket
// heads are read together, then the candidates in batches of eight, every
// load of a batch issued before any is used.  The grid is read-only in this
// phase and the grid barrier before it is a gpu-scope acquire, so the reads
// may go through L1, where neighbouring particles of a CTA share cells;
// under the cluster barrier (cluster-scope acquire) they stay L2 reads.
#define NC_SELF_BATCH 8u
// A particle's query: its buckets, the candidates each holds (prefix
// counts, a bucket met twice counts once) and their total.
struct SelfQuery {
    uint32_t bk[8];
    uint32_t pre[9];
};

// Buckets of the 2 x 2 x 2 cells on the particle's side of its cell centre
// and the heads of those within reach, loaded together.
__device__ __forceinline__ void self_heads(const Ctx& ctx, const float4& p, SelfQuery& q, unsigned long long hd[8],
                                           bool near[8]) {
    const DeviceCloth& d = ctx.d;
    const float inv_cell = 1.0f / (4.0f * ctx.c.radius);
    const bool l1 = d.cluster_barrier == 0u;
    int base[3], step[3];
    float gap2[3];   // squared distance to the probed neighbour cell, in cell units
    const float coord[3] = {p.x * inv_cell, p.y * inv_cell, p.z * inv_cell};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float c0 = floorf(coord[k]);
        const float frac = coord[k] - c0;
        base[k] = static_cast<int>(c0);
        step[k] = frac < 0.5f ? -1 : 1;
        const float gap = frac < 0.5f ? frac : 1.0f - frac;
        gap2[k] = gap * gap;
    }
#pragma unroll
    for (uint32_t c = 0; c < 8u; ++c)
        q.bk[c] = cell_bucket(base[0] + ((c & 1u) ? step[0] : 0), base[1] + ((c & 2u) ? step[1] : 0),
                              base[2] + ((c & 4u) ? step[2] : 0), d.hash_mask);
    // A neighbour cell farther than the contact distance (half a cell)
    // cannot hold a contact.  The margin covers the rounding of the cell
    // coordinates: 1e-3 cells plus a few ulps of the largest coordinate.
    // Only the heads of near cells are read.
    const float slack = 0.5f + 1.0e-3f + 2.4e-7f * fmaxf(fabsf(coord[0]), fmaxf(fabsf(coord[1]), fabsf(coord[2])));
    const float reach2 = slack * slack;
#pragma unroll
    for (uint32_t c = 0; c < 8u; ++c) {
        const float g2 = ((c & 1u) ? gap2[0] : 0.0f) + ((c & 2u) ? gap2[1] : 0.0f) + ((c & 4u) ? gap2[2] : 0.0f);
        near[c] = c == 0u || g2 < reach2;
        hd[c] = !near[c] ? 0ull : l1 ? __ldca(d.hash_head + q.bk[c]) : __ldcg(d.hash_head + q.bk[c]);
    }
}

// Candidates per bucket of this pass (a bucket met twice counts once).
__device__ __forceinline__ uint32_t self_counts(uint32_t tag, SelfQuery& q, const unsigned long long hd[8],
                                                const bool near[8]) {
    q.pre[0] = 0u;
#pragma unroll
    for (uint32_t c = 0; c < 8u; ++c) {
        bool repeat = false;
#pragma unroll
        for (uint32_t e = 0; e < c; ++e) repeat = repeat || (near[e] && q.bk[e] == q.bk[c]);
        const uint32_t cnt = (near[c] && !repeat && static_cast<uint32_t>(hd[c] >> 32) == tag)
                                 ? min(static_cast<uint32_t>(hd[c]), NC_HASH_CAP)
                                 : 0u;
        q.pre[c + 1u] = q.pre[c] + cnt;
    }
    return q.pre[8];
}

// Slot of candidate t (past the end: the last one again).
__device__ __forceinline__ uint32_t self_slot(const SelfQuery& q, uint32_t t, uint32_t total) {
    t = min(t, total - 1u);
    uint32_t bq = q.bk[0], pq = 0u;
#pragma unroll
    for (uint32_t k = 1; k < 8u; ++k)
        if (t >= q.pre[k]) {
            bq = q.bk[k];
            pq = q.pre[k];
        }
    return bq * NC_HASH_CAP + (t - pq);
}

// ---------------------------------------------------------------------------
// ---------------------------------------------------------------------------
// Point self contact in the batched order (the default): every non-local
// pair closer than 2r at the start of the pass, each particle's
// corrections from all its pairs summed in fixed point and applied once.
// Where every particle has at most one partner this makes the reference's
// moves (tools/cloth_bag.cpp:4249-4315); the reference-order form below
// keeps its Gauss-Seidel order everywhere.
// ---------------------------------------------------------------------------
// One candidate entry e of particle a at its start-of-pass position p: the
// reference pair correction (a's half), summed in fixed point.
__device__ __forceinline__ void self_pair(const Ctx& ctx, uint32_t a, const float4& p, const float4& e,
                                          long long sum[3], bool& touched, unsigned long long& contacts,
                                          float& max_pen) {
    const DeviceCloth& d = ctx.d;
    const float target = 2.0f * ctx.c.radius;
    const uint32_t b = __float_as_uint(e.w);
    if (b == a) return;
    const V3 diff = xyz(e) - xyz(p);
    const float L = len3(diff);
    if (L >= target || L < 1.0e-12f) return;
    // the partner's inverse mass (fixed; the corrections of this pass
    // rewrite only positions)
    const float den = p.w + px(ctx, b).w;
    if (den <= 0.0f) return;
    if (local_pair(d, a, b)) return;
    const V3 corr = diff * ((target - L) / (L * den));
    sum[0] += to_fixed(-(corr.x * p.w));
    sum[1] += to_fixed(-(corr.y * p.w));
    sum[2] += to_fixed(-(corr.z * p.w));
    touched = true;
    if (a < b) {
        ++contacts;
        max_pen = fmaxf(max_pen, target - L);
    }
}

// The overflow list (particles of full buckets), then the moved position.
__device__ __forceinline__ bool self_finish(const Ctx& ctx, uint32_t tag, uint32_t a, const float4& p,
                                            long long sum[3], bool touched, float4& moved,
                                            unsigned long long& contacts, float& max_pen) {
    const DeviceCloth& d = ctx.d;
    const bool l1 = d.cluster_barrier == 0u;
    const unsigned long long oh = l1 ? __ldca(d.hash_over_head) : __ldcg(d.hash_over_head);
    const uint32_t over = static_cast<uint32_t>(oh >> 32) == tag ? min(static_cast<uint32_t>(oh), d.n) : 0u;
    for (uint32_t o = 0; o < over; ++o) self_pair(ctx, a, p, __ldcg(&d.hash_over[o].pos), sum, touched, contacts, max_pen);
    if (touched) {
        const float dx = from_fixed(static_cast<unsigned long long>(sum[0]));
        const float dy = from_fixed(static_cast<unsigned long long>(sum[1]));
        const float dz = from_fixed(static_cast<unsigned long long>(sum[2]));
        moved = make_float4(p.x + dx, p.y + dy, p.z + dz, p.w);
    }
    return touched;
}

// Resolve every particle's pairs.  A cell is twice the contact distance,
// so the 2 x 2 x 2 cells on the particle's side of its own cell's centre
// hold every particle closer than the contact distance.  The eight bucket
// heads are read together, then the candidates in batches of eight, every
// load of a batch issued before any is used.  The grid is read-only in this
// phase and the grid barrier before it is a gpu-scope acquire, so the reads
// may go through L1, where neighbouring particles of a CTA share cells;
// under the cluster barrier (cluster-scope acquire) they stay L2 reads.
// The pass of particle a at its start-of-pass position p: true when a pair
// moved it, with the moved position in `moved`; counts the pairs a < b and the
// deepest penetration.
__device__ __forceinline__ bool self_solve_one(const Ctx& ctx, uint32_t tag, uint32_t a, const float4& p,
                                               float4& moved, unsigned long long& contacts, float& max_pen) {
    const DeviceCloth& d = ctx.d;
    const bool l1 = d.cluster_barrier == 0u;
    SelfQuery q;
    unsigned long long hd[8];
    bool near[8];
    self_heads(ctx, p, q, hd, near);
    const uint32_t total = self_counts(tag, q, hd, near);
    long long sum[3] = {0, 0, 0};
    bool touched = false;
    for (uint32_t t0 = 0; t0 < total; t0 += NC_SELF_BATCH) {
        float4 e[NC_SELF_BATCH];
#pragma unroll
        for (uint32_t j = 0; j < NC_SELF_BATCH; ++j) {
            const uint32_t slot = self_slot(q, t0 + j, total);
            e[j] = l1 ? __ldca(&d.hash[slot].pos) : __ldcg(&d.hash[slot].pos);
        }
#pragma unroll
        for (uint32_t j = 0; j < NC_SELF_BATCH; ++j)
            if (t0 + j < total) self_pair(ctx, a, p, e[j], sum, touched, contacts, max_pen);
    }
    return self_finish(ctx, tag, a, p, sum, touched, moved, contacts, max_pen);
}

// The self-contact statistics of a CTA's particles: one atomic pair per
// warp (an integer sum and the maximum of non-negative floats as integers:
// the order does not matter).
__device__ __forceinline__ void self_stats_flush(const DeviceCloth& d, unsigned long long contacts, float max_pen) {
    unsigned pen_bits = __float_as_uint(max_pen);
    for (int o = 16; o > 0; o >>= 1) {
        contacts += __shfl_xor_sync(0xffffffffu, contacts, o);
        pen_bits = max(pen_bits, __shfl_xor_sync(0xffffffffu, pen_bits, o));
    }
    if ((threadIdx.x & 31u) == 0u && contacts != 0ull) {
        atomicAdd(d.self_stats, contacts);
        atomicMax(d.self_stats + 1, static_cast<unsigned long long>(pen_bits));
    }
}

__device__ void self_solve(Ctx& ctx, uint32_t it) {
    const uint32_t tag = self_pass_tag(ctx, it);
    unsigned long long contacts = 0ull;
    float max_pen = 0.0f;
    for (Range r = particle_range(ctx); r.i < r.end; r.i += r.stride) {
        const uint32_t a = r.i;
        const float4 p = px(ctx, a);
        float4 q;
        if (self_solve_one(ctx, tag, a, p, q, contacts, max_pen)) px_set(ctx, a, q);
    }
    self_stats_flush(ctx.d, contacts, max_pen);
}

// Point self contact in the reference's Gauss-Seidel order
// (solveSelfCollision, tools/cloth_bag.cpp:4249-4315).
//
// The reference visits the particles in index order.  Particle a, from its
// position at its turn, resolves every non-local b > a whose start-of-pass
// cell (edge = the contact distance 2r) is one of the 27 around a's cell,
// cell by cell (z, then y, then x, each from -1) and by index within a
// cell, each pair on the current positions.  The kernel makes the same
// moves in parallel:
//  * phase A, every particle at its start-of-pass position: a particle that
//    touches nobody (no non-local particle closer than 2r) is no mover.  A
//    mover whose only particle within 4r is its one contact partner, and
//    whose partner's only particle within 4r is the mover itself, is one
//    side of an isolated pair: each side computes the reference correction
//    from the two start positions and applies its own half.  Every other
//    mover lists its pairs with all particles within 4r (it is coupled).
//  * the ordered pass, on one CTA and only where something was listed:
//    the listed particles go back to their start positions and the listed
//    pairs run serially in the reference's order.
// Why that is the reference's result: a pair nobody listed either starts
// 4r or more apart, or joins two particles that touch nobody.  The first
// kind can act only if its particles move by 2r together, the second only
// if one of them moves at all.  An isolated pair moves each of its
// particles by at most r (a deeper pair is listed instead); the ordered
// pass checks every listed particle's largest displacement against r and,
// for a listed particle that touched nobody at the start but moved, lists
// its own 4r neighbourhood and starts over.  Where a listed particle moves
// farther, the list overflows or a particle has too many listed partners,
// the ordered pass runs the reference loop itself on one thread over the
// whole cloth (exact, slow, and met only where layers interpenetrate by
// more than half the contact distance).
// ---------------------------------------------------------------------------
#define NC_SELF_LISTED 1ull
#define NC_SELF_KNOWN 2ull     // the particle's whole 4r neighbourhood is listed
#define NC_SELF_SIMPLE 4ull    // one side of an isolated pair (phase A)
#define NC_SELF_ROUNDS 8u      // ordered-pass rounds before the fallback
#define NC_SELF_GROUP 512u     // listed partners of one particle in one turn
#define NC_SELF_KNOWN_BIT 0x80000000u
#define NC_SELF_WAVE_MAX 8192u   // pairs in contact the wavefront form orders
#define NC_SELF_BAND 0.01f       // listed pairs within this fraction of the contact distance join the wavefronts

// Reference cell of a position (edge = the contact distance; the
// reference's floor(position * inverseCell)).
__device__ __forceinline__ int3 self_ref_cell(V3 p, float inv) {
    return make_int3(static_cast<int>(floorf(p.x * inv)), static_cast<int>(floorf(p.y * inv)),
                     static_cast<int>(floorf(p.z * inv)));
}
// Rank of cell b among the 27 around cell a in the reference's visit order
// (dz, then dy, then dx, each from -1), or -1 outside them.
__device__ __forceinline__ int self_visit_rank(int3 a, int3 b) {
    const int dx = b.x - a.x, dy = b.y - a.y, dz = b.z - a.z;
    if (dx < -1 || dx > 1 || dy < -1 || dy > 1 || dz < -1 || dz > 1) return -1;
    return (dz + 1) * 9 + (dy + 1) * 3 + (dx + 1);
}

// Every grid entry of this pass within one grid cell (4r) of p: the buckets
// of the 27 cells around p's cell that reach within a cell of p, then the
// overflow list.  Two cells that share a bucket repeat its entries; callers
// either tolerate repeats (a repeat only makes a particle look coupled) or
// remove them.
template <class F>
__device__ __forceinline__ void self_scan_cell(const Ctx& ctx, uint32_t tag, const float4& p, F&& visit) {
    const DeviceCloth& d = ctx.d;
    const float inv_cell = 1.0f / (4.0f * ctx.c.radius);
    const float coord[3] = {p.x * inv_cell, p.y * inv_cell, p.z * inv_cell};
    int base[3];
    float lo2[3], hi2[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float c0 = floorf(coord[k]);
        base[k] = static_cast<int>(c0);
        const float f = coord[k] - c0;
        lo2[k] = f * f;
        hi2[k] = (1.0f - f) * (1.0f - f);
    }
    const float slack = 1.0f + 1.0e-3f + 2.4e-7f * fmaxf(fabsf(coord[0]), fmaxf(fabsf(coord[1]), fabsf(coord[2])));
    const float reach2 = slack * slack;
    for (int dz = -1; dz <= 1; ++dz)
        for (int dy = -1; dy <= 1; ++dy)
            for (int dx = -1; dx <= 1; ++dx) {
                const float g2 = (dx < 0 ? lo2[0] : dx > 0 ? hi2[0] : 0.0f) +
                                 (dy < 0 ? lo2[1] : dy > 0 ? hi2[1] : 0.0f) +
                                 (dz < 0 ? lo2[2] : dz > 0 ? hi2[2] : 0.0f);
                if (g2 >= reach2) continue;
                const uint32_t bk = cell_bucket(base[0] + dx, base[1] + dy, base[2] + dz, d.hash_mask);
                const unsigned long long hd = __ldcg(d.hash_head + bk);
                if (static_cast<uint32_t>(hd >> 32) != tag) continue;
                const uint32_t cnt = min(static_cast<uint32_t>(hd), NC_HASH_CAP);
                for (uint32_t s = 0; s < cnt; ++s) visit(__ldcg(&d.hash[bk * NC_HASH_CAP + s].pos));
            }
    const unsigned long long oh = __ldcg(d.hash_over_head);
    const uint32_t over = static_cast<uint32_t>(oh >> 32) == tag ? min(static_cast<uint32_t>(oh), d.n) : 0u;
    for (uint32_t o = 0; o < over; ++o) visit(__ldcg(&d.hash_over[o].pos));
}

// A pair the pass can resolve: another particle, not local, not both
// fixed (w: the inverse masses).
__device__ __forceinline__ bool self_partner(const DeviceCloth& d, uint32_t a, uint32_t b, float wa, float wb) {
    return b != a && wa + wb > 0.0f && !local_pair(d, min(a, b), max(a, b));
}

// Entries within 4r of particle a (start position p, w = its inverse mass)
// that it may pair with, counted up to two.
__device__ __noinline__ uint32_t self_count_near(const Ctx& ctx, uint32_t tag, uint32_t a, const float4& p) {
    const float reach = 4.0f * ctx.c.radius;
    uint32_t n = 0u;
    self_scan_cell(ctx, tag, p, [&](const float4& e) {
        const uint32_t b = __float_as_uint(e.w);
        if (n >= 2u || b == a || len3(xyz(e) - xyz(p)) >= reach) return;
        if (self_partner(ctx.d, a, b, p.w, px(ctx, b).w)) ++n;
    });
    return n;
}

// List particle a's pairs with every particle within 4r (a's start position
// p; a's entry carries the known bit).  False where the list is full.
__device__ __noinline__ bool self_list_near(const Ctx& ctx, uint32_t tag, uint32_t a, const float4& p) {
    const DeviceCloth& d = ctx.d;
    const float reach = 4.0f * ctx.c.radius;
    bool room = true;
    self_scan_cell(ctx, tag, p, [&](const float4& e) {
        const uint32_t b = __float_as_uint(e.w);
        if (b == a || len3(xyz(e) - xyz(p)) >= reach || !self_partner(d, a, b, p.w, px(ctx, b).w)) return;
        atomicMax(d.self_list_head, static_cast<unsigned long long>(tag) << 32);
        const uint32_t k = static_cast<uint32_t>(atomicAdd(d.self_list_head, 1ull));
        if (k >= d.self_list_cap) {
            room = false;
            return;
        }
        const float4 ea = make_float4(p.x, p.y, p.z, __uint_as_float(a | NC_SELF_KNOWN_BIT));
        const float4 eb = make_float4(e.x, e.y, e.z, __uint_as_float(b));
        d.self_list[2u * k] = a < b ? ea : eb;
        d.self_list[2u * k + 1u] = a < b ? eb : ea;
    });
    return room;
}

// Phase A of a mover a (start position p) with `touches` contact partners,
// the last one `partner` (start position and inverse mass pe): the isolated
// pair's move, or the coupled particle's listing.  Out of line: only movers
// run it.
__device__ __noinline__ bool self_mover(const Ctx& ctx, uint32_t tag, uint32_t a, const float4& p, uint32_t touches,
                                        uint32_t partner, const float4& pe, float4& moved,
                                        unsigned long long& contacts, float& max_pen) {
    const DeviceCloth& d = ctx.d;
    const float target = 2.0f * ctx.c.radius;
    if (touches == 1u && self_count_near(ctx, tag, a, p) == 1u && self_count_near(ctx, tag, partner, pe) == 1u) {
        // isolated pair: the reference's correction with f < s
        const bool first = a < partner;
        const float4 xf = first ? p : pe, xs = first ? pe : p;
        const float inv_ref = 1.0f / target;
        const bool visited = self_visit_rank(self_ref_cell(xyz(xf), inv_ref), self_ref_cell(xyz(xs), inv_ref)) >= 0;
        const V3 diff = xyz(xs) - xyz(xf);
        const float L = len3(diff);
        if (!visited || L < 1.0e-12f) {
            d.self_mark[a] = (static_cast<unsigned long long>(tag) << 32) | NC_SELF_SIMPLE;
            return false;   // a pair the reference skips, and nothing else moves either side
        }
        const float den = xf.w + xs.w;
        const V3 corr = diff * ((target - L) / (L * den));
        const V3 cf = corr * xf.w, cs = corr * xs.w;
        const float lim = 0.5f * target * (1.0f - 1.0e-4f);
        if (len3(cf) <= lim && len3(cs) <= lim) {
            d.self_mark[a] = (static_cast<unsigned long long>(tag) << 32) | NC_SELF_SIMPLE;
            moved = with_xyz(p, first ? xyz(p) - cf : xyz(p) + cs);
            if (first) {
                ++contacts;
                max_pen = fmaxf(max_pen, target - L);
            }
            return true;
        }
    }
    (void)self_list_near(ctx, tag, a, p);   // a full list sends the ordered pass to the fallback
    return false;
}


// Phase A of particle a at its start-of-pass position p: true when its
// isolated pair moved it, with the moved position in `moved`; counts that
// pair (on its first particle) and its penetration.  A coupled particle is
// listed and left where it is.
__device__ __forceinline__ bool self_exact_one(const Ctx& ctx, uint32_t tag, uint32_t a, const float4& p,
                                               float4& moved, unsigned long long& contacts, float& max_pen) {
    const DeviceCloth& d = ctx.d;
    const bool l1 = d.cluster_barrier == 0u;
    const float target = 2.0f * ctx.c.radius;
    SelfQuery q;
    unsigned long long hd[8];
    bool near[8];
    self_heads(ctx, p, q, hd, near);
    const uint32_t total = self_counts(tag, q, hd, near);
    uint32_t touches = 0u, partner = 0u;
    float4 pe = p;
    auto touch = [&](const float4& e) {
        const uint32_t b = __float_as_uint(e.w);
        if (b == a || len3(xyz(e) - xyz(p)) >= target) return;
        const float wb = px(ctx, b).w;
        if (!self_partner(d, a, b, p.w, wb)) return;
        ++touches;
        partner = b;
        pe = make_float4(e.x, e.y, e.z, wb);
    };
    for (uint32_t t0 = 0; t0 < total; t0 += NC_SELF_BATCH) {
        float4 e[NC_SELF_BATCH];
#pragma unroll
        for (uint32_t j = 0; j < NC_SELF_BATCH; ++j) {
            const uint32_t slot = self_slot(q, t0 + j, total);
            e[j] = l1 ? __ldca(&d.hash[slot].pos) : __ldcg(&d.hash[slot].pos);
        }
#pragma unroll
        for (uint32_t j = 0; j < NC_SELF_BATCH; ++j)
            if (t0 + j < total) touch(e[j]);
    }
    {
        const unsigned long long oh = l1 ? __ldca(d.hash_over_head) : __ldcg(d.hash_over_head);
        const uint32_t over = static_cast<uint32_t>(oh >> 32) == tag ? min(static_cast<uint32_t>(oh), d.n) : 0u;
        for (uint32_t o = 0; o < over; ++o) touch(__ldcg(&d.hash_over[o].pos));
    }
    if (touches == 0u) return false;
    return self_mover(ctx, tag, a, p, touches, partner, pe, moved, contacts, max_pen);
}

// This pass's contact statistics of phase A: one atomic pair per warp (an
// integer sum and the maximum of non-negative floats as integers).
__device__ __forceinline__ void self_pass_flush(const DeviceCloth& d, unsigned long long contacts, float max_pen) {
    unsigned pen_bits = __float_as_uint(max_pen);
    for (int o = 16; o > 0; o >>= 1) {
        contacts += __shfl_xor_sync(0xffffffffu, contacts, o);
        pen_bits = max(pen_bits, __shfl_xor_sync(0xffffffffu, pen_bits, o));
    }
    if ((threadIdx.x & 31u) == 0u && contacts != 0ull) {
        atomicAdd(d.self_pass_stats, contacts);
        atomicMax(d.self_pass_stats + 1, static_cast<unsigned long long>(pen_bits));
    }
}

__device__ void self_solve_exact(Ctx& ctx, uint32_t it) {
    const uint32_t tag = self_pass_tag(ctx, it);
    unsigned long long contacts = 0ull;
    float max_pen = 0.0f;
    for (Range r = particle_range(ctx); r.i < r.end; r.i += r.stride) {
        const uint32_t a = r.i;
        const float4 p = px(ctx, a);
        float4 q;
        if (self_exact_one(ctx, tag, a, p, q, contacts, max_pen)) px_set(ctx, a, q);
    }
    self_pass_flush(ctx.d, contacts, max_pen);
}

// The pass's statistics into the cloth's (one thread, after the pass).
__device__ __forceinline__ void self_fold(const DeviceCloth& d) {
    const unsigned long long c = __ldcg(d.self_pass_stats);
    const unsigned long long pen = __ldcg(d.self_pass_stats + 1);
    if (c != 0ull) {
        d.self_stats[0] += c;
        d.self_stats[1] = max(d.self_stats[1], pen);
    }
    d.self_pass_stats[0] = 0ull;
    d.self_pass_stats[1] = 0ull;
}

// The reference pair body (first f < second s) on the current positions;
// with `x0` set, also the largest displacement of each side from its start
// position.  True where it acted, with its penetration.
__device__ __forceinline__ bool self_gs_pair(const Ctx& ctx, uint32_t f, uint32_t s, float target, bool track,
                                             float& pen) {
    const DeviceCloth& d = ctx.d;
    const float4 xf = px(ctx, f), xs = px(ctx, s);
    const V3 diff = xyz(xs) - xyz(xf);
    const float L = len3(diff);
    if (L >= target || L < 1.0e-12f) return false;
    const float den = xf.w + xs.w;
    if (den <= 0.0f) return false;
    const V3 corr = diff * ((target - L) / (L * den));
    const V3 nf = xyz(xf) - corr * xf.w, ns = xyz(xs) + corr * xs.w;
    px_set(ctx, f, with_xyz(xf, nf));
    px_set(ctx, s, with_xyz(xs, ns));
    if (track) {
        d.self_disp[f] = fmaxf(d.self_disp[f], len3(nf - xyz(d.self_x0[f])));
        d.self_disp[s] = fmaxf(d.self_disp[s], len3(ns - xyz(d.self_x0[s])));
    }
    pen = target - L;
    return true;
}

// Sort n keys (a power of two) ascending, the calling CTA together.
__device__ void self_bitonic(unsigned long long* keys, uint32_t n) {
    for (uint32_t size = 2u; size <= n; size <<= 1)
        for (uint32_t stride = size >> 1; stride > 0u; stride >>= 1) {
            for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
                const uint32_t j = i ^ stride;
                if (j <= i) continue;
                const unsigned long long ki = keys[i], kj = keys[j];
                const bool up = (i & size) == 0u;
                if ((ki > kj) == up) {
                    keys[i] = kj;
                    keys[j] = ki;
                }
            }
            __syncthreads();
        }
}

// Insertion sort of a short run of keys (one thread).
__device__ __forceinline__ void self_sort_run(unsigned long long* k, uint32_t n) {
    for (uint32_t i = 1; i < n; ++i) {
        const unsigned long long v = k[i];
        uint32_t j = i;
        while (j > 0u && k[j - 1u] > v) {
            k[j] = k[j - 1u];
            --j;
        }
        k[j] = v;
    }
}

// The reference loop itself, one thread, every particle from its
// start-of-pass position (its grid entry): the exact fallback.  False where
// a particle has more than NC_SELF_GROUP candidates in its 27 cells.
__device__ __noinline__ bool self_serial_all(const Ctx& ctx, uint32_t tag, unsigned long long& contacts, float& max_pen) {
    const DeviceCloth& d = ctx.d;
    const float target = 2.0f * ctx.c.radius;
    const float inv_ref = 1.0f / target;
    unsigned long long* run = d.self_keys + 3u * d.self_key_cap;
    const unsigned long long oh = __ldcg(d.hash_over_head);
    const uint32_t over = static_cast<uint32_t>(oh >> 32) == tag ? min(static_cast<uint32_t>(oh), d.n) : 0u;
    auto floor_half = [](int v) { return v >= 0 ? v / 2 : -((1 - v) / 2); };
    for (uint32_t a = 0; a < d.n; ++a) {
        const int3 tc = self_ref_cell(xyz(px(ctx, a)), inv_ref);
        uint32_t n = 0u;
        bool room = true;
        auto take = [&](const float4& e) {
            const uint32_t b = __float_as_uint(e.w);
            if (b <= a || local_pair(d, a, b)) return;
            const int rank = self_visit_rank(tc, self_ref_cell(xyz(e), inv_ref));
            if (rank < 0) return;
            if (n >= NC_SELF_GROUP) {
                room = false;
                return;
            }
            run[n++] = (static_cast<unsigned long long>(rank) << 32) | b;
        };
        // grid cells (edge 4r) that hold the reference cells tc - 1 .. tc + 1:
        // a grid coordinate is exactly half the reference one (1/(4r) is
        // 1/(2r) halved, so the products differ by an exact factor of two)
        const int gx0 = floor_half(tc.x - 1), gx1 = floor_half(tc.x + 1);
        const int gy0 = floor_half(tc.y - 1), gy1 = floor_half(tc.y + 1);
        const int gz0 = floor_half(tc.z - 1), gz1 = floor_half(tc.z + 1);
        for (int gz = gz0; gz <= gz1; ++gz)
            for (int gy = gy0; gy <= gy1; ++gy)
                for (int gx = gx0; gx <= gx1; ++gx) {
                    const uint32_t bk = cell_bucket(gx, gy, gz, d.hash_mask);
                    const unsigned long long hd = __ldcg(d.hash_head + bk);
                    if (static_cast<uint32_t>(hd >> 32) != tag) continue;
                    const uint32_t cnt = min(static_cast<uint32_t>(hd), NC_HASH_CAP);
                    for (uint32_t s = 0; s < cnt; ++s) take(__ldcg(&d.hash[bk * NC_HASH_CAP + s].pos));
                }
        for (uint32_t o = 0; o < over; ++o) take(__ldcg(&d.hash_over[o].pos));
        if (!room) return false;
        self_sort_run(run, n);
        for (uint32_t k = 0; k < n; ++k) {
            if (k > 0u && run[k] == run[k - 1u]) continue;   // a bucket met twice
            float pen;
            if (self_gs_pair(ctx, a, static_cast<uint32_t>(run[k]), target, false, pen)) {
                ++contacts;
                max_pen = fmaxf(max_pen, pen);
            }
        }
    }
    return true;
}

// The ordered pass's fast form (the calling CTA, all its threads): the
// listed pairs in contact at the start of the pass, or within NC_SELF_BAND
// of it, are ordered by the reference's key (first particle, rank of the
// second's cell around the first's, second particle) and run as wavefronts:
// a pair runs once the pairs before it in that order that share a particle
// have run, so each pair sees the positions the serial pass gives it (and
// acts or not as there).  The listed pairs farther apart run nowhere; they
// are proved idle afterwards (their start distance less both particles'
// largest displacements stays above the contact distance), as are the visit
// cells (every first particle's cell at its turn is its start cell).  False where a proof fails or the pairs do
// not fit the scratch: the caller then restores the start positions and
// runs the pairs serially.  Scratch (d.self_keys, u64 words): keys [0, K),
// predecessors [K, 2K) (via the first particle << 32 | via the second,
// 0xffffffff none), wavefront [2K, 3K) (bit 63: the first pair of its
// first particle's turn; low bits 0 pending, t run in wave t; ~0 a repeat),
// K = self_key_cap.  The predecessor search compares every pair with every
// other; beyond NC_SELF_WAVE_MAX pairs the serial form runs instead.
__device__ __noinline__ bool self_ordered_levels(const Ctx& ctx, uint32_t tag, uint32_t m,
                                                 unsigned long long& contacts_out, float& pen_out) {
    const DeviceCloth& d = ctx.d;
    const float target = 2.0f * ctx.c.radius;
    const float inv_ref = 1.0f / target;
    const float lim = 0.5f * target * (1.0f - 1.0e-4f);
    const uint32_t K = min(d.self_key_cap, NC_SELF_WAVE_MAX);
    unsigned long long* key = d.self_keys;
    unsigned long long* pred = d.self_keys + K;
    unsigned long long* wave = d.self_keys + 2u * K;
    constexpr uint32_t kNone = 0xffffffffu;
    __shared__ uint32_t s_k, s_bad, s_left;
    __shared__ unsigned long long s_contacts;
    __shared__ unsigned s_pen_bits;
    if (threadIdx.x == 0) {
        s_k = 0u;
        s_bad = 0u;
        s_contacts = 0ull;
        s_pen_bits = 0u;
    }
    // listed particles at their start positions, displacements cleared
    for (uint32_t k = threadIdx.x; k < 2u * m; k += blockDim.x) {
        const float4 en = __ldcg(d.self_list + k);
        const uint32_t i = __float_as_uint(en.w) & ~NC_SELF_KNOWN_BIT;
        d.self_x0[i] = make_float4(en.x, en.y, en.z, 0.0f);
        d.self_disp[i] = 0.0f;
        px_set(ctx, i, make_float4(en.x, en.y, en.z, px(ctx, i).w));
    }
    __syncthreads();
    // the pairs in contact at the start, keyed in the reference's order
    for (uint32_t k = threadIdx.x; k < m; k += blockDim.x) {
        const float4 ef = __ldcg(d.self_list + 2u * k), es = __ldcg(d.self_list + 2u * k + 1u);
        const uint32_t f = __float_as_uint(ef.w) & ~NC_SELF_KNOWN_BIT, s = __float_as_uint(es.w) & ~NC_SELF_KNOWN_BIT;
        const float L0 = len3(xyz(es) - xyz(ef));
        if (L0 >= target * (1.0f + NC_SELF_BAND)) continue;
        const int rank = self_visit_rank(self_ref_cell(xyz(ef), inv_ref), self_ref_cell(xyz(es), inv_ref));
        if (rank < 0 && L0 >= target) continue;   // never visited: the proof below covers it
        if (rank < 0 || s >= (1u << 27)) {
            s_bad = 1u;   // a touching pair outside the visit cells: the serial form decides
            continue;
        }
        const uint32_t slot = atomicAdd(&s_k, 1u);
        if (slot < K) key[slot] = (static_cast<unsigned long long>(f) << 32) |
                                  (static_cast<unsigned long long>(rank) << 27) | s;
    }
    __syncthreads();
    const uint32_t n = s_k;
    if (n > K || s_bad != 0u) return false;
    // predecessors through each particle (the latest earlier pair that
    // shares it; among equal keys the lowest slot), repeats, first pairs of
    // a turn
    for (uint32_t p = threadIdx.x; p < n; p += blockDim.x) {
        const unsigned long long kp = key[p];
        const uint32_t f = static_cast<uint32_t>(kp >> 32), s = static_cast<uint32_t>(kp) & ((1u << 27) - 1u);
        unsigned long long bf = 0ull, bs = 0ull;
        uint32_t pf = kNone, ps = kNone;
        bool repeat = false;
        for (uint32_t q = 0; q < n; ++q) {
            const unsigned long long kq = key[q];
            if (kq == kp) {
                repeat = repeat || q < p;
                continue;
            }
            if (kq > kp) continue;
            const uint32_t fq = static_cast<uint32_t>(kq >> 32), sq = static_cast<uint32_t>(kq) & ((1u << 27) - 1u);
            if ((fq == f || sq == f) && (pf == kNone || kq > bf)) {
                bf = kq;
                pf = q;
            }
            if ((fq == s || sq == s) && (ps == kNone || kq > bs)) {
                bs = kq;
                ps = q;
            }
        }
        pred[p] = (static_cast<unsigned long long>(pf) << 32) | ps;
        // first pair of f's turn: no earlier pair has f as its first particle
        const bool first = pf == kNone || static_cast<uint32_t>(bf >> 32) != f;
        wave[p] = repeat ? ~0ull : (first ? (1ull << 63) : 0ull);
    }
    if (threadIdx.x == 0) s_left = n;
    // wavefronts: a pair runs in wave t once both predecessors ran in an
    // earlier wave (every wave runs at least the earliest pending pair)
    for (uint32_t t = 1u;; ++t) {
        __syncthreads();   // the last wave's writes are visible
        const bool go = s_left != 0u && s_bad == 0u && t <= n + 1u;
        __syncthreads();   // everyone read the counters before any wave writes them
        if (!go) break;
        unsigned long long contacts = 0ull;
        float pen_max = 0.0f;
        uint32_t ran = 0u;
        for (uint32_t p = threadIdx.x; p < n; p += blockDim.x) {
            const unsigned long long w = wave[p];
            if (w == ~0ull) {
                if (t == 1u) ++ran;   // a repeat counts once, as done
                continue;
            }
            if ((w & ~(1ull << 63)) != 0ull) continue;
            const unsigned long long pp = pred[p];
            const uint32_t pf = static_cast<uint32_t>(pp >> 32), ps = static_cast<uint32_t>(pp);
            auto ready = [&](uint32_t q) {
                if (q == kNone) return true;
                const unsigned long long wq = wave[q] & ~(1ull << 63);
                return wq != 0ull && wq < t;
            };
            if (!ready(pf) || !ready(ps)) continue;
            const unsigned long long kp = key[p];
            const uint32_t f = static_cast<uint32_t>(kp >> 32), s = static_cast<uint32_t>(kp) & ((1u << 27) - 1u);
            if ((w >> 63) != 0ull) {
                // f's turn starts: its cell must still be its start cell
                const int3 tc = self_ref_cell(xyz(px(ctx, f)), inv_ref);
                const int3 sc = self_ref_cell(xyz(d.self_x0[f]), inv_ref);
                if (tc.x != sc.x || tc.y != sc.y || tc.z != sc.z) s_bad = 1u;
            }
            float pen;
            if (self_gs_pair(ctx, f, s, target, true, pen)) {
                ++contacts;
                pen_max = fmaxf(pen_max, pen);
            }
            wave[p] = (w & (1ull << 63)) | t;
            ++ran;
        }
        if (contacts != 0ull) {
            atomicAdd(&s_contacts, contacts);
            atomicMax(&s_pen_bits, __float_as_uint(pen_max));
        }
        if (ran != 0u) atomicSub(&s_left, ran);
    }
    if (threadIdx.x == 0 && s_left != 0u) s_bad = 1u;   // unreachable: the waves ran out
    // the proofs: every listed pair that started apart stays apart, and no
    // particle moved farther than the listing reach allows
    for (uint32_t k = threadIdx.x; k < m && s_bad == 0u; k += blockDim.x) {
        const float4 ef = __ldcg(d.self_list + 2u * k), es = __ldcg(d.self_list + 2u * k + 1u);
        const uint32_t f = __float_as_uint(ef.w) & ~NC_SELF_KNOWN_BIT, s = __float_as_uint(es.w) & ~NC_SELF_KNOWN_BIT;
        const float df = d.self_disp[f], ds = d.self_disp[s];
        if (df > lim || ds > lim) s_bad = 1u;
        const float L0 = len3(xyz(es) - xyz(ef));
        const int rank = self_visit_rank(self_ref_cell(xyz(ef), inv_ref), self_ref_cell(xyz(es), inv_ref));
        if (rank >= 0 && L0 < target * (1.0f + NC_SELF_BAND)) continue;   // one of the wavefront pairs
        if (L0 - (df + ds) <= target * (1.0f + 1.0e-5f)) s_bad = 1u;
    }
    __syncthreads();
    contacts_out = s_contacts;
    pen_out = __uint_as_float(s_pen_bits);
    return s_bad == 0u;
}

// The ordered pass (the CTA that calls it, all its threads): the listed
// pairs in the reference's order, the fallback where the checks fail, then
// the ground clamp of the particles it moved and the pass statistics.
__device__ __noinline__ void self_ordered(const Ctx& ctx, uint32_t tag, uint32_t listed) {
    const DeviceCloth& d = ctx.d;
    const SubCfg& c = ctx.c;
    const float target = 2.0f * c.radius;
    const float lim = 0.5f * target * (1.0f - 1.0e-4f);
    const unsigned long long mark_tag = static_cast<unsigned long long>(tag) << 32;
    __shared__ uint32_t s_state;   // 1: fallback, 2: the list grew
    __shared__ unsigned long long s_contacts;
    __shared__ float s_pen;
    uint32_t m = listed;
    bool fallback = m > d.self_list_cap;
    uint32_t rounds = 0u;
    unsigned long long fast_contacts = 0ull;
    float fast_pen = 0.0f;
    const bool fast = !fallback && self_ordered_levels(ctx, tag, m, fast_contacts, fast_pen);
    for (uint32_t round = 0; !fallback && !fast; ++round) {
        if (round == NC_SELF_ROUNDS) {
            fallback = true;
            break;
        }
        rounds = round + 1u;
        // listed particles back at their start positions
        for (uint32_t k = threadIdx.x; k < 2u * m; k += blockDim.x) {
            const float4 en = __ldcg(d.self_list + k);
            const uint32_t raw = __float_as_uint(en.w), i = raw & ~NC_SELF_KNOWN_BIT;
            atomicMax(d.self_mark + i, mark_tag);
            atomicOr(d.self_mark + i, NC_SELF_LISTED | ((raw & NC_SELF_KNOWN_BIT) ? NC_SELF_KNOWN : 0ull));
            d.self_x0[i] = make_float4(en.x, en.y, en.z, 0.0f);
            d.self_disp[i] = 0.0f;
            px_set(ctx, i, make_float4(en.x, en.y, en.z, px(ctx, i).w));
        }
        uint32_t pow2 = 1u;
        while (pow2 < m) pow2 <<= 1;
        for (uint32_t k = threadIdx.x; k < pow2; k += blockDim.x) {
            unsigned long long key = ~0ull;
            if (k < m) {
                const uint32_t f = __float_as_uint(__ldcg(&d.self_list[2u * k].w)) & ~NC_SELF_KNOWN_BIT;
                const uint32_t s = __float_as_uint(__ldcg(&d.self_list[2u * k + 1u].w)) & ~NC_SELF_KNOWN_BIT;
                key = (static_cast<unsigned long long>(f) << 32) | s;
            }
            d.self_keys[k] = key;
        }
        if (threadIdx.x == 0) s_state = 0u;
        __syncthreads();
        self_bitonic(d.self_keys, pow2);
        // the listed pairs, first particle by first particle; a turn's pairs
        // in the reference's cell order from the particle's position then
        if (threadIdx.x == 0) {
            const float inv_ref = 1.0f / target;
            unsigned long long* run = d.self_keys + 3u * d.self_key_cap;
            unsigned long long contacts = 0ull;
            float pen_max = 0.0f;
            for (uint32_t k = 0; k < m && s_state == 0u;) {
                const uint32_t a = static_cast<uint32_t>(d.self_keys[k] >> 32);
                const int3 tc = self_ref_cell(xyz(px(ctx, a)), inv_ref);
                uint32_t n = 0u;
                for (; k < m && static_cast<uint32_t>(d.self_keys[k] >> 32) == a; ++k) {
                    if (k > 0u && d.self_keys[k] == d.self_keys[k - 1u]) continue;   // listed by both sides
                    const uint32_t b = static_cast<uint32_t>(d.self_keys[k]);
                    const int rank = self_visit_rank(tc, self_ref_cell(xyz(d.self_x0[b]), inv_ref));
                    if (rank < 0) continue;
                    if (n == NC_SELF_GROUP) {
                        s_state = 1u;
                        break;
                    }
                    run[n++] = (static_cast<unsigned long long>(rank) << 32) | b;
                }
                self_sort_run(run, n);
                for (uint32_t j = 0; j < n; ++j) {
                    float pen;
                    if (self_gs_pair(ctx, a, static_cast<uint32_t>(run[j]), target, true, pen)) {
                        ++contacts;
                        pen_max = fmaxf(pen_max, pen);
                    }
                }
            }
            s_contacts = contacts;
            s_pen = pen_max;
        }
        __syncthreads();
        // the checks: every listed particle within r of its start; a moved
        // particle whose neighbourhood is not listed yet lists it
        for (uint32_t k = threadIdx.x; k < 2u * m; k += blockDim.x) {
            const uint32_t i = __float_as_uint(__ldcg(&d.self_list[k].w)) & ~NC_SELF_KNOWN_BIT;
            const float dsp = __ldcg(d.self_disp + i);
            if (dsp > lim) {
                atomicOr(&s_state, 1u);
            } else if (dsp > 0.0f) {
                const unsigned long long old = atomicOr(d.self_mark + i, NC_SELF_KNOWN);
                if ((old & NC_SELF_KNOWN) == 0ull) {
                    const float4 x0 = d.self_x0[i];
                    bool simple_met = false;
                    self_scan_cell(ctx, tag, x0, [&](const float4& e) {
                        const uint32_t b = __float_as_uint(e.w);
                        if (b == i || len3(xyz(e) - xyz(x0)) >= 2.0f * target) return;
                        const unsigned long long mb = __ldcg(d.self_mark + b);
                        if ((mb >> 32) == tag && (mb & NC_SELF_SIMPLE)) simple_met = true;
                    });
                    const float4 xi = make_float4(x0.x, x0.y, x0.z, px(ctx, i).w);
                    if (simple_met || !self_list_near(ctx, tag, i, xi)) atomicOr(&s_state, 1u);
                    atomicOr(&s_state, 2u);
                }
            }
        }
        __syncthreads();
        const uint32_t state = s_state;
        if (state & 1u) {
            fallback = true;
            break;
        }
        if ((state & 2u) == 0u) break;
        const unsigned long long head = __ldcg(d.self_list_head);
        m = static_cast<uint32_t>(head);
        fallback = m > d.self_list_cap;
        __syncthreads();
    }
    if (fallback) {
        // every particle back at its start-of-pass position
        for (uint32_t bk = threadIdx.x; bk <= d.hash_mask; bk += blockDim.x) {
            const unsigned long long hd = __ldcg(d.hash_head + bk);
            if (static_cast<uint32_t>(hd >> 32) != tag) continue;
            const uint32_t cnt = min(static_cast<uint32_t>(hd), NC_HASH_CAP);
            for (uint32_t s = 0; s < cnt; ++s) {
                const float4 e = __ldcg(&d.hash[bk * NC_HASH_CAP + s].pos);
                const uint32_t i = __float_as_uint(e.w);
                px_set(ctx, i, make_float4(e.x, e.y, e.z, px(ctx, i).w));
            }
        }
        {
            const unsigned long long oh = __ldcg(d.hash_over_head);
            const uint32_t over = static_cast<uint32_t>(oh >> 32) == tag ? min(static_cast<uint32_t>(oh), d.n) : 0u;
            for (uint32_t o = threadIdx.x; o < over; o += blockDim.x) {
                const float4 e = __ldcg(&d.hash_over[o].pos);
                const uint32_t i = __float_as_uint(e.w);
                px_set(ctx, i, make_float4(e.x, e.y, e.z, px(ctx, i).w));
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            unsigned long long contacts = 0ull;
            float pen = 0.0f;
            if (!self_serial_all(ctx, tag, contacts, pen)) fail(d, NUMI_CLOTH_FAILURE_RANGE);
            // the pass's statistics are this loop's alone
            d.self_pass_stats[0] = contacts;
            d.self_pass_stats[1] = __float_as_uint(pen);
        }
        __syncthreads();
        if (c.ground)
            for (uint32_t i = threadIdx.x; i < d.n; i += blockDim.x) {
                const float4 p = px(ctx, i);
                if (c.radius - p.z > 0.0f) px_set(ctx, i, make_float4(p.x, p.y, c.radius, p.w));
            }
    } else {
        if (c.ground)
            for (uint32_t k = threadIdx.x; k < 2u * m; k += blockDim.x) {
                const uint32_t i = __float_as_uint(__ldcg(&d.self_list[k].w)) & ~NC_SELF_KNOWN_BIT;
                const float4 p = px(ctx, i);
                if (c.radius - p.z > 0.0f) px_set(ctx, i, make_float4(p.x, p.y, c.radius, p.w));
            }
        const unsigned long long ordered_contacts = fast ? fast_contacts : s_contacts;
        const float ordered_pen = fast ? fast_pen : s_pen;
        if (threadIdx.x == 0 && ordered_contacts != 0ull) {
            d.self_pass_stats[0] += ordered_contacts;
            d.self_pass_stats[1] =
                max(d.self_pass_stats[1], static_cast<unsigned long long>(__float_as_uint(ordered_pen)));
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        self_fold(d);
        d.self_stats[2] += 1ull;
        d.self_stats[3] += m;
        d.self_stats[4] += rounds;
        d.self_stats[5] += fallback ? 1ull : 0ull;
    }
}

// After phase A and the barrier behind it, every CTA alike: the ordered
// pass where phase A listed pairs (then one more barrier), else only the
// statistics.
__device__ bool self_settle(Ctx& ctx, uint32_t it) {
    const DeviceCloth& d = ctx.d;
    const uint32_t tag = self_pass_tag(ctx, it);
    const unsigned long long head = __ldcg(d.self_list_head);
    const uint32_t listed = static_cast<uint32_t>(head >> 32) == tag ? static_cast<uint32_t>(head) : 0u;
    if (listed == 0u) {
        if (ctx.grip_cta && threadIdx.x == 0) self_fold(d);
        return true;
    }
    if (ctx.grip_cta) self_ordered(ctx, tag, listed);
    NC_SYNC(ctx);
    return true;
}


}  // namespace
}  // namespace nc

#include "cloth_edge.cuh"

namespace nc {
namespace {   // internal linkage: the edge kernels' unit includes these too

// Ground clamp (tools/cloth_bag.cpp:2655-2690).
__device__ void fruit_ground(Ctx& ctx);

__device__ void phase_ground(Ctx& ctx) {
    const SubCfg& c = ctx.c;
    fruit_flush(ctx);
    if (!c.ground) return;
    for (Range r = particle_range(ctx); r.i < r.end; r.i += r.stride) {
        const float4 p = px(ctx, r.i);
        if (c.radius - p.z > 0.0f) px_set(ctx, r.i, make_float4(p.x, p.y, c.radius, p.w));
    }
    fruit_ground(ctx);
}

// The fruits' ground clamp with its normal impulse (fruit CTA; ground on).
__device__ void fruit_ground(Ctx& ctx) {
    const DeviceCloth& d = ctx.d;
    const SubCfg& c = ctx.c;
    if (ctx.fruit_cta) {
        for (uint32_t f = threadIdx.x; f < d.f_count; f += blockDim.x) {
            NumiClothFruit& fr = d.fruits[f];
            const float pen = fr.previousAndRadius.w - fr.positionAndInverseMass.z;
            if (pen > 0.0f) {
                fr.velocityAndGroundImpulse.w =
                    fr.velocityAndGroundImpulse.w + pen / (fr.positionAndInverseMass.w * c.dt);
                fr.positionAndInverseMass.z = fr.previousAndRadius.w;
            }
        }
    }
}

template <bool kIlp>
__device__ bool strain_sweeps(Ctx& ctx) {
    const DeviceCloth& d = ctx.d;
    for (uint32_t sw = 0; sw < ctx.s.strain_sweeps; ++sw) {
        if constexpr (kIlp) {
            for (uint32_t b = 0; b < d.n_dist_batches; ++b) {
                const Batch bt = d.dist_batches[b];
                if (bt.limited == 0u) continue;
                fruit_flush(ctx);
                strain_colour(ctx, bt.first, bt.limited);
                NC_SYNC(ctx);
            }
        } else {
            for (uint32_t b = 0; b < d.n_dist_batches; ++b) {
                const Batch bt = d.dist_batches[b];
                if (bt.limited == 0u) continue;
                fruit_flush(ctx);
                for (Range r = colour_items(ctx, b, bt.limited); r.i < r.end; r.i += r.stride) {
                    const uint32_t k = colour_item(ctx, r.i);
                    if (k < bt.limited) limit_strain(ctx, bt.first + k);
                }
                // a colour follows: a later limited batch, or the next sweep
                bool more = sw + 1u < ctx.s.strain_sweeps;
                for (uint32_t c = b + 1u; c < d.n_dist_batches && !more; ++c) more = d.dist_batches[c].limited != 0u;
                NC_CSYNC(ctx, more);
            }
        }
    }
    return true;
}

// Residuals in FP64 (tools/cloth_bag.cpp:1765-1780, 1880-1895, 3111-3139);
// max over blocks, every CTA reads all partials and takes the same decision.
__device__ void residual_partials(Ctx& ctx, double* out3) {
    const DeviceCloth& d = ctx.d;
    const SubCfg& c = ctx.c;
    double strain = 0.0, ground = 0.0, fruit = 0.0;
    for (Range r = item_range(ctx, d.d_count); r.i < r.end; r.i += r.stride) {
        const uint32_t k = r.i;
        const float4 m = __ldg(d.d_mat + k);
        if (!(m.w > 0.0f)) continue;
        const uint2 ij = __ldg(d.d_ij + k);
        const float4 a = px(ctx, ij.x);
        const float4 b = px(ctx, ij.y);
        const double dx = static_cast<double>(b.x) - a.x, dy = static_cast<double>(b.y) - a.y,
                     dz = static_cast<double>(b.z) - a.z;
        const double L = sqrt((dx * dx + dy * dy) + dz * dz);
        const double maxL = static_cast<double>(m.x) * (1.0 + static_cast<double>(m.w));
        strain = fmax(strain, L - maxL);
    }
    if (c.ground) {
        for (Range r = particle_range(ctx); r.i < r.end; r.i += r.stride)
            ground = fmax(ground, static_cast<double>(c.radius) - static_cast<double>(px(ctx, r.i).z));
        if (ctx.rank == 0)
            for (uint32_t f = threadIdx.x; f < d.f_count; f += blockDim.x)
                ground = fmax(ground, static_cast<double>(__ldcg(&d.fruits[f].previousAndRadius.w)) -
                                          static_cast<double>(__ldcg(&d.fruits[f].positionAndInverseMass.z)));
    }
    if (d.f_count > 0u) {
        for (uint32_t b = 0; b < d.n_dist_batches; ++b) {
            const Batch bt = d.dist_batches[b];
            for (Range r = item_range(ctx, bt.yarn); r.i < r.end; r.i += r.stride) {
                const uint2 ij = __ldg(d.d_ij + bt.first + r.i);
                const float4 pa = px(ctx, ij.x);
                const float4 pb = px(ctx, ij.y);
                for (uint32_t f = 0; f < d.f_count; ++f) {
                    const NumiClothFruit& fr = d.fruits[f];
                    const double X[3] = {__ldcg(&fr.positionAndInverseMass.x), __ldcg(&fr.positionAndInverseMass.y),
                                         __ldcg(&fr.positionAndInverseMass.z)};
                    const double target = static_cast<double>(__ldcg(&fr.previousAndRadius.w)) + c.radius;
                    const double A[3] = {pa.x, pa.y, pa.z};
                    const double B[3] = {pb.x, pb.y, pb.z};
                    bool outside = false;
                    for (int e = 0; e < 3; ++e)
                        outside = outside || X[e] < fmin(A[e], B[e]) - target || X[e] > fmax(A[e], B[e]) + target;
                    if (outside) continue;
                    const double dir[3] = {B[0] - A[0], B[1] - A[1], B[2] - A[2]};
                    const double lb = (dir[0] * dir[0] + dir[1] * dir[1]) + dir[2] * dir[2];
                    double t = 0.0;
                    if (lb > 1.0e-20) {
                        const double proj = (dir[0] * (X[0] - A[0]) + dir[1] * (X[1] - A[1])) + dir[2] * (X[2] - A[2]);
                        t = fmin(fmax(proj / lb, 0.0), 1.0);
                    }
                    const double cx = A[0] + dir[0] * t - X[0], cy = A[1] + dir[1] * t - X[1],
                                 cz = A[2] + dir[2] * t - X[2];
                    fruit = fmax(fruit, target - sqrt((cx * cx + cy * cy) + cz * cz));
                }
            }
        }
    }
    double (*s_r)[NC_BLOCK_MAX] = nc_red_smem;
    s_r[0][threadIdx.x] = strain;
    s_r[1][threadIdx.x] = ground;
    s_r[2][threadIdx.x] = fruit;
    __syncthreads();
    for (uint32_t st = blockDim.x / 2u; st > 0u; st >>= 1u) {
        if (threadIdx.x < st)
            for (int e = 0; e < 3; ++e) s_r[e][threadIdx.x] = fmax(s_r[e][threadIdx.x], s_r[e][threadIdx.x + st]);
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int e = 0; e < 3; ++e) out3[3u * ctx.rank + e] = s_r[e][0];
    __syncthreads();
}

__device__ bool residuals_converged(Ctx& ctx) {
    const DeviceCloth& d = ctx.d;
    double (*s_r)[NC_BLOCK_MAX] = nc_red_smem;
    double r[3] = {0.0, 0.0, 0.0};
    for (uint32_t b = threadIdx.x; b < ctx.ranks; b += blockDim.x)
        for (int e = 0; e < 3; ++e) r[e] = fmax(r[e], __ldcg(d.red + 3u * b + e));
    for (int e = 0; e < 3; ++e) s_r[e][threadIdx.x] = r[e];
    __syncthreads();
    for (uint32_t st = blockDim.x / 2u; st > 0u; st >>= 1u) {
        if (threadIdx.x < st)
            for (int e = 0; e < 3; ++e) s_r[e][threadIdx.x] = fmax(s_r[e][threadIdx.x], s_r[e][threadIdx.x + st]);
        __syncthreads();
    }
    const bool ok = s_r[2][0] < 1.0e-6 && s_r[1][0] < 1.0e-9 && s_r[0][0] < 1.0e-6;
    __syncthreads();
    return ok;
}

template <bool kIlp>
__device__ bool contacts_pass(Ctx& ctx, bool with_strain) {
    // fruit pairs (fruit CTA) -> fruit/yarn -> [strain] -> ground
    if (ctx.fruit_cta && ctx.d.p_count > 0u) {
        fruit_flush(ctx);
        fruit_pair_sweep(ctx.d, *ctx.fs, ctx.c.dt);
    }
    if (ctx.d.p_count > 0u) NC_SYNC(ctx);
    if (!yarn_sweep(ctx)) return false;
    if (with_strain && !strain_sweeps<kIlp>(ctx)) return false;
    phase_ground(ctx);
    NC_SYNC(ctx);
    return true;
}

// Finalize + cloth/ground friction (tools/cloth_bag.cpp:5186-5211, 2076-2115).
// Finalize of one particle at its final position p: the velocity from the
// substep's motion with the ground normal impulse (velocity w) and the
// cloth/ground Coulomb friction; a particle of zero inverse mass returns to
// its rest position (true: p was moved).
__device__ __forceinline__ bool finalize_particle(const Ctx& ctx, uint32_t i, float4& p, const float4& vv,
                                                  float4& vout) {
    const DeviceCloth& d = ctx.d;
    const SubCfg& c = ctx.c;
    const float inv_dt = 1.0f / c.dt;
    const V3 prev = xyz(ld(d.xp + i));
    V3 pos = xyz(p);
    V3 vel;
    float gi = 0.0f;
    bool moved = false;
    if (p.w == 0.0f) {
        pos = xyz(__ldg(d.rest + i));
        vel = (pos - prev) * inv_dt;
        p = with_xyz(p, pos);
        moved = true;
    } else {
        vel = (pos - prev) * inv_dt;
        if (c.ground && pos.z <= c.radius + 1.0e-6f) {
            const float nvc = vel.z - vv.w;
            gi = fmaxf(0.0f, nvc / p.w);
        }
        if (ctx.s.frictions && gi > 0.0f) {
            const V3 tv{vel.x, vel.y, 0.0f};
            const float slip = len3(tv);
            if (!(slip < 1.0e-10f)) {
                const float limit = c.mu_cloth_ground * gi;
                const float ti = fminf(slip / p.w, limit);
                if (ti > 0.0f) vel = vel - tv * (ti * p.w / slip);
            }
        }
    }
    if (!finite3(vel)) fail(d, NUMI_CLOTH_FAILURE_NONFINITE);
    vout = make_float4(vel.x, vel.y, vel.z, gi);
    return moved;
}

__device__ void fruit_finalize(Ctx& ctx);

__device__ void phase_finalize(Ctx& ctx) {
    fruit_flush(ctx);
    for (Range r = particle_range(ctx); r.i < r.end; r.i += r.stride) {
        const uint32_t i = r.i;
        float4 p = px(ctx, i);
        float4 v;
        if (finalize_particle(ctx, i, p, pv(ctx, i), v)) px_set(ctx, i, p);
        pv_set(ctx, i, v);
    }
    fruit_finalize(ctx);
}

// The fruits' velocities from their substep motion (fruit CTA).
__device__ void fruit_finalize(Ctx& ctx) {
    const DeviceCloth& d = ctx.d;
    const float inv_dt = 1.0f / ctx.c.dt;
    if (ctx.fruit_cta) {
        for (uint32_t f = threadIdx.x; f < d.f_count; f += blockDim.x) {
            FruitState s = load_fruit(d.fruits[f]);
            s.v = (s.x - s.prev) * inv_dt;
            if (!finite3(s.x) || !finite3(s.v)) fail(d, NUMI_CLOTH_FAILURE_NONFINITE);
            store_fruit(d.fruits[f], s);
        }
    }
}

// Fruit/yarn Coulomb friction (tools/cloth_bag.cpp:3178-3270) of one
// recorded segment, with fruit velocities frozen over the sweep; the fruit
// velocity changes go into the CTA's fixed-point sums.
// A recorded segment's endpoints and slot states: what the friction of the
// segment reads that no yarn colour of the sweep changes.
struct FrictionSeg {
    uint32_t seg;
    uint2 ij;
    uint32_t st[NC_YARN_SLOTS];
};
__device__ __forceinline__ FrictionSeg friction_seg(const DeviceCloth& d, uint32_t seg) {
    FrictionSeg fs;
    fs.seg = seg;
    fs.ij = __ldg(d.d_ij + seg);
#pragma unroll
    for (uint32_t q = 0; q < NC_YARN_SLOTS; ++q)
        fs.st[q] = __float_as_uint(__ldcg(&d.yarn_slot_b[seg * NC_YARN_SLOTS + q].z));
    return fs;
}

// The friction of one segment on its loaded endpoints: positions pa, pb,
// velocities va, vb (updated), slot tags st and the slots' records ra, rb
// (only the live ones are read).
__device__ __forceinline__ void yarn_friction_core(const Ctx& ctx, const float4& pa, const float4& pb, float4& va,
                                                   float4& vb, const uint32_t* st, const float4* ra, const float4* rb,
                                                   const float4* s_vw, const float4* s_or, unsigned long long* s_sum) {
    const SubCfg& c = ctx.c;
    // Live records of this segment, visited in ascending fruit order.
    const uint32_t live = ctx.epoch & 0x3ffffffu;
    uint32_t fruit_of[NC_YARN_SLOTS];
    uint32_t nlive = 0;
#pragma unroll
    for (uint32_t q = 0; q < NC_YARN_SLOTS; ++q) {
        fruit_of[q] = ((st[q] >> 6) == live) ? (st[q] & 63u) : 0xffffffffu;
        nlive += fruit_of[q] != 0xffffffffu ? 1u : 0u;
    }
    for (uint32_t visit = 0; visit < nlive; ++visit) {
        uint32_t slot = 0;
        uint32_t f = 0xffffffffu;
#pragma unroll
        for (uint32_t q = 0; q < NC_YARN_SLOTS; ++q)
            if (fruit_of[q] < f) {
                f = fruit_of[q];
                slot = q;
            }
#pragma unroll
        for (uint32_t q = 0; q < NC_YARN_SLOTS; ++q)
            if (q == slot) fruit_of[q] = 0xffffffffu;
        float4 sa = ra[0], sb = rb[0];
#pragma unroll
        for (uint32_t q = 1; q < NC_YARN_SLOTS; ++q)
            if (q == slot) {
                sa = ra[q];
                sb = rb[q];
            }
        const float ni = sa.w;
        const V3 wn{sa.x, sa.y, sa.z};
        if (ni <= 0.0f || lsq(wn) < 1.0e-20f) continue;
        FruitState fr;
        {
            const float4 vw = s_vw[f];
            const float4 orr = s_or[f];
            fr.v = V3{vw.x, vw.y, vw.z};
            fr.w = vw.w;
            fr.omega = V3{orr.x, orr.y, orr.z};
            fr.radius = orr.w;
        }
        const V3 normal = normalized3(wn);
        float wt[2] = {sb.x / ni, sb.y / ni};
        const float sum = wt[0] + wt[1];
        if (sum <= 1.0e-12f) continue;
        wt[0] = wt[0] / sum;
        wt[1] = wt[1] / sum;
        const V3 yv = (V3{0.0f, 0.0f, 0.0f} + xyz(va) * wt[0]) + xyz(vb) * wt[1];
        const V3 off = normal * -fr.radius;
        const V3 bcv = fr.v + cross3(fr.omega, off);
        const V3 rel = bcv - yv;
        const V3 tv = rel - normal * dot3(rel, normal);
        const float slip = len3(tv);
        if (slip < 1.0e-10f) continue;
        const V3 t = vdiv(tv, slip);
        const float inv_i = inverse_inertia(fr.w, fr.radius);
        float den = fr.w + inv_i * lsq(cross3(off, t));
        V3 resp[2];
        const float4* pp[2] = {&pa, &pb};
        for (int s = 0; s < 2; ++s) {
            resp[s] = t * pp[s]->w;
            if (c.ground && pp[s]->z <= c.radius + 1.0e-6f && resp[s].z < 0.0f) resp[s].z = 0.0f;
            den = den + dot3(t, resp[s]) * wt[s] * wt[s];
        }
        if (den <= 0.0f) continue;
        const float limit = c.mu_fruit_yarn * ni;
        const float ti = fminf(slip / den, limit);
        if (ti <= 0.0f) continue;
        const V3 imp = t * -ti;
        const V3 dv = imp * fr.w;
        const V3 dw = cross3(off, imp) * inv_i;
        cta_sums_add(s_sum + 6u * f + 0u, dv.x);
        cta_sums_add(s_sum + 6u * f + 1u, dv.y);
        cta_sums_add(s_sum + 6u * f + 2u, dv.z);
        cta_sums_add(s_sum + 6u * f + 3u, dw.x);
        cta_sums_add(s_sum + 6u * f + 4u, dw.y);
        cta_sums_add(s_sum + 6u * f + 5u, dw.z);
        const V3 na = xyz(va) + resp[0] * (ti * wt[0]);
        const V3 nb = xyz(vb) + resp[1] * (ti * wt[1]);
        va = with_xyz(va, na);
        vb = with_xyz(vb, nb);
    }
}


// The slot records of a segment's live slots (the others zero).
__device__ __forceinline__ void friction_records(const Ctx& ctx, uint32_t seg, const uint32_t* st, float4* ra,
                                                 float4* rb) {
    const DeviceCloth& d = ctx.d;
    const uint32_t live = ctx.epoch & 0x3ffffffu;
#pragma unroll
    for (uint32_t q = 0; q < NC_YARN_SLOTS; ++q) {
        const bool on = (st[q] >> 6) == live;
        ra[q] = on ? __ldcg(&d.yarn_slot_a[seg * NC_YARN_SLOTS + q]) : make_float4(0, 0, 0, 0);
        rb[q] = on ? __ldcg(&d.yarn_slot_b[seg * NC_YARN_SLOTS + q]) : make_float4(0, 0, 0, 0);
    }
}

__device__ __forceinline__ void yarn_friction_segment(const Ctx& ctx, const FrictionSeg& fseg, const float4* s_vw,
                                                      const float4* s_or, unsigned long long* s_sum) {
    const uint2 ij = fseg.ij;
    const float4 pa = px(ctx, ij.x);
    const float4 pb = px(ctx, ij.y);
    float4 va = pv(ctx, ij.x);
    float4 vb = pv(ctx, ij.y);
    float4 ra[NC_YARN_SLOTS], rb[NC_YARN_SLOTS];
    friction_records(ctx, fseg.seg, fseg.st, ra, rb);
    yarn_friction_core(ctx, pa, pb, va, vb, fseg.st, ra, rb, s_vw, s_or, s_sum);
    pv_set(ctx, ij.x, va);
    pv_set(ctx, ij.y, vb);
}

// Fruit state of the fruit/yarn friction sweep (fruit CTA): the fixed-point
// velocity and spin sums, the staged velocities and spins.
__shared__ unsigned long long nc_fric_sum[6u * NC_MAX_FRUITS];
__shared__ float4 nc_fric_vw[NC_MAX_FRUITS];
__shared__ float4 nc_fric_or[NC_MAX_FRUITS];

// Stage the substep's recorded segments for the friction sweep (fruit CTA,
// tile mode): what the sweep reads that no later phase changes, read as
// soon as the fruit/yarn sweep has ended: segment, endpoints, slot tags and
// the live slots' records, and for every endpoint the first endpoint of the
// list with the same particle (where a later colour must see an earlier
// colour's velocity change).  More segments than NC_FRICTION_STAGE are not
// staged (the sweep reads them from global memory).
__device__ void friction_stage(const Ctx& ctx) {
    if (!ctx.fruit_cta || ctx.fst == nullptr) return;
    const DeviceCloth& d = ctx.d;
    FrictionStage& fs = *ctx.fst;
    const uint32_t listed = min(__ldcg(d.yarn_list_n), d.d_count);
    const uint32_t n = listed <= NC_FRICTION_STAGE ? listed : NC_FRICTION_STAGE + 1u;
    if (threadIdx.x == 0) fs.count = n;
    if (n <= NC_FRICTION_STAGE) {
        for (uint32_t k = threadIdx.x; k < n; k += blockDim.x) {
            const uint32_t seg = __ldcg(d.yarn_list + k);
            const uint2 ij = __ldg(d.d_ij + seg);
            fs.seg[k] = seg;
            fs.pid[2u * k] = ij.x;
            fs.pid[2u * k + 1u] = ij.y;
#pragma unroll
            for (uint32_t q = 0; q < NC_YARN_SLOTS; ++q)
                fs.tag[k][q] = __float_as_uint(__ldcg(&d.yarn_slot_b[seg * NC_YARN_SLOTS + q].z));
            friction_records(ctx, seg, fs.tag[k], fs.ra[k], fs.rb[k]);
        }
        __syncthreads();
        for (uint32_t e = threadIdx.x; e < 2u * n; e += blockDim.x) {
            uint32_t r = e;
            for (uint32_t o = 0; o < e; ++o)
                if (fs.pid[o] == fs.pid[e]) {
                    r = o;
                    break;
                }
            fs.rep[e] = static_cast<unsigned short>(r);
        }
    }
    __syncthreads();
}

// The fruit/yarn friction sweep on the fruit CTA: the yarn colours in order,
// each over its segments on the substep's recorded-segment list (a few per
// fruit), CTA barriers between the colours; segments of a colour share no
// particle.  The fruit velocity changes are exact integer sums, so adding
// them in this one CTA gives the same totals as summing per CTA; the CTA
// applies them itself.
__device__ void yarn_friction_sweep_global(Ctx& ctx) {
    const DeviceCloth& d = ctx.d;
    unsigned long long* s_sum = nc_fric_sum;
    float4* s_vw = nc_fric_vw;   // velocity xyz, inverse mass
    float4* s_or = nc_fric_or;   // spin xyz, radius
    // this thread's first listed segment, loaded once for all colours (the
    // colours then wait only on their particle loads; the loads overlap the
    // fruit staging); further ones (more segments listed than threads) are
    // loaded in their colour
    const uint32_t listed = min(__ldcg(d.yarn_list_n), d.d_count);
    FrictionSeg mine{};
    if (threadIdx.x < listed) mine = friction_seg(d, __ldcg(d.yarn_list + threadIdx.x));
    cta_sums_clear(s_sum, 6u * d.f_count);
    for (uint32_t f = threadIdx.x; f < d.f_count; f += blockDim.x) {
        const NumiClothFruit& fr = d.fruits[f];
        const float4 vg = __ldcg(reinterpret_cast<const float4*>(&fr.velocityAndGroundImpulse));
        const float4 om = __ldcg(reinterpret_cast<const float4*>(&fr.angularVelocity));
        s_vw[f] = make_float4(vg.x, vg.y, vg.z, __ldcg(&fr.positionAndInverseMass.w));
        s_or[f] = make_float4(om.x, om.y, om.z, __ldcg(&fr.previousAndRadius.w));
    }
    __syncthreads();
    for (uint32_t b = 0; b < d.n_dist_batches; ++b) {
        const Batch bt = d.dist_batches[b];
        if (bt.yarn == 0u) continue;
        if (threadIdx.x < listed && mine.seg >= bt.first && mine.seg < bt.first + bt.yarn)
            yarn_friction_segment(ctx, mine, s_vw, s_or, s_sum);
        for (uint32_t e = threadIdx.x + blockDim.x; e < listed; e += blockDim.x) {
            const uint32_t seg = __ldcg(d.yarn_list + e);
            if (seg < bt.first || seg >= bt.first + bt.yarn) continue;
            yarn_friction_segment(ctx, friction_seg(d, seg), s_vw, s_or, s_sum);
        }
        __syncthreads();
    }
    // the fruits' velocities and spins with the friction sums, handed to the
    // fruit tail in shared memory (the fruit CTA's own fruit state)
    for (uint32_t f = threadIdx.x; f < d.f_count; f += blockDim.x) {
        unsigned long long sm[6];
        for (int k = 0; k < 6; ++k) sm[k] = s_sum[6u * f + k];
        const float4 v = s_vw[f], w = s_or[f];
        ctx.fs->v[f] = make_float4(v.x + from_fixed(sm[0]), v.y + from_fixed(sm[1]), v.z + from_fixed(sm[2]), v.w);
        ctx.fs->o[f] = make_float4(w.x + from_fixed(sm[3]), w.y + from_fixed(sm[4]), w.z + from_fixed(sm[5]), w.w);
    }
    __syncthreads();
}

// The sweep on staged segments (friction_stage, tile mode): the endpoints
// are loaded once, the colours run in shared memory, the velocities are
// stored once; unstaged, the sweep over global memory.
__device__ void yarn_friction_sweep(Ctx& ctx) {
    if (!ctx.fruit_cta) return;
    if (ctx.fst == nullptr || ctx.fst->count > NC_FRICTION_STAGE) {
        yarn_friction_sweep_global(ctx);
        return;
    }
    const DeviceCloth& d = ctx.d;
    FrictionStage& fs = *ctx.fst;
    unsigned long long* s_sum = nc_fric_sum;
    float4* s_vw = nc_fric_vw;
    float4* s_or = nc_fric_or;
    const uint32_t n = fs.count;
    cta_sums_clear(s_sum, 6u * d.f_count);
    for (uint32_t f = threadIdx.x; f < d.f_count; f += blockDim.x) {
        const NumiClothFruit& fr = d.fruits[f];
        const float4 vg = __ldcg(reinterpret_cast<const float4*>(&fr.velocityAndGroundImpulse));
        const float4 om = __ldcg(reinterpret_cast<const float4*>(&fr.angularVelocity));
        s_vw[f] = make_float4(vg.x, vg.y, vg.z, __ldcg(&fr.positionAndInverseMass.w));
        s_or[f] = make_float4(om.x, om.y, om.z, __ldcg(&fr.previousAndRadius.w));
    }
    for (uint32_t e = threadIdx.x; e < 2u * n; e += blockDim.x)
        if (fs.rep[e] == e) {
            fs.x[e] = px(ctx, fs.pid[e]);
            fs.v[e] = pv(ctx, fs.pid[e]);
        }
    __syncthreads();
    for (uint32_t b = 0; b < d.n_dist_batches; ++b) {
        const Batch bt = d.dist_batches[b];
        if (bt.yarn == 0u) continue;
        for (uint32_t k = threadIdx.x; k < n; k += blockDim.x) {
            const uint32_t seg = fs.seg[k];
            if (seg < bt.first || seg >= bt.first + bt.yarn) continue;
            const uint32_t ea = fs.rep[2u * k], eb = fs.rep[2u * k + 1u];
            float4 va = fs.v[ea], vb = fs.v[eb];
            yarn_friction_core(ctx, fs.x[ea], fs.x[eb], va, vb, fs.tag[k], fs.ra[k], fs.rb[k], s_vw, s_or, s_sum);
            fs.v[ea] = va;
            fs.v[eb] = vb;
        }
        __syncthreads();
    }
    for (uint32_t e = threadIdx.x; e < 2u * n; e += blockDim.x)
        if (fs.rep[e] == e) pv_set(ctx, fs.pid[e], fs.v[e]);
    // the fruits' velocities and spins with the friction sums, handed to the
    // fruit tail in shared memory (the fruit CTA's own fruit state)
    for (uint32_t f = threadIdx.x; f < d.f_count; f += blockDim.x) {
        unsigned long long sm[6];
        for (int q = 0; q < 6; ++q) sm[q] = s_sum[6u * f + q];
        const float4 v = s_vw[f], w = s_or[f];
        ctx.fs->v[f] = make_float4(v.x + from_fixed(sm[0]), v.y + from_fixed(sm[1]), v.z + from_fixed(sm[2]), v.w);
        ctx.fs->o[f] = make_float4(w.x + from_fixed(sm[3]), w.y + from_fixed(sm[4]), w.z + from_fixed(sm[5]), w.w);
    }
    __syncthreads();
}

// ---------------------------------------------------------- release ----
// Released-fruit masks (updateReleasedFruit, tools/cloth_bag.cpp:4545-4597):
// the mouth frame from the ordered rim, a fruit's projection tested against
// the rim polygon, and the 0.025 m hysteresis on leaving through the mouth
// or around it.  FP64 throughout, in the reference's operation order, on
// the fruit CTA (one thread per fruit; the frame by one thread).
struct D3 {
    double x, y, z;
};
__device__ __forceinline__ D3 operator+(D3 a, D3 b) { return D3{a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ D3 operator-(D3 a, D3 b) { return D3{a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ D3 operator*(D3 a, double s) { return D3{a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ double dot_d(D3 a, D3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
__device__ __forceinline__ D3 cross_d(D3 a, D3 b) {
    return D3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ D3 vdiv_d(D3 a, double s) { return a * (1.0 / s); }
__device__ __forceinline__ D3 normalized_d(D3 a) {
    const double m = sqrt(dot_d(a, a));
    return m > 1.0e-14 ? vdiv_d(a, m) : D3{1.0, 0.0, 0.0};
}
__device__ __forceinline__ double clamp01_d(double v) { return v < 0.0 ? 0.0 : (1.0 < v ? 1.0 : v); }
__device__ __forceinline__ double min_d(double a, double b) { return b < a ? b : a; }
__device__ __forceinline__ D3 to_d3(float4 p) { return D3{static_cast<double>(p.x), static_cast<double>(p.y), static_cast<double>(p.z)}; }

__device__ void release_masks(Ctx& ctx) {
    const DeviceCloth& d = ctx.d;
    const NumiClothConfig& cf = d.cfg[ctx.s.cfg_offset + ctx.sub];
    const uint32_t m = cf.mouthControl.x;
    if (!ctx.s.release || d.rim == nullptr || m < 3u || m > NUMI_CLOTH_MOUTH_RIM_CAPACITY) return;
    __shared__ D3 s_ring[NUMI_CLOTH_MOUTH_RIM_CAPACITY];
    __shared__ D3 s_frame[4];   // centre, normal, tangent, bitangent
    __shared__ int s_ok;
    __shared__ unsigned s_mask[2];
    for (uint32_t k = threadIdx.x; k < m; k += blockDim.x) s_ring[k] = to_d3(px(ctx, __ldg(d.rim + k)));
    __syncthreads();
    if (threadIdx.x == 0) {
        D3 center{0.0, 0.0, 0.0};
        for (uint32_t k = 0; k < m; ++k) center = center + s_ring[k];
        center = vdiv_d(center, static_cast<double>(m));
        D3 area{0.0, 0.0, 0.0};
        for (uint32_t k = 0; k < m; ++k) area = area + cross_d(s_ring[k] - center, s_ring[(k + 1u) % m] - center);
        s_ok = dot_d(area, area) < 1.0e-16 ? 0 : 1;
        if (s_ok) {
            D3 normal = normalized_d(area);
            const D3 bc = to_d3(px(ctx, cf.mouthControl.y));
            if (dot_d(normal, center - bc) < 0.0) normal = normal * -1.0;
            D3 tangent = s_ring[0] - center;
            tangent = tangent - normal * dot_d(tangent, normal);
            if (dot_d(tangent, tangent) < 1.0e-16)
                tangent = cross_d(normal, fabs(normal.z) < 0.9 ? D3{0.0, 0.0, 1.0} : D3{1.0, 0.0, 0.0});
            tangent = normalized_d(tangent);
            s_frame[0] = center;
            s_frame[1] = normal;
            s_frame[2] = tangent;
            s_frame[3] = normalized_d(cross_d(normal, tangent));
        }
        s_mask[0] = d.release[0];
        s_mask[1] = d.release[1];
    }
    __syncthreads();
    if (!s_ok) return;
    const D3 center = s_frame[0], normal = s_frame[1], tangent = s_frame[2], bitangent = s_frame[3];
    const double hysteresis = static_cast<double>(cf.mouthMaterial.x);
    for (uint32_t f = threadIdx.x; f < d.f_count; f += blockDim.x) {
        const NumiClothFruit& fr = d.fruits[f];
        const D3 p{static_cast<double>(fr.positionAndInverseMass.x), static_cast<double>(fr.positionAndInverseMass.y),
                   static_cast<double>(fr.positionAndInverseMass.z)};
        const double need = static_cast<double>(fr.previousAndRadius.w) + static_cast<double>(ctx.c.radius);
        // projection inside the rim polygon, and its squared distance to it
        const D3 rel = p - center;
        const double qx = dot_d(rel, tangent), qy = dot_d(rel, bitangent);
        bool in = false;
        double best = INFINITY;
        for (uint32_t a = 0, b = m - 1u; a < m; b = a++) {
            const D3 ra = s_ring[a] - center, rb = s_ring[b] - center;
            const double ax = dot_d(ra, tangent), ay = dot_d(ra, bitangent);
            const double bx = dot_d(rb, tangent), by = dot_d(rb, bitangent);
            const double ex = bx - ax, ey = by - ay;
            const double el = ex * ex + ey * ey;
            const double t = el > 1.0e-20 ? clamp01_d(((qx - ax) * ex + (qy - ay) * ey) / el) : 0.0;
            const double sx = qx - (ax + t * ex), sy = qy - (ay + t * ey);
            best = min_d(best, sx * sx + sy * sy);
            if ((ay > qy) != (by > qy)) {
                const double cx = ax + (bx - ax) * (qy - ay) / (by - ay);
                if (qx < cx) in = !in;
            }
        }
        const bool in_proj = in || best <= 0.0;
        const bool near_proj = in || best <= need * need;
        // distance to the rim polyline in 3D
        double rim_best = INFINITY;
        for (uint32_t a = 0; a < m; ++a) {
            const D3 st = s_ring[a];
            const D3 e = s_ring[(a + 1u) % m] - st;
            const double el = dot_d(e, e);
            const double t = el > 1.0e-20 ? clamp01_d(dot_d(p - st, e) / el) : 0.0;
            const D3 off = p - (st + e * t);
            rim_best = min_d(rim_best, dot_d(off, off));
        }
        const double out = dot_d(p - center, normal);
        const unsigned bit = 1u << f;
        bool candidate = (s_mask[0] & bit) != 0u;
        if (in_proj && out > 0.0) candidate = true;
        const double axial = out - need;
        const double rim_clear = sqrt(rim_best) - need;
        const bool cap = near_proj && axial > hysteresis;
        const bool around = candidate && !in_proj && out > 0.0 && rim_clear > hysteresis;
        if (candidate) atomicOr(&s_mask[0], bit);
        if (cap || around) atomicOr(&s_mask[1], bit);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        d.release[0] = s_mask[0];
        d.release[1] = s_mask[1];
    }
}

// Fruit frictions and orientation in the fruit CTA: pair friction on
// fruit velocities staged in shared memory (one warp walks the colours),
// then ground friction, rolling resistance and orientation per fruit; the
// pair impulses of a launch's last substep are published to global memory
// for readback.
__device__ void fruit_tail(Ctx& ctx, bool last, bool staged) {
    if (!ctx.fruit_cta) return;
    const DeviceCloth& d = ctx.d;
    const SubCfg& c = ctx.c;
    FruitShared& fs = *ctx.fs;
    // velocities and spins: staged by the fruit/yarn friction sweep, else
    // from the fruit records
    for (uint32_t f = threadIdx.x; f < d.f_count && !staged; f += blockDim.x) {
        const NumiClothFruit& fr = d.fruits[f];
        fs.v[f] = make_float4(fr.velocityAndGroundImpulse.x, fr.velocityAndGroundImpulse.y,
                              fr.velocityAndGroundImpulse.z, fr.positionAndInverseMass.w);
        fs.o[f] = make_float4(fr.angularVelocity.x, fr.angularVelocity.y, fr.angularVelocity.z,
                              fr.previousAndRadius.w);
    }
    // Colours holding at least one loaded pair (marked by the pair sweeps);
    // the friction walk visits only those, in colour order.
    __syncthreads();
    const unsigned long long loaded_colours = fs.loaded;
    if (ctx.s.frictions && loaded_colours != 0ull && threadIdx.x < 32u) {
        for (unsigned long long m = loaded_colours; m != 0ull; m &= m - 1ull) {
            const uint32_t b = static_cast<uint32_t>(__ffsll(static_cast<long long>(m)) - 1);
            const Batch bt = d.pair_batches[b];
            for (uint32_t k = bt.first + threadIdx.x; k < bt.first + bt.count; k += 32u) {
                const float4 cw = fs.contact[k];
                if (cw.w <= 0.0f) continue;
                pair_friction_smem(fs.v, fs.o, fs.ab[k] & 0xffu, fs.ab[k] >> 8, xyz(cw), cw.w, c.mu_pair);
            }
            __syncwarp();
        }
    }
    __syncthreads();
    release_masks(ctx);
    for (uint32_t f = threadIdx.x; f < d.f_count; f += blockDim.x) {
        FruitState s = load_fruit(d.fruits[f]);
        s.v = xyz(fs.v[f]);
        s.omega = xyz(fs.o[f]);
        if (ctx.s.frictions) fruit_ground_friction(s, c);
        integrate_orientation(s, c.dt);
        store_fruit(d.fruits[f], s);
    }
    if (last) {   // the host reads the impulses of a launch's last substep
        for (uint32_t k = threadIdx.x; k < d.p_count; k += blockDim.x) {
            const float4 cw = fs.contact[k];
            d.pairs[k].contact = nf4<numi_float4>(cw.x, cw.y, cw.z, cw.w);
        }
    }
    __syncthreads();
}

// One substep.  Returns false when a barrier gave up.  kEdge: the kernel
// carries the edge/edge yarn self-collision phases (a separate kernel, so
// that the kernel without them keeps its registers).  kIlp: the constraint
// colours gather NC_ILP items per thread before computing them (the batched
// engine, where a CTA holds a whole cloth and every thread several items of
// a colour; with one item per thread, as on the cooperative grid, the wider
// loops only cost registers).
template <bool kEdge, bool kIlp>
__device__ __forceinline__ bool substep(Ctx& ctx, bool last) {
    const DeviceCloth& d = ctx.d;
    const Schedule& s = ctx.s;
    const float dt2 = ctx.c.dt * ctx.c.dt;
    phase_begin(ctx);
    NC_SYNC(ctx);
    if (s.aerodynamics) {
        float4* force = d.force;
        for (uint32_t i = ctx.tid; i < d.n; i += ctx.nthreads) force[i] = make_float4(0, 0, 0, 0);
        NC_SYNC(ctx);
        for (uint32_t b = 0; b < d.n_dist_batches; ++b) {
            if (d.dist_batches[b].yarn == 0u) continue;
            air_force_batch(ctx, d.dist_batches[b], force);
            NC_SYNC(ctx);
        }
        air_reduce_chunks(ctx, force);
        NC_SYNC(ctx);
        const float att = air_attenuation(ctx);
        air_apply_advance(ctx, force, att);
        NC_SYNC(ctx);
    }
    const bool prim = kEdge && s.primitive_self && d.edge_count != nullptr;
    if (prim && !edge_sweep(ctx, true)) return false;   // swept edge/edge (tools/cloth_bag.cpp:4921)
    if (s.swept_fruit_yarn && d.f_count > 0u) {
        uint32_t first = NC_MAX_BATCHES, last = 0;
        for (uint32_t b = 0; b < d.n_dist_batches; ++b)
            if (d.dist_batches[b].yarn != 0u) {
                first = min(first, b);
                last = b;
            }
        for (uint32_t b = first; b <= last && b < d.n_dist_batches; ++b) {
            if (d.dist_batches[b].yarn == 0u) continue;
            swept_contact_batch(ctx, d.dist_batches[b], b == first, b == last);
            NC_SYNC(ctx);
        }
        ctx.fruit_pending = true;
    }
    for (uint32_t it = 0; it < s.iterations; ++it) {
        if constexpr (kIlp) {
            for (uint32_t b = 0; b < d.n_dist_batches; ++b) {
                const Batch bt = d.dist_batches[b];
                fruit_flush(ctx);
                distance_colour(ctx, bt.first, bt.count, dt2);
                NC_SYNC(ctx);
            }
        } else {
            // a colour follows while batches of this sweep remain
            const bool bends_follow = (it & 1u) == 0u && d.n_bend_batches > 0u;
            for (uint32_t b = 0; b < d.n_dist_batches; ++b) {
                const Batch bt = d.dist_batches[b];
                fruit_flush(ctx);
                for (Range r = colour_items(ctx, b, bt.count); r.i < r.end; r.i += r.stride)
                    solve_distance(ctx, bt.first + colour_item(ctx, r.i), dt2);
                NC_CSYNC(ctx, b + 1u < d.n_dist_batches || d.n_knot_batches > 0u || bends_follow);
            }
            for (uint32_t b = 0; b < d.n_knot_batches; ++b) {
                const Batch bt = d.knot_batches[b];
                for (Range r = colour_items(ctx, d.n_dist_batches + b, bt.count); r.i < r.end; r.i += r.stride)
                    solve_knot(ctx, bt.first + colour_item(ctx, r.i), dt2);
                NC_CSYNC(ctx, b + 1u < d.n_knot_batches || bends_follow);
            }
        }
        if constexpr (kIlp) {
            for (uint32_t b = 0; b < d.n_knot_batches; ++b) {
                const Batch bt = d.knot_batches[b];
                for (Range r = item_range(ctx, bt.count); r.i < r.end; r.i += r.stride)
                    solve_knot(ctx, bt.first + r.i, dt2);
                NC_SYNC(ctx);
            }
        }
        if ((it & 1u) == 0u) {
            if constexpr (kIlp) {
                for (uint32_t b = 0; b < d.n_bend_batches; ++b) {
                    const Batch bt = d.bend_batches[b];
                    bend_colour(ctx, bt.first, bt.count, dt2, ctx.c.radius, ctx.c.ground);
                    NC_SYNC(ctx);
                }
            } else {
                const uint32_t slot0 = d.n_dist_batches + d.n_knot_batches;
                for (uint32_t b = 0; b < d.n_bend_batches; ++b) {
                    const Batch bt = d.bend_batches[b];
                    for (Range r = colour_items(ctx, slot0 + b, bt.count); r.i < r.end; r.i += r.stride)
                        solve_bend(ctx, bt.first + colour_item(ctx, r.i), dt2, ctx.c.radius, ctx.c.ground);
                    NC_CSYNC(ctx, b + 1u < d.n_bend_batches);
                }
            }
        }
        // grips (CTA 0) and fruit pairs (fruit CTA) touch disjoint state
        if (ctx.grip_cta) solve_grips(ctx);
        if (ctx.fruit_cta && d.p_count > 0u) {
            __syncthreads();
            fruit_pair_sweep(d, *ctx.fs, ctx.c.dt);
        }
        NC_SYNC(ctx);
        if (!yarn_sweep(ctx)) return false;
        if (s.self_collision && d.hash_head != nullptr) {
            fruit_flush(ctx);
            self_insert(ctx, it);
            NC_SYNC(ctx);
#ifdef NC_SELF_ORDER_KERNELS
            self_solve_exact(ctx, it);   // same particle ranges as the ground clamp below
#else
            self_solve(ctx, it);   // same particle ranges as the ground clamp below
#endif
        }
        phase_ground(ctx);
        NC_SYNC(ctx);
#ifdef NC_SELF_ORDER_KERNELS
        if (s.self_collision && d.hash_head != nullptr && !self_settle(ctx, it)) return false;
#endif
    }
    // reconciliation (tools/cloth_bag.cpp:4975-5058)
    uint32_t passes = 0;
    for (uint32_t p = 0; p < s.reconcile_passes; ++p) {
        if (!contacts_pass<kIlp>(ctx, true)) return false;
        passes = p + 1u;
        if (s.early_exit) {
            residual_partials(ctx, d.red);
            NC_SYNC(ctx);
            const bool ok = residuals_converged(ctx);
            NC_SYNC(ctx);
            if (ok) break;
        }
    }
    // endpoint: present edge/edge contacts, strain, final contacts
    // (tools/cloth_bag.cpp:5059-5142)
    if (prim && !edge_sweep(ctx, false)) return false;
    if (!strain_sweeps<kIlp>(ctx)) return false;
    for (uint32_t p = 0; p < s.final_passes; ++p)
        if (!contacts_pass<kIlp>(ctx, false)) return false;
    uint32_t cert = 0;
    if (last) {
        for (uint32_t p = 0; p < s.certificate_passes; ++p) {
            if (prim && !edge_sweep(ctx, false)) return false;
            if (!strain_sweeps<kIlp>(ctx)) return false;
            for (uint32_t q = 0; q < s.final_passes; ++q)
                if (!contacts_pass<kIlp>(ctx, false)) return false;
            cert = p + 1u;
            if (prim && !edge_measure(ctx)) return false;
            residual_partials(ctx, d.red);
            NC_SYNC(ctx);
            const bool ok = residuals_converged(ctx) && (!prim || edge_measured_clear(ctx));
            NC_SYNC(ctx);
            if (ok) break;
        }
    }
    phase_finalize(ctx);
    NC_SYNC(ctx);
    if (prim && s.frictions) {
        edge_friction(ctx);   // yarn/yarn self friction (tools/cloth_bag.cpp:3995-4090)
        NC_SYNC(ctx);
    }
    const bool friction_sweep = s.frictions && d.f_count > 0u;
    if (friction_sweep) yarn_friction_sweep(ctx);   // fruit CTA, no grid barrier
    fruit_tail(ctx, last, friction_sweep);
    if (ctx.ranks > 1u && ctx.grip_cta && !last) {   // the next substep's grip attach
        Ctx next = ctx;
        next.c = nc::load_cfg(d.cfg + s.cfg_offset + ctx.sub + 1u);
        grip_attach(next);
    }
    NC_SYNC(ctx);
    if (ctx.rank == 0 && threadIdx.x == 0) {
        d.stats[1] = max(d.stats[1], passes);
        d.stats[2] = max(d.stats[2], cert);
    }
    return true;
}

// Checks of caller-built records before an allocation-free launch steps
// anything, one CTA (the reference kernels make the same checks item by
// item, ClothBag.metal:1156-1175): every particle index below the particle
// count and the two (or four) particles of an item distinct, else RANGE;
// no two items of one colour run sharing a particle (or fruit), else BATCH.
// A run claims its particles with an atomic max of its own tag, which grows
// run by run, so an item that finds its tag already there shares a particle
// with an earlier item of the same run.  Returns false (failure bits set)
// when anything is wrong; the launch then steps nothing.
__device__ bool validate_records(const DeviceCloth& d, const SubCfg& c0) {
    uint32_t* stamp = d.check_stamp;
    for (uint32_t i = threadIdx.x; i < d.n + NC_MAX_FRUITS; i += blockDim.x) stamp[i] = 0u;
    __syncthreads();
    unsigned bad = 0u;
    uint32_t tag = 0u;
    auto claim = [&](uint32_t slot) {
        if (atomicMax(stamp + slot, tag) == tag) bad |= NUMI_CLOTH_FAILURE_BATCH;
    };
    for (uint32_t b = 0; b < d.n_dist_batches; ++b) {
        const Batch bt = d.dist_batches[b];
        ++tag;
        for (uint32_t k = threadIdx.x; k < bt.count; k += blockDim.x) {
            const uint2 ij = d.d_ij[bt.first + k];
            if (ij.x >= d.n || ij.y >= d.n || ij.x == ij.y) {
                bad |= NUMI_CLOTH_FAILURE_RANGE;
                continue;
            }
            claim(ij.x);
            claim(ij.y);
        }
        __syncthreads();
    }
    for (uint32_t b = 0; b < d.n_knot_batches; ++b) {
        const Batch bt = d.knot_batches[b];
        ++tag;
        for (uint32_t k = threadIdx.x; k < bt.count; k += blockDim.x) {
            const uint4 q = d.k_ij[bt.first + k];
            if (q.x >= d.n || q.y >= d.n || q.z >= d.n || q.w >= d.n || q.x == q.y || q.x == q.z ||
                q.x == q.w || q.y == q.z || q.y == q.w || q.z == q.w) {
                bad |= NUMI_CLOTH_FAILURE_RANGE;
                continue;
            }
            claim(q.x);
            claim(q.y);
            claim(q.z);
            claim(q.w);
        }
        __syncthreads();
    }
    for (uint32_t b = 0; b < d.n_bend_batches; ++b) {
        const Batch bt = d.bend_batches[b];
        ++tag;
        for (uint32_t k = threadIdx.x; k < bt.count; k += blockDim.x) {
            const uint4 q = d.b_ij[bt.first + k];
            if (q.x >= d.n || q.y >= d.n || q.z >= d.n || q.x == q.z) {
                bad |= NUMI_CLOTH_FAILURE_RANGE;
                continue;
            }
            claim(q.x);
            claim(q.z);
        }
        __syncthreads();
    }
    for (uint32_t b = 0; b < d.n_pair_batches; ++b) {
        const Batch bt = d.pair_batches[b];
        ++tag;
        for (uint32_t k = threadIdx.x; k < bt.count; k += blockDim.x) {
            const numi_uint4 fc = d.pairs[bt.first + k].fruitsAndColor;
            if (fc.x >= d.f_count || fc.y >= d.f_count || fc.x == fc.y) {
                bad |= NUMI_CLOTH_FAILURE_RANGE;
                continue;
            }
            claim(d.n + fc.x);
            claim(d.n + fc.y);
        }
        __syncthreads();
    }
    for (uint32_t g = threadIdx.x; g < d.g_count; g += blockDim.x)
        if (d.grips[g].particle.x >= d.n) bad |= NUMI_CLOTH_FAILURE_RANGE;
    if (c0.grip_select == 1u)
        for (uint32_t k = threadIdx.x; k < 2u * c0.ring_count; k += blockDim.x)
            if (d.cuff[k] >= d.n) bad |= NUMI_CLOTH_FAILURE_RANGE;
    const int any = __syncthreads_or(bad != 0u);
    if (bad != 0u) fail(d, bad);
    return any == 0;
}

}  // namespace
}  // namespace nc

#include "cloth_bulk.cuh"
#include "cloth_tile.cuh"

// One cloth's frame on `ranks` CTAs (this one is `rank`): all substeps of
// the launch's Configs, particles optionally resident in (distributed)
// shared memory.
// The descriptor is copied into shared memory first, so both kernels run
// the phases on the same (shared-memory) view of it.
template <bool kEdge, bool kIlp>
__device__ __forceinline__ void run_frame(const DeviceCloth& src, const Schedule& s, uint32_t rank, uint32_t ranks,
                                          unsigned char* dynamic_smem) {
    {
        const uint32_t* from = reinterpret_cast<const uint32_t*>(&src);
        uint32_t* to = reinterpret_cast<uint32_t*>(dynamic_smem);
        for (uint32_t w = threadIdx.x; w < sizeof(DeviceCloth) / 4u; w += blockDim.x) to[w] = from[w];
        __syncthreads();
    }
    const DeviceCloth& d = *reinterpret_cast<const DeviceCloth*>(dynamic_smem);
    if (d.check_stamp != nullptr && s.substeps > 0u && !nc::validate_records(d, nc::load_cfg(d.cfg + s.cfg_offset)))
        return;
    FruitShared& fruit_shared = *reinterpret_cast<FruitShared*>(dynamic_smem + nc_fruit_offset());
    nc::Ctx ctx{d, s};
    ctx.gx = d.x;
    ctx.gv = d.v;
    ctx.fs = &fruit_shared;
    ctx.tid = rank * blockDim.x + threadIdx.x;
    ctx.nthreads = ranks * blockDim.x;
    ctx.fruit_cta = rank == ranks - 1u;
    ctx.grip_cta = rank == 0u;
    ctx.fruit_pending = false;
    ctx.seq = 0;
    ctx.nseq = 0;
    ctx.resident = d.resident != 0u;
    ctx.rank = rank;
    ctx.ranks = ranks;
    ctx.shift = d.resident_shift;
    uint32_t own_first = 0, own_end = 0;
    if (ctx.resident) {
        // Stage this CTA's particles into shared memory for the whole launch
        // (bulk copies of its slices of x and v).
        ctx.xs = reinterpret_cast<float4*>(dynamic_smem + nc_resident_offset());
        ctx.vs = ctx.xs + (1u << ctx.shift);
        own_first = min(ctx.rank << ctx.shift, d.n);
        own_end = min(own_first + (1u << ctx.shift), d.n);
        const uint32_t bytes = (own_end - own_first) * static_cast<uint32_t>(sizeof(float4));
        const nc::BulkJob jobs[2] = {{ctx.xs, d.x + own_first, bytes}, {ctx.vs, d.v + own_first, bytes}};
        const bool staged = nc::bulk_load(d, jobs, 2u);
        // a cluster's CTAs all pass its barrier; a copy that timed out has
        // raised TIMEOUT and the abort flag for the host
        if (ranks > 1u)
            cooperative_groups::this_cluster().sync();
        else if (!staged)
            return;
    }
    if (s.tiles) {
        // tile mode: the CTA's plan and its local particles after the
        // descriptor (the fruit CTA keeps its fruit state there instead)
        uint32_t* plan = reinterpret_cast<uint32_t*>(dynamic_smem + nc_fruit_offset());
        ctx.tp = plan;
        if (ctx.fruit_cta) ctx.fst = reinterpret_cast<FrictionStage*>(dynamic_smem + nc_resident_offset());
        if (!ctx.fruit_cta) {
            if (!nc::tile_stage(ctx, plan)) return;
            ctx.tx = reinterpret_cast<float4*>(
                dynamic_smem + nc_fruit_offset() + 4u * (d.tile_off[rank + 1u] - d.tile_off[rank]));
            ctx.tile_box = nc::tile_closure_box(ctx);
        }
    } else {
        nc::neighbour_stage(ctx);
    }
    if (ctx.fruit_cta) {
        for (uint32_t k = threadIdx.x; k < d.p_count; k += blockDim.x)
            fruit_shared.ab[k] =
                static_cast<unsigned short>(d.pairs[k].fruitsAndColor.x | (d.pairs[k].fruitsAndColor.y << 8));
        __syncthreads();
    }
    const uint32_t epoch_base = s.epoch_ptr != nullptr ? *s.epoch_ptr : d.epoch_base;
    if (ranks > 1u && s.substeps > 0u) {
        // the first substep's grip attach, before any CTA predicts (later
        // substeps attach at the end of the one before)
        ctx.sub = 0;
        ctx.c = nc::load_cfg(d.cfg + s.cfg_offset);
        ctx.barriers = 0;
        if (ctx.grip_cta) nc::grip_attach(ctx);
        if (!nc::grid_sync(ctx)) return;
    }
    for (uint32_t sub = 0; sub < s.substeps; ++sub) {
        ctx.sub = sub;
        ctx.c = nc::load_cfg(d.cfg + s.cfg_offset + sub);
        ctx.epoch = epoch_base + sub;
        ctx.barriers = 0;
        if (d.tape != nullptr && ranks == 1u) {
            // adjoint tape: state at the start of the substep
            float4* slot = d.tape + static_cast<size_t>(sub) * d.tape_slots * d.n;
            for (uint32_t i = threadIdx.x; i < d.n; i += blockDim.x) {
                slot[i] = px(ctx, i);
                d.tape_v[static_cast<size_t>(sub) * d.n + i] = pv(ctx, i);
            }
            __syncthreads();
        }
        if constexpr (!kEdge && !kIlp) {
            if (s.tiles) {
                if (!nc::substep_tiles(ctx, sub + 1u == s.substeps)) return;
                if (rank == 0 && threadIdx.x == 0) d.stats[0] = ctx.barriers;
                continue;
            }
        }
        if (!nc::substep<kEdge, kIlp>(ctx, sub + 1u == s.substeps)) return;
        if (rank == 0 && threadIdx.x == 0) d.stats[0] = ctx.barriers;
    }
    if (ctx.gx != d.x || ctx.gv != d.v) {
        // tile mode ended on the alternate buffers: copy them back (every
        // store of the launch ended at its last barrier)
        for (nc::Range r = nc::particle_range(ctx); r.i < r.end; r.i += r.stride) {
            if (ctx.gx != d.x) d.x[r.i] = __ldcg(ctx.gx + r.i);
            if (ctx.gv != d.v) d.v[r.i] = __ldcg(ctx.gv + r.i);
        }
    }
    if (ctx.resident) {
        // Every remote access ended at the last barrier: write the CTA's own
        // particles back (bulk copies).
        const uint32_t bytes = (own_end - own_first) * static_cast<uint32_t>(sizeof(float4));
        const nc::BulkJob jobs[2] = {{ctx.xs, d.x + own_first, bytes}, {ctx.vs, d.v + own_first, bytes}};
        nc::bulk_store(jobs, 2u);
    }
}

// The frame and batch kernels with the edge/edge yarn self-collision phases
// are defined in cloth_edge_kernels.cu, a translation unit of their own: with
// them in the same unit the compiler inlines the shared phases differently
// and the default kernels grow a call frame.
__global__ void numi_cloth_frame_edge_kernel(DeviceCloth d, Schedule s);
__global__ void numi_cloth_batch_edge_kernel(const DeviceCloth* cloths, uint32_t count, Schedule s,
                                             unsigned int* queue);
// The frame kernels whose point self contact keeps the reference's
// Gauss-Seidel order are likewise in cloth_self_order_kernels.cu: its
// out-of-line ordered pass would otherwise cost the default kernels
// registers in every phase.
__global__ void numi_cloth_frame_exact_kernel(DeviceCloth d, Schedule s);
__global__ void numi_cloth_frame_edge_exact_kernel(DeviceCloth d, Schedule s);

// Many independent cloths in one persistent launch: every CTA takes the
// next cloth from a device work queue (cloths ordered by work, largest
// first) and runs its whole frame alone, until the queue is empty.
#define NC_BATCH_BODY(kEdge)                                                  \
    extern __shared__ __align__(16) unsigned char nc_dynamic_smem[];          \
    __shared__ uint32_t s_next;                                               \
    for (;;) {                                                                \
        if (threadIdx.x == 0) s_next = atomicAdd(queue, 1u);                  \
        __syncthreads();                                                      \
        const uint32_t k = s_next;                                            \
        if (k >= count) break;                                                \
        run_frame<kEdge, true>(cloths[k], s, 0u, 1u, nc_dynamic_smem);        \
        __syncthreads();                                                      \
    }

#ifndef NC_EDGE_KERNELS
// One cloth on the whole grid (one CTA, a cooperative grid or a cluster).
__global__ void __launch_bounds__(NC_BLOCK_MAX, 1) numi_cloth_frame_kernel(DeviceCloth d, Schedule s) {
    extern __shared__ __align__(16) unsigned char nc_dynamic_smem[];
    run_frame<false, false>(d, s, blockIdx.x, gridDim.x, nc_dynamic_smem);
}
__global__ void __launch_bounds__(NC_BLOCK_MAX, 1) numi_cloth_batch_kernel(const DeviceCloth* cloths, uint32_t count,
                                                                         Schedule s, unsigned int* queue) {
    NC_BATCH_BODY(false)
}

// Advance the batch substep counter after a batch launch.
__global__ void numi_cloth_epoch_kernel(uint32_t* epoch, uint32_t substeps) { *epoch += substeps; }
#endif
