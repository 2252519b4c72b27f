// Edge/edge yarn self-collision and yarn/yarn self friction.
//
// The reference resolves every non-local pair of yarn segments closer than
// the yarn diameter one pair after another (solvePrimitiveSelfCollision,
// tools/cloth_bag.cpp:3880-3993): segment by segment, each segment's
// candidates from a box tree, once swept (conservative advancement from the
// substep start) before the constraint iterations and once present at every
// endpoint.  A pair's solve reads and writes only its four particles, so two
// solves commute unless they share a particle, and the solve of a pair whose
// segments stay farther apart than the yarn diameter does nothing.  The
// kernels keep the reference's Gauss-Seidel order exactly:
//   1. a pair list holds every non-local segment pair whose spheres came
//      within a skin of each other when it was built; it is rebuilt (through
//      a hashed grid of segment spheres) only when some position has moved a
//      sixth of the skin since, so it always holds every pair whose
//      pass-start spheres (edgeCollisionSphere) overlap;
//   2. every listed pair whose pass-start spheres overlap (the reference's
//      sphere filter) becomes a candidate with a lower bound on every
//      distance its solve could see: the pass-start distance (present pass)
//      or half the start and end distances less the endpoints' motion (swept
//      pass).  Candidates whose bound is within a margin of contact are
//      "ordered";
//   3. one thread resolves the ordered pairs in the reference's order (first
//      segment ascending, then the second) with the reference's own tests:
//      the pass-start box of the second segment against the current box of
//      the first, then the solve.  Each particle's path length is recorded;
//   4. every other candidate is checked: its bound less the path lengths of
//      its segments' particles must still clear contact, which proves its
//      solve would have changed nothing.  A candidate that fails joins the
//      ordered pairs and the pass is redone from the pass-start positions.
// The one departure from the reference order: the candidates of a segment
// are taken in ascending index order, not in the box tree's leaf order.
#pragma once

namespace nc {
namespace {   // internal linkage: the edge kernels' unit includes these too

// Margin of the ordered set (fraction of the yarn diameter) and the most
// redo rounds of one pass.
#define NC_EDGE_MARGIN 0.125f
#define NC_EDGE_ROUNDS 64u
// Skin of the pair list, in yarn diameters.
#define NC_EDGE_SKIN 1.0f

__device__ __forceinline__ float clamp01f(float v) {
    const float a = v < 0.0f ? 0.0f : v;
    return 1.0f < a ? 1.0f : a;
}

// closestPointsOnSegments (tools/cloth_bag.cpp:2751-2824): cp = p0 + (p1 -
// p0) s and cq = q0 + (q1 - q0) t.
__device__ __forceinline__ void segment_closest(V3 p0, V3 p1, V3 q0, V3 q1, V3& cp, V3& cq, float& s, float& t) {
    const V3 d1 = p1 - p0, d2 = q1 - q0, off = p0 - q0;
    const float l1 = lsq(d1), l2 = lsq(d2), sp = dot3(d2, off);
    const float eps = 1.0e-20f;
    s = 0.0f;
    t = 0.0f;
    if (l1 <= eps && l2 <= eps) {
        cp = p0;
        cq = q0;
        return;
    }
    if (l1 <= eps) {
        t = clamp01f(sp / l2);
    } else {
        const float fp = dot3(d1, off);
        if (l2 <= eps) {
            s = clamp01f(-fp / l1);
        } else {
            const float c = dot3(d1, d2);
            const float den = l1 * l2 - c * c;
            if (den > eps) s = clamp01f((c * sp - fp * l2) / den);
            t = (c * s + sp) / l2;
            if (t < 0.0f) {
                t = 0.0f;
                s = clamp01f(-fp / l1);
            } else if (t > 1.0f) {
                t = 1.0f;
                s = clamp01f((c - fp) / l1);
            }
        }
    }
    cp = p0 + d1 * s;
    cq = q0 + d2 * t;
}

__device__ __forceinline__ float segment_distance(V3 p0, V3 p1, V3 q0, V3 q1) {
    V3 cp, cq;
    float s, t;
    segment_closest(p0, p1, q0, q1, cp, cq, s, t);
    return len3(cq - cp);
}

// selfContactNormal (tools/cloth_bag.cpp:3400-3414).
__device__ __forceinline__ V3 edge_normal(V3 sep, V3 fa, V3 fb, V3 prev_off) {
    const float L = len3(sep);
    if (L > 1.0e-12f) return vdiv(sep, L);
    V3 nrm = normalized3(cross3(fa, fb));
    if (dot3(prev_off, nrm) > 0.0f) nrm = nrm * -1.0f;
    return nrm;
}

struct EdgeBox {
    V3 lo, hi;
};

// edgeBounds (tools/cloth_bag.cpp:3675-3691): the segment, with its
// substep-start copy when swept, grown by the expansion.
__device__ __forceinline__ EdgeBox edge_box(V3 a, V3 b, V3 ap, V3 bp, bool swept, float ex) {
    EdgeBox r;
    r.lo = V3{fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z)};
    r.hi = V3{fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)};
    if (swept) {
        r.lo = V3{fminf(r.lo.x, fminf(ap.x, bp.x)), fminf(r.lo.y, fminf(ap.y, bp.y)), fminf(r.lo.z, fminf(ap.z, bp.z))};
        r.hi = V3{fmaxf(r.hi.x, fmaxf(ap.x, bp.x)), fmaxf(r.hi.y, fmaxf(ap.y, bp.y)), fmaxf(r.hi.z, fmaxf(ap.z, bp.z))};
    }
    r.lo = r.lo - V3{ex, ex, ex};
    r.hi = r.hi + V3{ex, ex, ex};
    return r;
}

// overlapBounds (tools/cloth_bag.cpp:3758-3768).
__device__ __forceinline__ bool boxes_overlap(const EdgeBox& a, const EdgeBox& b) {
    return a.lo.x <= b.hi.x && a.hi.x >= b.lo.x && a.lo.y <= b.hi.y && a.hi.y >= b.lo.y && a.lo.z <= b.hi.z &&
           a.hi.z >= b.lo.z;
}

// edgeCollisionSphere (tools/cloth_bag.cpp:3697-3720): centre and radius
// (grown by the expansion) of the segment's points, with the substep-start
// points when swept.
__device__ __forceinline__ float4 edge_sphere(V3 a, V3 b, V3 ap, V3 bp, bool swept, float ex) {
    V3 c = V3{0.0f, 0.0f, 0.0f} + a;
    c = c + b;
    if (swept) {
        c = c + ap;
        c = c + bp;
    }
    c = vdiv(c, swept ? 4.0f : 2.0f);
    float r = 0.0f;
    r = fmaxf(r, len3(a - c));
    r = fmaxf(r, len3(b - c));
    if (swept) {
        r = fmaxf(r, len3(ap - c));
        r = fmaxf(r, len3(bp - c));
    }
    return make_float4(c.x, c.y, c.z, r + ex);
}

// overlapSpheres (tools/cloth_bag.cpp:3722-3728).
__device__ __forceinline__ bool spheres_overlap(float4 a, float4 b) {
    const float r = a.w + b.w;
    return lsq(xyz(a) - xyz(b)) <= r * r;
}

// edgePairLocal (tools/cloth_bag.cpp:2740-2749).
__device__ __forceinline__ bool edge_local(const DeviceCloth& d, uint2 a, uint2 b) {
    return local_pair(d, a.x, b.x) || local_pair(d, a.x, b.y) || local_pair(d, a.y, b.x) || local_pair(d, a.y, b.y);
}

// Pass tag of the segment grid: 23 bits of the substep counter and the
// pass within the substep (the host clears the heads when they wrap).
__device__ __forceinline__ uint32_t edge_tag(const Ctx& ctx) { return ((ctx.epoch & 0x7fffffu) << 9) | (ctx.edge_pass & 511u); }

__device__ __forceinline__ unsigned long long edge_key(uint32_t i, uint32_t j) {
    return (static_cast<unsigned long long>(i) << 32) | j;
}

// The impulse of one solve into a zeroed record (tools/cloth_bag.cpp:3545-3557).
__device__ __forceinline__ void edge_impulse(EdgeRecord& rec, V3 nrm, const float fw[2], const float sw[2], float lam,
                                             float dt) {
    const float imp = lam / dt;
    rec.wn[0] = rec.wn[0] - nrm.x * imp;
    rec.wn[1] = rec.wn[1] - nrm.y * imp;
    rec.wn[2] = rec.wn[2] - nrm.z * imp;
    for (int e = 0; e < 2; ++e) {
        rec.wf[e] = rec.wf[e] + fw[e] * imp;
        rec.ws[e] = rec.ws[e] + sw[e] * imp;
    }
    rec.ni = rec.ni + imp;
}

// Positions of the four particles of a pair, read and written through the
// launch's particle view.
struct EdgeQuad {
    uint32_t id[4];
    float4 x[4];   // current (xyz, inverse mass)
    V3 p[4];       // substep start
};

// solveSweptEdgeEdge (tools/cloth_bag.cpp:3452-3567).  Returns true when it
// moved the particles (and filled rec).
__device__ bool edge_swept(EdgeQuad& q, float radius, float dt, EdgeRecord& rec) {
    const float target = 2.0f * radius;
    const float tol = 1.0e-9f;
    float bound = 0.0f;
    for (int e = 0; e < 4; ++e) bound = bound + len3(xyz(q.x[e]) - q.p[e]);
    if (bound < 1.0e-14f) return false;
    V3 P[4], cp, cq;
    float s = 0.0f, t = 0.0f, dist = 0.0f;
    auto sample = [&](float time) {
        for (int e = 0; e < 4; ++e) P[e] = q.p[e] + (xyz(q.x[e]) - q.p[e]) * time;
        segment_closest(P[0], P[1], P[2], P[3], cp, cq, s, t);
        dist = len3(cq - cp);
    };
    float time = 0.0f;
    sample(0.0f);
    bool found = dist <= target + tol;
    if (!found) {
        for (uint32_t k = 0; k < 80u; ++k) {
            sample(time);
            const float gap = dist - target;
            if (gap <= tol) {
                found = true;
                break;
            }
            const float adv = 0.9f * gap / bound;
            if (!isfinite(adv) || adv <= 0.0f || time + adv >= 1.0f) break;
            time = time + (adv < 1.0e-10f ? 1.0e-10f : adv);
        }
    }
    if (!found) return false;
    const float fw[2] = {1.0f - s, s}, sw[2] = {1.0f - t, t};
    const V3 fprev = q.p[0] * fw[0] + q.p[1] * fw[1];
    const V3 sprev = q.p[2] * sw[0] + q.p[3] * sw[1];
    const V3 nrm = edge_normal(cq - cp, P[1] - P[0], P[3] - P[2], fprev - sprev);
    V3 frem{0.0f, 0.0f, 0.0f}, srem{0.0f, 0.0f, 0.0f};
    for (int e = 0; e < 2; ++e) {
        frem = frem + (xyz(q.x[e]) - P[e]) * fw[e];
        srem = srem + (xyz(q.x[e + 2]) - P[e + 2]) * sw[e];
    }
    const float removed = dot3(frem - srem, nrm);
    if (removed <= 0.0f) return false;
    float den = 0.0f;
    for (int e = 0; e < 2; ++e) {
        den = den + q.x[e].w * fw[e] * fw[e];
        den = den + q.x[e + 2].w * sw[e] * sw[e];
    }
    if (den <= 0.0f) return false;
    const float lam = removed / den;
    for (int e = 0; e < 2; ++e) {
        q.x[e] = with_xyz(q.x[e], xyz(q.x[e]) - nrm * (q.x[e].w * fw[e] * lam));
        q.x[e + 2] = with_xyz(q.x[e + 2], xyz(q.x[e + 2]) + nrm * (q.x[e + 2].w * sw[e] * lam));
    }
    edge_impulse(rec, nrm, fw, sw, lam, dt);
    return true;
}

// solveEdgeEdge (tools/cloth_bag.cpp:3569-3640).
__device__ bool edge_present(EdgeQuad& q, float radius, float dt, EdgeRecord& rec) {
    const float target = 2.0f * radius;
    V3 cp, cq;
    float s, t;
    segment_closest(xyz(q.x[0]), xyz(q.x[1]), xyz(q.x[2]), xyz(q.x[3]), cp, cq, s, t);
    const V3 sep = cq - cp;
    const float dist = len3(sep);
    if (dist >= target) return false;
    const float fw[2] = {1.0f - s, s}, sw[2] = {1.0f - t, t};
    const V3 fprev = q.p[0] * fw[0] + q.p[1] * fw[1];
    const V3 sprev = q.p[2] * sw[0] + q.p[3] * sw[1];
    const V3 nrm = edge_normal(sep, xyz(q.x[1]) - xyz(q.x[0]), xyz(q.x[3]) - xyz(q.x[2]), fprev - sprev);
    float den = 0.0f;
    for (int e = 0; e < 2; ++e) {
        den = den + q.x[e].w * fw[e] * fw[e];
        den = den + q.x[e + 2].w * sw[e] * sw[e];
    }
    if (den <= 0.0f) return false;
    const float lam = (target - dist) / den;
    for (int e = 0; e < 2; ++e) {
        q.x[e] = with_xyz(q.x[e], xyz(q.x[e]) - nrm * (q.x[e].w * fw[e] * lam));
        q.x[e + 2] = with_xyz(q.x[e + 2], xyz(q.x[e + 2]) + nrm * (q.x[e + 2].w * sw[e] * lam));
    }
    edge_impulse(rec, nrm, fw, sw, lam, dt);
    return true;
}

// Cover sphere of a segment for the pair list: centred on the segment's
// midpoint, large enough to hold both its present and its swept sphere,
// plus half the skin.
__device__ __forceinline__ float4 edge_cover(V3 a, V3 b, V3 ap, V3 bp, float ex, float skin) {
    const float4 ps = edge_sphere(a, b, ap, bp, false, ex);
    const float4 ss = edge_sphere(a, b, ap, bp, true, ex);
    const float r = fmaxf(ps.w, len3(xyz(ss) - xyz(ps)) + ss.w) + 0.5f * skin;
    return make_float4(ps.x, ps.y, ps.z, r);
}

__device__ __forceinline__ float edge_skin(const Ctx& ctx) { return NC_EDGE_SKIN * (2.0f * ctx.c.radius); }

// Phase 1: snapshot the pass-start positions, clear the path lengths, write
// every segment's pass sphere and this CTA's largest displacement (of x and
// of the substep-start positions) since the pair list was built.
__device__ void edge_begin(Ctx& ctx, bool swept) {
    const DeviceCloth& d = ctx.d;
    const float ex = 0.5f * (2.0f * ctx.c.radius);
    float moved = 0.0f;
    for (Range r = particle_range(ctx); r.i < r.end; r.i += r.stride) {
        const float4 p = px(ctx, r.i);
        d.edge_x0[r.i] = p;
        d.edge_path[r.i] = 0.0f;
        const V3 dx = xyz(p) - xyz(ld(d.edge_xb + r.i));
        const V3 dp = xyz(ld(d.xp + r.i)) - xyz(ld(d.edge_pb + r.i));
        moved = fmaxf(moved, fmaxf(len3(dx), len3(dp)));
        if (!(len3(dx) == len3(dx))) moved = INFINITY;   // NaN: rebuild, and the bound checks fail later
    }
    for (Range r = item_range(ctx, d.y_count); r.i < r.end; r.i += r.stride) {
        const uint2 ab = __ldg(d.y_ij + r.i);
        d.edge_sph[r.i] = edge_sphere(xyz(px(ctx, ab.x)), xyz(px(ctx, ab.y)), xyz(ld(d.xp + ab.x)),
                                      xyz(ld(d.xp + ab.y)), swept, ex);
    }
    double (*s_r)[NC_BLOCK_MAX] = nc_red_smem;
    s_r[0][threadIdx.x] = static_cast<double>(moved);
    __syncthreads();
    for (uint32_t st = blockDim.x / 2u; st > 0u; st >>= 1u) {
        if (threadIdx.x < st) s_r[0][threadIdx.x] = fmax(s_r[0][threadIdx.x], s_r[0][threadIdx.x + st]);
        __syncthreads();
    }
    if (threadIdx.x == 0) d.edge_red[ctx.ranks + ctx.rank] = s_r[0][0];
    __syncthreads();
    if (ctx.rank == 0 && threadIdx.x == 0) {
        d.edge_ctl[0] = 0u;   // candidates
        d.edge_ctl[1] = 0u;   // ordered pairs
        d.edge_ctl[4] = 0u;   // records of the pass
        if (swept) d.edge_ctl[3] = 0u;   // records of the substep
    }
}

// The pair list holds every non-local pair whose present or swept spheres
// were within the skin of each other when it was built.  A sphere's centre
// moves at most as far as its points and its radius changes at most twice
// that, so while every position moved less than a sixth of the skin since
// the build, every pair whose spheres overlap now is on the list.
__device__ bool edge_list_valid(const Ctx& ctx) {
    const DeviceCloth& d = ctx.d;
    if (__ldcg(d.edge_ctl + 6) == 0u || __ldcg(d.edge_built_radius) != ctx.c.radius) return false;
    double moved = 0.0;
    for (uint32_t r = 0; r < ctx.ranks; ++r) moved = fmax(moved, __ldcg(d.edge_red + ctx.ranks + r));
    return 6.0 * moved + 1.0e-6 < static_cast<double>(edge_skin(ctx));
}

// Rebuild, step 1: put every segment's cover sphere into the grid (or the
// list) and remember the positions of the build.
__device__ void edge_build_insert(Ctx& ctx) {
    const DeviceCloth& d = ctx.d;
    const float ex = 0.5f * (2.0f * ctx.c.radius);
    const float skin = edge_skin(ctx);
    const float inv_cell = 1.0f / d.edge_cell;
    const float grid_radius = 0.25f * d.edge_cell;
    const unsigned long long tag = edge_tag(ctx);
    for (Range r = particle_range(ctx); r.i < r.end; r.i += r.stride) {
        d.edge_xb[r.i] = ld(d.edge_x0 + r.i);
        d.edge_pb[r.i] = ld(d.xp + r.i);
    }
    for (Range r = item_range(ctx, d.y_count); r.i < r.end; r.i += r.stride) {
        const uint32_t k = r.i;
        const uint2 ab = __ldg(d.y_ij + k);
        const float4 sph = edge_cover(xyz(ld(d.edge_x0 + ab.x)), xyz(ld(d.edge_x0 + ab.y)), xyz(ld(d.xp + ab.x)),
                                      xyz(ld(d.xp + ab.y)), ex, skin);
        bool listed = !(sph.w <= grid_radius);
        HashSlot* e = nullptr;
        if (!listed) {
            const uint32_t bucket = cell_bucket(static_cast<int>(floorf(sph.x * inv_cell)),
                                                static_cast<int>(floorf(sph.y * inv_cell)),
                                                static_cast<int>(floorf(sph.z * inv_cell)), d.edge_mask);
            unsigned long long* head = d.edge_head + bucket;
            atomicMax(head, tag << 32);
            const uint32_t slot = static_cast<uint32_t>(atomicAdd(head, 1ull));
            if (slot < NC_HASH_CAP)
                e = d.edge_slot + bucket * NC_HASH_CAP + slot;
            else
                listed = true;
        }
        if (listed) {
            atomicMax(d.edge_list_head, tag << 32);
            const uint32_t o = static_cast<uint32_t>(atomicAdd(d.edge_list_head, 1ull));
            if (o >= d.y_count) {   // cannot happen: at most one entry per segment
                fail(d, NUMI_CLOTH_FAILURE_RANGE);
                continue;
            }
            e = d.edge_list + o;
        }
        e->pos = sph;
        e->meta = make_uint4(k, 0u, 0u, 0u);
        d.edge_flag[k] = listed ? 1u : 0u;
    }
    if (ctx.rank == 0 && threadIdx.x == 0) {
        d.edge_ctl[5] = 0u;   // pairs on the list
        *d.edge_built_radius = ctx.c.radius;
    }
}

// Rebuild, step 2: every pair of overlapping cover spheres (a < b) once.
// Grid segments query the 2 x 2 x 2 cells on their centre's side (a cell
// is at least twice the largest distance between the centres of two
// overlapping grid spheres) and scan the list; list segments scan only the
// list.  A pair of grid segments is met by its lower index, a grid/list
// pair by the grid segment, a pair of list segments by its lower index.
__device__ void edge_build_pairs(Ctx& ctx) {
    const DeviceCloth& d = ctx.d;
    const float ex = 0.5f * (2.0f * ctx.c.radius);
    const float skin = edge_skin(ctx);
    const float inv_cell = 1.0f / d.edge_cell;
    const uint32_t tag = edge_tag(ctx);
    const unsigned long long lh = __ldcg(d.edge_list_head);
    const uint32_t listed_count = static_cast<uint32_t>(lh >> 32) == tag ? min(static_cast<uint32_t>(lh), d.y_count) : 0u;
    // the exact test of the build: present or swept spheres within the skin
    auto keep = [&](uint32_t a, uint32_t b) {
        const uint2 sa = __ldg(d.y_ij + a), sb = __ldg(d.y_ij + b);
        if (edge_local(d, sa, sb)) return;
        const V3 xa0 = xyz(ld(d.edge_x0 + sa.x)), xa1 = xyz(ld(d.edge_x0 + sa.y));
        const V3 xb0 = xyz(ld(d.edge_x0 + sb.x)), xb1 = xyz(ld(d.edge_x0 + sb.y));
        const V3 pa0 = xyz(ld(d.xp + sa.x)), pa1 = xyz(ld(d.xp + sa.y));
        const V3 pb0 = xyz(ld(d.xp + sb.x)), pb1 = xyz(ld(d.xp + sb.y));
        bool near = false;
        for (int v = 0; v < 2 && !near; ++v) {
            const float4 s1 = edge_sphere(xa0, xa1, pa0, pa1, v == 1, ex);
            const float4 s2 = edge_sphere(xb0, xb1, pb0, pb1, v == 1, ex);
            const float r = s1.w + s2.w + skin;
            near = lsq(xyz(s1) - xyz(s2)) <= r * r;
        }
        if (!near) return;
        const uint32_t k = atomicAdd(d.edge_ctl + 5, 1u);
        if (k >= d.edge_list_cap) {
            fail(d, NUMI_CLOTH_FAILURE_RANGE);
            return;
        }
        d.edge_pairs[k] = make_uint2(a, b);
    };
    for (Range r = item_range(ctx, d.y_count); r.i < r.end; r.i += r.stride) {
        const uint32_t i = r.i;
        const uint2 ai = __ldg(d.y_ij + i);
        const float4 si = edge_cover(xyz(ld(d.edge_x0 + ai.x)), xyz(ld(d.edge_x0 + ai.y)), xyz(ld(d.xp + ai.x)),
                                     xyz(ld(d.xp + ai.y)), ex, skin);
        const bool listed = __ldcg(d.edge_flag + i) != 0u;
        if (!listed) {
            int base[3], step[3];
            float gap2[3];
            const float coord[3] = {si.x * inv_cell, si.y * inv_cell, si.z * inv_cell};
            for (int k = 0; k < 3; ++k) {
                const float c0 = floorf(coord[k]);
                const float frac = coord[k] - c0;
                base[k] = static_cast<int>(c0);
                step[k] = frac < 0.5f ? -1 : 1;
                const float gap = frac < 0.5f ? frac : 1.0f - frac;
                gap2[k] = gap * gap;
            }
            // neighbour cells farther than this sphere's reach (its radius
            // plus the largest grid radius, a quarter cell) hold no partner;
            // the margin covers the rounding of the cell coordinates
            const float reach = si.w * inv_cell + 0.25f + 1.0e-3f +
                                2.4e-7f * fmaxf(fabsf(coord[0]), fmaxf(fabsf(coord[1]), fabsf(coord[2])));
            const float reach2 = reach * reach;
            uint32_t bk[8];
            bool near[8];
            for (uint32_t q = 0; q < 8u; ++q) {
                bk[q] = cell_bucket(base[0] + ((q & 1u) ? step[0] : 0), base[1] + ((q & 2u) ? step[1] : 0),
                                    base[2] + ((q & 4u) ? step[2] : 0), d.edge_mask);
                const float g2 =
                    ((q & 1u) ? gap2[0] : 0.0f) + ((q & 2u) ? gap2[1] : 0.0f) + ((q & 4u) ? gap2[2] : 0.0f);
                bool repeat = false;
                for (uint32_t e = 0; e < q; ++e) repeat = repeat || (near[e] && bk[e] == bk[q]);
                near[q] = (q == 0u || g2 < reach2) && !repeat;
            }
            for (uint32_t q = 0; q < 8u; ++q) {
                if (!near[q]) continue;
                const unsigned long long hd = __ldcg(d.edge_head + bk[q]);
                if (static_cast<uint32_t>(hd >> 32) != tag) continue;
                const uint32_t cnt = min(static_cast<uint32_t>(hd), NC_HASH_CAP);
                for (uint32_t k = 0; k < cnt; ++k) {
                    const HashSlot* e = d.edge_slot + bk[q] * NC_HASH_CAP + k;
                    const uint32_t j = __ldcg(&e->meta.x);
                    if (j <= i || !spheres_overlap(si, __ldcg(&e->pos))) continue;
                    keep(i, j);
                }
            }
        }
        for (uint32_t o = 0; o < listed_count; ++o) {
            const uint32_t j = __ldcg(&d.edge_list[o].meta.x);
            if (j == i || (listed && j < i)) continue;
            if (!spheres_overlap(si, __ldcg(&d.edge_list[o].pos))) continue;
            if (j > i)
                keep(i, j);
            else
                keep(j, i);
        }
    }
}

// Phases 1 and the rebuild when it is due.  Returns false when a barrier
// gave up.
__device__ __forceinline__ bool edge_prepare(Ctx& ctx, bool swept) {
    edge_begin(ctx, swept);
    NC_SYNC(ctx);
    if (!edge_list_valid(ctx)) {
        edge_build_insert(ctx);
        NC_SYNC(ctx);
        edge_build_pairs(ctx);
        NC_SYNC(ctx);
        if (ctx.rank == 0 && threadIdx.x == 0) ctx.d.edge_ctl[6] = 1u;   // the list is built
    }
    return true;
}

// Phase 2: the pairs of the list whose pass spheres overlap (the
// reference's sphere filter) are the candidates, each with a lower bound
// (less the rounding slack) on every distance its solve could see; those
// within the margin of contact are ordered.
__device__ void edge_candidates(Ctx& ctx, bool swept) {
    const DeviceCloth& d = ctx.d;
    const float target = 2.0f * ctx.c.radius;
    const float thr = (swept ? target + 1.0e-9f : target) + NC_EDGE_MARGIN * target;
    const uint32_t listed = min(__ldcg(d.edge_ctl + 5), d.edge_list_cap);
    for (Range r = item_range(ctx, listed); r.i < r.end; r.i += r.stride) {
        const uint2 ab = __ldcg(d.edge_pairs + r.i);
        const uint32_t a = ab.x, b = ab.y;
        if (!spheres_overlap(ld(d.edge_sph + a), ld(d.edge_sph + b))) continue;
        const uint2 sa = __ldg(d.y_ij + a), sb = __ldg(d.y_ij + b);
        const V3 x0[4] = {xyz(ld(d.edge_x0 + sa.x)), xyz(ld(d.edge_x0 + sa.y)), xyz(ld(d.edge_x0 + sb.x)),
                          xyz(ld(d.edge_x0 + sb.y))};
        float bound;
        float big = 0.0f;
        for (int e = 0; e < 4; ++e) big = fmaxf(big, fmaxf(fabsf(x0[e].x), fmaxf(fabsf(x0[e].y), fabsf(x0[e].z))));
        if (swept) {
            const V3 p[4] = {xyz(ld(d.xp + sa.x)), xyz(ld(d.xp + sa.y)), xyz(ld(d.xp + sb.x)), xyz(ld(d.xp + sb.y))};
            for (int e = 0; e < 4; ++e) big = fmaxf(big, fmaxf(fabsf(p[e].x), fmaxf(fabsf(p[e].y), fabsf(p[e].z))));
            const float d_start = segment_distance(p[0], p[1], p[2], p[3]);
            const float d_end = segment_distance(x0[0], x0[1], x0[2], x0[3]);
            const float motion = fmaxf(len3(x0[0] - p[0]), len3(x0[1] - p[1])) +
                                 fmaxf(len3(x0[2] - p[2]), len3(x0[3] - p[3]));
            bound = 0.5f * (d_start + d_end - motion);
        } else {
            bound = segment_distance(x0[0], x0[1], x0[2], x0[3]);
        }
        // rounding of the distances, the paths and the solve's own distance
        bound = bound - (1.0e-6f + 1.0e-6f * big);
        const uint32_t k = atomicAdd(d.edge_ctl + 0, 1u);
        if (k >= d.edge_cap) {
            fail(d, NUMI_CLOTH_FAILURE_RANGE);
            continue;
        }
        const bool ordered = !(bound >= thr);
        d.edge_cand[k] = make_uint4(a, b, __float_as_uint(bound), ordered ? 1u : 0u);
        if (ordered) d.edge_order[atomicAdd(d.edge_ctl + 1, 1u)] = edge_key(a, b);
    }
}

// Phase 3 (CTA 0): sort the ordered pairs, undo the previous round, then
// resolve them one after another on thread 0.
__device__ void edge_resolve(Ctx& ctx, bool swept, bool redo) {
    if (ctx.rank != 0) return;
    const DeviceCloth& d = ctx.d;
    const uint32_t count = min(__ldcg(d.edge_ctl + 1), d.edge_cap);
    // rank sort: the keys are distinct
    for (uint32_t k = threadIdx.x; k < count; k += blockDim.x) {
        const unsigned long long key = __ldcg(d.edge_order + k);
        uint32_t rank = 0;
        for (uint32_t m = 0; m < count; ++m) rank += __ldcg(d.edge_order + m) < key ? 1u : 0u;
        d.edge_sorted[rank] = key;
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    const float ex = 0.5f * (2.0f * ctx.c.radius);
    if (redo) {
        // back to the pass-start positions of every particle the last round moved
        const uint32_t done = d.edge_ctl[4];
        for (uint32_t r = 0; r < done; ++r) {
            const uint2 sa = __ldg(d.y_ij + d.edge_new[r].i), sb = __ldg(d.y_ij + d.edge_new[r].j);
            const uint32_t id[4] = {sa.x, sa.y, sb.x, sb.y};
            for (int e = 0; e < 4; ++e) {
                px_set(ctx, id[e], ld(d.edge_x0 + id[e]));
                d.edge_path[id[e]] = 0.0f;
            }
        }
        d.edge_ctl[4] = 0u;
    }
    uint32_t done = 0;
    uint32_t first = 0xffffffffu;
    EdgeBox qi{};
    for (uint32_t k = 0; k < count; ++k) {
        const unsigned long long key = d.edge_sorted[k];
        const uint32_t i = static_cast<uint32_t>(key >> 32), j = static_cast<uint32_t>(key);
        const uint2 sa = __ldg(d.y_ij + i), sb = __ldg(d.y_ij + j);
        EdgeQuad q;
        q.id[0] = sa.x;
        q.id[1] = sa.y;
        q.id[2] = sb.x;
        q.id[3] = sb.y;
        for (int e = 0; e < 4; ++e) {
            q.x[e] = px(ctx, q.id[e]);
            q.p[e] = xyz(ld(d.xp + q.id[e]));
        }
        // the reference's tree query: the first segment's box when its turn
        // comes (before any of its own pairs), against the second segment's
        // pass-start box
        if (i != first) {
            first = i;
            qi = edge_box(xyz(q.x[0]), xyz(q.x[1]), q.p[0], q.p[1], swept, ex);
        }
        const EdgeBox bj = edge_box(xyz(ld(d.edge_x0 + sb.x)), xyz(ld(d.edge_x0 + sb.y)), q.p[2], q.p[3], swept, ex);
        if (!boxes_overlap(bj, qi)) continue;
        EdgeRecord rec{};
        rec.i = i;
        rec.j = j;
        const bool moved = swept ? edge_swept(q, ctx.c.radius, ctx.c.dt, rec) : edge_present(q, ctx.c.radius, ctx.c.dt, rec);
        if (!moved) continue;
        for (int e = 0; e < 4; ++e) {
            const float4 before = px(ctx, q.id[e]);
            d.edge_path[q.id[e]] = d.edge_path[q.id[e]] + len3(xyz(q.x[e]) - xyz(before));
            px_set(ctx, q.id[e], q.x[e]);
        }
        if (done < d.edge_cap) d.edge_new[done++] = rec;
    }
    d.edge_ctl[4] = done;
}

// Phase 4: every candidate outside the ordered set must have stayed clear
// of contact; one that may not joins the ordered set.
__device__ void edge_verify(Ctx& ctx, bool swept) {
    const DeviceCloth& d = ctx.d;
    const float target = 2.0f * ctx.c.radius;
    const float thr = swept ? target + 1.0e-9f : target;
    const uint32_t count = min(__ldcg(d.edge_ctl + 0), d.edge_cap);
    for (Range r = item_range(ctx, count); r.i < r.end; r.i += r.stride) {
        const uint4 c = __ldcg(d.edge_cand + r.i);
        if (c.w != 0u) continue;
        const uint2 sa = __ldg(d.y_ij + c.x), sb = __ldg(d.y_ij + c.y);
        const float pa = fmaxf(__ldcg(d.edge_path + sa.x), __ldcg(d.edge_path + sa.y));
        const float pb = fmaxf(__ldcg(d.edge_path + sb.x), __ldcg(d.edge_path + sb.y));
        if (pa == 0.0f && pb == 0.0f) continue;   // no particle of the pair moved
        if (__uint_as_float(c.z) - (pa + pb) >= thr) continue;
        d.edge_cand[r.i].w = 1u;
        d.edge_order[atomicAdd(d.edge_ctl + 1, 1u)] = edge_key(c.x, c.y);
        atomicAdd(d.edge_ctl + 2, 1u);
    }
}

// Merge the pass's records (ascending keys) into the substep's records
// (ascending keys), adding the sums of a pair met before
// (tools/cloth_bag.cpp:3962-3985).  Thread 0 of CTA 0.
__device__ void edge_commit(const Ctx& ctx) {
    if (ctx.rank != 0 || threadIdx.x != 0) return;
    const DeviceCloth& d = ctx.d;
    const uint32_t fresh = d.edge_ctl[4];
    uint32_t have = d.edge_ctl[3];
    auto key = [](const EdgeRecord& r) { return edge_key(r.i, r.j); };
    uint32_t inserts = 0;
    for (uint32_t k = 0, r = 0; k < fresh; ++k) {
        const EdgeRecord& n = d.edge_new[k];
        while (r < have && key(d.edge_rec[r]) < key(n)) ++r;
        if (r < have && key(d.edge_rec[r]) == key(n)) {
            EdgeRecord& o = d.edge_rec[r];
            for (int e = 0; e < 3; ++e) o.wn[e] = o.wn[e] + n.wn[e];
            for (int e = 0; e < 2; ++e) {
                o.wf[e] = o.wf[e] + n.wf[e];
                o.ws[e] = o.ws[e] + n.ws[e];
            }
            o.ni = o.ni + n.ni;
        } else {
            ++inserts;
        }
    }
    if (have + inserts > d.edge_cap) {
        fail(d, NUMI_CLOTH_FAILURE_RANGE);
        inserts = 0;
    }
    // new keys, merged in from the back
    int w = static_cast<int>(have + inserts) - 1, p = static_cast<int>(have) - 1;
    for (int k = static_cast<int>(fresh) - 1; k >= 0 && inserts > 0u; --k) {
        const EdgeRecord& n = d.edge_new[k];
        while (p >= 0 && key(d.edge_rec[p]) > key(n)) d.edge_rec[w--] = d.edge_rec[p--];
        if (p >= 0 && key(d.edge_rec[p]) == key(n)) continue;
        EdgeRecord o{};
        o.i = n.i;
        o.j = n.j;
        for (int e = 0; e < 3; ++e) o.wn[e] = 0.0f + n.wn[e];
        for (int e = 0; e < 2; ++e) {
            o.wf[e] = 0.0f + n.wf[e];
            o.ws[e] = 0.0f + n.ws[e];
        }
        o.ni = 0.0f + n.ni;
        d.edge_rec[w--] = o;
    }
    d.edge_ctl[3] = have + inserts;
    d.edge_stats[0] += fresh;
}

// One edge/edge pass (swept or present).  Returns false when a barrier
// gave up.
__device__ __forceinline__ bool edge_sweep(Ctx& ctx, bool swept) {
    const DeviceCloth& d = ctx.d;
    if (!edge_prepare(ctx, swept)) return false;
    edge_candidates(ctx, swept);
    NC_SYNC(ctx);
    uint32_t seen = __ldcg(d.edge_ctl + 2);
    for (uint32_t round = 0;; ++round) {
        edge_resolve(ctx, swept, round > 0u);
        NC_SYNC(ctx);
        edge_verify(ctx, swept);
        NC_SYNC(ctx);
        const uint32_t now = __ldcg(d.edge_ctl + 2);
        if (now == seen) break;
        seen = now;
        if (round + 1u >= NC_EDGE_ROUNDS) {
            fail(d, NUMI_CLOTH_FAILURE_RANGE);
            break;
        }
    }
    edge_commit(ctx);
    ++ctx.edge_pass;
    return true;
}

// The deepest non-local pair of the current positions
// (measurePrimitiveSelfPenetration, tools/cloth_bag.cpp:4182-4247): every
// pair closer than the yarn diameter passes the reference's box and sphere
// filters (and is on the pair list), so the maximum over the listed pairs
// whose present spheres overlap (and 0) is the reference's value.  Writes
// this CTA's maximum to edge_red[rank].
__device__ void edge_deepest(Ctx& ctx) {
    const DeviceCloth& d = ctx.d;
    const float target = 2.0f * ctx.c.radius;
    float pen = 0.0f;
    const uint32_t listed = min(__ldcg(d.edge_ctl + 5), d.edge_list_cap);
    for (Range r = item_range(ctx, listed); r.i < r.end; r.i += r.stride) {
        const uint2 ab = __ldcg(d.edge_pairs + r.i);
        if (!spheres_overlap(ld(d.edge_sph + ab.x), ld(d.edge_sph + ab.y))) continue;
        const uint2 sa = __ldg(d.y_ij + ab.x), sb = __ldg(d.y_ij + ab.y);
        const float depth = target - segment_distance(xyz(ld(d.edge_x0 + sa.x)), xyz(ld(d.edge_x0 + sa.y)),
                                                      xyz(ld(d.edge_x0 + sb.x)), xyz(ld(d.edge_x0 + sb.y)));
        pen = pen < depth ? depth : pen;
    }
    double (*s_r)[NC_BLOCK_MAX] = nc_red_smem;
    s_r[0][threadIdx.x] = static_cast<double>(pen);
    __syncthreads();
    for (uint32_t st = blockDim.x / 2u; st > 0u; st >>= 1u) {
        if (threadIdx.x < st) s_r[0][threadIdx.x] = fmax(s_r[0][threadIdx.x], s_r[0][threadIdx.x + st]);
        __syncthreads();
    }
    if (threadIdx.x == 0) d.edge_red[ctx.rank] = s_r[0][0];
    __syncthreads();
}

// Certificate measure: pass spheres (and the list, when due), then the
// deepest pair.
__device__ __forceinline__ bool edge_measure(Ctx& ctx) {
    if (!edge_prepare(ctx, false)) return false;
    edge_deepest(ctx);
    ++ctx.edge_pass;
    return true;
}

__device__ __forceinline__ bool edge_measured_clear(const Ctx& ctx) {
    double m = 0.0;
    for (uint32_t r = 0; r < ctx.ranks; ++r) m = fmax(m, __ldcg(ctx.d.edge_red + r));
    return static_cast<float>(m) < 1.0e-6f;
}

// applyClothSelfFriction (tools/cloth_bag.cpp:3995-4090): Coulomb friction
// on every record in key order, thread 0 of CTA 0.
__device__ __forceinline__ void edge_friction(const Ctx& ctx) {
    if (ctx.rank != 0 || threadIdx.x != 0) return;
    const DeviceCloth& d = ctx.d;
    const float mu = ctx.c.mu_self;
    const uint32_t count = d.edge_ctl[3];
    unsigned long long applied = 0;
    for (uint32_t k = 0; k < count; ++k) {
        const EdgeRecord r = d.edge_rec[k];
        const V3 wn{r.wn[0], r.wn[1], r.wn[2]};
        if (r.ni <= 0.0f || lsq(wn) < 1.0e-20f) continue;
        const V3 nrm = normalized3(wn);
        float fw[2], sw[2];
        float fsum = 0.0f, ssum = 0.0f;
        for (int e = 0; e < 2; ++e) {
            fw[e] = r.wf[e] / r.ni;
            sw[e] = r.ws[e] / r.ni;
            fsum = fsum + fw[e];
            ssum = ssum + sw[e];
        }
        if (fsum <= 1.0e-12f || ssum <= 1.0e-12f) continue;
        const uint2 sa = __ldg(d.y_ij + r.i), sb = __ldg(d.y_ij + r.j);
        const uint32_t fi[2] = {sa.x, sa.y}, si[2] = {sb.x, sb.y};
        float4 fvv[2], svv[2];
        float fwm[2], swm[2];
        V3 fv{0.0f, 0.0f, 0.0f}, sv{0.0f, 0.0f, 0.0f};
        for (int e = 0; e < 2; ++e) {
            fw[e] = fw[e] / fsum;
            sw[e] = sw[e] / ssum;
            fvv[e] = pv(ctx, fi[e]);
            svv[e] = pv(ctx, si[e]);
            fwm[e] = px(ctx, fi[e]).w;
            swm[e] = px(ctx, si[e]).w;
            fv = fv + xyz(fvv[e]) * fw[e];
            sv = sv + xyz(svv[e]) * sw[e];
        }
        const V3 rel = fv - sv;
        const V3 tv = rel - nrm * dot3(rel, nrm);
        const float slip = len3(tv);
        if (slip < 1.0e-10f) continue;
        const V3 tn = vdiv(tv, slip);
        float den = 0.0f;
        for (int e = 0; e < 2; ++e) {
            den = den + fwm[e] * fw[e] * fw[e];
            den = den + swm[e] * sw[e] * sw[e];
        }
        if (den <= 0.0f) continue;
        const float limit = mu * r.ni;
        const float a = slip / den;
        const float imp = limit < a ? limit : a;
        if (imp <= 0.0f) continue;
        const V3 on_first = tn * (-imp);
        // the two segments share no particle (the pair is not local), but a
        // segment's own endpoints are read back after each write
        for (int e = 0; e < 2; ++e) {
            const float4 v1 = pv(ctx, fi[e]);
            pv_set(ctx, fi[e], with_xyz(v1, xyz(v1) + on_first * (fwm[e] * fw[e])));
            const float4 v2 = pv(ctx, si[e]);
            pv_set(ctx, si[e], with_xyz(v2, xyz(v2) - on_first * (swm[e] * sw[e])));
        }
        ++applied;
    }
    d.edge_stats[1] += applied;
}

}  // namespace
}  // namespace nc
