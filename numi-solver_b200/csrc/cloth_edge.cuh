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
#define NC_EDGE_SKIN 2.0f

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

// Segments a < b local to each other (edgePairLocal,
// tools/cloth_bag.cpp:2740-2749: any endpoint pair is local): b on a's list
// of local segments of higher index (ascending), built on the host.
__device__ __forceinline__ bool seg_local(const DeviceCloth& d, uint32_t a, uint32_t b) {
    uint32_t lo = __ldg(d.edge_loc_off + a), hi = __ldg(d.edge_loc_off + a + 1u);
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        const uint32_t v = __ldg(d.edge_loc_idx + mid);
        if (v == b) return true;
        if (v < b) lo = mid + 1u;
        else hi = mid;
    }
    return false;
}

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

// A slot of an append counter: one atomic add for the lanes of a warp that
// append together, each lane getting the next slot in lane order.
__device__ __forceinline__ uint32_t warp_append(uint32_t* counter) {
    const unsigned m = __activemask();
    const uint32_t lane = threadIdx.x & 31u;
    const int leader = __ffs(m) - 1;
    uint32_t base = 0;
    if (lane == static_cast<uint32_t>(leader)) base = atomicAdd(counter, static_cast<uint32_t>(__popc(m)));
    base = __shfl_sync(m, base, leader);
    return base + static_cast<uint32_t>(__popc(m & ((1u << lane) - 1u)));
}

__device__ __forceinline__ float edge_skin(const Ctx& ctx) { return NC_EDGE_SKIN * (2.0f * ctx.c.radius); }

// Phase 1: snapshot the pass-start positions, clear the path lengths, write
// every segment's pass sphere, and this CTA's largest displacement since the
// pair list was built (of x and of the substep-start positions) and largest
// motion over the substep so far (x - substep start).
__device__ void edge_begin(Ctx& ctx, bool swept) {
    const DeviceCloth& d = ctx.d;
    const float ex = 0.5f * (2.0f * ctx.c.radius);
    float moved = 0.0f, motion = 0.0f;
    for (Range r = particle_range(ctx); r.i < r.end; r.i += r.stride) {
        const float4 p = px(ctx, r.i);
        const V3 prev = xyz(ld(d.xp + r.i));
        d.edge_x0[r.i] = p;
        d.edge_path[r.i] = 0.0f;
        const float dx = len3(xyz(p) - xyz(ld(d.edge_xb + r.i)));
        const float dp = len3(prev - xyz(ld(d.edge_pb + r.i)));
        const float dm = len3(xyz(p) - prev);
        moved = fmaxf(moved, fmaxf(dx, dp));
        motion = fmaxf(motion, dm);
        if (!(dx == dx && dp == dp && dm == dm)) moved = INFINITY;   // NaN: rebuild; the bound checks fail later
    }
    for (Range r = item_range(ctx, d.y_count); r.i < r.end; r.i += r.stride) {
        const uint2 ab = __ldg(d.y_ij + r.i);
        d.edge_sph[r.i] = edge_sphere(xyz(px(ctx, ab.x)), xyz(px(ctx, ab.y)), xyz(ld(d.xp + ab.x)),
                                      xyz(ld(d.xp + ab.y)), swept, ex);
    }
    double (*s_r)[NC_BLOCK_MAX] = nc_red_smem;
    s_r[0][threadIdx.x] = static_cast<double>(moved);
    s_r[1][threadIdx.x] = static_cast<double>(motion);
    __syncthreads();
    for (uint32_t st = blockDim.x / 2u; st > 0u; st >>= 1u) {
        if (threadIdx.x < st) {
            s_r[0][threadIdx.x] = fmax(s_r[0][threadIdx.x], s_r[0][threadIdx.x + st]);
            s_r[1][threadIdx.x] = fmax(s_r[1][threadIdx.x], s_r[1][threadIdx.x + st]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        d.edge_red[ctx.ranks + ctx.rank] = s_r[0][0];
        d.edge_red[2u * ctx.ranks + ctx.rank] = s_r[1][0];
    }
    __syncthreads();
    if (ctx.rank == 0 && threadIdx.x == 0) {
        d.edge_ctl[0] = 0u;   // candidates
        d.edge_ctl[1] = 0u;   // ordered pairs
        d.edge_ctl[4] = 0u;   // records of the pass
        d.edge_ctl[7] = 0u;   // segments too long for the build grid
        if (swept) d.edge_ctl[3] = 0u;   // records of the substep
    }
}

// The pair list holds every non-local pair whose segments were within the
// yarn diameter plus the skin of each other at the build, at the build's
// positions or at its substep-start positions.  Every position has moved at
// most D since (D: the larger of the two displacements), and every endpoint
// at most M over the substep so far, so an unlisted pair is at least
// diameter + skin - 2D apart now, and its swept bound (half the start and end
// distances less the motion) is at least diameter + skin - 2D - M.  While
// 2D + M + the ordering margin stays below the skin, no unlisted pair can be
// a candidate, and no pair closer than the diameter is unlisted.
__device__ bool edge_list_valid(const Ctx& ctx) {
    const DeviceCloth& d = ctx.d;
    if (__ldcg(d.edge_ctl + 6) == 0u || __ldcg(d.edge_built_radius) != ctx.c.radius) return false;
    double moved = 0.0, motion = 0.0;
    for (uint32_t r = 0; r < ctx.ranks; ++r) {
        moved = fmax(moved, __ldcg(d.edge_red + ctx.ranks + r));
        motion = fmax(motion, __ldcg(d.edge_red + 2u * ctx.ranks + r));
    }
    const double target = 2.0 * static_cast<double>(ctx.c.radius);
    return 2.0 * moved + motion + NC_EDGE_MARGIN * target + 1.0e-6 < static_cast<double>(edge_skin(ctx));
}

// Build-grid cells of a segment: its current and substep-start endpoints'
// box grown by half of (diameter + skin), so that two segments within
// diameter + skin of each other share a cell.  A span of 0 marks a segment
// the grid does not hold (more than 27 cells, or not finite).
struct EdgeCells {
    int lo[3];
    int span[3];
};
__device__ __forceinline__ EdgeCells edge_cells(V3 a, V3 b, V3 ap, V3 bp, float h, float inv_cell) {
    const float lo[3] = {fminf(fminf(a.x, b.x), fminf(ap.x, bp.x)) - h, fminf(fminf(a.y, b.y), fminf(ap.y, bp.y)) - h,
                         fminf(fminf(a.z, b.z), fminf(ap.z, bp.z)) - h};
    const float hi[3] = {fmaxf(fmaxf(a.x, b.x), fmaxf(ap.x, bp.x)) + h, fmaxf(fmaxf(a.y, b.y), fmaxf(ap.y, bp.y)) + h,
                         fmaxf(fmaxf(a.z, b.z), fmaxf(ap.z, bp.z)) + h};
    EdgeCells c;
    bool ok = true;
    for (int k = 0; k < 3; ++k) {
        const float l = floorf(lo[k] * inv_cell), u = floorf(hi[k] * inv_cell);
        ok = ok && l >= -1048576.0f && u <= 1048575.0f && u - l <= 2.0f;   // finite, biased key, at most 3 cells
        c.lo[k] = ok ? static_cast<int>(l) : 0;
        c.span[k] = ok ? static_cast<int>(u - l) + 1 : 0;
    }
    if (!ok)
        for (int k = 0; k < 3; ++k) c.span[k] = 0;
    return c;
}

// Exclusive-scan chunk of the buckets handled by this CTA.
__device__ __forceinline__ uint32_t edge_chunk(const Ctx& ctx) {
    const uint32_t buckets = ctx.d.edge_mask + 1u;
    return (buckets + ctx.ranks - 1u) / ctx.ranks;
}

// Rebuild, step 1: remember the build's positions and count every
// segment's cells into its bucket (cells hash as the point grid's); a
// segment the grid does not hold goes to the long-segment list.
__device__ void edge_build_count(Ctx& ctx) {
    const DeviceCloth& d = ctx.d;
    const float h = 0.5f * (2.0f * ctx.c.radius + edge_skin(ctx));
    const float inv_cell = 1.0f / d.edge_cell;
    for (Range r = particle_range(ctx); r.i < r.end; r.i += r.stride) {
        d.edge_xb[r.i] = ld(d.edge_x0 + r.i);
        d.edge_pb[r.i] = ld(d.xp + r.i);
    }
    for (Range r = item_range(ctx, d.y_count); r.i < r.end; r.i += r.stride) {
        const uint2 ab = __ldg(d.y_ij + r.i);
        const V3 a = xyz(ld(d.edge_x0 + ab.x)), b = xyz(ld(d.edge_x0 + ab.y)), ap = xyz(ld(d.xp + ab.x)),
                 bp = xyz(ld(d.xp + ab.y));
        // the grown box, for the pair search's first test
        d.edge_bbox[2u * r.i] = make_float4(fminf(fminf(a.x, b.x), fminf(ap.x, bp.x)) - h,
                                            fminf(fminf(a.y, b.y), fminf(ap.y, bp.y)) - h,
                                            fminf(fminf(a.z, b.z), fminf(ap.z, bp.z)) - h, 0.0f);
        d.edge_bbox[2u * r.i + 1u] = make_float4(fmaxf(fmaxf(a.x, b.x), fmaxf(ap.x, bp.x)) + h,
                                                 fmaxf(fmaxf(a.y, b.y), fmaxf(ap.y, bp.y)) + h,
                                                 fmaxf(fmaxf(a.z, b.z), fmaxf(ap.z, bp.z)) + h, 0.0f);
        const EdgeCells c = edge_cells(a, b, ap, bp, h, inv_cell);
        if (c.span[0] == 0) {
            d.edge_giant[atomicAdd(d.edge_ctl + 7, 1u)] = r.i;
            continue;
        }
        for (int z = 0; z < c.span[2]; ++z)
            for (int y = 0; y < c.span[1]; ++y)
                for (int x = 0; x < c.span[0]; ++x)
                    atomicAdd(d.edge_count + cell_bucket(c.lo[0] + x, c.lo[1] + y, c.lo[2] + z, d.edge_mask), 1u);
    }
    if (ctx.rank == 0 && threadIdx.x == 0) {
        d.edge_ctl[5] = 0u;   // pairs on the list
        *d.edge_built_radius = ctx.c.radius;
    }
}

// Rebuild, step 2: exclusive scan of the bucket counts.  Each CTA scans its
// chunk of buckets into edge_offs (chunk-local) and publishes the chunk's
// total; the counts are zeroed to serve as fill cursors.
__device__ void edge_build_scan(Ctx& ctx) {
    const DeviceCloth& d = ctx.d;
    __shared__ uint32_t s_part[NC_BLOCK_MAX];
    const uint32_t buckets = d.edge_mask + 1u;
    const uint32_t chunk = edge_chunk(ctx);
    const uint32_t first = min(ctx.rank * chunk, buckets), end = min(first + chunk, buckets);
    const uint32_t per = (end - first + blockDim.x - 1u) / blockDim.x;
    const uint32_t lo = min(first + threadIdx.x * per, end), hi = min(lo + per, end);
    uint32_t sum = 0;
    for (uint32_t b = lo; b < hi; ++b) sum += __ldcg(d.edge_count + b);
    s_part[threadIdx.x] = sum;
    __syncthreads();
    if (threadIdx.x == 0) {   // the CTA's thread totals, in order
        uint32_t run = 0;
        for (uint32_t t = 0; t < blockDim.x; ++t) {
            const uint32_t v = s_part[t];
            s_part[t] = run;
            run += v;
        }
        d.edge_chunk_total[ctx.rank] = run;
    }
    __syncthreads();
    uint32_t run = s_part[threadIdx.x];
    for (uint32_t b = lo; b < hi; ++b) {
        const uint32_t v = __ldcg(d.edge_count + b);
        d.edge_offs[b] = run;
        d.edge_count[b] = 0u;
        run += v;
    }
}

// The start of every CTA's chunk: exclusive prefix of the chunk totals.
__device__ __forceinline__ void edge_chunk_starts(const Ctx& ctx, uint32_t* s_start) {
    if (threadIdx.x == 0) {
        uint32_t run = 0;
        for (uint32_t r = 0; r < ctx.ranks; ++r) {
            s_start[r] = run;
            run += __ldcg(ctx.d.edge_chunk_total + r);
        }
    }
    __syncthreads();
}

// Rebuild, step 3: every segment's cells into the sorted entry array; an
// entry is the segment's grown box (its cells follow from the box) with
// the segment index in the lower corner's w.
__device__ void edge_build_scatter(Ctx& ctx, uint32_t* s_start) {
    const DeviceCloth& d = ctx.d;
    const float h = 0.5f * (2.0f * ctx.c.radius + edge_skin(ctx));
    const float inv_cell = 1.0f / d.edge_cell;
    const uint32_t chunk = edge_chunk(ctx);
    edge_chunk_starts(ctx, s_start);
    for (Range r = item_range(ctx, d.y_count); r.i < r.end; r.i += r.stride) {
        const uint2 ab = __ldg(d.y_ij + r.i);
        const EdgeCells c = edge_cells(xyz(ld(d.edge_x0 + ab.x)), xyz(ld(d.edge_x0 + ab.y)), xyz(ld(d.xp + ab.x)),
                                       xyz(ld(d.xp + ab.y)), h, inv_cell);
        if (c.span[0] == 0) continue;
        float4 lo = __ldcg(d.edge_bbox + 2u * r.i);
        const float4 hi = __ldcg(d.edge_bbox + 2u * r.i + 1u);
        lo.w = __uint_as_float(r.i);
        for (int z = 0; z < c.span[2]; ++z)
            for (int y = 0; y < c.span[1]; ++y)
                for (int x = 0; x < c.span[0]; ++x) {
                    const uint32_t b = cell_bucket(c.lo[0] + x, c.lo[1] + y, c.lo[2] + z, d.edge_mask);
                    const uint32_t at = s_start[b / chunk] + __ldcg(d.edge_offs + b) + atomicAdd(d.edge_count + b, 1u);
                    d.edge_entries[2u * at] = lo;
                    d.edge_entries[2u * at + 1u] = hi;
                }
    }
}

// Rebuild, step 4: the pairs, one warp per segment.  The warp visits the
// segment's cells and its lanes take the cell's entries side by side; an
// entry of a later segment is a pair when the visited cell lies in that
// segment's range and is the lowest cell of the two ranges' overlap, so
// that every pair is met once.  Long segments: every held segment scans
// their list, and they pair among themselves by index.  A pair is listed
// when it is not local (the segment's local list, held in the warp's
// registers) and its segments are within diameter + skin at the build's
// positions or at its substep-start positions.
__device__ void edge_build_pairs(Ctx& ctx, const uint32_t* s_start) {
    const DeviceCloth& d = ctx.d;
    const float target = 2.0f * ctx.c.radius;
    const float reach = target + edge_skin(ctx);
    const float h = 0.5f * reach;
    const float inv_cell = 1.0f / d.edge_cell;
    const uint32_t chunk = edge_chunk(ctx);
    const uint32_t giants = min(__ldcg(d.edge_ctl + 7), d.y_count);
    const uint32_t lane = threadIdx.x & 31u;
    // the positions and entries are not written in this phase: the reads
    // may go through L1 after a grid barrier (a gpu-scope acquire), not
    // after the cluster barrier (cluster scope)
    const bool l1 = d.cluster_barrier == 0u;
    auto rd = [l1](const float4* p) { return l1 ? __ldca(p) : __ldcg(p); };
    auto rdu = [l1](const uint32_t* p) { return l1 ? __ldca(p) : __ldcg(p); };
    auto keep_far = [&](uint32_t a, uint32_t b) {   // a non-local pair: the distance test
        const uint2 sa = __ldg(d.y_ij + a), sb = __ldg(d.y_ij + b);
        const bool near = segment_distance(xyz(rd(d.edge_x0 + sa.x)), xyz(rd(d.edge_x0 + sa.y)),
                                           xyz(rd(d.edge_x0 + sb.x)), xyz(rd(d.edge_x0 + sb.y))) <= reach ||
                          segment_distance(xyz(rd(d.xp + sa.x)), xyz(rd(d.xp + sa.y)), xyz(rd(d.xp + sb.x)),
                                           xyz(rd(d.xp + sb.y))) <= reach;
        if (!near) return;
        const uint32_t k = warp_append(d.edge_ctl + 5);
        if (k >= d.edge_list_cap) {
            fail(d, NUMI_CLOTH_FAILURE_RANGE);
            return;
        }
        d.edge_pairs[k] = make_uint2(a, b);
    };
    // Non-local candidates queue up per warp (in the reduction scratch) and
    // take the distance test 32 at a time, one per lane, instead of one or
    // two lanes at a time as they turn up.
    static_assert(2u * NC_BLOCK_MAX * sizeof(uint2) <= sizeof(nc_red_smem), "pair queues exceed the scratch");
    uint2* queue = reinterpret_cast<uint2*>(&nc_red_smem[0][0]) + 64u * (threadIdx.x >> 5);
    uint32_t queued = 0;   // warp-uniform
    auto flush = [&]() {
        __syncwarp();
        for (uint32_t k = lane; k < queued; k += 32u) {
            const uint2 pr = queue[k];
            keep_far(pr.x, pr.y);
        }
        __syncwarp();
        queued = 0;
    };
    // warps over the segments, as item_range spreads threads
    const uint32_t warps = blockDim.x >> 5;
    uint32_t i, end, stride;
    if (ctx.resident) {
        i = static_cast<uint32_t>(static_cast<unsigned long long>(d.y_count) * ctx.rank / ctx.ranks) +
            (threadIdx.x >> 5);
        end = static_cast<uint32_t>(static_cast<unsigned long long>(d.y_count) * (ctx.rank + 1u) / ctx.ranks);
        stride = warps;
    } else {
        i = ctx.tid >> 5;
        end = d.y_count;
        stride = ctx.nthreads >> 5;
    }
    for (; i < end; i += stride) {   // warp-uniform from here on
        const uint2 ab = __ldg(d.y_ij + i);
        const EdgeCells c = edge_cells(xyz(ld(d.edge_x0 + ab.x)), xyz(ld(d.edge_x0 + ab.y)), xyz(ld(d.xp + ab.x)),
                                       xyz(ld(d.xp + ab.y)), h, inv_cell);
        const float4 blo = rd(d.edge_bbox + 2u * i), bhi = rd(d.edge_bbox + 2u * i + 1u);
        // the segment's local list: up to 64 entries in two registers per lane
        const uint32_t llo = __ldg(d.edge_loc_off + i), llen = __ldg(d.edge_loc_off + i + 1u) - llo;
        const uint32_t la = lane < llen ? __ldg(d.edge_loc_idx + llo + lane) : 0xffffffffu;
        const uint32_t lb = lane + 32u < llen ? __ldg(d.edge_loc_idx + llo + 32u + lane) : 0xffffffffu;
        if (c.span[0] != 0) {
            // the segment's cells, one per lane: bucket range and cell
            const uint32_t cells = static_cast<uint32_t>(c.span[0] * c.span[1] * c.span[2]);
            uint32_t my_start = 0, my_stop = 0;
            if (lane < cells) {
                const int x = static_cast<int>(lane) % c.span[0], y = (static_cast<int>(lane) / c.span[0]) % c.span[1],
                          z = static_cast<int>(lane) / (c.span[0] * c.span[1]);
                const uint32_t b = cell_bucket(c.lo[0] + x, c.lo[1] + y, c.lo[2] + z, d.edge_mask);
                my_start = s_start[b / chunk] + rdu(d.edge_offs + b);
                my_stop = my_start + rdu(d.edge_count + b);
            }
            for (uint32_t t = 0; t < cells; ++t) {
                const int cx = c.lo[0] + static_cast<int>(t) % c.span[0];
                const int cy = c.lo[1] + (static_cast<int>(t) / c.span[0]) % c.span[1];
                const int cz = c.lo[2] + static_cast<int>(t) / (c.span[0] * c.span[1]);
                const uint32_t start = __shfl_sync(0xffffffffu, my_start, t);
                const uint32_t stop = __shfl_sync(0xffffffffu, my_stop, t);
                for (uint32_t base = start; base < stop; base += 32u) {
                    const uint32_t e = base + lane;
                    bool cand = e < stop;
                    uint32_t j = 0;
                    if (cand) {
                        const float4 olo = rd(d.edge_entries + 2u * e), ohi = rd(d.edge_entries + 2u * e + 1u);
                        j = __float_as_uint(olo.w);
                        // the other segment's cells, as edge_cells finds them from the same box
                        const int jx = static_cast<int>(floorf(olo.x * inv_cell)),
                                  jy = static_cast<int>(floorf(olo.y * inv_cell)),
                                  jz = static_cast<int>(floorf(olo.z * inv_cell));
                        const int ux = static_cast<int>(floorf(ohi.x * inv_cell)),
                                  uy = static_cast<int>(floorf(ohi.y * inv_cell)),
                                  uz = static_cast<int>(floorf(ohi.z * inv_cell));
                        // a later segment; the visited cell in its range and the lowest
                        // common cell; the grown boxes meet (not farther apart than
                        // diameter + skin)
                        cand = j > i && cx >= jx && cx <= ux && cy >= jy && cy <= uy && cz >= jz && cz <= uz &&
                               cx == max(c.lo[0], jx) && cy == max(c.lo[1], jy) && cz == max(c.lo[2], jz) &&
                               !(olo.x > bhi.x || ohi.x < blo.x || olo.y > bhi.y || ohi.y < blo.y || olo.z > bhi.z ||
                                 ohi.z < blo.z);
                    }
                    if (!__any_sync(0xffffffffu, cand)) continue;
                    bool local = false;
                    if (llen > 64u) {
                        local = cand && seg_local(d, i, j);
                    } else {
                        for (uint32_t q = 0; q < min(llen, 32u); ++q) local |= __shfl_sync(0xffffffffu, la, q) == j;
                        for (uint32_t q = 32u; q < llen; ++q) local |= __shfl_sync(0xffffffffu, lb, q - 32u) == j;
                    }
                    const bool push = cand && !local;
                    const unsigned m = __ballot_sync(0xffffffffu, push);
                    if (push) queue[queued + __popc(m & ((1u << lane) - 1u))] = make_uint2(i, j);
                    queued += static_cast<uint32_t>(__popc(m));
                    if (queued >= 32u) flush();
                }
            }
        }
        for (uint32_t g = lane; g < giants; g += 32u) {
            const uint32_t j = __ldcg(d.edge_giant + g);
            if (j == i || (c.span[0] == 0 && j < i)) continue;
            if (!seg_local(d, min(i, j), max(i, j))) keep_far(min(i, j), max(i, j));
        }
    }
    flush();
}

// Phase 1 and, when due, the rebuild of the pair list.  Returns false
// when a barrier gave up; rebuilt tells the candidates phase to clear the
// build counts.
__device__ __forceinline__ bool edge_prepare(Ctx& ctx, bool swept, bool& rebuilt) {
    __shared__ uint32_t s_start[1024];
    edge_begin(ctx, swept);
    NC_SYNC(ctx);
    rebuilt = !edge_list_valid(ctx);
    if (rebuilt) {
        if (ctx.ranks > 1024u) {   // the chunk starts live in shared memory
            fail(ctx.d, NUMI_CLOTH_FAILURE_RANGE);
            rebuilt = false;
            return true;
        }
        edge_build_count(ctx);
        NC_SYNC(ctx);
        edge_build_scan(ctx);
        NC_SYNC(ctx);
        edge_build_scatter(ctx, s_start);
        NC_SYNC(ctx);
        edge_build_pairs(ctx, s_start);
        NC_SYNC(ctx);
        if (ctx.rank == 0 && threadIdx.x == 0) ctx.d.edge_ctl[6] = 1u;   // the list is built
    }
    return true;
}

// The build counts serve as fill cursors and ranges until the pairs are
// listed; clear them for the next build.
__device__ __forceinline__ void edge_clear_counts(const Ctx& ctx) {
    for (uint32_t b = ctx.tid; b <= ctx.d.edge_mask; b += ctx.nthreads) ctx.d.edge_count[b] = 0u;
}

// Phase 2: the pairs of the list whose pass spheres overlap (the
// reference's sphere filter) are the candidates, each with a lower bound
// (less the rounding slack) on every distance its solve could see; those
// within the margin of contact are ordered.
__device__ void edge_candidates(Ctx& ctx, bool swept, bool rebuilt) {
    const DeviceCloth& d = ctx.d;
    if (rebuilt) edge_clear_counts(ctx);
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
        const uint32_t k = warp_append(d.edge_ctl + 0);
        if (k >= d.edge_cap) {
            fail(d, NUMI_CLOTH_FAILURE_RANGE);
            continue;
        }
        const bool ordered = !(bound >= thr);
        d.edge_cand[k] = make_uint4(a, b, __float_as_uint(bound), ordered ? 1u : 0u);
        if (ordered) d.edge_order[warp_append(d.edge_ctl + 1)] = edge_key(a, b);
    }
}

// The leaf order of the reference's box tree over the pass-start segment
// boxes (makeCollisionBVH / buildCollisionBVHNode,
// tools/cloth_bag.cpp:3780-3842), in which a segment meets its candidates
// (gatherCollisionCandidates :3844-3878 visits the left subtree first, so
// the candidates come in ascending tree position).  A node of more than 8
// primitives orders them by box centre along the longest axis of its
// centres (ties by index) and splits them at the middle; the node ranges
// follow from the count alone, so the tree is built level by level.  The
// segments are sorted once along each axis (x, y, z lists); every level
// then keeps each node's members in one range of all three lists, each in
// its own axis order: a splitting node sends the first half of its axis
// list to the left child, and a stable partition (one CTA-wide prefix count
// per list) moves every list's members to their child, in order.  A leaf's
// order is its parent's axis list.  CTA 0, all threads; at most
// NC_EDGE_TREE_MAX segments.  edge_tree: [m] segment at each leaf position,
// [m] position of each segment, then the build's scratch (two sets of the
// three lists, the side of each segment, the parent axis of each position).
#define NC_EDGE_TREE_MAX 4096u
#define NC_EDGE_TREE_KEY_BYTES (NC_EDGE_TREE_MAX * 8u)
#define NC_EDGE_TREE_WORDS 14u   /* edge_tree words per segment (13, and one flag word) */
#define NC_EDGE_TREE_WARM 8u     /* odd-even passes tried on the previous order before a full sort */
__shared__ unsigned char nc_edge_tree_axis[NC_EDGE_TREE_MAX / 8u];
__shared__ uint32_t nc_edge_scan[3][32];

// The node of position p (or of index j, a path of `level` left/right bits)
// at depth `level`; false past a leaf.
__device__ __forceinline__ bool tree_node_of_path(uint32_t m, uint32_t level, uint32_t j, uint32_t& b, uint32_t& e) {
    b = 0u;
    e = m;
    for (uint32_t l = 0; l < level; ++l) {
        if (e - b <= 8u) return false;
        const uint32_t mid = b + (e - b) / 2u;
        if ((j >> (level - 1u - l)) & 1u)
            b = mid;
        else
            e = mid;
    }
    return true;
}
__device__ __forceinline__ uint32_t tree_path_of_position(uint32_t m, uint32_t level, uint32_t p, uint32_t& b,
                                                          uint32_t& e) {
    b = 0u;
    e = m;
    uint32_t j = 0u;
    for (uint32_t l = 0; l < level && e - b > 8u; ++l) {
        const uint32_t mid = b + (e - b) / 2u;
        j <<= 1;
        if (p >= mid) {
            b = mid;
            j |= 1u;
        } else {
            e = mid;
        }
    }
    return j;
}
// Float bits in an order of unsigned integers (zeros of either sign equal).
__device__ __forceinline__ uint32_t ordered_bits(float v) {
    if (v == 0.0f) v = 0.0f;
    const uint32_t u = __float_as_uint(v);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

// Ascending bitonic sort of E * blockDim.x keys in shared memory.  Each
// thread holds E consecutive keys in registers: compare distances below E
// stay in the thread, distances below 32 E go between the lanes of a warp
// (shuffles), and only the longer ones pass through shared memory between
// CTA barriers.
template <int E>
__device__ void block_sort_keys(unsigned long long* keys) {
    const uint32_t t = threadIdx.x;
    const uint32_t n = static_cast<uint32_t>(E) * blockDim.x;
    unsigned long long v[E];
#pragma unroll
    for (int r = 0; r < E; ++r) v[r] = keys[t * E + r];
    for (uint32_t k = 2u; k <= n; k <<= 1) {
        for (uint32_t jj = k >> 1; jj >= static_cast<uint32_t>(E); jj >>= 1) {
            if (jj < 32u * E) {
                const uint32_t lm = jj / E;
#pragma unroll
                for (int r = 0; r < E; ++r) {
                    const uint32_t i = t * E + r;
                    const unsigned long long o = __shfl_xor_sync(0xffffffffu, v[r], lm);
                    const bool keep_min = ((i & jj) == 0u) == ((i & k) == 0u);
                    v[r] = keep_min ? (o < v[r] ? o : v[r]) : (o > v[r] ? o : v[r]);
                }
            } else {
                __syncthreads();
#pragma unroll
                for (int r = 0; r < E; ++r) keys[t * E + r] = v[r];
                __syncthreads();
#pragma unroll
                for (int r = 0; r < E; ++r) {
                    const uint32_t i = t * E + r;
                    const unsigned long long o = keys[i ^ jj];
                    const bool keep_min = ((i & jj) == 0u) == ((i & k) == 0u);
                    v[r] = keep_min ? (o < v[r] ? o : v[r]) : (o > v[r] ? o : v[r]);
                }
            }
        }
#pragma unroll
        for (int q = E / 2; q >= 1; q >>= 1) {
            if (static_cast<uint32_t>(q) < k) {
#pragma unroll
                for (int r = 0; r < E; ++r) {
                    const int pr = r ^ q;
                    if (pr > r) {
                        const bool asc = ((t * E + r) & k) == 0u;
                        const unsigned long long a = v[r], b = v[pr];
                        const bool swap = asc ? (a > b) : (a < b);
                        v[r] = swap ? b : a;
                        v[pr] = swap ? a : b;
                    }
                }
            }
        }
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < E; ++r) keys[t * E + r] = v[r];
    __syncthreads();
}

// Sort the first n keys (n a power of two, blockDim.x <= n <= 16 blockDim.x).
__device__ void block_sort(unsigned long long* keys, uint32_t n) {
    switch (n / blockDim.x) {
    case 1u: block_sort_keys<1>(keys); break;
    case 2u: block_sort_keys<2>(keys); break;
    case 4u: block_sort_keys<4>(keys); break;
    case 8u: block_sort_keys<8>(keys); break;
    default: block_sort_keys<16>(keys); break;
    }
}

// Exclusive prefix counts, for each of the three lists L[a][0..m), of the
// members that go right (right[segment] = 1), into pre[a][0..m) (shared
// memory; counts below 65,536): every thread a contiguous run of each list.
__device__ void tree_prefix3(const uint32_t* L, const uint32_t* right, unsigned short* pre, uint32_t m) {
    const uint32_t per = (m + blockDim.x - 1u) / blockDim.x;
    const uint32_t lo = min(threadIdx.x * per, m), hi = min(lo + per, m);
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    uint32_t sum[3], incl[3];
#pragma unroll
    for (uint32_t a = 0; a < 3u; ++a) {
        sum[a] = 0u;
        for (uint32_t p = lo; p < hi; ++p) sum[a] += right[L[a * m + p]];
        incl[a] = sum[a];
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, incl[a], o);
            if (lane >= static_cast<uint32_t>(o)) incl[a] += y;
        }
        if (lane == 31u) nc_edge_scan[a][warp] = incl[a];
    }
    __syncthreads();
    if (warp < 3u) {
        const uint32_t warps = blockDim.x >> 5;
        uint32_t w = lane < warps ? nc_edge_scan[warp][lane] : 0u;
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= static_cast<uint32_t>(o)) w += y;
        }
        if (lane < warps) nc_edge_scan[warp][lane] = w;
    }
    __syncthreads();
#pragma unroll
    for (uint32_t a = 0; a < 3u; ++a) {
        uint32_t run = (warp > 0u ? nc_edge_scan[a][warp - 1u] : 0u) + incl[a] - sum[a];
        for (uint32_t p = lo; p < hi; ++p) {
            pre[a * m + p] = static_cast<unsigned short>(run);
            run += right[L[a * m + p]];
        }
    }
    __syncthreads();
}

__device__ void edge_tree_order(const Ctx& ctx, bool swept) {
    const DeviceCloth& d = ctx.d;
    // the sort keys, then the prefix counts, in the launch's dynamic shared
    // memory
    unsigned long long* keys = reinterpret_cast<unsigned long long*>(nc_frame_smem + ctx.s.tree_keys);
    unsigned short* pre = reinterpret_cast<unsigned short*>(keys);
    const uint32_t m = d.y_count;
    const float ex = 0.5f * (2.0f * ctx.c.radius);
    uint32_t* ord = d.edge_tree;
    uint32_t* lists = d.edge_tree + 2u * m;   // [2][3][m]
    uint32_t* right = lists + 6u * m;         // per segment: goes to the right child
    uint32_t* leaf_axis = right + m;          // per position: axis of its deepest split
    uint32_t* gsort = leaf_axis + m;          // [3][m] the last build's order along each axis
    uint32_t* valid = gsort + 3u * m;         // 1 once a tree was built
    float4* prev = d.edge_centre + m;         // the last build's centres
    // Every array here is written and read by this CTA alone between CTA
    // barriers, which make the writes visible to its threads: plain loads,
    // served from L1.
    const bool warm = *valid != 0u;
    bool changed = !warm;
    for (uint32_t k = threadIdx.x; k < m; k += blockDim.x) {
        const uint2 ab = __ldg(d.y_ij + k);
        const EdgeBox bx = edge_box(xyz(ld(d.edge_x0 + ab.x)), xyz(ld(d.edge_x0 + ab.y)), xyz(ld(d.xp + ab.x)),
                                    xyz(ld(d.xp + ab.y)), swept, ex);
        const float4 c = make_float4(0.5f * (bx.lo.x + bx.hi.x), 0.5f * (bx.lo.y + bx.hi.y),
                                     0.5f * (bx.lo.z + bx.hi.z), 0.0f);
        d.edge_centre[k] = c;
        if (warm) {
            const float4 q = prev[k];
            changed = changed || __float_as_uint(c.x) != __float_as_uint(q.x) ||
                      __float_as_uint(c.y) != __float_as_uint(q.y) || __float_as_uint(c.z) != __float_as_uint(q.z);
        }
        leaf_axis[k] = 3u;
    }
    // the same centres as the last build: the same tree
    if (!__syncthreads_or(changed)) return;
    uint32_t size = blockDim.x;
    while (size < m) size <<= 1;
    // the three axis lists, (centre, index) order: from the last build's
    // order, a few odd-even transposition passes while it is not sorted
    // (the centres move little from pass to pass), else a full sort
    for (uint32_t a = 0; a < 3u; ++a) {
        for (uint32_t p = threadIdx.x; p < size; p += blockDim.x) {
            unsigned long long key = ~0ull;
            if (p < m) {
                const uint32_t sg = warm ? gsort[a * m + p] : p;
                const float4 c = d.edge_centre[sg];
                const float v = a == 0u ? c.x : (a == 1u ? c.y : c.z);
                key = (static_cast<unsigned long long>(ordered_bits(v)) << 12) | sg;
            }
            keys[p] = key;
        }
        __syncthreads();
        bool sorted = false;
        for (uint32_t t = 0; warm && t <= NC_EDGE_TREE_WARM; ++t) {
            bool out = false;
            for (uint32_t p = threadIdx.x; p + 1u < m; p += blockDim.x) out = out || keys[p] > keys[p + 1u];
            if (!__syncthreads_or(out)) {
                sorted = true;
                break;
            }
            if (t == NC_EDGE_TREE_WARM) break;
            for (uint32_t phase = 0; phase < 2u; ++phase) {
                for (uint32_t p = 2u * threadIdx.x + phase; p + 1u < m; p += 2u * blockDim.x) {
                    const unsigned long long x = keys[p], y = keys[p + 1u];
                    if (x > y) {
                        keys[p] = y;
                        keys[p + 1u] = x;
                    }
                }
                __syncthreads();
            }
        }
        if (!sorted) block_sort(keys, size);
        for (uint32_t p = threadIdx.x; p < m; p += blockDim.x) {
            const uint32_t sg = static_cast<uint32_t>(keys[p] & 0xfffull);
            lists[a * m + p] = sg;
            gsort[a * m + p] = sg;
        }
        __syncthreads();
    }
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u, warps = blockDim.x >> 5;
    uint32_t cur = 0u;
    for (uint32_t level = 0; level < 32u; ++level) {
        const uint32_t* L = lists + cur * 3u * m;
        uint32_t* N = lists + (cur ^ 1u) * 3u * m;
        // centre bounds and axis of every node of the level that splits
        const uint32_t nodes = 1u << level;
        bool any = false;
        for (uint32_t j = warp; j < nodes && j < NC_EDGE_TREE_MAX / 8u; j += warps) {
            uint32_t b, e;
            if (!tree_node_of_path(m, level, j, b, e) || e - b <= 8u) continue;
            V3 lo{INFINITY, INFINITY, INFINITY}, hi{-INFINITY, -INFINITY, -INFINITY};
            for (uint32_t p = b + lane; p < e; p += 32u) {
                const float4 c = d.edge_centre[L[p]];
                lo = V3{fminf(lo.x, c.x), fminf(lo.y, c.y), fminf(lo.z, c.z)};
                hi = V3{fmaxf(hi.x, c.x), fmaxf(hi.y, c.y), fmaxf(hi.z, c.z)};
            }
            for (int o = 16; o > 0; o >>= 1) {
                lo.x = fminf(lo.x, __shfl_xor_sync(0xffffffffu, lo.x, o));
                lo.y = fminf(lo.y, __shfl_xor_sync(0xffffffffu, lo.y, o));
                lo.z = fminf(lo.z, __shfl_xor_sync(0xffffffffu, lo.z, o));
                hi.x = fmaxf(hi.x, __shfl_xor_sync(0xffffffffu, hi.x, o));
                hi.y = fmaxf(hi.y, __shfl_xor_sync(0xffffffffu, hi.y, o));
                hi.z = fmaxf(hi.z, __shfl_xor_sync(0xffffffffu, hi.z, o));
            }
            const V3 ext = hi - lo;
            if (lane == 0)
                nc_edge_tree_axis[j] = static_cast<unsigned char>(
                    ext.y > ext.x ? (ext.z > ext.y ? 2u : 1u) : (ext.z > ext.x ? 2u : 0u));
            any = true;
        }
        if (!__syncthreads_or(any)) break;
        // sides: the second half of a splitting node's axis list goes right
        for (uint32_t p = threadIdx.x; p < m; p += blockDim.x) {
            uint32_t b, e;
            const uint32_t j = tree_path_of_position(m, level, p, b, e);
            if (e - b <= 8u) {
                right[L[p]] = 0u;
                continue;
            }
            const uint32_t a = nc_edge_tree_axis[j];
            right[L[a * m + p]] = p - b >= (e - b) / 2u ? 1u : 0u;
            leaf_axis[p] = a;
        }
        __syncthreads();
        // every list: stable partition of each splitting node's range
        tree_prefix3(L, right, pre, m);
        for (uint32_t q = threadIdx.x; q < 3u * m; q += blockDim.x) {
            const uint32_t a = q / m, p = q - a * m;
            uint32_t b, e;
            tree_path_of_position(m, level, p, b, e);
            const uint32_t sg = L[q];
            uint32_t to = p;
            if (e - b > 8u) {
                const uint32_t rights = static_cast<uint32_t>(pre[q]) - static_cast<uint32_t>(pre[a * m + b]);
                to = right[sg] != 0u ? b + (e - b) / 2u + rights : p - rights;
            }
            N[a * m + to] = sg;
        }
        __syncthreads();
        cur ^= 1u;
    }
    const uint32_t* L = lists + cur * 3u * m;
    for (uint32_t p = threadIdx.x; p < m; p += blockDim.x) {
        const uint32_t a = leaf_axis[p];
        ord[p] = a < 3u ? L[a * m + p] : p;
        prev[p] = d.edge_centre[p];
    }
    __syncthreads();
    for (uint32_t p = threadIdx.x; p < m; p += blockDim.x) ord[m + ord[p]] = p;
    if (threadIdx.x == 0) *valid = 1u;
    __syncthreads();
}

// Phase 3 (CTA 0): sort the ordered pairs, undo the previous round, then
// resolve them in the reference's order as wavefronts: a pair's level is one
// more than the last level of any of its four particles, so pairs of one
// level share no particle and every pair runs after all earlier pairs it
// shares a particle with, which is all the serial order requires.  The first
// segment's box of the tree test is taken at its first pair.  Up to
// NC_EDGE_STAGED ordered pairs the sort and the levels run in shared memory
// (each pair finds, in parallel, the last earlier pair of each of its
// particles; one thread then chains the levels); more go through global
// memory with a per-particle level array.
#define NC_EDGE_STAGED 256u
__device__ void edge_resolve(Ctx& ctx, bool swept, bool redo) {
    if (ctx.rank != 0) return;
    const DeviceCloth& d = ctx.d;
    const uint32_t count = min(__ldcg(d.edge_ctl + 1), d.edge_cap);
    const bool staged = count <= NC_EDGE_STAGED;
    // the reduction scratch holds the staged arrays
    static_assert(NC_EDGE_STAGED * (8u + 8u + 16u + 8u + 4u) <= sizeof(nc_red_smem), "staged arrays exceed the scratch");
    unsigned char* scratch = reinterpret_cast<unsigned char*>(&nc_red_smem[0][0]);
    unsigned long long* s_key = reinterpret_cast<unsigned long long*>(scratch);
    unsigned long long* s_sorted = s_key + NC_EDGE_STAGED;
    uint4* s_id = reinterpret_cast<uint4*>(s_sorted + NC_EDGE_STAGED);
    uint2* s_pred = reinterpret_cast<uint2*>(s_id + NC_EDGE_STAGED);   // 16-bit pair indices, 0xffff: none
    uint32_t* s_lv = reinterpret_cast<uint32_t*>(s_pred + NC_EDGE_STAGED);
    if (redo) {
        // back to the pass-start positions of every particle the last round
        // moved (particles shared by records get the same values)
        const uint32_t done = __ldcg(d.edge_ctl + 4);
        for (uint32_t r = threadIdx.x; r < done; r += blockDim.x) {
            const EdgeRecord& rec = d.edge_new[__ldcg(d.edge_done + r)];
            const uint2 sa = __ldg(d.y_ij + rec.i), sb = __ldg(d.y_ij + rec.j);
            const uint32_t id[4] = {sa.x, sa.y, sb.x, sb.y};
            for (int e = 0; e < 4; ++e) {
                px_set(ctx, id[e], ld(d.edge_x0 + id[e]));
                d.edge_path[id[e]] = 0.0f;
            }
        }
    }
    __shared__ uint32_t s_top;
    // A segment with several ordered pairs meets them in the tree's leaf
    // order (edge_tree_order), else the first segments' order is all that
    // matters: pairs are sorted by (first, tree position of the second).
    bool mine = false;
    if (staged) {
        // the first segments in shared memory (the staged key array, filled
        // again below), compared there
        uint32_t* s_first = reinterpret_cast<uint32_t*>(s_key);
        for (uint32_t k = threadIdx.x; k < count; k += blockDim.x)
            s_first[k] = static_cast<uint32_t>(__ldcg(d.edge_order + k) >> 32);
        __syncthreads();
        for (uint32_t k = threadIdx.x; k < count && !mine; k += blockDim.x) {
            const uint32_t first = s_first[k];
            for (uint32_t m = 0; m < count && !mine; ++m) mine = m != k && s_first[m] == first;
        }
    } else {
        for (uint32_t k = threadIdx.x; k < count && !mine; k += blockDim.x) {
            const uint32_t first = static_cast<uint32_t>(__ldcg(d.edge_order + k) >> 32);
            for (uint32_t m = 0; m < count && !mine; ++m)
                mine = m != k && static_cast<uint32_t>(__ldcg(d.edge_order + m) >> 32) == first;
        }
    }
    const bool tree = __syncthreads_or(mine) != 0 && d.y_count <= NC_EDGE_TREE_MAX && ctx.s.tree_keys != 0u;
    if (tree) edge_tree_order(ctx, swept);
    const uint32_t* tpos = d.edge_tree + d.y_count;
    auto sort_key = [&](unsigned long long key) {
        return tree ? ((key & 0xffffffff00000000ull) | __ldcg(tpos + static_cast<uint32_t>(key))) : key;
    };
    if (staged) {
        __syncthreads();   // the first-segment comparisons are done with the scratch
        for (uint32_t k = threadIdx.x; k < count; k += blockDim.x) s_key[k] = sort_key(__ldcg(d.edge_order + k));
        __syncthreads();
        // rank sort: the keys are distinct
        for (uint32_t k = threadIdx.x; k < count; k += blockDim.x) {
            const unsigned long long key = s_key[k];
            uint32_t rank = 0;
            for (uint32_t m = 0; m < count; ++m) rank += s_key[m] < key ? 1u : 0u;
            const unsigned long long orig = __ldcg(d.edge_order + k);
            s_sorted[rank] = orig;
            d.edge_sorted[rank] = orig;
            const uint2 sa = __ldg(d.y_ij + static_cast<uint32_t>(orig >> 32)),
                        sb = __ldg(d.y_ij + static_cast<uint32_t>(orig));
            s_id[rank] = make_uint4(sa.x, sa.y, sb.x, sb.y);
        }
        __syncthreads();
        // the last earlier pair of each particle
        for (uint32_t k = threadIdx.x; k < count; k += blockDim.x) {
            const uint4 me = s_id[k];
            const uint32_t id[4] = {me.x, me.y, me.z, me.w};
            uint32_t pred[4] = {0xffffu, 0xffffu, 0xffffu, 0xffffu};
            uint32_t open = 4u;
            for (uint32_t m = k; m-- > 0u && open > 0u;) {
                const uint4 o = s_id[m];
                for (int e = 0; e < 4; ++e)
                    if (pred[e] == 0xffffu && (o.x == id[e] || o.y == id[e] || o.z == id[e] || o.w == id[e])) {
                        pred[e] = m;
                        --open;
                    }
            }
            s_pred[k] = make_uint2(pred[0] | (pred[1] << 16), pred[2] | (pred[3] << 16));
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t top = 0;
            for (uint32_t k = 0; k < count; ++k) {
                const uint2 pr = s_pred[k];
                const uint32_t pk[4] = {pr.x & 0xffffu, pr.x >> 16, pr.y & 0xffffu, pr.y >> 16};
                uint32_t lv = 0;
                for (int e = 0; e < 4; ++e)
                    if (pk[e] != 0xffffu) lv = max(lv, s_lv[pk[e]] & 0x3fffffffu);
                ++lv;
                const bool first = k == 0u || (s_sorted[k - 1u] >> 32) != (s_sorted[k] >> 32);
                s_lv[k] = lv | (first ? 0x80000000u : 0u);
                top = max(top, lv);
            }
            s_top = top;
        }
    } else {
        // rank sort: the keys are distinct
        for (uint32_t k = threadIdx.x; k < count; k += blockDim.x) {
            const unsigned long long orig = __ldcg(d.edge_order + k);
            const unsigned long long key = sort_key(orig);
            uint32_t rank = 0;
            for (uint32_t m = 0; m < count; ++m) rank += sort_key(__ldcg(d.edge_order + m)) < key ? 1u : 0u;
            d.edge_sorted[rank] = orig;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t top = 0;
            for (uint32_t k = 0; k < count; ++k) {
                const unsigned long long key = d.edge_sorted[k];
                const uint32_t i = static_cast<uint32_t>(key >> 32);
                const uint2 sa = __ldg(d.y_ij + i), sb = __ldg(d.y_ij + static_cast<uint32_t>(key));
                const uint32_t id[4] = {sa.x, sa.y, sb.x, sb.y};
                uint32_t lv = 0;
                for (int e = 0; e < 4; ++e) lv = max(lv, d.edge_level[id[e]]);
                ++lv;
                for (int e = 0; e < 4; ++e) d.edge_level[id[e]] = lv;
                const bool first = k == 0u || static_cast<uint32_t>(d.edge_sorted[k - 1u] >> 32) != i;
                d.edge_lv[k] = lv | (first ? 0x80000000u : 0u);
                top = max(top, lv);
            }
            for (uint32_t k = 0; k < count; ++k) {   // leave the level marks zero for the next pass
                const unsigned long long key = d.edge_sorted[k];
                const uint2 sa = __ldg(d.y_ij + static_cast<uint32_t>(key >> 32)),
                            sb = __ldg(d.y_ij + static_cast<uint32_t>(key));
                d.edge_level[sa.x] = d.edge_level[sa.y] = d.edge_level[sb.x] = d.edge_level[sb.y] = 0u;
            }
            s_top = top;
        }
    }
    __syncthreads();
    uint32_t* lvp = staged ? s_lv : d.edge_lv;
    const uint32_t top = s_top;
    const float ex = 0.5f * (2.0f * ctx.c.radius);
    for (uint32_t level = 1; level <= top; ++level) {
        for (uint32_t k = threadIdx.x; k < count; k += blockDim.x) {
            const uint32_t tagged = lvp[k];
            if ((tagged & 0x3fffffffu) != level) continue;
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
            // the reference's tree query: the first segment's box when its
            // turn comes (before any of its own pairs), against the second
            // segment's pass-start box
            EdgeBox qi;
            if (tagged & 0x80000000u) {
                qi = edge_box(xyz(q.x[0]), xyz(q.x[1]), q.p[0], q.p[1], swept, ex);
                float* qb = d.edge_qbox_raw + 6u * i;
                qb[0] = qi.lo.x; qb[1] = qi.lo.y; qb[2] = qi.lo.z;
                qb[3] = qi.hi.x; qb[4] = qi.hi.y; qb[5] = qi.hi.z;
            } else {
                const float* qb = d.edge_qbox_raw + 6u * i;   // written at a lower level
                qi.lo = V3{qb[0], qb[1], qb[2]};
                qi.hi = V3{qb[3], qb[4], qb[5]};
            }
            const EdgeBox bj =
                edge_box(xyz(ld(d.edge_x0 + sb.x)), xyz(ld(d.edge_x0 + sb.y)), q.p[2], q.p[3], swept, ex);
            EdgeRecord rec{};
            rec.i = i;
            rec.j = j;
            bool moved = false;
            if (boxes_overlap(bj, qi))
                moved = swept ? edge_swept(q, ctx.c.radius, ctx.c.dt, rec) : edge_present(q, ctx.c.radius, ctx.c.dt, rec);
            if (moved) {
                for (int e = 0; e < 4; ++e) {
                    const float4 before = px(ctx, q.id[e]);
                    d.edge_path[q.id[e]] = d.edge_path[q.id[e]] + len3(xyz(q.x[e]) - xyz(before));
                    px_set(ctx, q.id[e], q.x[e]);
                }
                d.edge_new[k] = rec;
                lvp[k] = tagged | 0x40000000u;
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {   // the pairs that moved, in key order
        uint32_t done = 0;
        for (uint32_t k = 0; k < count; ++k)
            if (lvp[k] & 0x40000000u) d.edge_done[done++] = k;
        if (tree) {
            // in tree order within a first segment: back to key order
            for (uint32_t a = 1; a < done; ++a) {
                const uint32_t v = d.edge_done[a];
                const unsigned long long kv = d.edge_sorted[v];
                uint32_t b = a;
                while (b > 0u && d.edge_sorted[d.edge_done[b - 1u]] > kv) {
                    d.edge_done[b] = d.edge_done[b - 1u];
                    --b;
                }
                d.edge_done[b] = v;
            }
        }
        d.edge_ctl[4] = done;
    }
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
        const EdgeRecord& n = d.edge_new[d.edge_done[k]];
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
        const EdgeRecord& n = d.edge_new[d.edge_done[k]];
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
    bool rebuilt = false;
    if (!edge_prepare(ctx, swept, rebuilt)) return false;
    edge_candidates(ctx, swept, rebuilt);
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
    return true;
}

// The deepest non-local pair of the current positions
// (measurePrimitiveSelfPenetration, tools/cloth_bag.cpp:4182-4247): every
// pair closer than the yarn diameter passes the reference's box and sphere
// filters (and is on the pair list), so the maximum over the listed pairs
// whose present spheres overlap (and 0) is the reference's value.  Writes
// this CTA's maximum to edge_red[rank].
__device__ void edge_deepest(Ctx& ctx, bool rebuilt) {
    const DeviceCloth& d = ctx.d;
    if (rebuilt) edge_clear_counts(ctx);
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
    bool rebuilt = false;
    if (!edge_prepare(ctx, false, rebuilt)) return false;
    edge_deepest(ctx, rebuilt);
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
