// C ABI of the cloth solver: handle lifetime, validation, colour batches,
// AoS <-> SoA conversion at the boundary, and the cooperative launch.
//
// Replaces the reference Metal host runGPU (tools/cloth_bag_metal.mm:4010-4760):
// buffer allocation (:4091-4202), per-substep encoding (:4211-4709), commit
// and readback (:4710-4757), and the colouring check verifyColoring
// (tools/cloth_bag_metal.mm:1705-1819).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <mutex>
#include <vector>

#include "cloth_frame.cuh"
#include "cloth_adjoint.cuh"
#include "numi_cloth.h"

static_assert(sizeof(NumiClothConfig) == 224, "Config layout");
static_assert(sizeof(NumiClothParticle) == 48, "Particle layout");
static_assert(sizeof(NumiClothDistance) == 32, "Distance layout");
static_assert(sizeof(NumiClothGrip) == 48, "Grip layout");
static_assert(sizeof(NumiClothKnot) == 48, "Knot layout");
static_assert(sizeof(NumiClothBend) == 32, "Bend layout");
static_assert(sizeof(NumiClothFruit) == 96, "Fruit layout");
static_assert(sizeof(NumiClothFruitPair) == 32, "FruitPair layout");
static_assert(sizeof(NumiClothBatch) == 16, "Batch layout");
static_assert(offsetof(NumiClothConfig, gravityAndTimestep) == 48, "Config offsets");
static_assert(offsetof(NumiClothConfig, mouthMaterial) == 208, "Config offsets");
static_assert(sizeof(DeviceCloth) % 4u == 0u, "DeviceCloth is copied as 32-bit words");

__global__ void __launch_bounds__(NC_THREADS) numi_cloth_residual_kernel(DeviceCloth d, NumiClothConfig cfg) {
    Schedule s{};
    nc::Ctx ctx{d, s};
    ctx.gx = d.x;
    ctx.gv = d.v;
    ctx.c = nc::load_cfg(&cfg);
    ctx.tid = blockIdx.x * blockDim.x + threadIdx.x;
    ctx.nthreads = gridDim.x * blockDim.x;
    ctx.rank = blockIdx.x;
    ctx.ranks = gridDim.x;
    nc::residual_partials(ctx, d.red);
}

namespace {

constexpr uint32_t kSnapshotSlots = 8;
constexpr uint32_t kTuneSlot = kSnapshotSlots;   // snapshot slot of the launch-shape tuners
constexpr uint32_t kResidentChunk = 4096;   // particles a CTA holds in resident mode
constexpr uint32_t kResidentClusterChunk = 256;   // default chunk of a small resident cloth
constexpr uint32_t kBarrierWords = 48;   // barrier counter, abort, release and fruit flags: three 128-byte lines

struct Snapshot {
    bool valid = false;
    void* mem = nullptr;
    size_t bytes = 0;
};

struct DeviceBuffers {
    std::vector<void*> owned;
    template <class T>
    T* alloc(size_t count) {
        if (count == 0) count = 1;
        void* p = nullptr;
        if (cudaMalloc(&p, count * sizeof(T)) != cudaSuccess) return nullptr;
        cudaMemset(p, 0, count * sizeof(T));
        owned.push_back(p);
        return static_cast<T*>(p);
    }
    ~DeviceBuffers() {
        for (void* p : owned) cudaFree(p);
    }
};

bool env_u32(const char* name, uint32_t& out) {
    const char* v = std::getenv(name);
    if (v == nullptr || *v == 0) return false;
    out = static_cast<uint32_t>(std::strtoul(v, nullptr, 10));
    return true;
}

}  // namespace

struct numi_cloth {
    int device = 0;
    cudaStream_t stream = nullptr;
    DeviceBuffers buf;
    DeviceCloth d{};
    NumiClothConfig base{};
    NumiClothConfig* d_cfg = nullptr;
    uint32_t cfg_capacity = 0;
    uint32_t epoch = 1;
    uint32_t host_failure = 0;
    bool poisoned = false;
    bool self_exact = false;   // point self contact in the reference's order (NUMI_CLOTH_SELF_ORDER=reference)
    uint32_t grid = 1;
    uint32_t block = NC_THREADS;
    uint32_t cluster = 0;   // > 0: the grid is one cluster of this many CTAs
    size_t smem = nc_resident_offset();   // dynamic shared memory of a frame launch
    uint32_t launches = 0;
    uint32_t trace_capacity = 0;   // substeps the trace buffer holds
    uint32_t last_substeps = 0;
    float yarn_rest_median = 0.0f;   // median yarn segment rest length
    bool neighbours = false;         // neighbour-sync tables built for the cooperative grid
    size_t nbr_smem = 0;             // dynamic shared memory of a frame launch with them
    // tile mode (cloth_tile.cuh): launch shape and shared memory of a tile
    // launch; the plan is rebuilt before the next launch when a material
    // changed (its items carry the materials)
    bool tiles = false;
    bool tiles_dirty = false;
    uint32_t tile_grid = 0, tile_block = 0;
    size_t tile_smem = 0;
    uint32_t last_grid = 0, last_block = 0;
    bool last_tiles = false;
    // host copies for the edge/edge local lists, built with the edge buffers
    std::vector<uint2> host_yarn;
    std::vector<uint32_t> host_local_off, host_local_idx;
    Snapshot snaps[kSnapshotSlots + 1u];   // the callers' slots, then the tuners' own
    // dynamic state regions copied by snapshot/restore
    struct Region {
        void* ptr;
        size_t bytes;
    };
    std::vector<Region> dynamic;
    // device staging of particle records for the host copies (one transfer
    // each way, transposed to and from the state arrays on the device)
    NumiClothParticle* io = nullptr;
};

namespace {

// cudaFuncAttributeMaxDynamicSharedMemorySize is per function, not per
// launch, and cloths with different launch modes share the frame kernel: only
// ever raise it, so that creating one cloth never breaks another's launch.
// The frame and batch kernels come in two builds: without and with the
// edge/edge yarn self-collision phases (primitiveSelf).
// A third pair resolves point self contact in the reference's Gauss-Seidel
// order (NUMI_CLOTH_SELF_ORDER=reference at create).
const void* frame_fn(bool edge, bool exact = false) {
    if (exact)
        return edge ? reinterpret_cast<const void*>(numi_cloth_frame_edge_exact_kernel)
                    : reinterpret_cast<const void*>(numi_cloth_frame_exact_kernel);
    return edge ? reinterpret_cast<const void*>(numi_cloth_frame_edge_kernel)
                : reinterpret_cast<const void*>(numi_cloth_frame_kernel);
}
const void* batch_fn(bool edge) {
    return edge ? reinterpret_cast<const void*>(numi_cloth_batch_edge_kernel)
                : reinterpret_cast<const void*>(numi_cloth_batch_kernel);
}

cudaError_t raise_smem(const void* fn, size_t bytes) {
    cudaFuncAttributes fa{};
    cudaError_t e = cudaFuncGetAttributes(&fa, fn);
    if (e != cudaSuccess) return e;
    if (static_cast<size_t>(fa.maxDynamicSharedSizeBytes) >= bytes) return cudaSuccess;
    return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes));
}
cudaError_t raise_frame_smem(size_t bytes) {
    cudaError_t e = cudaSuccess;
    for (bool exact : {false, true})
        for (bool edge : {false, true})
            if (e == cudaSuccess) e = raise_smem(frame_fn(edge, exact), bytes);
    return e;
}
void allow_large_clusters() {
    for (bool exact : {false, true})
        for (bool edge : {false, true})
            cudaFuncSetAttribute(frame_fn(edge, exact), cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
}
// Clusters of cfg's shape that every frame kernel can place at once.
int frame_clusters(const cudaLaunchConfig_t& cfg) {
    int lo = 1 << 30;
    for (bool exact : {false, true})
        for (bool edge : {false, true}) {
            int clusters = 0;
            if (cudaOccupancyMaxActiveClusters(&clusters, frame_fn(edge, exact), &cfg) != cudaSuccess) return 0;
            lo = std::min(lo, clusters);
        }
    return lo;
}

bool finite4(const numi_float4& v) {
    return std::isfinite(v.x) && std::isfinite(v.y) && std::isfinite(v.z) && std::isfinite(v.w);
}

// Host twin of the reference validConfig (ClothBag.metal:16-55).
uint32_t validate_config(const NumiClothConfig& c, const NumiClothConfig& base) {
    if (c.control.x != NUMI_CLOTH_ABI_VERSION) return NUMI_CLOTH_FAILURE_ABI;
    if (c.control.y != base.control.y || c.control.z != base.control.z || c.control.w != base.control.w ||
        c.constraintCounts.x != base.constraintCounts.x || c.constraintCounts.y != base.constraintCounts.y ||
        c.constraintCounts.w != base.constraintCounts.w || c.contactCounts.x != base.contactCounts.x)
        return NUMI_CLOTH_FAILURE_RANGE;
    const float dt = c.gravityAndTimestep.w;
    bool ok = dt > 0.0f && std::isfinite(dt) && finite4(c.gravityAndTimestep) && finite4(c.gripTargetAndActive) &&
              finite4(c.gripOrientation) && finite4(c.gripMaterial) && finite4(c.clothMaterial) &&
              finite4(c.fruitMaterial) && finite4(c.airVelocityAndDensity) && finite4(c.aerodynamicCoefficients) &&
              finite4(c.mouthMaterial) && c.clothMaterial.x >= 0.0f && c.airVelocityAndDensity.w >= 0.0f &&
              c.aerodynamicCoefficients.x >= 0.0f && c.aerodynamicCoefficients.y >= 0.0f &&
              c.aerodynamicCoefficients.z >= 0.0f && c.aerodynamicCoefficients.w >= 0.0f &&
              c.gripMaterial.x >= 0.0f && c.gripControl.y <= 1u && c.mouthMaterial.x >= 0.0f &&
              c.mouthControl.x <= NUMI_CLOTH_MOUTH_RIM_CAPACITY;
    if (ok && c.gripTargetAndActive.w > 0.0f) {
        const numi_float4& q = c.gripOrientation;
        const float len = std::sqrt(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w);
        ok = std::fabs(len - 1.0f) <= 1.0e-4f && c.gripControl.x != 0u && c.gripMaterial.x > 0.0f;
    }
    if (ok && c.gripControl.y == 1u) {
        ok = c.gripControl.z >= 2u * c.gripControl.w + 1u && c.gripControl.z <= NUMI_CLOTH_MOUTH_RIM_CAPACITY &&
             c.gripControl.w <= 16u && c.control.w == 2u * (2u * c.gripControl.w + 1u);
    }
    return ok ? 0u : NUMI_CLOTH_FAILURE_NONFINITE;
}

// Colour runs -> batches; checks contiguity and one writer per particle.
template <class Rec, class ColourFn, class WritersFn, class YarnFn, class LimitFn>
int make_batches(const Rec* recs, uint32_t count, uint32_t n_targets, ColourFn colour, WritersFn writers,
                 YarnFn yarn, LimitFn limited, Batch* out, uint32_t& n_out) {
    n_out = 0;
    std::vector<uint32_t> stamp(n_targets, 0xffffffffu);
    std::vector<uint32_t> seen_colours;
    uint32_t k = 0;
    while (k < count) {
        const uint32_t col = colour(recs[k]);
        if (std::find(seen_colours.begin(), seen_colours.end(), col) != seen_colours.end()) return NUMI_CLOTH_EBATCH;
        seen_colours.push_back(col);
        if (n_out >= NC_MAX_BATCHES) return NUMI_CLOTH_EINVAL;
        Batch b{k, 0, 0, 0};
        bool yarn_open = true;
        while (k < count && colour(recs[k]) == col) {
            uint32_t w[4];
            const int nw = writers(recs[k], w);
            if (nw < 0) return NUMI_CLOTH_EINVAL;
            for (int e = 0; e < nw; ++e) {
                if (w[e] >= n_targets) return NUMI_CLOTH_EINVAL;
                if (stamp[w[e]] == n_out) return NUMI_CLOTH_EBATCH;
                stamp[w[e]] = n_out;
            }
            if (yarn(recs[k])) {
                if (!yarn_open) return NUMI_CLOTH_EINVAL;   // yarn segments lead their colour
                b.yarn = k - b.first + 1u;
            } else {
                yarn_open = false;
            }
            if (limited(recs[k])) b.limited = k - b.first + 1u;
            ++k;
        }
        b.count = k - b.first;
        out[n_out++] = b;
    }
    return NUMI_CLOTH_OK;
}

// Neighbour syncs of the cooperative grid.  CTA r takes, in every colour
// batch, the items whose lowest particle lies in its equal share
// [r n / R, (r + 1) n / R) of the particle range (a list of batch-relative
// indices per colour, staged in its shared memory); its neighbours are the
// CTAs whose items share a particle with its own in any colour (reads
// included: a bend's middle particle).  Built when no CTA has more than
// NC_NBR_MAX neighbours, its lists fit NC_NBR_WORDS words, and the grid
// stays co-resident with them; otherwise every colour ends with the grid
// barrier.  NUMI_CLOTH_NEIGHBOUR_SYNC=0 keeps the grid barrier.
#define NC_NBR_WORDS 4096u
bool prepare_neighbours(numi_cloth* h, const NumiClothScene* scene) {
    DeviceCloth& d = h->d;
    const uint32_t R = h->grid, n = d.n;
    const uint32_t slots = d.n_dist_batches + d.n_knot_batches + d.n_bend_batches;
    uint32_t want = 1;
    env_u32("NUMI_CLOTH_NEIGHBOUR_SYNC", want);
    if (want == 0u || R < 2u || h->cluster != 0u || d.resident != 0u || n == 0u || slots == 0u ||
        slots > 3u * NC_MAX_BATCHES)
        return false;
    auto cta_of = [&](uint32_t p) { return static_cast<uint32_t>(static_cast<uint64_t>(p) * R / n); };
    // lists[r][slot]: CTA r's items of the colour, ascending
    std::vector<std::vector<std::vector<uint32_t>>> lists(R, std::vector<std::vector<uint32_t>>(slots));
    std::vector<std::vector<uint32_t>> touch(n);   // CTAs touching each particle
    auto batch = [&](uint32_t slot, const Batch& bt, auto parts) {
        for (uint32_t k = 0; k < bt.count; ++k) {
            uint32_t p[4];
            const int np = parts(bt.first + k, p);
            uint32_t lowest = p[0];
            for (int e = 1; e < np; ++e) lowest = std::min(lowest, p[e]);
            const uint32_t c = cta_of(lowest);
            lists[c][slot].push_back(k);
            for (int e = 0; e < np; ++e) {
                std::vector<uint32_t>& t = touch[p[e]];
                if (std::find(t.begin(), t.end(), c) == t.end()) t.push_back(c);
            }
        }
    };
    for (uint32_t b = 0; b < d.n_dist_batches; ++b)
        batch(b, d.dist_batches[b], [&](uint32_t i, uint32_t* p) {
            p[0] = scene->distances[i].particlesAndColor.x;
            p[1] = scene->distances[i].particlesAndColor.y;
            return 2;
        });
    for (uint32_t b = 0; b < d.n_knot_batches; ++b)
        batch(d.n_dist_batches + b, d.knot_batches[b], [&](uint32_t i, uint32_t* p) {
            const NumiClothKnot& r = scene->knots[i];
            p[0] = r.particles.x;
            p[1] = r.particles.y;
            p[2] = r.particles.z;
            p[3] = r.particles.w;
            return 4;
        });
    for (uint32_t b = 0; b < d.n_bend_batches; ++b)
        batch(d.n_dist_batches + d.n_knot_batches + b, d.bend_batches[b], [&](uint32_t i, uint32_t* p) {
            p[0] = scene->bends[i].particlesAndColor.x;
            p[1] = scene->bends[i].particlesAndColor.y;
            p[2] = scene->bends[i].particlesAndColor.z;
            return 3;
        });
    std::vector<std::vector<uint32_t>> nbr(R);
    for (const std::vector<uint32_t>& t : touch)
        for (uint32_t c : t)
            for (uint32_t o : t)
                if (o != c && std::find(nbr[c].begin(), nbr[c].end(), o) == nbr[c].end()) {
                    if (nbr[c].size() >= NC_NBR_MAX) return false;
                    nbr[c].push_back(o);
                }
    std::vector<uint32_t> off(R + 1u, 0u), idx, block(R + 1u, 0u), items;
    uint32_t widest = 0;
    for (uint32_t r = 0; r < R; ++r) {
        std::sort(nbr[r].begin(), nbr[r].end());
        idx.insert(idx.end(), nbr[r].begin(), nbr[r].end());
        off[r + 1u] = static_cast<uint32_t>(idx.size());
        // the CTA's block: slot offsets, then the items
        uint32_t at = 0;
        for (uint32_t b = 0; b < slots; ++b) {
            items.push_back(at);
            at += static_cast<uint32_t>(lists[r][b].size());
        }
        items.push_back(at);
        for (uint32_t b = 0; b < slots; ++b) items.insert(items.end(), lists[r][b].begin(), lists[r][b].end());
        block[r + 1u] = static_cast<uint32_t>(items.size());
        widest = std::max(widest, block[r + 1u] - block[r]);
    }
    if (widest > NC_NBR_WORDS) return false;
    const size_t smem = nc_resident_offset() + static_cast<size_t>(widest) * sizeof(uint32_t);
    int per_sm = 0;
    if (raise_frame_smem(smem) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, frame_fn(false, h->self_exact), static_cast<int>(h->block), smem) !=
            cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device);
    if (static_cast<uint64_t>(per_sm) * static_cast<uint64_t>(sms) < R) return false;   // must stay co-resident
    uint32_t* d_block = h->buf.alloc<uint32_t>(block.size());
    uint32_t* d_items = h->buf.alloc<uint32_t>(items.size());
    uint32_t* d_off = h->buf.alloc<uint32_t>(off.size());
    uint32_t* d_idx = h->buf.alloc<uint32_t>(std::max<size_t>(idx.size(), 1));
    unsigned int* d_flag = h->buf.alloc<unsigned int>(static_cast<size_t>(NC_NBR_FLAG_STRIDE) * R);
    if (!d_block || !d_items || !d_off || !d_idx || !d_flag) return false;
    if (cudaMemcpy(d_block, block.data(), block.size() * sizeof(uint32_t), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(d_items, items.data(), items.size() * sizeof(uint32_t), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(d_off, off.data(), off.size() * sizeof(uint32_t), cudaMemcpyHostToDevice) != cudaSuccess ||
        (!idx.empty() &&
         cudaMemcpy(d_idx, idx.data(), idx.size() * sizeof(uint32_t), cudaMemcpyHostToDevice) != cudaSuccess))
        return false;
    d.colour_slots = slots;
    d.nbr_block = d_block;
    d.nbr_items = d_items;
    d.nbr_off = d_off;
    d.nbr_idx = d_idx;
    d.nbr_flag = d_flag;
    h->nbr_smem = smem;
    return true;
}

// Tile plans of the cooperative grid (cloth_tile.cuh).  CTA t < T owns a
// tile: for a row-major grid cloth a block of a x b particles (the shape
// with the fewest estimated closure particles among those giving at most T
// tiles), else an index strip; the last CTA is the fruit CTA and owns none.
// For each chain of colours the closure of a tile is found backwards: the
// items of the last colour touching an owned particle, then those of the
// colour before touching an owned particle or a particle of an item found,
// and so on.  Local particles are ordered own, then the fruit/yarn and
// strain chains' other particles, then the constraint chain's, so every
// chain reads a prefix.  Returns false (tile mode off) when a plan would not
// fit the shared memory of one CTA per SM or a closure holds 65,536
// particles or more.
struct TileColour {
    uint32_t family, first, count;
};

bool build_tiles(numi_cloth* h, uint32_t grid_width, const std::vector<uint2>& dij, const std::vector<float4>& dmat,
                 const std::vector<uint4>& bij, const std::vector<float2>& bmat, size_t smem_budget) {
    const DeviceCloth& d = h->d;
    const uint32_t n = d.n, R = h->tile_grid, T = R - 1u;
    if (R < 3u || n == 0u) return false;
    // tiles
    std::vector<uint32_t> tile_of(n);
    uint32_t tiles = 0;
    if (grid_width > 0u && n % grid_width == 0u) {
        const uint32_t W = grid_width, H = n / grid_width;
        uint32_t best_a = 0, best_b = 0;
        uint64_t best = ~0ull;
        for (uint32_t a = 1; a <= std::min(H, 512u); ++a)
            for (uint32_t b = 1; b <= std::min(W, 512u); ++b) {
                const uint64_t count = static_cast<uint64_t>((H + a - 1u) / a) * ((W + b - 1u) / b);
                if (count > T) continue;
                const uint64_t cost = static_cast<uint64_t>(a + 12u) * (b + 12u);
                if (cost < best) {
                    best = cost;
                    best_a = a;
                    best_b = b;
                }
            }
        if (best_a == 0u) return false;
        const uint32_t across = (W + best_b - 1u) / best_b;
        for (uint32_t i = 0; i < n; ++i) tile_of[i] = (i / W / best_a) * across + (i % W) / best_b;
        tiles = ((H + best_a - 1u) / best_a) * across;
    } else {
        for (uint32_t i = 0; i < n; ++i) tile_of[i] = static_cast<uint32_t>(static_cast<uint64_t>(i) * T / n);
        tiles = T;
    }
    // chains
    std::vector<std::vector<TileColour>> chains(NC_TILE_CHAINS);
    for (uint32_t b = 0; b < d.n_dist_batches; ++b) {
        const Batch& bt = d.dist_batches[b];
        chains[NC_TILE_CONSTRAINTS].push_back({NC_TILE_DISTANCE, bt.first, bt.count});
        if (bt.yarn) chains[NC_TILE_YARN].push_back({NC_TILE_SEGMENT, bt.first, bt.yarn});
        if (bt.limited) chains[NC_TILE_STRAIN].push_back({NC_TILE_LIMIT, bt.first, bt.limited});
    }
    for (uint32_t b = 0; b < d.n_bend_batches; ++b)
        chains[NC_TILE_CONSTRAINTS].push_back({NC_TILE_BEND, d.bend_batches[b].first, d.bend_batches[b].count});
    // particle -> records (CSR), distances and bends
    auto csr = [&](uint32_t records, auto ends, std::vector<uint32_t>& off, std::vector<uint32_t>& idx) {
        off.assign(n + 1u, 0u);
        for (uint32_t k = 0; k < records; ++k) {
            const uint2 e = ends(k);
            ++off[e.x + 1u];
            ++off[e.y + 1u];
        }
        for (uint32_t i = 0; i < n; ++i) off[i + 1u] += off[i];
        idx.assign(off[n], 0u);
        std::vector<uint32_t> at(off.begin(), off.end() - 1);
        for (uint32_t k = 0; k < records; ++k) {
            const uint2 e = ends(k);
            idx[at[e.x]++] = k;
            idx[at[e.y]++] = k;
        }
    };
    std::vector<uint32_t> doff, didx, boff, bidx;
    csr(d.d_count, [&](uint32_t k) { return dij[k]; }, doff, didx);
    csr(d.b_count, [&](uint32_t k) { return make_uint2(bij[k].x, bij[k].z); }, boff, bidx);
    auto ends = [&](uint32_t family, uint32_t rec) {
        return family == NC_TILE_BEND ? make_uint2(bij[rec].x, bij[rec].z) : dij[rec];
    };
    std::vector<uint32_t> owner(n, 0u), local_of(n, 0u);
    std::vector<uint32_t> need_stamp(n, 0u), item_stamp_d(d.d_count, 0u), item_stamp_b(d.b_count, 0u);
    std::vector<int32_t> lidx(n, -1);
    uint32_t stamp = 0;
    std::vector<std::vector<uint32_t>> plans(R);
    size_t widest = 0;
    std::vector<std::vector<uint32_t>> own_of(tiles);
    for (uint32_t i = 0; i < n; ++i) own_of[tile_of[i]].push_back(i);
    for (uint32_t t = 0; t < R; ++t) {
        const std::vector<uint32_t> none;
        const std::vector<uint32_t>& own = t < tiles ? own_of[t] : none;
        // closures: per chain, the items of every colour and the particles
        std::vector<std::vector<std::vector<uint32_t>>> items(NC_TILE_CHAINS);
        std::vector<std::vector<uint32_t>> parts(NC_TILE_CHAINS);
        for (uint32_t k = 0; k < NC_TILE_CHAINS; ++k) {
            const uint32_t g = ++stamp;
            std::vector<uint32_t> cur(own.begin(), own.end());
            for (uint32_t p : cur) need_stamp[p] = g;
            items[k].resize(chains[k].size());
            for (size_t c = chains[k].size(); c-- > 0;) {
                const TileColour& col = chains[k][c];
                const uint32_t cs = ++stamp;
                std::vector<uint32_t>& its = items[k][c];
                const size_t upto = cur.size();
                for (size_t q = 0; q < upto; ++q) {
                    const uint32_t p = cur[q];
                    const bool bend = col.family == NC_TILE_BEND;
                    const std::vector<uint32_t>& off = bend ? boff : doff;
                    const std::vector<uint32_t>& idx = bend ? bidx : didx;
                    std::vector<uint32_t>& ist = bend ? item_stamp_b : item_stamp_d;
                    for (uint32_t e = off[p]; e < off[p + 1u]; ++e) {
                        const uint32_t rec = idx[e];
                        if (rec < col.first || rec >= col.first + col.count || ist[rec] == cs) continue;
                        ist[rec] = cs;
                        its.push_back(rec);
                        const uint2 pe = ends(col.family, rec);
                        for (uint32_t v : {pe.x, pe.y})
                            if (need_stamp[v] != g) {
                                need_stamp[v] = g;
                                cur.push_back(v);
                            }
                    }
                }
                std::sort(its.begin(), its.end());
            }
            parts[k] = cur;
        }
        // local order: own, then the yarn and strain chains' others, then
        // the constraint chain's
        std::vector<uint32_t> local(own.begin(), own.end());
        for (uint32_t p : own) lidx[p] = 0;
        auto add = [&](std::initializer_list<uint32_t> ks) {
            std::vector<uint32_t> extra;
            for (uint32_t k : ks)
                for (uint32_t p : parts[k])
                    if (lidx[p] < 0) {
                        lidx[p] = 0;
                        extra.push_back(p);
                    }
            std::sort(extra.begin(), extra.end());
            local.insert(local.end(), extra.begin(), extra.end());
        };
        add({NC_TILE_YARN, NC_TILE_STRAIN});
        const uint32_t small = static_cast<uint32_t>(local.size());
        add({NC_TILE_CONSTRAINTS});
        for (uint32_t l = 0; l < local.size(); ++l) lidx[local[l]] = static_cast<int32_t>(l);
        if (local.size() >= 65536u) return false;
        for (uint32_t l = 0; l < own.size(); ++l) {
            owner[own[l]] = t;
            local_of[own[l]] = l;
        }
        // plan words
        uint32_t colours = 0, nitems = 0;
        for (uint32_t k = 0; k < NC_TILE_CHAINS; ++k) {
            colours += static_cast<uint32_t>(chains[k].size());
            for (const auto& its : items[k]) nitems += static_cast<uint32_t>(its.size());
        }
        std::vector<uint32_t>& w = plans[t];
        const uint32_t table_at = NC_TILE_HEADER;
        const uint32_t list_at = table_at + 2u * colours;
        const uint32_t items_at = (list_at + static_cast<uint32_t>(local.size()) + 3u) & ~3u;
        w.assign(items_at + 4u * nitems, 0u);
        w[0] = static_cast<uint32_t>(local.size());
        w[1] = static_cast<uint32_t>(own.size());
        w[2] = list_at;
        w[3] = items_at;
        w[4u + NC_TILE_CONSTRAINTS] = static_cast<uint32_t>(local.size());
        w[4u + NC_TILE_YARN] = small;
        w[4u + NC_TILE_STRAIN] = small;
        uint32_t tat = table_at, item = 0;
        for (uint32_t k = 0; k < NC_TILE_CHAINS; ++k) {
            w[8u + 2u * k] = tat;
            w[9u + 2u * k] = static_cast<uint32_t>(chains[k].size());
            for (size_t c = 0; c < chains[k].size(); ++c) {
                const TileColour& col = chains[k][c];
                const std::vector<uint32_t>& its = items[k][c];
                w[tat++] = item;
                w[tat++] = static_cast<uint32_t>(its.size()) | (col.family << 28);
                for (uint32_t rec : its) {
                    const uint2 pe = ends(col.family, rec);
                    uint32_t* o = w.data() + items_at + 4u * item++;
                    o[0] = static_cast<uint32_t>(lidx[pe.x]) | (static_cast<uint32_t>(lidx[pe.y]) << 16);
                    o[1] = rec | ((t < tiles && tile_of[pe.x] == t) ? 0x80000000u : 0u);
                    float m0 = 0.0f, m1 = 0.0f;
                    if (col.family == NC_TILE_DISTANCE) {
                        m0 = dmat[rec].x;
                        m1 = dmat[rec].y;
                    } else if (col.family == NC_TILE_BEND) {
                        m0 = bmat[rec].x;
                        m1 = bmat[rec].y;
                    } else if (col.family == NC_TILE_LIMIT) {
                        m0 = dmat[rec].x;
                        m1 = dmat[rec].w;
                    }
                    std::memcpy(o + 2, &m0, 4);
                    std::memcpy(o + 3, &m1, 4);
                }
            }
        }
        for (uint32_t l = 0; l < local.size(); ++l) w[list_at + l] = local[l];
        for (uint32_t p : local) lidx[p] = -1;
        widest = std::max(widest, w.size() * 4u + local.size() * sizeof(float4));
    }
    // the fruit CTA holds its fruit state and the staged friction sweep
    const size_t smem = std::max(nc_resident_offset() + sizeof(FrictionStage), nc_fruit_offset() + widest);
    if (smem > smem_budget) return false;
    std::vector<uint32_t> off(R + 1u, 0u), words;
    for (uint32_t t = 0; t < R; ++t) {
        words.insert(words.end(), plans[t].begin(), plans[t].end());
        off[t + 1u] = static_cast<uint32_t>(words.size());
    }
    std::vector<uint32_t> owner_word(n);
    for (uint32_t i = 0; i < n; ++i) owner_word[i] = (owner[i] << 16) | local_of[i];
    DeviceCloth& dd = h->d;
    if (dd.x_alt == nullptr) {
        dd.x_alt = h->buf.alloc<float4>(n);
        dd.v_alt = h->buf.alloc<float4>(n);
        dd.tile_owner = h->buf.alloc<uint32_t>(n);
        dd.tile_off = h->buf.alloc<uint32_t>(R + 1u);
    }
    // the words are replaced on a rebuild (their size can change)
    uint32_t* dw = h->buf.alloc<uint32_t>(words.size());
    if (!dd.x_alt || !dd.v_alt || !dd.tile_owner || !dd.tile_off || !dw) return false;
    if (cudaMemcpy(const_cast<uint32_t*>(dd.tile_owner), owner_word.data(), n * sizeof(uint32_t),
                   cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(const_cast<uint32_t*>(dd.tile_off), off.data(), off.size() * sizeof(uint32_t),
                   cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(dw, words.data(), words.size() * sizeof(uint32_t), cudaMemcpyHostToDevice) != cudaSuccess)
        return false;
    dd.tile_words = dw;
    h->tile_smem = smem;
    return true;
}

// Rebuild the tile plan from the device records (after a material change).
bool rebuild_tiles(numi_cloth* h) {
    const DeviceCloth& d = h->d;
    std::vector<uint2> dij(d.d_count);
    std::vector<float4> dmat(d.d_count);
    std::vector<uint4> bij(d.b_count);
    std::vector<float2> bmat(d.b_count);
    if (cudaStreamSynchronize(h->stream) != cudaSuccess ||
        (d.d_count && (cudaMemcpy(dij.data(), d.d_ij, d.d_count * sizeof(uint2), cudaMemcpyDeviceToHost) != cudaSuccess ||
                       cudaMemcpy(dmat.data(), d.d_mat, d.d_count * sizeof(float4), cudaMemcpyDeviceToHost) != cudaSuccess)) ||
        (d.b_count && (cudaMemcpy(bij.data(), d.b_ij, d.b_count * sizeof(uint4), cudaMemcpyDeviceToHost) != cudaSuccess ||
                       cudaMemcpy(bmat.data(), d.b_mat, d.b_count * sizeof(float2), cudaMemcpyDeviceToHost) != cudaSuccess)))
        return false;
    int max_optin = 0;
    cudaDeviceGetAttribute(&max_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, h->device);
    cudaFuncAttributes fa{};
    cudaFuncGetAttributes(&fa, frame_fn(false, h->self_exact));
    return build_tiles(h, d.grid_width, dij, dmat, bij, bmat, static_cast<size_t>(max_optin) - fa.sharedSizeBytes);
}

// A launch runs in tile mode when the cloth has tile plans and the
// schedule is one the tile substep covers.
bool tile_schedule(const numi_cloth* h, const Schedule& s) {
    return h->tiles && s.iterations == 1u && s.aerodynamics == 0u && s.swept_fruit_yarn == 0u &&
           s.primitive_self == 0u && s.reconcile_passes == 0u && s.final_passes == 0u && s.certificate_passes == 0u;
}

cudaError_t launch(numi_cloth* h, uint32_t substeps, const Schedule& s, uint32_t cfg_offset = 0) {
    DeviceCloth d = h->d;
    d.cfg = h->d_cfg + cfg_offset;
    d.epoch_base = h->epoch;
    Schedule sc = s;
    sc.substeps = substeps;
    void* args[] = {&d, &sc};
    const bool edge = sc.primitive_self != 0u && d.edge_count != nullptr;
    if (d.trace != nullptr && substeps > h->trace_capacity) d.trace = nullptr;
    if (d.trace == nullptr) d.trace_cta = nullptr;
    cudaError_t e = cudaMemsetAsync(h->d.bar_count, 0, kBarrierWords * sizeof(unsigned long long), h->stream);
    if (e != cudaSuccess) return e;
    h->last_substeps = substeps;
    size_t smem = h->smem;
    if (edge) {
        // the edge/edge phases' box-tree sort keys after the launch's own
        // shared memory, where the device has room
        int max_optin = 0;
        cudaDeviceGetAttribute(&max_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, h->device);
        cudaFuncAttributes fe{};
        cudaFuncGetAttributes(&fe, frame_fn(true, h->self_exact));
        const size_t at = nc_round256(smem);
        if (at + NC_EDGE_TREE_KEY_BYTES + fe.sharedSizeBytes <= static_cast<size_t>(max_optin) &&
            raise_smem(frame_fn(true, h->self_exact), at + NC_EDGE_TREE_KEY_BYTES) == cudaSuccess) {
            sc.tree_keys = static_cast<uint32_t>(at);
            smem = at + NC_EDGE_TREE_KEY_BYTES;
        }
        cudaGetLastError();
    }
    if (h->cluster > 0) {
        cudaLaunchConfig_t cfg{};
        cfg.gridDim = dim3(h->cluster);
        cfg.blockDim = dim3(h->block);
        cfg.dynamicSmemBytes = smem;
        cfg.stream = h->stream;
        cudaLaunchAttribute attr{};
        attr.id = cudaLaunchAttributeClusterDimension;
        attr.val.clusterDim.x = h->cluster;
        attr.val.clusterDim.y = 1;
        attr.val.clusterDim.z = 1;
        cfg.attrs = &attr;
        cfg.numAttrs = 1;
        d.cluster_barrier = 1u;
        e = cudaLaunchKernelExC(&cfg, frame_fn(edge, h->self_exact), args);
    } else if (h->grid == 1) {
        e = cudaLaunchKernel(frame_fn(edge, h->self_exact), dim3(1), dim3(h->block), args, smem, h->stream);
    } else if (tile_schedule(h, sc)) {
        if (h->tiles_dirty) {
            if (!rebuild_tiles(h)) return cudaErrorUnknown;
            h->tiles_dirty = false;
            d.tile_words = h->d.tile_words;
        }
        sc.tiles = 1u;
        if (h->tile_grid > h->grid) d.trace_cta = nullptr;
        e = raise_frame_smem(h->tile_smem);
        if (e == cudaSuccess)
            e = cudaLaunchCooperativeKernel(frame_fn(false, h->self_exact), dim3(h->tile_grid), dim3(h->tile_block), args,
                                            h->tile_smem, h->stream);
        h->last_grid = h->tile_grid;
        h->last_block = h->tile_block;
        h->last_tiles = true;
        if (e == cudaSuccess) ++h->launches;
        return e;
    } else {
        // neighbour syncs between colours (the kernel without the edge/edge
        // phases; its flags start at zero in every launch)
        if (h->neighbours && !edge) {
            d.nbr_on = 1u;
            e = cudaMemsetAsync(d.nbr_flag, 0, NC_NBR_FLAG_STRIDE * h->grid * sizeof(unsigned int), h->stream);
            if (e != cudaSuccess) return e;
        }
        e = cudaLaunchCooperativeKernel(frame_fn(edge, h->self_exact), dim3(h->grid), dim3(h->block), args,
                                        d.nbr_on ? h->nbr_smem : smem, h->stream);
    }
    h->last_grid = h->cluster > 0 ? h->cluster : h->grid;
    h->last_block = h->block;
    h->last_tiles = false;
    if (e == cudaSuccess) ++h->launches;
    return e;
}

Schedule device_schedule(const NumiClothSchedule& schedule) {
    Schedule s{};
    s.iterations = schedule.iterations;
    s.strain_sweeps = schedule.strainSweeps;
    s.reconcile_passes = schedule.reconcilePasses;
    s.final_passes = schedule.finalPasses;
    s.certificate_passes = schedule.certificatePasses;
    s.early_exit = schedule.earlyExit;
    s.self_collision = schedule.selfCollision;
    s.aerodynamics = schedule.aerodynamics;
    s.swept_ground = schedule.sweptGround;
    s.swept_fruit_yarn = schedule.sweptFruitYarn;
    s.frictions = schedule.frictions;
    s.release = schedule.release;
    s.damping = schedule.damping;
    s.primitive_self = schedule.primitiveSelf;
    return s;
}

// Point self-contact grid of a cloth, allocated on first use (about two
// buckets per particle); the bucket heads are cleared when the 26-bit
// substep part of their tags wraps within the next `substeps`.
int prepare_self_grid(numi_cloth* h, bool self_collision, uint32_t substeps) {
    if (self_collision && h->d.hash_head == nullptr) {
        uint32_t buckets = 1024u;
        while (buckets < 2u * h->d.n) buckets <<= 1;
        DeviceCloth& d = h->d;
        d.hash_head = h->buf.alloc<unsigned long long>(buckets);
        d.hash_over_head = h->buf.alloc<unsigned long long>(1);
        d.hash_over = h->buf.alloc<HashSlot>(h->d.n);
        d.hash = h->buf.alloc<HashSlot>(static_cast<size_t>(buckets) * NC_HASH_CAP);
        d.self_stats = h->buf.alloc<unsigned long long>(8);
        // the ordered pass's list: room for three pairs per particle (a
        // power of two, at least 4,096); scratch of three words per listed
        // pair (sort keys, or the wavefront form's keys, predecessors and
        // waves) plus one turn's partners
        uint32_t list_cap = 4096u;
        while (list_cap < 3u * h->d.n) list_cap <<= 1;
        bool order_ok = true;
        if (h->self_exact) {
            d.self_list = h->buf.alloc<float4>(2u * static_cast<size_t>(list_cap));
            d.self_list_head = h->buf.alloc<unsigned long long>(1);
            d.self_pass_stats = h->buf.alloc<unsigned long long>(2);
            d.self_keys = h->buf.alloc<unsigned long long>(3u * static_cast<size_t>(list_cap) + NC_SELF_GROUP);
            d.self_mark = h->buf.alloc<unsigned long long>(h->d.n);
            d.self_x0 = h->buf.alloc<float4>(h->d.n);
            d.self_disp = h->buf.alloc<float>(h->d.n);
            order_ok = d.self_list != nullptr && d.self_list_head != nullptr && d.self_pass_stats != nullptr &&
                       d.self_keys != nullptr && d.self_mark != nullptr && d.self_x0 != nullptr &&
                       d.self_disp != nullptr;
        }
        if (d.hash_head == nullptr || d.hash == nullptr || d.self_stats == nullptr || d.hash_over_head == nullptr ||
            d.hash_over == nullptr || !order_ok) {
            d.hash_head = nullptr;
            return NUMI_CLOTH_ENOMEM;
        }
        d.self_list_cap = list_cap;
        d.self_key_cap = list_cap;
        d.hash_mask = buckets - 1u;
    }
    if (h->d.hash_head != nullptr && ((h->epoch + substeps) >> 26) != (h->epoch >> 26)) {
        if (cudaMemsetAsync(h->d.hash_head, 0, (static_cast<size_t>(h->d.hash_mask) + 1u) * sizeof(unsigned long long),
                            h->stream) != cudaSuccess ||
            cudaMemsetAsync(h->d.hash_over_head, 0, sizeof(unsigned long long), h->stream) != cudaSuccess ||
            (h->self_exact &&
             (cudaMemsetAsync(h->d.self_list_head, 0, sizeof(unsigned long long), h->stream) != cudaSuccess ||
              cudaMemsetAsync(h->d.self_mark, 0, static_cast<size_t>(h->d.n) * sizeof(unsigned long long),
                              h->stream) != cudaSuccess)))
            return NUMI_CLOTH_ECUDA;
    }
    return NUMI_CLOTH_OK;
}

// Edge/edge buffers of a cloth, allocated on first use: a build grid of
// about four buckets per yarn segment with room for 27 cells per segment, 32
// listed pairs and 16 candidate pairs per segment.  The build cell is a
// median yarn segment plus the yarn diameter and skin (three diameters), so
// that a typical segment's grown box spans at most two cells a side.
// Every yarn segment's local segments of higher index, ascending: the pairs
// the edge/edge family skips (edgePairLocal, tools/cloth_bag.cpp:2740-2749:
// some endpoint of one is local to some endpoint of the other, by the 2-hop
// topology list or, on a row-major grid cloth, the 5 x 5 block).
bool build_local_lists(const numi_cloth* h, std::vector<uint32_t>& off, std::vector<uint32_t>& idx) {
    const DeviceCloth& d = h->d;
    const std::vector<uint2>& y = h->host_yarn;
    const bool csr = !h->host_local_off.empty();
    auto local = [&](uint32_t a, uint32_t b) {
        if (csr) {
            const uint32_t* lo = h->host_local_idx.data() + h->host_local_off[a];
            const uint32_t* hi = h->host_local_idx.data() + h->host_local_off[a + 1u];
            return std::binary_search(lo, hi, b);
        }
        if (d.grid_width == 0u) return a == b;
        const int ra = static_cast<int>(a / d.grid_width), ca = static_cast<int>(a % d.grid_width);
        const int rb = static_cast<int>(b / d.grid_width), cb = static_cast<int>(b % d.grid_width);
        return std::abs(ra - rb) <= 2 && std::abs(ca - cb) <= 2;
    };
    // segments at each particle
    std::vector<uint32_t> at_off(d.n + 1u, 0u), at(2u * y.size());
    for (const uint2& s : y) {
        ++at_off[s.x + 1u];
        ++at_off[s.y + 1u];
    }
    for (uint32_t p = 0; p < d.n; ++p) at_off[p + 1u] += at_off[p];
    std::vector<uint32_t> fill(at_off.begin(), at_off.end() - 1);
    for (uint32_t k = 0; k < y.size(); ++k) {
        at[fill[y[k].x]++] = k;
        at[fill[y[k].y]++] = k;
    }
    // the particles an endpoint can be local to
    std::vector<uint32_t> near;
    auto gather = [&](uint32_t a) {
        near.push_back(a);
        if (csr) {
            near.insert(near.end(), h->host_local_idx.begin() + h->host_local_off[a],
                        h->host_local_idx.begin() + h->host_local_off[a + 1u]);
        } else if (d.grid_width != 0u) {
            const int w = static_cast<int>(d.grid_width), rows = static_cast<int>((d.n + d.grid_width - 1u) / d.grid_width);
            const int ra = static_cast<int>(a / d.grid_width), ca = static_cast<int>(a % d.grid_width);
            for (int r = std::max(ra - 2, 0); r <= std::min(ra + 2, rows - 1); ++r)
                for (int c = std::max(ca - 2, 0); c <= std::min(ca + 2, w - 1); ++c) {
                    const uint32_t q = static_cast<uint32_t>(r * w + c);
                    if (q < d.n) near.push_back(q);
                }
        }
    };
    off.assign(y.size() + 1u, 0u);
    idx.clear();
    std::vector<uint32_t> cand;
    for (uint32_t i = 0; i < y.size(); ++i) {
        near.clear();
        gather(y[i].x);
        gather(y[i].y);
        cand.clear();
        for (uint32_t q : near)
            for (uint32_t k = at_off[q]; k < at_off[q + 1u]; ++k)
                if (at[k] > i) cand.push_back(at[k]);
        std::sort(cand.begin(), cand.end());
        cand.erase(std::unique(cand.begin(), cand.end()), cand.end());
        for (uint32_t j : cand)
            if (local(y[i].x, y[j].x) || local(y[i].x, y[j].y) || local(y[i].y, y[j].x) || local(y[i].y, y[j].y))
                idx.push_back(j);
        off[i + 1u] = static_cast<uint32_t>(idx.size());
    }
    return true;
}

int prepare_edge_grid(numi_cloth* h, bool primitive, uint32_t substeps, float radius) {
    (void)substeps;
    DeviceCloth& d = h->d;
    if (primitive && d.edge_count == nullptr && d.y_count > 0u) {
        uint32_t buckets = 1024u;
        while (buckets < 4u * d.y_count) buckets <<= 1;
        const uint32_t cap = std::max(1024u, 16u * d.y_count);
        const uint32_t list_cap = std::max(2048u, 32u * d.y_count);
        const uint32_t ctas = std::max<uint32_t>(h->grid, 1u);
        DeviceCloth e = d;
        e.edge_count = h->buf.alloc<uint32_t>(buckets);
        e.edge_offs = h->buf.alloc<uint32_t>(buckets);
        e.edge_chunk_total = h->buf.alloc<uint32_t>(ctas);
        e.edge_entries = h->buf.alloc<float4>(static_cast<size_t>(54u) * d.y_count);
        e.edge_giant = h->buf.alloc<uint32_t>(d.y_count);
        e.edge_bbox = h->buf.alloc<float4>(2u * d.y_count);
        std::vector<uint32_t> loc_off, loc_idx;
        build_local_lists(h, loc_off, loc_idx);
        uint32_t* d_loc_off = h->buf.alloc<uint32_t>(loc_off.size());
        uint32_t* d_loc_idx = h->buf.alloc<uint32_t>(std::max<size_t>(loc_idx.size(), 1));
        if (d_loc_off != nullptr && d_loc_idx != nullptr &&
            (cudaMemcpy(d_loc_off, loc_off.data(), loc_off.size() * sizeof(uint32_t), cudaMemcpyHostToDevice) !=
                 cudaSuccess ||
             (!loc_idx.empty() && cudaMemcpy(d_loc_idx, loc_idx.data(), loc_idx.size() * sizeof(uint32_t),
                                             cudaMemcpyHostToDevice) != cudaSuccess)))
            d_loc_off = nullptr;
        e.edge_loc_off = d_loc_off;
        e.edge_loc_idx = d_loc_idx;
        e.edge_pairs = h->buf.alloc<uint2>(list_cap);
        e.edge_xb = h->buf.alloc<float4>(d.n);
        e.edge_pb = h->buf.alloc<float4>(d.n);
        e.edge_built_radius = h->buf.alloc<float>(1);
        e.edge_sph = h->buf.alloc<float4>(d.y_count);
        e.edge_x0 = h->buf.alloc<float4>(d.n);
        e.edge_path = h->buf.alloc<float>(d.n);
        e.edge_cand = h->buf.alloc<uint4>(cap);
        e.edge_order = h->buf.alloc<unsigned long long>(cap);
        e.edge_sorted = h->buf.alloc<unsigned long long>(cap);
        e.edge_new = h->buf.alloc<EdgeRecord>(cap);
        e.edge_done = h->buf.alloc<uint32_t>(cap);
        e.edge_lv = h->buf.alloc<uint32_t>(cap);
        e.edge_level = h->buf.alloc<uint32_t>(d.n);
        e.edge_qbox_raw = h->buf.alloc<float>(6u * d.y_count);
        e.edge_tree = h->buf.alloc<uint32_t>(static_cast<size_t>(NC_EDGE_TREE_WORDS) * d.y_count);
        e.edge_centre = h->buf.alloc<float4>(2u * static_cast<size_t>(d.y_count));   // centres, last build's
        e.edge_rec = h->buf.alloc<EdgeRecord>(cap);
        e.edge_ctl = h->buf.alloc<uint32_t>(8);
        e.edge_stats = h->buf.alloc<unsigned long long>(2);
        e.edge_red = h->buf.alloc<double>(3u * ctas);
        if (!e.edge_count || !e.edge_offs || !e.edge_chunk_total || !e.edge_entries || !e.edge_giant ||
            !e.edge_pairs || !e.edge_xb || !e.edge_pb || !e.edge_built_radius || !e.edge_sph || !e.edge_x0 ||
            !e.edge_path || !e.edge_cand || !e.edge_order || !e.edge_sorted || !e.edge_new || !e.edge_done || !e.edge_rec ||
            !e.edge_ctl || !e.edge_stats || !e.edge_red || !e.edge_lv || !e.edge_level || !e.edge_qbox_raw || !e.edge_bbox ||
            !e.edge_tree || !e.edge_centre ||
            !e.edge_loc_off || !e.edge_loc_idx)
            return NUMI_CLOTH_ENOMEM;
        e.edge_mask = buckets - 1u;
        e.edge_cap = cap;
        e.edge_list_cap = list_cap;
        d = e;
    }
    if (d.edge_count != nullptr) {
        d.edge_cell = h->yarn_rest_median + 3.0f * (2.0f * radius);
        if (const char* v = std::getenv("NUMI_CLOTH_EDGE_CELL")) {
            const float cell = std::strtof(v, nullptr);   // test hook: force long segments or crowded cells
            if (cell > 0.0f) d.edge_cell = cell;
        }
    }
    return NUMI_CLOTH_OK;
}

}  // namespace

extern "C" {

const char* numi_cloth_version(void) { return "numi-cloth-b200 0.1 (sm_100a, ABI 13)"; }

int numi_cloth_create(const NumiClothScene* scene, numi_cloth_t** out) {
    if (scene == nullptr || out == nullptr || scene->config == nullptr || scene->particles == nullptr)
        return NUMI_CLOTH_EINVAL;
    *out = nullptr;
    const NumiClothConfig& cfg = *scene->config;
    if (cfg.control.x != NUMI_CLOTH_ABI_VERSION) return NUMI_CLOTH_EINVAL;
    const uint32_t n = cfg.control.y, D = cfg.control.z, G = cfg.control.w;
    const uint32_t K = cfg.constraintCounts.x, B = cfg.constraintCounts.y, F = cfg.constraintCounts.w;
    const uint32_t P = cfg.contactCounts.x;
    if (n == 0 || F > NC_MAX_FRUITS || G > NC_MAX_GRIPS || P > NC_MAX_PAIRS) return NUMI_CLOTH_EINVAL;
    if ((D && !scene->distances) || (K && !scene->knots) || (B && !scene->bends) || (G && !scene->grips) ||
        (F && !scene->fruits) || (P && !scene->fruitPairs))
        return NUMI_CLOTH_EINVAL;
    if (validate_config(cfg, cfg) != 0u) return NUMI_CLOTH_EINVAL;
    if (cfg.gripControl.y == 1u && scene->cuffParticles == nullptr) return NUMI_CLOTH_EINVAL;

    numi_cloth* h = new (std::nothrow) numi_cloth();
    if (h == nullptr) return NUMI_CLOTH_ENOMEM;
    cudaGetDevice(&h->device);
    h->base = cfg;

    // Batches.
    int rc = make_batches(
        scene->distances, D, n, [](const NumiClothDistance& r) { return r.particlesAndColor.z; },
        [](const NumiClothDistance& r, uint32_t* w) {
            w[0] = r.particlesAndColor.x;
            w[1] = r.particlesAndColor.y;
            return w[0] == w[1] ? -1 : 2;
        },
        [](const NumiClothDistance& r) { return r.particlesAndColor.w != 3u; },
        [](const NumiClothDistance& r) { return r.material.w > 0.0f; }, h->d.dist_batches, h->d.n_dist_batches);
    if (rc == NUMI_CLOTH_OK)
        rc = make_batches(
            scene->knots, K, n, [](const NumiClothKnot& r) { return r.control.x; },
            [](const NumiClothKnot& r, uint32_t* w) {
                w[0] = r.particles.x;
                w[1] = r.particles.y;
                w[2] = r.particles.z;
                w[3] = r.particles.w;
                return 4;
            },
            [](const NumiClothKnot&) { return false; }, [](const NumiClothKnot&) { return false; },
            h->d.knot_batches, h->d.n_knot_batches);
    if (rc == NUMI_CLOTH_OK)
        rc = make_batches(
            scene->bends, B, n, [](const NumiClothBend& r) { return r.particlesAndColor.w; },
            [](const NumiClothBend& r, uint32_t* w) {
                w[0] = r.particlesAndColor.x;
                w[1] = r.particlesAndColor.z;
                return w[0] == w[1] ? -1 : 2;
            },
            [](const NumiClothBend&) { return false; }, [](const NumiClothBend&) { return false; },
            h->d.bend_batches, h->d.n_bend_batches);
    if (rc == NUMI_CLOTH_OK)
        rc = make_batches(
            scene->fruitPairs, P, F, [](const NumiClothFruitPair& r) { return r.fruitsAndColor.z; },
            [](const NumiClothFruitPair& r, uint32_t* w) {
                w[0] = r.fruitsAndColor.x;
                w[1] = r.fruitsAndColor.y;
                return w[0] == w[1] ? -1 : 2;
            },
            [](const NumiClothFruitPair&) { return false; }, [](const NumiClothFruitPair&) { return false; },
            h->d.pair_batches, h->d.n_pair_batches);
    // the middle particle of a bend is read-only but must still exist
    for (uint32_t k = 0; rc == NUMI_CLOTH_OK && k < B; ++k)
        if (scene->bends[k].particlesAndColor.y >= n) rc = NUMI_CLOTH_EINVAL;
    for (uint32_t g = 0; rc == NUMI_CLOTH_OK && g < G; ++g) {
        if (scene->grips[g].particle.x >= n) rc = NUMI_CLOTH_EINVAL;
        for (uint32_t e = 0; e < g && rc == NUMI_CLOTH_OK; ++e)
            if (scene->grips[e].particle.x == scene->grips[g].particle.x) rc = NUMI_CLOTH_EBATCH;
    }
    if (rc == NUMI_CLOTH_OK && cfg.gripControl.y == 1u)
        for (uint32_t k = 0; k < 2u * cfg.gripControl.z; ++k)
            if (scene->cuffParticles[k] >= n) rc = NUMI_CLOTH_EINVAL;
    if (rc != NUMI_CLOTH_OK) {
        delete h;
        return rc;
    }

    // Device buffers.
    DeviceCloth& d = h->d;
    d.n = n;
    d.d_count = D;
    d.k_count = K;
    d.b_count = B;
    d.g_count = G;
    d.f_count = F;
    d.p_count = P;
    d.grid_width = scene->gridWidth;
    d.damping = -1.0f;
    d.x = h->buf.alloc<float4>(n);
    d.xp = h->buf.alloc<float4>(n);
    d.v = h->buf.alloc<float4>(n);
    float4* rest = h->buf.alloc<float4>(n);
    d.rest = rest;
    uint2* d_ij = h->buf.alloc<uint2>(D);
    float4* d_mat = h->buf.alloc<float4>(D);
    d.d_ij = d_ij;
    d.d_mat = d_mat;
    d.d_lambda = h->buf.alloc<float>(D);
    uint4* k_ij = h->buf.alloc<uint4>(K);
    float2* k_mat = h->buf.alloc<float2>(K);
    d.k_ij = k_ij;
    d.k_mat = k_mat;
    d.k_lambda = h->buf.alloc<float>(K);
    uint4* b_ij = h->buf.alloc<uint4>(B);
    float2* b_mat = h->buf.alloc<float2>(B);
    d.b_ij = b_ij;
    d.b_mat = b_mat;
    d.b_lambda = h->buf.alloc<float>(B);
    d.grips = h->buf.alloc<NumiClothGrip>(G);
    d.fruits = h->buf.alloc<NumiClothFruit>(F);
    d.pairs = h->buf.alloc<NumiClothFruitPair>(P);
    uint32_t* cuff = h->buf.alloc<uint32_t>(cfg.gripControl.y == 1u ? 2u * cfg.gripControl.z : 1u);
    d.cuff = cuff;
    const uint32_t rim_count = scene->mouthRim != nullptr ? cfg.mouthControl.x : 0u;
    uint32_t* rim = h->buf.alloc<uint32_t>(rim_count);
    d.rim = rim_count >= 3u ? rim : nullptr;
    d.release = h->buf.alloc<uint32_t>(2);
    d.yarn_slot_a = h->buf.alloc<float4>(static_cast<size_t>(F ? D : 1) * NC_YARN_SLOTS);
    d.yarn_slot_b = h->buf.alloc<float4>(static_cast<size_t>(F ? D : 1) * NC_YARN_SLOTS);
    d.yarn_live = h->buf.alloc<uint32_t>(F ? D : 1);
    d.yarn_list = h->buf.alloc<uint32_t>(F ? D : 1);
    d.yarn_list_n = h->buf.alloc<uint32_t>(1);
    d.force = h->buf.alloc<float4>(n);
    d.fruit_partial = h->buf.alloc<float4>(NC_MAX_FRUITS * 9u / 2u + 1u);
    d.failure = h->buf.alloc<unsigned int>(1);
    // barrier counter (u64) and abort flag share one 16-byte block so one
    // memset resets both before a launch
    d.bar_count = h->buf.alloc<unsigned long long>(kBarrierWords);
    d.abort_flag = reinterpret_cast<unsigned int*>(d.bar_count + 1);
    d.bar_flag = d.bar_count + 16;     // 128 bytes away from the arrival counter
    d.fruit_flag = d.bar_count + 32;   // and 128 more
    d.stats = h->buf.alloc<uint32_t>(4);

    // Point self contact in the reference's Gauss-Seidel order
    // (NUMI_CLOTH_SELF_ORDER=reference): the frame kernels of
    // cloth_self_order_kernels.cu; else the batched (Jacobi) order.
    if (const char* order = std::getenv("NUMI_CLOTH_SELF_ORDER")) h->self_exact = std::strcmp(order, "reference") == 0;

    // Launch geometry: one resident CTA for a small cloth, else a full
    // cooperative grid (as many CTAs as can be co-resident).
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device);
    int per_sm = 0;
    raise_frame_smem(nc_resident_offset());
    // NUMI_CLOTH_BLOCK=512 runs the cooperative grid with 512-thread CTAs
    // (one per SM) instead of 256 (two per SM); NUMI_CLOTH_BLOCK=256 runs a
    // one-CTA cloth with 256 threads instead of 512.
    uint32_t block = NC_THREADS;
    const bool forced_block = env_u32("NUMI_CLOTH_BLOCK", block);
    if (forced_block && block != NC_BLOCK_MAX) block = NC_THREADS;
    h->block = block;
    for (bool edge : {false, true}) {
        int k = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&k, frame_fn(edge, h->self_exact), static_cast<int>(block),
                                                      nc_resident_offset());
        per_sm = edge ? std::min(per_sm, k) : k;
    }
    uint32_t work = std::max({n, D, K, B});
    uint32_t grid = (work <= 8192u) ? 1u : std::min<uint32_t>(sms * std::max(per_sm, 1), (work + block - 1u) / block);
    uint32_t forced = 0;
    if (env_u32("NUMI_CLOTH_GRID", forced) && forced > 0) grid = std::min<uint32_t>(forced, sms * std::max(per_sm, 1));
    h->grid = std::max(grid, 1u);
    // one CTA holds the whole cloth: every phase is latency-bound on one SM,
    // so it runs with the most threads (16 warps instead of 8: 20 % less
    // time per frame on the produce bag)
    if (h->grid == 1u && !forced_block) h->block = NC_BLOCK_MAX;
    // NUMI_CLOTH_CLUSTER=8 or =16 runs a large cloth as one thread-block
    // cluster (hardware cluster barrier) when the device can place it; the
    // default is the cooperative grid.
    uint32_t want_cluster = 0;
    env_u32("NUMI_CLOTH_CLUSTER", want_cluster);
    // Resident mode: particle positions and velocities stay in the shared
    // memory of one CTA (n <= 4096, the default) or, with
    // NUMI_CLOTH_RESIDENT=2, of one thread-block cluster of up to 16 CTAs
    // holding 4096 particles each (n <= 65536) for the whole frame, where
    // accesses to another CTA's particles go through distributed shared
    // memory.  NUMI_CLOTH_RESIDENT=0 keeps them in global memory.  The
    // cluster form is off by default: 16 CTAs leave too few threads to hide
    // the latency of a 65,536-particle cloth's colour batches, and it
    // measured slower than the cooperative grid.
    uint32_t want_resident = 1;
    env_u32("NUMI_CLOTH_RESIDENT", want_resident);
    const uint32_t resident_limit = want_resident >= 2u ? 16u * kResidentChunk : kResidentChunk;
    // Particles each CTA of a resident cluster holds: a cloth of up to
    // 4096 particles runs on a cluster of ceil(n / 256) CTAs (up to 16),
    // which measured 1.3-1.5x faster on the 1,400-particle bag than one CTA
    // holding it all (more threads per colour batch, the same bits); with
    // NUMI_CLOTH_RESIDENT=2 each CTA holds 4096.  NUMI_CLOTH_RESIDENT_CHUNK
    // (a power of two, 64 to 4096) overrides it.
    uint32_t chunk = want_resident >= 2u ? kResidentChunk : kResidentClusterChunk;
    env_u32("NUMI_CLOTH_RESIDENT_CHUNK", chunk);
    if (chunk < 64u || chunk > kResidentChunk || (chunk & (chunk - 1u)) != 0u) chunk = kResidentChunk;
    if (want_resident != 0u && forced == 0 && n > 0u && n <= resident_limit && (n + chunk - 1u) / chunk <= 16u) {
        uint32_t shift = 4u;
        while ((1u << shift) < std::min(n, chunk)) ++shift;
        const uint32_t ranks = (n + (1u << shift) - 1u) >> shift;
        const size_t smem = nc_resident_offset() + 2u * (static_cast<size_t>(1u) << shift) * sizeof(float4);
        int max_optin = 0;
        cudaDeviceGetAttribute(&max_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, h->device);
        cudaFuncAttributes fa{}, fe{};
        cudaFuncGetAttributes(&fa, frame_fn(false, h->self_exact));
        cudaFuncGetAttributes(&fe, frame_fn(true, h->self_exact));
        bool ok = smem + std::max(fa.sharedSizeBytes, fe.sharedSizeBytes) <= static_cast<size_t>(max_optin) &&
                  raise_frame_smem(smem) == cudaSuccess;
        if (ok && ranks > 1u) {
            allow_large_clusters();
            cudaLaunchConfig_t cfg{};
            cfg.gridDim = dim3(ranks);
            cfg.blockDim = dim3(NC_BLOCK_MAX);
            cfg.dynamicSmemBytes = smem;
            cudaLaunchAttribute attr{};
            attr.id = cudaLaunchAttributeClusterDimension;
            attr.val.clusterDim.x = ranks;
            attr.val.clusterDim.y = 1;
            attr.val.clusterDim.z = 1;
            cfg.attrs = &attr;
            cfg.numAttrs = 1;
            ok = frame_clusters(cfg) >= 1;
        }
        cudaGetLastError();
        if (ok) {
            d.resident = 1u;
            d.resident_shift = shift;
            h->smem = smem;
            h->grid = ranks;
            if (ranks > 1u) {
                h->cluster = ranks;
                h->block = NC_BLOCK_MAX;
            }
            want_cluster = 0;
        }
    }
    if (h->grid > 1 && want_cluster > 0 && forced == 0) {
        allow_large_clusters();
        for (uint32_t c : {want_cluster, 8u}) {
            if (c > 16u || c < 2u) continue;
            cudaLaunchConfig_t cfg{};
            cfg.gridDim = dim3(c);
            cfg.blockDim = dim3(NC_BLOCK_MAX);
            cfg.dynamicSmemBytes = nc_resident_offset();
            cudaLaunchAttribute attr{};
            attr.id = cudaLaunchAttributeClusterDimension;
            attr.val.clusterDim.x = c;
            attr.val.clusterDim.y = 1;
            attr.val.clusterDim.z = 1;
            cfg.attrs = &attr;
            cfg.numAttrs = 1;
            if (frame_clusters(cfg) >= 1) {
                h->cluster = c;
                h->grid = c;
                h->block = NC_BLOCK_MAX;
                break;
            }
        }
        cudaGetLastError();
    }
    // Bounded waits: NUMI_CLOTH_WAIT_LIMIT sets the polls a barrier or
    // neighbour wait makes before it raises TIMEOUT (default 2^22, a few
    // seconds).  NUMI_CLOTH_TEST_MISSING_CTA=1 is a failure-path test hook:
    // every grid barrier of the cooperative grid also waits for a CTA that
    // does not exist, so the first wait runs out and the launch ends with
    // TIMEOUT.
    env_u32("NUMI_CLOTH_WAIT_LIMIT", d.spin_limit);
    env_u32("NUMI_CLOTH_TEST_MISSING_CTA", d.bar_phantom);
    if (d.bar_phantom > 1u) d.bar_phantom = 1u;
    uint32_t trace_substeps = 0;
    if (env_u32("NUMI_CLOTH_TRACE", trace_substeps) && trace_substeps > 0) {
        d.trace = h->buf.alloc<unsigned long long>(static_cast<size_t>(trace_substeps) * NC_TRACE_SLOTS);
        h->trace_capacity = d.trace ? trace_substeps : 0u;
        uint32_t per_cta = 0;
        if (env_u32("NUMI_CLOTH_TRACE_CTA", per_cta) && per_cta > 0)
            d.trace_cta = h->buf.alloc<unsigned long long>(static_cast<size_t>(trace_substeps) * NC_TRACE_SLOTS *
                                                           std::max<uint32_t>(h->grid, 1u));
    }
    const uint32_t chunks = (n + NC_THREADS - 1u) / NC_THREADS;
    d.red = h->buf.alloc<double>(std::max<size_t>(3u * 4096u, 2u * chunks + 8u));

    bool ok = d.x && d.xp && d.v && rest && d_ij && d_mat && d.d_lambda && k_ij && k_mat && d.k_lambda && b_ij &&
              b_mat && d.b_lambda && d.grips && d.fruits && d.pairs && cuff && d.yarn_slot_a && d.yarn_slot_b && d.yarn_live && d.yarn_list && d.yarn_list_n &&
              d.force && d.fruit_partial && d.failure && d.bar_count && d.abort_flag && d.stats && d.red && rim &&
              d.release;
    if (!ok) {
        delete h;
        return NUMI_CLOTH_ENOMEM;
    }

    // AoS -> SoA.
    std::vector<float4> hx(n), hxp(n), hv(n), hr(n);
    for (uint32_t i = 0; i < n; ++i) {
        const NumiClothParticle& p = scene->particles[i];
        hx[i] = make_float4(p.positionAndInverseMass.x, p.positionAndInverseMass.y, p.positionAndInverseMass.z,
                            p.positionAndInverseMass.w);
        hxp[i] = make_float4(p.previousAndMass.x, p.previousAndMass.y, p.previousAndMass.z, p.previousAndMass.w);
        hv[i] = make_float4(p.velocity.x, p.velocity.y, p.velocity.z, p.velocity.w);
        if (scene->restPositions != nullptr)
            hr[i] = make_float4(scene->restPositions[i].x, scene->restPositions[i].y, scene->restPositions[i].z, 0.0f);
        else
            hr[i] = make_float4(hx[i].x, hx[i].y, hx[i].z, 0.0f);
    }
    std::vector<uint2> hij(D);
    std::vector<float4> hdm(D);
    std::vector<float> hdl(D);
    for (uint32_t k = 0; k < D; ++k) {
        const NumiClothDistance& r = scene->distances[k];
        hij[k] = make_uint2(r.particlesAndColor.x, r.particlesAndColor.y);
        hdm[k] = make_float4(r.material.x, r.material.y, 0.0f, r.material.w);
        hdl[k] = r.material.z;
    }
    std::vector<uint4> hkij(K);
    std::vector<float2> hkm(K);
    std::vector<float> hkl(K);
    for (uint32_t k = 0; k < K; ++k) {
        const NumiClothKnot& r = scene->knots[k];
        hkij[k] = make_uint4(r.particles.x, r.particles.y, r.particles.z, r.particles.w);
        hkm[k] = make_float2(r.material.x, r.material.y);
        hkl[k] = r.material.z;
    }
    std::vector<uint4> hbij(B);
    std::vector<float2> hbm(B);
    std::vector<float> hbl(B);
    for (uint32_t k = 0; k < B; ++k) {
        const NumiClothBend& r = scene->bends[k];
        hbij[k] = make_uint4(r.particlesAndColor.x, r.particlesAndColor.y, r.particlesAndColor.z, 0u);
        hbm[k] = make_float2(r.material.x, r.material.z);
        hbl[k] = r.material.w;
    }
    cudaError_t e = cudaSuccess;
    auto up = [&](void* dst, const void* src, size_t bytes) {
        if (e == cudaSuccess && bytes) e = cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice);
    };
    up(d.x, hx.data(), n * sizeof(float4));
    up(d.xp, hxp.data(), n * sizeof(float4));
    up(d.v, hv.data(), n * sizeof(float4));
    up(rest, hr.data(), n * sizeof(float4));
    up(d_ij, hij.data(), D * sizeof(uint2));
    {
        // yarn segments: the distances that are not shear diagonals, in array order
        std::vector<uint2> hy;
        std::vector<float> rest_lengths;
        for (uint32_t k = 0; k < D; ++k) {
            const NumiClothDistance& r = scene->distances[k];
            if (r.particlesAndColor.w == 3u) continue;
            hy.push_back(make_uint2(r.particlesAndColor.x, r.particlesAndColor.y));
            rest_lengths.push_back(r.material.x);
        }
        if (!rest_lengths.empty()) {
            std::nth_element(rest_lengths.begin(), rest_lengths.begin() + rest_lengths.size() / 2, rest_lengths.end());
            h->yarn_rest_median = rest_lengths[rest_lengths.size() / 2];
        }
        uint2* y_ij = h->buf.alloc<uint2>(hy.size());
        if (y_ij == nullptr && e == cudaSuccess) e = cudaErrorMemoryAllocation;
        d.y_ij = y_ij;
        d.y_count = static_cast<uint32_t>(hy.size());
        up(y_ij, hy.data(), hy.size() * sizeof(uint2));
        h->host_yarn = hy;
    }
    up(d_mat, hdm.data(), D * sizeof(float4));
    up(d.d_lambda, hdl.data(), D * sizeof(float));
    up(k_ij, hkij.data(), K * sizeof(uint4));
    up(k_mat, hkm.data(), K * sizeof(float2));
    up(d.k_lambda, hkl.data(), K * sizeof(float));
    up(b_ij, hbij.data(), B * sizeof(uint4));
    up(b_mat, hbm.data(), B * sizeof(float2));
    up(d.b_lambda, hbl.data(), B * sizeof(float));
    up(d.grips, scene->grips, G * sizeof(NumiClothGrip));
    up(d.fruits, scene->fruits, F * sizeof(NumiClothFruit));
    up(d.pairs, scene->fruitPairs, P * sizeof(NumiClothFruitPair));
    if (cfg.gripControl.y == 1u) up(cuff, scene->cuffParticles, 2u * cfg.gripControl.z * sizeof(uint32_t));
    if (rim_count > 0u) up(rim, scene->mouthRim, rim_count * sizeof(uint32_t));
    if (scene->localOffsets != nullptr && scene->localIndices != nullptr) {
        // 2-hop topology CSR of the point self-contact exclusion
        const uint32_t entries = scene->localOffsets[n];
        uint32_t* off = h->buf.alloc<uint32_t>(n + 1u);
        uint32_t* idx = h->buf.alloc<uint32_t>(entries);
        if (off == nullptr || idx == nullptr) {
            delete h;
            return NUMI_CLOTH_ENOMEM;
        }
        up(off, scene->localOffsets, (n + 1u) * sizeof(uint32_t));
        up(idx, scene->localIndices, entries * sizeof(uint32_t));
        h->host_local_off.assign(scene->localOffsets, scene->localOffsets + n + 1u);
        h->host_local_idx.assign(scene->localIndices, scene->localIndices + entries);
        d.local_off = off;
        d.local_idx = idx;
    }
    if (e != cudaSuccess) {
        delete h;
        return NUMI_CLOTH_ECUDA;
    }
    h->neighbours = prepare_neighbours(h, scene);
    // Tile mode of the cooperative grid (cloth_tile.cuh): one 512-thread CTA
    // per SM, used by the launches whose schedule it covers;
    // on by default; NUMI_CLOTH_TILES=0 keeps the colour-by-colour schedule.
    uint32_t want_tiles = 1;
    env_u32("NUMI_CLOTH_TILES", want_tiles);
    if (want_tiles != 0u && h->grid > 1u && h->cluster == 0u && d.resident == 0u && K == 0u) {
        int max_optin = 0;
        cudaDeviceGetAttribute(&max_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, h->device);
        cudaFuncAttributes fa{};
        cudaFuncGetAttributes(&fa, frame_fn(false, h->self_exact));
        uint32_t tgrid = static_cast<uint32_t>(sms);
        env_u32("NUMI_CLOTH_TILE_GRID", tgrid);
        h->tile_grid = std::max(tgrid, 3u);
        h->tile_block = NC_BLOCK_MAX;
        h->tiles = build_tiles(h, scene->gridWidth, hij, hdm, hbij, hbm,
                               static_cast<size_t>(max_optin) - fa.sharedSizeBytes);
        if (h->tiles) {
            int k = 0;
            h->tiles = raise_frame_smem(h->tile_smem) == cudaSuccess &&
                       cudaOccupancyMaxActiveBlocksPerMultiprocessor(&k, frame_fn(false, h->self_exact), NC_BLOCK_MAX,
                                                                     h->tile_smem) == cudaSuccess &&
                       static_cast<uint64_t>(k) * static_cast<uint64_t>(sms) >= h->tile_grid;
        }
        cudaGetLastError();
    }
    h->dynamic = {{d.x, n * sizeof(float4)},
                  {d.xp, n * sizeof(float4)},
                  {d.v, n * sizeof(float4)},
                  {d.d_lambda, std::max<size_t>(D, 1) * sizeof(float)},
                  {d.k_lambda, std::max<size_t>(K, 1) * sizeof(float)},
                  {d.b_lambda, std::max<size_t>(B, 1) * sizeof(float)},
                  {d.grips, std::max<size_t>(G, 1) * sizeof(NumiClothGrip)},
                  {d.fruits, std::max<size_t>(F, 1) * sizeof(NumiClothFruit)},
                  {d.pairs, std::max<size_t>(P, 1) * sizeof(NumiClothFruitPair)},
                  {d.release, 2u * sizeof(uint32_t)}};
    *out = h;
    return NUMI_CLOTH_OK;
}

void numi_cloth_destroy(numi_cloth_t* h) {
    if (h == nullptr) return;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    for (auto& s : h->snaps)
        if (s.mem) cudaFree(s.mem);
    cudaFree(h->d_cfg);
    delete h;
}

int numi_cloth_set_damping(numi_cloth_t* h, float damping) {
    if (h == nullptr || !std::isfinite(damping)) return NUMI_CLOTH_EINVAL;
    h->d.damping = damping < 0.0f ? -1.0f : damping;
    return NUMI_CLOTH_OK;
}

int numi_cloth_set_stream(numi_cloth_t* h, void* stream) {
    if (h == nullptr) return NUMI_CLOTH_EINVAL;
    h->stream = static_cast<cudaStream_t>(stream);
    return NUMI_CLOTH_OK;
}

int numi_cloth_step(numi_cloth_t* h, const NumiClothConfig* configs, uint32_t count,
                    const NumiClothSchedule* schedule) {
    if (h == nullptr || configs == nullptr || schedule == nullptr || count == 0) return NUMI_CLOTH_EINVAL;
    if (h->poisoned) return NUMI_CLOTH_ESTATE;
    cudaSetDevice(h->device);
    for (uint32_t k = 0; k < count; ++k) {
        const uint32_t bad = validate_config(configs[k], h->base);
        if (bad) {
            h->host_failure |= bad;
            return NUMI_CLOTH_OK;   // the failure word reports it; nothing ran
        }
    }
    if (count > h->cfg_capacity) {
        cudaFree(h->d_cfg);
        h->d_cfg = nullptr;
        if (cudaMalloc(&h->d_cfg, count * sizeof(NumiClothConfig)) != cudaSuccess) return NUMI_CLOTH_ECUDA;
        h->cfg_capacity = count;
    }
    if (cudaMemcpyAsync(h->d_cfg, configs, count * sizeof(NumiClothConfig), cudaMemcpyHostToDevice, h->stream) !=
        cudaSuccess)
        return NUMI_CLOTH_ECUDA;
    const Schedule s = device_schedule(*schedule);
    int rc = prepare_self_grid(h, s.self_collision != 0u, count);
    if (rc == NUMI_CLOTH_OK) rc = prepare_edge_grid(h, s.primitive_self != 0u, count, configs[0].clothMaterial.x);
    if (rc != NUMI_CLOTH_OK) return rc;
    const cudaError_t e = launch(h, count, s);
    h->epoch += count;
    if (e != cudaSuccess) {
        h->poisoned = true;
        return NUMI_CLOTH_ECUDA;
    }
    return NUMI_CLOTH_OK;
}

uint32_t numi_cloth_failure(numi_cloth_t* h) {
    if (h == nullptr) return NUMI_CLOTH_FAILURE_RANGE;
    cudaSetDevice(h->device);
    uint32_t f = 0;
    if (cudaStreamSynchronize(h->stream) != cudaSuccess ||
        cudaMemcpy(&f, h->d.failure, sizeof(f), cudaMemcpyDeviceToHost) != cudaSuccess) {
        h->poisoned = true;
        return h->host_failure | NUMI_CLOTH_FAILURE_RANGE;
    }
    return f | h->host_failure;
}

// Particle records <-> the state arrays (x, previous, v), one thread per
// particle: coalesced 16-byte loads and stores on both sides.
__global__ void numi_cloth_unpack_particles_kernel(const NumiClothParticle* in, float4* x, float4* xp, float4* v,
                                                   uint32_t n) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4* r = reinterpret_cast<const float4*>(in + i);
        x[i] = __ldcs(r);
        xp[i] = __ldcs(r + 1);
        v[i] = __ldcs(r + 2);
    }
}

__global__ void numi_cloth_pack_particles_kernel(const float4* x, const float4* xp, const float4* v,
                                                 NumiClothParticle* out, uint32_t n) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float4* r = reinterpret_cast<float4*>(out + i);
        __stcs(r, x[i]);
        __stcs(r + 1, xp[i]);
        __stcs(r + 2, v[i]);
    }
}

static_assert(sizeof(NumiClothParticle) == 3u * sizeof(float4), "particle record: three float4 words");

// The handle's staging buffer for particle records, allocated on first use.
static NumiClothParticle* particle_io(numi_cloth_t* h) {
    if (h->io == nullptr) h->io = h->buf.alloc<NumiClothParticle>(h->d.n);
    return h->io;
}

int numi_cloth_read_particles(numi_cloth_t* h, NumiClothParticle* out, uint32_t count) {
    if (h == nullptr || out == nullptr || count != h->d.n) return NUMI_CLOTH_EINVAL;
    cudaSetDevice(h->device);
    NumiClothParticle* io = particle_io(h);
    if (io == nullptr) return NUMI_CLOTH_ECUDA;
    const uint32_t blocks = std::min<uint32_t>((count + 255u) / 256u, 1184u);
    numi_cloth_pack_particles_kernel<<<blocks, 256, 0, h->stream>>>(h->d.x, h->d.xp, h->d.v, io, count);
    if (cudaGetLastError() != cudaSuccess ||
        cudaMemcpyAsync(out, io, count * sizeof(NumiClothParticle), cudaMemcpyDeviceToHost, h->stream) !=
            cudaSuccess ||
        cudaStreamSynchronize(h->stream) != cudaSuccess)
        return NUMI_CLOTH_ECUDA;
    return NUMI_CLOTH_OK;
}

int numi_cloth_write_particles(numi_cloth_t* h, const NumiClothParticle* in, uint32_t count) {
    if (h == nullptr || in == nullptr || count != h->d.n) return NUMI_CLOTH_EINVAL;
    cudaSetDevice(h->device);
    NumiClothParticle* io = particle_io(h);
    if (io == nullptr) return NUMI_CLOTH_ECUDA;
    const uint32_t blocks = std::min<uint32_t>((count + 255u) / 256u, 1184u);
    if (cudaMemcpyAsync(io, in, count * sizeof(NumiClothParticle), cudaMemcpyHostToDevice, h->stream) !=
        cudaSuccess)
        return NUMI_CLOTH_ECUDA;
    numi_cloth_unpack_particles_kernel<<<blocks, 256, 0, h->stream>>>(io, h->d.x, h->d.xp, h->d.v, count);
    // synchronous: the caller may reuse its buffer on return
    if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(h->stream) != cudaSuccess)
        return NUMI_CLOTH_ECUDA;
    return NUMI_CLOTH_OK;
}

static int copy_records(numi_cloth_t* h, void* dst, const void* src, size_t bytes, cudaMemcpyKind kind) {
    cudaSetDevice(h->device);
    if (cudaStreamSynchronize(h->stream) != cudaSuccess) return NUMI_CLOTH_ECUDA;
    if (bytes && cudaMemcpy(dst, src, bytes, kind) != cudaSuccess) return NUMI_CLOTH_ECUDA;
    return NUMI_CLOTH_OK;
}

int numi_cloth_read_fruits(numi_cloth_t* h, NumiClothFruit* out, uint32_t count) {
    if (h == nullptr || (out == nullptr && count) || count != h->d.f_count) return NUMI_CLOTH_EINVAL;
    return copy_records(h, out, h->d.fruits, count * sizeof(NumiClothFruit), cudaMemcpyDeviceToHost);
}

int numi_cloth_write_fruits(numi_cloth_t* h, const NumiClothFruit* in, uint32_t count) {
    if (h == nullptr || (in == nullptr && count) || count != h->d.f_count) return NUMI_CLOTH_EINVAL;
    return copy_records(h, h->d.fruits, in, count * sizeof(NumiClothFruit), cudaMemcpyHostToDevice);
}

int numi_cloth_read_grips(numi_cloth_t* h, NumiClothGrip* out, uint32_t count) {
    if (h == nullptr || (out == nullptr && count) || count != h->d.g_count) return NUMI_CLOTH_EINVAL;
    return copy_records(h, out, h->d.grips, count * sizeof(NumiClothGrip), cudaMemcpyDeviceToHost);
}

int numi_cloth_read_distances(numi_cloth_t* h, NumiClothDistance* out, uint32_t count) {
    if (h == nullptr || out == nullptr || count != h->d.d_count) return NUMI_CLOTH_EINVAL;
    std::vector<uint2> ij(count);
    std::vector<float4> m(count);
    std::vector<float> l(count);
    int rc = copy_records(h, ij.data(), h->d.d_ij, count * sizeof(uint2), cudaMemcpyDeviceToHost);
    if (rc == NUMI_CLOTH_OK) rc = copy_records(h, m.data(), h->d.d_mat, count * sizeof(float4), cudaMemcpyDeviceToHost);
    if (rc == NUMI_CLOTH_OK) rc = copy_records(h, l.data(), h->d.d_lambda, count * sizeof(float), cudaMemcpyDeviceToHost);
    if (rc != NUMI_CLOTH_OK) return rc;
    for (uint32_t k = 0; k < count; ++k) {
        out[k].particlesAndColor.x = ij[k].x;
        out[k].particlesAndColor.y = ij[k].y;
        out[k].material = {m[k].x, m[k].y, l[k], m[k].w};
    }
    return NUMI_CLOTH_OK;
}

int numi_cloth_residuals(numi_cloth_t* h, double out[4]) {
    if (h == nullptr || out == nullptr) return NUMI_CLOTH_EINVAL;
    cudaSetDevice(h->device);
    const uint32_t grid = std::max<uint32_t>(1u, std::min<uint32_t>(h->grid, 4096u));
    DeviceCloth d = h->d;
    NumiClothConfig cfg = h->base;
    numi_cloth_residual_kernel<<<grid, NC_THREADS, 0, h->stream>>>(d, cfg);
    std::vector<double> r(3u * grid);
    if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(h->stream) != cudaSuccess ||
        cudaMemcpy(r.data(), d.red, r.size() * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
        return NUMI_CLOTH_ECUDA;
    out[0] = out[1] = out[2] = out[3] = 0.0;
    for (uint32_t b = 0; b < grid; ++b)
        for (int e = 0; e < 3; ++e) out[e] = std::max(out[e], r[3u * b + e]);
    return NUMI_CLOTH_OK;
}

int numi_cloth_self_contacts(numi_cloth_t* h, unsigned long long* contacts, double* max_penetration) {
    if (h == nullptr || contacts == nullptr || max_penetration == nullptr) return NUMI_CLOTH_EINVAL;
    *contacts = 0ull;
    *max_penetration = 0.0;
    if (h->d.self_stats == nullptr) return NUMI_CLOTH_OK;
    cudaSetDevice(h->device);
    unsigned long long st[2] = {0ull, 0ull};
    if (cudaStreamSynchronize(h->stream) != cudaSuccess ||
        cudaMemcpy(st, h->d.self_stats, sizeof(st), cudaMemcpyDeviceToHost) != cudaSuccess)
        return NUMI_CLOTH_ECUDA;
    *contacts = st[0];
    float pen = 0.0f;
    const uint32_t bits = static_cast<uint32_t>(st[1]);
    std::memcpy(&pen, &bits, sizeof(pen));
    *max_penetration = pen;
    return NUMI_CLOTH_OK;
}

int numi_cloth_self_order_stats(numi_cloth_t* h, unsigned long long out[4]) {
    if (h == nullptr || out == nullptr) return NUMI_CLOTH_EINVAL;
    for (int k = 0; k < 4; ++k) out[k] = 0ull;
    if (h->d.self_stats == nullptr) return NUMI_CLOTH_OK;
    cudaSetDevice(h->device);
    if (cudaStreamSynchronize(h->stream) != cudaSuccess ||
        cudaMemcpy(out, h->d.self_stats + 2, 4 * sizeof(unsigned long long), cudaMemcpyDeviceToHost) != cudaSuccess)
        return NUMI_CLOTH_ECUDA;
    return NUMI_CLOTH_OK;
}

int numi_cloth_edge_contacts(numi_cloth_t* h, unsigned long long out[2]) {
    if (h == nullptr || out == nullptr) return NUMI_CLOTH_EINVAL;
    out[0] = out[1] = 0ull;
    if (h->d.edge_stats == nullptr) return NUMI_CLOTH_OK;
    cudaSetDevice(h->device);
    if (cudaStreamSynchronize(h->stream) != cudaSuccess ||
        cudaMemcpy(out, h->d.edge_stats, 2u * sizeof(unsigned long long), cudaMemcpyDeviceToHost) != cudaSuccess)
        return NUMI_CLOTH_ECUDA;
    return NUMI_CLOTH_OK;
}

int numi_cloth_release_masks(numi_cloth_t* h, uint32_t out[2]) {
    if (h == nullptr || out == nullptr) return NUMI_CLOTH_EINVAL;
    out[0] = out[1] = 0u;
    cudaSetDevice(h->device);
    if (cudaStreamSynchronize(h->stream) != cudaSuccess ||
        cudaMemcpy(out, h->d.release, 2u * sizeof(uint32_t), cudaMemcpyDeviceToHost) != cudaSuccess)
        return NUMI_CLOTH_ECUDA;
    return NUMI_CLOTH_OK;
}

namespace {
int snapshot_slot(numi_cloth_t* h, uint32_t slot);
int restore_slot(numi_cloth_t* h, uint32_t slot);
}  // namespace

int numi_cloth_snapshot(numi_cloth_t* h, uint32_t slot) {
    if (h == nullptr || slot >= kSnapshotSlots) return NUMI_CLOTH_EINVAL;
    return snapshot_slot(h, slot);
}

int numi_cloth_restore(numi_cloth_t* h, uint32_t slot) {
    if (h == nullptr || slot >= kSnapshotSlots || !h->snaps[slot].valid) return NUMI_CLOTH_EINVAL;
    return restore_slot(h, slot);
}

}  // extern "C"

namespace {
int snapshot_slot(numi_cloth_t* h, uint32_t slot) {
    cudaSetDevice(h->device);
    size_t total = 0;
    for (const auto& r : h->dynamic) total += (r.bytes + 255u) & ~size_t(255u);
    Snapshot& s = h->snaps[slot];
    if (s.mem == nullptr) {
        if (cudaMalloc(&s.mem, total) != cudaSuccess) return NUMI_CLOTH_ENOMEM;
        s.bytes = total;
    }
    size_t off = 0;
    for (const auto& r : h->dynamic) {
        if (cudaMemcpyAsync(static_cast<char*>(s.mem) + off, r.ptr, r.bytes, cudaMemcpyDeviceToDevice, h->stream) !=
            cudaSuccess)
            return NUMI_CLOTH_ECUDA;
        off += (r.bytes + 255u) & ~size_t(255u);
    }
    s.valid = true;
    return NUMI_CLOTH_OK;
}

int restore_slot(numi_cloth_t* h, uint32_t slot) {
    cudaSetDevice(h->device);
    size_t off = 0;
    for (const auto& r : h->dynamic) {
        if (cudaMemcpyAsync(r.ptr, static_cast<char*>(h->snaps[slot].mem) + off, r.bytes, cudaMemcpyDeviceToDevice,
                            h->stream) != cudaSuccess)
            return NUMI_CLOTH_ECUDA;
        off += (r.bytes + 255u) & ~size_t(255u);
    }
    return NUMI_CLOTH_OK;
}
}  // namespace

extern "C" {

int numi_cloth_trace(numi_cloth_t* h, unsigned long long* out, uint32_t substeps, uint32_t slots) {
    if (h == nullptr || out == nullptr || slots != NC_TRACE_SLOTS) return NUMI_CLOTH_EINVAL;
    if (h->d.trace == nullptr || substeps > h->trace_capacity) return NUMI_CLOTH_ESTATE;
    cudaSetDevice(h->device);
    if (cudaStreamSynchronize(h->stream) != cudaSuccess ||
        cudaMemcpy(out, h->d.trace, static_cast<size_t>(substeps) * NC_TRACE_SLOTS * sizeof(unsigned long long),
                   cudaMemcpyDeviceToHost) != cudaSuccess)
        return NUMI_CLOTH_ECUDA;
    return NUMI_CLOTH_OK;
}

int numi_cloth_trace_cta(numi_cloth_t* h, unsigned long long* out, uint32_t substeps) {
    if (h == nullptr || out == nullptr) return NUMI_CLOTH_EINVAL;
    if (h->d.trace_cta == nullptr || substeps > h->trace_capacity) return NUMI_CLOTH_ESTATE;
    cudaSetDevice(h->device);
    // the last launch's CTAs (a tile launch may use fewer than the grid)
    const uint32_t grid = h->last_grid != 0u ? h->last_grid : h->grid;
    if (grid > h->grid) return NUMI_CLOTH_ESTATE;   // not traced per CTA
    if (cudaStreamSynchronize(h->stream) != cudaSuccess ||
        cudaMemcpy(out, h->d.trace_cta,
                   static_cast<size_t>(substeps) * NC_TRACE_SLOTS * grid * sizeof(unsigned long long),
                   cudaMemcpyDeviceToHost) != cudaSuccess)
        return NUMI_CLOTH_ECUDA;
    return NUMI_CLOTH_OK;
}

int numi_cloth_pass_counts(numi_cloth_t* h, uint32_t out[3]) {
    if (h == nullptr || out == nullptr) return NUMI_CLOTH_EINVAL;
    cudaSetDevice(h->device);
    uint32_t stats[4] = {0, 0, 0, 0};
    if (cudaStreamSynchronize(h->stream) != cudaSuccess ||
        cudaMemcpy(stats, h->d.stats, sizeof(stats), cudaMemcpyDeviceToHost) != cudaSuccess)
        return NUMI_CLOTH_ECUDA;
    out[0] = stats[0];
    out[1] = stats[1];
    out[2] = stats[2];
    return NUMI_CLOTH_OK;
}

}  // extern "C"

namespace {

// Tile plans for a tile launch of `grid` CTAs, and whether the device holds
// that grid co-resident with their shared memory.
bool configure_tiles(numi_cloth* h, uint32_t grid) {
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device);
    h->tile_grid = grid;
    h->tiles = rebuild_tiles(h);
    h->tiles_dirty = false;
    if (h->tiles) {
        int k = 0;
        h->tiles = raise_frame_smem(h->tile_smem) == cudaSuccess &&
                   cudaOccupancyMaxActiveBlocksPerMultiprocessor(&k, frame_fn(false, h->self_exact), NC_BLOCK_MAX, h->tile_smem) ==
                       cudaSuccess &&
                   static_cast<uint64_t>(k) * static_cast<uint64_t>(sms) >= h->tile_grid;
    }
    cudaGetLastError();
    return h->tiles;
}

}  // namespace

extern "C" int numi_cloth_tune(numi_cloth_t* h, const NumiClothConfig* configs, uint32_t count,
                               const NumiClothSchedule* schedule, uint32_t out[4]) {
    if (h == nullptr || configs == nullptr || schedule == nullptr || count == 0 || out == nullptr)
        return NUMI_CLOTH_EINVAL;
    if (h->poisoned) return NUMI_CLOTH_ESTATE;
    cudaSetDevice(h->device);
    if (numi_cloth_failure(h) != 0u) return NUMI_CLOTH_ESTATE;   // a failed cloth is not timed
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device);
    const Schedule sched = device_schedule(*schedule);
    const uint32_t colours = h->d.n_dist_batches + h->d.n_bend_batches;
    // the candidates: one colour per synchronisation (the colour-by-colour
    // launch), and tile mode at three CTA counts
    struct Shape {
        bool tiles;
        uint32_t grid;
    };
    std::vector<Shape> shapes;
    const bool had_tiles = h->tiles;
    const uint32_t had_grid = h->tile_grid;
    const bool tile_capable = h->tile_block != 0u && h->grid > 1u && h->cluster == 0u && h->d.resident == 0u;
    if (h->grid > 1u) shapes.push_back({false, h->grid});
    if (tile_capable) {
        h->tiles = true;   // tile_schedule asks only whether the schedule is covered
        const bool covered = tile_schedule(h, sched);
        h->tiles = had_tiles;
        if (covered)
            for (uint32_t g : {static_cast<uint32_t>(sms), static_cast<uint32_t>(3 * sms / 4), static_cast<uint32_t>(sms / 2)})
                shapes.push_back({true, std::max(g, 3u)});
    }
    auto report = [&](float us) {
        out[0] = h->tiles ? colours : 1u;
        out[1] = h->tiles ? h->tile_grid : h->grid;
        out[2] = h->tiles ? h->tile_block : h->block;
        out[3] = static_cast<uint32_t>(us);
    };
    if (shapes.size() < 2u) {
        report(0.0f);
        return NUMI_CLOTH_OK;
    }
    int rc = snapshot_slot(h, kTuneSlot);
    if (rc != NUMI_CLOTH_OK) return rc;
    cudaEvent_t t0, t1;
    cudaEventCreate(&t0);
    cudaEventCreate(&t1);
    float best_ms = INFINITY;
    size_t best = shapes.size();
    for (size_t k = 0; k < shapes.size() && rc == NUMI_CLOTH_OK; ++k) {
        if (shapes[k].tiles) {
            if (!configure_tiles(h, shapes[k].grid)) continue;
        } else {
            h->tiles = false;
        }
        float ms = 0.0f;
        for (int rep = 0; rep < 2 && rc == NUMI_CLOTH_OK; ++rep) {   // a warm-up run, then the timed one
            rc = restore_slot(h, kTuneSlot);
            if (rc == NUMI_CLOTH_OK) cudaEventRecord(t0, h->stream);
            if (rc == NUMI_CLOTH_OK) rc = numi_cloth_step(h, configs, count, schedule);
            if (rc == NUMI_CLOTH_OK) {
                cudaEventRecord(t1, h->stream);
                if (cudaEventSynchronize(t1) != cudaSuccess) rc = NUMI_CLOTH_ECUDA;
            }
        }
        if (rc != NUMI_CLOTH_OK) break;
        cudaEventElapsedTime(&ms, t0, t1);
        if (numi_cloth_failure(h) != 0u || h->host_failure != 0u) {
            // this shape failed (the caller's state comes back below)
            cudaMemsetAsync(h->d.failure, 0, sizeof(uint32_t), h->stream);
            h->host_failure = 0u;
            continue;
        }
        if (ms < best_ms) {
            best_ms = ms;
            best = k;
        }
    }
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    // keep the fastest shape (else the one the cloth had) and its state
    if (best < shapes.size() && shapes[best].tiles) {
        if (!configure_tiles(h, shapes[best].grid)) best = shapes.size();
    } else if (best < shapes.size()) {
        h->tiles = false;
    }
    if (best == shapes.size()) {
        if (had_tiles)
            configure_tiles(h, had_grid);
        else
            h->tiles = false;
    }
    const int rrc = restore_slot(h, kTuneSlot);
    if (rc == NUMI_CLOTH_OK) rc = rrc;
    if (rc == NUMI_CLOTH_OK && cudaStreamSynchronize(h->stream) != cudaSuccess) rc = NUMI_CLOTH_ECUDA;
    report(best < shapes.size() ? 1000.0f * best_ms : 0.0f);
    return rc;
}

extern "C" {

int numi_cloth_launch_info(numi_cloth_t* h, uint32_t out[6]) {
    if (h == nullptr || out == nullptr) return NUMI_CLOTH_EINVAL;
    cudaSetDevice(h->device);
    uint32_t stats[4] = {0, 0, 0, 0};
    if (cudaStreamSynchronize(h->stream) != cudaSuccess ||
        cudaMemcpy(stats, h->d.stats, sizeof(stats), cudaMemcpyDeviceToHost) != cudaSuccess)
        return NUMI_CLOTH_ECUDA;
    // the shape of the last launch (tile mode has its own), else the default
    out[0] = h->last_grid != 0u ? h->last_grid : h->grid;
    out[1] = h->last_block != 0u ? h->last_block : h->block;
    out[2] = stats[0];
    out[3] = h->launches;
    out[4] = h->cluster;
    out[5] = h->d.resident | (h->neighbours ? 2u : 0u) | (h->tiles ? 4u : 0u) | (h->last_tiles ? 8u : 0u) |
             (h->self_exact ? 16u : 0u);
    return NUMI_CLOTH_OK;
}

}  // extern "C"

// ------------------------------------------------------------------------
// Allocation-free stepping (numi_cloth_step_noalloc in numi_cloth.h).  The
// array below is the only device memory this path uses besides the
// caller's buffers: contact records, air forces, fixed-point fruit sums,
// reduction partials and the substep Configs of one call.
namespace {

struct NoAllocScratch {
    float4 slot_a[NUMI_CLOTH_NOALLOC_MAX_DISTANCES * NC_YARN_SLOTS];
    float4 slot_b[NUMI_CLOTH_NOALLOC_MAX_DISTANCES * NC_YARN_SLOTS];
    uint32_t live[NUMI_CLOTH_NOALLOC_MAX_DISTANCES];
    uint32_t list[NUMI_CLOTH_NOALLOC_MAX_DISTANCES];
    uint32_t list_n[4];
    float4 force[NUMI_CLOTH_NOALLOC_MAX_PARTICLES];
    unsigned long long fruit_sums[9u * NC_MAX_FRUITS + 8u];
    double red[256];
    uint32_t stamp[NUMI_CLOTH_NOALLOC_MAX_PARTICLES + NC_MAX_FRUITS];
    NumiClothConfig configs[NUMI_CLOTH_NOALLOC_MAX_SUBSTEPS];
    unsigned long long barrier[32];
    uint32_t stats[4];
};

// File-scope device array.  In host code this name is only a stand-in for
// the symbol, never a device address; the address comes from
// cudaGetSymbolAddress, once per device.
static __device__ __align__(256) unsigned char g_noalloc_scratch[sizeof(NoAllocScratch)];

// The scratch array's device address on each device, looked up on the
// first call with that device current and kept for the process (stale after
// a cudaDeviceReset of the device).  The lookup runs under a mutex, so two
// host threads making their first calls on one device at once agree.
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mutex;
NoAllocScratch* g_noalloc_ptr[kMaxDevices] = {};

NoAllocScratch* noalloc_scratch(int device) {
    if (device < 0 || device >= kMaxDevices) return nullptr;
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (g_noalloc_ptr[device] == nullptr) {
        void* ptr = nullptr;
        if (cudaGetSymbolAddress(&ptr, g_noalloc_scratch) != cudaSuccess || ptr == nullptr) return nullptr;
        g_noalloc_ptr[device] = static_cast<NoAllocScratch*>(ptr);
    }
    return g_noalloc_ptr[device];
}

int noalloc_reject(const char* what) {
    std::fprintf(stderr, "numi_cloth_step_noalloc: %s\n", what);
    return NUMI_CLOTH_EINVAL;
}

}  // namespace

extern "C" int numi_cloth_step_noalloc(const NumiClothConfig* base, const NumiClothDeviceState* st,
                                       const NumiClothBatch* batches, const uint32_t batchCounts[4],
                                       const NumiClothConfig* configs, uint32_t count,
                                       const NumiClothSchedule* schedule, void* stream_ptr) {
    if (base == nullptr || st == nullptr || configs == nullptr || schedule == nullptr || batchCounts == nullptr ||
        count == 0)
        return noalloc_reject("null argument or zero substeps");
    const uint32_t n = base->control.y, D = base->control.z, G = base->control.w;
    const uint32_t K = base->constraintCounts.x, B = base->constraintCounts.y, F = base->constraintCounts.w;
    const uint32_t P = base->contactCounts.x;
    if (n == 0 || n > NUMI_CLOTH_NOALLOC_MAX_PARTICLES)
        return noalloc_reject("particle count is zero or above NUMI_CLOTH_NOALLOC_MAX_PARTICLES (4096)");
    if (D > NUMI_CLOTH_NOALLOC_MAX_DISTANCES)
        return noalloc_reject("distance count above NUMI_CLOTH_NOALLOC_MAX_DISTANCES (8192)");
    if (count > NUMI_CLOTH_NOALLOC_MAX_SUBSTEPS)
        return noalloc_reject("substeps per call above NUMI_CLOTH_NOALLOC_MAX_SUBSTEPS (256)");
    if (F > NC_MAX_FRUITS || G > NC_MAX_GRIPS || P > NC_MAX_PAIRS)
        return noalloc_reject("fruit, grip or fruit-pair count above its limit");
    for (int k = 0; k < 4; ++k)
        if (batchCounts[k] > NC_MAX_BATCHES) return noalloc_reject("more than 64 colour runs in one family");
    if ((batchCounts[0] + batchCounts[1] + batchCounts[2] + batchCounts[3]) != 0u && batches == nullptr)
        return noalloc_reject("null batches");
    {
        // every colour run stays inside its family's records, and a distance
        // run's yarn and strain-limited prefixes inside the run
        const uint32_t records[4] = {D, K, B, P};
        const NumiClothBatch* run = batches;
        for (int fam = 0; fam < 4; ++fam)
            for (uint32_t k = 0; k < batchCounts[fam]; ++k, ++run) {
                const uint64_t first = run->control.x, cnt = run->control.y;
                if (first + cnt > records[fam]) return noalloc_reject("a colour run reaches past its family's records");
                if (fam == 0 && ((run->control.w & 0xffffu) > cnt || (run->control.w >> 16) > cnt))
                    return noalloc_reject("a distance run's yarn or strain-limited prefix is longer than the run");
            }
    }
    if (schedule->selfCollision)
        return noalloc_reject("selfCollision needs the point self-contact hash grid, which this path does not hold");
    if (schedule->release)
        return noalloc_reject("release needs the mouth rim, which NumiClothDeviceState does not carry");
    if (schedule->primitiveSelf)
        return noalloc_reject("primitiveSelf needs the edge/edge pass buffers, which this path does not hold");
    if (!st->positions || !st->previous || !st->velocities || !st->rest || !st->failure ||
        (D && (!st->distanceIJ || !st->distanceMaterial || !st->distanceLambda)) ||
        (K && (!st->knotIJ || !st->knotMaterial || !st->knotLambda)) ||
        (B && (!st->bendIJ || !st->bendMaterial || !st->bendLambda)) || (G && !st->grips) || (F && !st->fruits) ||
        (P && !st->fruitPairs) || (base->gripControl.y == 1u && !st->cuffParticles))
        return noalloc_reject("null device buffer");
    uint32_t bad = 0;
    for (uint32_t k = 0; k < count && bad == 0u; ++k) bad = validate_config(configs[k], *base);
    if (bad != 0u) return static_cast<int>(bad);
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) return NUMI_CLOTH_ECUDA;
    NoAllocScratch* scratch = noalloc_scratch(device);
    if (scratch == nullptr) return NUMI_CLOTH_ECUDA;
    cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);

    DeviceCloth d{};
    d.x = reinterpret_cast<float4*>(st->positions);
    d.xp = reinterpret_cast<float4*>(st->previous);
    d.v = reinterpret_cast<float4*>(st->velocities);
    d.rest = reinterpret_cast<const float4*>(st->rest);
    d.n = n;
    d.d_ij = reinterpret_cast<const uint2*>(st->distanceIJ);
    d.d_mat = reinterpret_cast<const float4*>(st->distanceMaterial);
    d.d_lambda = st->distanceLambda;
    d.d_count = D;
    d.k_ij = reinterpret_cast<const uint4*>(st->knotIJ);
    d.k_mat = reinterpret_cast<const float2*>(st->knotMaterial);
    d.k_lambda = st->knotLambda;
    d.k_count = K;
    d.b_ij = reinterpret_cast<const uint4*>(st->bendIJ);
    d.b_mat = reinterpret_cast<const float2*>(st->bendMaterial);
    d.b_lambda = st->bendLambda;
    d.b_count = B;
    d.grips = st->grips;
    d.g_count = G;
    d.fruits = st->fruits;
    d.f_count = F;
    d.pairs = st->fruitPairs;
    d.p_count = P;
    d.cuff = st->cuffParticles;
    d.failure = st->failure;
    d.yarn_slot_a = scratch->slot_a;
    d.yarn_slot_b = scratch->slot_b;
    d.yarn_live = scratch->live;
    d.yarn_list = scratch->list;
    d.yarn_list_n = scratch->list_n;
    d.force = scratch->force;
    d.fruit_partial = reinterpret_cast<float4*>(scratch->fruit_sums);
    d.red = scratch->red;
    d.bar_count = scratch->barrier;
    d.abort_flag = reinterpret_cast<unsigned int*>(scratch->barrier + 1);
    d.bar_flag = scratch->barrier + 16;
    d.stats = scratch->stats;
    d.cfg = scratch->configs;
    d.epoch_base = 1u;   // contact records are cleared below, so epochs restart at 1
    d.damping = -1.0f;   // the schedule's damping applies (as on the handle path)
    d.check_stamp = scratch->stamp;   // the kernel checks the caller's records first
    Batch* families[4] = {d.dist_batches, d.knot_batches, d.bend_batches, d.pair_batches};
    uint32_t* family_counts[4] = {&d.n_dist_batches, &d.n_knot_batches, &d.n_bend_batches, &d.n_pair_batches};
    const NumiClothBatch* b = batches;
    for (int fam = 0; fam < 4; ++fam) {
        *family_counts[fam] = batchCounts[fam];
        for (uint32_t k = 0; k < batchCounts[fam]; ++k, ++b) {
            Batch& o = families[fam][k];
            o.first = b->control.x;
            o.count = b->control.y;
            o.yarn = fam == 0 ? (b->control.w & 0xffffu) : 0u;
            o.limited = fam == 0 ? (b->control.w >> 16) : 0u;
        }
    }
    // Every call shares the scratch: clear what must start at zero (contact
    // records and their live epochs, fixed-point fruit sums, barrier words,
    // stats) and the caller's failure word.
    cudaError_t e = cudaMemsetAsync(scratch->slot_b, 0, sizeof(scratch->slot_b), stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(scratch->live, 0, sizeof(scratch->live), stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(scratch->fruit_sums, 0, sizeof(scratch->fruit_sums), stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(scratch->barrier, 0, sizeof(scratch->barrier), stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(scratch->stats, 0, sizeof(scratch->stats), stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(st->failure, 0, sizeof(uint32_t), stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(scratch->configs, configs, count * sizeof(NumiClothConfig), cudaMemcpyHostToDevice,
                            stream);
    if (e != cudaSuccess) return NUMI_CLOTH_ECUDA;
    Schedule s{};
    s.iterations = schedule->iterations;
    s.strain_sweeps = schedule->strainSweeps;
    s.reconcile_passes = schedule->reconcilePasses;
    s.final_passes = schedule->finalPasses;
    s.certificate_passes = schedule->certificatePasses;
    s.early_exit = schedule->earlyExit;
    s.self_collision = schedule->selfCollision;
    s.aerodynamics = schedule->aerodynamics;
    s.swept_ground = schedule->sweptGround;
    s.swept_fruit_yarn = schedule->sweptFruitYarn;
    s.frictions = schedule->frictions;
    s.release = schedule->release;
    s.damping = schedule->damping;
    s.substeps = count;
    void* args[] = {&d, &s};
    e = raise_frame_smem(nc_resident_offset());
    if (e == cudaSuccess)
        e = cudaLaunchKernel(reinterpret_cast<const void*>(numi_cloth_frame_kernel), dim3(1), dim3(NC_THREADS), args,
                             nc_resident_offset(), stream);
    return e == cudaSuccess ? NUMI_CLOTH_OK : NUMI_CLOTH_ECUDA;
}

// ------------------------------------------------------------------------
// Batched stepping (numi_cloth_batch_* in numi_cloth.h): many independent
// cloths in one persistent launch.  Each CTA takes the next cloth from a
// device work queue (largest cloths first, so the last wave is short) and
// runs its whole frame alone with CTA barriers; the cloths' device state is
// their handles' own, so every per-handle read/write call still works.

struct numi_cloth_batch {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::vector<numi_cloth*> cloths;   // caller order
    std::vector<uint32_t> order;       // launch position -> caller index
    DeviceBuffers buf;
    DeviceCloth* d_cloths = nullptr;   // launch order
    NumiClothConfig* d_cfg = nullptr;  // caller order, cloth-major
    uint32_t cfg_capacity = 0;         // substeps per cloth d_cfg holds
    uint32_t layout_substeps = 0;      // substeps the uploaded descriptors assume
    bool layout_valid = false;
    unsigned int* queue = nullptr;
    uint32_t* epoch = nullptr;         // device substep counter
    uint32_t epoch_host = 1;
    uint32_t block = NC_THREADS;
    uint32_t chunk = 0;                // resident particle chunk (0: none)
    bool edge_room = true;             // the shape leaves room for the box tree's sort keys
    uint32_t ctas = 0;
    size_t smem = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    const NumiClothConfig* graph_cfg = nullptr;
    uint32_t graph_substeps = 0;
};

namespace {

uint32_t log2_pow2(uint32_t v) {
    uint32_t s = 0;
    while ((1u << s) < v) ++s;
    return s;
}

// Launch shape: resident chunk (0 or a power of two), threads per CTA, and
// as many CTAs as fit on the device (never more than the cloths).
int batch_shape(numi_cloth_batch* b, uint32_t chunk, uint32_t block) {
    const size_t smem = nc_resident_offset() + (chunk ? 2u * static_cast<size_t>(chunk) * sizeof(float4) : 0u);
    int optin = 0, sms = 0;
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, b->device);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device);
    int per_sm = 1 << 30;
    bool edge_room = false;
    for (bool edge : {false, true}) {
        // the edge/edge kernel also holds the box tree's sort keys; a shape
        // without room for them serves only schedules without that family
        const size_t bytes = edge ? nc_round256(smem) + NC_EDGE_TREE_KEY_BYTES : smem;
        cudaFuncAttributes fa{};
        if (cudaFuncGetAttributes(&fa, batch_fn(edge)) != cudaSuccess) return NUMI_CLOTH_ECUDA;
        if (bytes + fa.sharedSizeBytes > static_cast<size_t>(optin)) {
            if (edge) continue;
            return NUMI_CLOTH_EINVAL;
        }
        if (raise_smem(batch_fn(edge), bytes) != cudaSuccess) return NUMI_CLOTH_ECUDA;
        if (edge) {
            edge_room = true;
            continue;   // launched without co-residence
        }
        int k = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&k, batch_fn(edge), static_cast<int>(block), bytes) !=
            cudaSuccess)
            return NUMI_CLOTH_EINVAL;
        per_sm = std::min(per_sm, k);
    }
    if (per_sm < 1) return NUMI_CLOTH_EINVAL;
    b->edge_room = edge_room;
    b->chunk = chunk;
    b->block = block;
    b->smem = smem;
    b->ctas = std::min<uint32_t>(static_cast<uint32_t>(b->cloths.size()), static_cast<uint32_t>(sms * per_sm));
    b->layout_valid = false;
    return NUMI_CLOTH_OK;
}

// Descriptors of every cloth for a launch of `substeps` Configs each.
int batch_layout(numi_cloth_batch* b, uint32_t substeps) {
    if (b->layout_valid && b->layout_substeps == substeps) return NUMI_CLOTH_OK;
    const uint32_t count = static_cast<uint32_t>(b->cloths.size());
    std::vector<DeviceCloth> host(count);
    for (uint32_t j = 0; j < count; ++j) {
        const uint32_t k = b->order[j];
        DeviceCloth d = b->cloths[k]->d;
        d.cfg = b->d_cfg + static_cast<size_t>(k) * substeps;
        d.trace = nullptr;
        d.trace_cta = nullptr;
        d.cluster_barrier = 0u;
        d.resident = (b->chunk != 0u && d.n <= b->chunk) ? 1u : 0u;
        d.resident_shift = b->chunk ? log2_pow2(b->chunk) : 0u;
        host[j] = d;
    }
    if (cudaMemcpyAsync(b->d_cloths, host.data(), count * sizeof(DeviceCloth), cudaMemcpyHostToDevice, b->stream) !=
        cudaSuccess)
        return NUMI_CLOTH_ECUDA;
    if (cudaStreamSynchronize(b->stream) != cudaSuccess) return NUMI_CLOTH_ECUDA;
    b->layout_substeps = substeps;
    b->layout_valid = true;
    return NUMI_CLOTH_OK;
}

// Validate and stage one launch: Configs, self-contact grids, descriptors.
int batch_prepare(numi_cloth_batch* b, const NumiClothConfig* configs, uint32_t substeps, const NumiClothSchedule& sched) {
    if (sched.primitiveSelf != 0u && !b->edge_room) return NUMI_CLOTH_EINVAL;   // set a smaller shape first
    const uint32_t count = static_cast<uint32_t>(b->cloths.size());
    for (uint32_t k = 0; k < count; ++k) {
        numi_cloth* h = b->cloths[k];
        if (h->poisoned) return NUMI_CLOTH_ESTATE;
        for (uint32_t q = 0; q < substeps; ++q) {
            const uint32_t bad = validate_config(configs[static_cast<size_t>(k) * substeps + q], h->base);
            if (bad) {
                h->host_failure |= bad;
                return static_cast<int>(bad);
            }
        }
    }
    if (substeps > b->cfg_capacity) {
        NumiClothConfig* cfg = b->buf.alloc<NumiClothConfig>(static_cast<size_t>(count) * substeps);
        if (cfg == nullptr) return NUMI_CLOTH_ENOMEM;
        b->d_cfg = cfg;
        b->cfg_capacity = substeps;
        b->layout_valid = false;
    }
    for (size_t k = 0; k < b->cloths.size(); ++k) {
        numi_cloth* h = b->cloths[k];
        void* before = h->d.hash_head;
        void* edge_before = h->d.edge_count;
        const float cell_before = h->d.edge_cell;
        h->epoch = b->epoch_host;
        int rc = prepare_self_grid(h, sched.selfCollision != 0u, substeps);
        if (rc == NUMI_CLOTH_OK)
            rc = prepare_edge_grid(h, sched.primitiveSelf != 0u, substeps,
                                   configs[k * substeps].clothMaterial.x);
        if (rc != NUMI_CLOTH_OK) return rc;
        if (h->d.hash_head != before || h->d.edge_count != edge_before || h->d.edge_cell != cell_before)
            b->layout_valid = false;
        if (h->stream != b->stream && h->stream != nullptr && cudaStreamSynchronize(h->stream) != cudaSuccess)
            return NUMI_CLOTH_ECUDA;
    }
    return batch_layout(b, substeps);
}

cudaError_t batch_launch(numi_cloth_batch* b, const NumiClothConfig* configs, uint32_t substeps, const Schedule& s) {
    const uint32_t count = static_cast<uint32_t>(b->cloths.size());
    cudaError_t e = cudaMemcpyAsync(b->d_cfg, configs, static_cast<size_t>(count) * substeps * sizeof(NumiClothConfig),
                                    cudaMemcpyHostToDevice, b->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(b->queue, 0, sizeof(unsigned int), b->stream);
    if (e != cudaSuccess) return e;
    Schedule sc = s;
    sc.substeps = substeps;
    sc.epoch_ptr = b->epoch;
    unsigned int* queue = b->queue;
    const DeviceCloth* cloths = b->d_cloths;
    void* args[] = {&cloths, const_cast<uint32_t*>(&count), &sc, &queue};
    size_t smem = b->smem;
    if (sc.primitive_self != 0u) {   // the box tree's sort keys (batch_shape checked the room)
        sc.tree_keys = static_cast<uint32_t>(nc_round256(smem));
        smem = nc_round256(smem) + NC_EDGE_TREE_KEY_BYTES;
    }
    e = cudaLaunchKernel(batch_fn(sc.primitive_self != 0u), dim3(b->ctas), dim3(b->block), args, smem, b->stream);
    if (e != cudaSuccess) return e;
    numi_cloth_epoch_kernel<<<1, 1, 0, b->stream>>>(b->epoch, substeps);
    return cudaGetLastError();
}

void batch_advance(numi_cloth_batch* b, uint32_t substeps) {
    b->epoch_host += substeps;
    for (numi_cloth* h : b->cloths) {
        h->epoch = b->epoch_host;
        h->last_substeps = substeps;
        ++h->launches;
    }
}

void batch_drop_graph(numi_cloth_batch* b) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
    b->graph_cfg = nullptr;
}

}  // namespace

extern "C" {

int numi_cloth_batch_create(numi_cloth_t* const* cloths, uint32_t count, numi_cloth_batch_t** out) {
    if (cloths == nullptr || out == nullptr || count == 0) return NUMI_CLOTH_EINVAL;
    *out = nullptr;
    auto* b = new numi_cloth_batch();
    b->device = cloths[0] ? cloths[0]->device : 0;
    for (uint32_t k = 0; k < count; ++k) {
        if (cloths[k] == nullptr || cloths[k]->device != b->device) {
            delete b;
            return NUMI_CLOTH_EINVAL;
        }
        for (uint32_t j = 0; j < k; ++j)
            if (cloths[j] == cloths[k]) {
                delete b;
                return NUMI_CLOTH_EINVAL;
            }
        b->cloths.push_back(cloths[k]);
        b->epoch_host = std::max(b->epoch_host, cloths[k]->epoch);
    }
    cudaSetDevice(b->device);
    // largest work first: particles plus constraints
    b->order.resize(count);
    for (uint32_t k = 0; k < count; ++k) b->order[k] = k;
    auto work = [&](uint32_t k) {
        const DeviceCloth& d = b->cloths[k]->d;
        return static_cast<uint64_t>(d.n) + d.d_count + d.k_count + d.b_count;
    };
    std::stable_sort(b->order.begin(), b->order.end(), [&](uint32_t a, uint32_t c) { return work(a) > work(c); });
    b->d_cloths = b->buf.alloc<DeviceCloth>(count);
    b->queue = b->buf.alloc<unsigned int>(1);
    b->epoch = b->buf.alloc<uint32_t>(1);
    if (!b->d_cloths || !b->queue || !b->epoch ||
        cudaMemcpy(b->epoch, &b->epoch_host, sizeof(uint32_t), cudaMemcpyHostToDevice) != cudaSuccess) {
        delete b;
        return NUMI_CLOTH_ENOMEM;
    }
    // default shape: particles from global memory, 256 threads per CTA
    const int rc = batch_shape(b, 0u, NC_THREADS);
    if (rc != NUMI_CLOTH_OK) {
        delete b;
        return rc;
    }
    *out = b;
    return NUMI_CLOTH_OK;
}

void numi_cloth_batch_destroy(numi_cloth_batch_t* b) {
    if (b == nullptr) return;
    cudaSetDevice(b->device);
    cudaStreamSynchronize(b->stream);
    batch_drop_graph(b);
    delete b;
}

int numi_cloth_batch_set_stream(numi_cloth_batch_t* b, void* stream) {
    if (b == nullptr) return NUMI_CLOTH_EINVAL;
    b->stream = static_cast<cudaStream_t>(stream);
    batch_drop_graph(b);
    return NUMI_CLOTH_OK;
}

int numi_cloth_batch_set_shape(numi_cloth_batch_t* b, uint32_t resident_chunk, uint32_t threads) {
    if (b == nullptr || (threads != NC_THREADS && threads != NC_BLOCK_MAX) ||
        (resident_chunk != 0u && (resident_chunk & (resident_chunk - 1u)) != 0u) || resident_chunk > 4096u)
        return NUMI_CLOTH_EINVAL;
    cudaSetDevice(b->device);
    batch_drop_graph(b);
    return batch_shape(b, resident_chunk, threads);
}

int numi_cloth_batch_shape(numi_cloth_batch_t* b, uint32_t out[3]) {
    if (b == nullptr || out == nullptr) return NUMI_CLOTH_EINVAL;
    out[0] = b->chunk;
    out[1] = b->block;
    out[2] = b->ctas;
    return NUMI_CLOTH_OK;
}

int numi_cloth_batch_step(numi_cloth_batch_t* b, const NumiClothConfig* configs, uint32_t substeps,
                          const NumiClothSchedule* schedule) {
    if (b == nullptr || configs == nullptr || schedule == nullptr || substeps == 0) return NUMI_CLOTH_EINVAL;
    cudaSetDevice(b->device);
    const int rc = batch_prepare(b, configs, substeps, *schedule);
    if (rc > 0) return NUMI_CLOTH_OK;   // a rejected Config: its cloth's failure word reports it
    if (rc != NUMI_CLOTH_OK) return rc;
    const cudaError_t e = batch_launch(b, configs, substeps, device_schedule(*schedule));
    batch_advance(b, substeps);
    if (e != cudaSuccess) {
        for (numi_cloth* h : b->cloths) h->poisoned = true;
        return NUMI_CLOTH_ECUDA;
    }
    return NUMI_CLOTH_OK;
}

int numi_cloth_batch_tune(numi_cloth_batch_t* b, const NumiClothConfig* configs, uint32_t substeps,
                          const NumiClothSchedule* schedule, uint32_t out[3]) {
    if (b == nullptr || configs == nullptr || schedule == nullptr || substeps == 0) return NUMI_CLOTH_EINVAL;
    cudaSetDevice(b->device);
    batch_drop_graph(b);
    uint32_t largest = 0;
    for (numi_cloth* h : b->cloths) largest = std::max(largest, h->d.n);
    const uint32_t slot = kTuneSlot;
    for (numi_cloth* h : b->cloths) {
        const int rc = snapshot_slot(h, slot);
        if (rc != NUMI_CLOTH_OK) return rc;
        if (h->stream && cudaStreamSynchronize(h->stream) != cudaSuccess) return NUMI_CLOTH_ECUDA;
    }
    if (cudaDeviceSynchronize() != cudaSuccess) return NUMI_CLOTH_ECUDA;
    cudaEvent_t t0, t1;
    cudaEventCreate(&t0);
    cudaEventCreate(&t1);
    float best_ms = INFINITY;
    uint32_t best_chunk = 0, best_block = NC_THREADS;
    const uint32_t chunks[] = {0u, 256u, 512u, 1024u, 2048u, 4096u};
    const uint32_t blocks[] = {NC_THREADS, NC_BLOCK_MAX};
    const Schedule s = device_schedule(*schedule);
    int rc = NUMI_CLOTH_OK;
    for (uint32_t chunk : chunks) {
        if (chunk > 0u && chunk / 2u >= largest) continue;   // same as a smaller chunk
        for (uint32_t block : blocks) {
            if (batch_shape(b, chunk, block) != NUMI_CLOTH_OK) continue;
            if (schedule->primitiveSelf != 0u && !b->edge_room) continue;
            rc = batch_prepare(b, configs, substeps, *schedule);
            if (rc != NUMI_CLOTH_OK) break;
            cudaEventRecord(t0, b->stream);
            const cudaError_t e = batch_launch(b, configs, substeps, s);
            cudaEventRecord(t1, b->stream);
            if (e != cudaSuccess || cudaEventSynchronize(t1) != cudaSuccess) {
                rc = NUMI_CLOTH_ECUDA;
                break;
            }
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, t0, t1);
            batch_advance(b, substeps);
            if (ms < best_ms) {
                best_ms = ms;
                best_chunk = chunk;
                best_block = block;
            }
            for (numi_cloth* h : b->cloths) restore_slot(h, slot);
            if (cudaDeviceSynchronize() != cudaSuccess) {
                rc = NUMI_CLOTH_ECUDA;
                break;
            }
        }
        if (rc != NUMI_CLOTH_OK) break;
    }
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    if (rc != NUMI_CLOTH_OK) return rc;
    rc = batch_shape(b, best_chunk, best_block);
    if (rc == NUMI_CLOTH_OK && out != nullptr) numi_cloth_batch_shape(b, out);
    return rc;
}

int numi_cloth_batch_capture(numi_cloth_batch_t* b, const NumiClothConfig* configs, uint32_t substeps,
                             const NumiClothSchedule* schedule) {
    if (b == nullptr || configs == nullptr || schedule == nullptr || substeps == 0) return NUMI_CLOTH_EINVAL;
    cudaSetDevice(b->device);
    batch_drop_graph(b);
    int rc = batch_prepare(b, configs, substeps, *schedule);
    if (rc > 0) return NUMI_CLOTH_EINVAL;
    if (rc != NUMI_CLOTH_OK) return rc;
    cudaStream_t cap = nullptr;
    if (cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking) != cudaSuccess) return NUMI_CLOTH_ECUDA;
    cudaStream_t saved = b->stream;
    b->stream = cap;
    cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        const cudaError_t le = batch_launch(b, configs, substeps, device_schedule(*schedule));
        e = cudaStreamEndCapture(cap, &b->graph);
        if (le != cudaSuccess) e = le;
    }
    b->stream = saved;
    cudaStreamDestroy(cap);
    if (e == cudaSuccess) e = cudaGraphInstantiate(&b->exec, b->graph, 0);
    if (e != cudaSuccess) {
        batch_drop_graph(b);
        cudaGetLastError();
        return NUMI_CLOTH_ECUDA;
    }
    b->graph_cfg = configs;
    b->graph_substeps = substeps;
    return NUMI_CLOTH_OK;
}

int numi_cloth_batch_replay(numi_cloth_batch_t* b) {
    if (b == nullptr || b->exec == nullptr) return NUMI_CLOTH_ESTATE;
    cudaSetDevice(b->device);
    const uint32_t count = static_cast<uint32_t>(b->cloths.size());
    for (uint32_t k = 0; k < count; ++k) {
        numi_cloth* h = b->cloths[k];
        if (h->poisoned) return NUMI_CLOTH_ESTATE;
        for (uint32_t q = 0; q < b->graph_substeps; ++q) {
            const uint32_t bad = validate_config(b->graph_cfg[static_cast<size_t>(k) * b->graph_substeps + q], h->base);
            if (bad) {
                h->host_failure |= bad;
                return NUMI_CLOTH_OK;
            }
        }
        if (h->d.hash_head != nullptr && ((b->epoch_host + b->graph_substeps) >> 26) != (b->epoch_host >> 26))
            return NUMI_CLOTH_ESTATE;   // tag wrap: capture again after a plain step
    }
    const cudaError_t e = cudaGraphLaunch(b->exec, b->stream);
    batch_advance(b, b->graph_substeps);
    if (e != cudaSuccess) {
        for (numi_cloth* h : b->cloths) h->poisoned = true;
        return NUMI_CLOTH_ECUDA;
    }
    return NUMI_CLOTH_OK;
}

}  // extern "C"

// ------------------------------------------------------------------------
// Reverse-mode gradients of a rollout (numi_cloth_rollout_grad).

namespace {

// Barrier sequence of one substep for the schedules the adjoint supports
// (one iteration, no reconciliation / final / certificate passes, no air
// load, no self contact): mirrors nc::substep.
std::vector<uint2> adjoint_phases(const DeviceCloth& d, const Schedule& s) {
    std::vector<uint2> ph;
    ph.push_back(make_uint2(ADJ_BEGIN, 0u));
    for (uint32_t b = 0; b < d.n_dist_batches; ++b) ph.push_back(make_uint2(ADJ_DIST, b));
    for (uint32_t b = 0; b < d.n_knot_batches; ++b) ph.push_back(make_uint2(ADJ_KNOT, b));
    for (uint32_t b = 0; b < d.n_bend_batches; ++b) ph.push_back(make_uint2(ADJ_BEND, b));
    ph.push_back(make_uint2(ADJ_GRIP, 0u));
    if (d.f_count > 0u)
        for (uint32_t b = 0; b < d.n_dist_batches; ++b)
            if (d.dist_batches[b].yarn != 0u) ph.push_back(make_uint2(ADJ_YARN, b));
    ph.push_back(make_uint2(ADJ_GROUND, 0u));
    for (uint32_t sw = 0; sw < s.strain_sweeps; ++sw)
        for (uint32_t b = 0; b < d.n_dist_batches; ++b)
            if (d.dist_batches[b].limited != 0u) ph.push_back(make_uint2(ADJ_STRAIN, b));
    ph.push_back(make_uint2(ADJ_FINAL, 0u));
    // fruit/yarn friction and the fruit tail share the substep's last phase
    ph.push_back(make_uint2(ADJ_TAIL, 0u));
    return ph;
}

// Device allocations of one rollout, freed on scope exit.
struct Scratch {
    std::vector<void*> owned;
    template <class T>
    T* get(size_t count) {
        void* p = nullptr;
        if (cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T)) != cudaSuccess) return nullptr;
        cudaMemset(p, 0, std::max<size_t>(count, 1) * sizeof(T));
        owned.push_back(p);
        return static_cast<T*>(p);
    }
    ~Scratch() {
        for (void* p : owned) cudaFree(p);
    }
};

// Compliance groups: the distinct compliance values of each constraint
// family (distance, knot, bend, grip), ascending, numbered family by family.
struct Groups {
    std::vector<uint32_t> family;
    std::vector<float> value;
    std::vector<uint8_t> d, k, b, g;   // per record
};

int compliance_groups(numi_cloth* h, Groups& out) {
    const DeviceCloth& d = h->d;
    std::vector<float4> dm(d.d_count);
    std::vector<float2> km(d.k_count), bm(d.b_count);
    std::vector<NumiClothGrip> gr(d.g_count);
    cudaError_t e = cudaStreamSynchronize(h->stream);
    if (e == cudaSuccess && d.d_count) e = cudaMemcpy(dm.data(), d.d_mat, d.d_count * sizeof(float4), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && d.k_count) e = cudaMemcpy(km.data(), d.k_mat, d.k_count * sizeof(float2), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && d.b_count) e = cudaMemcpy(bm.data(), d.b_mat, d.b_count * sizeof(float2), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && d.g_count)
        e = cudaMemcpy(gr.data(), d.grips, d.g_count * sizeof(NumiClothGrip), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return NUMI_CLOTH_ECUDA;
    auto assign = [&](uint32_t family, const std::vector<float>& values, std::vector<uint8_t>& ids) {
        std::vector<float> distinct = values;
        std::sort(distinct.begin(), distinct.end());
        distinct.erase(std::unique(distinct.begin(), distinct.end()), distinct.end());
        const uint32_t base = static_cast<uint32_t>(out.value.size());
        for (float v : distinct) {
            out.family.push_back(family);
            out.value.push_back(v);
        }
        ids.resize(values.size());
        for (size_t r = 0; r < values.size(); ++r)
            ids[r] = static_cast<uint8_t>(
                base + (std::lower_bound(distinct.begin(), distinct.end(), values[r]) - distinct.begin()));
    };
    std::vector<float> v;
    v.clear();
    for (const float4& m : dm) v.push_back(m.y);
    assign(0u, v, out.d);
    v.clear();
    for (const float2& m : km) v.push_back(m.y);
    assign(1u, v, out.k);
    v.clear();
    for (const float2& m : bm) v.push_back(m.y);
    assign(2u, v, out.b);
    v.clear();
    for (const NumiClothGrip& g : gr) v.push_back(g.targetOffsetAndCompliance.w);
    assign(3u, v, out.g);
    return out.value.size() <= NUMI_CLOTH_MAX_GROUPS ? NUMI_CLOTH_OK : NUMI_CLOTH_EINVAL;
}

__global__ void numi_cloth_replace_compliance_kernel(DeviceCloth d, uint32_t family, float from, float to) {
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;; k += stride) {
        bool any = false;
        if (family == 0u && k < d.d_count) {
            any = true;
            float4* m = const_cast<float4*>(d.d_mat) + k;
            if (m->y == from) m->y = to;
        }
        if (family == 1u && k < d.k_count) {
            any = true;
            float2* m = const_cast<float2*>(d.k_mat) + k;
            if (m->y == from) m->y = to;
        }
        if (family == 2u && k < d.b_count) {
            any = true;
            float2* m = const_cast<float2*>(d.b_mat) + k;
            if (m->y == from) m->y = to;
        }
        if (family == 3u && k < d.g_count) {
            any = true;
            if (d.grips[k].targetOffsetAndCompliance.w == from) d.grips[k].targetOffsetAndCompliance.w = to;
        }
        if (!any) break;
    }
}

}  // namespace

extern "C" int numi_cloth_compliance_groups(numi_cloth_t* h, uint32_t family[NUMI_CLOTH_MAX_GROUPS],
                                            float compliance[NUMI_CLOTH_MAX_GROUPS], uint32_t* count) {
    if (h == nullptr || family == nullptr || compliance == nullptr || count == nullptr) return NUMI_CLOTH_EINVAL;
    cudaSetDevice(h->device);
    Groups g;
    const int rc = compliance_groups(h, g);
    if (rc != NUMI_CLOTH_OK) return rc;
    *count = static_cast<uint32_t>(g.value.size());
    for (size_t k = 0; k < g.value.size(); ++k) {
        family[k] = g.family[k];
        compliance[k] = g.value[k];
    }
    return NUMI_CLOTH_OK;
}

extern "C" int numi_cloth_replace_compliance(numi_cloth_t* h, uint32_t family, float from, float to) {
    if (h == nullptr || family > 3u || !(to >= 0.0f) || !std::isfinite(to)) return NUMI_CLOTH_EINVAL;
    cudaSetDevice(h->device);
    h->tiles_dirty = h->tiles;   // the tile plan's items carry the materials
    numi_cloth_replace_compliance_kernel<<<64, 256, 0, h->stream>>>(h->d, family, from, to);
    return cudaGetLastError() == cudaSuccess ? NUMI_CLOTH_OK : NUMI_CLOTH_ECUDA;
}

extern "C" int numi_cloth_rollout_grad(numi_cloth_t* h, const NumiClothConfig* configs, uint32_t substeps,
                                       const NumiClothSchedule* schedule, uint32_t checkpoint_every,
                                       const uint32_t* tracked, uint32_t n_tracked, const double* targets,
                                       uint32_t loss_every, double* loss, double* grads, double* grip_grads,
                                       uint32_t* nonsmooth) {
    if (h == nullptr || configs == nullptr || schedule == nullptr || substeps == 0 || checkpoint_every == 0 ||
        loss == nullptr || grads == nullptr || (n_tracked > 0 && (tracked == nullptr || targets == nullptr)) ||
        loss_every == 0)
        return NUMI_CLOTH_EINVAL;
    if (h->poisoned) return NUMI_CLOTH_ESTATE;
    const NumiClothSchedule& sc = *schedule;
    if (sc.iterations != 1u || sc.reconcilePasses != 0u || sc.finalPasses != 0u || sc.certificatePasses != 0u ||
        sc.aerodynamics != 0u || sc.selfCollision != 0u || sc.primitiveSelf != 0u)
        return NUMI_CLOTH_EINVAL;
    for (uint32_t t = 0; t < n_tracked; ++t)
        if (tracked[t] >= h->d.n) return NUMI_CLOTH_EINVAL;
    cudaSetDevice(h->device);
    for (uint32_t k = 0; k < substeps; ++k) {
        const uint32_t bad = validate_config(configs[k], h->base);
        if (bad) {
            h->host_failure |= bad;
            return static_cast<int>(bad);
        }
    }
    if (substeps > h->cfg_capacity) {
        cudaFree(h->d_cfg);
        h->d_cfg = nullptr;
        if (cudaMalloc(&h->d_cfg, substeps * sizeof(NumiClothConfig)) != cudaSuccess) return NUMI_CLOTH_ECUDA;
        h->cfg_capacity = substeps;
    }
    if (cudaMemcpyAsync(h->d_cfg, configs, substeps * sizeof(NumiClothConfig), cudaMemcpyHostToDevice, h->stream) !=
        cudaSuccess)
        return NUMI_CLOTH_ECUDA;
    const Schedule s = device_schedule(sc);
    const std::vector<uint2> phases = adjoint_phases(h->d, s);
    const uint32_t slots = static_cast<uint32_t>(phases.size()) + 1u;
    const uint32_t n = h->d.n;
    const uint32_t segs = (substeps + checkpoint_every - 1u) / checkpoint_every;
    const uint32_t losses = substeps / loss_every;

    Groups groups;
    {
        const int rc = compliance_groups(h, groups);
        if (rc != NUMI_CLOTH_OK) return rc;
    }
    const uint32_t ngroups = static_cast<uint32_t>(groups.value.size());
    Scratch mem;
    size_t state_bytes = 0;
    for (const auto& r : h->dynamic) state_bytes += (r.bytes + 255u) & ~size_t(255u);
    char* ckpt = mem.get<char>((segs + 1u) * state_bytes);
    float4* tape = mem.get<float4>(static_cast<size_t>(checkpoint_every) * slots * n);
    float4* tape_v = mem.get<float4>(static_cast<size_t>(checkpoint_every) * n);
    uint2* d_phases = mem.get<uint2>(phases.size());
    DeviceCloth* d_cloth = mem.get<DeviceCloth>(1);
    uint32_t* d_tracked = mem.get<uint32_t>(n_tracked);
    double* d_targets = mem.get<double>(static_cast<size_t>(losses) * n_tracked * 3u);
    double4* gx = mem.get<double4>(n);
    double4* gv = mem.get<double4>(n);
    double4* gprev = mem.get<double4>(n);
    double* d_out = mem.get<double>(ngroups + 2u);   // group gradients, damping, loss
    uint8_t* gd = mem.get<uint8_t>(groups.d.size());
    uint8_t* gk = mem.get<uint8_t>(groups.k.size());
    uint8_t* gb = mem.get<uint8_t>(groups.b.size());
    uint8_t* gg = mem.get<uint8_t>(groups.g.size());
    double* d_grip = mem.get<double>(static_cast<size_t>(substeps) * 6u);
    unsigned int* d_rough = mem.get<unsigned int>(1);
    if (!ckpt || !tape || !tape_v || !d_phases || !d_cloth || !d_tracked || !d_targets || !gx || !gv || !gprev ||
        !d_out || !d_grip || !d_rough || !gd || !gk || !gb || !gg)
        return NUMI_CLOTH_ENOMEM;
    cudaError_t e = cudaMemcpyAsync(d_phases, phases.data(), phases.size() * sizeof(uint2), cudaMemcpyHostToDevice,
                                    h->stream);
    if (e == cudaSuccess && n_tracked)
        e = cudaMemcpyAsync(d_tracked, tracked, n_tracked * sizeof(uint32_t), cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess && n_tracked && losses)
        e = cudaMemcpyAsync(d_targets, targets, static_cast<size_t>(losses) * n_tracked * 3u * sizeof(double),
                            cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_cloth, &h->d, sizeof(DeviceCloth), cudaMemcpyHostToDevice, h->stream);
    const std::vector<uint8_t>* lists[4] = {&groups.d, &groups.k, &groups.b, &groups.g};
    uint8_t* dst[4] = {gd, gk, gb, gg};
    for (int f = 0; f < 4 && e == cudaSuccess; ++f)
        if (!lists[f]->empty())
            e = cudaMemcpyAsync(dst[f], lists[f]->data(), lists[f]->size(), cudaMemcpyHostToDevice, h->stream);
    if (e != cudaSuccess) return NUMI_CLOTH_ECUDA;

    auto save = [&](uint32_t slot) {
        size_t off = 0;
        for (const auto& r : h->dynamic) {
            if (cudaMemcpyAsync(ckpt + slot * state_bytes + off, r.ptr, r.bytes, cudaMemcpyDeviceToDevice, h->stream) !=
                cudaSuccess)
                return false;
            off += (r.bytes + 255u) & ~size_t(255u);
        }
        return true;
    };
    auto load = [&](uint32_t slot) {
        size_t off = 0;
        for (const auto& r : h->dynamic) {
            if (cudaMemcpyAsync(r.ptr, ckpt + slot * state_bytes + off, r.bytes, cudaMemcpyDeviceToDevice, h->stream) !=
                cudaSuccess)
                return false;
            off += (r.bytes + 255u) & ~size_t(255u);
        }
        return true;
    };

    // forward in the handle's own launch shape, checkpointing every segment
    std::vector<uint32_t> seg_epoch(segs);
    for (uint32_t g = 0; g < segs; ++g) {
        const uint32_t first = g * checkpoint_every;
        const uint32_t count = std::min(checkpoint_every, substeps - first);
        seg_epoch[g] = h->epoch;
        if (!save(g)) return NUMI_CLOTH_ECUDA;
        e = launch(h, count, s, first);
        h->epoch += count;
        if (e != cudaSuccess) {
            h->poisoned = true;
            return NUMI_CLOTH_ECUDA;
        }
    }
    const uint32_t end_epoch = h->epoch;
    if (!save(segs)) return NUMI_CLOTH_ECUDA;

    // backward: replay each segment on one CTA with the tape, then reverse it
    const float damping = h->d.damping >= 0.0f ? h->d.damping : s.damping;
    const bool resident_one = h->d.resident != 0u && h->grid == 1u;
    for (uint32_t g = segs; g-- > 0u;) {
        const uint32_t first = g * checkpoint_every;
        const uint32_t count = std::min(checkpoint_every, substeps - first);
        if (!load(g)) return NUMI_CLOTH_ECUDA;
        DeviceCloth d = h->d;
        d.cfg = h->d_cfg + first;
        d.epoch_base = seg_epoch[g];
        d.trace = nullptr;
        d.trace_cta = nullptr;
        d.cluster_barrier = 0u;
        d.resident = resident_one ? 1u : 0u;
        d.tape = tape;
        d.tape_v = tape_v;
        d.tape_slots = slots;
        Schedule st = s;
        st.substeps = count;
        const size_t smem = resident_one ? h->smem : nc_resident_offset();
        numi_cloth_frame_kernel<<<1, h->block, smem, h->stream>>>(d, st);
        AdjointArgs A{};
        A.cloth = d_cloth;
        A.cfg = h->d_cfg + first;
        A.tape = tape;
        A.tape_v = tape_v;
        A.phases = d_phases;
        A.slots = slots;
        A.substeps = count;
        A.first_substep = first;
        A.damping = damping;
        A.frictions = s.frictions;
        A.tracked = d_tracked;
        A.n_tracked = n_tracked;
        A.targets = d_targets;
        A.loss_every = loss_every;
        A.gx = gx;
        A.gv = gv;
        A.gprev = gprev;
        A.d_group = gd;
        A.k_group = gk;
        A.b_group = gb;
        A.g_group = gg;
        A.groups = ngroups;
        A.grads = d_out;
        A.loss = d_out + ngroups + 1u;
        A.grip_grads = d_grip;
        A.nonsmooth = d_rough;
        numi_cloth_adjoint_kernel<<<1, NC_THREADS, 0, h->stream>>>(A);
        if (cudaGetLastError() != cudaSuccess) {
            h->poisoned = true;
            return NUMI_CLOTH_ECUDA;
        }
        uint32_t barriers = 0;
        if (cudaMemcpyAsync(&barriers, h->d.stats, sizeof(uint32_t), cudaMemcpyDeviceToHost, h->stream) != cudaSuccess ||
            cudaStreamSynchronize(h->stream) != cudaSuccess) {
            h->poisoned = true;
            return NUMI_CLOTH_ECUDA;
        }
        if (barriers + 1u != slots) return NUMI_CLOTH_ESTATE;   // the phase list does not match the kernel
    }
    if (!load(segs)) return NUMI_CLOTH_ECUDA;
    h->epoch = end_epoch;
    std::vector<double> out(ngroups + 2u);
    unsigned int rough = 0;
    e = cudaMemcpyAsync(out.data(), d_out, out.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&rough, d_rough, sizeof(rough), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess && grip_grads)
        e = cudaMemcpyAsync(grip_grads, d_grip, static_cast<size_t>(substeps) * 6u * sizeof(double),
                            cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) {
        h->poisoned = true;
        return NUMI_CLOTH_ECUDA;
    }
    for (uint32_t k = 0; k <= ngroups; ++k) grads[k] = out[k];
    *loss = out[ngroups + 1u];
    if (nonsmooth) *nonsmooth = rough;
    return NUMI_CLOTH_OK;
}

// ------------------------------------------------------------------------
// Batched rollout gradients (numi_cloth_batch_rollout_grad): the forward of
// every cloth in one persistent launch per segment, the taped replays in one
// launch per segment, and the adjoint of every cloth's segment in one grid
// (a CTA per cloth).  Checkpoints are moved by one copy kernel per segment.

extern "C" int numi_cloth_batch_rollout_grad(numi_cloth_batch_t* b, const NumiClothConfig* configs, uint32_t substeps,
                                             const NumiClothSchedule* schedule, uint32_t checkpoint_every,
                                             const uint32_t* tracked, uint32_t n_tracked, const double* targets,
                                             uint32_t loss_every, double* loss, double* grads, uint32_t* groups_out,
                                             uint32_t* nonsmooth) {
    if (b == nullptr || configs == nullptr || schedule == nullptr || substeps == 0 || checkpoint_every == 0 ||
        loss == nullptr || grads == nullptr || loss_every == 0 || (n_tracked > 0 && (tracked == nullptr || targets == nullptr)))
        return NUMI_CLOTH_EINVAL;
    const NumiClothSchedule& sc = *schedule;
    if (sc.iterations != 1u || sc.reconcilePasses != 0u || sc.finalPasses != 0u || sc.certificatePasses != 0u ||
        sc.aerodynamics != 0u || sc.selfCollision != 0u || sc.primitiveSelf != 0u)
        return NUMI_CLOTH_EINVAL;
    cudaSetDevice(b->device);
    batch_drop_graph(b);
    const uint32_t count = static_cast<uint32_t>(b->cloths.size());
    for (numi_cloth* h : b->cloths)
        for (uint32_t t = 0; t < n_tracked; ++t)
            if (tracked[t] >= h->d.n) return NUMI_CLOTH_EINVAL;
    // Configs, descriptors (always rebuilt: damping and compliances may have
    // changed since the last launch)
    b->layout_valid = false;
    {
        const int rc = batch_prepare(b, configs, substeps, sc);
        if (rc > 0) return rc;
        if (rc != NUMI_CLOTH_OK) return rc;
    }
    cudaError_t e = cudaMemcpyAsync(b->d_cfg, configs, static_cast<size_t>(count) * substeps * sizeof(NumiClothConfig),
                                    cudaMemcpyHostToDevice, b->stream);
    if (e != cudaSuccess) return NUMI_CLOTH_ECUDA;
    const Schedule s = device_schedule(sc);
    const uint32_t segs = (substeps + checkpoint_every - 1u) / checkpoint_every;
    const uint32_t losses = substeps / loss_every;

    Scratch mem;
    // per cloth: groups, phase list, tape, checkpoints, adjoint arrays
    std::vector<Groups> groups(count);
    std::vector<std::vector<uint2>> phases(count);
    std::vector<size_t> state_bytes(count), tape_off(count), ckpt_off(count);
    size_t tape_total = 0, ckpt_total = 0;
    uint32_t max_slots = 0;
    for (uint32_t k = 0; k < count; ++k) {
        numi_cloth* h = b->cloths[k];
        const int rc = compliance_groups(h, groups[k]);
        if (rc != NUMI_CLOTH_OK) return rc;
        phases[k] = adjoint_phases(h->d, s);
        const uint32_t slots = static_cast<uint32_t>(phases[k].size()) + 1u;
        max_slots = std::max(max_slots, slots);
        tape_off[k] = tape_total;
        tape_total += static_cast<size_t>(checkpoint_every) * (slots + 1u) * h->d.n;   // positions + velocities
        size_t bytes = 0;
        for (const auto& r : h->dynamic) bytes += (r.bytes + 255u) & ~size_t(255u);
        state_bytes[k] = bytes;
        ckpt_off[k] = ckpt_total;
        ckpt_total += (segs + 1u) * bytes;
    }
    float4* tape = mem.get<float4>(tape_total);
    char* ckpt = mem.get<char>(ckpt_total);
    uint32_t* d_tracked = mem.get<uint32_t>(n_tracked);
    double* d_targets = mem.get<double>(static_cast<size_t>(count) * losses * n_tracked * 3u);
    double* d_out = mem.get<double>(static_cast<size_t>(count) * (NUMI_CLOTH_MAX_GROUPS + 2u));
    unsigned int* d_rough = mem.get<unsigned int>(count);
    DeviceCloth* d_replay = mem.get<DeviceCloth>(count);   // launch order, tape set
    DeviceCloth* d_plain = mem.get<DeviceCloth>(count);    // caller order, for the adjoint
    AdjointArgs* d_args = mem.get<AdjointArgs>(count);
    CopyOp* d_save = mem.get<CopyOp>(static_cast<size_t>(count) * 16u);
    if (!tape || !ckpt || !d_tracked || !d_targets || !d_out || !d_rough || !d_replay || !d_plain || !d_args || !d_save)
        return NUMI_CLOTH_ENOMEM;
    std::vector<AdjointArgs> args(count);
    std::vector<DeviceCloth> replay(count), plain(count);
    // one arena for every cloth's phase list, adjoint arrays and group ids
    auto round256 = [](size_t v) { return (v + 255u) & ~size_t(255u); };
    size_t arena_bytes = 0;
    for (uint32_t k = 0; k < count; ++k)
        arena_bytes += round256(phases[k].size() * sizeof(uint2)) + round256(3u * sizeof(double4) * b->cloths[k]->d.n) +
                       round256(groups[k].d.size() + 1u) + round256(groups[k].k.size() + 1u) +
                       round256(groups[k].b.size() + 1u) + round256(groups[k].g.size() + 1u);
    char* arena = mem.get<char>(arena_bytes);
    if (!arena) return NUMI_CLOTH_ENOMEM;
    size_t cursor = 0;
    auto carve = [&](size_t bytes) {
        char* p = arena + cursor;
        cursor += round256(bytes);
        return p;
    };
    for (uint32_t k = 0; k < count; ++k) {
        numi_cloth* h = b->cloths[k];
        const uint32_t n = h->d.n;
        const uint32_t slots = static_cast<uint32_t>(phases[k].size()) + 1u;
        uint2* ph = reinterpret_cast<uint2*>(carve(phases[k].size() * sizeof(uint2)));
        double4* gx = reinterpret_cast<double4*>(carve(3u * sizeof(double4) * n));
        uint8_t* gd = reinterpret_cast<uint8_t*>(carve(groups[k].d.size() + 1u));
        uint8_t* gk = reinterpret_cast<uint8_t*>(carve(groups[k].k.size() + 1u));
        uint8_t* gb = reinterpret_cast<uint8_t*>(carve(groups[k].b.size() + 1u));
        uint8_t* gg = reinterpret_cast<uint8_t*>(carve(groups[k].g.size() + 1u));
        e = cudaMemcpyAsync(ph, phases[k].data(), phases[k].size() * sizeof(uint2), cudaMemcpyHostToDevice, b->stream);
        const std::vector<uint8_t>* lists[4] = {&groups[k].d, &groups[k].k, &groups[k].b, &groups[k].g};
        uint8_t* dst[4] = {gd, gk, gb, gg};
        for (int f = 0; f < 4 && e == cudaSuccess; ++f)
            if (!lists[f]->empty())
                e = cudaMemcpyAsync(dst[f], lists[f]->data(), lists[f]->size(), cudaMemcpyHostToDevice, b->stream);
        if (e != cudaSuccess) return NUMI_CLOTH_ECUDA;
        plain[k] = h->d;
        AdjointArgs& A = args[k];
        A.cloth = d_plain + k;
        A.tape = tape + tape_off[k];
        A.tape_v = A.tape + static_cast<size_t>(checkpoint_every) * slots * n;
        A.phases = ph;
        A.slots = slots;
        A.damping = h->d.damping >= 0.0f ? h->d.damping : s.damping;
        A.frictions = s.frictions;
        A.tracked = d_tracked;
        A.n_tracked = n_tracked;
        A.targets = d_targets + static_cast<size_t>(k) * losses * n_tracked * 3u;
        A.loss_every = loss_every;
        A.gx = gx;
        A.gv = gx + n;
        A.gprev = gx + 2u * static_cast<size_t>(n);
        A.d_group = gd;
        A.k_group = gk;
        A.b_group = gb;
        A.g_group = gg;
        A.groups = static_cast<uint32_t>(groups[k].value.size());
        A.grads = d_out + static_cast<size_t>(k) * (NUMI_CLOTH_MAX_GROUPS + 2u);
        A.loss = A.grads + NUMI_CLOTH_MAX_GROUPS + 1u;
        A.grip_grads = nullptr;
        A.nonsmooth = d_rough + k;
    }
    // replay descriptors: the batch's launch-order descriptors with tapes
    {
        std::vector<DeviceCloth> base(count);
        e = cudaMemcpy(base.data(), b->d_cloths, count * sizeof(DeviceCloth), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return NUMI_CLOTH_ECUDA;
        for (uint32_t j = 0; j < count; ++j) {
            const uint32_t k = b->order[j];
            replay[j] = base[j];
            replay[j].tape = const_cast<float4*>(args[k].tape);
            replay[j].tape_v = const_cast<float4*>(args[k].tape_v);
            replay[j].tape_slots = args[k].slots;
        }
    }
    e = cudaMemcpyAsync(d_replay, replay.data(), count * sizeof(DeviceCloth), cudaMemcpyHostToDevice, b->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_plain, plain.data(), count * sizeof(DeviceCloth), cudaMemcpyHostToDevice, b->stream);
    if (e == cudaSuccess && n_tracked)
        e = cudaMemcpyAsync(d_tracked, tracked, n_tracked * sizeof(uint32_t), cudaMemcpyHostToDevice, b->stream);
    if (e == cudaSuccess && n_tracked && losses)
        e = cudaMemcpyAsync(d_targets, targets, static_cast<size_t>(count) * losses * n_tracked * 3u * sizeof(double),
                            cudaMemcpyHostToDevice, b->stream);
    if (e != cudaSuccess) return NUMI_CLOTH_ECUDA;

    // one copy kernel per checkpoint move: op tables for save (state ->
    // checkpoint) and load (checkpoint -> state) of every slot
    std::vector<CopyOp> save_ops, load_ops;
    uint32_t regions = 0;
    for (numi_cloth* h : b->cloths) regions += static_cast<uint32_t>(h->dynamic.size());
    CopyOp* d_ops = mem.get<CopyOp>(2u * static_cast<size_t>(segs + 1u) * regions);
    if (!d_ops) return NUMI_CLOTH_ENOMEM;
    for (uint32_t g = 0; g <= segs; ++g) {
        for (uint32_t k = 0; k < count; ++k) {
            numi_cloth* h = b->cloths[k];
            size_t off = 0;
            for (const auto& r : h->dynamic) {
                char* slot = ckpt + ckpt_off[k] + g * state_bytes[k] + off;
                save_ops.push_back(CopyOp{r.ptr, slot, r.bytes});
                load_ops.push_back(CopyOp{slot, r.ptr, r.bytes});
                off += (r.bytes + 255u) & ~size_t(255u);
            }
        }
    }
    e = cudaMemcpyAsync(d_ops, save_ops.data(), save_ops.size() * sizeof(CopyOp), cudaMemcpyHostToDevice, b->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_ops + save_ops.size(), load_ops.data(), load_ops.size() * sizeof(CopyOp),
                            cudaMemcpyHostToDevice, b->stream);
    if (e != cudaSuccess) return NUMI_CLOTH_ECUDA;
    auto move = [&](bool save, uint32_t g) {
        const CopyOp* ops = d_ops + (save ? 0u : save_ops.size()) + static_cast<size_t>(g) * regions;
        numi_cloth_copy_kernel<<<regions, 256, 0, b->stream>>>(ops);
    };
    auto set_epoch = [&](uint32_t value) {
        return cudaMemcpyAsync(b->epoch, &value, sizeof(uint32_t), cudaMemcpyHostToDevice, b->stream) == cudaSuccess &&
               cudaStreamSynchronize(b->stream) == cudaSuccess;
    };

    // forward
    std::vector<uint32_t> seg_epoch(segs);
    const uint32_t epoch0 = b->epoch_host;
    if (!set_epoch(epoch0)) return NUMI_CLOTH_ECUDA;
    for (uint32_t g = 0; g < segs; ++g) {
        const uint32_t first = g * checkpoint_every;
        const uint32_t cnt = std::min(checkpoint_every, substeps - first);
        seg_epoch[g] = epoch0 + first;
        move(true, g);
        Schedule st = s;
        st.substeps = cnt;
        st.cfg_offset = first;
        st.epoch_ptr = b->epoch;
        cudaMemsetAsync(b->queue, 0, sizeof(unsigned int), b->stream);
        numi_cloth_batch_kernel<<<b->ctas, b->block, b->smem, b->stream>>>(b->d_cloths, count, st, b->queue);
        numi_cloth_epoch_kernel<<<1, 1, 0, b->stream>>>(b->epoch, cnt);
    }
    move(true, segs);
    // backward
    for (uint32_t g = segs; g-- > 0u;) {
        const uint32_t first = g * checkpoint_every;
        const uint32_t cnt = std::min(checkpoint_every, substeps - first);
        move(false, g);
        if (!set_epoch(seg_epoch[g])) return NUMI_CLOTH_ECUDA;
        Schedule st = s;
        st.substeps = cnt;
        st.cfg_offset = first;
        st.epoch_ptr = b->epoch;
        cudaMemsetAsync(b->queue, 0, sizeof(unsigned int), b->stream);
        numi_cloth_batch_kernel<<<b->ctas, b->block, b->smem, b->stream>>>(d_replay, count, st, b->queue);
        for (uint32_t k = 0; k < count; ++k) {
            args[k].cfg = b->d_cfg + static_cast<size_t>(k) * substeps + first;
            args[k].substeps = cnt;
            args[k].first_substep = first;
        }
        e = cudaMemcpyAsync(d_args, args.data(), count * sizeof(AdjointArgs), cudaMemcpyHostToDevice, b->stream);
        if (e != cudaSuccess) return NUMI_CLOTH_ECUDA;
        numi_cloth_adjoint_batch_kernel<<<count, NC_THREADS, 0, b->stream>>>(d_args);
        // args is rewritten next segment: wait for this copy to be consumed
        if (cudaStreamSynchronize(b->stream) != cudaSuccess) {
            for (numi_cloth* h : b->cloths) h->poisoned = true;
            return NUMI_CLOTH_ECUDA;
        }
    }
    move(false, segs);
    const uint32_t end_epoch = epoch0 + substeps;
    if (!set_epoch(end_epoch)) return NUMI_CLOTH_ECUDA;
    b->epoch_host = end_epoch;
    for (numi_cloth* h : b->cloths) {
        h->epoch = end_epoch;
        h->last_substeps = substeps;
    }
    std::vector<double> out(static_cast<size_t>(count) * (NUMI_CLOTH_MAX_GROUPS + 2u));
    std::vector<unsigned int> rough(count);
    e = cudaMemcpyAsync(out.data(), d_out, out.size() * sizeof(double), cudaMemcpyDeviceToHost, b->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(rough.data(), d_rough, count * sizeof(unsigned int), cudaMemcpyDeviceToHost, b->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
    if (e != cudaSuccess) {
        for (numi_cloth* h : b->cloths) h->poisoned = true;
        return NUMI_CLOTH_ECUDA;
    }
    for (uint32_t k = 0; k < count; ++k) {
        const double* o = out.data() + static_cast<size_t>(k) * (NUMI_CLOTH_MAX_GROUPS + 2u);
        for (uint32_t q = 0; q <= NUMI_CLOTH_MAX_GROUPS; ++q) grads[static_cast<size_t>(k) * (NUMI_CLOTH_MAX_GROUPS + 1u) + q] = o[q];
        loss[k] = o[NUMI_CLOTH_MAX_GROUPS + 1u];
        if (groups_out) groups_out[k] = static_cast<uint32_t>(groups[k].value.size());
        if (nonsmooth) nonsmooth[k] = rough[k];
    }
    return NUMI_CLOTH_OK;
}
