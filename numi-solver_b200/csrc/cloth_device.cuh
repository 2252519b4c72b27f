// Device-side layout of one cloth solver handle.
//
// HBM layout (structure of arrays; every array is 16-byte aligned):
//   x      float4[N]  position xyz, inverse mass w
//   xp     float4[N]  position at substep start xyz, mass w
//   v      float4[N]  velocity xyz; w holds the predicted vertical velocity
//                     during a substep and the cloth/ground normal impulse
//                     after finalize (the reference's velocity.w)
//   rest   float4[N]  rest position xyz (used for inverse mass 0)
//   dist   uint2 ij[D], float4 mat[D] (rest, compliance, -, max extension),
//          float lambda[D]
//   knot   uint4 ij[K], float2 mat[K] (rest cosine, compliance), float lambda[K]
//   bend   uint4 ij[B] (first, middle, third, -), float2 mat[B]
//          (rest chord, compliance), float lambda[B]
//   grips / fruits / fruit pairs keep the 48/96/32-byte ABI records (tiny).
// Constraint arrays are grouped by colour; a batch is a contiguous run.
#pragma once

#include <stdint.h>

#include "numi_cloth.h"

#define NC_MAX_FRUITS 64u
#define NC_MAX_GRIPS 32u
#define NC_MAX_BATCHES 64u
#define NC_YARN_SLOTS 4u
#define NC_MAX_PAIRS 2016u
#define NC_TRACE_SLOTS 128u
#define NC_HASH_CAP 8u      /* particles one self-contact bucket holds */
#define NC_FRICTION_STAGE 128u   /* recorded segments the staged friction sweep holds */

struct Batch {
    uint32_t first;
    uint32_t count;      // all records of the colour
    uint32_t limited;    // leading records that may carry a strain limit
    uint32_t yarn;       // leading records that are yarn segments
};

// One particle in the self-contact grid: its start-of-pass position and,
// in w, its index (bits); two slots per 32-byte sector.
struct __align__(16) HashSlot {
    float4 pos;
};

// One edge/edge pair record of a substep (SelfEdgeEdgeContactImpulse,
// tools/cloth_bag.cpp:3962-3985): the two yarn segments and the sums of
// their solves' impulse-weighted normal on the first segment, barycentric
// weights and normal impulse.
struct EdgeRecord {
    uint32_t i, j;
    float wn[3];
    float wf[2], ws[2];
    float ni;
};

struct DeviceCloth {
    // particles
    float4* x;
    float4* xp;
    float4* v;
    const float4* rest;
    uint32_t n;
    // distances
    const uint2* d_ij;
    const float4* d_mat;
    float* d_lambda;
    uint32_t d_count;
    // knots
    const uint4* k_ij;
    const float2* k_mat;
    float* k_lambda;
    uint32_t k_count;
    // bends
    const uint4* b_ij;
    const float2* b_mat;
    float* b_lambda;
    uint32_t b_count;
    // grips, fruits, pairs (ABI records)
    NumiClothGrip* grips;
    uint32_t g_count;
    NumiClothFruit* fruits;
    uint32_t f_count;
    NumiClothFruitPair* pairs;
    uint32_t p_count;
    const uint32_t* cuff;
    const uint32_t* rim;           // ordered mouth-rim particles (Config mouthControl.x of them)
    uint32_t* release;             // [0] mouth candidates, [1] released fruits (sticky bit masks)
    // fruit/yarn contact records, NC_YARN_SLOTS per yarn segment:
    //   a = (impulse-weighted normal on the fruit xyz, normal impulse)
    //   b = (impulse-weighted segment weights xy, tag bits, 0)
    // tag = (substep epoch << 6) | fruit; a record is live only while its
    // epoch is the current substep, so nothing is cleared between substeps.
    float4* yarn_slot_a;
    float4* yarn_slot_b;
    // substep epoch of the latest fruit/yarn contact record of each segment
    uint32_t* yarn_live;
    // segments recorded this substep, each once, in no particular order (the
    // friction sweep picks each colour's own), and their count
    uint32_t* yarn_list;
    uint32_t* yarn_list_n;
    // per-particle yarn air force of the current substep
    float4* force;
    // 2^-40 fixed-point fruit sums (int64 two's complement):
    // [0, 3*64) displacement xyz, [3*64, 9*64) velocity and spin xyz
    float4* fruit_partial;
    // batches
    Batch dist_batches[NC_MAX_BATCHES];
    Batch knot_batches[NC_MAX_BATCHES];
    Batch bend_batches[NC_MAX_BATCHES];
    Batch pair_batches[NC_MAX_BATCHES];
    uint32_t n_dist_batches, n_knot_batches, n_bend_batches, n_pair_batches;
    // configs for this launch
    const NumiClothConfig* cfg;
    // control
    unsigned int* failure;
    // grid barrier: monotonically increasing arrival counter (reset to 0 by
    // the host before every launch) and a sticky abort flag
    unsigned long long* bar_count;
    unsigned long long* bar_flag;   // barrier number released last (own 128-byte line)
    unsigned long long* fruit_flag; // tile mode: substeps whose fruit-CTA tail is done (own line)
    unsigned int* abort_flag;
    // polls a barrier or neighbour wait makes before it gives up (0: the
    // default NC_BARRIER_SPIN_LIMIT)
    uint32_t spin_limit;
    // failure-path tests only: grid barriers also wait for this many CTAs
    // that do not exist, so every bounded wait runs out (0 in production)
    uint32_t bar_phantom;
    // optional per-barrier globaltimer trace: [substep][NC_TRACE_SLOTS]
    unsigned long long* trace;
    // optional per-CTA barrier arrival stamps: [substep][NC_TRACE_SLOTS][grid]
    unsigned long long* trace_cta;
    // 1: the grid is one thread-block cluster and phases are separated by
    // the hardware cluster barrier instead of the global-memory barrier
    uint32_t cluster_barrier;
    // Neighbour syncs between constraint colours (cooperative grid, particles
    // in global memory): CTA r solves, in every colour, the items whose
    // lowest particle lies in its equal share of the particle range (its
    // list: nbr_items[nbr_block[r] .. nbr_block[r + 1]], colour_slots + 1
    // offsets then batch-relative item indices), and between two colours
    // waits only for the CTAs whose items share a particle with its own in
    // any colour (nbr_idx[nbr_off[r] .. nbr_off[r + 1]]).
    // nbr_flag[32 r] counts the colours CTA r has finished in the launch
    // (zeroed before every launch).
    uint32_t nbr_on;
    uint32_t colour_slots;         // distance + knot + bend batches
    const uint32_t* nbr_block;     // [grid + 1]
    const uint32_t* nbr_items;
    const uint32_t* nbr_off;       // [grid + 1]
    const uint32_t* nbr_idx;
    unsigned int* nbr_flag;        // [32 * grid]
    // resident mode: 1 when particle positions and velocities live in the
    // (distributed) shared memory of the grid's CTAs for the whole launch;
    // CTA r owns particles [r << resident_shift, (r + 1) << resident_shift)
    uint32_t resident;
    uint32_t resident_shift;
    double* red;          // [blocks * 8] reduction partials
    uint32_t* stats;      // [0] barriers of the last substep, [1] reconcile passes max, [2] certificate passes max
    uint32_t epoch_base;  // substep counter of the handle at launch
    float damping;        // velocity damping c of v <- v / (1 + c dt); < 0: the schedule's
    uint32_t grid_width;  // row-major grid topology (square cloth) or 0
    const uint32_t* local_off;
    const uint32_t* local_idx;
    // point self-contact hash grid: cells of twice the contact distance,
    // hashed into hash_mask + 1 buckets (about two per particle) of
    // NC_HASH_CAP slots; a bucket head is (pass tag << 32) | count, so
    // buckets of older passes read as empty and nothing is cleared between
    // passes
    unsigned long long* hash_head;
    HashSlot* hash;       // [buckets * NC_HASH_CAP]
    // particles whose bucket was full: (pass tag << 32) | count, and [n]
    // slots, so no particle is ever dropped
    unsigned long long* hash_over_head;
    HashSlot* hash_over;
    uint32_t hash_mask;
    // [0] self contacts (a < b pairs resolved), [1] max self penetration
    // (float bits; non-negative so unsigned max orders them)
    unsigned long long* self_stats;
    // point self contact in the reference order: pairs phase A lists for the
    // ordered pass (two entries each: start position, index | known bit),
    // the list head (tag << 32 | entries), this pass's statistics, sort keys
    // (self_key_cap, then room for one particle's turn), and per particle
    // the ordered pass's marks (tag << 32 | bits), start positions and
    // largest displacements
    float4* self_list;
    unsigned long long* self_list_head;
    uint32_t self_list_cap;
    unsigned long long* self_pass_stats;
    unsigned long long* self_keys;
    uint32_t self_key_cap;
    unsigned long long* self_mark;
    float4* self_x0;
    float* self_disp;
    // edge/edge yarn self-collision.  Yarn segments: the distances that are
    // not shear diagonals, in array order.  Buffers (allocated on first use):
    //   pair list: every non-local segment pair (first < second) within the
    //     yarn diameter plus the skin at its build, the positions of the
    //     build, and for the build a hashed cell grid sorted by counting
    //     (per-bucket counts and offsets, the cells' entries: segment, lower
    //     cell corner key, spans) with a list of segments too long for it;
    //   pass: the pass-start positions and spheres, each particle's path
    //     length, the candidates (first, second, distance bound bits, ordered
    //     flag), the keys (first << 32 | second) of the ordered pairs and
    //     their sorted copy, the pass's records and the substep's records
    //     (ascending keys)
    const uint2* y_ij;
    uint32_t y_count;
    uint32_t edge_mask;
    float edge_cell;
    uint32_t edge_cap;            // candidates, ordered pairs, records
    uint32_t edge_list_cap;       // pairs on the list
    uint32_t* edge_count;         // [buckets]
    uint32_t* edge_offs;          // [buckets], within the bucket's scan chunk
    uint32_t* edge_chunk_total;   // [CTAs] entries of each CTA's chunk of buckets
    float4* edge_entries;         // [2 * 27 * y_count] grown box per entry, segment index in the first w
    uint32_t* edge_giant;         // [y_count] segments the grid does not hold
    float4* edge_bbox;            // [2 * y_count] grown boxes of the build
    const uint32_t* edge_loc_off; // [y_count + 1] CSR of every segment's local segments of higher index
    const uint32_t* edge_loc_idx; //   (ascending)
    uint2* edge_pairs;            // [edge_list_cap]
    float4* edge_xb;              // [n] positions at the build
    float4* edge_pb;              // [n] substep-start positions at the build
    float* edge_built_radius;     // yarn radius of the build
    float4* edge_x0;              // [n]
    float4* edge_sph;             // [y_count] pass spheres (centre, radius)
    float* edge_qbox_raw;         // [6 * y_count] a first segment's tree-query box of the pass
    uint32_t* edge_tree;          // [14 * y_count] the pass's box-tree leaf order: position -> segment,
                                  //   then segment -> position, the build's scratch and the last
                                  //   build's axis orders (edge_tree_order)
    float4* edge_centre;          // [2 * y_count] centres of the pass-start boxes of the tree, then
                                  //   those of the last build
    float* edge_path;             // [n]
    uint4* edge_cand;             // [edge_cap]
    unsigned long long* edge_order;    // [edge_cap]
    unsigned long long* edge_sorted;   // [edge_cap]
    EdgeRecord* edge_new;         // [edge_cap] records of the pass's ordered pairs, by sorted index
    uint32_t* edge_done;          // [edge_cap] sorted indices of the pairs that moved, ascending
    uint32_t* edge_lv;            // [edge_cap] wavefront level of each ordered pair (+ first / moved bits)
    uint32_t* edge_level;         // [n] last wavefront level of each particle (zero between passes)
    EdgeRecord* edge_rec;         // [edge_cap]
    // [0] candidates, [1] ordered pairs, [2] violations found (only grows),
    // [3] records of the substep, [4] records of the pass, [5] pairs on the
    // list, [6] 1 once the list is built, [7] long segments of the build
    uint32_t* edge_ctl;
    // [0] edge/edge contacts resolved, [1] self-friction contacts
    unsigned long long* edge_stats;
    // [0, CTAs) deepest non-local pair of the last measure, [CTAs, 2 CTAs)
    // largest displacement since the build, [2 CTAs, 3 CTAs) largest motion
    // over the substep
    double* edge_red;
    // adjoint tape (one-CTA launches only): positions at the start of every
    // substep and after every barrier, [substep][tape_slots][n], and
    // velocities at the start of every substep, [substep][n]
    float4* tape;
    float4* tape_v;
    uint32_t tape_slots;
    // tile mode of the cooperative grid (cloth_tile.cuh): CTA r's plan is
    // tile_words[tile_off[r] .. tile_off[r + 1]); tile_owner[i] = (owning
    // CTA << 16) | local index of particle i; positions and velocities
    // alternate between x, v and x_alt, v_alt
    const uint32_t* tile_off;
    const uint32_t* tile_words;
    const uint32_t* tile_owner;
    float4* x_alt;
    float4* v_alt;
    // allocation-free launches: [n + NC_MAX_FRUITS] words of scratch; when
    // set, the launch first checks every record's indices and the colouring
    // of every run (validate_records) and steps nothing if one is wrong
    uint32_t* check_stamp;
};

struct Schedule {
    uint32_t iterations;
    uint32_t strain_sweeps;
    uint32_t reconcile_passes;
    uint32_t final_passes;
    uint32_t certificate_passes;
    uint32_t early_exit;
    uint32_t self_collision;
    uint32_t aerodynamics;
    uint32_t swept_ground;
    uint32_t swept_fruit_yarn;
    uint32_t frictions;
    uint32_t release;
    float damping;
    uint32_t substeps;
    uint32_t primitive_self;   // edge/edge yarn self-collision and self friction
    // batch launches: the substep counter of the batch in device memory
    // (advanced by a kernel after each launch, so a captured graph can be
    // replayed); null: DeviceCloth::epoch_base
    const uint32_t* epoch_ptr;
    // first Config of the launch within DeviceCloth::cfg
    uint32_t cfg_offset;
    // 1: the launch runs in tile mode (cloth_tile.cuh)
    uint32_t tiles;
    // edge/edge launches: byte offset in dynamic shared memory of the box
    // tree's sort keys (edge_tree_order), 0 when the launch has none
    uint32_t tree_keys;
};

// Fruit-side state kept in the shared memory of the fruit CTA for a whole
// launch: compact pair indices (loaded once) and the pair contact impulses
// of the current substep (the only readers and writers are fruit-CTA
// phases), plus staging for the fruit sweeps.
struct FruitShared {
    unsigned short ab[NC_MAX_PAIRS];       // fruit a | fruit b << 8, colour order
    float4 contact[NC_MAX_PAIRS];          // weighted normal xyz, normal impulse
    float4 fx[NC_MAX_FRUITS];              // position xyz, inverse mass
    float fr[NC_MAX_FRUITS];               // radius
    float4 v[NC_MAX_FRUITS];               // velocity xyz, inverse mass
    float4 o[NC_MAX_FRUITS];               // spin xyz, radius
    unsigned long long loaded;             // pair colours with an impulse this substep
};

// The fruit/yarn friction sweep's recorded segments, staged by the fruit CTA
// in tile mode (friction_stage, after FruitShared in its shared memory):
// segment, slot tags and records, endpoint particles, for every endpoint
// the first endpoint slot with the same particle, endpoint positions and
// velocities.
struct FrictionStage {
    uint32_t count;                        // staged segments (NC_FRICTION_STAGE + 1: too many)
    uint32_t seg[NC_FRICTION_STAGE];
    uint32_t tag[NC_FRICTION_STAGE][NC_YARN_SLOTS];
    uint32_t pid[2 * NC_FRICTION_STAGE];
    unsigned short rep[2 * NC_FRICTION_STAGE];
    float4 x[2 * NC_FRICTION_STAGE];
    float4 v[2 * NC_FRICTION_STAGE];
    float4 ra[NC_FRICTION_STAGE][NC_YARN_SLOTS];
    float4 rb[NC_FRICTION_STAGE][NC_YARN_SLOTS];
};
