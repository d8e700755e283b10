// Per-element bodies of the TERRAIN-step kernels (host + device).
//
// Each body computes one work item of one kernel from the Batch it is given, so the
// sm_100a kernels in terrain.cu are one-line wrappers, and a test-only host build can
// run the same bodies to check generated code on the CPU.
//
// Stage -> reference (cpu/src/terrain.cpp unless noted):
//   biome chunks      cpu_chunk_biomes :152-176 (climate, quantize, R-tree chain)
//   corner channels   VolumeEvaluator::sample_interpolated_block_step, volume_eval.cpp:619-674
//   surface levels    Aquifer::max_surface_level / surface_level :307-331 (volume vs point)
//   aquifer cells     Aquifer location / compute_fluid :225-241, :343-408
//   fill              cpu_terrain_from_biomes :782-805, Aquifer::compute_substance :217-272
//   surface           Surface::build :477-522 and its extensions :677-725
#pragma once

#include <climits>

#include "model_gen.cuh"
#include "tb_host.h"

namespace tb {

constexpr int kQuartsPerChunk = 16 * (tbm::kHeight / 4);
constexpr int kBlocksPerChunk = 256 * tbm::kHeight;
constexpr int kRows = tbm::kHeight / 8 + 1;              // 4x8 cell corner rows
constexpr int kCellsY = tbm::kHeight / 8;
constexpr int kMaxY = tbm::kMinY + tbm::kHeight - 1;
// Column masks: 32 heights per word, air words then fluid words.
constexpr int kMaskWords = tbm::kHeight / 32;
static_assert(tbm::kHeight % 32 == 0, "column mask words");
// Per-block bytes the column walk reads (zoomed biome, ore-vein bits) in column order: 4
// heights per 32-bit word, word (y - kMinY) >> 2 of column lz * 16 + lx at
// (c * kColWords + word) * 256 + column, byte (y - kMinY) & 3 of it (little-endian), so that
// a warp's 32 columns read 128 contiguous bytes per 4 heights.
constexpr int kColWords = tbm::kHeight / 4;
TB_HD TB_FI size_t colbyte(int c, int col, int y) {
    const int r = y - tbm::kMinY;
    return ((static_cast<size_t>(c) * kColWords + (r >> 2)) * 256 + col) * 4 + (r & 3);
}
constexpr int kGridX = 27, kGridZ = 19, kGrid = kGridX * kGridZ;   // surface-level quarts per chunk
constexpr int kAqX = 3, kAqY = 35, kAqZ = 3, kAqCells = kAqX * kAqY * kAqZ;
constexpr int kAqMinGridY = -7;
// Nearest-cell queries per chunk: the lowest of the three candidate layers (33 for the world
// height) x the two x and two z candidate columns a block of the chunk can start from.
constexpr int kAqQueryLayers = kAqY - 2, kAqQueries = kAqQueryLayers * 4;
constexpr int kWayBelowMinY = -2032 * 16;   // DimensionType.WAY_BELOW_MIN_Y
constexpr int kMaxGradientRandoms = 8;
constexpr int kSearchStack = 16;
// quart vertices a chunk's BiomeManager lookups can reach: x and z from 4c - 1 to 4c + 4,
// y from ((min_y - 2) >> 2) to ((max_y + 1 - 2) >> 2) + 1
constexpr int kZoomQyMin = (tbm::kMinY - 2) >> 2;
constexpr int kZoomQyMax = ((tbm::kMinY + tbm::kHeight - 2) >> 2) + 1;
constexpr int kZoomY = kZoomQyMax - kZoomQyMin + 1;
constexpr int kZoomVerts = 36 * kZoomY;
static_assert(tbm::kNumGradientRandoms <= kMaxGradientRandoms, "too many vertical-gradient random names");
static_assert(tbm::kHeight % 16 == 0 && tbm::kMinY % 16 == 0, "world height must be section aligned");

// ---- device-resident model and per-seed tables -------------------------------------------------
struct DevModel {
    const RBox* boxes;              // null when the 32-bit search does not apply; root is box 0
    const int32_t* box_leaf;        // parameter index -> box index
    const RNode* tree;
    const int32_t* children;
    const int32_t* leaf_biome;
    const int32_t* leaf_node;
    const int32_t* leaf_rank;
    int32_t root;
    int32_t depth;                  // levels of the climate tree (root = 1)
    const uint8_t* block_flags;     // 1 air, 2 water, 4 lava, 8 fluid
    const float* biome_temp;
    const uint8_t* biome_frozen;
    Simplex2 temp, frozen[3], info;
    float frozen_amp[3];
    double f2, g2;
};

struct DevSeed {
    NoiseTables nt;
    const AxisRec* ytab;   // per corner row, the y record of each corner-context volume layer
    Positional random, aquifer, ore;
    Positional gradient[kMaxGradientRandoms];
    int64_t zoom_seed;
    uint16_t clay[192];
};

// Open-addressing table deduplicating 64-bit position keys; unique keys get dense
// indices in insertion order of the winning thread.
// Open-addressing key set of one dedupe stage. Inserting records, per slot, the least item
// that inserted the key; compaction then numbers the keys in the order of those first items
// (uniq), so neighbouring entries of uniq come from neighbouring items (nearby chunks).
struct HashTab {
    unsigned long long* keys;   // kEmpty when free
    int32_t* vals;
    unsigned long long* uniq;
    int32_t* count;
    uint32_t mask;
    int32_t* owner;             // per slot: least inserting item (INT32_MAX-like when free)
    uint32_t* err;              // sticky error bits of the lane: kErrTableFull, kErrKeyMissing
};
// Device-side error bits, read by the host after the work: the tables are sized so that
// neither can happen (capacity >= 2 x the keys a batch can insert); they turn a broken
// invariant into an error status instead of a silent wrong index.
constexpr uint32_t kErrTableFull = 1u;    // an insert's probe sequence met no free slot
constexpr uint32_t kErrKeyMissing = 2u;   // a resolve did not find its key (index 0 used instead)
constexpr unsigned long long kEmpty = ~0ull;

// One aquifer grid cell (NoiseBasedAquifer's aquiferLocationCache and aquiferCache entries
// together): its jittered location and its fluid status packed as level * 4 + fluid block,
// 16 bytes so that the nearest-cell scan reads a cell with one vector load.
struct alignas(16) AqCell {
    int32_t x, y, z, st;
};

// What the 12 candidate cells of one nearest-cell query decide without their distances:
// the status all of them share (kAqMixed when they differ) and the height from which every
// block is air (the highest level + 5).
struct alignas(8) AqQuery {
    int32_t uni, air_from;
};
constexpr int32_t kAqMixed = INT32_MIN;   // no status packs to it (fluid blocks are 2 or 3)

struct Batch {
    DevModel M;
    const DevSeed* seeds;
    const int32_t* n_dev;             // chunks in the batch (device memory, so one graph serves any size)
    const int32_t* cx;                // chunk coordinates, seed slot
    const int32_t* cz;
    const int32_t* cseed;
    // biome chunks: the union of the 3x3 neighbourhoods
    HashTab hb;
    int32_t nb_cap;
    int32_t* nb9;                     // n * 9 biome-chunk indices, (dz + 1) * 3 + dx + 1
    float* bcol;                      // nb_cap * 16 * kClimateCols
    long long* tgt;                   // nb_cap * kQuartsPerChunk * 6, chain order
    int32_t* lstar;                   // first minimal leaf per quart, chain order
    long long* mdist;                 // its distance
    uint8_t* qbiome;                  // nb_cap * kQuartsPerChunk, (qy * 4 + qz) * 4 + qx
    // corner columns of the 4x8 channels
    HashTab hc;
    int32_t cc_cap;
    int32_t* c25;                     // n * 25 corner-column indices, (k) * 5 + i
    float* ccol;                      // cc_cap * kCornerCols
    // per-batch axis tables of the corner kernel: the distinct corner x (and z) coordinates
    // of each seed slot, and per coordinate the x (z) record of every axis-table layer
    HashTab ha;                       // keys (slot, qx, 0, 0) and (slot, 0, qz, 1)
    AxisRec* axtab;                   // ha's keys * kAxisLayers
    int32_t* colax;                   // cc_cap * 2: per corner column its x row and z row of axtab
    float* corners;                   // cc_cap * kRows * kNumChannels
    // surface-level quarts (find_top_surface), volume or point semantics
    HashTab hs;
    int32_t sg_cap;
    int32_t* g513;                    // n * kGrid indices
    float* sfts;                      // sg_cap: find_top_surface value per unique quart
    // aquifer
    AqCell* aq_cell;                  // n * kAqCells, (iy * kAqZ + iz) * kAqX + ix
    AqQuery* aq_query;                // n * kAqQueries, (layer * 2 + z column) * 2 + x column
    int32_t* aq_skip;                 // n
    // outputs and heights
    uint16_t* blocks;                 // n * kBlocksPerChunk
    float* density;                   // optional n * kBlocksPerChunk final density per block (block layout)
    int32_t* h0;                      // n * 256, x * 16 + z: heights after the fill
    int32_t* h1;                      // after the eroded-badlands extension
    int32_t* h2;                      // after the frozen-ocean extension (dry run)
    uint8_t* biomes_out;              // n * kQuartsPerChunk
    uint32_t* zoom_tab;               // n * kZoomVerts packed fiddle draws per quart vertex
    uint8_t* zoom_uni;                // n * kZoomCells: the biome all 8 corners of a zoom cell store, or kZoomMixed
    uint8_t* bbiome;                  // n * kBlocksPerChunk zoomed biome per block up to the column height, colbyte order
    uint8_t* oremask;                 // n * kBlocksPerChunk ore-vein density tests passed, bit per vein, colbyte order
    uint32_t* colmask;                // n * 2 * kMaskWords * 256: word w of column lz * 16 + lx at
                                      // (c * 2 * kMaskWords + w) * 256 + column; words below
                                      // kMaskWords hold air, the rest fluid; bit k = y kMinY + 32 w + k
    struct ColumnRec* colrec;         // n * 256 per-column surface context
    struct DeferRec* defer;           // blocks the walk leaves to the deferred pass (nullptr: none)
    int32_t* defer_count;             // blocks appended (may pass defer_cap; the rest stay in the walk)
    int32_t defer_cap;
};

// Per-column context of the material rules (MaterialSystem column state).
struct ColumnRec {
    double secondary;                 // surface_secondary noise at (x, 0, z)
    int32_t surface_depth, min_surface, grad_x, grad_z;
    int32_t surface_biome, start_h;
};
// A block whose rule evaluation reaches a per-block noise or an ore vein past its density
// bit: the walk's inputs to the rules, for the deferred pass (body_walk_deferred).
struct DeferRec {
    int32_t column;                   // chunk * 256 + x * 16 + z
    int16_t y, stone_above, stone_below, water_height;   // water_height kNoWater for none
    uint8_t biome, ore_bits;
    uint16_t pad;
};
constexpr int16_t kNoWater = INT16_MIN;
#ifndef TB_DEFER_ORE
#define TB_DEFER_ORE 0   // also defer blocks that reach an ore vein past its density bit
#endif

// Per block, bit k: whether ore vein k's density test passes (its density is not <= 0),
// decided by the fill from the channel values it already holds, so that the rule tree
// interpolates channels only inside veins.
#ifndef TB_ORE_MASK
#define TB_ORE_MASK (tbm::kNumOres <= 8)
#endif

// ---- atomics (device) / plain operations (host test build) --------------------------------------
TB_HD TB_FI unsigned long long cas64(unsigned long long* p, unsigned long long cmp, unsigned long long val) {
#if defined(__CUDA_ARCH__)
    return atomicCAS(p, cmp, val);
#else
    const unsigned long long old = *p;
    if (old == cmp) *p = val;
    return old;
#endif
}
TB_HD TB_FI int32_t add32(int32_t* p, int32_t v) {
#if defined(__CUDA_ARCH__)
    return atomicAdd(p, v);
#else
    const int32_t old = *p;
    *p += v;
    return old;
#endif
}
// The largest v over the warp's lanes that run together here (device) or v itself (host
// build, where items run one at a time). Either way the result is at least v.
TB_HD TB_FI int warp_max(int v) {
#if defined(__CUDA_ARCH__)
    return __reduce_max_sync(__activemask(), v);
#else
    return v;
#endif
}
TB_HD TB_FI void min32(int32_t* p, int32_t v) {
#if defined(__CUDA_ARCH__)
    atomicMin(p, v);
#else
    if (v < *p) *p = v;
#endif
}
TB_HD TB_FI void or32(uint32_t* p, uint32_t v) {
#if defined(__CUDA_ARCH__)
    atomicOr(p, v);
#else
    *p |= v;
#endif
}
TB_HD TB_FI void max32(int32_t* p, int32_t v) {
#if defined(__CUDA_ARCH__)
    atomicMax(p, v);
#else
    if (v > *p) *p = v;
#endif
}

TB_HD TB_FI uint32_t hash_slot(unsigned long long k, uint32_t mask) {
    unsigned long long h = k * 0x9E3779B97F4A7C15ull;
    h ^= h >> 29;
    h *= 0xBF58476D1CE4E5B9ull;
    h ^= h >> 32;
    return static_cast<uint32_t>(h) & mask;
}

TB_HD inline void ht_insert(const HashTab& t, unsigned long long key, int32_t item) {
    uint32_t s = hash_slot(key, t.mask);
    for (uint32_t probe = 0; probe <= t.mask; ++probe) {
        const unsigned long long prev = cas64(&t.keys[s], kEmpty, key);
        if (prev == kEmpty || prev == key) {
            min32(&t.owner[s], item);
            return;
        }
        s = (s + 1) & t.mask;
    }
    or32(t.err, kErrTableFull);
}

// The slot holding key (inserted), or the table size when absent.
TB_HD inline uint32_t ht_slot(const HashTab& t, unsigned long long key) {
    uint32_t s = hash_slot(key, t.mask);
    for (uint32_t probe = 0; probe <= t.mask; ++probe) {
        const unsigned long long k = t.keys[s];
        if (k == key) return s;
        if (k == kEmpty) break;
        s = (s + 1) & t.mask;
    }
    return t.mask + 1;
}

// Compaction, one item at a time in item order (the host build): the key's first item
// gives it the next index.
TB_HD inline void ht_number(const HashTab& t, unsigned long long key, int32_t item) {
    const uint32_t s = ht_slot(t, key);
    if (s > t.mask || t.owner[s] != item) return;
    const int32_t idx = add32(t.count, 1);
    t.vals[s] = idx;
    t.uniq[idx] = key;
}

TB_HD inline int32_t ht_find(const HashTab& t, unsigned long long key) {
    uint32_t s = hash_slot(key, t.mask);
    for (uint32_t probe = 0; probe <= t.mask; ++probe) {
        const unsigned long long k = t.keys[s];
        if (k == key) return t.vals[s];
        if (k == kEmpty) return -1;
        s = (s + 1) & t.mask;
    }
    return -1;
}

// ht_find for an inserted key; a missing one sets kErrKeyMissing and gives index 0, so
// that no later access goes out of bounds.
TB_HD TB_FI int32_t ht_resolve(const HashTab& t, unsigned long long key) {
    const int32_t v = ht_find(t, key);
    if (v >= 0) return v;
    or32(t.err, kErrKeyMissing);
    return 0;
}

// Keys: 27-bit offset coordinates (|v| < 2^26), a semantics bit and a 9-bit seed slot.
constexpr int64_t kKeyBias = 1ll << 26;
TB_HD TB_FI unsigned long long pack_key(int32_t slot, int32_t a, int32_t b, int32_t sem) {
    return (static_cast<unsigned long long>(slot) << 55) | (static_cast<unsigned long long>(sem & 1) << 54) |
           (static_cast<unsigned long long>(static_cast<int64_t>(a) + kKeyBias) << 27) | static_cast<unsigned long long>(static_cast<int64_t>(b) + kKeyBias);
}
TB_HD TB_FI void unpack_key(unsigned long long k, int32_t& slot, int32_t& a, int32_t& b, int32_t& sem) {
    slot = static_cast<int32_t>(k >> 55);
    sem = static_cast<int32_t>((k >> 54) & 1);
    a = static_cast<int32_t>(static_cast<int64_t>((k >> 27) & ((1ull << 27) - 1)) - kKeyBias);
    b = static_cast<int32_t>(static_cast<int64_t>(k & ((1ull << 27) - 1)) - kKeyBias);
}

// ---- dedupe stages ----------------------------------------------------------------------------
// Each stage inserts its keys, numbers them (ht_number on the host, k_number on the device),
// then resolves every item to its key's index.
// biome chunks (item = chunk * 9 + neighbour)
TB_HD TB_FI unsigned long long nb_key(const Batch& B, int i) {
    const int c = i / 9, k = i % 9;
    return pack_key(B.cseed[c], B.cx[c] + k % 3 - 1, B.cz[c] + k / 3 - 1, 0);
}
TB_HD inline void body_nb_insert(const Batch& B, int i) { ht_insert(B.hb, nb_key(B, i), i); }
TB_HD inline void body_nb_resolve(const Batch& B, int i) { B.nb9[i] = ht_resolve(B.hb, nb_key(B, i)); }
// corner columns in quart units (item = chunk * 25 + k * 5 + i)
TB_HD TB_FI unsigned long long cc_key(const Batch& B, int it) {
    const int c = it / 25, k = (it % 25) / 5, i = it % 5;
    return pack_key(B.cseed[c], B.cx[c] * 4 + i, B.cz[c] * 4 + k, 0);
}
TB_HD inline void body_cc_insert(const Batch& B, int it) { ht_insert(B.hc, cc_key(B, it), it); }
TB_HD inline void body_cc_resolve(const Batch& B, int it) { B.c25[it] = ht_resolve(B.hc, cc_key(B, it)); }
// surface-level quarts: 27 x 19 per chunk; the 11 x 11 window of the aquifer's
// constructor uses volume semantics (sem 1), the rest the lazy point path (sem 0).
TB_HD TB_FI unsigned long long sg_key(const Batch& B, int c, int g) {
    const int gx = g % kGridX, gz = g / kGridX;
    const int qx = B.cx[c] * 4 - 16 + gx, qz = B.cz[c] * 4 - 8 + gz;
    const bool win = qx >= B.cx[c] * 4 - 4 && qx <= B.cx[c] * 4 + 6 && qz >= B.cz[c] * 4 - 4 && qz <= B.cz[c] * 4 + 6;
    return pack_key(B.cseed[c], qx, qz, win ? 1 : 0);
}
TB_HD TB_FI unsigned long long sg_key_item(const Batch& B, int it) { return sg_key(B, it / kGrid, it % kGrid); }
TB_HD inline void body_sg_insert(const Batch& B, int it) { ht_insert(B.hs, sg_key_item(B, it), it); }
TB_HD inline void body_sg_resolve(const Batch& B, int it) { B.g513[it] = ht_resolve(B.hs, sg_key(B, it / kGrid, it % kGrid)); }

// ---- biomes -------------------------------------------------------------------------------------
// chain position p -> quart (qx, qy, qz): vanilla order sections, x, y, z
TB_HD TB_FI void chain_quart(int p, int& qx, int& qy, int& qz) {
    qz = p & 3;
    const int y = (p >> 2) & 3;
    qx = (p >> 4) & 3;
    qy = (p >> 6) * 4 + y;
}
TB_HD TB_FI int chain_pos(int qx, int qy, int qz) { return (((qy >> 2) * 4 + qx) * 4 + (qy & 3)) * 4 + qz; }

TB_HD inline void body_climate_col(const Batch& B, int it) {
    const int b = it / 16, col = it % 16;
    if (b >= *B.hb.count) return;
    int32_t slot, bx, bz, sem;
    unpack_key(B.hb.uniq[b], slot, bx, bz, sem);
    const DevSeed& S = B.seeds[slot];
    tbgen::gen_climate_col(S.nt, bx * 16 + 4 * (col & 3), bz * 16 + 4 * (col >> 2), B.bcol + static_cast<size_t>(it) * tbm::kClimateCols);
}

TB_HD TB_FI long long param_dist(const RNode& n, const long long* t) {
    long long d = 0;
#pragma unroll
    for (int i = 0; i < 7; ++i) {
        const long long tv = i < 6 ? t[i] : 0;
        const long long above = tv - n.mx[i], below = n.mn[i] - tv;
        const long long p = above > 0 ? above : (below > 0 ? below : 0);
        d += p * p;
    }
    return d;
}

// First minimal leaf in depth-first order: the minimum of (distance, leaf rank) over
// all leaves, pruned with a known leaf as the starting best.
TB_HD inline int tree_first_min(const DevModel& M, const long long* t, int start_leaf, long long& best_d) {
    int best = start_leaf;
    int best_rank = M.leaf_rank[start_leaf];
    best_d = param_dist(M.tree[M.leaf_node[start_leaf]], t);
    int stack_node[kSearchStack], stack_next[kSearchStack];
    int sp = 0;
    stack_node[0] = M.root;
    stack_next[0] = 0;
    sp = 1;
    while (sp > 0) {
        const RNode& nd = M.tree[stack_node[sp - 1]];
        const int k = stack_next[sp - 1];
        if (k >= nd.child_count) {
            --sp;
            continue;
        }
        stack_next[sp - 1] = k + 1;
        const int ci = M.children[nd.first_child + k];
        const RNode& ch = M.tree[ci];
        const long long d = param_dist(ch, t);
        if (d < best_d || (d == best_d && ch.rank < best_rank)) {
            if (ch.leaf >= 0) {
                best = ch.leaf;
                best_rank = ch.rank;
                best_d = d;
            } else if (sp < kSearchStack) {
                stack_node[sp] = ci;
                stack_next[sp] = 0;
                ++sp;
            }
        }
    }
    return best;
}

// 32-bit form of the same search (exact: every bound and target is within +/-2^29, so
// no difference overflows and each squared term fits 60 bits).
TB_HD TB_FI long long box_dist32(const RBox& n, const int32_t* t) {
    long long d = 0;
#pragma unroll
    for (int i = 0; i < 7; ++i) {
        const int32_t tv = i < 6 ? t[i] : 0;
        int32_t p = tv - n.mx[i];
        const int32_t q = n.mn[i] - tv;
        p = p > q ? p : q;
        p = p > 0 ? p : 0;
        d += static_cast<long long>(static_cast<unsigned long long>(static_cast<uint32_t>(p)) * static_cast<uint32_t>(p));
    }
    return d;
}

TB_HD inline int tree_first_min32(const DevModel& M, const int32_t* t, int start_leaf, long long& best_d) {
    int best = start_leaf;
    int best_rank = M.leaf_rank[start_leaf];
    best_d = box_dist32(M.boxes[M.box_leaf[start_leaf]], t);
    int stack_node[kSearchStack], stack_next[kSearchStack];
    int sp = 1;
    stack_node[0] = 0;
    stack_next[0] = 0;
    while (sp > 0) {
        const int info = M.boxes[stack_node[sp - 1]].info;
        const int k = stack_next[sp - 1];
        if (k >= (info & 31)) {
            --sp;
            continue;
        }
        stack_next[sp - 1] = k + 1;
        const int ci = (info >> 5) + k;
        const RBox ch = M.boxes[ci];
        const long long d = box_dist32(ch, t);
        if (d < best_d || (d == best_d && ch.rank < best_rank)) {
            if (ch.info < 0) {
                best = ~ch.info;
                best_rank = ch.rank;
                best_d = d;
            } else if (sp < kSearchStack) {
                stack_node[sp] = ci;
                stack_next[sp] = 0;
                ++sp;
            }
        }
    }
    return best;
}

// The same search with the descent as nested loops over the tree levels (children of a box
// are consecutive boxes), for trees of at most kRecDepth levels: the loop state of every
// level stays in registers instead of a stack in local memory. Same visiting order.
constexpr int kRecDepth = 6;
template <int L>
TB_HD TB_FI void search_level32(const DevModel& M, const int32_t* t, int node, int& best, int& best_rank, long long& best_d) {
    const int info = M.boxes[node].info;
    const int first = info >> 5, cnt = info & 31;
    for (int k = 0; k < cnt; ++k) {
        const RBox ch = M.boxes[first + k];
        const long long d = box_dist32(ch, t);
        if (d < best_d || (d == best_d && ch.rank < best_rank)) {
            if (ch.info < 0) {
                best = ~ch.info;
                best_rank = ch.rank;
                best_d = d;
            } else if constexpr (L > 1) {
                search_level32<L - 1>(M, t, first + k, best, best_rank, best_d);
            }
        }
    }
}
TB_HD inline int tree_first_min32_levels(const DevModel& M, const int32_t* t, int start_leaf, long long& best_d) {
    int best = start_leaf;
    int best_rank = M.leaf_rank[start_leaf];
    best_d = box_dist32(M.boxes[M.box_leaf[start_leaf]], t);
    search_level32<kRecDepth - 1>(M, t, 0, best, best_rank, best_d);
    return best;
}
#ifndef TB_SEARCH_LEVELS
#define TB_SEARCH_LEVELS 1
#endif

#if defined(__CUDA_ARCH__)
// The first minimal leaf for one target t held by every lane, searched by the whole warp: lane
// k tests child k of a node (a node has at most 31 children), the warp takes the least
// (distance, rank) among the leaf children, then enters the other children in order while
// they can still hold a better leaf. The same result as tree_first_min32; every lane ends
// with it. All 32 lanes must take part (full mask).
#ifndef TB_WARP_START
#define TB_WARP_START 1
#endif
template <int L>
__device__ __forceinline__ void warp_search32(const DevModel& M, const int32_t* t, int node, int lane, long long& best_d, int& best_rank, int& best_leaf) {
    const unsigned full = 0xFFFFFFFFu;
    const int info = M.boxes[node].info;
    const int first = info >> 5, cnt = info & 31;
    long long d = LLONG_MAX;
    int rank = INT_MAX, cinfo = 0;
    if (lane < cnt) {
        const RBox ch = M.boxes[first + lane];
        d = box_dist32(ch, t);
        rank = ch.rank;
        cinfo = ch.info;
    }
    // least (distance, rank, leaf) over the leaf children
    long long ld = (lane < cnt && cinfo < 0) ? d : LLONG_MAX;
    int lr = (lane < cnt && cinfo < 0) ? rank : INT_MAX, ll = (lane < cnt && cinfo < 0) ? ~cinfo : 0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const long long od = __shfl_xor_sync(full, ld, o);
        const int orr = __shfl_xor_sync(full, lr, o), ol = __shfl_xor_sync(full, ll, o);
        if (od < ld || (od == ld && orr < lr)) {
            ld = od;
            lr = orr;
            ll = ol;
        }
    }
    if (ld < best_d || (ld == best_d && lr < best_rank)) {
        best_d = ld;
        best_rank = lr;
        best_leaf = ll;
    }
    if constexpr (L > 1) {
        unsigned todo = __ballot_sync(full, lane < cnt && cinfo >= 0);
        while (todo) {
            const int k = __ffs(static_cast<int>(todo)) - 1;
            todo &= todo - 1u;
            const long long dk = __shfl_sync(full, d, k);
            const int rk = __shfl_sync(full, rank, k);
            if (dk < best_d || (dk == best_d && rk < best_rank)) warp_search32<L - 1>(M, t, first + k, lane, best_d, best_rank, best_leaf);
        }
    }
}
__device__ inline int warp_first_min32(const DevModel& M, const int32_t* t) {
    const int lane = static_cast<int>(threadIdx.x & 31u);
    long long best_d = LLONG_MAX;
    int best_rank = INT_MAX, best_leaf = 0;
    warp_search32<kRecDepth - 1>(M, t, 0, lane, best_d, best_rank, best_leaf);
    return best_leaf;
}
#endif

// The first minimal leaf for G targets that agree in every coordinate but depth (index 4),
// in one descent of the tree: a box's terms of the other coordinates are summed once, each
// target adds its own depth term and keeps its own best (distance, rank, leaf), and a box is
// entered when any target could find a better leaf in it. Each result is the one
// tree_first_min32 gives for that target alone: both are the least (distance, rank) over
// all leaves, and a box is skipped only when it cannot hold a better pair for any target.
template <int G>
struct MultiBest {
    long long d[G];
    int rank[G], leaf[G];
};
TB_HD TB_FI long long box_dist32_no_depth(const RBox& n, const int32_t* t) {
    long long d = 0;
#pragma unroll
    for (int i = 0; i < 7; ++i) {
        if (i == 4) continue;
        const int32_t tv = i < 6 ? t[i] : 0;
        int32_t p = tv - n.mx[i];
        const int32_t q = n.mn[i] - tv;
        p = p > q ? p : q;
        p = p > 0 ? p : 0;
        d += static_cast<long long>(static_cast<unsigned long long>(static_cast<uint32_t>(p)) * static_cast<uint32_t>(p));
    }
    return d;
}
TB_HD TB_FI long long depth_term32(const RBox& n, int32_t depth) {
    int32_t p = depth - n.mx[4];
    const int32_t q = n.mn[4] - depth;
    p = p > q ? p : q;
    p = p > 0 ? p : 0;
    return static_cast<long long>(static_cast<unsigned long long>(static_cast<uint32_t>(p)) * static_cast<uint32_t>(p));
}
template <int L, int G>
TB_HD TB_FI void search_multi32(const DevModel& M, const int32_t* t, const int32_t* depth, int node, MultiBest<G>& b) {
    const int info = M.boxes[node].info;
    const int first = info >> 5, cnt = info & 31;
    for (int k = 0; k < cnt; ++k) {
        const RBox ch = M.boxes[first + k];
        const long long a = box_dist32_no_depth(ch, t);
        bool enter = false;
#pragma unroll
        for (int g = 0; g < G; ++g) {
            const long long d = a + depth_term32(ch, depth[g]);
            const bool better = d < b.d[g] || (d == b.d[g] && ch.rank < b.rank[g]);
            if (ch.info < 0) {
                if (better) {
                    b.d[g] = d;
                    b.rank[g] = ch.rank;
                    b.leaf[g] = ~ch.info;
                }
            } else {
                enter = enter || better;
            }
        }
        if constexpr (L > 1) {
            if (ch.info >= 0 && enter) search_multi32<L - 1, G>(M, t, depth, first + k, b);
        }
    }
}
// Starts every target from start_leaf (the previous result), as tree_first_min32 does.
template <int G>
TB_HD inline void tree_first_min32_multi(const DevModel& M, const int32_t* t, const int32_t* depth, int start_leaf, MultiBest<G>& b) {
    const RBox& s0 = M.boxes[M.box_leaf[start_leaf]];
    const long long a = box_dist32_no_depth(s0, t);
    const int r0 = M.leaf_rank[start_leaf];
#pragma unroll
    for (int g = 0; g < G; ++g) {
        b.d[g] = a + depth_term32(s0, depth[g]);
        b.rank[g] = r0;
        b.leaf[g] = start_leaf;
    }
    search_multi32<kRecDepth - 1, G>(M, t, depth, 0, b);
}

// Whether a leaf other than `leaf` reaches distance m (the minimum) from target t: then the
// chain's previous result may be kept over the first minimal leaf. Boxes farther than m
// are pruned.
template <int L>
TB_HD TB_FI bool other_min_level32(const DevModel& M, const int32_t* t, int node, int leaf, long long m) {
    const int info = M.boxes[node].info;
    const int first = info >> 5, cnt = info & 31;
    for (int k = 0; k < cnt; ++k) {
        const RBox ch = M.boxes[first + k];
        const long long d = box_dist32(ch, t);
        if (d > m) continue;
        if (ch.info < 0) {
            if (~ch.info != leaf) return true;
        } else if constexpr (L > 1) {
            if (other_min_level32<L - 1>(M, t, first + k, leaf, m)) return true;
        }
    }
    return false;
}
TB_HD inline bool tree_other_min(const DevModel& M, const long long* t, int leaf, long long m) {
    int stack_node[kSearchStack], stack_next[kSearchStack];
    int sp = 1;
    stack_node[0] = M.root;
    stack_next[0] = 0;
    while (sp > 0) {
        const RNode& nd = M.tree[stack_node[sp - 1]];
        const int k = stack_next[sp - 1];
        if (k >= nd.child_count) {
            --sp;
            continue;
        }
        stack_next[sp - 1] = k + 1;
        const int ci = M.children[nd.first_child + k];
        const RNode& ch = M.tree[ci];
        if (param_dist(ch, t) > m) continue;
        if (ch.leaf >= 0) {
            if (ch.leaf != leaf) return true;
        } else if (sp < kSearchStack) {
            stack_node[sp] = ci;
            stack_next[sp] = 0;
            ++sp;
        }
    }
    return false;
}

// One quart on its own (biome lookups): climate, quantized target, the first minimal leaf,
// the minimum distance, and whether another leaf reaches it. (X, Z) are absolute quart
// coordinates, qy the quart row 0..height/4-1.
struct QuartLeaf {
    int leaf;
    bool tie;
    long long m;
    long long t[6];
};
// Quantized climate target of quart (X, qy, Z) from its column's climate terms col.
TB_HD TB_FI void quart_target(const DevSeed& S, const float* col, int X, int qy, int Z, long long* t) {
    float cl[6];
    tbgen::gen_climate(S.nt, 4 * X, tbm::kMinY + 4 * qy, 4 * Z, col, cl);
    for (int k = 0; k < 6; ++k) t[k] = f2l(cl[k] * 10000.0f);
}

// First minimal leaf of quart (X, qy, Z) and whether another leaf ties it, from the quart
// column's climate terms col (gen_climate_col at x = 4 X, z = 4 Z). The search starts from
// leaf start (any leaf: it only bounds the search, the result is the same).
TB_HD TB_NOINLINE inline QuartLeaf quart_leaf_col(const DevModel& M, const DevSeed& S, const float* col, int X, int qy, int Z, int start = 0) {
    QuartLeaf q;
    quart_target(S, col, X, qy, Z, q.t);
    bool small = M.boxes != nullptr && M.depth <= kRecDepth;
    int32_t t32[6];
    for (int k = 0; k < 6; ++k) {
        small = small && q.t[k] >= -kBox32Limit && q.t[k] <= kBox32Limit;
        t32[k] = static_cast<int32_t>(q.t[k]);
    }
    if (small) {
        q.leaf = tree_first_min32_levels(M, t32, start, q.m);
        q.tie = other_min_level32<kRecDepth - 1>(M, t32, 0, q.leaf, q.m);
    } else {
        q.leaf = tree_first_min(M, q.t, start, q.m);
        q.tie = tree_other_min(M, q.t, q.leaf, q.m);
    }
    return q;
}
TB_HD TB_NOINLINE inline QuartLeaf quart_leaf(const DevModel& M, const DevSeed& S, int X, int qy, int Z) {
    float col[tbm::kClimateCols];
    tbgen::gen_climate_col(S.nt, 4 * X, 4 * Z, col);
    return quart_leaf_col(M, S, col, X, qy, Z);
}

// One quart column run: climate per quart, quantized targets, first minimal leaf.
// item = run * (biome chunks * 16) + biome chunk * 16 + column; a run is kRun
// consecutive quarts in y. A warp holds 32 neighbouring columns at the same heights,
// whose targets (and so tree paths) are alike.
#ifndef TB_QUART_RUN
#define TB_QUART_RUN 16
#endif
constexpr int kRun = TB_QUART_RUN;
// quarts of a run searched together (one descent of the tree for the group)
#ifndef TB_QUART_GROUP
#define TB_QUART_GROUP 4
#endif
constexpr int kQuartGroup = TB_QUART_GROUP;
static_assert(kRun % kQuartGroup == 0, "quart group must divide the run");
constexpr int kRuns = (tbm::kHeight / 4) / kRun;
static_assert((tbm::kHeight / 4) % kRun == 0, "quart run must divide the quart height");
TB_HD inline void body_climate_quart(const Batch& B, int it) {
    const int ncol = *B.hb.count * 16;
    const int run = it / ncol, cidx = it % ncol, b = cidx / 16, col = cidx % 16;
    if (run >= kRuns) return;
    int32_t slot, bx, bz, sem;
    unpack_key(B.hb.uniq[b], slot, bx, bz, sem);
    const DevSeed& S = B.seeds[slot];
    const int qx = col & 3, qz = col >> 2;
    const int x = bx * 16 + 4 * qx, z = bz * 16 + 4 * qz;
    const float* colv = B.bcol + static_cast<size_t>(cidx) * tbm::kClimateCols;
    int prev = 0;
    for (int r0 = 0; r0 < kRun; r0 += kQuartGroup) {
        // The group's targets go out as they are computed; the shared search needs 32-bit
        // targets that agree outside depth.
        bool shared = B.M.boxes != nullptr && TB_SEARCH_LEVELS && B.M.depth <= kRecDepth;
        int32_t t32[6], depth[kQuartGroup];
        for (int g = 0; g < kQuartGroup; ++g) {
            float cl[6];
            tbgen::gen_climate(S.nt, x, tbm::kMinY + 4 * (run * kRun + r0 + g), z, colv, cl);
            long long* tg = B.tgt + (static_cast<size_t>(b) * kQuartsPerChunk + chain_pos(qx, run * kRun + r0 + g, qz)) * 6;
            for (int k = 0; k < 6; ++k) {
                const long long v = f2l(cl[k] * 10000.0f);
                tg[k] = v;
                shared = shared && v >= -kBox32Limit && v <= kBox32Limit;
                if (g == 0) t32[k] = static_cast<int32_t>(v);
                else if (k != 4) shared = shared && static_cast<int32_t>(v) == t32[k];
                if (k == 4) depth[g] = static_cast<int32_t>(v);
            }
        }
#if defined(__CUDA_ARCH__)
        // A run's first group has no previous result; neighbouring columns (the warp's lanes)
        // have close climates, so the warp searches lane 0's first target once and every
        // lane starts from that leaf (the results do not depend on the starting leaf).
        if (TB_WARP_START && r0 == 0 && B.M.boxes != nullptr && B.M.depth <= kRecDepth) {
            const unsigned m = __activemask();
            if (m == 0xFFFFFFFFu) {
                int32_t tr[6];
#pragma unroll
                for (int k = 0; k < 6; ++k) tr[k] = __shfl_sync(m, k == 4 ? depth[0] : t32[k], 0);
                prev = warp_first_min32(B.M, tr);
            }
        }
#endif
        if (shared) {
            MultiBest<kQuartGroup> mb;
            tree_first_min32_multi<kQuartGroup>(B.M, t32, depth, prev, mb);
            // each quart's least (distance, rank) is the same whichever leaf its search starts from
            for (int g = 0; g < kQuartGroup; ++g) {
                const size_t p = static_cast<size_t>(b) * kQuartsPerChunk + chain_pos(qx, run * kRun + r0 + g, qz);
                B.lstar[p] = mb.leaf[g];
                B.mdist[p] = mb.d[g];
            }
            prev = mb.leaf[kQuartGroup - 1];
        } else {
            for (int g = 0; g < kQuartGroup; ++g) {
                const size_t p = static_cast<size_t>(b) * kQuartsPerChunk + chain_pos(qx, run * kRun + r0 + g, qz);
                const long long* t = B.tgt + p * 6;
                bool small = B.M.boxes != nullptr;
                int32_t u32[6];
                for (int k = 0; k < 6; ++k) {
                    small = small && t[k] >= -kBox32Limit && t[k] <= kBox32Limit;
                    u32[k] = static_cast<int32_t>(t[k]);
                }
                long long md;
                const int leaf = !small                                     ? tree_first_min(B.M, t, prev, md)
                                 : (TB_SEARCH_LEVELS && B.M.depth <= kRecDepth) ? tree_first_min32_levels(B.M, u32, prev, md)
                                                                                : tree_first_min32(B.M, u32, prev, md);
                B.lstar[p] = leaf;
                B.mdist[p] = md;
                prev = leaf;
            }
        }
    }
}

// The last-result rule: the previous result is kept while it reaches the minimum.
TB_HD inline void body_chain(const Batch& B, int b) {
    if (b >= *B.hb.count) return;
    const size_t base = static_cast<size_t>(b) * kQuartsPerChunk;
    int last = -1;
    for (int p = 0; p < kQuartsPerChunk; ++p) {
        int r = B.lstar[base + p];
        if (last >= 0 && last != r) {
            if (param_dist(B.M.tree[B.M.leaf_node[last]], B.tgt + (base + p) * 6) == B.mdist[base + p]) r = last;
        }
        last = r;
        int qx, qy, qz;
        chain_quart(p, qx, qy, qz);
        B.qbiome[base + (qy * 4 + qz) * 4 + qx] = static_cast<uint8_t>(B.M.leaf_biome[r]);
    }
}

// ---- corner channels ----------------------------------------------------------------------------
// ---- axis tables of the corner kernel ------------------------------------------------------------
// item = corner column * 2 + (0: its x, 1: its z)
TB_HD TB_FI unsigned long long axis_key(const Batch& B, int it) {
    int32_t slot, qx, qz, sem;
    unpack_key(B.hc.uniq[it >> 1], slot, qx, qz, sem);
    return (it & 1) ? pack_key(slot, 0, qz, 1) : pack_key(slot, qx, 0, 0);
}
TB_HD inline void body_axis_insert(const Batch& B, int it) { ht_insert(B.ha, axis_key(B, it), it); }
// numbering in arrival order: the table rows are found by lookup, so their order is free
TB_HD inline void body_axis_number(const Batch& B, int it) {
    const unsigned long long key = axis_key(B, it);
    const uint32_t s = ht_slot(B.ha, key);
    if (s > B.ha.mask || B.ha.owner[s] != it) return;
    const int32_t idx = add32(B.ha.count, 1);
    B.ha.vals[s] = idx;
    B.ha.uniq[idx] = key;
}
// item = row * kAxisLayers + entry: the x (or z) record of one axis-table layer at one
// coordinate, the arithmetic of axis_setup in the octave it replaces
TB_HD inline void body_axis_fill(const Batch& B, int it) {
    if (tbm::kAxisLayers == 0) return;
    const int row = it / tbm::kAxisLayers, e = it % tbm::kAxisLayers;
    int32_t slot, qx, qz, sem;
    unpack_key(B.ha.uniq[row], slot, qx, qz, sem);
    const NoiseTables& T = B.seeds[slot].nt;
#if defined(__CUDA_ARCH__)
    const Layer L = T.layer[tbm::kAxisLayerDev[e]];
    const double scale = tbm::kAxisScaleDev[e] * L.freq;
#else
    const Layer L = T.layer[tbm::kAxisLayer[e]];
    const double scale = tbm::kAxisScale[e] * L.freq;
#endif
    const OctaveOff o = T.off[L.oct];
    const AxisSetup a = axis_setup((sem ? qz : qx) * 4, scale, sem ? o.oz : o.ox);
    // an x record also holds the octave's first hash lookup, which depends on x alone
    const int32_t hx = sem ? 0 : static_cast<int32_t>(T.perm2[256 * L.oct + (static_cast<uint32_t>(a.f) & 255u)]);
    B.axtab[static_cast<size_t>(row) * tbm::kAxisLayers + e] = AxisRec{a.f, a.r, a.a, hx};
}

TB_HD inline void body_corner_col(const Batch& B, int u) {
    if (u >= *B.hc.count) return;
    int32_t slot, qx, qz, sem;
    unpack_key(B.hc.uniq[u], slot, qx, qz, sem);
    tbgen::gen_corner_col(B.seeds[slot].nt, qx * 4, qz * 4, B.ccol + static_cast<size_t>(u) * tbm::kCornerCols);
#if TB_AXIS_TABLE
    B.colax[2 * u] = ht_resolve(B.ha, pack_key(slot, qx, 0, 0));
    B.colax[2 * u + 1] = ht_resolve(B.ha, pack_key(slot, 0, qz, 1));
#endif
}
// item = row * count + column: a warp evaluates one corner row over neighbouring
// columns, where the lazy branches (surface, caves, blended-noise limits) agree most.
TB_HD inline void body_corner(const Batch& B, int it) {
    const int cnt = *B.hc.count;
    const int u = it % cnt, row = it / cnt;
    if (row >= kRows) return;
    int32_t slot, qx, qz, sem;
    unpack_key(B.hc.uniq[u], slot, qx, qz, sem);
#if TB_AXIS_TABLE
    const AxisRec* ax = B.axtab + static_cast<size_t>(B.colax[2 * u]) * tbm::kAxisLayers;
    const AxisRec* az = B.axtab + static_cast<size_t>(B.colax[2 * u + 1]) * tbm::kAxisLayers;
#else
    const AxisRec* ax = nullptr;
    const AxisRec* az = nullptr;
#endif
    const AxisRec* ay = B.seeds[slot].ytab + static_cast<size_t>(row) * tbm::kYLayers;
    tbgen::gen_corner(B.seeds[slot].nt, qx * 4, tbm::kMinY + 8 * row, qz * 4, B.ccol + static_cast<size_t>(u) * tbm::kCornerCols, ax, az, ay,
                      B.corners + (static_cast<size_t>(u) * kRows + row) * tbm::kNumChannels);
}

// ---- surface levels and aquifer cells ---------------------------------------------------------------
TB_HD inline void body_surface_level(const Batch& B, int u) {
    if (u >= *B.hs.count) return;
    int32_t slot, qx, qz, sem;
    unpack_key(B.hs.uniq[u], slot, qx, qz, sem);
    const NoiseTables& T = B.seeds[slot].nt;
    B.sfts[u] = sem ? tbgen::gen_fts_vol(T, qx * 4, qz * 4) : tbgen::gen_fts_pt(T, qx * 4, qz * 4);
}

struct Fluid {
    int32_t level, type;
    TB_HD TB_FI int at(int y) const { return y < level ? type : tbm::kAir; }
};
// Aquifer status packing: the fluid block is water or lava (below 4), the level at least
// kWayBelowMinY, so level * 4 + type fits and the arithmetic shift gives the level back.
static_assert(tbm::kWater >= 0 && tbm::kWater < 4 && tbm::kLava >= 0 && tbm::kLava < 4 && tbm::kDefaultFluid < 4, "fluid packing");
TB_HD TB_FI int32_t fluid_pack(Fluid f) { return f.level * 4 + f.type; }
TB_HD TB_FI Fluid fluid_unpack(int32_t st) { return Fluid{st >> 2, st & 3}; }
TB_HD TB_FI Fluid global_fluid(int y) {
    constexpr int lava_level = tbm::kTmSeaLevel < -54 ? tbm::kTmSeaLevel : -54;
    return y < lava_level ? Fluid{-54, tbm::kLava} : Fluid{tbm::kTmSeaLevel, tbm::kDefaultFluid};
}

// BlockPos packing: 26 bits x, 12 bits y, 26 bits z (two's complement fields)
TB_HD TB_FI void blockpos_wrap(int32_t& x, int32_t& y, int32_t& z) {
    const uint64_t v = ((static_cast<uint64_t>(static_cast<int64_t>(x)) & 0x3FFFFFFull) << 38) |
                       ((static_cast<uint64_t>(static_cast<int64_t>(z)) & 0x3FFFFFFull) << 12) | (static_cast<uint64_t>(static_cast<int64_t>(y)) & 0xFFFull);
    const int64_t s = static_cast<int64_t>(v);
    x = static_cast<int32_t>(s >> 38);
    y = static_cast<int32_t>(static_cast<int64_t>(v << 52) >> 52);
    z = static_cast<int32_t>(static_cast<int64_t>(v << 26) >> 38);
}

// Surface level at block (sx, sz) as seen by chunk c (NoiseBasedAquifer's surface-level
// cache, cpu/src/terrain.cpp:324-331): the chunk's grid of surface quarts, which holds every
// unwrapped position the aquifer cells ask for. Cell locations that the BlockPos packing
// wrapped (chunks from |c| = 2^21 - 1 on) lie 2^26 blocks away, outside the cached window,
// so the point path evaluates them.
TB_HD TB_FI int surface_at(const Batch& B, const NoiseTables& T, int c, int sx, int sz) {
    const int gx = (sx >> 2) - (B.cx[c] * 4 - 16), gz = (sz >> 2) - (B.cz[c] * 4 - 8);
    if (gx >= 0 && gx < kGridX && gz >= 0 && gz < kGridZ)
        return jfloor(static_cast<double>(B.sfts[B.g513[static_cast<size_t>(c) * kGrid + gz * kGridX + gx]]));
    return jfloor(static_cast<double>(tbgen::gen_fts_pt(T, (sx >> 2) * 4, (sz >> 2) * 4)));
}

TB_HD inline void body_aquifer_cell(const Batch& B, int it) {
    const int c = it / kAqCells, cell = it % kAqCells;
    const int ix = cell % kAqX, iz = (cell / kAqX) % kAqZ, iy = cell / (kAqX * kAqZ);
    const int gx = B.cx[c] - 1 + ix, gy = kAqMinGridY + iy, gz = B.cz[c] - 1 + iz;
    const DevSeed& S = B.seeds[B.cseed[c]];
    Xoro r = S.aquifer.at(gx, gy, gz);
    int32_t x = gx * 16 + r.next_int(10);
    int32_t y = gy * 12 + r.next_int(9);
    int32_t z = gz * 16 + r.next_int(10);
    blockpos_wrap(x, y, z);
    // NoiseBasedAquifer.computeFluid
    const Fluid glob = global_fluid(y);
    Fluid res{0, 0};
    bool done = false;
    int lowest = INT_MAX;
    const int top = y + 12, bottom = y - 12;
    bool center_under = false;
    const signed char off[13][2] = {{0, 0}, {-2, -1}, {-1, -1}, {0, -1}, {1, -1}, {-3, 0}, {-2, 0}, {-1, 0}, {1, 0}, {-2, 1}, {-1, 1}, {0, 1}, {1, 1}};
    for (int k = 0; k < 13 && !done; ++k) {
        const int sx = x + (off[k][0] << 4), sz = z + (off[k][1] << 4);
        const int level = surface_at(B, S.nt, c, sx, sz);
        const int adjusted = level + 8;
        const bool start = k == 0;
        if (start && bottom > adjusted) {
            res = glob;
            done = true;
            break;
        }
        const bool pokes = top > adjusted;
        if (pokes || start) {
            const Fluid at_s = global_fluid(adjusted);
            if (at_s.at(adjusted) != tbm::kAir) {
                if (start) center_under = true;
                if (pokes) {
                    res = at_s;
                    done = true;
                    break;
                }
            }
        }
        lowest = lowest < level ? lowest : level;
    }
    if (!done) {
        const NoiseTables& T = S.nt;
        double partially, fully;
        if (tbgen::gen_aq_exclusion(T, x, y, z) > 0.0f) {
            partially = -1.0;
            fully = -1.0;
        } else {
            const int below = lowest + 8 - y;
            double factor = 0.0;
            if (center_under) {
                const double f = (static_cast<double>(below) - 0.0) / (64.0 - 0.0);
                factor = f < 0.0 ? 1.0 : (f > 1.0 ? 0.0 : 1.0 + f * (0.0 - 1.0));
            }
            const double noise = jclampd(static_cast<double>(tbgen::gen_aq_fluid_level_floodedness(T, x, y, z)), -1.0, 1.0);
            const double fully_t = -0.3 + ((factor - 1.0) / (0.0 - 1.0)) * (0.8 - -0.3);
            const double partial_t = -0.8 + ((factor - 1.0) / (0.0 - 1.0)) * (0.4 - -0.8);
            partially = noise - partial_t;
            fully = noise - fully_t;
        }
        int level;
        if (fully > 0.0) {
            level = glob.level;
        } else if (partially > 0.0) {
            const int scx = fdiv(x, 16), scy = fdiv(y, 40), scz = fdiv(z, 16);
            const int middle = scy * 40 + 20;
            const double spread = static_cast<double>(tbgen::gen_aq_fluid_level_spread(T, scx, scy, scz) * 10.0f);
            const int q = jfloor(spread / 3.0) * 3;
            level = lowest < middle + q ? lowest : middle + q;
        } else {
            level = kWayBelowMinY;
        }
        int type = glob.type;
        if (level <= -10 && level != kWayBelowMinY && glob.type != tbm::kLava) {
            const double lv = static_cast<double>(tbgen::gen_aq_lava(T, fdiv(x, 64), fdiv(y, 40), fdiv(z, 64)));
            if (dabs(lv) > 0.3) type = tbm::kLava;
        }
        res = Fluid{level, type};
    }
    B.aq_cell[it] = AqCell{x, y, z, fluid_pack(res)};
}

// The 12 cells of one query: x columns xa..xa+1 (outer), layers (middle), z columns (inner).
TB_HD TB_FI int aq_query_cell(int base, int j) {
    const int ox = j >= 6 ? 1 : 0, r = j - 6 * ox;
    return base + ((r >> 1) * kAqZ + (r & 1)) * kAqX + ox;
}

// Shortcuts of NoiseBasedAquifer.computeSubstance (cpu/src/terrain.cpp:215-275) that hold for
// every block of a query, whatever its distances to the cells:
//  - all 12 statuses equal: each pressure is 0 (equal levels), so no barrier test can make
//    the block solid and the result is that status's fluid at y;
//  - y >= every level + 5: for any two cells, above = y + 0.5 - average exceeds diff / 2 + 5,
//    so the gradient is at most -5.5 / 2.5 < -2, the barrier noise is not sampled, every
//    pressure is negative and no test makes the block solid; the nearest cell's fluid at y
//    is air.
TB_HD inline void body_aquifer_query(const Batch& B, int it) {
    const int c = it / kAqQueries, q = it % kAqQueries;
    const int layer = q >> 2, zc = (q >> 1) & 1, xc = q & 1;
    const AqCell* cell = B.aq_cell + static_cast<size_t>(c) * kAqCells;
    const int base = (layer * kAqZ + zc) * kAqX + xc;
    const int32_t st0 = cell[base].st;
    bool uni = true;
    int top = INT_MIN;
    for (int j = 0; j < 12; ++j) {
        const int32_t st = cell[aq_query_cell(base, j)].st;
        uni = uni && st == st0;
        const int level = fluid_unpack(st).level;
        top = level > top ? level : top;
    }
    B.aq_query[it] = AqQuery{uni ? st0 : kAqMixed, top + 5};
}

// per-chunk skip height from the volume-semantics window maximum
TB_HD inline void body_aquifer_skip(const Batch& B, int c) {
    int mx = INT_MIN;
    for (int gz = 4; gz <= 14; ++gz)
        for (int gx = 12; gx <= 22; ++gx) {
            const int v = jfloor(static_cast<double>(B.sfts[B.g513[static_cast<size_t>(c) * kGrid + gz * kGridX + gx]]));
            mx = v > mx ? v : mx;
        }
    const int adjusted = mx + 8;
    const int skip_grid_y = fdiv(adjusted + 12, 12) + 1;
    B.aq_skip[c] = skip_grid_y * 12 + 11 - 1;
}

// ---- fill: channels, final density, aquifer substance --------------------------------------------
// b - a wraps like the reference's int subtraction (distances of wrapped locations overflow)
TB_HD TB_FI double aq_similarity(int a, int b) { return 1.0 - static_cast<double>(isub(b, a)) / 25.0; }

struct AqBlock {
    const AqCell* cell;
    const AqQuery* query;
    int cx, cz;
    bool keyed;   // aq_keyed(cx, cz)
};
// Chunks this far from the BlockPos wrap have unwrapped cell locations and squared
// distances below 2^13, so distance * 16 + scan position fits an int.
constexpr int kAqKeyedMax = (1 << 21) - 4;
TB_HD TB_FI bool aq_keyed(int cx, int cz) { return cx >= -kAqKeyedMax && cx <= kAqKeyedMax && cz >= -kAqKeyedMax && cz <= kAqKeyedMax; }

TB_HD inline double aq_pressure(const NoiseTables& T, int x, int y, int z, double& barrier, bool& barrier_set, Fluid a, Fluid b) {
    const int t1 = a.at(y), t2 = b.at(y);
    if ((t1 == tbm::kLava && t2 == tbm::kWater) || (t1 == tbm::kWater && t2 == tbm::kLava)) return 2.0;
    const int diff = a.level - b.level < 0 ? b.level - a.level : a.level - b.level;
    if (diff == 0) return 0.0;
    const double average = 0.5 * static_cast<double>(a.level + b.level);
    const double above = static_cast<double>(y) + 0.5 - average;
    const double base = static_cast<double>(diff) / 2.0;
    const double towards = base - dabs(above);
    double gradient;
    if (above > 0.0) {
        const double center = 0.0 + towards;
        gradient = center > 0.0 ? center / 1.5 : center / 2.5;
    } else {
        const double center = 3.0 + towards;
        gradient = center > 0.0 ? center / 3.0 : center / 10.0;
    }
    double noise;
    if (!(gradient < -2.0) && !(gradient > 2.0)) {
        if (!barrier_set) {
            barrier = static_cast<double>(tbgen::gen_aq_barrier(T, x, y, z));
            barrier_set = true;
        }
        noise = barrier;
    } else {
        noise = 0.0;
    }
    return 2.0 * (noise + gradient);
}

// NoiseBasedAquifer.computeSubstance; -1 = keep the default block.
TB_HD inline int aq_substance(const NoiseTables& T, const AqBlock& A, int skip, int x, int y, int z, double density) {
    if (density > 0.0) return -1;
    const Fluid glob = global_fluid(y);
    if (y > skip) return glob.at(y);
    if (glob.at(y) == tbm::kLava) return tbm::kLava;
    const int xa = (x - 5) >> 4, ya = fdiv(y + 1, 12), za = (z - 5) >> 4;
    const int layer = ya - 1 - kAqMinGridY, zc = za - (A.cz - 1), xc = xa - (A.cx - 1);
    const AqQuery Q = A.query[(layer * 2 + zc) * 2 + xc];
    if (Q.uni != kAqMixed) return fluid_unpack(Q.uni).at(y);
    if (y >= Q.air_from) return tbm::kAir;
    // the three nearest of the 12 candidate cells, later ones first on equal distance
    int d1 = INT_MAX, d2 = INT_MAX, d3 = INT_MAX, i1 = 0, i2 = 0, i3 = 0;
    const int base = (layer * kAqZ + zc) * kAqX + xc;
    if (A.keyed) {
        // Each candidate as one key, distance * 16 + (15 - scan position): ascending keys are
        // ascending distances with later cells first, so the insertion chain's order is the
        // order of the three smallest keys, kept by a min/max network.
        int k1 = INT_MAX, k2 = INT_MAX, k3 = INT_MAX;
        int j = 15;
        for (int ox = 0; ox <= 1; ++ox)
            for (int oy = 0; oy <= 2; ++oy)
                for (int oz = 0; oz <= 1; ++oz, --j) {
                    const AqCell l = A.cell[base + (oy * kAqZ + oz) * kAqX + ox];
                    const int dx = l.x - x, dy = l.y - y, dz = l.z - z;
                    const int key = (dx * dx + dy * dy + dz * dz) * 16 + j;
                    k3 = imin(k3, imax(k2, key));
                    k2 = imin(k2, imax(k1, key));
                    k1 = imin(k1, key);
                }
        auto cell_of = [&](int k) { return aq_query_cell(base, 15 - (k & 15)); };
        d1 = k1 >> 4; d2 = k2 >> 4; d3 = k3 >> 4;
        i1 = cell_of(k1); i2 = cell_of(k2); i3 = cell_of(k3);
    } else {
        for (int ox = 0; ox <= 1; ++ox)
            for (int oy = 0; oy <= 2; ++oy)
                for (int oz = 0; oz <= 1; ++oz) {
                    const int idx = base + (oy * kAqZ + oz) * kAqX + ox;
                    const AqCell l = A.cell[idx];
                    const int dx = l.x - x, dy = l.y - y, dz = l.z - z;
                    const int nd = iadd(iadd(imul(dx, dx), imul(dy, dy)), imul(dz, dz));
                    if (d1 >= nd) {
                        i3 = i2; i2 = i1; i1 = idx;
                        d3 = d2; d2 = d1; d1 = nd;
                    } else if (d2 >= nd) {
                        i3 = i2; i2 = idx;
                        d3 = d2; d2 = nd;
                    } else if (d3 >= nd) {
                        i3 = idx;
                        d3 = nd;
                    }
                }
    }
    const int32_t t1 = A.cell[i1].st;
    const Fluid s1 = fluid_unpack(t1);
    const int fluid = s1.at(y);
    // similarity(a, b) = 1 - (b - a) / 25: the quotient of an integer below 25 by 25 rounds
    // below 1 (and a wrapped negative difference gives a similarity above 1), so the
    // similarity is <= 0 exactly when the wrapped b - a is >= 25
    if (isub(d2, d1) >= 25) return fluid;
    if (fluid == tbm::kWater && global_fluid(y - 1).at(y - 1) == tbm::kLava) return fluid;
    const double sim12 = aq_similarity(d1, d2);
    double barrier = 0.0;
    bool barrier_set = false;
    const Fluid s2 = fluid_unpack(A.cell[i2].st);
    const double b12 = sim12 * aq_pressure(T, x, y, z, barrier, barrier_set, s1, s2);
    if (density + b12 > 0.0) return -1;
    const Fluid s3 = fluid_unpack(A.cell[i3].st);
    if (isub(d3, d1) < 25) {
        const double b13 = sim12 * aq_similarity(d1, d3) * aq_pressure(T, x, y, z, barrier, barrier_set, s1, s3);
        if (density + b13 > 0.0) return -1;
    }
    if (isub(d3, d2) < 25) {
        const double b23 = sim12 * aq_similarity(d2, d3) * aq_pressure(T, x, y, z, barrier, barrier_set, s2, s3);
        if (density + b23 > 0.0) return -1;
    }
    return fluid;
}

// Channel values for the 8 blocks of one column cell: the block-step interpolation
// order of InterpolatedFunction (z, then x, then y in increments).
struct CellInterp {
    float a0[tbm::kNumChannels], step[tbm::kNumChannels];
};
TB_HD inline void cell_interp(const Batch& B, int c, int lx, int lz, int cell_y, CellInterp& out) {
    const int ci = lx >> 2, xi = lx & 3, ck = lz >> 2, zi = lz & 3;
    const int32_t* cc = B.c25 + static_cast<size_t>(c) * 25;
    const size_t u00 = cc[ck * 5 + ci], u10 = cc[ck * 5 + ci + 1], u01 = cc[(ck + 1) * 5 + ci], u11 = cc[(ck + 1) * 5 + ci + 1];
    const int C = tbm::kNumChannels;
    const float* p00 = B.corners + (u00 * kRows + cell_y) * C;
    const float* p10 = B.corners + (u10 * kRows + cell_y) * C;
    const float* p01 = B.corners + (u01 * kRows + cell_y) * C;
    const float* p11 = B.corners + (u11 * kRows + cell_y) * C;
    const float az = static_cast<float>(zi) * 0.25f, ax = static_cast<float>(xi) * 0.25f;
    // the two rows of the four corner columns (2 x C channels each), as 16-byte loads on the
    // device where a row is a whole number of them (the buffer is cudaMalloc-aligned)
    float r00[2 * C], r10[2 * C], r01[2 * C], r11[2 * C];
#if defined(__CUDA_ARCH__)
    if (C % 4 == 0) {
        auto put = [](float* r, const float4 v) {
            r[0] = v.x;
            r[1] = v.y;
            r[2] = v.z;
            r[3] = v.w;
        };
#pragma unroll
        for (int k = 0; k < 2 * C; k += 4) {
            put(r00 + k, __ldg(reinterpret_cast<const float4*>(p00 + k)));
            put(r10 + k, __ldg(reinterpret_cast<const float4*>(p10 + k)));
            put(r01 + k, __ldg(reinterpret_cast<const float4*>(p01 + k)));
            put(r11 + k, __ldg(reinterpret_cast<const float4*>(p11 + k)));
        }
    } else
#endif
    {
        for (int k = 0; k < 2 * C; ++k) {
            r00[k] = p00[k];
            r10[k] = p10[k];
            r01[k] = p01[k];
            r11[k] = p11[k];
        }
    }
    for (int k = 0; k < C; ++k) {
        const float v000 = r00[k], v100 = r10[k], v001 = r01[k], v101 = r11[k];
        const float v010 = r00[C + k], v110 = r10[C + k], v011 = r01[C + k], v111 = r11[C + k];
        const float v00 = lerpf(az, v000, v001), v01 = lerpf(az, v010, v011);
        const float v10 = lerpf(az, v100, v101), v11 = lerpf(az, v110, v111);
        const float a0 = lerpf(ax, v00, v10), a1 = lerpf(ax, v01, v11);
        out.step[k] = (a1 - a0) * 0.125f;
        out.a0[k] = a0 + out.step[k] * 0.0f;
    }
}

// Column lz * 16 + lx of item `it` when each warp's 32 items cover a tile of TW columns in x by
// 32 / TW in z (TW 16: two rows of 16, the plain order).
template <int TW>
TB_HD TB_FI int tile_column(int it) {
    static_assert(TW == 4 || TW == 8 || TW == 16, "tile width");
    constexpr int th = 32 / TW, across = 16 / TW;
    const int w = (it >> 5) & 7, l = it & 31;
    return (th * (w / across) + l / TW) * 16 + TW * (w % across) + l % TW;
}
// the fill's warps hold 4 x 8 column tiles: their cell columns read fewer distinct corner
// columns than a 16 x 2 strip (fill 6.43 -> 6.29 ms per 12,288-chunk step)
#ifndef TB_FILL_TILE
#define TB_FILL_TILE 4
#endif

// The 8 blocks of one cell column. ORES: evaluate the ore veins of ore_live (else their bits
// are 0, and the channels only they read are neither interpolated nor stepped).
template <bool ORES>
TB_HD TB_FI void fill_cell(const Batch& B, int c, int col, int cell_y, uint32_t ore_live) {
    const int lx = col & 15, lz = col >> 4;
    const int bx = B.cx[c] * 16 + lx, bz = B.cz[c] * 16 + lz;
    const DevSeed& S = B.seeds[B.cseed[c]];
    CellInterp ci;
    cell_interp(B, c, lx, lz, cell_y, ci);
    float ch[tbm::kNumChannels];
    for (int k = 0; k < tbm::kNumChannels; ++k) ch[k] = ci.a0[k];
    const AqBlock A{B.aq_cell + static_cast<size_t>(c) * kAqCells, B.aq_query + static_cast<size_t>(c) * kAqQueries, B.cx[c], B.cz[c],
                    aq_keyed(B.cx[c], B.cz[c])};
    const int skip = B.aq_skip[c];
    uint16_t* out = B.blocks + static_cast<size_t>(c) * kBlocksPerChunk;
    int top = INT_MIN;
    uint32_t air = 0, fluid = 0, ore_lo = 0, ore_hi = 0;
    // the fill's blocks are the default block, air or a fluid: the flags of states 0..3 in
    // one register word instead of a table load per block
    const uint32_t flags4 = static_cast<uint32_t>(B.M.block_flags[0]) | (static_cast<uint32_t>(B.M.block_flags[1]) << 8) |
                            (static_cast<uint32_t>(B.M.block_flags[2]) << 16) | (static_cast<uint32_t>(B.M.block_flags[3]) << 24);
    for (int k = 0; k < 8; ++k) {
        const int y = tbm::kMinY + cell_y * 8 + k;
        const float d = tbgen::gen_final_density(S.nt, bx, y, bz, ch);
        int s = aq_substance(S.nt, A, skip, bx, y, bz, static_cast<double>(d));
        if (s < 0) s = tbm::kDefaultBlock;
        const size_t bi = ((y - tbm::kMinY) * 16 + lz) * 16 + lx;
        out[bi] = static_cast<uint16_t>(s);
        if (B.density) B.density[static_cast<size_t>(c) * kBlocksPerChunk + bi] = d;
        if (ORES) {
            uint32_t om = 0;
            for (int v = 0; v < tbm::kNumOres; ++v)
                if (((ore_live >> v) & 1u) && !(tbgen::gen_ore_density(v, S.nt, bx, y, bz, ch) <= 0.0f)) om |= 1u << v;
            if (k < 4) ore_lo |= om << (8 * k);
            else ore_hi |= om << (8 * (k - 4));
        }
        const uint8_t f = s < 4 ? static_cast<uint8_t>(flags4 >> (8 * s)) : B.M.block_flags[s];
        if (!(f & 1)) top = y;
        air |= static_cast<uint32_t>(f & 1) << k;
        fluid |= static_cast<uint32_t>((f >> 3) & 1) << k;
        for (int q = 0; q < tbm::kNumChannels; ++q) ch[q] += ci.step[q];
    }
    // the cell's 8 heights are byte cell_y & 3 of mask word cell_y >> 2 (little-endian words)
    uint8_t* cm = reinterpret_cast<uint8_t*>(B.colmask + (static_cast<size_t>(c) * 2 * kMaskWords + (cell_y >> 2)) * 256 + col) + (cell_y & 3);
    cm[0] = static_cast<uint8_t>(air);
    cm[static_cast<size_t>(kMaskWords) * 256 * 4] = static_cast<uint8_t>(fluid);
    if (TB_ORE_MASK) {
        // the cell's 8 heights are words 2 cell_y and 2 cell_y + 1 of the column
        uint32_t* ow = reinterpret_cast<uint32_t*>(B.oremask) + (static_cast<size_t>(c) * kColWords + 2 * cell_y) * 256 + col;
        ow[0] = ore_lo;
        ow[256] = ore_hi;
    }
    if (top != INT_MIN) max32(B.h0 + static_cast<size_t>(c) * 256 + lx * 16 + lz, top + 1);
}

// item = (chunk * kCellsY + cell_y) * 256 + tile_column: the 8 blocks of one cell column
TB_HD inline void body_fill(const Batch& B, int it) {
    const int col = tile_column<TB_FILL_TILE>(it), cell_y = (it >> 8) % kCellsY, c = (it >> 8) / kCellsY;
    // the ore veins whose density can be above zero in this cell row, the same for the whole
    // warp (its items share cell_y): rows where none can be skip the ore work
#if defined(__CUDA_ARCH__)
    const uint32_t ore_live = tbm::kOreLiveCellsDev[cell_y];
#else
    const uint32_t ore_live = tbm::kOreLiveCells[cell_y];
#endif
    if (TB_ORE_MASK && ore_live)
        fill_cell<true>(B, c, col, cell_y, ore_live);
    else
        fill_cell<false>(B, c, col, cell_y, 0u);
}

// ---- BiomeManager zoom ---------------------------------------------------------------------
// The three fiddle draws of quart vertex (qx, qy, qz): the LCG chain of
// BiomeManager.getFiddledDistance (cpu/src/biome.cpp:255-268), as floorMod(r >> 24, 1024)
// each, packed in 10-bit fields.
TB_HD TB_FI uint32_t zoom_fiddles(int64_t seed, int qx, int qy, int qz) {
    int64_t r = seed;
    r = zoom_lcg(r, qx);
    r = zoom_lcg(r, qy);
    r = zoom_lcg(r, qz);
    r = zoom_lcg(r, qx);
    r = zoom_lcg(r, qy);
    r = zoom_lcg(r, qz);
    const uint32_t mx = static_cast<uint32_t>(zoom_fiddle_m(r));
    r = zoom_lcg(r, seed);
    const uint32_t my = static_cast<uint32_t>(zoom_fiddle_m(r));
    r = zoom_lcg(r, seed);
    const uint32_t mz = static_cast<uint32_t>(zoom_fiddle_m(r));
    return mx | (my << 10) | (mz << 20);
}

// BiomeManager.getBiome: the quart whose fiddled corner is nearest (first on ties), then
// its stored biome from the chunk's 3x3 neighbourhood (qy clamped to the world).
TB_HD TB_FI int zoom_stored(const Batch& B, int c, int best, int px, int py, int pz) {
    const int qx = (best & 4) == 0 ? px : px + 1;
    const int qy = (best & 2) == 0 ? py : py + 1;
    const int qz = (best & 1) == 0 ? pz : pz + 1;
    const int dcx = (qx >> 2) - B.cx[c], dcz = (qz >> 2) - B.cz[c];
    constexpr int qmin = tbm::kMinY >> 2, qh = tbm::kHeight / 4;
    const int cqy = (qy < qmin ? qmin : (qy > qmin + qh - 1 ? qmin + qh - 1 : qy)) - qmin;
    const int b = B.nb9[static_cast<size_t>(c) * 9 + (dcz + 1) * 3 + dcx + 1];
    return B.qbiome[static_cast<size_t>(b) * kQuartsPerChunk + (cqy * 4 + (qz & 3)) * 4 + (qx & 3)];
}
// The index (x 4 + y 2 + z 1 steps) of the fiddled corner nearest to block (x, y, z).
template <class Fiddles>
TB_HD TB_FI int zoom_best(int x, int y, int z, Fiddles fid) {
    const int ax = x - 2, ay = y - 2, az = z - 2;
    const int px = ax >> 2, py = ay >> 2, pz = az >> 2;
    const double fx = static_cast<double>(ax & 3) / 4.0, fy = static_cast<double>(ay & 3) / 4.0, fz = static_cast<double>(az & 3) / 4.0;
    int best = 0;
    double best_d = 0.0;
    for (int i = 0; i < 8; ++i) {
        const bool xe = (i & 4) == 0, ye = (i & 2) == 0, ze = (i & 1) == 0;
        const uint32_t m = fid(xe ? px : px + 1, ye ? py : py + 1, ze ? pz : pz + 1);
        const double ox = zoom_fiddle(static_cast<int32_t>(m & 1023u));
        const double oy = zoom_fiddle(static_cast<int32_t>((m >> 10) & 1023u));
        const double oz = zoom_fiddle(static_cast<int32_t>(m >> 20));
        const double dx = xe ? fx : fx - 1.0, dy = ye ? fy : fy - 1.0, dz = ze ? fz : fz - 1.0;
        const double sz = (dz + oz) * (dz + oz), sy = (dy + oy) * (dy + oy), sx = (dx + ox) * (dx + ox);
        const double d = sz + sy + sx;
        if (i == 0 || best_d > d) {
            best = i;
            best_d = d;
        }
    }
    return best;
}
template <class Fiddles>
TB_HD TB_FI int zoom_pick(const Batch& B, int c, int x, int y, int z, Fiddles fid) {
    const int best = zoom_best(x, y, z, fid);
    return zoom_stored(B, c, best, (x - 2) >> 2, (y - 2) >> 2, (z - 2) >> 2);
}

// any position (biome lookups): the LCG chains computed in place
TB_HD inline int zoom_biome(const Batch& B, int c, int64_t seed, int x, int y, int z) {
    return zoom_pick(B, c, x, y, z, [&](int qx, int qy, int qz) { return zoom_fiddles(seed, qx, qy, qz); });
}

// blocks of chunk c (and its surface height): the chunk's precomputed vertex table
TB_HD TB_NOINLINE inline int zoom_biome_tab(const Batch& B, int c, int x, int y, int z) {
    const uint32_t* tab = B.zoom_tab + static_cast<size_t>(c) * kZoomVerts;
    const int qx0 = B.cx[c] * 4 - 1, qz0 = B.cz[c] * 4 - 1;
    return zoom_pick(B, c, x, y, z, [&](int qx, int qy, int qz) { return tab[((qy - kZoomQyMin) * 6 + (qz - qz0)) * 6 + (qx - qx0)]; });
}

// BiomeManager.getBiome at one block with the chunk chain's exact result, from the quart
// alone where its minimum is unique (the chain's previous result cannot be kept there) and
// otherwise from the nearest earlier quart of the chunk's chain order whose result is
// fixed (unique minimum, or the chunk's first quart), replaying the chain from it.
// The quart BiomeManager.getBiome reads for block (x, y, z): absolute quart x / z, the quart
// row clamped to the world, and its index in the chunk's chain order.
struct LookupQuart {
    int qx, cqy, qz, p;
};
TB_HD TB_FI LookupQuart lookup_quart(int64_t zoom_seed, int x, int y, int z) {
    const int best = zoom_best(x, y, z, [&](int qx, int qy, int qz) { return zoom_fiddles(zoom_seed, qx, qy, qz); });
    const int px = (x - 2) >> 2, py = (y - 2) >> 2, pz = (z - 2) >> 2;
    LookupQuart L;
    L.qx = (best & 4) == 0 ? px : px + 1;
    const int qy = (best & 2) == 0 ? py : py + 1;
    L.qz = (best & 1) == 0 ? pz : pz + 1;
    constexpr int qmin = tbm::kMinY >> 2, qh = tbm::kHeight / 4;
    L.cqy = (qy < qmin ? qmin : (qy > qmin + qh - 1 ? qmin + qh - 1 : qy)) - qmin;
    L.p = chain_pos(L.qx & 3, L.cqy, L.qz & 3);
    return L;
}
TB_HD inline int biome_point(const DevModel& M, const DevSeed& S, int x, int y, int z) {
    const LookupQuart L = lookup_quart(S.zoom_seed, x, y, z);
    const int X0 = (L.qx >> 2) * 4, Z0 = (L.qz >> 2) * 4;   // the chunk's first quart column
    const int p = L.p;
    QuartLeaf q = quart_leaf(M, S, L.qx, L.cqy, L.qz);
    if (!q.tie || p == 0) return M.leaf_biome[q.leaf];
    int j = p - 1, a, b, c;
    for (;; --j) {
        chain_quart(j, a, b, c);
        q = quart_leaf(M, S, X0 + a, b, Z0 + c);
        if (!q.tie || j == 0) break;
    }
    int r = q.leaf;
    for (int k = j + 1; k <= p; ++k) {
        chain_quart(k, a, b, c);
        const QuartLeaf u = quart_leaf(M, S, X0 + a, b, Z0 + c);
        r = (r != u.leaf && param_dist(M.tree[M.leaf_node[r]], u.t) == u.m) ? r : u.leaf;
    }
    return M.leaf_biome[r];
}

// item = chunk * kZoomVerts + vertex
TB_HD inline void body_zoom_table(const Batch& B, int it) {
    const int c = it / kZoomVerts, v = it % kZoomVerts;
    const int qx = B.cx[c] * 4 - 1 + v % 6, qz = B.cz[c] * 4 - 1 + (v / 6) % 6, qy = kZoomQyMin + v / 36;
    B.zoom_tab[it] = zoom_fiddles(B.seeds[B.cseed[c]].zoom_seed, qx, qy, qz);
}

// Zoomed biomes of the blocks under the surface, for the rule tree. Blocks y = 4 py + 2 ..
// 4 py + 5 share py = (y - 2) >> 2 and so the 8 candidate vertices: their fiddles and the
// x and z distance terms are computed once per group, and each block adds its own y term
// in zoom_pick's order ((z term + y term) + x term), so every value is zoom_pick's.
constexpr int kZoomPyMin = (tbm::kMinY - 2) >> 2;
constexpr int kZoomGroups = ((kMaxY - 2) >> 2) - kZoomPyMin + 1;

// Zoom cells of a chunk: the corner quart (px, py, pz) of the 8 candidates of its blocks,
// px and pz over the 5 values ((cx * 16 - 2) >> 2 .. (cx * 16 + 13) >> 2), py over the groups.
constexpr int kZoomCells = kZoomGroups * 25;
constexpr uint8_t kZoomMixed = 0xFF;
static_assert(tbm::kNumBiomes < kZoomMixed, "biome ids below the mixed marker");

// item = chunk * kZoomCells + (group * 5 + pz - (cz * 4 - 1)) * 5 + px - (cx * 4 - 1). When
// the 8 candidate quarts of a cell store one biome, every block of the cell zooms to it,
// whichever corner is nearest.
TB_HD inline void body_zoom_uniform(const Batch& B, int it) {
    const int c = it / kZoomCells, r = it % kZoomCells;
    const int px = B.cx[c] * 4 - 1 + r % 5, pz = B.cz[c] * 4 - 1 + (r / 5) % 5, py = kZoomPyMin + r / 25;
    const int b0 = zoom_stored(B, c, 0, px, py, pz);
    bool uni = true;
    for (int i = 1; i < 8; ++i) uni = uni && zoom_stored(B, c, i, px, py, pz) == b0;
    B.zoom_uni[it] = uni ? static_cast<uint8_t>(b0) : kZoomMixed;
}

// item = chunk * 256 + z * 16 + x: the zoomed biome of every block of the column up to its
// height, written 4 heights to a word (column order). Blocks of a uniform zoom cell take its
// biome; the others pick the nearest fiddled corner in FP64, the 8 candidates' x and z terms
// once per group of 4 heights.
// block_biome's warps hold 4 x 8 column tiles (fewer distinct zoom cells per warp, and more
// lanes in the same uniform or mixed cell: 1.62 -> 1.52 ms per 12,288-chunk step)
#ifndef TB_BB_TILE
#define TB_BB_TILE 4
#endif
TB_HD inline void body_block_biome(const Batch& B, int it) {
    const int c = it >> 8, col = tile_column<TB_BB_TILE>(it), lx = col & 15, lz = col >> 4;
    const int h = B.h1[(static_cast<size_t>(c) << 8) | (lx << 4) | lz];
    const int top = h > kMaxY ? kMaxY : h;
    if (top < tbm::kMinY) return;
    const int x = B.cx[c] * 16 + lx, z = B.cz[c] * 16 + lz;
    const int ax = x - 2, az = z - 2, px = ax >> 2, pz = az >> 2;
    const int qx0 = B.cx[c] * 4 - 1, qz0 = B.cz[c] * 4 - 1;
    const uint8_t* uni_of = B.zoom_uni + static_cast<size_t>(c) * kZoomCells + (pz - qz0) * 5 + px - qx0;
    const uint32_t* tab = B.zoom_tab + static_cast<size_t>(c) * kZoomVerts;
    uint32_t* words = reinterpret_cast<uint32_t*>(B.bbiome) + static_cast<size_t>(c) * kColWords * 256 + col;
    double sx[8], sz[8], oy[8];
    int g_cur = -1;
    uint8_t uni = 0;
    uint32_t word = 0;
    for (int y = tbm::kMinY; y <= top; ++y) {
        const int py = (y - 2) >> 2, g = py - kZoomPyMin;
        if (g != g_cur) {
            g_cur = g;
            uni = uni_of[g * 25];
            if (uni == kZoomMixed) {
                const double fx = static_cast<double>(ax & 3) / 4.0, fz = static_cast<double>(az & 3) / 4.0;
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    const bool xe = (i & 4) == 0, ye = (i & 2) == 0, ze = (i & 1) == 0;
                    const int qx = xe ? px : px + 1, qy = ye ? py : py + 1, qz = ze ? pz : pz + 1;
                    const uint32_t m = tab[((qy - kZoomQyMin) * 6 + (qz - qz0)) * 6 + (qx - qx0)];
                    const double ox = zoom_fiddle(static_cast<int32_t>(m & 1023u));
                    oy[i] = zoom_fiddle(static_cast<int32_t>((m >> 10) & 1023u));
                    const double oz = zoom_fiddle(static_cast<int32_t>(m >> 20));
                    const double dx = xe ? fx : fx - 1.0, dz = ze ? fz : fz - 1.0;
                    sz[i] = (dz + oz) * (dz + oz);
                    sx[i] = (dx + ox) * (dx + ox);
                }
            }
        }
        uint32_t biome = uni;
        if (uni == kZoomMixed) {
            const double fy = static_cast<double>((y - 2) & 3) / 4.0;
            int best = 0;
            double best_d = 0.0;
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                const double dy = (i & 2) == 0 ? fy : fy - 1.0;
                const double sy = (dy + oy[i]) * (dy + oy[i]);
                const double d = sz[i] + sy + sx[i];
                if (i == 0 || best_d > d) {
                    best = i;
                    best_d = d;
                }
            }
            biome = static_cast<uint32_t>(zoom_stored(B, c, best, px, py, pz));
        }
        const int r = y - tbm::kMinY;
        word |= biome << (8 * (r & 3));
        if ((r & 3) == 3 || y == top) {
            words[(r >> 2) * 256] = word;
            word = 0;
        }
    }
}

TB_HD TB_NOINLINE inline float biome_temperature(const DevModel& M, int biome, int x, int y, int z) {
    float adjusted = M.biome_temp[biome];
    if (M.biome_frozen[biome]) {
        float fv = 0.0f;
        const double freq[3] = {1.0, 0.5, 0.25};
        for (int i = 0; i < 3; ++i)
            fv = fv + M.frozen_amp[i] * simplex2(M.frozen[i], static_cast<double>(x) * 0.05 * freq[i], static_cast<double>(z) * 0.05 * freq[i], M.f2, M.g2);
        const double large = static_cast<double>(fv * 7.0f);
        const double edge = static_cast<double>(simplex2(M.info, static_cast<double>(x) * 0.2, static_cast<double>(z) * 0.2, M.f2, M.g2));
        if (large + edge < 0.3) {
            const double small = static_cast<double>(simplex2(M.info, static_cast<double>(x) * 0.09, static_cast<double>(z) * 0.09, M.f2, M.g2));
            if (small < 0.8) adjusted = 0.2f;
        }
    }
    constexpr int snow = tbm::kTmSeaLevel + 17;
    if (y > snow) {
        const float v = simplex2(M.temp, static_cast<double>(static_cast<float>(x) / 8.0f), static_cast<double>(static_cast<float>(z) / 8.0f), M.f2, M.g2) * 8.0f;
        float t = v + static_cast<float>(y);
        t = t - static_cast<float>(snow);
        t = t * 0.05f;
        t = t / 40.0f;
        return adjusted - t;
    }
    return adjusted;
}

// ---- surface: one column ----------------------------------------------------------------------
struct Column {
    const Batch* B;
    const DevSeed* S;
    uint16_t* blocks;     // chunk blocks
    int c, lx, lz, bx, bz;
    int hm;               // live WORLD_SURFACE_WG value of this column (first available y)

    TB_HD TB_FI size_t idx(int y) const { return static_cast<size_t>(((y - tbm::kMinY) * 16 + lz) * 16 + lx); }
    TB_HD TB_FI int get(int y) const { return (y < tbm::kMinY || y > kMaxY) ? tbm::kAir : blocks[idx(y)]; }
    TB_HD TB_FI uint8_t flags(int s) const { return B->M.block_flags[s]; }
    // ProtoChunk.setBlockState plus the heightmap update
    TB_HD inline void set(int y, int state) {
        if (y < tbm::kMinY || y > kMaxY) return;
        blocks[idx(y)] = static_cast<uint16_t>(state);
        const int first = hm;
        if (y <= first - 2) return;
        if (!(flags(state) & 1)) {
            if (y >= first) hm = y + 1;
        } else if (first - 1 == y) {
            for (int yy = y - 1; yy >= tbm::kMinY; --yy)
                if (!(flags(blocks[idx(yy)]) & 1)) {
                    hm = yy + 1;
                    return;
                }
            hm = tbm::kMinY;
        }
    }
    template <int K>
    TB_HD TB_FI double noise(double x, double y, double z) const {
        constexpr int first = tbm::kNoiseFirst[K], count = tbm::kNoiseCount[K];
        return static_cast<double>(stack_point<first, count, false>(S->nt, x, y, z));
    }
};

TB_HD inline void eroded_badlands(Column& C, int height) {
    const double a = dabs(C.noise<tbm::kNoise_badlands_surface>(C.bx, 0.0, C.bz) * 8.25);
    const double b = static_cast<double>(static_cast<float>(C.noise<tbm::kNoise_badlands_pillar>(C.bx * 0.2, 0.0, C.bz * 0.2)) * 15.0f);
    const double pillar = jmind(a, b);
    if (pillar <= 0.0) return;
    const double floor_v = dabs(C.noise<tbm::kNoise_badlands_pillar_roof>(C.bx * 0.75, 0.0, C.bz * 0.75) * 1.5);
    const double top = 64.0 + jmind(pillar * pillar * 2.5, ::ceil(floor_v * 50.0) + 24.0);
    const int start = jfloor(top);
    if (height > start) return;
    for (int y = start; y >= tbm::kMinY; --y) {
        const int old = C.get(y);
        if (old == tbm::kDefaultBlock) break;
        if (C.flags(old) & 2) return;
    }
    for (int y = start; y >= tbm::kMinY && (C.flags(C.get(y)) & 1); --y) C.set(y, tbm::kDefaultBlock);
}

// Frozen-ocean iceberg extension; with write == false only the heightmap effect is
// simulated (the rule tree never turns air or fluid into anything else, so the
// decisions are the same before and after the rules).
TB_HD inline void frozen_ocean(Column& C, int min_surface, int biome, int height, bool write) {
    const double a = dabs(C.noise<tbm::kNoise_iceberg_surface>(C.bx, 0.0, C.bz) * 8.25);
    const double b = static_cast<double>(static_cast<float>(C.noise<tbm::kNoise_iceberg_pillar>(C.bx * 1.28, 0.0, C.bz * 1.28)) * 15.0f);
    const double berg = jmind(a, b);
    if (berg <= 1.8) return;
    const double roof = dabs(C.noise<tbm::kNoise_iceberg_pillar_roof>(C.bx * 1.17, 0.0, C.bz * 1.17) * 1.5);
    double top = jmind(berg * berg * 1.2, ::ceil(roof * 40.0) + 14.0);
    constexpr int sea = tbm::kTmSeaLevel;
    if (biome_temperature(C.B->M, biome, C.bx, sea, C.bz) > 0.1f) top -= 2.0;
    if (top <= 2.0) return;
    const double bottom = static_cast<double>(sea) - top - 7.0;
    top += static_cast<double>(sea);
    Xoro r = C.S->random.at(C.bx, 0, C.bz);
    const int max_snow = 2 + r.next_int(4);
    const int min_snow_height = sea + 18 + r.next_int(10);
    int snow = 0;
    const int itop = d2i(top), ibottom = d2i(bottom);
    const int y0 = height > itop + 1 ? height : itop + 1;
    for (int y = y0; y >= min_surface; --y) {
        const int g = C.get(y);
        bool place = false;
        if ((C.flags(g) & 1) && y < itop && r.next_double() > 0.01) place = true;
        else if (g == tbm::kWater && y > ibottom && y < sea && r.next_double() > 0.15) place = true;
        if (place) {
            int state;
            if (snow <= max_snow && y > min_snow_height) {
                state = tbm::kSnowBlock;
                ++snow;
            } else {
                state = tbm::kPackedIce;
            }
            if (write) {
                C.set(y, state);
            } else if (y >= tbm::kMinY && y <= kMaxY) {
                // heightmap effect of set() for a solid state, without writing
                if (!(y <= C.hm - 2) && y >= C.hm) C.hm = y + 1;
            }
        }
    }
}

// surface/chunk_surface_level at column (lx, lz): InterpolatedFunction 16x1 over the
// four chunk-corner find_top_surface values (volume semantics, in the aquifer window).
TB_HD TB_FI float prelim_surface(const Batch& B, int c, int lx, int lz) {
    const int32_t* g = B.g513 + static_cast<size_t>(c) * kGrid;
    const float c00 = B.sfts[g[8 * kGridX + 16]], c10 = B.sfts[g[8 * kGridX + 20]];
    const float c01 = B.sfts[g[12 * kGridX + 16]], c11 = B.sfts[g[12 * kGridX + 20]];
    const float az = static_cast<float>(lz) * 0.0625f, ax = static_cast<float>(lx) * 0.0625f;
    const float v00 = lerpf(az, c00, c01), v01 = lerpf(az, c00, c01);
    const float v10 = lerpf(az, c10, c11), v11 = lerpf(az, c10, c11);
    const float a0 = lerpf(ax, v00, v10), a1 = lerpf(ax, v01, v11);
    const float step = (a1 - a0) * 1.0f;
    return a0 + step * 0.0f;
}

// Channel k of one block: cell_interp's arithmetic for that channel, then the step added
// once per block above the cell floor, as in the fill. Out of line.
TB_HD TB_NOINLINE inline float block_channel(const Batch& B, int c, int lx, int lz, int y, int k) {
    const int cell_y = (y - tbm::kMinY) >> 3, yi = (y - tbm::kMinY) & 7;
    const int ci = lx >> 2, xi = lx & 3, ck = lz >> 2, zi = lz & 3;
    const int32_t* cc = B.c25 + static_cast<size_t>(c) * 25;
    const size_t u00 = cc[ck * 5 + ci], u10 = cc[ck * 5 + ci + 1], u01 = cc[(ck + 1) * 5 + ci], u11 = cc[(ck + 1) * 5 + ci + 1];
    const int C = tbm::kNumChannels;
    const float* p00 = B.corners + (u00 * kRows + cell_y) * C;
    const float* p10 = B.corners + (u10 * kRows + cell_y) * C;
    const float* p01 = B.corners + (u01 * kRows + cell_y) * C;
    const float* p11 = B.corners + (u11 * kRows + cell_y) * C;
    const float az = static_cast<float>(zi) * 0.25f, ax = static_cast<float>(xi) * 0.25f;
    const float v000 = p00[k], v100 = p10[k], v001 = p01[k], v101 = p11[k];
    const float v010 = p00[C + k], v110 = p10[C + k], v011 = p01[C + k], v111 = p11[C + k];
    const float v00 = lerpf(az, v000, v001), v01 = lerpf(az, v010, v011);
    const float v10 = lerpf(az, v100, v101), v11 = lerpf(az, v110, v111);
    const float a0 = lerpf(ax, v00, v10), a1 = lerpf(ax, v01, v11);
    const float step = (a1 - a0) * 0.125f;
    float v = a0 + step * 0.0f;
    for (int q = 0; q < yi; ++q) v += step;
    return v;
}

// Channel values of one block, each interpolated on its first use: the generated ore
// functions read a channel only under the guards that need it (a vein's y range, for one),
// and a vein reads few of them (its density one, its richness two more).
struct LazyChannels {
    const Batch* B;
    int c, lx, lz, y;
    mutable uint32_t set;
    mutable float v[tbm::kNumChannels];
    TB_HD TB_FI float operator[](int k) const {
        if (!((set >> k) & 1u)) {
            v[k] = block_channel(*B, c, lx, lz, y, k);
            set |= 1u << k;
        }
        return v[k];
    }
};

// OreVeinRule past its density test (density > 0): the positional draw, richness on the
// volume path (channel values), the filler gap on the point path. Inputs by value, so
// that the rule context of the caller stays in registers.
TB_HD TB_NOINLINE inline int ore_vein_hit(const Batch& B, int c, int lx, int lz, int bx, int y, int bz, const DevSeed& S, int k, int ore, int raw,
                                          int filler, float chance, float density) {
    const NoiseTables& T = S.nt;
    Xoro r = S.ore.at(bx, y, bz);
    if (r.next_float() > density) return -1;
    const LazyChannels ch{&B, c, lx, lz, y, 0u, {}};
    const float richness = tbgen::gen_ore_richness(k, T, bx, y, bz, ch);
    if (r.next_float() < richness && tbgen::gen_ore_gap(k, T, bx, y, bz) < 0.0f) return r.next_float() < chance ? raw : ore;
    return filler;
}

// Block context handed to the generated rule tree (MaterialSystem's per-block state).
static_assert(tbgen::kRuleNoise2d <= 32, "2-D threshold noise memo slots fit one 32-bit mask");
struct RuleCtx {
    Column* col;
    const Batch* B;
    int c;
    // column
    int surface_depth, grad_x, grad_z;
    bool sec_set, min_set;
    double secondary;
    int min_surf;
    float prelim;
    // column values the rules read, each evaluated at its first use and kept for the
    // column's other blocks: the 2-D threshold noises (by memo slot) and the clay-band offset
    double n2d[tbgen::kRuleNoise2d > 0 ? tbgen::kRuleNoise2d : 1];
    uint32_t n2d_set;
    int band_off;
    bool band_set;
    // block
    int y, stone_above, stone_below, water_height;
    int biome_v;        // zoomed biome of the block
    uint32_t ore_bits;  // its ore-vein density tests

    TB_HD TB_FI int biome() const { return biome_v; }
    TB_HD TB_FI double noise2d(int slot, int first, int count) {
        if (!((n2d_set >> slot) & 1u)) {
            n2d[slot] = static_cast<double>(stack_point_rt(col->S->nt, first, count, col->bx, 0.0, col->bz));
            n2d_set |= 1u << slot;
        }
        return n2d[slot];
    }
    // The walk leaves a block whose rules need a per-block noise or an ore vein past its
    // density bit (rare, costly, and in different iterations of each thread's walk) to the
    // deferred pass, where the threads of a warp evaluate such blocks side by side: with
    // defer set these set deferred and give NaN / nothing, and the walk discards the state.
    bool defer, deferred;
    TB_HD TB_FI double noise3d(int k, int first, int count) {
        if (defer) {
            deferred = true;
            return bitsd(0x7FF8000000000000ull);   // a quiet NaN: its tests come out false
        }
        return static_cast<double>(stack_point_rt(col->S->nt, first, count, col->bx, y, col->bz));
    }
    TB_HD TB_FI bool vgradient(int k, int true_at, int false_at) const {
        if (y <= true_at) return true;
        if (y >= false_at) return false;
        const double t = (static_cast<double>(y) - true_at) / static_cast<double>(false_at - true_at);
        const double probability = 1.0 + t * (0.0 - 1.0);
        Xoro r = col->S->gradient[k].at(col->bx, y, col->bz);
        return static_cast<double>(r.next_float()) < probability;
    }
    TB_HD TB_FI bool cold() { return !(biome_temperature(B->M, biome(), col->bx, y, col->bz) >= 0.15f); }
    TB_HD TB_FI int min_surface() {
        if (!min_set) {
            min_surf = jfloor(static_cast<double>(prelim)) + surface_depth - 8;
            min_set = true;
        }
        return min_surf;
    }
    TB_HD TB_FI int secondary_depth(int range) {
        if (!sec_set) {
            secondary = col->noise<tbm::kNoise_surface_secondary>(col->bx, 0.0, col->bz);
            sec_set = true;
        }
        const double t = (secondary - -1.0) / (1.0 - -1.0);
        return d2i(0.0 + t * (static_cast<double>(range) - 0.0));
    }
    TB_HD TB_FI int band() {
        if (!band_set) {
            band_off = jround(static_cast<float>(col->noise<tbm::kNoise_clay_bands_offset>(col->bx, 0.0, col->bz)) * 4.0f);
            band_set = true;
        }
        return col->S->clay[(y + band_off + 192) % 192];
    }
    // OreVeinRule: the density inline (its guards usually end it after a y test), the rest
    // out of line
    TB_HD TB_FI int ore_vein(int k, int ore, int raw, int filler, float chance) {
        if (TB_ORE_MASK && !((ore_bits >> k) & 1)) return -1;
        if (TB_DEFER_ORE && defer) {
            deferred = true;
            return -1;
        }
        const LazyChannels ch{B, c, col->lx, col->lz, y, 0u, {}};
        const float density = tbgen::gen_ore_density(k, col->S->nt, col->bx, y, col->bz, ch);
        if (density <= 0.0f) return -1;
        return ore_vein_hit(*B, c, col->lx, col->lz, col->bx, y, col->bz, *col->S, k, ore, raw, filler, chance, density);
    }
};

// pass 1 (item = chunk * 256 + z * 16 + x): eroded badlands (writes), heights after it
// and after a dry run of the frozen-ocean extension
// Air and fluid words of one column rebuilt from its blocks, after a pass that turned air
// into other blocks.
TB_HD inline void column_mask_rebuild(const Batch& B, const Column& C) {
    uint32_t* cm = B.colmask + static_cast<size_t>(C.c) * 2 * kMaskWords * 256 + C.lz * 16 + C.lx;
    for (int w = 0; w < kMaskWords; ++w) {
        uint32_t air = 0, fluid = 0;
        for (int k = 0; k < 32; ++k) {
            const uint8_t f = C.flags(C.get(tbm::kMinY + 32 * w + k));
            air |= static_cast<uint32_t>(f & 1) << k;
            fluid |= static_cast<uint32_t>((f >> 3) & 1) << k;
        }
        cm[w * 256] = air;
        cm[(kMaskWords + w) * 256] = fluid;
    }
}

// surface1's warps hold 4 x 8 column tiles too (0.491 -> 0.484 ms per 12,288-chunk step)
#ifndef TB_S1_TILE
#define TB_S1_TILE 4
#endif
TB_HD inline void body_surface1(const Batch& B, int it) {
    const int c = it >> 8, col1 = tile_column<TB_S1_TILE>(it), lz = col1 >> 4, lx = col1 & 15;
    const int ci = (c << 8) | (lx << 4) | lz;   // x * 16 + z column index
    Column C{&B, &B.seeds[B.cseed[c]], B.blocks + static_cast<size_t>(c) * kBlocksPerChunk, c, lx, lz, B.cx[c] * 16 + lx, B.cz[c] * 16 + lz,
             B.h0[ci]};
    const int start_h = C.hm;
    const int surface_biome = zoom_biome_tab(B, c, C.bx, start_h, C.bz);
    if (surface_biome == tbm::kBiomeErodedBadlands) {
        eroded_badlands(C, start_h);
        column_mask_rebuild(B, C);
    }
    B.h1[ci] = C.hm;
    if (surface_biome == tbm::kBiomeFrozenOcean || surface_biome == tbm::kBiomeDeepFrozenOcean) {
        const double n = C.noise<tbm::kNoise_surface>(C.bx, 0.0, C.bz);
        const double rr = C.S->random.at(C.bx, 0, C.bz).next_double();
        const int sd = d2i(n * 2.75 + 3.0 + rr * 0.25);
        const int min_surface = jfloor(static_cast<double>(prelim_surface(B, c, lx, lz))) + sd - 8;
        frozen_ocean(C, min_surface, surface_biome, start_h, false);
    }
    B.h2[ci] = C.hm;
}

// pass 2 fused (item = chunk * 256 + z * 16 + x): the column context and the top-down walk,
// applying the rule tree to each solid block as the walk reaches it (the blocks below it,
// which the walk still reads, are untouched; the rules never turn a block into air or a
// fluid). A warp holds 32 columns of one chunk at the same y, as the per-block pass does.
// The walk's item order: the 32 lanes of a warp hold a tile of TB_WALK_TILE columns in x by
// 32 / TB_WALK_TILE in z (a compact tile has closer heights and rule paths than a strip).
#ifndef TB_WALK_TILE
#define TB_WALK_TILE 8
#endif
TB_HD TB_FI int walk_column(int it) { return tile_column<TB_WALK_TILE>(it); }
TB_HD inline void body_surface_walk_rules(const Batch& B, int it) {
    const int wcol = walk_column(it);
    const int c = it >> 8, lz = wcol >> 4, lx = wcol & 15;
    const int ci = (c << 8) | (lx << 4) | lz;   // x * 16 + z column index
    const size_t hb = static_cast<size_t>(c) * 256;
    Column C{&B, &B.seeds[B.cseed[c]], B.blocks + static_cast<size_t>(c) * kBlocksPerChunk, c, lx, lz, B.cx[c] * 16 + lx, B.cz[c] * 16 + lz,
             B.h1[ci]};
    auto H = [&](int x, int z) -> int {
        if (x == lx && z == lz) return B.h1[hb + x * 16 + z] - 1;
        const bool done = x < lx || (x == lx && z < lz);
        return (done ? B.h2[hb + x * 16 + z] : B.h0[hb + x * 16 + z]) - 1;
    };
    ColumnRec r;
    r.start_h = B.h0[ci];
    r.surface_biome = zoom_biome_tab(B, c, C.bx, r.start_h, C.bz);
    r.grad_x = H(lx + 1 < 15 ? lx + 1 : 15, lz) - H(lx - 1 > 0 ? lx - 1 : 0, lz);
    r.grad_z = H(lx, lz + 1 < 15 ? lz + 1 : 15) - H(lx, lz - 1 > 0 ? lz - 1 : 0);
    const double n = C.noise<tbm::kNoise_surface>(C.bx, 0.0, C.bz);
    const double rr = C.S->random.at(C.bx, 0, C.bz).next_double();
    r.surface_depth = d2i(n * 2.75 + 3.0 + rr * 0.25);
    r.min_surface = jfloor(static_cast<double>(prelim_surface(B, c, lx, lz))) + r.surface_depth - 8;
    r.secondary = C.noise<tbm::kNoise_surface_secondary>(C.bx, 0.0, C.bz);
    B.colrec[ci] = r;
    RuleCtx R{};
    R.col = &C;
    R.B = &B;
    R.c = c;
    R.surface_depth = r.surface_depth;
    R.grad_x = r.grad_x;
    R.grad_z = r.grad_z;
    R.min_set = true;
    R.min_surf = r.min_surface;
    R.sec_set = true;
    R.secondary = r.secondary;
    R.defer = B.defer != nullptr;
    // The walk reads the column's air and fluid bits, which stay true while it runs (the rules
    // never make air or fluid). All lanes of a warp walk the same height: above its own
    // height a column holds air, which leaves the walk state as it starts.
    const uint32_t* cm = B.colmask + static_cast<size_t>(c) * 2 * kMaskWords * 256 + wcol;
    const int height = C.hm;
#if defined(__CUDA_ARCH__)
    const int start = warp_max(height > kMaxY ? kMaxY : height);
#else
    // the host build takes the maximum over the same 32 items a device warp holds
    int start = INT_MIN;
    for (int j = it & ~31; j < (it & ~31) + 32; ++j) {
        const int jc = walk_column(j);
        const int h = B.h1[(static_cast<size_t>(c) << 8) | ((jc & 15) << 4) | (jc >> 4)];
        start = imax(start, h > kMaxY ? kMaxY : h);
    }
#endif
    // Zoomed biomes and ore bits, 4 heights per word: the walk descends one height at a time,
    // so the word below is loaded while the current one is in use.
    const uint32_t* bwords = reinterpret_cast<const uint32_t*>(B.bbiome) + static_cast<size_t>(c) * kColWords * 256 + wcol;
    const uint32_t* owords = reinterpret_cast<const uint32_t*>(B.oremask) + static_cast<size_t>(c) * kColWords * 256 + wcol;
    int wq = (start - tbm::kMinY) >> 2;
    uint32_t bq = bwords[wq * 256], oq = TB_ORE_MASK ? owords[wq * 256] : 0u;
    uint32_t bq_next = 0, oq_next = 0;
    if (wq > 0) {
        bq_next = bwords[(wq - 1) * 256];
        if (TB_ORE_MASK) oq_next = owords[(wq - 1) * 256];
    }
    int stone_above = 0, water_height = INT_MIN, next_ceiling = INT_MAX;
    int wi = -1;
    uint32_t aw = 0, fw = 0;
    for (int y = start; y >= tbm::kMinY; --y) {
        const int r = y - tbm::kMinY;
        if ((r >> 5) != wi) {
            wi = r >> 5;
            aw = cm[wi * 256];
            fw = cm[(kMaskWords + wi) * 256];
        }
        if ((r >> 2) != wq) {
            wq = r >> 2;
            bq = bq_next;
            oq = oq_next;
            if (wq > 0) {
                bq_next = bwords[(wq - 1) * 256];
                if (TB_ORE_MASK) oq_next = owords[(wq - 1) * 256];
            }
        }
        const uint32_t bit = 1u << (r & 31);
        if (aw & bit) {
            stone_above = 0;
            water_height = INT_MIN;
        } else if (fw & bit) {
            if (water_height == INT_MIN) water_height = y + 1;
        } else {
            if (next_ceiling >= y) {
                // one above the highest air or fluid block below y; below the world is air
                uint32_t m = (aw | fw) & (bit - 1u);
                int w = wi;
                while (m == 0 && w > 0) {
                    --w;
                    m = cm[w * 256] | cm[(kMaskWords + w) * 256];
                }
                next_ceiling = m != 0 ? tbm::kMinY + 32 * w + hibit(m) + 1 : tbm::kMinY;
            }
            ++stone_above;
            R.y = y;
            R.stone_above = stone_above;
            R.stone_below = y - next_ceiling + 1;
            R.water_height = water_height;
            R.biome_v = static_cast<int>((bq >> (8 * (r & 3))) & 255u);
            R.ore_bits = (oq >> (8 * (r & 3))) & 255u;
            R.deferred = false;
            int state = tbgen::apply_rules(R);
            if (R.deferred) {
                const int32_t slot = add32(B.defer_count, 1);
                if (slot < B.defer_cap) {
                    B.defer[slot] = DeferRec{ci, static_cast<int16_t>(y), static_cast<int16_t>(stone_above), static_cast<int16_t>(R.stone_below),
                                             water_height == INT_MIN ? kNoWater : static_cast<int16_t>(water_height), static_cast<uint8_t>(R.biome_v),
                                             static_cast<uint8_t>(R.ore_bits), 0};
                    continue;
                }
                // the list is full: the block's rules run here after all
                R.defer = false;
                state = tbgen::apply_rules(R);
                R.defer = true;
            }
            if (state >= 0) C.blocks[C.idx(y)] = static_cast<uint16_t>(state);
        }
    }
}

// deferred pass (item = index into the walk's deferred list): the material rules of a block
// the walk left, from the inputs it recorded and its column's context (ColumnRec)
TB_HD inline void body_walk_deferred(const Batch& B, int it) {
    if (it >= B.defer_cap) return;
    const DeferRec d = B.defer[it];
    const int c = d.column >> 8, ci = d.column & 255, lx = ci >> 4, lz = ci & 15;
    Column C{&B, &B.seeds[B.cseed[c]], B.blocks + static_cast<size_t>(c) * kBlocksPerChunk, c, lx, lz, B.cx[c] * 16 + lx, B.cz[c] * 16 + lz,
             B.h1[d.column]};
    const ColumnRec& r = B.colrec[d.column];
    RuleCtx R{};
    R.col = &C;
    R.B = &B;
    R.c = c;
    R.surface_depth = r.surface_depth;
    R.grad_x = r.grad_x;
    R.grad_z = r.grad_z;
    R.min_set = true;
    R.min_surf = r.min_surface;
    R.sec_set = true;
    R.secondary = r.secondary;
    R.y = d.y;
    R.stone_above = d.stone_above;
    R.stone_below = d.stone_below;
    R.water_height = d.water_height == kNoWater ? INT_MIN : d.water_height;
    R.biome_v = d.biome;
    R.ore_bits = d.ore_bits;
    const int state = tbgen::apply_rules(R);
    if (state >= 0) C.blocks[C.idx(d.y)] = static_cast<uint16_t>(state);
}

// pass 2c (item = chunk * 256 + z * 16 + x): the frozen-ocean extension after the rules
TB_HD inline void body_surface_frozen(const Batch& B, int it) {
    const int c = it >> 8, lz = (it >> 4) & 15, lx = it & 15;
    const int ci = (c << 8) | (lx << 4) | lz;   // x * 16 + z column index
    const ColumnRec& r = B.colrec[ci];
    if (r.surface_biome != tbm::kBiomeFrozenOcean && r.surface_biome != tbm::kBiomeDeepFrozenOcean) return;
    Column C{&B, &B.seeds[B.cseed[c]], B.blocks + static_cast<size_t>(c) * kBlocksPerChunk, c, lx, lz, B.cx[c] * 16 + lx, B.cz[c] * 16 + lz,
             B.h1[ci]};
    frozen_ocean(C, r.min_surface, r.surface_biome, r.start_h, true);
}

// centre chunk's quart biomes to the output (item = chunk * kQuartsPerChunk + q)
TB_HD inline void body_gather(const Batch& B, int it) {
    const int c = it / kQuartsPerChunk, q = it % kQuartsPerChunk;
    B.biomes_out[it] = B.qbiome[static_cast<size_t>(B.nb9[static_cast<size_t>(c) * 9 + 4]) * kQuartsPerChunk + q];
}

}  // namespace tb
