// Test-only host build of the TERRAIN-step kernel bodies.
//
// Runs the same per-element bodies as the sm_100a kernels (csrc/tb_pipeline.cuh), in
// the same stage order, sequentially on the CPU, so the CPU test suite can compare the
// generated evaluators and every pipeline stage with the reference oracle without a
// GPU. It is a checker of the device code's arithmetic, not a product path: the
// product library (libterrain_b200.so) has no host fallback and never loads this file.
#include <cstdint>
#include <cstring>
#include <vector>

#include "tb_pipeline.cuh"

namespace tb {
long long tb_count_sink[kOpKinds];   // counts of calls made outside a counted stage
thread_local long long* tb_op_counts = tb_count_sink;
}
using namespace tb;

namespace {

// stage sink when nothing is counted
long long g_discard[kOpKinds];

struct HostRun {
    ModelHost m;
    SeedHost s;
    DevModel M{};
    DevSeed D{};
    std::vector<uint8_t> flags;
    std::vector<float> btemp;
    std::vector<uint8_t> bfrozen;

    explicit HostRun(int64_t seed) {
        build_model_host(m);
        build_seed_host(seed, s);
        flags.assign(tbm::kBlockFlags, tbm::kBlockFlags + tbm::kPaletteSize);
        btemp.assign(tbm::kBiomeTemp, tbm::kBiomeTemp + tbm::kNumBiomes);
        bfrozen.assign(tbm::kBiomeFrozen, tbm::kBiomeFrozen + tbm::kNumBiomes);
        M.boxes = m.boxes.empty() ? nullptr : m.boxes.data();
        M.box_leaf = m.box_leaf.empty() ? nullptr : m.box_leaf.data();
        M.tree = m.nodes.data();
        M.children = m.children.data();
        M.leaf_biome = m.leaf_biome.data();
        M.leaf_node = m.leaf_node.data();
        M.leaf_rank = m.leaf_rank.data();
        M.root = m.root;
        M.depth = m.depth;
        M.block_flags = flags.data();
        M.biome_temp = btemp.data();
        M.biome_frozen = bfrozen.data();
        M.temp = m.temp;
        for (int i = 0; i < 3; ++i) {
            M.frozen[i] = m.frozen[i];
            M.frozen_amp[i] = m.frozen_amp[i];
        }
        M.info = m.info;
        M.f2 = m.f2;
        M.g2 = m.g2;
        D.nt = NoiseTables{s.off.data(), s.perm.data(), s.layers.data(), s.perm2.data()};
        D.ytab = s.ytab.data();
        D.random = s.random;
        D.aquifer = s.aquifer;
        D.ore = s.ore;
        for (size_t k = 0; k < s.gradient.size(); ++k) D.gradient[k] = s.gradient[k];
        D.zoom_seed = s.zoom_seed;
        std::memcpy(D.clay, s.clay, sizeof D.clay);
    }
};

struct Table {
    std::vector<unsigned long long> keys, uniq;
    std::vector<int32_t> vals, owner;
    int32_t count = 0;
    uint32_t err = 0;
    uint32_t cap = 0;
    void init(size_t max_keys) {
        cap = 1024;
        while (cap < 2 * max_keys) cap <<= 1;
        keys.assign(cap, kEmpty);
        vals.assign(cap, -1);
        owner.assign(cap, 0x7F7F7F7F);
        uniq.assign(max_keys, 0);
        count = 0;
    }
    HashTab view() { return HashTab{keys.data(), vals.data(), uniq.data(), &count, cap - 1, owner.data(), &err}; }
};

template <class F>
void each(int n, F f) {
    for (int i = 0; i < n; ++i) f(i);
}

}  // namespace

extern "C" {

// Stages of the pipeline in the order (and with the names) of the library's tunable kernels.
enum Stage { S_NB_INSERT, S_NB_RESOLVE, S_CLIMATE_COL, S_CLIMATE_QUART, S_CHAIN, S_CC_INSERT, S_CC_RESOLVE, S_CORNER_COL, S_CORNER, S_ZOOM_TABLE,
             S_ZOOM_UNIFORM, S_SG_INSERT, S_SG_RESOLVE, S_SURFACE_LEVEL, S_AQ_CELL, S_AQ_QUERY, S_AQ_SKIP, S_INIT_HEIGHTS, S_FILL, S_SURFACE1,
             S_BLOCK_BIOME, S_WALK, S_FROZEN, S_GATHER, S_AXIS_INSERT, S_AXIS_NUMBER, S_AXIS_FILL, S_WALK_DEFER, S_COUNT };

// blocks per chunk the host twin's deferred list holds (hc_set_defer; the library's default)
int g_defer_per_chunk = 8192;

// The pipeline for n chunks of one seed, stage by stage; with counts (S_COUNT x kOpKinds),
// each stage's octave and simplex samples are counted into its row.
int run_generate(int64_t seed, const int32_t* cx, const int32_t* cz, int32_t n, uint16_t* blocks, uint8_t* biomes, uint16_t* aquifer, long long* counts,
                 int32_t* meta) {
    auto stage = [&](int k) { tb_op_counts = counts ? counts + static_cast<size_t>(k) * kOpKinds : g_discard; };
    tb_op_counts = g_discard;
    HostRun R(seed);
    std::vector<int32_t> vcx(cx, cx + n), vcz(cz, cz + n), vcs(n, 0);
    Table hb, hc, hs, ha;
    hb.init(9 * static_cast<size_t>(n));
    hc.init(25 * static_cast<size_t>(n));
    hs.init(static_cast<size_t>(kGrid) * n);
    ha.init(10 * static_cast<size_t>(n));
    const size_t N = n, nb = 9 * N, cc = 25 * N, sg = kGrid * N;
    std::vector<int32_t> nb9(9 * N), c25(25 * N), g513(sg), aq_skip(N);
    std::vector<AqCell> aq_cell(N * kAqCells);
    std::vector<AqQuery> aq_query(N * kAqQueries);
    std::vector<float> bcol(nb * 16 * tbm::kClimateCols), ccol(cc * tbm::kCornerCols), corners(cc * kRows * tbm::kNumChannels), sfts(sg);
    std::vector<long long> tgt(nb * kQuartsPerChunk * 6), mdist(nb * kQuartsPerChunk);
    std::vector<int32_t> lstar(nb * kQuartsPerChunk), h0(256 * N, tbm::kMinY), h1(256 * N), h2(256 * N);
    std::vector<uint8_t> qbiome(nb * kQuartsPerChunk), bout(N * kQuartsPerChunk);
    std::vector<uint16_t> bl(N * kBlocksPerChunk);
    std::vector<uint32_t> ztab(N * kZoomVerts);
    std::vector<uint8_t> bbiome(N * kBlocksPerChunk), oremask(N * kBlocksPerChunk);
    std::vector<uint32_t> colmask(N * 2 * kMaskWords * 256);
    std::vector<uint8_t> zuni(N * kZoomCells);
    std::vector<ColumnRec> colrec(N * 256);
    std::vector<AxisRec> axtab(10 * N * std::max(1, tbm::kAxisLayers));
    std::vector<int32_t> colax(2 * 25 * N);
    Batch B{};
    B.M = R.M;
    B.seeds = &R.D;
    B.n_dev = &n;
    B.cx = vcx.data();
    B.cz = vcz.data();
    B.cseed = vcs.data();
    B.hb = hb.view();
    B.nb_cap = static_cast<int32_t>(nb);
    B.nb9 = nb9.data();
    B.bcol = bcol.data();
    B.tgt = tgt.data();
    B.lstar = lstar.data();
    B.mdist = mdist.data();
    B.qbiome = qbiome.data();
    B.hc = hc.view();
    B.cc_cap = static_cast<int32_t>(cc);
    B.c25 = c25.data();
    B.ccol = ccol.data();
    B.ha = ha.view();
    B.axtab = axtab.data();
    B.colax = colax.data();
    B.corners = corners.data();
    B.hs = hs.view();
    B.sg_cap = static_cast<int32_t>(sg);
    B.g513 = g513.data();
    B.sfts = sfts.data();
    B.aq_cell = aq_cell.data();
    B.aq_query = aq_query.data();
    B.aq_skip = aq_skip.data();
    B.blocks = bl.data();
    B.h0 = h0.data();
    B.h1 = h1.data();
    B.h2 = h2.data();
    B.biomes_out = bout.data();
    B.zoom_tab = ztab.data();
    B.zoom_uni = zuni.data();
    B.bbiome = bbiome.data();
    B.oremask = oremask.data();
    B.colmask = colmask.data();
    B.colrec = colrec.data();
    int32_t defer_count = 0;
    std::vector<DeferRec> defer(static_cast<size_t>(g_defer_per_chunk) * N);
    B.defer = g_defer_per_chunk > 0 ? defer.data() : nullptr;
    B.defer_count = &defer_count;
    B.defer_cap = static_cast<int32_t>(defer.size());
    stage(S_NB_INSERT);
    each(9 * n, [&](int i) { body_nb_insert(B, i); });
    each(9 * n, [&](int i) { ht_number(B.hb, nb_key(B, i), i); });
    stage(S_NB_RESOLVE);
    each(9 * n, [&](int i) { body_nb_resolve(B, i); });
    stage(S_CLIMATE_COL);
    each(hb.count * 16, [&](int i) { body_climate_col(B, i); });
    stage(S_CLIMATE_QUART);
    each(hb.count * 16 * kRuns, [&](int i) { body_climate_quart(B, i); });
    stage(S_CHAIN);
    each(hb.count, [&](int i) { body_chain(B, i); });
    stage(S_CC_INSERT);
    each(25 * n, [&](int i) { body_cc_insert(B, i); });
    each(25 * n, [&](int i) { ht_number(B.hc, cc_key(B, i), i); });
    stage(S_CC_RESOLVE);
    each(25 * n, [&](int i) { body_cc_resolve(B, i); });
    if (TB_AXIS_TABLE && tbm::kAxisLayers > 0) {
        stage(S_AXIS_INSERT);
        each(hc.count * 2, [&](int i) { body_axis_insert(B, i); });
        stage(S_AXIS_NUMBER);
        each(hc.count * 2, [&](int i) { body_axis_number(B, i); });
        stage(S_AXIS_FILL);
        each(ha.count * tbm::kAxisLayers, [&](int i) { body_axis_fill(B, i); });
    }
    stage(S_CORNER_COL);
    each(hc.count, [&](int i) { body_corner_col(B, i); });
    stage(S_CORNER);
    each(hc.count * kRows, [&](int i) { body_corner(B, i); });
    stage(S_ZOOM_TABLE);
    each(kZoomVerts * n, [&](int i) { body_zoom_table(B, i); });
    stage(S_ZOOM_UNIFORM);
    each(kZoomCells * n, [&](int i) { body_zoom_uniform(B, i); });
    stage(S_SG_INSERT);
    each(kGrid * n, [&](int i) { body_sg_insert(B, i); });
    each(kGrid * n, [&](int i) { ht_number(B.hs, sg_key_item(B, i), i); });
    stage(S_SG_RESOLVE);
    each(kGrid * n, [&](int i) { body_sg_resolve(B, i); });
    stage(S_SURFACE_LEVEL);
    each(hs.count, [&](int i) { body_surface_level(B, i); });
    stage(S_AQ_CELL);
    each(kAqCells * n, [&](int i) { body_aquifer_cell(B, i); });
    stage(S_AQ_QUERY);
    each(kAqQueries * n, [&](int i) { body_aquifer_query(B, i); });
    stage(S_AQ_SKIP);
    each(n, [&](int i) { body_aquifer_skip(B, i); });
    stage(S_FILL);
    each(256 * kCellsY * n, [&](int i) { body_fill(B, i); });
    if (aquifer) std::memcpy(aquifer, bl.data(), sizeof(uint16_t) * bl.size());
    stage(S_SURFACE1);
    each(256 * n, [&](int i) { body_surface1(B, i); });
    stage(S_BLOCK_BIOME);
    each(256 * n, [&](int i) { body_block_biome(B, i); });
    stage(S_WALK);
    each(256 * n, [&](int i) { body_surface_walk_rules(B, i); });
    stage(S_WALK_DEFER);
    if (B.defer) each(std::min(defer_count, B.defer_cap), [&](int i) { body_walk_deferred(B, i); });
    if (meta) meta[3] = defer_count;
    stage(S_FROZEN);
    each(256 * n, [&](int i) { body_surface_frozen(B, i); });
    stage(S_GATHER);
    each(kQuartsPerChunk * n, [&](int i) { body_gather(B, i); });
    tb_op_counts = g_discard;
    if (meta) {
        meta[0] = hc.count;
        meta[1] = hs.count;
        meta[2] = hb.count;
    }
    std::memcpy(blocks, bl.data(), sizeof(uint16_t) * bl.size());
    if (biomes) std::memcpy(biomes, bout.data(), bout.size());
    return 0;
}

// Full pipeline for n chunks of one seed. blocks: n * 16 * 16 * height u16; biomes: n * 1536 u8
// (may be null); aquifer: blocks after the fill (may be null).
int hc_generate(int64_t seed, const int32_t* cx, const int32_t* cz, int32_t n, uint16_t* blocks, uint8_t* biomes, uint16_t* aquifer) {
    return run_generate(seed, cx, cz, n, blocks, biomes, aquifer, nullptr, nullptr);
}

// The samples each stage evaluates for n chunks (one batch): counts is S_COUNT x kOpKinds
// (volume, smeared volume, point, smeared point octave samples; simplex samples), and
// meta[0..2] the batch's distinct corner columns, surface-level quarts and biome chunks,
// meta[3] the blocks the column walk left to the deferred pass.
// Blocks per chunk of the deferred list in the following calls (0: the walk keeps every
// block), so that the tests can run the walk with a full list.
void hc_set_defer(int32_t per_chunk) { g_defer_per_chunk = per_chunk; }

int hc_count_ops(int64_t seed, const int32_t* cx, const int32_t* cz, int32_t n, long long* counts, int32_t* meta) {
    std::vector<uint16_t> bl(static_cast<size_t>(n) * kBlocksPerChunk);
    std::memset(counts, 0, sizeof(long long) * S_COUNT * kOpKinds);
    return run_generate(seed, cx, cz, n, bl.data(), nullptr, nullptr, counts, meta);
}

// Point-path root values at positions (root: 0 barrier, 1 floodedness, 2 spread, 3 lava,
// 4 exclusion, 5 find_top_surface density, 6 fts volume (x, z), 7 fts point (x, z)).
int hc_point(int64_t seed, int32_t root, const int32_t* xyz, int32_t n, float* out) {
    HostRun R(seed);
    const NoiseTables& T = R.D.nt;
    for (int i = 0; i < n; ++i) {
        const int x = xyz[3 * i], y = xyz[3 * i + 1], z = xyz[3 * i + 2];
        float v = 0.0f;
        switch (root) {
            case 0: v = tbgen::gen_aq_barrier(T, x, y, z); break;
            case 1: v = tbgen::gen_aq_fluid_level_floodedness(T, x, y, z); break;
            case 2: v = tbgen::gen_aq_fluid_level_spread(T, x, y, z); break;
            case 3: v = tbgen::gen_aq_lava(T, x, y, z); break;
            case 4: v = tbgen::gen_aq_exclusion(T, x, y, z); break;
            case 5: v = tbgen::gen_fts_density(T, x, y, z); break;
            case 6: v = tbgen::gen_fts_vol(T, x, z); break;
            case 7: v = tbgen::gen_fts_pt(T, x, z); break;
            default: return -1;
        }
        out[i] = v;
    }
    return 0;
}

// Climate roots (volume path) at quart positions: out 6 floats per position.
int hc_climate(int64_t seed, const int32_t* xyz, int32_t n, float* out) {
    HostRun R(seed);
    float col[tbm::kClimateCols];
    for (int i = 0; i < n; ++i) {
        tbgen::gen_climate_col(R.D.nt, xyz[3 * i], xyz[3 * i + 2], col);
        tbgen::gen_climate(R.D.nt, xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2], col, out + 6 * i);
    }
    return 0;
}

// Interpolation-channel inputs (volume path) at cell-corner positions: kNumChannels floats each.
// The axis-table records of every table layer at one x (or z) block coordinate, as the
// batch's axis_fill stage writes them.
void axis_row(const NoiseTables& T, int32_t b, bool z, AxisRec* row) {
    for (int e = 0; e < tbm::kAxisLayers; ++e) {
        const Layer L = T.layer[tbm::kAxisLayer[e]];
        const OctaveOff o = T.off[L.oct];
        const AxisSetup a = axis_setup(b, tbm::kAxisScale[e] * L.freq, z ? o.oz : o.ox);
        row[e] = AxisRec{a.f, a.r, a.a, z ? 0 : static_cast<int32_t>(T.perm2[256 * L.oct + (static_cast<uint32_t>(a.f) & 255u)])};
    }
}

int hc_corners(int64_t seed, const int32_t* xyz, int32_t n, float* out) {
    HostRun R(seed);
    float col[tbm::kCornerCols];
    std::vector<AxisRec> ax(std::max(1, tbm::kAxisLayers)), az(std::max(1, tbm::kAxisLayers)), ay(std::max(1, tbm::kYLayers));
    for (int i = 0; i < n; ++i) {
        tbgen::gen_corner_col(R.D.nt, xyz[3 * i], xyz[3 * i + 2], col);
        axis_row(R.D.nt, xyz[3 * i], false, ax.data());
        axis_row(R.D.nt, xyz[3 * i + 2], true, az.data());
        // the y records at this height, as the seed's table holds them for a corner row
        for (int e = 0; e < tbm::kYLayers; ++e) ay[e] = y_record(R.D.nt, tbm::kYLayer[e], tbm::kYScale[e], tbm::kYSmeared[e], xyz[3 * i + 1]);
        tbgen::gen_corner(R.D.nt, xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2], col, ax.data(), az.data(), ay.data(), out + tbm::kNumChannels * i);
    }
    return 0;
}

int hc_num_channels() { return tbm::kNumChannels; }

// Per-seed host scalars: zoom seed, positional factories (random, aquifer, ore), clay bands.
int hc_seed_scalars(int64_t seed, int64_t* out7, int32_t* clay) {
    SeedHost s;
    build_seed_host(seed, s);
    out7[0] = s.zoom_seed;
    out7[1] = static_cast<int64_t>(s.random.lo);
    out7[2] = static_cast<int64_t>(s.random.hi);
    out7[3] = static_cast<int64_t>(s.aquifer.lo);
    out7[4] = static_cast<int64_t>(s.aquifer.hi);
    out7[5] = static_cast<int64_t>(s.ore.lo);
    out7[6] = static_cast<int64_t>(s.ore.hi);
    for (int i = 0; i < 192; ++i) clay[i] = s.clay[i];
    return 0;
}

// Layers of one noise key index: frequency, amplitude, offsets, permutations.
int hc_noise_layers(int64_t seed, int32_t key, double* freq, float* amp, double* offs, uint8_t* perms) {
    SeedHost s;
    build_seed_host(seed, s);
    const int first = tbm::kNoiseFirst[key], count = tbm::kNoiseCount[key];
    for (int i = 0; i < count; ++i) {
        const Layer& L = s.layers[first + i];
        freq[i] = L.freq;
        amp[i] = L.amp;
        offs[3 * i] = s.off[L.oct].ox;
        offs[3 * i + 1] = s.off[L.oct].oy;
        offs[3 * i + 2] = s.off[L.oct].oz;
        std::memcpy(perms + 256 * i, s.perm.data() + 256 * L.oct, 256);
    }
    return count;
}

void hc_md5(const uint8_t* d, int64_t n, uint8_t* out) { md5(d, static_cast<size_t>(n), out); }
void hc_sha256(const uint8_t* d, int64_t n, uint8_t* out) { sha256(d, static_cast<size_t>(n), out); }

}  // extern "C"

extern "C" {
// Distance evaluations of the first-minimal-leaf search for each target (6 int64 each),
// starting from the previous target's leaf (a column run), for search-cost studies.
int hc_tree_visits(const long long* t, int32_t n, int32_t* visits, int32_t* leaves) {
    ModelHost m;
    build_model_host(m);
    int prev = 0;
    for (int i = 0; i < n; ++i) {
        const long long* q = t + 6 * i;
        int best = prev, best_rank = m.leaf_rank[prev];
        auto dist = [&](const RNode& nd) {
            long long d = 0;
            for (int k = 0; k < 7; ++k) {
                const long long tv = k < 6 ? q[k] : 0;
                const long long a = tv - nd.mx[k], b = nd.mn[k] - tv;
                const long long p = a > 0 ? a : (b > 0 ? b : 0);
                d += p * p;
            }
            return d;
        };
        long long best_d = dist(m.nodes[m.leaf_node[prev]]);
        int cnt = 0;
        std::vector<std::pair<int, int>> st{{m.root, 0}};
        while (!st.empty()) {
            auto& f = st.back();
            const RNode& nd = m.nodes[f.first];
            if (f.second >= nd.child_count) { st.pop_back(); continue; }
            const int ci = m.children[nd.first_child + f.second++];
            const RNode& ch = m.nodes[ci];
            const long long d = dist(ch);
            ++cnt;
            if (d < best_d || (d == best_d && ch.rank < best_rank)) {
                if (ch.leaf >= 0) { best = ch.leaf; best_rank = ch.rank; best_d = d; }
                else st.push_back({ci, 0});
            }
        }
        visits[i] = cnt;
        leaves[i] = best;
        prev = best;
    }
    return 0;
}
}

extern "C" {
// Biome lookups of one seed through the single-block path (biome_point): n xyz triples.
int hc_biome_point(int64_t seed, const int32_t* xyz, int32_t n, uint8_t* out) {
    HostRun R(seed);
    for (int i = 0; i < n; ++i) out[i] = static_cast<uint8_t>(biome_point(R.M, R.D, xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]));
    return 0;
}
}

extern "C" {
// Climate tree shape: depth (root = 1), node count, whether the 32-bit search applies.
int hc_tree_info(int32_t* out3) {
    ModelHost m;
    build_model_host(m);
    out3[0] = m.depth;
    out3[1] = static_cast<int32_t>(m.nodes.size());
    out3[2] = m.boxes.empty() ? 0 : 1;
    return 0;
}
}

extern "C" {
// Java-semantics helpers and random sources of the product, for known-answer tests.
int32_t hc_d2i(double v) { return d2i(v); }
int32_t hc_jfloor(double v) { return jfloor(v); }
int32_t hc_fdiv(int32_t a, int32_t b) { return fdiv(a, b); }
int32_t hc_fmod(int32_t a, int32_t b) { return fmod_i(a, b); }
float hc_jmin(float a, float b) { return jmin(a, b); }
float hc_jmax(float a, float b) { return jmax(a, b); }
float hc_fabs(float a) { return fabs_j(a); }
int64_t hc_f2l(float v) { return f2l(v); }
double hc_nwrap(double v) { return nwrap(v); }
float hc_grad(int32_t h, int32_t c) { return c == 0 ? gx_of(static_cast<uint32_t>(h)) : (c == 1 ? gy_of(static_cast<uint32_t>(h)) : gz_of(static_cast<uint32_t>(h))); }
int64_t hc_pos_seed(int32_t x, int32_t y, int32_t z) { return pos_seed(x, y, z); }
int hc_xoroshiro_longs(int64_t seed, int32_t n, int64_t* out) {
    Xoro r = Xoro::from_seed(seed);
    for (int i = 0; i < n; ++i) out[i] = static_cast<int64_t>(r.next());
    return n;
}
int hc_xoroshiro_ints(int64_t seed, int32_t bound, int32_t n, int32_t* out) {
    Xoro r = Xoro::from_seed(seed);
    for (int i = 0; i < n; ++i) out[i] = r.next_int(bound);
    return n;
}
double hc_stream_sum(const double* v, int32_t n) { return java_stream_sum(std::vector<double>(v, v + n)); }
int64_t hc_zoom_seed(int64_t seed) {
    SeedHost s;
    build_seed_host(seed, s);
    return s.zoom_seed;
}
}

extern "C" {
// The dedupe tables' error bits on the host build of the same insert / resolve code: n keys
// into a table of cap slots (a power of two), then every key resolved; returns the error
// bits (kErrTableFull when the keys outnumber the slots, kErrKeyMissing for the keys left
// out) and writes each resolved index (0 for a missing key) to idx.
uint32_t hc_table_errors(int32_t n, uint32_t cap, int32_t* idx) {
    std::vector<unsigned long long> keys(cap, kEmpty), uniq(static_cast<size_t>(n));
    std::vector<int32_t> vals(cap, -1), owner(cap, 0x7F7F7F7F);
    int32_t count = 0;
    uint32_t err = 0;
    const HashTab t{keys.data(), vals.data(), uniq.data(), &count, cap - 1, owner.data(), &err};
    auto key = [](int i) { return pack_key(0, i, -i, 0); };
    for (int i = 0; i < n; ++i) ht_insert(t, key(i), i);
    for (int i = 0; i < n; ++i) ht_number(t, key(i), i);
    for (int i = 0; i < n; ++i) idx[i] = ht_resolve(t, key(i));
    return err;
}
}
