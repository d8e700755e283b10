// C binding around the reference's own single-threaded C++ port (cpu/ of
// bonquifo/minecraft-terrain-cuda), compiled from its sources in place by
// oracle/Makefile into oracle/_ref/libref_terrain.so.
//
// TEST INFRASTRUCTURE ONLY. Nothing in the product links or loads this file;
// tests/, bench.py's CPU-baseline leg and __graft_entry__.smoke() use it as the
// checker.
//
// Every entry point forwards to the reference's functions unchanged:
//   model loading        cpu/src/ir.cpp:63 load_ir, cpu/src/terrain_model.cpp:111 load_terrain_model
//   per-seed state       cpu/src/terrain.cpp:112 TerrainSeed::TerrainSeed
//   chunk biomes         cpu/src/terrain.cpp:152 cpu_chunk_biomes
//   fill + surface       cpu/src/terrain.cpp:765 cpu_terrain_from_biomes
//   zoomed block biome   cpu/src/biome.cpp:272 zoomed_biome
//   volume / point eval  cpu/src/volume_eval.cpp:111 VolumeEvaluator::sample, :357 ::point
// The region form mirrors bench/bench_main.cpp:253-304 (biomes of the region plus
// a one-chunk border, computed once per chunk, then fill + surface per chunk).
#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "mccuda/biome.h"
#include "mccuda/ir.h"
#include "mccuda/rng.h"
#include "mccuda/seed_tables.h"
#include "mccuda/terrain.h"
#include "mccuda/terrain_model.h"
#include "mccuda/volume_eval.h"

using namespace mcc;

namespace {

struct Model {
    IR ir;
    TerrainModel tm;
};

struct Seeded {
    Model* m;
    std::unique_ptr<TerrainSeed> ts;
};

thread_local std::string g_err;

template <typename F>
void pool_for(int threads, int count, F&& f) {
    if (threads <= 1) {
        for (int i = 0; i < count; ++i) f(0, i);
        return;
    }
    std::atomic<int> next{0};
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t)
        pool.emplace_back([&, t] {
            int i;
            while ((i = next.fetch_add(1)) < count) f(t, i);
        });
    for (auto& th : pool) th.join();
}

int64_t ckey(int32_t x, int32_t z) { return (static_cast<int64_t>(z) << 32) | static_cast<uint32_t>(x); }

}  // namespace

extern "C" {

const char* ref_last_error() { return g_err.c_str(); }

void* ref_open(const char* ir_path, const char* terrain_path) {
    try {
        auto* m = new Model{load_ir(ir_path), load_terrain_model(terrain_path)};
        return m;
    } catch (const std::exception& e) {
        g_err = e.what();
        return nullptr;
    }
}

void ref_close(void* m) { delete static_cast<Model*>(m); }

int ref_model_info(void* mp, int32_t* out) {
    Model* m = static_cast<Model*>(mp);
    out[0] = m->ir.min_y;
    out[1] = m->ir.height;
    out[2] = m->ir.sea_level;
    out[3] = static_cast<int32_t>(m->ir.nodes.size());
    out[4] = static_cast<int32_t>(m->tm.palette.size());
    out[5] = static_cast<int32_t>(m->tm.biome_names.size());
    out[6] = static_cast<int32_t>(m->tm.params.size());
    out[7] = static_cast<int32_t>(m->tm.conds.size());
    out[8] = static_cast<int32_t>(m->tm.rules.size());
    return 0;
}

int ref_root(void* mp, const char* name) {
    Model* m = static_cast<Model*>(mp);
    auto it = m->ir.roots.find(name);
    return it == m->ir.roots.end() ? -1 : it->second;
}

void* ref_seed(void* mp, int64_t seed) {
    try {
        Model* m = static_cast<Model*>(mp);
        auto* s = new Seeded{m, std::make_unique<TerrainSeed>(m->ir, m->tm, seed)};
        return s;
    } catch (const std::exception& e) {
        g_err = e.what();
        return nullptr;
    }
}

void ref_seed_free(void* s) { delete static_cast<Seeded*>(s); }

// Biomes of one chunk, vanilla quart order (qy*4+qz)*4+qx, 16*height/4 bytes.
int ref_chunk_biomes(void* sp, int32_t cx, int32_t cz, uint8_t* out) {
    try {
        Seeded* s = static_cast<Seeded*>(sp);
        VolumeEvaluator ev(s->m->ir, s->ts->tables);
        cpu_chunk_biomes(*s->ts, ev, cx, cz, out);
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

// Full TERRAIN step for an arbitrary chunk list. Each distinct chunk of the union of
// 3x3 neighbourhoods gets its biomes once; outputs are chunk-major in list order.
// blocks: n*16*16*height u16; biomes/aquifer/density may be null.
int ref_generate(void* sp, const int32_t* cx, const int32_t* cz, int32_t n, int32_t threads, uint16_t* blocks, uint8_t* biomes,
                 uint16_t* aquifer, float* density) {
    try {
        Seeded* s = static_cast<Seeded*>(sp);
        const IR& ir = s->m->ir;
        const int qper = 16 * (ir.height / 4);
        const size_t per = static_cast<size_t>(256) * ir.height;
        std::vector<int64_t> keys;
        std::unordered_map<int64_t, int> slot;
        for (int i = 0; i < n; ++i)
            for (int dz = -1; dz <= 1; ++dz)
                for (int dx = -1; dx <= 1; ++dx) {
                    int64_t k = ckey(cx[i] + dx, cz[i] + dz);
                    if (slot.emplace(k, static_cast<int>(keys.size())).second) keys.push_back(k);
                }
        std::vector<uint8_t> bb(keys.size() * static_cast<size_t>(qper));
        std::vector<std::unique_ptr<VolumeEvaluator>> evals(static_cast<size_t>(std::max(threads, 1)));
        auto ev_for = [&](int t) -> VolumeEvaluator& {
            if (!evals[static_cast<size_t>(t)]) evals[static_cast<size_t>(t)] = std::make_unique<VolumeEvaluator>(ir, s->ts->tables);
            return *evals[static_cast<size_t>(t)];
        };
        pool_for(threads, static_cast<int>(keys.size()), [&](int t, int i) {
            int64_t k = keys[static_cast<size_t>(i)];
            int32_t x = static_cast<int32_t>(static_cast<uint32_t>(k & 0xFFFFFFFFll));
            int32_t z = static_cast<int32_t>(k >> 32);
            cpu_chunk_biomes(*s->ts, ev_for(t), x, z, bb.data() + static_cast<size_t>(i) * qper);
        });
        pool_for(threads, n, [&](int t, int i) {
            const uint8_t* nb[9];
            for (int dz = -1; dz <= 1; ++dz)
                for (int dx = -1; dx <= 1; ++dx)
                    nb[(dz + 1) * 3 + dx + 1] = bb.data() + static_cast<size_t>(slot.at(ckey(cx[i] + dx, cz[i] + dz))) * qper;
            ChunkTerrain c;
            cpu_terrain_from_biomes(*s->ts, ev_for(t), cx[i], cz[i], nb, c);
            std::copy(c.terrain.begin(), c.terrain.end(), blocks + static_cast<size_t>(i) * per);
            if (biomes) std::copy(c.biomes.begin(), c.biomes.end(), biomes + static_cast<size_t>(i) * qper);
            if (aquifer) std::copy(c.aquifer.begin(), c.aquifer.end(), aquifer + static_cast<size_t>(i) * per);
            if (density) std::copy(c.density.begin(), c.density.end(), density + static_cast<size_t>(i) * per);
        });
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

// BiomeManager.getBiome at block positions (cpu/src/biome.cpp:272), with the quart
// biomes of every chunk computed by cpu_chunk_biomes (R-tree candidate reset per chunk).
int ref_biome_lookup(void* sp, const int32_t* xyz, int32_t n, int32_t threads, uint8_t* out) {
    try {
        Seeded* s = static_cast<Seeded*>(sp);
        const IR& ir = s->m->ir;
        const int qh = ir.height / 4, qmin = ir.min_y >> 2, qper = 16 * qh;
        std::mutex mu;
        std::unordered_map<int64_t, std::shared_ptr<std::vector<uint8_t>>> cache;
        std::vector<std::unique_ptr<VolumeEvaluator>> evals(static_cast<size_t>(std::max(threads, 1)));
        pool_for(threads, n, [&](int t, int i) {
            if (!evals[static_cast<size_t>(t)]) evals[static_cast<size_t>(t)] = std::make_unique<VolumeEvaluator>(ir, s->ts->tables);
            auto quart = [&](int qx, int qy, int qz) -> int {
                int ccx = qx >> 2, ccz = qz >> 2;
                int64_t k = ckey(ccx, ccz);
                std::shared_ptr<std::vector<uint8_t>> b;
                {
                    std::lock_guard<std::mutex> g(mu);
                    auto it = cache.find(k);
                    if (it != cache.end()) b = it->second;
                }
                if (!b) {
                    b = std::make_shared<std::vector<uint8_t>>(static_cast<size_t>(qper));
                    cpu_chunk_biomes(*s->ts, *evals[static_cast<size_t>(t)], ccx, ccz, b->data());
                    std::lock_guard<std::mutex> g(mu);
                    cache.emplace(k, b);
                }
                int cqy = std::min(std::max(qy, qmin), qmin + qh - 1) - qmin;
                return (*b)[static_cast<size_t>((cqy * 4 + (qz & 3)) * 4 + (qx & 3))];
            };
            out[i] = static_cast<uint8_t>(zoomed_biome(s->ts->zoom_seed, xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2], quart));
        });
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

// VolumeEvaluator::sample of one node over a volume (buffer order y + (x + z*sx)*sy).
int ref_sample(void* sp, int32_t node, const int32_t* vol /* sx,sy,sz,minx,miny,minz,stx,sty,stz */, float* out) {
    try {
        Seeded* s = static_cast<Seeded*>(sp);
        VolumeEvaluator ev(s->m->ir, s->ts->tables);
        Volume v{vol[0], vol[1], vol[2], vol[3], vol[4], vol[5], vol[6], vol[7], vol[8]};
        ev.sample(node, v, out);
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

// VolumeEvaluator::point of one node at n positions.
int ref_point(void* sp, int32_t node, const int32_t* xyz, int32_t n, float* out) {
    try {
        Seeded* s = static_cast<Seeded*>(sp);
        VolumeEvaluator ev(s->m->ir, s->ts->tables);
        for (int i = 0; i < n; ++i) out[i] = ev.point(node, xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]);
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

// Per-seed scalars the pipeline derives on the host (cpu/src/terrain.cpp:112-149).
int ref_seed_scalars(void* sp, int64_t* out /* zoom_seed, random lo, hi, aquifer lo, hi, ore lo, hi */, int32_t* clay /* 192 */) {
    Seeded* s = static_cast<Seeded*>(sp);
    out[0] = s->ts->zoom_seed;
    out[1] = static_cast<int64_t>(s->ts->random.lo());
    out[2] = static_cast<int64_t>(s->ts->random.hi());
    out[3] = static_cast<int64_t>(s->ts->aquifer_random.lo());
    out[4] = static_cast<int64_t>(s->ts->aquifer_random.hi());
    out[5] = static_cast<int64_t>(s->ts->ore_random.lo());
    out[6] = static_cast<int64_t>(s->ts->ore_random.hi());
    if (clay) std::memcpy(clay, s->ts->clay_bands, sizeof(int32_t) * 192);
    return 0;
}

// Octave table of one noise key: per layer {frequency, amplitude, octave offsets x/y/z}
// and the permutation; lets tests pin the per-seed noise construction layer by layer.
int ref_noise_layers(void* sp, const char* key, int32_t max_layers, double* freq, float* amp, double* offs, uint8_t* perms) {
    Seeded* s = static_cast<Seeded*>(sp);
    auto it = s->ts->tables.noise.find(key);
    if (it == s->ts->tables.noise.end()) return -1;
    const StackRef& r = it->second;
    int n = std::min(r.count, max_layers);
    for (int i = 0; i < n; ++i) {
        const StackLayer& L = s->ts->tables.layers[static_cast<size_t>(r.first_layer + i)];
        const PerlinOctave& o = s->ts->tables.octaves[static_cast<size_t>(L.octave)];
        freq[i] = L.frequency;
        amp[i] = L.amplitude;
        offs[3 * i] = o.ox;
        offs[3 * i + 1] = o.oy;
        offs[3 * i + 2] = o.oz;
        std::memcpy(perms + 256 * i, o.perm, 256);
    }
    return r.count;
}

// Unit primitives for the known-answer checks (cpu/src/rng.cpp, cpu/src/biome.cpp).
void ref_md5(const uint8_t* data, int64_t len, uint8_t* out16) { md5(data, static_cast<size_t>(len), out16); }
int64_t ref_zoom_seed(int64_t world_seed) { return biome_zoom_seed(world_seed); }
int64_t ref_xoroshiro_longs(int64_t seed, int32_t n, int64_t* out) {
    XoroshiroRandom r(seed);
    for (int i = 0; i < n; ++i) out[i] = r.next_long();
    return n;
}
int64_t ref_mth_get_seed(int32_t x, int32_t y, int32_t z) { return mth_get_seed(x, y, z); }
int64_t ref_quantize(float v) { return quantize_coord(v); }
double ref_stream_sum(const double* v, int32_t n) { return java_double_stream_sum(std::vector<double>(v, v + n)); }

}  // extern "C"
