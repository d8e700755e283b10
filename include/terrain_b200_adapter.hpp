// terrain_b200_adapter.hpp: the reference's GPU generator class over the C ABI.
//
// A drop-in for mcc::cuda::FullTerrainGenerator (cuda/include/mccuda_cuda/terrain_gpu.h:31-53
// of bonquifo/minecraft-terrain-cuda): a maintainer replaces cuda/src/terrain.cu with this
// header and links libterrain_b200.so; callers keep their code, including the output type:
// generate() takes the reference's u8 palette-index buffers (terrain_gpu.h:41-43) and calls
// tg_generate_u8. An added overload takes u16 buffers (tg_generate), the CPU port's state type.
// Errors become std::runtime_error, as the reference throws.
#pragma once
#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>
#include "terrain_b200.h"

namespace mcc::cuda {
struct ChunkXZ { int32_t x, z; };                       // generator.h:14-16
struct TerrainTiming {                                  // terrain_gpu.h:15-22
    float h2d_ms = 0, biome_ms = 0, noise_ms = 0, aquifer_ms = 0, fill_ms = 0, surface_ms = 0, d2h_ms = 0;
    float kernel_ms() const { return biome_ms + noise_ms + aquifer_ms + fill_ms + surface_ms; }
};

class FullTerrainGenerator {
public:
    FullTerrainGenerator(const std::string& ir_json, const std::string& terrain_json, int max_batch_chunks = 256, int pipeline_slots = 2) {
        tg_config c{max_batch_chunks, pipeline_slots, 0};
        check(tg_create(ir_json.c_str(), terrain_json.c_str(), &c, &g_));
    }
    ~FullTerrainGenerator() { tg_destroy(g_); }
    void set_seed(int64_t seed) { check(tg_set_seed(g_, seed)); }
    // terrain_gpu.h:43, same signature
    void generate(const ChunkXZ* chunks, int count, uint8_t* terrain_out, uint8_t* biomes_out, uint8_t* aquifer_out,
                  TerrainTiming* timing = nullptr) {
        tg_timing t{};
        check(tg_generate_u8(g_, reinterpret_cast<const tg_chunk_xz*>(chunks), count, terrain_out, biomes_out, aquifer_out, timing ? &t : nullptr));
        if (timing) *timing = TerrainTiming{t.h2d_ms, t.biome_ms, t.noise_ms, t.aquifer_ms, t.fill_ms, t.surface_ms, t.d2h_ms};
    }
    // u16 block states (the CPU port's type)
    void generate(const ChunkXZ* chunks, int count, uint16_t* terrain_out, uint8_t* biomes_out = nullptr,
                  uint16_t* aquifer_out = nullptr, TerrainTiming* timing = nullptr) {
        tg_timing t{};
        check(tg_generate(g_, reinterpret_cast<const tg_chunk_xz*>(chunks), count, terrain_out, biomes_out, aquifer_out, timing ? &t : nullptr));
        if (timing) *timing = TerrainTiming{t.h2d_ms, t.biome_ms, t.noise_ms, t.aquifer_ms, t.fill_ms, t.surface_ms, t.d2h_ms};
    }

private:
    static void check(tg_status s) {
        if (s != TG_OK) throw std::runtime_error(tg_last_error_string());   // the reference throws runtime_error
    }
    tg_generator* g_ = nullptr;
};

inline uint8_t* alloc_pinned(size_t bytes) { return static_cast<uint8_t*>(tg_alloc_pinned(bytes)); }   // terrain_gpu.h:62
inline void free_pinned(void* p) { tg_free_pinned(p); }                                                  // terrain_gpu.h:63
}  // namespace mcc::cuda
