// C binding around the reference's own GPU TERRAIN generator (cuda/src/terrain.cu of
// bonquifo/minecraft-terrain-cuda, class mcc::cuda::FullTerrainGenerator,
// cuda/include/mccuda_cuda/terrain_gpu.h:31-53), compiled unchanged for sm_100a by
// baseline/Makefile, with its evaluators generated by the reference's own code generator
// (cuda/codegen/gen_router.py) from the same model files this repository's library is
// built from.
//
// A timed side arm of bench.py only: it gives the reference GPU pipeline's chunks/s on
// the same B200 and the same model. Nothing in the product links or loads it.
#include <cstdint>
#include <cstring>
#include <exception>
#include <memory>
#include <string>

#include "mccuda/ir.h"
#include "mccuda/terrain_model.h"
#include "mccuda_cuda/terrain_gpu.h"

using namespace mcc;

namespace {
thread_local std::string g_err;

struct Handle {
    IR ir;
    TerrainModel tm;
    std::unique_ptr<cuda::FullTerrainGenerator> gen;
};
}  // namespace

extern "C" {

const char* refgpu_last_error() { return g_err.c_str(); }

// FullTerrainGenerator(ir, tm, max_batch_chunks, pipeline_slots) (terrain_gpu.h:33)
void* refgpu_open(const char* ir_path, const char* terrain_path, int32_t max_batch, int32_t slots) {
    try {
        auto h = std::make_unique<Handle>();
        h->ir = load_ir(ir_path);
        h->tm = load_terrain_model(terrain_path);
        h->gen = std::make_unique<cuda::FullTerrainGenerator>(h->ir, h->tm, max_batch, slots);
        return h.release();
    } catch (const std::exception& e) {
        g_err = e.what();
        return nullptr;
    }
}

void refgpu_close(void* p) { delete static_cast<Handle*>(p); }

int refgpu_set_seed(void* p, int64_t seed) {
    try {
        static_cast<Handle*>(p)->gen->set_seed(seed);
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

// generate(chunks, count, terrain_out u8, biomes_out, aquifer_out, timing) (terrain_gpu.h:41-43);
// stage_ms (may be null) receives h2d, biome, noise, aquifer, fill, surface, d2h, wall ms.
int refgpu_generate(void* p, const int32_t* chunks_xz, int32_t count, uint8_t* terrain, uint8_t* biomes, uint8_t* aquifer, double* stage_ms) {
    try {
        static_assert(sizeof(cuda::ChunkXZ) == 8, "ChunkXZ is two int32");
        cuda::TerrainTiming t;
        static_cast<Handle*>(p)->gen->generate(reinterpret_cast<const cuda::ChunkXZ*>(chunks_xz), count, terrain, biomes, aquifer, stage_ms ? &t : nullptr);
        if (stage_ms) {
            const double v[8] = {t.h2d_ms, t.biome_ms, t.noise_ms, t.aquifer_ms, t.fill_ms, t.surface_ms, t.d2h_ms, t.wall_ms};
            std::memcpy(stage_ms, v, sizeof v);
        }
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

void* refgpu_alloc_pinned(size_t bytes) { return cuda::alloc_pinned(bytes); }
void refgpu_free_pinned(void* p) { cuda::free_pinned(p); }

}  // extern "C"
