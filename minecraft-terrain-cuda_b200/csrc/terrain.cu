// TERRAIN step on sm_100a: kernels, the batch pipeline and the C ABI of
// include/terrain_b200.h.
//
// Pipeline of one batch (all on one stream, all positions deduplicated on the device
// through hash tables, so nothing returns to the host until the outputs):
//   biome stage    neighbourhood union -> climate columns -> climate + first minimal
//                  leaf per quart -> last-result chain per biome chunk
//   noise stage    corner-column union -> hoisted y = 0 values -> 4x8 channel corners
//   aquifer stage  surface-level quart union (volume / point) -> find_top_surface ->
//                  aquifer cell locations and fluid status, skip heights
//   fill           per 8-block cell column: channels, final density, substance, heights
//   surface        per column: eroded badlands + frozen-ocean dry run, then the rule
//                  walk and the frozen-ocean extension
// Reference: cuda/src/terrain.cu:1259-1332 (run_batch) and cpu/src/terrain.cpp:750-810.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <climits>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <memory>
#include <mutex>
#include <sstream>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/terrain_b200.h"
#include "tb_pipeline.cuh"

namespace tb {
namespace {

thread_local std::string g_error;

struct Error : std::runtime_error {
    tg_status code;
    Error(tg_status c, const std::string& m) : std::runtime_error(m), code(c) {}
};

void ck(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        if (e == cudaErrorMemoryAllocation) throw Error(TG_ERR_OUT_OF_MEMORY, std::string(what) + ": " + cudaGetErrorString(e));
        throw Error(TG_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
    }
}

// ---- kernels: grid-stride loops over the bodies --------------------------------------------------
// Minimum resident 256-thread blocks per SM for the register-heavy kernels (caps registers).
#ifndef TB_MINB_SURFACE2
#define TB_MINB_SURFACE2 3
#endif
#ifndef TB_MINB_FILL
#define TB_MINB_FILL 1
#endif
#ifndef TB_MINB_CORNER
#define TB_MINB_CORNER 1
#endif
#ifndef TB_MINB_QUART
#define TB_MINB_QUART 2
#endif

template <void (*F)(const Batch&, int), int MINB = 1>
__global__ void __launch_bounds__(256, MINB) k_items(const __grid_constant__ Batch B, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) F(B, i);
}

// item count = *count * MUL (a device-side dedupe count)
template <void (*F)(const Batch&, int), int MUL, int MINB = 1>
__global__ void __launch_bounds__(256, MINB) k_dyn(const __grid_constant__ Batch B, const int32_t* count) {
    const int n = *count * MUL;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) F(B, i);
}

__global__ void k_fill_i32(int32_t* p, int32_t v, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) p[i] = v;
}

__global__ void k_split_chunks(const tg_chunk_xz* ch, int n, int32_t slot, int32_t* cx, int32_t* cz, int32_t* cs) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        cx[i] = ch[i].x;
        cz[i] = ch[i].z;
        cs[i] = slot;
    }
}

// one lookup position per item: the zoomed biome from its chunk's neighbourhood
__global__ void k_biome_lookup(const __grid_constant__ Batch B, const int32_t* xyz, uint8_t* out, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        out[i] = static_cast<uint8_t>(zoom_biome(B, i, B.seeds[B.cseed[i]].zoom_seed, xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]));
}

int g_sm_count = 148;
thread_local int g_launches = 0;

template <typename K, typename... Args>
void launch(K kernel, cudaStream_t s, int items_hint, Args... args) {
    const int threads = 256;
    long blocks = (static_cast<long>(items_hint) + threads - 1) / threads;
    const long cap = static_cast<long>(g_sm_count) * 8;
    blocks = std::max(1L, std::min(blocks, cap));
    kernel<<<static_cast<unsigned>(blocks), threads, 0, s>>>(args...);
    ++g_launches;
}

uint32_t pow2_at_least(uint64_t v) {
    uint32_t p = 1024;
    while (p < v) p <<= 1;
    return p;
}

// ---- device memory ---------------------------------------------------------------------------------
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() {
        if (p) cudaFree(p);
    }
    void alloc(size_t b) {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = b;
        if (b) ck(cudaMalloc(&p, b), "cudaMalloc");
    }
    template <class T>
    T* as() const {
        return static_cast<T*>(p);
    }
};

struct TableBufs {
    DevBuf keys, vals, uniq, count;
    uint32_t cap = 0;
    void alloc(uint64_t max_keys) {
        cap = pow2_at_least(2 * max_keys);
        keys.alloc(sizeof(unsigned long long) * cap);
        vals.alloc(sizeof(int32_t) * cap);
        uniq.alloc(sizeof(unsigned long long) * max_keys);
        count.alloc(sizeof(int32_t));
    }
    HashTab view() const { return HashTab{keys.as<unsigned long long>(), vals.as<int32_t>(), uniq.as<unsigned long long>(), count.as<int32_t>(), cap - 1}; }
    void reset(cudaStream_t s) {
        ck(cudaMemsetAsync(keys.p, 0xFF, keys.bytes, s), "memset");
        ck(cudaMemsetAsync(count.p, 0, sizeof(int32_t), s), "memset");
    }
};

constexpr int kMaxSlots = 512;

struct SeedSlot {
    int64_t seed = 0;
    bool valid = false;
    uint64_t last_use = 0;
    DevBuf off, perm, layers;
};

}  // namespace

// ---- the generator ----------------------------------------------------------------------------------
struct Generator {
    int device = 0;
    int max_batch = 2048;
    cudaStream_t stream = nullptr;      // the stream all work runs on
    cudaStream_t own_stream = nullptr;
    cudaEvent_t ev[8] = {};
    // model
    DevBuf d_boxes, d_tree, d_children, d_leaf_biome, d_leaf_node, d_leaf_rank, d_flags, d_btemp, d_bfrozen;
    DevModel model{};
    int tree_depth = 0;
    // seeds
    std::unique_ptr<SeedSlot[]> slots;
    DevBuf d_seeds;                 // kMaxSlots DevSeed
    std::vector<DevSeed> h_seeds;
    uint64_t use_clock = 0;
    int current_slot = -1;
    // batch buffers
    DevBuf d_chunks, d_cx, d_cz, d_cs, d_nb9, d_bcol, d_tgt, d_lstar, d_mdist, d_qbiome, d_c25, d_ccol, d_corners, d_g513, d_sfts, d_aq_loc,
        d_aq_status, d_aq_skip, d_blocks, d_h0, d_h1, d_h2, d_biomes, d_aqcopy, d_zoom, d_walk, d_colrec;
    TableBufs tb_b, tb_c, tb_s;
    // pinned staging
    tg_chunk_xz* h_chunks = nullptr;

    Generator(int dev, int batch) : device(dev), max_batch(batch) {
        ck(cudaSetDevice(device), "cudaSetDevice");
        cudaDeviceProp prop{};
        ck(cudaGetDeviceProperties(&prop, device), "cudaGetDeviceProperties");
        g_sm_count = prop.multiProcessorCount;
        ck(cudaStreamCreateWithFlags(&own_stream, cudaStreamNonBlocking), "cudaStreamCreate");
        stream = own_stream;
        for (auto& e : ev) ck(cudaEventCreate(&e), "cudaEventCreate");
        // generated evaluators and the rule tree use deep inlined frames
        ck(cudaDeviceSetLimit(cudaLimitStackSize, 16384), "cudaDeviceSetLimit");
        upload_model();
        slots.reset(new SeedSlot[kMaxSlots]);
        h_seeds.resize(kMaxSlots);
        d_seeds.alloc(sizeof(DevSeed) * kMaxSlots);
        alloc_batch(max_batch);
        ck(cudaMallocHost(reinterpret_cast<void**>(&h_chunks), sizeof(tg_chunk_xz) * max_batch), "cudaMallocHost");
    }
    ~Generator() {
        if (h_chunks) cudaFreeHost(h_chunks);
        for (auto& e : ev)
            if (e) cudaEventDestroy(e);
        if (own_stream) cudaStreamDestroy(own_stream);
    }

    template <class T>
    void upload(DevBuf& b, const std::vector<T>& v) {
        b.alloc(sizeof(T) * std::max<size_t>(v.size(), 1));
        if (!v.empty()) ck(cudaMemcpy(b.p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice), "upload");
    }

    void upload_model() {
        ModelHost m;
        build_model_host(m);
        upload(d_tree, m.nodes);
        if (!m.boxes.empty()) upload(d_boxes, m.boxes);
        upload(d_children, m.children);
        upload(d_leaf_biome, m.leaf_biome);
        upload(d_leaf_node, m.leaf_node);
        upload(d_leaf_rank, m.leaf_rank);
        std::vector<uint8_t> flags(tbm::kBlockFlags, tbm::kBlockFlags + tbm::kPaletteSize);
        upload(d_flags, flags);
        std::vector<float> bt(tbm::kBiomeTemp, tbm::kBiomeTemp + tbm::kNumBiomes);
        upload(d_btemp, bt);
        std::vector<uint8_t> bf(tbm::kBiomeFrozen, tbm::kBiomeFrozen + tbm::kNumBiomes);
        upload(d_bfrozen, bf);
        if (m.depth >= kSearchStack) throw Error(TG_ERR_INTERNAL, "climate tree deeper than the search stack");
        tree_depth = m.depth;
        model.boxes = m.boxes.empty() ? nullptr : d_boxes.as<RBox>();
        model.tree = d_tree.as<RNode>();
        model.children = d_children.as<int32_t>();
        model.leaf_biome = d_leaf_biome.as<int32_t>();
        model.leaf_node = d_leaf_node.as<int32_t>();
        model.leaf_rank = d_leaf_rank.as<int32_t>();
        model.root = m.root;
        model.block_flags = d_flags.as<uint8_t>();
        model.biome_temp = d_btemp.as<float>();
        model.biome_frozen = d_bfrozen.as<uint8_t>();
        model.temp = m.temp;
        for (int i = 0; i < 3; ++i) {
            model.frozen[i] = m.frozen[i];
            model.frozen_amp[i] = m.frozen_amp[i];
        }
        model.info = m.info;
        model.f2 = m.f2;
        model.g2 = m.g2;
    }

    void alloc_batch(int n) {
        const size_t N = static_cast<size_t>(n);
        d_chunks.alloc(sizeof(tg_chunk_xz) * N);
        d_cx.alloc(4 * N);
        d_cz.alloc(4 * N);
        d_cs.alloc(4 * N);
        tb_b.alloc(9 * N);
        tb_c.alloc(25 * N);
        tb_s.alloc(static_cast<uint64_t>(kGrid) * N);
        const size_t nb = 9 * N, cc = 25 * N, sg = static_cast<size_t>(kGrid) * N;
        d_nb9.alloc(4 * 9 * N);
        d_bcol.alloc(sizeof(float) * nb * 16 * tbm::kClimateCols);
        d_tgt.alloc(sizeof(long long) * nb * kQuartsPerChunk * 6);
        d_lstar.alloc(sizeof(int32_t) * nb * kQuartsPerChunk);
        d_mdist.alloc(sizeof(long long) * nb * kQuartsPerChunk);
        d_qbiome.alloc(nb * kQuartsPerChunk);
        d_c25.alloc(4 * 25 * N);
        d_ccol.alloc(sizeof(float) * cc * tbm::kCornerCols);
        d_corners.alloc(sizeof(float) * cc * kRows * tbm::kNumChannels);
        d_g513.alloc(4 * sg);
        d_sfts.alloc(sizeof(float) * sg);
        d_aq_loc.alloc(sizeof(int32_t) * N * kAqCells * 3);
        d_aq_status.alloc(sizeof(int32_t) * N * kAqCells * 2);
        d_aq_skip.alloc(4 * N);
        d_blocks.alloc(sizeof(uint16_t) * N * kBlocksPerChunk);
        d_h0.alloc(4 * 256 * N);
        d_h1.alloc(4 * 256 * N);
        d_h2.alloc(4 * 256 * N);
        d_biomes.alloc(N * kQuartsPerChunk);
        d_zoom.alloc(sizeof(uint32_t) * N * kZoomVerts);
        d_walk.alloc(sizeof(uint32_t) * N * kBlocksPerChunk);
        d_colrec.alloc(sizeof(ColumnRec) * N * 256);
    }

    // Resident per-seed tables: returns the slot, building and uploading on a miss.
    int seed_slot(int64_t seed, const std::vector<int>& pinned_slots = {}) {
        ++use_clock;
        int free_slot = -1, lru = -1;
        for (int i = 0; i < kMaxSlots; ++i) {
            if (slots[i].valid && slots[i].seed == seed) {
                slots[i].last_use = use_clock;
                return i;
            }
            if (!slots[i].valid && free_slot < 0) free_slot = i;
        }
        int s = free_slot;
        if (s < 0) {
            for (int i = 0; i < kMaxSlots; ++i) {
                if (std::find(pinned_slots.begin(), pinned_slots.end(), i) != pinned_slots.end()) continue;
                if (lru < 0 || slots[i].last_use < slots[lru].last_use) lru = i;
            }
            s = lru;
        }
        if (s < 0) throw Error(TG_ERR_INTERNAL, "no free seed slot");
        SeedHost h;
        build_seed_host(seed, h);
        SeedSlot& sl = slots[s];
        upload(sl.off, h.off);
        upload(sl.perm, h.perm);
        upload(sl.layers, h.layers);
        DevSeed d{};
        d.nt = NoiseTables{sl.off.as<OctaveOff>(), sl.perm.as<uint8_t>(), sl.layers.as<Layer>()};
        d.random = h.random;
        d.aquifer = h.aquifer;
        d.ore = h.ore;
        for (size_t k = 0; k < h.gradient.size(); ++k) d.gradient[k] = h.gradient[k];
        d.zoom_seed = h.zoom_seed;
        std::memcpy(d.clay, h.clay, sizeof d.clay);
        h_seeds[s] = d;
        ck(cudaMemcpy(d_seeds.as<DevSeed>() + s, &d, sizeof(DevSeed), cudaMemcpyHostToDevice), "seed upload");
        sl.seed = seed;
        sl.valid = true;
        sl.last_use = use_clock;
        return s;
    }

    Batch batch_view(int n) const {
        Batch B{};
        B.M = model;
        B.seeds = d_seeds.as<DevSeed>();
        B.n = n;
        B.cx = d_cx.as<int32_t>();
        B.cz = d_cz.as<int32_t>();
        B.cseed = d_cs.as<int32_t>();
        B.hb = tb_b.view();
        B.nb_cap = 9 * n;
        B.nb9 = d_nb9.as<int32_t>();
        B.bcol = d_bcol.as<float>();
        B.tgt = d_tgt.as<long long>();
        B.lstar = d_lstar.as<int32_t>();
        B.mdist = d_mdist.as<long long>();
        B.qbiome = d_qbiome.as<uint8_t>();
        B.hc = tb_c.view();
        B.cc_cap = 25 * n;
        B.c25 = d_c25.as<int32_t>();
        B.ccol = d_ccol.as<float>();
        B.corners = d_corners.as<float>();
        B.hs = tb_s.view();
        B.sg_cap = kGrid * n;
        B.g513 = d_g513.as<int32_t>();
        B.sfts = d_sfts.as<float>();
        B.aq_loc = d_aq_loc.as<int32_t>();
        B.aq_status = d_aq_status.as<int32_t>();
        B.aq_skip = d_aq_skip.as<int32_t>();
        B.blocks = d_blocks.as<uint16_t>();
        B.h0 = d_h0.as<int32_t>();
        B.h1 = d_h1.as<int32_t>();
        B.h2 = d_h2.as<int32_t>();
        B.biomes_out = d_biomes.as<uint8_t>();
        B.zoom_tab = d_zoom.as<uint32_t>();
        B.walk = d_walk.as<uint32_t>();
        B.colrec = d_colrec.as<ColumnRec>();
        return B;
    }

    // biome stage only (shared by the TERRAIN step and biome lookups)
    void run_biomes(const Batch& B, int n) {
        cudaStream_t s = stream;
        tb_b.reset(s);
        launch(k_items<body_nb_insert>, s, 9 * n, B, 9 * n);
        launch(k_items<body_nb_resolve>, s, 9 * n, B, 9 * n);
        launch(k_dyn<body_climate_col, 16>, s, n * 16 * 2, B, static_cast<const int32_t*>(tb_b.count.as<int32_t>()));
        launch(k_dyn<body_climate_quart, 16 * kRuns, TB_MINB_QUART>, s, n * 16 * kRuns * 2, B, static_cast<const int32_t*>(tb_b.count.as<int32_t>()));
        launch(k_dyn<body_chain, 1>, s, n * 2, B, static_cast<const int32_t*>(tb_b.count.as<int32_t>()));
    }

    // One device batch of n chunks whose coordinates are already in d_cx/d_cz/d_cs.
    void run_batch(int n, tg_timing* t) {
        cudaStream_t s = stream;
        const Batch B = batch_view(n);
        const int32_t* cnt_c = tb_c.count.as<int32_t>();
        const int32_t* cnt_s = tb_s.count.as<int32_t>();
        ck(cudaEventRecord(ev[0], s), "event");
        run_biomes(B, n);
        ck(cudaEventRecord(ev[1], s), "event");
        // noise stage
        tb_c.reset(s);
        launch(k_items<body_cc_insert>, s, 25 * n, B, 25 * n);
        launch(k_items<body_cc_resolve>, s, 25 * n, B, 25 * n);
        launch(k_dyn<body_corner_col, 1>, s, 16 * n, B, cnt_c);
        launch(k_dyn<body_corner, kRows, TB_MINB_CORNER>, s, 16 * n * kRows, B, cnt_c);
        launch(k_items<body_zoom_table>, s, kZoomVerts * n, B, kZoomVerts * n);
        ck(cudaEventRecord(ev[2], s), "event");
        // aquifer stage
        tb_s.reset(s);
        launch(k_items<body_sg_insert>, s, kGrid * n, B, kGrid * n);
        launch(k_items<body_sg_resolve>, s, kGrid * n, B, kGrid * n);
        launch(k_dyn<body_surface_level, 1>, s, 2 * n * 100, B, cnt_s);
        launch(k_items<body_aquifer_cell>, s, kAqCells * n, B, kAqCells * n);
        launch(k_items<body_aquifer_skip>, s, n, B, n);
        ck(cudaEventRecord(ev[3], s), "event");
        // fill
        launch(k_fill_i32, s, 256 * n, B.h0, static_cast<int32_t>(tbm::kMinY), 256 * n);
        launch(k_items<body_fill, TB_MINB_FILL>, s, 256 * kCellsY * n, B, 256 * kCellsY * n);
        ck(cudaEventRecord(ev[4], s), "event");
        // surface
        launch(k_items<body_surface1>, s, 256 * n, B, 256 * n);
        launch(k_items<body_surface_walk>, s, 256 * n, B, 256 * n);
        launch(k_items<body_surface_rules, TB_MINB_SURFACE2>, s, kBlocksPerChunk * n, B, kBlocksPerChunk * n);
        launch(k_items<body_surface_frozen>, s, 256 * n, B, 256 * n);
        launch(k_items<body_gather>, s, kQuartsPerChunk * n, B, kQuartsPerChunk * n);
        ck(cudaEventRecord(ev[5], s), "event");
        ck(cudaGetLastError(), "kernel launch");
        if (t) {
            ck(cudaEventSynchronize(ev[5]), "sync");
            float ms[5];
            for (int i = 0; i < 5; ++i) ck(cudaEventElapsedTime(&ms[i], ev[i], ev[i + 1]), "elapsed");
            t->biome_ms += ms[0];
            t->noise_ms += ms[1];
            t->aquifer_ms += ms[2];
            t->fill_ms += ms[3];
            t->surface_ms += ms[4];
            t->kernel_ms += ms[0] + ms[1] + ms[2] + ms[3] + ms[4];
            t->batches += 1;
            t->launches = g_launches;
        }
    }

    void check_chunks(const tg_chunk_xz* c, int n) {
        const int32_t lim = 1 << 23;
        for (int i = 0; i < n; ++i)
            if (c[i].x <= -lim || c[i].x >= lim || c[i].z <= -lim || c[i].z >= lim) throw Error(TG_ERR_RANGE, "chunk coordinate outside |c| < 2^23");
    }

    void generate(const tg_chunk_xz* chunks, int count, uint16_t* blocks, uint8_t* biomes, uint16_t* aquifer, tg_timing* t) {
        if (current_slot < 0) throw Error(TG_ERR_NO_SEED, "tg_set_seed has not been called");
        check_chunks(chunks, count);
        for (int off = 0; off < count; off += max_batch) {
            const int n = std::min(max_batch, count - off);
            std::memcpy(h_chunks, chunks + off, sizeof(tg_chunk_xz) * n);
            ck(cudaMemcpyAsync(d_chunks.p, h_chunks, sizeof(tg_chunk_xz) * n, cudaMemcpyHostToDevice, stream), "h2d");
            launch(k_split_chunks, stream, n, d_chunks.as<tg_chunk_xz>(), n, static_cast<int32_t>(current_slot), d_cx.as<int32_t>(), d_cz.as<int32_t>(),
                   d_cs.as<int32_t>());
            run_batch(n, t);
            if (aquifer) throw Error(TG_ERR_INVALID_ARGUMENT, "aquifer_out is not supported yet");
            ck(cudaMemcpyAsync(blocks + static_cast<size_t>(off) * kBlocksPerChunk, d_blocks.p, sizeof(uint16_t) * n * kBlocksPerChunk,
                               cudaMemcpyDeviceToHost, stream),
               "d2h");
            if (biomes)
                ck(cudaMemcpyAsync(biomes + static_cast<size_t>(off) * kQuartsPerChunk, d_biomes.p, static_cast<size_t>(n) * kQuartsPerChunk,
                                   cudaMemcpyDeviceToHost, stream),
                   "d2h");
            ck(cudaStreamSynchronize(stream), "sync");
        }
    }

    void generate_device(const tg_chunk_xz* chunks_dev, int count, uint16_t* blocks_dev, uint8_t* biomes_dev, tg_timing* t) {
        if (current_slot < 0) throw Error(TG_ERR_NO_SEED, "tg_set_seed has not been called");
        if (count > max_batch) throw Error(TG_ERR_INVALID_ARGUMENT, "count exceeds max_batch_chunks");
        launch(k_split_chunks, stream, count, chunks_dev, count, static_cast<int32_t>(current_slot), d_cx.as<int32_t>(), d_cz.as<int32_t>(),
               d_cs.as<int32_t>());
        run_batch(count, t);
        ck(cudaMemcpyAsync(blocks_dev, d_blocks.p, sizeof(uint16_t) * count * kBlocksPerChunk, cudaMemcpyDeviceToDevice, stream), "d2d");
        if (biomes_dev) ck(cudaMemcpyAsync(biomes_dev, d_biomes.p, static_cast<size_t>(count) * kQuartsPerChunk, cudaMemcpyDeviceToDevice, stream), "d2d");
        ck(cudaStreamSynchronize(stream), "sync");
    }

    void biome_lookup(const int64_t* seeds, const int32_t* xyz, int n, uint8_t* out) {
        std::vector<int32_t> cx, cz, cs, pos;
        for (int off = 0; off < n; off += max_batch) {
            const int m = std::min(max_batch, n - off);
            cx.resize(m);
            cz.resize(m);
            cs.resize(m);
            std::vector<int> used;
            for (int i = 0; i < m; ++i) {
                const int32_t* p = xyz + 3 * (off + i);
                cx[i] = p[0] >> 4;
                cz[i] = p[2] >> 4;
                if (cx[i] <= -(1 << 23) || cx[i] >= (1 << 23) || cz[i] <= -(1 << 23) || cz[i] >= (1 << 23)) throw Error(TG_ERR_RANGE, "position out of range");
                cs[i] = seed_slot(seeds[off + i], used);
                used.push_back(cs[i]);
            }
            DevBuf d_xyz, d_out;
            d_xyz.alloc(sizeof(int32_t) * 3 * m);
            d_out.alloc(m);
            ck(cudaMemcpyAsync(d_xyz.p, xyz + 3 * off, sizeof(int32_t) * 3 * m, cudaMemcpyHostToDevice, stream), "h2d");
            ck(cudaMemcpyAsync(d_cx.p, cx.data(), 4 * m, cudaMemcpyHostToDevice, stream), "h2d");
            ck(cudaMemcpyAsync(d_cz.p, cz.data(), 4 * m, cudaMemcpyHostToDevice, stream), "h2d");
            ck(cudaMemcpyAsync(d_cs.p, cs.data(), 4 * m, cudaMemcpyHostToDevice, stream), "h2d");
            const Batch B = batch_view(m);
            run_biomes(B, m);
            launch(k_biome_lookup, stream, m, B, d_xyz.as<int32_t>(), d_out.as<uint8_t>(), m);
            ck(cudaMemcpyAsync(out + off, d_out.p, m, cudaMemcpyDeviceToHost, stream), "d2h");
            ck(cudaStreamSynchronize(stream), "sync");
        }
    }

    void generate_batch(const tg_request* req, int n, tg_timing* t) {
        // flatten requests into device batches; each request's seed gets a resident slot
        std::vector<int32_t> cx, cz, cs;
        struct Piece {
            int req, first, count;
        };
        std::vector<Piece> pieces;
        std::vector<int> used;
        auto flush = [&]() {
            const int m = static_cast<int>(cx.size());
            if (!m) return;
            ck(cudaMemcpyAsync(d_cx.p, cx.data(), 4 * m, cudaMemcpyHostToDevice, stream), "h2d");
            ck(cudaMemcpyAsync(d_cz.p, cz.data(), 4 * m, cudaMemcpyHostToDevice, stream), "h2d");
            ck(cudaMemcpyAsync(d_cs.p, cs.data(), 4 * m, cudaMemcpyHostToDevice, stream), "h2d");
            run_batch(m, t);
            int at = 0;
            for (const Piece& p : pieces) {
                ck(cudaMemcpyAsync(req[p.req].blocks_out + static_cast<size_t>(p.first) * kBlocksPerChunk,
                                   d_blocks.as<uint16_t>() + static_cast<size_t>(at) * kBlocksPerChunk, sizeof(uint16_t) * p.count * kBlocksPerChunk,
                                   cudaMemcpyDeviceToHost, stream),
                   "d2h");
                if (req[p.req].biomes_out)
                    ck(cudaMemcpyAsync(req[p.req].biomes_out + static_cast<size_t>(p.first) * kQuartsPerChunk,
                                       d_biomes.as<uint8_t>() + static_cast<size_t>(at) * kQuartsPerChunk, static_cast<size_t>(p.count) * kQuartsPerChunk,
                                       cudaMemcpyDeviceToHost, stream),
                       "d2h");
                at += p.count;
            }
            ck(cudaStreamSynchronize(stream), "sync");
            cx.clear();
            cz.clear();
            cs.clear();
            pieces.clear();
            used.clear();
        };
        for (int r = 0; r < n; ++r) {
            if (!req[r].chunks || !req[r].blocks_out || req[r].count < 0) throw Error(TG_ERR_INVALID_ARGUMENT, "bad request");
            check_chunks(req[r].chunks, req[r].count);
            int done = 0;
            while (done < req[r].count) {
                if (static_cast<int>(cx.size()) == max_batch || static_cast<int>(used.size()) >= kMaxSlots) flush();
                const int slot = seed_slot(req[r].seed, used);
                if (std::find(used.begin(), used.end(), slot) == used.end()) used.push_back(slot);
                const int take = std::min(req[r].count - done, max_batch - static_cast<int>(cx.size()));
                pieces.push_back({r, done, take});
                for (int i = 0; i < take; ++i) {
                    cx.push_back(req[r].chunks[done + i].x);
                    cz.push_back(req[r].chunks[done + i].z);
                    cs.push_back(slot);
                }
                done += take;
            }
        }
        flush();
    }
};

std::string read_file(const char* path) {
    std::ifstream f(path, std::ios::binary);
    if (!f) throw Error(TG_ERR_INVALID_ARGUMENT, std::string("cannot open ") + path);
    std::stringstream ss;
    ss << f.rdbuf();
    return ss.str();
}

template <class F>
tg_status guarded(F&& f) {
    try {
        f();
        g_error.clear();
        return TG_OK;
    } catch (const Error& e) {
        g_error = e.what();
        return e.code;
    } catch (const std::bad_alloc&) {
        g_error = "host allocation failed";
        return TG_ERR_OUT_OF_MEMORY;
    } catch (const std::exception& e) {
        g_error = e.what();
        return TG_ERR_INTERNAL;
    }
}

}  // namespace tb

struct tg_generator {
    std::unique_ptr<tb::Generator> g;
};

extern "C" {

tg_status tg_create(const char* ir_json_path, const char* terrain_json_path, const tg_config* config, tg_generator** out) {
    return tb::guarded([&] {
        if (!out) throw tb::Error(TG_ERR_INVALID_ARGUMENT, "out is null");
        *out = nullptr;
        if (ir_json_path && tb::sha256_hex(tb::read_file(ir_json_path)) != tbm::kModelIrSha256)
            throw tb::Error(TG_ERR_MODEL_MISMATCH, "IR file differs from the compiled model");
        if (terrain_json_path && tb::sha256_hex(tb::read_file(terrain_json_path)) != tbm::kModelTerrainSha256)
            throw tb::Error(TG_ERR_MODEL_MISMATCH, "terrain model file differs from the compiled model");
        int batch = config && config->max_batch_chunks > 0 ? config->max_batch_chunks : 2048;
        if (batch > (1 << 16)) throw tb::Error(TG_ERR_INVALID_ARGUMENT, "max_batch_chunks too large");
        const int dev = config ? config->device : 0;
        auto* h = new tg_generator;
        try {
            h->g = std::make_unique<tb::Generator>(dev, batch);
        } catch (...) {
            delete h;
            throw;
        }
        *out = h;
    });
}

tg_status tg_destroy(tg_generator* gen) {
    return tb::guarded([&] { delete gen; });
}

tg_status tg_set_stream(tg_generator* gen, void* cuda_stream) {
    return tb::guarded([&] {
        if (!gen) throw tb::Error(TG_ERR_INVALID_ARGUMENT, "gen is null");
        gen->g->stream = cuda_stream ? static_cast<cudaStream_t>(cuda_stream) : gen->g->own_stream;
    });
}

tg_status tg_set_seed(tg_generator* gen, int64_t seed) {
    return tb::guarded([&] {
        if (!gen) throw tb::Error(TG_ERR_INVALID_ARGUMENT, "gen is null");
        tb::ck(cudaSetDevice(gen->g->device), "cudaSetDevice");
        gen->g->current_slot = gen->g->seed_slot(seed);
    });
}

tg_status tg_generate(tg_generator* gen, const tg_chunk_xz* chunks, int32_t count, uint16_t* blocks_out, uint8_t* biomes_out, uint16_t* aquifer_out,
                      tg_timing* timing) {
    return tb::guarded([&] {
        if (!gen || (count > 0 && (!chunks || !blocks_out)) || count < 0) throw tb::Error(TG_ERR_INVALID_ARGUMENT, "bad argument");
        tb::ck(cudaSetDevice(gen->g->device), "cudaSetDevice");
        const auto t0 = std::chrono::steady_clock::now();
        if (timing) std::memset(timing, 0, sizeof *timing);
        tb::g_launches = 0;
        gen->g->generate(chunks, count, blocks_out, biomes_out, aquifer_out, timing);
        if (timing) timing->launches = tb::g_launches;
        if (timing) timing->wall_ms = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
    });
}

tg_status tg_generate_device(tg_generator* gen, const tg_chunk_xz* chunks_dev, int32_t count, uint16_t* blocks_dev, uint8_t* biomes_dev, tg_timing* timing) {
    return tb::guarded([&] {
        if (!gen || count <= 0 || !chunks_dev || !blocks_dev) throw tb::Error(TG_ERR_INVALID_ARGUMENT, "bad argument");
        tb::ck(cudaSetDevice(gen->g->device), "cudaSetDevice");
        if (timing) std::memset(timing, 0, sizeof *timing);
        tb::g_launches = 0;
        gen->g->generate_device(chunks_dev, count, blocks_dev, biomes_dev, timing);
        if (timing) timing->launches = tb::g_launches;
    });
}

tg_status tg_generate_batch(tg_generator* gen, const tg_request* requests, int32_t n, tg_timing* timing) {
    return tb::guarded([&] {
        if (!gen || n < 0 || (n > 0 && !requests)) throw tb::Error(TG_ERR_INVALID_ARGUMENT, "bad argument");
        tb::ck(cudaSetDevice(gen->g->device), "cudaSetDevice");
        const auto t0 = std::chrono::steady_clock::now();
        if (timing) std::memset(timing, 0, sizeof *timing);
        tb::g_launches = 0;
        gen->g->generate_batch(requests, n, timing);
        if (timing) timing->launches = tb::g_launches;
        if (timing) timing->wall_ms = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
    });
}

tg_status tg_biome_lookup(tg_generator* gen, const int64_t* seeds, const int32_t* xyz, int32_t n, uint8_t* out) {
    return tb::guarded([&] {
        if (!gen || n < 0 || (n > 0 && (!seeds || !xyz || !out))) throw tb::Error(TG_ERR_INVALID_ARGUMENT, "bad argument");
        tb::ck(cudaSetDevice(gen->g->device), "cudaSetDevice");
        gen->g->biome_lookup(seeds, xyz, n, out);
    });
}

void* tg_alloc_pinned(size_t bytes) {
    void* p = nullptr;
    if (cudaMallocHost(&p, bytes) != cudaSuccess) return nullptr;
    return p;
}

void tg_free_pinned(void* p) {
    if (p) cudaFreeHost(p);
}

tg_status tg_model_info(int32_t* min_y, int32_t* height, int32_t* sea_level, int32_t* palette_size, int32_t* biome_count) {
    if (min_y) *min_y = tbm::kMinY;
    if (height) *height = tbm::kHeight;
    if (sea_level) *sea_level = tbm::kSeaLevel;
    if (palette_size) *palette_size = tbm::kPaletteSize;
    if (biome_count) *biome_count = tbm::kNumBiomes;
    return TG_OK;
}

const char* tg_last_error_string(void) { return tb::g_error.c_str(); }

}  // extern "C"
