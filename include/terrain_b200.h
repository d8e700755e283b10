/* terrain_b200: the overworld TERRAIN step on one B200, behind a C ABI.
 *
 * Drop-in for the reference's GPU generator class mcc::cuda::FullTerrainGenerator
 * (cuda/include/mccuda_cuda/terrain_gpu.h:31-53 of bonquifo/minecraft-terrain-cuda):
 * the same chunk-list-in, buffers-out pipeline, with plain pointers, status codes
 * instead of C++ exceptions, and u16 block-state ids instead of the reference's u8.
 *
 * Layouts (identical to the reference's CPU port, cpu/include/mccuda/terrain.h:55-60):
 *   blocks   per chunk 16 * 16 * height u16, index ((y - min_y) * 16 + z) * 16 + x
 *   biomes   per chunk 16 * height / 4 u8, index (qy * 4 + qz) * 4 + qx
 *   chunks   back to back in list order
 *
 * Threading: one generator per host thread; calls on one generator are serialised by
 * the caller. Every call is synchronous on return unless its name says otherwise.
 */
#ifndef TERRAIN_B200_H
#define TERRAIN_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum tg_status {
    TG_OK = 0,
    TG_ERR_INVALID_ARGUMENT = 1,  /* null pointer, bad count, bad config */
    TG_ERR_MODEL_MISMATCH = 2,    /* model files differ from the model compiled in */
    TG_ERR_CUDA = 3,              /* a CUDA runtime call failed (message in tg_last_error_string) */
    TG_ERR_OUT_OF_MEMORY = 4,     /* device or pinned allocation failed */
    TG_ERR_RANGE = 5,             /* chunk coordinate outside |c| < 2^23 */
    TG_ERR_NO_SEED = 6,           /* tg_generate before tg_set_seed */
    TG_ERR_DEVICE_TIMEOUT = 7,    /* a bounded device-side wait expired */
    TG_ERR_INTERNAL = 8,
    TG_ERR_IO = 9,                /* a region file could not be written */
    TG_ERR_CANCELLED = 10         /* tg_server_wait: the request was cancelled (tg_server_cancel) */
} tg_status;

/* reference: mcc::cuda::ChunkXZ (cuda/include/mccuda_cuda/generator.h:14-16) */
typedef struct tg_chunk_xz {
    int32_t x, z;
} tg_chunk_xz;

/* reference: FullTerrainGenerator(ir, tm, max_batch_chunks, pipeline_slots)
 * (cuda/include/mccuda_cuda/terrain_gpu.h:33); device selects the CUDA device. */
typedef struct tg_config {
    int32_t max_batch_chunks; /* chunks per device batch; 0 = 2048 */
    int32_t pipeline_slots;   /* batches in flight (1 or 2); 0 = 2 */
    int32_t device;           /* CUDA device ordinal */
} tg_config;

/* reference: TerrainTiming (cuda/include/mccuda_cuda/terrain_gpu.h:15-22); milliseconds
 * of device time per stage summed over batches, plus host wall time of the call. */
typedef struct tg_timing {
    float h2d_ms, biome_ms, noise_ms, aquifer_ms, fill_ms, surface_ms, d2h_ms, kernel_ms, wall_ms;
    int32_t batches;
    int32_t launches;     /* kernels launched by the call */
    float walk_rules_ms;  /* the column walk with the rule tree and its deferred pass (part of surface_ms) */
    float corner_ms;      /* the channel-corner kernel (part of noise_ms) */
} tg_timing;

/* Creates a generator for the model compiled into the library. ir_json_path and
 * terrain_json_path, when not NULL, must be the files it was generated from
 * (checked by SHA-256; TG_ERR_MODEL_MISMATCH otherwise).
 * reference: FullTerrainGenerator::FullTerrainGenerator (cuda/src/terrain.cu:1375, :1105-1122) */
tg_status tg_create(const char* ir_json_path, const char* terrain_json_path, const tg_config* config, struct tg_generator** out);

/* reference: ~FullTerrainGenerator */
tg_status tg_destroy(struct tg_generator* gen);

/* Runs the generator's work on the caller's CUDA stream (a cudaStream_t; NULL restores
 * the generator's own stream): each batch starts after the work already queued there, and
 * the stages it runs on the generator's internal side streams fork from and join back into
 * that stream. Calls still return only when their work is done.
 * No counterpart in the reference (its streams are internal). */
tg_status tg_set_stream(struct tg_generator* gen, void* cuda_stream);

/* Builds the per-seed noise tables, random factories and zoom seed on the host and
 * uploads them. reference: FullTerrainGenerator::set_seed (cuda/src/terrain.cu:1387, :1176-1255) */
tg_status tg_set_seed(struct tg_generator* gen, int64_t seed);

/* The TERRAIN step for count chunks. blocks_out: count * 16 * 16 * height u16 (required);
 * biomes_out: count * 16 * height / 4 u8 (may be NULL); aquifer_out: the blocks after the
 * aquifer fill and before the material rules (may be NULL); timing may be NULL.
 * Host buffers; pinned ones (tg_alloc_pinned) copy fastest. The chunks go in device
 * batches, each batch's copy to the host running while the next one computes; the batch
 * sizes follow the launch table's host_u16 line (tg_set_launch_table).
 * reference: FullTerrainGenerator::generate (cuda/src/terrain.cu:1392-1417) */
tg_status tg_generate(struct tg_generator* gen, const tg_chunk_xz* chunks, int32_t count, uint16_t* blocks_out, uint8_t* biomes_out,
                      uint16_t* aquifer_out, tg_timing* timing);

/* The same step in the reference generator's own output form: terrain_out and aquifer_out
 * (may be NULL) hold one u8 palette index per block, biomes_out u8 per quart (may be NULL),
 * in the same layouts as tg_generate. Each value is the u16 state of tg_generate narrowed
 * (every state id is below the palette size); half the bytes cross the host link. The
 * narrowing runs on the GPU after each batch; the batch sizes follow the launch table's
 * host_u8 line.
 * reference: FullTerrainGenerator::generate (cuda/include/mccuda_cuda/terrain_gpu.h:41-43,
 * cuda/src/terrain.cu:1392-1417), same argument types and order */
tg_status tg_generate_u8(struct tg_generator* gen, const tg_chunk_xz* chunks, int32_t count, uint8_t* terrain_out, uint8_t* biomes_out,
                         uint8_t* aquifer_out, tg_timing* timing);

/* Region outputs for consumers. Sets the generator's seed to seed, generates the
 * region x region chunks from chunk (x0, z0) in u8 form, row-major by chunk
 * ((cz - z0) * region + (cx - x0)), and writes
 *   - when dump_dir is not NULL (created if missing): dump_dir/terrain.u8 (u8 palette index
 *     per block, chunks back to back), dump_dir/biomes.u8 (u8 per quart) and
 *     dump_dir/meta.json {seed, x0, z0, region, height, min_y, chunk_bytes, biome_bytes};
 *   - when topdown_path is not NULL: the top-down map, "MCTD", int32 {1, region, x0, z0,
 *     min_y}, then 8 bytes per block column row-major over the region: u8 top state (highest
 *     non-air block), u8 floor state (first non-fluid block at or below it), u8 fluid depth
 *     (at most 255), u8 0, int16 top y, int16 floor y.
 * region in [1, 2048]; the files are written a slab of chunk rows at a time (host memory of at
 * most 4,096 chunks' outputs); TG_ERR_IO when a file cannot be written.
 * reference: write_dump (bench/bench_main.cpp:170-187) and write_topdown (:134-165); the dump
 * is what the client maps (client/src/main/java/mccuda/client/GpuDump.java:88-104) */
tg_status tg_write_region(struct tg_generator* gen, int64_t seed, int32_t x0, int32_t z0, int32_t region, const char* dump_dir,
                          const char* topdown_path);

/* Device-resident form: chunks, blocks_out and biomes_out (may be NULL) are device
 * pointers; count <= max_batch_chunks; runs on the generator's stream and returns
 * when the work is done. The kernels write blocks_out and biomes_out in place when both
 * are 16-byte aligned (else through the generator's buffers and a device copy). No
 * counterpart in the reference (its buffers are host-side); used to measure the kernels
 * with inputs already in HBM. */
tg_status tg_generate_device(struct tg_generator* gen, const tg_chunk_xz* chunks_dev, int32_t count, uint16_t* blocks_dev, uint8_t* biomes_dev,
                             tg_timing* timing);

/* Final density of every block of count chunks: the f32 value the fill tests (with the
 * aquifer) before the material rules, in the block layout, count * 16 * 16 * height floats
 * of host memory. The whole TERRAIN step runs; the fill also writes each density it
 * evaluates. For parity checks at the density level.
 * reference: TerrainGenerator::generate's density_out (cuda/include/mccuda_cuda/generator.h:38-39);
 * the CPU port's ChunkTerrain::density (cpu/include/mccuda/terrain.h:59, filled at
 * cpu/src/terrain.cpp:787-795) */
tg_status tg_generate_density(struct tg_generator* gen, const tg_chunk_xz* chunks, int32_t count, float* density_out);

/* Multi-seed batch: each request is its own seed and chunk list; all requests run in
 * shared device batches with positions deduplicated per seed. Output buffers are host
 * memory per request. No counterpart in the reference (single seed per generator). */
typedef struct tg_request {
    int64_t seed;
    const tg_chunk_xz* chunks;
    int32_t count;
    uint16_t* blocks_out;
    uint8_t* biomes_out; /* may be NULL */
} tg_request;
tg_status tg_generate_batch(struct tg_generator* gen, const tg_request* requests, int32_t n, tg_timing* timing);

/* Device-resident multi-seed batch: every request's chunk list and outputs are device
 * memory (outputs 16-byte aligned). The requests become one device work queue of
 * (chunk, seed) items; each iteration takes the next batch of at most max_batch_chunks
 * items, runs the TERRAIN step on it and copies each chunk's outputs to its request. By
 * default the iterations run as a loop on the device: one CUDA-graph launch (a WHILE
 * conditional node) drains the whole queue with no host round trip between batches;
 * TG_BATCH_HOST_LOOP launches one graph per batch from the host instead (same kernels).
 * Requests with more than 256 distinct seeds go in groups, one launch per group. Returns
 * when the work is done. No counterpart in the reference (single seed per generator). */
typedef struct tg_request_device {
    int64_t seed;
    const tg_chunk_xz* chunks;   /* device memory, count entries */
    int32_t count;
    uint16_t* blocks_out;        /* device memory, count * 16 * 16 * height u16 */
    uint8_t* biomes_out;         /* device memory, count * 16 * height / 4 u8, or NULL */
} tg_request_device;
#define TG_BATCH_HOST_LOOP 1
tg_status tg_generate_batch_device(struct tg_generator* gen, const tg_request_device* requests, int32_t n, int32_t flags, tg_timing* timing);

/* BiomeManager.getBiome at block positions (xyz triples) for one seed per position,
 * with the chunk's R-tree chain exactly as the TERRAIN step computes it.
 * reference semantics: zoomed_biome over cpu_chunk_biomes (cpu/src/biome.cpp:272-289,
 * cpu/src/terrain.cpp:152-176). */
tg_status tg_biome_lookup(struct tg_generator* gen, const int64_t* seeds, const int32_t* xyz, int32_t n, uint8_t* out);

/* Biome lookups for the seed of tg_set_seed that allocate nothing: for callers that cannot
 * allocate device memory after start-up (a server that reserves its whole HBM budget when
 * it creates the generator, so that a lookup cannot fail later on an allocation; a caller
 * that must not cause the device-wide wait of cudaFree while other libraries' kernels run
 * on other streams). Positions and results pass through one fixed device scratch array of
 * 53,504 bytes, so n <= 4,096 and n <= max_batch_chunks; larger n returns
 * TG_ERR_INVALID_ARGUMENT. xyz (3 x n int32) and out (n u8) are host memory. The call
 * reuses the generator's batch buffers: it first waits for that generator's earlier work,
 * so it runs on the generator's own thread, not beside its batches, and a generator owned
 * by a server refuses it. The first call on a device resolves the scratch address; make
 * it before any stream capture begins. Every call on a device shares the array: calls that
 * overlap on the GPU race (each call waits for its own copies before it returns). Results
 * equal tg_biome_lookup with every seed = the current seed. No counterpart in the
 * reference. */
tg_status tg_biome_lookup_noalloc(struct tg_generator* gen, const int32_t* xyz, int32_t n, uint8_t* out);

/* ---- serving: continuous batching ---------------------------------------------------
 * A server owns its generator (which then rejects direct calls until the server is
 * destroyed). A worker thread admits submitted requests while the chunks in flight, priced
 * at the HBM a chunk of batch capacity takes (tg_server_stats.device_bytes_per_chunk), stay
 * within the budget; it cuts device batches across all admitted requests (seeds, request
 * sizes and output forms mixed), and copies each batch out on a second stream while the
 * next one computes; per-seed tables stay resident on the device. Results are
 * byte-identical to tg_generate / tg_generate_u8 for the same seed and chunks, alone or in
 * any mix. No counterpart in the reference (it has no serving form). */
typedef struct tg_server_config {
    int32_t batch_chunks;       /* chunks per device batch (<= max_batch_chunks); 0 = max_batch_chunks */
    int64_t hbm_budget_bytes;   /* device memory of the chunks admitted and not yet issued; 0 = 8 batches */
    int32_t reserved;
} tg_server_config;

typedef struct tg_server_stats {
    int64_t completed_requests, completed_chunks;
    double p50_ms, p99_ms, mean_ms, max_ms;  /* submit -> last byte on the host, completed requests */
    double chunks_per_s;                     /* completed chunks / (first submit -> last completion) */
    int32_t batches, queued_requests, active_requests;
    int64_t cancelled_requests;
    double device_bytes_per_chunk;           /* HBM per chunk of batch capacity (admission price) */
    int64_t max_active_chunks;               /* the budget in chunks */
} tg_server_stats;

tg_status tg_server_create(struct tg_generator* gen, const tg_server_config* config, struct tg_server** out);
/* Queues a request; blocks_out (count * 16 * 16 * height u16) and biomes_out (may be NULL)
 * are host buffers that must stay valid until the request completes. Non-blocking. */
tg_status tg_server_submit(struct tg_server* srv, int64_t seed, const tg_chunk_xz* chunks, int32_t count, uint16_t* blocks_out, uint8_t* biomes_out,
                           uint64_t* ticket);
/* The same in the reference generator's u8 form: terrain_out holds count * 16 * 16 * height
 * u8 palette indices (the u16 states narrowed on the GPU), half the bytes to copy. */
tg_status tg_server_submit_u8(struct tg_server* srv, int64_t seed, const tg_chunk_xz* chunks, int32_t count, uint8_t* terrain_out, uint8_t* biomes_out,
                              uint64_t* ticket);
/* *done = 1 once the request's outputs are on the host (the ticket is then released);
 * timeout_ms: 0 polls, < 0 waits without limit. A cancelled request returns
 * TG_ERR_CANCELLED once its chunks in flight have landed (the ticket is then released). */
tg_status tg_server_wait(struct tg_server* srv, uint64_t ticket, int32_t timeout_ms, int32_t* done);
/* Cancels a request: a queued one is dropped at once, an admitted one issues no more chunks
 * (its outputs hold only the chunks already in flight); *was_pending (may be NULL) = 0 when
 * it had already completed, whose result stands. Its buffers must stay valid until
 * tg_server_wait reports it. */
tg_status tg_server_cancel(struct tg_server* srv, uint64_t ticket, int32_t* was_pending);
tg_status tg_server_get_stats(struct tg_server* srv, tg_server_stats* stats);
/* Latencies (ms, submit -> last byte on the host) of the requests completed since the last
 * reset, in completion order: up to cap values into ms, their total count into *n. */
tg_status tg_server_latencies(struct tg_server* srv, double* ms, int32_t cap, int32_t* n);
tg_status tg_server_reset_stats(struct tg_server* srv);
/* Finishes the work in flight, then stops the worker. */
tg_status tg_server_destroy(struct tg_server* srv);

/* ---- live flythrough renderer -----------------------------------------------------------
 * A viewer keeps a toroidal window of window_chunks x window_chunks generated chunks on the
 * device (u8 palette index per block) and ray traces frames of it. tg_viewer_update
 * generates the chunks within a radius of the camera's chunk that the window does not hold,
 * nearest first, with the generator (its seed of tg_set_seed) straight into the window: the
 * blocks never leave the device. tg_viewer_render traces one width x height frame: 2 x 2
 * rays per pixel through the voxels (whole 4 x 4-column cells skipped while a ray stays
 * above their blocks, water seen through), a shadow ray toward the sun, ambient occlusion,
 * water tint and reflection, distance haze. The generator serves the viewer on the same
 * host thread (not while a server owns it).
 * reference: the flythrough renderer viz/fly.cu (k_render :249-310, k_scatter :312-320,
 * k_cells :322-334, the frame loop :486-560), which copies each chunk to the host and back. */
typedef struct tg_viewer_config {
    int32_t window_chunks;   /* window side in chunks, a multiple of 4 in 4..256; 0 = 64 */
    int32_t width, height;   /* frame size; 0 = 1280 x 720 */
    int32_t reserved;
} tg_viewer_config;

typedef struct tg_camera {
    float x, y, z;                 /* eye position, blocks */
    float yaw_deg, pitch_deg;      /* yaw 0 looks along +z, 90 along +x; pitch > 0 looks up */
    float fov_deg;                 /* vertical field of view; 0 = 70 */
    float sun_x, sun_y, sun_z;     /* direction toward the sun (any length > 0) */
    float fog;                     /* haze distance in blocks; 0 = the window's reach */
} tg_camera;

tg_status tg_viewer_create(struct tg_generator* gen, const tg_viewer_config* config, struct tg_viewer** out);
/* Generates up to cap (0: max_batch_chunks) missing chunks within radius (at most
 * window_chunks / 2 - 1) of chunk (cx, cz), marking them born at frame; *generated (may
 * be NULL) receives their number and *ms (may be NULL) the device time of the generation
 * and window update. */
tg_status tg_viewer_update(struct tg_viewer* viewer, int32_t cx, int32_t cz, int32_t radius, int32_t cap, int32_t frame, int32_t* generated, float* ms);
/* Traces one frame. rgb_out (may be NULL): width * height * 3 u8, rows top to bottom;
 * hits_out (may be NULL): per pixel 4 int32 {palette index or -1, x, y, z} of the first
 * ray's hit; ms (may be NULL): the render kernel's device time. Chunks generated within 8
 * frames before frame are tinted green. */
tg_status tg_viewer_render(struct tg_viewer* viewer, const tg_camera* camera, int32_t frame, uint8_t* rgb_out, int32_t* hits_out, float* ms);
/* The window state for checks (each may be NULL): voxels (height * (16 * window_chunks)^2
 * u8, [y][z][x]), cells ((4 * window_chunks)^2 u32: 1 + highest non-air height index per
 * 4 x 4-column cell), slots (2 * window_chunks^2 int32: chunk x, z held per slot, INT32_MIN
 * when empty), born (window_chunks^2 int32). */
tg_status tg_viewer_state(struct tg_viewer* viewer, uint8_t* voxels, uint32_t* cells, int32_t* slots, int32_t* born);
/* The parameters a frame is traced with, for checks (each may be NULL): the camera record
 * (18 floats: eye, forward, right, up, tan(fov / 2), aspect, unit sun direction, haze
 * distance), the linear colours of the palette (64 x 3 floats of top faces, 64 x 3 of
 * sides), capped texel rows (64 int32), and {window_chunks, air, water, lava, bedrock,
 * min_y, height}. */
tg_status tg_viewer_params(struct tg_viewer* viewer, const tg_camera* camera, float* cam_out, float* top, float* side, int32_t* caps, int32_t* ids);
tg_status tg_viewer_destroy(struct tg_viewer* viewer);

/* ---- launch shapes and per-kernel times (the autotuner's interface) -----------------------
 * The batch pipeline's kernels run in the shapes of a launch table: the autotuned table
 * compiled into the library (minecraft-terrain-cuda_b200/tuning/launch_table.txt) unless one
 * is set here. Text format, one line per kernel, '#' starts a comment:
 *   <kernel> <threads 32..256, multiple of 32> <blocks_per_sm 1..32> <grab 0..64>
 *   table_load <2..8>
 *   host_u8 <batch> <tail_min> <tail_pct 0..99> <head_min> <head_pct 0|101..1000>
 *   host_u16 (the same)
 *   walk_defer <0..65536>       blocks per chunk of batch capacity in the column walk's
 *                               deferred list (blocks whose material rules need a per-block
 *                               noise; 0: no deferred pass)
 * host_u8 / host_u16: the batches of calls with host outputs in that form hold at most
 * batch chunks (0: max_batch_chunks); at the end of a call they shrink, each tail_pct % of
 * the one before, down to tail_min chunks; at the start they grow from head_min chunks by
 * head_pct % each (pct 0: no tail / no head).
 * grab 0 runs the kernel as a grid-stride loop; grab g > 0 as a persistent work queue whose
 * blocks take runs of g * threads items from a device counter. table_load sizes the dedupe
 * hash tables (capacity >= table_load x the keys a batch can insert). Kernel names, in
 * pipeline order: nb_insert nb_resolve climate_col climate_quart chain cc_insert cc_resolve
 * corner_col corner zoom_table zoom_uniform sg_insert sg_resolve surface_level aquifer_cell
 * aquifer_query aquifer_skip init_heights fill surface1 block_biome walk_rules
 * surface_frozen gather axis_insert axis_number axis_fill walk_deferred (the chain kernel has no
 * work-queue form). Results do not depend on the table. No counterpart in the reference (its launch shapes are constants). */
tg_status tg_set_launch_table(struct tg_generator* gen, const char* text);   /* NULL: the compiled-in table */
/* The table in use, as text (needed: its size with the terminating zero). */
tg_status tg_get_launch_table(struct tg_generator* gen, char* buf, size_t cap, size_t* needed);
/* The batch sizes a call with host outputs makes under a launch table (NULL: the compiled-in
 * one): count chunks in the u8 (u8 = 1) or u16 form on a generator of max_batch_chunks.
 * Writes at most cap sizes, in call order, and their number to n. Host only: needs no GPU. */
tg_status tg_host_schedule(const char* text, int32_t u8, int32_t count, int32_t max_batch_chunks, int32_t* sizes, int32_t cap, int32_t* n);
/* Per-kernel device times of timed batches (those of calls given a tg_timing): writes the
 * milliseconds and launch counts gathered since the previous call (cap entries, pipeline
 * order), clears them, and enables (enable = 1) or disables the per-kernel events. */
tg_status tg_kernel_times(struct tg_generator* gen, int32_t enable, float* ms, int32_t* calls, int32_t cap);

/* Pinned host memory for outputs. reference: alloc_pinned / free_pinned
 * (cuda/include/mccuda_cuda/terrain_gpu.h:62-63) */
void* tg_alloc_pinned(size_t bytes);
void tg_free_pinned(void* p);

/* Model constants: min_y, height, sea_level, palette size, biome count. */
tg_status tg_model_info(int32_t* min_y, int32_t* height, int32_t* sea_level, int32_t* palette_size, int32_t* biome_count);

/* Message of the last failing call on this thread (empty if none). */
const char* tg_last_error_string(void);

#ifdef __cplusplus
}
#endif

#endif /* TERRAIN_B200_H */
