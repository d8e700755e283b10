// TERRAIN step on sm_100a: kernels, the batch pipeline, the continuous-batching server
// and the C ABI of include/terrain_b200.h.
//
// Pipeline of one batch (all on one stream, all positions deduplicated on the device
// through hash tables, so nothing returns to the host until the outputs):
//   biome stage    neighbourhood union -> climate columns -> climate + first minimal
//                  leaf per quart -> last-result chain per biome chunk
//   noise stage    corner-column union -> hoisted y = 0 values -> 4x8 channel corners,
//                  zoom fiddle table
//   aquifer stage  surface-level quart union (volume / point) -> find_top_surface ->
//                  aquifer cell locations and fluid status, skip heights
//   fill           per 8-block cell column: channels, final density, substance, heights
//   surface        eroded badlands + frozen-ocean dry run per column, the walk state per
//                  column, the rule tree per block, the frozen-ocean extension per column
// The batch size lives in device memory and every kernel is a grid-stride loop, so the
// whole batch is captured once as a CUDA graph per output buffer and replayed for any
// batch size up to the capacity. Outputs are double-buffered: the copy stream drains
// batch k while batch k + 1 computes.
// Reference: cuda/src/terrain.cu:1259-1417 (run_batch / generate) and
// cpu/src/terrain.cpp:750-810.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <climits>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <filesystem>
#include <fstream>
#include <memory>
#include <mutex>
#include <sstream>
#include <stdexcept>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/terrain_b200.h"
#include "launch_table.h"   // generated from tuning/launch_table.txt: kLaunchTableText
#include "tb_pipeline.cuh"
#include "tb_viewer.cuh"

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

double now_ms() { return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count(); }

// ---- kernels: grid-stride loops over the bodies --------------------------------------------------
// Minimum resident 256-thread blocks per SM for the register-heavy kernels (caps registers).
#ifndef TB_MINB_WALK
#define TB_MINB_WALK 4
#endif
#ifndef TB_CHAIN_WARP
#define TB_CHAIN_WARP 1     // last-result chain with one warp per biome chunk
#endif
#ifndef TB_MINB_FILL
#define TB_MINB_FILL 1
#endif
#ifndef TB_MINB_CORNER
#define TB_MINB_CORNER 3
#endif
#ifndef TB_MINB_QUART
#define TB_MINB_QUART 4
#endif

// The per-item bodies of a batch run in one of two kernel forms, chosen per kernel by the
// launch table (an autotuned, committed table; see launch_shape below). Items number
// *count * MUL (count: the batch's chunk count or a device-side dedupe count).
//   k_body    grid-stride loop: thread t takes items t, t + grid, ...
//   k_body_q  persistent work queue: each block takes runs of grab * blockDim.x consecutive
//             items from a device counter (one atomicAdd per run) until the items run out,
//             so blocks that meet cheap items take more of them. Consecutive items stay on
//             consecutive lanes, as in the stride form.
template <void (*F)(const Batch&, int), int MUL, int MINB = 1>
__global__ void __launch_bounds__(256, MINB) k_body(const __grid_constant__ Batch B, const int32_t* count) {
    const int n = *count * MUL;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) F(B, i);
}

template <void (*F)(const Batch&, int), int MUL, int MINB = 1>
__global__ void __launch_bounds__(256, MINB) k_body_q(const __grid_constant__ Batch B, const int32_t* count, int32_t* next, int grab) {
    const int n = *count * MUL;
    const int run = grab * static_cast<int>(blockDim.x);
    __shared__ int32_t base;
    for (;;) {
        if (threadIdx.x == 0) base = atomicAdd(next, run);
        __syncthreads();
        const int b = base;
        __syncthreads();   // every thread has read base before thread 0 takes the next run
        if (b >= n) break;
        const int end = min(n, b + run);
        for (int i = b + static_cast<int>(threadIdx.x); i < end; i += blockDim.x) F(B, i);
    }
}

// Numbers the keys of one dedupe stage (TAB 0 biome chunks, 1 corner columns, 2 surface
// quarts): within each tile of 256 items, the items that are their key's first insert
// (ht_insert keeps the least item per key) take consecutive indices from one atomicAdd, so
// neighbouring entries of uniq come from neighbouring items. The host build numbers in plain
// item order (ht_number).
template <int TAB>
__device__ __forceinline__ const HashTab& dedupe_table(const Batch& B) {
    return TAB == 0 ? B.hb : (TAB == 1 ? B.hc : B.hs);
}
template <int TAB, unsigned long long (*K)(const Batch&, int), int MUL>
__global__ void __launch_bounds__(256) k_number(const __grid_constant__ Batch B) {
    const HashTab& t = dedupe_table<TAB>(B);
    const int n = *B.n_dev * MUL;
    __shared__ int32_t warp_off[8];
    __shared__ int32_t tile_base;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int tile = blockIdx.x * 256; tile < n; tile += gridDim.x * 256) {
        const int it = tile + static_cast<int>(threadIdx.x);
        bool first = false;
        unsigned long long key = 0;
        uint32_t slot = 0;
        if (it < n) {
            key = K(B, it);
            slot = ht_slot(t, key);
            first = slot <= t.mask && t.owner[slot] == it;
        }
        const unsigned ball = __ballot_sync(0xFFFFFFFFu, first);
        if (lane == 0) warp_off[wid] = __popc(ball);
        __syncthreads();
        if (threadIdx.x == 0) {
            int32_t sum = 0;
            for (int w = 0; w < 8; ++w) {
                const int32_t v = warp_off[w];
                warp_off[w] = sum;
                sum += v;
            }
            tile_base = sum ? atomicAdd(t.count, sum) : 0;
        }
        __syncthreads();
        if (first) {
            const int32_t idx = tile_base + warp_off[wid] + __popc(ball & ((1u << lane) - 1u));
            t.vals[slot] = idx;
            t.uniq[idx] = key;
        }
        __syncthreads();
    }
}

__device__ __forceinline__ void body_init_heights(const Batch& B, int i) { B.h0[i] = tbm::kMinY; }

__global__ void k_split_chunks(const tg_chunk_xz* ch, int n, int32_t slot, int32_t* cx, int32_t* cz, int32_t* cs, int32_t* n_dev) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        cx[i] = ch[i].x;
        cz[i] = ch[i].z;
        cs[i] = slot;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) *n_dev = n;
}

// Fills of a lane's dedupe tables and work-queue counters before a batch, as one launch:
// each segment is words 32-bit words at p set to value (16-byte stores for the bulk; every
// segment starts at an allocation's base, so p is 16-byte aligned).
struct ResetSeg {
    uint32_t* p;
    uint32_t words, value;
};
struct ResetList {
    ResetSeg seg[16];
    int n = 0;
    void add(void* p, size_t bytes, uint32_t value) {
        if (n == 16) throw Error(TG_ERR_INTERNAL, "reset list full");
        seg[n++] = ResetSeg{static_cast<uint32_t*>(p), static_cast<uint32_t>(bytes / 4), value};
    }
};
__global__ void k_reset(const ResetList L) {
    const uint32_t stride = gridDim.x * blockDim.x, t = blockIdx.x * blockDim.x + threadIdx.x;
    for (int j = 0; j < L.n; ++j) {
        const ResetSeg S = L.seg[j];
        const uint4 v = make_uint4(S.value, S.value, S.value, S.value);
        const uint32_t n4 = S.words >> 2;
        for (uint32_t i = t; i < n4; i += stride) reinterpret_cast<uint4*>(S.p)[i] = v;
        for (uint32_t i = 4 * n4 + t; i < S.words; i += stride) S.p[i] = S.value;
    }
}

// The last-result chain of body_chain with one warp per biome chunk. Lane k of a block of
// 32 quarts p first assumes the chain entered p holding L*(p - 1) (the previous quart's
// first minimal leaf; for lane 0 the true previous result) and decides whether that leaf is
// kept (it differs from L*(p) and reaches the minimum distance of p). While the assumption
// holds the block resolves from those decisions; a leaf that is carried past its own quart
// is tested against the following quarts of the block in one parallel round. Every result
// equals body_chain's.
__device__ void chain_warp(const Batch& B, int b, int lane) {
    const size_t base = static_cast<size_t>(b) * kQuartsPerChunk;
    const unsigned full = 0xFFFFFFFFu;
    int last = -1;
    for (int p0 = 0; p0 < kQuartsPerChunk; p0 += 32) {
        const size_t q = base + p0 + lane;
        const int ls = B.lstar[q];
        const long long md = B.mdist[q];
        const long long* t = B.tgt + q * 6;
        int prev = __shfl_up_sync(full, ls, 1);
        if (lane == 0) prev = last;
        const bool keep = prev >= 0 && prev != ls && param_dist(B.M.tree[B.M.leaf_node[prev]], t) == md;
        const unsigned keeps = __ballot_sync(full, keep);
        int r = ls;                 // this lane's result
        int v = last;               // chain value entering position pos (warp-uniform)
        int pos = 0;
        while (pos < 32) {
            const int spec = pos == 0 ? last : __shfl_sync(full, ls, pos - 1);
            if (v == spec) {
                const unsigned m = keeps & (full << pos);
                if (!m) {
                    pos = 32;
                    break;
                }
                const int j = __ffs(m) - 1;
                if (lane == j) r = prev;
                v = __shfl_sync(full, prev, j);
                pos = j + 1;
            } else {
                const bool carry = lane >= pos && v != ls && param_dist(B.M.tree[B.M.leaf_node[v]], t) == md;
                const unsigned run = __ballot_sync(full, carry) | ~(full << pos);
                const int j = (~run) ? __ffs(~run) - 1 : 32;   // first lane at or after pos that does not keep v
                if (lane >= pos && lane < j) r = v;
                if (j < 32) v = __shfl_sync(full, ls, j);
                pos = j + 1;
            }
        }
        last = __shfl_sync(full, r, 31);
        int qx, qy, qz;
        chain_quart(p0 + lane, qx, qy, qz);
        B.qbiome[base + (qy * 4 + qz) * 4 + qx] = static_cast<uint8_t>(B.M.leaf_biome[r]);
    }
}

__global__ void __launch_bounds__(256) k_chain_warp(const __grid_constant__ Batch B, const int32_t* count) {
    const int n = *count, lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < n; w += warps) chain_warp(B, w, lane);
}

// Biome lookups in two passes. Pass 1, one thread per position: the zoomed quart, its
// climate, first minimal leaf and tie test; a quart whose minimum is unique (or the chunk's
// first in chain order) has its result fixed, and the rest go to a list. Pass 2, one warp
// per listed position: the chain is replayed from the nearest earlier quart whose result is
// fixed, 32 quarts of the walk evaluated at a time (biome_point's result, without one thread
// walking hundreds of quarts while the rest of its warp waits).
struct TiedLookup {
    int32_t i, qx, cqy, qz, leaf;   // leaf: the quart's own first minimal leaf
};
__global__ void k_biome_point1(const __grid_constant__ DevModel M, const DevSeed* seeds, const int32_t* slot, const int32_t* xyz, int n, uint8_t* out,
                               TiedLookup* tied, int32_t* n_tied) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const DevSeed& S = seeds[slot[i]];
        const LookupQuart L = lookup_quart(S.zoom_seed, xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]);
        const QuartLeaf q = quart_leaf(M, S, L.qx, L.cqy, L.qz);
        if (!q.tie || L.p == 0) {
            out[i] = static_cast<uint8_t>(M.leaf_biome[q.leaf]);
        } else {
            tied[atomicAdd(n_tied, 1)] = TiedLookup{i, L.qx, L.cqy, L.qz, q.leaf};
        }
    }
}

// Leaves of the quarts a tied lookup walks back over, one 16-bit entry per chain position
// (index p - j), per warp of a 256-thread block.
constexpr int kTiedWarps = 8;
static_assert(tbm::kNumParams < 32768, "leaves are kept as 16-bit indices");

// The zoomed lookup of a tied quart (chain position p of its chunk): the reference's
// last-result chain from the nearest earlier quart whose result is fixed (unique minimum, or
// position 0). Only the column climate terms carry noise, so the chunk's 16 quart columns are
// evaluated once, lane c < 16 holding column (c >> 2, c & 3); the walk back keeps each quart's
// first minimal leaf in lf, and the replay needs per quart only its target and one leaf
// distance (the minimum it is compared with is the distance of that quart's own leaf).
__device__ int tied_chain(const DevModel& M, const DevSeed& S, const TiedLookup& T, int lane, int16_t* lf) {
    const unsigned full = 0xFFFFFFFFu;
    const int X0 = (T.qx >> 2) * 4, Z0 = (T.qz >> 2) * 4;
    const int p = chain_pos(T.qx & 3, T.cqy, T.qz & 3);
    float colv[tbm::kClimateCols];
    for (int k = 0; k < tbm::kClimateCols; ++k) colv[k] = 0.0f;
    if (lane < 16) tbgen::gen_climate_col(S.nt, 4 * (X0 + (lane >> 2)), 4 * (Z0 + (lane & 3)), colv);
    auto column_of = [&](int j, float* c) {
        const int src = ((j >> 4) & 3) * 4 + (j & 3);
        for (int k = 0; k < tbm::kClimateCols; ++k) c[k] = __shfl_sync(full, colv[k], src);
    };
    int a, b, cz;
    float c[tbm::kClimateCols];
    // walk back from p itself (lane 0 of the first window) to the nearest fixed j < p; a
    // lane's next quart is two layers below its last one in the same column, whose leaf
    // starts its search
    int anchor = -1, r = -1, start = T.leaf;
    __syncwarp();
    for (int base = p; anchor < 0; base -= 32) {
        const int j = base - lane;
        column_of(j < 0 ? 0 : j, c);
        bool fixed = false;
        int leaf = -1;
        if (j >= 0) {
            chain_quart(j, a, b, cz);
            const QuartLeaf q = quart_leaf_col(M, S, c, X0 + a, b, Z0 + cz, start);
            lf[p - j] = static_cast<int16_t>(q.leaf);
            fixed = j < p && (!q.tie || j == 0);
            leaf = start = q.leaf;
        }
        const unsigned m = __ballot_sync(full, fixed);
        if (m) {
            const int k = __ffs(m) - 1;
            anchor = base - k;
            r = __shfl_sync(full, leaf, k);
        }
    }
    __syncwarp();
    // replay the chain from the anchor to p, 32 quarts at a time (chain_warp's resolution)
    for (int k0 = anchor + 1; k0 <= p; k0 += 32) {
        const int nvalid = min(32, p - k0 + 1);
        const int k = k0 + lane;
        column_of(k > p ? p : k, c);
        long long t[6] = {0, 0, 0, 0, 0, 0}, um = 0;
        int ls = -1;
        if (lane < nvalid) {
            chain_quart(k, a, b, cz);
            quart_target(S, c, X0 + a, b, Z0 + cz, t);
            ls = lf[p - k];
            um = param_dist(M.tree[M.leaf_node[ls]], t);
        }
        int prev = __shfl_up_sync(full, ls, 1);
        if (lane == 0) prev = r;
        const bool keep = lane < nvalid && prev >= 0 && prev != ls && param_dist(M.tree[M.leaf_node[prev]], t) == um;
        const unsigned keeps = __ballot_sync(full, keep);
        int res = ls, v = r, pos = 0;
        while (pos < nvalid) {
            const int spec = pos == 0 ? r : __shfl_sync(full, ls, pos - 1);
            if (v == spec) {
                const unsigned mk = keeps & (full << pos);
                if (!mk) {
                    pos = nvalid;
                    break;
                }
                const int jj = __ffs(mk) - 1;
                if (jj >= nvalid) {
                    pos = nvalid;
                    break;
                }
                if (lane == jj) res = prev;
                v = __shfl_sync(full, prev, jj);
                pos = jj + 1;
            } else {
                const bool carry = lane >= pos && lane < nvalid && v != ls && param_dist(M.tree[M.leaf_node[v]], t) == um;
                const unsigned run = __ballot_sync(full, carry) | ~(full << pos);
                int jj = (~run) ? __ffs(~run) - 1 : 32;
                if (jj > nvalid) jj = nvalid;
                if (lane >= pos && lane < jj) res = v;
                if (jj < nvalid) v = __shfl_sync(full, ls, jj);
                pos = jj + 1;
            }
        }
        r = __shfl_sync(full, res, nvalid - 1);
    }
    __syncwarp();
    return r;
}

__global__ void __launch_bounds__(32 * kTiedWarps) k_biome_tied(const __grid_constant__ DevModel M, const DevSeed* seeds, const int32_t* slot, const TiedLookup* tied, const int32_t* n_tied,
                             uint8_t* out) {
    __shared__ int16_t lf[kTiedWarps][kQuartsPerChunk];
    const int n = *n_tied, lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < n; w += warps) {
        const TiedLookup T = tied[w];
        const int r = tied_chain(M, seeds[slot[T.i]], T, lane, lf[threadIdx.x >> 5]);
        if (lane == 0) out[T.i] = static_cast<uint8_t>(M.leaf_biome[r]);
    }
}


// u8 copies of u16 block states (the reference generator's output type: one palette index per
// block). Every state id is below the palette size, so the narrowing is exact. n8 groups of 8
// states: one 16-byte load and one 8-byte store each.
static_assert(tbm::kPaletteSize <= 256, "u8 block output needs every state id below 256");
__global__ void k_narrow_u8(const uint4* in, uint2* out, long n8) {
    for (long i = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x; i < n8; i += static_cast<long>(gridDim.x) * blockDim.x) {
        const uint4 v = in[i];
        uint2 o;
        o.x = (v.x & 0xFFu) | ((v.x >> 8) & 0xFF00u) | ((v.y & 0xFFu) << 16) | ((v.y >> 16) << 24);
        o.y = (v.z & 0xFFu) | ((v.z >> 8) & 0xFF00u) | ((v.w & 0xFFu) << 16) | ((v.w >> 16) << 24);
        out[i] = o;
    }
}

// Top-down records (the region writer's map) of n chunks of u16 states in HBM: chunk c is
// number first + c of a slab of whole chunk rows, region chunks per row, and its records go
// to rec (the slab's block rows, region * 16 columns each, 8 bytes per column). One thread
// per block column; a warp reads 32 neighbouring columns (64 contiguous bytes) per height.
// Per column: the highest non-air block (y 0 when all is air), then down while fluid and
// y > 0; u8 top, u8 floor, u8 min(255, depth), u8 0, int16 top y, int16 floor y.
__global__ void k_topdown(const uint16_t* blocks, const uint8_t* flags, int n, int first, int region, uint2* rec) {
    const long total = static_cast<long>(n) * 256;
    for (long t = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x; t < total; t += static_cast<long>(gridDim.x) * blockDim.x) {
        const int c = static_cast<int>(t >> 8), z = static_cast<int>(t >> 4) & 15, x = static_cast<int>(t) & 15;
        const uint16_t* b = blocks + static_cast<size_t>(c) * kBlocksPerChunk + z * 16 + x;
        int y = tbm::kHeight - 1;
        while (y > 0 && (flags[b[y * 256]] & 1)) --y;
        const uint32_t top = b[y * 256];
        const int top_y = y;
        while (y > 0 && (flags[b[y * 256]] & 8)) --y;
        const int g = first + c, r = g / region, i = g % region;
        const size_t side = static_cast<size_t>(region) * 16;
        uint2 v;
        v.x = top | (static_cast<uint32_t>(b[y * 256]) << 8) | (static_cast<uint32_t>(min(255, top_y - y)) << 16);
        v.y = static_cast<uint32_t>(static_cast<uint16_t>(tbm::kMinY + top_y)) | (static_cast<uint32_t>(static_cast<uint16_t>(tbm::kMinY + y)) << 16);
        rec[(static_cast<size_t>(r) * 16 + z) * side + static_cast<size_t>(i) * 16 + x] = v;
    }
}

// ---- device work queue of the device-resident multi-seed batch ----------------------------------
// The whole request list sits in HBM as a queue of (chunk, seed slot, request, index) items.
// Each iteration of a batch takes the next at most `cap` items (k_queue_take), runs the
// TERRAIN step on them, copies each chunk's outputs to its request's buffers
// (k_queue_scatter) and advances the queue (k_queue_advance), which also decides whether
// another iteration follows: inside one CUDA graph that decision is the condition of a
// WHILE node, so a whole request list runs from one graph launch.
struct QueueReq {                    // one request of the list
    const tg_chunk_xz* chunks;       // device memory
    uint16_t* blocks;                // device memory, 16-byte aligned
    uint8_t* biomes;                 // device memory, 16-byte aligned, or null
    int32_t first, count, slot, pad;
};
struct QueueView {
    const QueueReq* req;
    int32_t* cx;                     // items: chunk x, z, seed slot, request, index in the request
    int32_t* cz;
    int32_t* cs;
    int32_t* rq;
    int32_t* ix;
    int32_t* state;                  // head, total, iterations, iteration limit, items of the batch in flight
    int32_t n_req;
};

// The items of every request (one thread per item; the request found by binary search over
// the requests' first items).
__global__ void k_queue_fill(QueueView Q) {
    const int total = Q.state[1];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        int lo = 0, hi = Q.n_req - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (Q.req[mid].first <= i) lo = mid;
            else hi = mid - 1;
        }
        const QueueReq& r = Q.req[lo];
        const int j = i - r.first;
        Q.cx[i] = r.chunks[j].x;
        Q.cz[i] = r.chunks[j].z;
        Q.cs[i] = r.slot;
        Q.rq[i] = lo;
        Q.ix[i] = j;
    }
}

// The next batch: items [head, head + n), n = min(cap, total - head), into the batch's chunk
// arrays and its device-side count.
__global__ void k_queue_take(QueueView Q, int cap, int32_t* cx, int32_t* cz, int32_t* cs, int32_t* n_dev) {
    const int head = Q.state[0];
    const int n = max(0, min(cap, Q.state[1] - head));
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        cx[i] = Q.cx[head + i];
        cz[i] = Q.cz[head + i];
        cs[i] = Q.cs[head + i];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        *n_dev = n;
        Q.state[4] = n;
    }
}

// Each chunk of the batch in flight to its request's output buffers, 16 bytes per thread
// (12,288 of the blocks and 96 of the biomes per chunk).
constexpr int kScatterBlockVecs = kBlocksPerChunk * 2 / 16, kScatterBiomeVecs = kQuartsPerChunk / 16;
__global__ void k_queue_scatter(QueueView Q, const uint4* blocks, const uint4* biomes) {
    const int head = Q.state[0], n = Q.state[4];
    constexpr int per = kScatterBlockVecs + kScatterBiomeVecs;
    const long total = static_cast<long>(n) * per;
    for (long t = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x; t < total; t += static_cast<long>(gridDim.x) * blockDim.x) {
        const int c = static_cast<int>(t / per), k = static_cast<int>(t % per);
        const QueueReq& r = Q.req[Q.rq[head + c]];
        const size_t j = static_cast<size_t>(Q.ix[head + c]);
        if (k < kScatterBlockVecs) {
            reinterpret_cast<uint4*>(r.blocks)[j * kScatterBlockVecs + k] = blocks[static_cast<size_t>(c) * kScatterBlockVecs + k];
        } else if (r.biomes) {
            const int b = k - kScatterBlockVecs;
            reinterpret_cast<uint4*>(r.biomes)[j * kScatterBiomeVecs + b] = biomes[static_cast<size_t>(c) * kScatterBiomeVecs + b];
        }
    }
}

// Advances the queue past the batch in flight; with a graph loop, sets its condition: another
// iteration while items remain and the iteration limit (more than the list needs) is not
// reached. The head grows by at least one item per iteration that has items, so the loop ends.
__global__ void k_queue_advance(QueueView Q, cudaGraphConditionalHandle h, int looped) {
    const int head = Q.state[0] + Q.state[4];
    const int iters = Q.state[2] + 1;
    Q.state[0] = head;
    Q.state[2] = iters;
    Q.state[4] = 0;
    if (looped) cudaGraphSetConditional(h, (head < Q.state[1] && iters < Q.state[3]) ? 1u : 0u);
}

// ---- scratch of the no-allocation biome lookup ---------------------------------------------------
// tg_biome_lookup_noalloc stages its positions and results in this fixed device array
// instead of device buffers allocated per call. Callers that cannot allocate device memory
// after start-up use it: a server that reserves its whole HBM budget when it creates the
// generator (an allocation in the middle of a tick could fail), and a caller that must not
// cause the device-wide wait of cudaFree while other libraries' kernels run on other
// streams. The call still reuses the generator's batch buffers, so it waits for that
// generator's earlier work first. Layout: [0, 256) header, the u32 count of finished
// positions at offset 0, which must start at zero and is cleared by every call; then 3 x int32
// positions; then the u8 biomes. At most 4,096 positions per call: 53,504 bytes.
// Every call on a device shares this one array, so calls that overlap on the GPU race;
// each call waits for its own copies before it returns.
constexpr int kNoAllocMaxLookups = 4096;
constexpr size_t kNoAllocXyzOff = 256;
constexpr size_t kNoAllocOutOff = kNoAllocXyzOff + sizeof(int32_t) * 3 * kNoAllocMaxLookups;
constexpr size_t kNoAllocBytes = kNoAllocOutOff + kNoAllocMaxLookups;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

// Zoomed biomes of the positions staged in the no-allocation scratch, each from its chunk's
// neighbourhood computed by the biome stage; writes them to the scratch and counts the
// positions it finished into the scratch header.
__global__ void k_biome_lookup_scratch(const __grid_constant__ Batch B, unsigned char* scratch) {
    const int n = *B.n_dev;
    const int32_t* xyz = reinterpret_cast<const int32_t*>(scratch + kNoAllocXyzOff);
    uint8_t* out = scratch + kNoAllocOutOff;
    unsigned int finished = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        out[i] = static_cast<uint8_t>(zoom_biome(B, i, B.seeds[B.cseed[i]].zoom_seed, xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]));
        ++finished;
    }
    if (finished) atomicAdd(reinterpret_cast<unsigned int*>(scratch), finished);
}

// Device address of the scratch array on `device`, resolved once per device with that
// device current. The first call on a device does this set-up; make it before any
// stream capture begins.
unsigned char* noalloc_scratch(int device) {
    constexpr int kMaxDevices = 64;
    static std::mutex mu;
    static unsigned char* addr[kMaxDevices] = {};
    if (device < 0 || device >= kMaxDevices) throw Error(TG_ERR_INVALID_ARGUMENT, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(mu);
    if (!addr[device]) {
        int current = -1;
        ck(cudaGetDevice(&current), "cudaGetDevice");
        if (current != device) ck(cudaSetDevice(device), "cudaSetDevice");
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) throw Error(TG_ERR_CUDA, std::string("cudaGetSymbolAddress(no-allocation scratch): ") + cudaGetErrorString(e));
        addr[device] = static_cast<unsigned char*>(p);
    }
    return addr[device];
}

int g_sm_count = 148;
thread_local int g_launches = 0;

// grid for a grid-stride kernel: enough blocks for the items, at most 8 per SM
template <typename K, typename... Args>
void launch(K kernel, cudaStream_t s, long items_hint, Args... args) {
    const int threads = 256;
    long blocks = (items_hint + threads - 1) / threads;
    blocks = std::max(1L, std::min(blocks, static_cast<long>(g_sm_count) * 8));
    kernel<<<static_cast<unsigned>(blocks), threads, 0, s>>>(args...);
    ++g_launches;
}

// ---- launch shapes ------------------------------------------------------------------------------
// The tunable kernels of a batch, in pipeline order. Their shapes come from a launch table:
// the committed, autotuned table compiled in (tuning/launch_table.txt) or one set at run
// time (tg_set_launch_table). A line "kernel threads blocks_per_sm grab" per kernel (grab 0:
// grid-stride form; grab g > 0: work-queue form taking g * threads items per run), and
// "table_load f": dedupe hash tables of at least f times the most keys a batch can insert
// (rounded up to a power of two). "host_u8" and "host_u16" set how calls with host outputs
// of that form cut their chunks into batches (host_schedule): "host_u8 batch tail_min
// tail_pct head_min head_pct": batches of at most batch chunks (0: max_batch_chunks); the
// batches at the end of a call shrink, each at most tail_pct % of the one before
// it, down to tail_min chunks (tail_pct 0: no tail); the batches at the start grow from
// head_min chunks by head_pct % each (head_pct 0: no head).
enum KernelId {
    K_NB_INSERT, K_NB_RESOLVE, K_CLIMATE_COL, K_CLIMATE_QUART, K_CHAIN, K_CC_INSERT, K_CC_RESOLVE, K_CORNER_COL, K_CORNER, K_ZOOM_TABLE,
    K_ZOOM_UNIFORM, K_SG_INSERT, K_SG_RESOLVE, K_SURFACE_LEVEL, K_AQ_CELL, K_AQ_QUERY, K_AQ_SKIP, K_INIT_HEIGHTS, K_FILL, K_SURFACE1,
    K_BLOCK_BIOME, K_WALK, K_FROZEN, K_GATHER, K_AXIS_INSERT, K_AXIS_NUMBER, K_AXIS_FILL, K_WALK_DEFER, K_COUNT
};
const char* const kKernelNames[K_COUNT] = {"nb_insert", "nb_resolve", "climate_col", "climate_quart", "chain", "cc_insert", "cc_resolve",
                                           "corner_col", "corner", "zoom_table", "zoom_uniform", "sg_insert", "sg_resolve", "surface_level",
                                           "aquifer_cell", "aquifer_query", "aquifer_skip", "init_heights", "fill", "surface1", "block_biome",
                                           "walk_rules", "surface_frozen", "gather", "axis_insert", "axis_number", "axis_fill",
                                           "walk_deferred"};

struct LaunchShape {
    int threads = 256;        // 32 .. 256, a multiple of 32 (the kernels are built for at most 256)
    int blocks_per_sm = 8;    // grid = min(blocks for the items, blocks_per_sm * SMs)
    int grab = 0;             // 0: grid-stride; > 0: work queue, grab * threads items per run
};
#ifndef TB_HOST_BATCH
#define TB_HOST_BATCH 2048
#endif
#ifndef TB_DEFER_PER_CHUNK
#define TB_DEFER_PER_CHUNK 8192
#endif
#ifndef TB_HOST_BATCH_U8
#define TB_HOST_BATCH_U8 4096
#endif
#ifndef TB_TAIL_MIN
#define TB_TAIL_MIN 512
#endif
struct HostSchedule {
    int batch, tail_min, tail_pct, head_min, head_pct;
};
struct LaunchTable {
    LaunchShape k[K_COUNT];
    int table_load = 2;
    // "walk_defer n": the column walk's deferred list holds n blocks per chunk of batch
    // capacity (0: no deferred pass, every block's rules run in the walk)
    int defer_per_chunk = TB_DEFER_PER_CHUNK;
    // host[0]: the u16 output form, host[1]: u8. The u16 form's copies are slower than its
    // kernels, so smaller batches start them sooner; the u8 form's are faster, the kernels
    // bound the step and larger batches win.
    HostSchedule host[2] = {{TB_HOST_BATCH, TB_TAIL_MIN, 50, 0, 0}, {TB_HOST_BATCH_U8, TB_TAIL_MIN, 50, 0, 0}};
};

// The batch sizes of a call with host outputs: count chunks in batches of at most hb. The
// copy of the last batch is the one no compute hides, so the batches at the end shrink
// (tail); the first copy starts only when the first batch is done, so the batches at the
// start may grow (head). Full batches in between; a part batch goes first (or after the head).
std::vector<int> host_schedule(int count, int hb, const HostSchedule& t) {
    std::vector<int> tail, head, mid;
    long rem = count;
    if (t.tail_pct > 0 && t.tail_min > 0)
        for (long b = t.tail_min; rem > 0 && b < hb; b = std::max(b + 1, b * 100 / t.tail_pct)) {
            const int take = static_cast<int>(std::min(b, rem));
            tail.push_back(take);
            rem -= take;
        }
    if (t.head_pct > 100 && t.head_min > 0)
        for (long b = t.head_min; rem > 0 && b < hb; b = b * t.head_pct / 100) {
            const int take = static_cast<int>(std::min(b, rem));
            head.push_back(take);
            rem -= take;
        }
    const long part = rem % hb;
    if (part) mid.push_back(static_cast<int>(part));
    for (long i = 0; i < rem / hb; ++i) mid.push_back(hb);
    head.insert(head.end(), mid.begin(), mid.end());
    head.insert(head.end(), tail.rbegin(), tail.rend());
    return head;
}

// Parses a launch table; unknown kernels, bad values and malformed lines are errors.
LaunchTable parse_launch_table(const std::string& text) {
    LaunchTable t;
    std::istringstream in(text);
    std::string line;
    int ln = 0;
    while (std::getline(in, line)) {
        ++ln;
        const size_t hash = line.find('#');
        if (hash != std::string::npos) line.resize(hash);
        std::istringstream ls(line);
        std::string name;
        if (!(ls >> name)) continue;
        auto bad = [&](const char* why) { throw Error(TG_ERR_INVALID_ARGUMENT, "launch table line " + std::to_string(ln) + ": " + why); };
        if (name == "table_load") {
            if (!(ls >> t.table_load) || t.table_load < 2 || t.table_load > 8) bad("table_load must be 2..8");
            continue;
        }
        if (name == "walk_defer") {
            if (!(ls >> t.defer_per_chunk) || t.defer_per_chunk < 0 || t.defer_per_chunk > 65536) bad("walk_defer must be 0..65536");
            continue;
        }
        if (name == "host_u8" || name == "host_u16") {
            HostSchedule& h = t.host[name == "host_u8" ? 1 : 0];
            if (!(ls >> h.batch >> h.tail_min >> h.tail_pct >> h.head_min >> h.head_pct)) bad("expected: host_u8|host_u16 batch tail_min tail_pct head_min head_pct");
            if (h.batch < 0 || h.tail_min < 0 || h.head_min < 0) bad("host schedule sizes must be >= 0");
            if (h.tail_pct < 0 || h.tail_pct >= 100) bad("tail_pct must be 0..99");
            if (h.head_pct != 0 && (h.head_pct <= 100 || h.head_pct > 1000)) bad("head_pct must be 0 or 101..1000");
            continue;
        }
        int id = -1;
        for (int i = 0; i < K_COUNT; ++i)
            if (name == kKernelNames[i]) id = i;
        if (id < 0) bad("unknown kernel");
        LaunchShape& k = t.k[id];
        if (!(ls >> k.threads >> k.blocks_per_sm >> k.grab)) bad("expected: kernel threads blocks_per_sm grab");
        if (k.threads < 32 || k.threads > 256 || k.threads % 32) bad("threads must be a multiple of 32 in 32..256");
        if (k.blocks_per_sm < 1 || k.blocks_per_sm > 32) bad("blocks_per_sm must be 1..32");
        if (k.grab < 0 || k.grab > 64) bad("grab must be 0..64");
        if (id == K_CHAIN && k.grab) bad("the chain kernel has no work-queue form");
    }
    return t;
}

std::string format_launch_table(const LaunchTable& t) {
    std::ostringstream o;
    o << "table_load " << t.table_load << "\n";
    o << "walk_defer " << t.defer_per_chunk << "\n";
    for (int f = 1; f >= 0; --f) {
        const HostSchedule& h = t.host[f];
        o << (f ? "host_u8 " : "host_u16 ") << h.batch << ' ' << h.tail_min << ' ' << h.tail_pct << ' ' << h.head_min << ' ' << h.head_pct << "\n";
    }
    for (int i = 0; i < K_COUNT; ++i) o << kKernelNames[i] << ' ' << t.k[i].threads << ' ' << t.k[i].blocks_per_sm << ' ' << t.k[i].grab << "\n";
    return o.str();
}

uint32_t pow2_at_least(uint64_t v) {
    uint32_t p = 1024;
    while (p < v) p <<= 1;
    return p;
}

// ---- device and pinned memory -------------------------------------------------------------------
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    bool owned = true;   // false: a view into another buffer
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() {
        if (p && owned) cudaFree(p);
    }
    void alloc(size_t b) {
        if (p && owned) cudaFree(p);
        p = nullptr;
        owned = true;
        bytes = b;
        if (b) ck(cudaMalloc(&p, b), "cudaMalloc");
    }
    void view(void* base, size_t b) {
        if (p && owned) cudaFree(p);
        p = base;
        bytes = b;
        owned = false;
    }
    template <class T>
    T* as() const {
        return static_cast<T*>(p);
    }
};

struct PinBuf {
    void* p = nullptr;
    PinBuf() = default;
    PinBuf(const PinBuf&) = delete;
    PinBuf& operator=(const PinBuf&) = delete;
    ~PinBuf() {
        if (p) cudaFreeHost(p);
    }
    void alloc(size_t b) {
        if (p) cudaFreeHost(p);
        p = nullptr;
        if (b) ck(cudaMallocHost(&p, b), "cudaMallocHost");
    }
    template <class T>
    T* as() const {
        return static_cast<T*>(p);
    }
};

struct TableBufs {
    DevBuf keys, vals, uniq, count, owner;
    uint32_t cap = 0;
    uint32_t* err = nullptr;   // the lane's error word (Work::d_err)
    void alloc(uint64_t max_keys, int load) {
        cap = pow2_at_least(static_cast<uint64_t>(load) * max_keys);
        keys.alloc(sizeof(unsigned long long) * cap);
        vals.alloc(sizeof(int32_t) * cap);
        owner.alloc(sizeof(int32_t) * cap);
        uniq.alloc(sizeof(unsigned long long) * max_keys);
        count.alloc(sizeof(int32_t));
    }
    HashTab view() const {
        return HashTab{keys.as<unsigned long long>(), vals.as<int32_t>(), uniq.as<unsigned long long>(), count.as<int32_t>(), cap - 1, owner.as<int32_t>(), err};
    }
    // free slots; owners above every item index (0x7F7F7F7F)
    void add_reset(ResetList& L) const {
        L.add(keys.p, keys.bytes, 0xFFFFFFFFu);
        L.add(owner.p, owner.bytes, 0x7F7F7F7Fu);
        L.add(count.p, sizeof(int32_t), 0u);
    }
};

constexpr int kMaxSlots = 512;   // resident seeds (the 9-bit seed field of the position keys)

struct SeedSlot {
    int64_t seed = 0;
    bool valid = false;
    uint64_t last_use = 0;
    DevBuf tables;   // octave offsets | layers | paired permutations | byte permutations | corner y records, 256-byte aligned
};

// one output buffer set (the pipeline's outputs are double-buffered)
struct OutSlot {
    DevBuf blocks, biomes, aquifer;
    DevBuf blocks8, aquifer8;  // u8 copies for the u8 output form, allocated on first use
    PinBuf coords;             // staged cx | cz | cs | n of the batch
    cudaEvent_t computed = nullptr, drained = nullptr;
    cudaGraphExec_t graph = nullptr;
    bool graph_aquifer = false;
    cudaStream_t graph_stream = nullptr;
    bool busy = false;         // outputs not yet drained to the host
    int lane = 0;              // working buffers and stream its batches use
};

// The working buffers of one batch in flight (tables, climate, corners, aquifer, heights,
// per-block biomes). A generator holds one set per lane; two lanes let the batches of the
// two output slots run concurrently on two streams.
struct Work {
    DevBuf d_coords, d_n, d_cx, d_cz, d_cs, d_nb9, d_bcol, d_tgt, d_lstar, d_mdist, d_qbiome, d_c25, d_ccol, d_corners, d_g513, d_sfts, d_aq_cell,
        d_aq_query, d_aq_skip, d_h0, d_h1, d_h2, d_zoom, d_zoom_uni, d_bbiome, d_oremask, d_colmask, d_colrec, d_qnext, d_err, d_axtab, d_colax,
        d_defer, d_defer_count;
    TableBufs tb_b, tb_c, tb_s, tb_a;
    int32_t defer_cap = 0;
    void alloc(int n, int load, int defer_per_chunk) {
        const size_t N = static_cast<size_t>(n);
        // chunk x | chunk z | seed slot | count, the layout of an output slot's staged
        // coordinates, so that one copy uploads them
        d_coords.alloc(4 * (3 * N + 1));
        d_cx.view(d_coords.as<int32_t>(), 4 * N);
        d_cz.view(d_coords.as<int32_t>() + N, 4 * N);
        d_cs.view(d_coords.as<int32_t>() + 2 * N, 4 * N);
        d_n.view(d_coords.as<int32_t>() + 3 * N, 4);
        d_err.alloc(sizeof(uint32_t));
        ck(cudaMemset(d_err.p, 0, sizeof(uint32_t)), "memset");
        tb_b.err = tb_c.err = tb_s.err = tb_a.err = d_err.as<uint32_t>();
        if (TB_AXIS_TABLE) {
            // at most 5 distinct corner x and 5 distinct corner z per chunk
            tb_a.alloc(10 * N, load);
            d_axtab.alloc(sizeof(AxisRec) * 10 * N * std::max(1, tbm::kAxisLayers));
            d_colax.alloc(sizeof(int32_t) * 2 * 25 * N);
        }
        d_qnext.alloc(sizeof(int32_t) * K_COUNT);   // work-queue counters, one per kernel
        tb_b.alloc(9 * N, load);
        tb_c.alloc(25 * N, load);
        tb_s.alloc(static_cast<uint64_t>(kGrid) * N, load);
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
        d_aq_cell.alloc(sizeof(AqCell) * N * kAqCells);
        d_aq_query.alloc(sizeof(AqQuery) * N * kAqQueries);
        d_aq_skip.alloc(4 * N);
        d_h0.alloc(4 * 256 * N);
        d_h1.alloc(4 * 256 * N);
        d_h2.alloc(4 * 256 * N);
        d_zoom.alloc(sizeof(uint32_t) * N * kZoomVerts);
        d_zoom_uni.alloc(N * kZoomCells);
        d_bbiome.alloc(N * kBlocksPerChunk);
        if (TB_ORE_MASK) d_oremask.alloc(N * kBlocksPerChunk);
        d_colmask.alloc(sizeof(uint32_t) * N * 2 * kMaskWords * 256);
        d_colrec.alloc(sizeof(ColumnRec) * N * 256);
        defer_cap = static_cast<int32_t>(std::min<size_t>(static_cast<size_t>(defer_per_chunk) * N, INT32_MAX / 2));
        d_defer.alloc(sizeof(DeferRec) * static_cast<size_t>(defer_cap));
        d_defer_count.alloc(sizeof(int32_t));
    }
};

}  // namespace

// ---- the generator ----------------------------------------------------------------------------------
struct Generator {
#ifndef TB_ORDERED_BATCH
#define TB_ORDERED_BATCH 2048
#endif
    static constexpr int kOrderedBatch = TB_ORDERED_BATCH;   // batches this large run one after another
    int device = 0;
    int max_batch = 2048;
    cudaStream_t stream = nullptr;      // compute stream (the caller's, when set)
    cudaStream_t own_stream = nullptr;
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t ev[10] = {};
    bool use_graphs = true;
    std::atomic<bool> served{false};    // owned by a server's worker thread
    // model
    DevBuf d_boxes, d_box_leaf, d_tree, d_children, d_leaf_biome, d_leaf_node, d_leaf_rank, d_flags, d_btemp, d_bfrozen;
    DevModel model{};
    int tree_depth = 0;
    // seeds
    std::unique_ptr<SeedSlot[]> slots;
    DevBuf d_seeds;
    DevBuf call_chunks;   // the chunk list of a call with host outputs (grown to the largest call)
    uint64_t use_clock = 0;
    int current_slot = -1;
    // working buffers per lane: lane 0 runs on `stream`, lane 1 on lane_stream
    Work work[2];
    int lanes = 2;
    cudaStream_t lane_stream = nullptr;
    cudaEvent_t ev_entry = nullptr;
    // per lane: the streams the biome and aquifer stages run on beside the lane's other
    // stages, and the events that fork them from and join them back into the lane's stream
    cudaStream_t side_stream[2] = {nullptr, nullptr}, aq_stream[2] = {nullptr, nullptr};
    cudaEvent_t ev_fork[2] = {nullptr, nullptr}, ev_join[2] = {nullptr, nullptr}, ev_join_aq[2] = {nullptr, nullptr};
    OutSlot out[2];
    int next_out = 0;
    int graph_launches = 0;
    LaunchTable lt = parse_launch_table(kLaunchTableText);
    // per-kernel event times of timed batches (tg_kernel_times); prof_now while a timed
    // batch is being enqueued with prof set
    bool prof = false, prof_now = false;
    cudaEvent_t prof_ev[2 * K_COUNT] = {};
    bool prof_marked[K_COUNT] = {};
    double prof_ms[K_COUNT] = {};
    int prof_calls[K_COUNT] = {};

    Generator(int dev, int batch, int pipeline_slots) : device(dev), max_batch(batch), lanes(pipeline_slots == 1 ? 1 : 2) {
        ck(cudaSetDevice(device), "cudaSetDevice");
        cudaDeviceProp prop{};
        ck(cudaGetDeviceProperties(&prop, device), "cudaGetDeviceProperties");
        g_sm_count = prop.multiProcessorCount;
        ck(cudaStreamCreateWithFlags(&own_stream, cudaStreamNonBlocking), "cudaStreamCreate");
        ck(cudaStreamCreateWithFlags(&copy_stream, cudaStreamNonBlocking), "cudaStreamCreate");
        ck(cudaStreamCreateWithFlags(&lane_stream, cudaStreamNonBlocking), "cudaStreamCreate");
        ck(cudaEventCreateWithFlags(&ev_entry, cudaEventDisableTiming), "cudaEventCreate");
        for (int l = 0; l < 2; ++l) {
            ck(cudaStreamCreateWithFlags(&side_stream[l], cudaStreamNonBlocking), "cudaStreamCreate");
            ck(cudaStreamCreateWithFlags(&aq_stream[l], cudaStreamNonBlocking), "cudaStreamCreate");
            ck(cudaEventCreateWithFlags(&ev_fork[l], cudaEventDisableTiming), "cudaEventCreate");
            ck(cudaEventCreateWithFlags(&ev_join[l], cudaEventDisableTiming), "cudaEventCreate");
            ck(cudaEventCreateWithFlags(&ev_join_aq[l], cudaEventDisableTiming), "cudaEventCreate");
        }
        stream = own_stream;
        out[1].lane = lanes == 2 ? 1 : 0;
        for (auto& e : ev) ck(cudaEventCreate(&e), "cudaEventCreate");
        for (auto& e : prof_ev) ck(cudaEventCreate(&e), "cudaEventCreate");
        for (auto& o : out) {
            ck(cudaEventCreateWithFlags(&o.computed, cudaEventDisableTiming), "cudaEventCreate");
            ck(cudaEventCreateWithFlags(&o.drained, cudaEventDisableTiming), "cudaEventCreate");
        }
        upload_model();
        slots.reset(new SeedSlot[kMaxSlots]);
        d_seeds.alloc(sizeof(DevSeed) * kMaxSlots);
        alloc_batch(max_batch);
    }
    ~Generator() {
        cudaSetDevice(device);
        cudaDeviceSynchronize();
        destroy_queue_graphs();
        for (auto& o : out) {
            if (o.graph) cudaGraphExecDestroy(o.graph);
            if (o.computed) cudaEventDestroy(o.computed);
            if (o.drained) cudaEventDestroy(o.drained);
        }
        for (auto& e : ev)
            if (e) cudaEventDestroy(e);
        for (auto& e : prof_ev)
            if (e) cudaEventDestroy(e);
        if (ev_entry) cudaEventDestroy(ev_entry);
        for (int l = 0; l < 2; ++l) {
            if (ev_fork[l]) cudaEventDestroy(ev_fork[l]);
            if (ev_join[l]) cudaEventDestroy(ev_join[l]);
            if (ev_join_aq[l]) cudaEventDestroy(ev_join_aq[l]);
            if (side_stream[l]) cudaStreamDestroy(side_stream[l]);
            if (aq_stream[l]) cudaStreamDestroy(aq_stream[l]);
        }
        if (lane_stream) cudaStreamDestroy(lane_stream);
        if (copy_stream) cudaStreamDestroy(copy_stream);
        if (own_stream) cudaStreamDestroy(own_stream);
    }

    template <class T>
    void upload(DevBuf& b, const std::vector<T>& v) {
        b.alloc(sizeof(T) * std::max<size_t>(v.size(), 1));
        if (!v.empty()) ck(cudaMemcpy(b.p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice), "upload");
    }

    std::vector<uint8_t> seed_image;   // host image of one seed's tables, reused

    void upload_model() {
        ModelHost m;
        build_model_host(m);
        upload(d_tree, m.nodes);
        if (!m.boxes.empty()) {
            upload(d_boxes, m.boxes);
            upload(d_box_leaf, m.box_leaf);
        }
        upload(d_children, m.children);
        upload(d_leaf_biome, m.leaf_biome);
        upload(d_leaf_node, m.leaf_node);
        upload(d_leaf_rank, m.leaf_rank);
        upload(d_flags, std::vector<uint8_t>(tbm::kBlockFlags, tbm::kBlockFlags + tbm::kPaletteSize));
        upload(d_btemp, std::vector<float>(tbm::kBiomeTemp, tbm::kBiomeTemp + tbm::kNumBiomes));
        upload(d_bfrozen, std::vector<uint8_t>(tbm::kBiomeFrozen, tbm::kBiomeFrozen + tbm::kNumBiomes));
        if (m.depth >= kSearchStack) throw Error(TG_ERR_INTERNAL, "climate tree deeper than the search stack");
        tree_depth = m.depth;
        model.boxes = m.boxes.empty() ? nullptr : d_boxes.as<RBox>();
        model.box_leaf = m.boxes.empty() ? nullptr : d_box_leaf.as<int32_t>();
        model.tree = d_tree.as<RNode>();
        model.children = d_children.as<int32_t>();
        model.leaf_biome = d_leaf_biome.as<int32_t>();
        model.leaf_node = d_leaf_node.as<int32_t>();
        model.leaf_rank = d_leaf_rank.as<int32_t>();
        model.root = m.root;
        model.depth = m.depth;
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
        for (int l = 0; l < lanes; ++l) work[l].alloc(n, lt.table_load, lt.defer_per_chunk);
        for (auto& o : out) {
            o.blocks.alloc(sizeof(uint16_t) * N * kBlocksPerChunk);
            o.biomes.alloc(N * kQuartsPerChunk);
            o.coords.alloc(sizeof(int32_t) * (3 * N + 1));
        }
    }

    // HBM the batch buffers take per chunk of batch capacity: both lanes' working buffers and
    // both output slots (u16 blocks and biomes, and their u8 copies once allocated)
    double device_bytes_per_chunk() const {
        size_t b = 0;
        for (int l = 0; l < lanes; ++l) {
            const Work& W = work[l];
            for (const DevBuf* d : {&W.d_cx, &W.d_cz, &W.d_cs, &W.d_nb9, &W.d_bcol, &W.d_tgt, &W.d_lstar, &W.d_mdist, &W.d_qbiome, &W.d_c25, &W.d_ccol,
                                    &W.d_corners, &W.d_g513, &W.d_sfts, &W.d_aq_cell, &W.d_aq_query, &W.d_aq_skip, &W.d_h0, &W.d_h1, &W.d_h2,
                                    &W.d_zoom, &W.d_zoom_uni, &W.d_bbiome, &W.d_oremask, &W.d_colmask, &W.d_colrec, &W.d_axtab, &W.d_colax,
                                    &W.d_defer})
                b += d->bytes;
            for (const TableBufs* t : {&W.tb_b, &W.tb_c, &W.tb_s, &W.tb_a}) b += t->keys.bytes + t->vals.bytes + t->uniq.bytes + t->owner.bytes;
        }
        for (const OutSlot& o : out) b += o.blocks.bytes + o.biomes.bytes + o.blocks8.bytes;
        return static_cast<double>(b) / static_cast<double>(max_batch);
    }

    // Resident per-seed tables: the slot of a seed, built and uploaded on a miss; slots
    // listed in `keep` are not evicted.
    // The slot holding seed's tables (refreshing its use), or -1.
    int resident_slot(int64_t seed) {
        for (int i = 0; i < kMaxSlots; ++i)
            if (slots[i].valid && slots[i].seed == seed) {
                slots[i].last_use = ++use_clock;
                return i;
            }
        return -1;
    }

    int seed_slot(int64_t seed, const std::vector<int>& keep = {}) {
        const int r = resident_slot(seed);
        if (r >= 0) return r;
        SeedHost h;
        build_seed_host(seed, h);
        return install_seed(seed, h, keep);
    }

    // Puts host tables h of seed into a free slot, else the least recently used one not in
    // keep, and returns it.
    // sync = false: the caller guarantees that no queued work reads a slot outside keep.
    int install_seed(int64_t seed, const SeedHost& h, const std::vector<int>& keep, bool sync = true) {
        ++use_clock;
        int free_slot = -1, lru = -1;
        for (int i = 0; i < kMaxSlots; ++i)
            if (!slots[i].valid && free_slot < 0) free_slot = i;
        int s = free_slot;
        if (s < 0) {
            for (int i = 0; i < kMaxSlots; ++i) {
                if (std::find(keep.begin(), keep.end(), i) != keep.end()) continue;
                if (lru < 0 || slots[i].last_use < slots[lru].last_use) lru = i;
            }
            s = lru;
        }
        if (s < 0) throw Error(TG_ERR_INTERNAL, "no free seed slot");
        // queued work may still read the tables this slot held
        if (slots[s].valid && sync) ck(cudaDeviceSynchronize(), "sync");
        SeedSlot& sl = slots[s];
        // one image and one copy per seed; the byte permutation table is read only by the
        // unpaired hash form
        auto al = [](size_t v) { return (v + 255) & ~static_cast<size_t>(255); };
        const size_t b_off = sizeof(OctaveOff) * h.off.size(), b_lay = sizeof(Layer) * h.layers.size(), b_p2 = sizeof(uint16_t) * h.perm2.size();
        const size_t b_p = TB_PERM_PAIRS ? 0 : h.perm.size();
        const size_t b_y = sizeof(AxisRec) * h.ytab.size();
        const size_t o_lay = al(b_off), o_p2 = o_lay + al(b_lay), o_p = o_p2 + al(b_p2), o_y = o_p + al(b_p), total = o_y + al(b_y);
        seed_image.assign(total, 0);
        std::memcpy(seed_image.data(), h.off.data(), b_off);
        std::memcpy(seed_image.data() + o_lay, h.layers.data(), b_lay);
        std::memcpy(seed_image.data() + o_p2, h.perm2.data(), b_p2);
        if (b_p) std::memcpy(seed_image.data() + o_p, h.perm.data(), b_p);
        if (b_y) std::memcpy(seed_image.data() + o_y, h.ytab.data(), b_y);
        if (!sl.tables.p || sl.tables.bytes != total) sl.tables.alloc(total);
        ck(cudaMemcpy(sl.tables.p, seed_image.data(), total, cudaMemcpyHostToDevice), "seed upload");
        const uint8_t* base = sl.tables.as<uint8_t>();
        DevSeed d{};
        d.nt = NoiseTables{reinterpret_cast<const OctaveOff*>(base), b_p ? base + o_p : nullptr, reinterpret_cast<const Layer*>(base + o_lay),
                           reinterpret_cast<const uint16_t*>(base + o_p2)};
        d.ytab = reinterpret_cast<const AxisRec*>(base + o_y);
        d.random = h.random;
        d.aquifer = h.aquifer;
        d.ore = h.ore;
        for (size_t k = 0; k < h.gradient.size(); ++k) d.gradient[k] = h.gradient[k];
        d.zoom_seed = h.zoom_seed;
        std::memcpy(d.clay, h.clay, sizeof d.clay);
        ck(cudaMemcpy(d_seeds.as<DevSeed>() + s, &d, sizeof(DevSeed), cudaMemcpyHostToDevice), "seed upload");
        sl.seed = seed;
        sl.valid = true;
        sl.last_use = use_clock;
        return s;
    }

    Batch batch_view(const Work& W, const OutSlot* o) const {
        Batch B{};
        B.M = model;
        B.seeds = d_seeds.as<DevSeed>();
        B.n_dev = W.d_n.as<int32_t>();
        B.cx = W.d_cx.as<int32_t>();
        B.cz = W.d_cz.as<int32_t>();
        B.cseed = W.d_cs.as<int32_t>();
        B.hb = W.tb_b.view();
        B.nb_cap = 9 * max_batch;
        B.nb9 = W.d_nb9.as<int32_t>();
        B.bcol = W.d_bcol.as<float>();
        B.tgt = W.d_tgt.as<long long>();
        B.lstar = W.d_lstar.as<int32_t>();
        B.mdist = W.d_mdist.as<long long>();
        B.qbiome = W.d_qbiome.as<uint8_t>();
        B.hc = W.tb_c.view();
        B.cc_cap = 25 * max_batch;
        B.c25 = W.d_c25.as<int32_t>();
        B.ccol = W.d_ccol.as<float>();
        B.ha = W.tb_a.view();
        B.axtab = W.d_axtab.as<AxisRec>();
        B.colax = W.d_colax.as<int32_t>();
        B.corners = W.d_corners.as<float>();
        B.hs = W.tb_s.view();
        B.sg_cap = kGrid * max_batch;
        B.g513 = W.d_g513.as<int32_t>();
        B.sfts = W.d_sfts.as<float>();
        B.aq_cell = W.d_aq_cell.as<AqCell>();
        B.aq_query = W.d_aq_query.as<AqQuery>();
        B.aq_skip = W.d_aq_skip.as<int32_t>();
        B.blocks = o ? o->blocks.as<uint16_t>() : nullptr;
        B.h0 = W.d_h0.as<int32_t>();
        B.h1 = W.d_h1.as<int32_t>();
        B.h2 = W.d_h2.as<int32_t>();
        B.biomes_out = o ? o->biomes.as<uint8_t>() : nullptr;
        B.zoom_tab = W.d_zoom.as<uint32_t>();
        B.zoom_uni = W.d_zoom_uni.as<uint8_t>();
        B.bbiome = W.d_bbiome.as<uint8_t>();
        B.oremask = W.d_oremask.as<uint8_t>();
        B.colmask = W.d_colmask.as<uint32_t>();
        B.colrec = W.d_colrec.as<ColumnRec>();
        B.defer = W.defer_cap > 0 ? W.d_defer.as<DeferRec>() : nullptr;
        B.defer_count = W.d_defer_count.as<int32_t>();
        B.defer_cap = W.defer_cap;
        return B;
    }

    // One tunable body kernel in the shape the launch table gives it; items_hint (an upper
    // bound of the items) sizes the grid, count (device memory) x MUL is the item count.
    template <void (*F)(const Batch&, int), int MUL, int MINB = 1>
    void run_body(KernelId id, const Work& W, cudaStream_t s, long items_hint, const Batch& B, const int32_t* count) {
        const LaunchShape& k = lt.k[id];
        long blocks = (items_hint + k.threads - 1) / k.threads;
        blocks = std::max(1L, std::min(blocks, static_cast<long>(g_sm_count) * k.blocks_per_sm));
        if (prof_now) ck(cudaEventRecord(prof_ev[2 * id], s), "event");
        if (k.grab > 0)
            k_body_q<F, MUL, MINB><<<static_cast<unsigned>(blocks), k.threads, 0, s>>>(B, count, W.d_qnext.as<int32_t>() + id, k.grab);
        else
            k_body<F, MUL, MINB><<<static_cast<unsigned>(blocks), k.threads, 0, s>>>(B, count);
        ++g_launches;
        if (prof_now) {
            ck(cudaEventRecord(prof_ev[2 * id + 1], s), "event");
            prof_marked[id] = true;
        }
    }

    // One launch that clears the lane's work-queue counters and dedupe tables for a batch:
    // the biome stage's table, and with all those of the whole step. (Separate memsets, six
    // to a batch, each waited behind the copies of the other output slot on the copy engines.)
    void reset_lane(const Work& W, cudaStream_t s, bool all) {
        ResetList L;
        L.add(W.d_qnext.p, W.d_qnext.bytes, 0u);
        W.tb_b.add_reset(L);
        if (all) {
            L.add(W.d_defer_count.p, W.d_defer_count.bytes, 0u);
            W.tb_c.add_reset(L);
            W.tb_s.add_reset(L);
            if (TB_AXIS_TABLE && tbm::kAxisLayers > 0) W.tb_a.add_reset(L);
        }
        size_t words = 0;
        for (int i = 0; i < L.n; ++i) words += L.seg[i].words;
        launch(k_reset, s, static_cast<long>(words / 4), L);
    }

    // biome stage (shared by the TERRAIN step and biome lookups); nmax sizes the grids;
    // reset: clear the counters and the table first (else reset_lane ran before)
    void enqueue_biomes(const Work& W, const Batch& B, cudaStream_t s, long nmax, bool reset = true) {
        const int32_t* n_dev = B.n_dev;
        const int32_t* cnt_b = W.tb_b.count.as<int32_t>();
        if (reset) reset_lane(W, s, false);
        run_body<body_nb_insert, 9>(K_NB_INSERT, W, s, 9 * nmax, B, n_dev);
        launch(k_number<0, nb_key, 9>, s, 9 * nmax, B);
        run_body<body_nb_resolve, 9>(K_NB_RESOLVE, W, s, 9 * nmax, B, n_dev);
        run_body<body_climate_col, 16>(K_CLIMATE_COL, W, s, nmax * 16 * 2, B, cnt_b);
        run_body<body_climate_quart, 16 * kRuns, TB_MINB_QUART>(K_CLIMATE_QUART, W, s, nmax * 16 * kRuns * 2, B, cnt_b);
        {
            const LaunchShape& k = lt.k[K_CHAIN];
            long blocks = (nmax * 2 * 32 + k.threads - 1) / k.threads;
            blocks = std::max(1L, std::min(blocks, static_cast<long>(g_sm_count) * k.blocks_per_sm));
            if (prof_now) ck(cudaEventRecord(prof_ev[2 * K_CHAIN], s), "event");
            k_chain_warp<<<static_cast<unsigned>(blocks), k.threads, 0, s>>>(B, cnt_b);
            ++g_launches;
            if (prof_now) {
                ck(cudaEventRecord(prof_ev[2 * K_CHAIN + 1], s), "event");
                prof_marked[K_CHAIN] = true;
            }
        }
    }

    // every kernel of one batch; with timed set, events split the stages; reset: clear the
    // lane's counters and tables first (else the caller ran reset_lane before).
    // fork (untimed batches): the biome stage reads only the chunk list, as do the noise,
    // aquifer and fill stages, so it runs on the lane's side stream beside them, followed by
    // the zoom tables and the quart biome output, and joins before the surface stage; the
    // aquifer stage does not
    // read the noise stage's corners either, so it runs on a second side stream beside the
    // noise stage and joins before the fill. The long last items of each stage's kernels then
    // overlap the other stages' kernels instead of leaving SMs idle.
    // Timed batches keep one stream, so that events split the stages.
    void enqueue_batch(const Work& W, const Batch& B, cudaStream_t s, long nmax, uint16_t* aquifer_dev, bool timed, bool reset = true,
                       bool fork = true) {
        auto mark = [&](int i) {
            if (timed) ck(cudaEventRecord(ev[i], s), "event");
        };
        const int32_t* cnt_c = W.tb_c.count.as<int32_t>();
        const int32_t* cnt_s = W.tb_s.count.as<int32_t>();
        prof_now = timed && prof;
        if (reset) reset_lane(W, s, true);
        mark(0);
        const int li = &W == &work[0] ? 0 : 1;
        const bool side = fork && !timed;
        cudaStream_t sb = side ? side_stream[li] : s;
        cudaStream_t sq = side ? aq_stream[li] : s;
        if (side) {
            ck(cudaEventRecord(ev_fork[li], s), "event");
            ck(cudaStreamWaitEvent(sb, ev_fork[li], 0), "wait");
            ck(cudaStreamWaitEvent(sq, ev_fork[li], 0), "wait");
        }
        const int32_t* n_dev = B.n_dev;
        enqueue_biomes(W, B, sb, nmax, false);
        // the zoom tables and the quart biome output need only the chunk list and the biomes
        run_body<body_zoom_table, kZoomVerts>(K_ZOOM_TABLE, W, sb, kZoomVerts * nmax, B, n_dev);
        run_body<body_zoom_uniform, kZoomCells>(K_ZOOM_UNIFORM, W, sb, kZoomCells * nmax, B, n_dev);
        run_body<body_gather, kQuartsPerChunk>(K_GATHER, W, sb, static_cast<long>(kQuartsPerChunk) * nmax, B, n_dev);
        if (side) ck(cudaEventRecord(ev_join[li], sb), "event");
        mark(1);
        run_body<body_cc_insert, 25>(K_CC_INSERT, W, s, 25 * nmax, B, n_dev);
        launch(k_number<1, cc_key, 25>, s, 25 * nmax, B);
        run_body<body_cc_resolve, 25>(K_CC_RESOLVE, W, s, 25 * nmax, B, n_dev);
        if (TB_AXIS_TABLE && tbm::kAxisLayers > 0) {
            const int32_t* cnt_a = W.tb_a.count.as<int32_t>();
            run_body<body_axis_insert, 2>(K_AXIS_INSERT, W, s, 2 * 16 * nmax, B, cnt_c);
            run_body<body_axis_number, 2>(K_AXIS_NUMBER, W, s, 2 * 16 * nmax, B, cnt_c);
            run_body<body_axis_fill, std::max(1, tbm::kAxisLayers)>(K_AXIS_FILL, W, s, 2L * nmax * std::max(1, tbm::kAxisLayers), B, cnt_a);
        }
        run_body<body_corner_col, 1>(K_CORNER_COL, W, s, 16 * nmax, B, cnt_c);
        mark(8);
        run_body<body_corner, kRows, TB_MINB_CORNER>(K_CORNER, W, s, 16 * nmax * kRows, B, cnt_c);
        mark(9);
        mark(2);
        run_body<body_sg_insert, kGrid>(K_SG_INSERT, W, sq, kGrid * nmax, B, n_dev);
        launch(k_number<2, sg_key_item, kGrid>, sq, kGrid * nmax, B);
        run_body<body_sg_resolve, kGrid>(K_SG_RESOLVE, W, sq, kGrid * nmax, B, n_dev);
        run_body<body_surface_level, 1>(K_SURFACE_LEVEL, W, sq, 2 * nmax * 100, B, cnt_s);
        run_body<body_aquifer_cell, kAqCells>(K_AQ_CELL, W, sq, kAqCells * nmax, B, n_dev);
        run_body<body_aquifer_query, kAqQueries>(K_AQ_QUERY, W, sq, kAqQueries * nmax, B, n_dev);
        run_body<body_aquifer_skip, 1>(K_AQ_SKIP, W, sq, nmax, B, n_dev);
        if (side) ck(cudaEventRecord(ev_join_aq[li], sq), "event");
        mark(3);
        run_body<body_init_heights, 256>(K_INIT_HEIGHTS, W, s, 256 * nmax, B, n_dev);
        if (side) ck(cudaStreamWaitEvent(s, ev_join_aq[li], 0), "wait");
        run_body<body_fill, 256 * kCellsY, TB_MINB_FILL>(K_FILL, W, s, 256L * kCellsY * nmax, B, n_dev);
        if (aquifer_dev)
            ck(cudaMemcpyAsync(aquifer_dev, B.blocks, sizeof(uint16_t) * static_cast<size_t>(max_batch) * kBlocksPerChunk, cudaMemcpyDeviceToDevice, s),
               "d2d");
        mark(4);
        if (side) ck(cudaStreamWaitEvent(s, ev_join[li], 0), "wait");
        run_body<body_surface1, 256>(K_SURFACE1, W, s, 256 * nmax, B, n_dev);
        run_body<body_block_biome, 256>(K_BLOCK_BIOME, W, s, 256L * nmax, B, n_dev);
        mark(6);
        run_body<body_surface_walk_rules, 256, TB_MINB_WALK>(K_WALK, W, s, 256 * nmax, B, n_dev);
        if (W.defer_cap > 0) run_body<body_walk_deferred, 1>(K_WALK_DEFER, W, s, W.defer_cap, B, W.d_defer_count.as<int32_t>());
        mark(7);
        run_body<body_surface_frozen, 256>(K_FROZEN, W, s, 256 * nmax, B, n_dev);
        mark(5);
        prof_now = false;
    }

    // per-kernel times of the last timed batch into prof_ms (after its events completed)
    void collect_kernel_times() {
        for (int i = 0; i < K_COUNT; ++i)
            if (prof_marked[i]) {
                float ms = 0.0f;
                ck(cudaEventSynchronize(prof_ev[2 * i + 1]), "sync");
                ck(cudaEventElapsedTime(&ms, prof_ev[2 * i], prof_ev[2 * i + 1]), "elapsed");
                prof_ms[i] += ms;
                ++prof_calls[i];
                prof_marked[i] = false;
            }
    }

    // a new launch table: graphs and (for a new table load) the batch buffers are rebuilt
    void set_launch_table(const LaunchTable& t) {
        finish();
        const bool realloc = t.table_load != lt.table_load || t.defer_per_chunk != lt.defer_per_chunk;
        lt = t;
        for (auto& o : out)
            if (o.graph) {
                cudaGraphExecDestroy(o.graph);
                o.graph = nullptr;
            }
        destroy_queue_graphs();
        graph_launches = 0;
        if (realloc) alloc_batch(max_batch);
    }

    void add_stage_times(tg_timing* t) {
        ck(cudaEventSynchronize(ev[5]), "sync");
        float ms[5];
        for (int i = 0; i < 5; ++i) ck(cudaEventElapsedTime(&ms[i], ev[i], ev[i + 1]), "elapsed");
        t->biome_ms += ms[0];
        t->noise_ms += ms[1];
        t->aquifer_ms += ms[2];
        t->fill_ms += ms[3];
        t->surface_ms += ms[4];
        t->kernel_ms += ms[0] + ms[1] + ms[2] + ms[3] + ms[4];
        float rules = 0.0f;
        ck(cudaEventElapsedTime(&rules, ev[6], ev[7]), "elapsed");
        t->walk_rules_ms += rules;
        float corner = 0.0f;
        ck(cudaEventElapsedTime(&corner, ev[8], ev[9]), "elapsed");
        t->corner_ms += corner;
        collect_kernel_times();
        t->batches += 1;
    }

    // the staged coordinates of o (cx | cz | seed slot | n) into lane W's batch buffers
    // (one copy: the lane's coordinate buffer has the staging layout)
    void upload_coords(const Work& W, const OutSlot& o, int n, cudaStream_t s) {
        (void)n;
        ck(cudaMemcpyAsync(W.d_coords.p, o.coords.p, 4 * (3 * static_cast<size_t>(max_batch) + 1), cudaMemcpyHostToDevice, s), "h2d");
    }

    // Runs one batch into output slot o: its chunks from dev_chunks (n entries of a device
    // chunk list, current seed) or, when that is null, the staged coordinates in o.coords.
    // narrow: also write u8 copies of the blocks (and aquifer blocks) for the u8 output form.
    void run_batch(OutSlot& o, int n, tg_timing* t, bool want_aquifer, bool narrow = false, const tg_chunk_xz* dev_chunks = nullptr) {
        Work& W = work[o.lane];
        cudaStream_t s = o.lane ? lane_stream : stream;
        if (o.busy) ck(cudaStreamWaitEvent(s, o.drained, 0), "wait");   // the slot's previous outputs are copied out
        // the lane's own buffers: ready while the other lane's batch still runs
        if (dev_chunks)
            launch(k_split_chunks, s, n, dev_chunks, n, static_cast<int32_t>(current_slot), W.d_cx.as<int32_t>(), W.d_cz.as<int32_t>(),
                   W.d_cs.as<int32_t>(), W.d_n.as<int32_t>());
        else
            upload_coords(W, o, n, s);
        reset_lane(W, s, true);
        // A batch that fills the GPU alone runs after the previous one rather than beside it,
        // so each finishes (and its copy starts) as early as possible; smaller ones overlap.
        OutSlot& other = out[&o == &out[0] ? 1 : 0];
        if (lanes > 1 && n >= kOrderedBatch && other.lane != o.lane && other.busy) ck(cudaStreamWaitEvent(s, other.computed, 0), "wait");
        if (want_aquifer && !o.aquifer.p) o.aquifer.alloc(sizeof(uint16_t) * static_cast<size_t>(max_batch) * kBlocksPerChunk);
        const Batch B = batch_view(W, &o);
        uint16_t* aq = want_aquifer ? o.aquifer.as<uint16_t>() : nullptr;
        if (t) {
            enqueue_batch(W, B, s, max_batch, aq, true, false);
            add_stage_times(t);
        } else if (use_graphs) {
            if (!o.graph || o.graph_aquifer != want_aquifer || o.graph_stream != s) {
                if (o.graph) cudaGraphExecDestroy(o.graph);
                o.graph = nullptr;
                cudaGraph_t g;
                ck(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "capture");
                const int before = g_launches;
                enqueue_batch(W, B, s, max_batch, aq, false, false);
                ck(cudaStreamEndCapture(s, &g), "capture");
                ck(cudaGraphInstantiate(&o.graph, g, 0), "graph instantiate");
                cudaGraphDestroy(g);
                graph_launches = g_launches - before;
                g_launches = before;
                o.graph_aquifer = want_aquifer;
                o.graph_stream = s;
            }
            ck(cudaGraphLaunch(o.graph, s), "graph launch");
            g_launches += graph_launches;
        } else {
            enqueue_batch(W, B, s, max_batch, aq, false, false);
        }
        if (narrow) {
            const size_t cap = static_cast<size_t>(max_batch) * kBlocksPerChunk;
            const long n8 = static_cast<long>(n) * (kBlocksPerChunk / 8);
            if (!o.blocks8.p) o.blocks8.alloc(cap);
            launch(k_narrow_u8, s, n8, o.blocks.as<uint4>(), o.blocks8.as<uint2>(), n8);
            if (want_aquifer) {
                if (!o.aquifer8.p) o.aquifer8.alloc(cap);
                launch(k_narrow_u8, s, n8, o.aquifer.as<uint4>(), o.aquifer8.as<uint2>(), n8);
            }
        }
        ck(cudaGetLastError(), "kernel launch");
        ck(cudaEventRecord(o.computed, s), "event");
    }

    void stage(OutSlot& o, int n, const int32_t* cx, const int32_t* cz, const int32_t* cs) {
        if (o.busy) ck(cudaEventSynchronize(o.computed), "sync");   // the slot's staged coordinates were consumed
        int32_t* h = o.coords.as<int32_t>();
        std::memcpy(h, cx, 4 * static_cast<size_t>(n));
        std::memcpy(h + max_batch, cz, 4 * static_cast<size_t>(n));
        std::memcpy(h + 2 * max_batch, cs, 4 * static_cast<size_t>(n));
        h[3 * max_batch] = n;
    }

    void check_chunks(const tg_chunk_xz* c, int n) {
        const int32_t lim = 1 << 23;
        for (int i = 0; i < n; ++i)
            if (c[i].x <= -lim || c[i].x >= lim || c[i].z <= -lim || c[i].z >= lim) throw Error(TG_ERR_RANGE, "chunk coordinate outside |c| < 2^23");
    }

    struct Piece {
        uint16_t* blocks;
        uint8_t* biomes;
        uint16_t* aquifer;
        int first, count;      // position in the batch
        uint8_t* blocks8 = nullptr;    // u8 output form: these replace blocks / aquifer
        uint8_t* aquifer8 = nullptr;
    };

    // copies of a computed batch to host buffers, on the copy stream
    void drain(OutSlot& o, const std::vector<Piece>& pieces) {
        ck(cudaStreamWaitEvent(copy_stream, o.computed, 0), "wait");
        for (const Piece& p : pieces) {
            if (p.blocks8)
                ck(cudaMemcpyAsync(p.blocks8, o.blocks8.as<uint8_t>() + static_cast<size_t>(p.first) * kBlocksPerChunk,
                                   static_cast<size_t>(p.count) * kBlocksPerChunk, cudaMemcpyDeviceToHost, copy_stream),
                   "d2h");
            else
                ck(cudaMemcpyAsync(p.blocks, o.blocks.as<uint16_t>() + static_cast<size_t>(p.first) * kBlocksPerChunk,
                                   sizeof(uint16_t) * p.count * kBlocksPerChunk, cudaMemcpyDeviceToHost, copy_stream),
                   "d2h");
            if (p.aquifer8)
                ck(cudaMemcpyAsync(p.aquifer8, o.aquifer8.as<uint8_t>() + static_cast<size_t>(p.first) * kBlocksPerChunk,
                                   static_cast<size_t>(p.count) * kBlocksPerChunk, cudaMemcpyDeviceToHost, copy_stream),
                   "d2h");
            if (p.biomes)
                ck(cudaMemcpyAsync(p.biomes, o.biomes.as<uint8_t>() + static_cast<size_t>(p.first) * kQuartsPerChunk,
                                   static_cast<size_t>(p.count) * kQuartsPerChunk, cudaMemcpyDeviceToHost, copy_stream),
                   "d2h");
            if (p.aquifer)
                ck(cudaMemcpyAsync(p.aquifer, o.aquifer.as<uint16_t>() + static_cast<size_t>(p.first) * kBlocksPerChunk,
                                   sizeof(uint16_t) * p.count * kBlocksPerChunk, cudaMemcpyDeviceToHost, copy_stream),
                   "d2h");
        }
        ck(cudaEventRecord(o.drained, copy_stream), "event");
        o.busy = true;
    }

    void finish() {
        for (auto& o : out)
            if (o.busy) {
                ck(cudaEventSynchronize(o.drained), "sync");
                o.busy = false;
            }
        ck(cudaStreamSynchronize(stream), "sync");
        ck(cudaStreamSynchronize(lane_stream), "sync");
        check_device_errors();
    }

    // The lanes' sticky device error words (kErrTableFull, kErrKeyMissing): any bit set is
    // an internal error of the work that ran (and stays reported until the generator is
    // destroyed). Called with no work in flight.
    void check_device_errors() {
        for (int l = 0; l < lanes; ++l) {
            uint32_t e = 0;
            ck(cudaMemcpy(&e, work[l].d_err.p, sizeof e, cudaMemcpyDeviceToHost), "d2h");
            if (e)
                throw Error(TG_ERR_INTERNAL, std::string("device error bits ") + std::to_string(e) +
                                                 ((e & kErrTableFull) ? " (a dedupe hash table was full)" : "") +
                                                 ((e & kErrKeyMissing) ? " (a dedupe key was missing at resolve)" : ""));
        }
    }

    // lane 1's stream starts after the work already queued on `stream` (the caller's)
    void order_lanes() {
        if (lanes < 2) return;
        ck(cudaEventRecord(ev_entry, stream), "event");
        ck(cudaStreamWaitEvent(lane_stream, ev_entry, 0), "wait");
    }

    // The TERRAIN step with host outputs: u16 blocks (blocks, aquifer) or, with blocks8 set,
    // the reference generator's u8 form (blocks8, aquifer8).
    void generate(const tg_chunk_xz* chunks, int count, uint16_t* blocks, uint8_t* biomes, uint16_t* aquifer, tg_timing* t,
                  uint8_t* blocks8 = nullptr, uint8_t* aquifer8 = nullptr) {
        if (current_slot < 0) throw Error(TG_ERR_NO_SEED, "tg_set_seed has not been called");
        check_chunks(chunks, count);
        // The call's chunk list goes to the device once, ahead of lane 1's start; each batch
        // takes its part on its lane (k_split_chunks), so the host queues every batch without
        // waiting for earlier ones (the slots' events order the reuse of their buffers) and a
        // late host thread leaves no gap between batches.
        if (count > 0) {
            if (call_chunks.bytes < sizeof(tg_chunk_xz) * static_cast<size_t>(count)) call_chunks.alloc(sizeof(tg_chunk_xz) * static_cast<size_t>(count));
            ck(cudaMemcpyAsync(call_chunks.p, chunks, sizeof(tg_chunk_xz) * static_cast<size_t>(count), cudaMemcpyHostToDevice, stream), "h2d");
        }
        order_lanes();
        const HostSchedule& hs = lt.host[blocks8 ? 1 : 0];
        const int hb = hs.batch > 0 ? std::min(max_batch, hs.batch) : max_batch;
        int off = 0;
        for (const int n : host_schedule(count, hb, hs)) {
            OutSlot& o = out[next_out];
            next_out ^= 1;
            const bool narrow = blocks8 != nullptr;
            run_batch(o, n, t, narrow ? aquifer8 != nullptr : aquifer != nullptr, narrow, call_chunks.as<tg_chunk_xz>() + off);
            const size_t at = static_cast<size_t>(off) * kBlocksPerChunk;
            drain(o, {Piece{narrow ? nullptr : blocks + at, biomes ? biomes + static_cast<size_t>(off) * kQuartsPerChunk : nullptr,
                            (!narrow && aquifer) ? aquifer + at : nullptr, 0, n, narrow ? blocks8 + at : nullptr,
                            (narrow && aquifer8) ? aquifer8 + at : nullptr}});
            off += n;
        }
        finish();
    }

    // Region outputs for consumers: the region x region chunks from (x0, z0) for seed, row-major
    // by chunk ((cz - z0) * region + (cx - x0)), generated in u8 form a slab of chunk rows at a
    // time. dump_dir gets terrain.u8 (one u8 palette index per block, chunks back to back),
    // biomes.u8 (one u8 per quart) and meta.json; topdown_path gets the top-down map: "MCTD",
    // int32 {1, region, x0, z0, min_y}, then per block column (row-major over the region's
    // blocks) u8 top state, u8 floor state, u8 fluid depth (at most 255), u8 0, int16 top y,
    // int16 floor y, where top is the highest non-air block (y 0 of the column when all is
    // air) and floor the first non-fluid block at or below it.
    // reference: write_dump (bench/bench_main.cpp:170-187), write_topdown (:134-165); the dump's
    // reader is the client's GpuDump (client/src/main/java/mccuda/client/GpuDump.java:88-104).
    void write_region(int64_t seed, int x0, int z0, int region, const char* dump_dir, const char* topdown_path) {
        if (region <= 0 || region > 2048) throw Error(TG_ERR_INVALID_ARGUMENT, "region must be in [1, 2048] chunks");
        const int64_t lim = 1 << 23;
        if (x0 <= -lim || z0 <= -lim || static_cast<int64_t>(x0) + region - 1 >= lim || static_cast<int64_t>(z0) + region - 1 >= lim)
            throw Error(TG_ERR_RANGE, "region outside |c| < 2^23");
        current_slot = seed_slot(seed);
        if (!dump_dir) return topdown_on_device(x0, z0, region, topdown_path);
        const int rows_per_slab = std::max(1, std::min(region, 4096 / region));
        const size_t slab_chunks = static_cast<size_t>(rows_per_slab) * region;
        PinBuf blk, bio;
        blk.alloc(slab_chunks * kBlocksPerChunk);
        bio.alloc(slab_chunks * kQuartsPerChunk);
        std::ofstream ft, fb;
        if (dump_dir) {
            std::error_code ec;
            std::filesystem::create_directories(dump_dir, ec);
            ft.open(std::filesystem::path(dump_dir) / "terrain.u8", std::ios::binary);
            fb.open(std::filesystem::path(dump_dir) / "biomes.u8", std::ios::binary);
            if (!ft || !fb) throw Error(TG_ERR_IO, std::string("cannot write the region dump in ") + dump_dir);
        }
        const size_t side = static_cast<size_t>(region) * 16;
        // top-down records go to the file a slab at a time (each slab's rows are contiguous in it)
        std::ofstream ftd;
        if (topdown_path) ftd = open_topdown_file(topdown_path, region, x0, z0);
        std::vector<uint8_t> rec(topdown_path ? static_cast<size_t>(rows_per_slab) * 16 * side * 8 : 0, 0);
        std::vector<tg_chunk_xz> chunks(slab_chunks);
        for (int r0 = 0; r0 < region; r0 += rows_per_slab) {
            const int rows = std::min(rows_per_slab, region - r0);
            const int n = rows * region;
            for (int r = 0; r < rows; ++r)
                for (int i = 0; i < region; ++i) chunks[static_cast<size_t>(r) * region + i] = tg_chunk_xz{x0 + i, z0 + r0 + r};
            generate(chunks.data(), n, nullptr, bio.as<uint8_t>(), nullptr, nullptr, blk.as<uint8_t>(), nullptr);
            if (dump_dir) {
                ft.write(blk.as<const char>(), static_cast<std::streamsize>(static_cast<size_t>(n) * kBlocksPerChunk));
                fb.write(bio.as<const char>(), static_cast<std::streamsize>(static_cast<size_t>(n) * kQuartsPerChunk));
                if (!ft || !fb) throw Error(TG_ERR_IO, std::string("cannot write the region dump in ") + dump_dir);
            }
            if (topdown_path) {
                topdown_records(blk.as<const uint8_t>(), rows, region, side, rec.data());
                write_topdown_rows(ftd, topdown_path, rec.data(), static_cast<size_t>(rows) * 16 * side * 8);
            }
        }
        if (dump_dir) {
            ft.close();
            fb.close();
            std::ofstream m(std::filesystem::path(dump_dir) / "meta.json");
            m << "{\"seed\": " << seed << ", \"x0\": " << x0 << ", \"z0\": " << z0 << ", \"region\": " << region << ", \"height\": " << tbm::kHeight
              << ", \"min_y\": " << tbm::kMinY << ", \"chunk_bytes\": " << kBlocksPerChunk << ", \"biome_bytes\": " << kQuartsPerChunk << "}\n";
            if (!m || ft.fail() || fb.fail()) throw Error(TG_ERR_IO, std::string("cannot write the region dump in ") + dump_dir);
        }
        if (topdown_path) {
            ftd.close();
            if (ftd.fail()) throw Error(TG_ERR_IO, std::string("cannot write the top-down map ") + topdown_path);
        }
    }

    // The top-down map alone: each slab of chunk rows is generated into HBM in pieces of at
    // most max_batch chunks, each piece straight into the output slot that k_topdown reads
    // (stream order keeps the next piece from overwriting it before k_topdown has run), so
    // only the 8-byte records per block column cross the host link; the slab's records go to
    // the file once its copy has landed.
    void topdown_on_device(int x0, int z0, int region, const char* path) {
        const int rows_per_slab = std::max(1, std::min(region, 4096 / region));
        const size_t slab_chunks = static_cast<size_t>(rows_per_slab) * region;
        const size_t side = static_cast<size_t>(region) * 16;
        const int piece_max = std::min<int>(max_batch, static_cast<int>(slab_chunks));
        const size_t slab_bytes = static_cast<size_t>(rows_per_slab) * 16 * side * 8;
        std::vector<tg_chunk_xz> chunks(slab_chunks);
        DevBuf d_chunks, d_rec;
        PinBuf h_rec;
        d_chunks.alloc(sizeof(tg_chunk_xz) * slab_chunks);
        d_rec.alloc(slab_bytes);
        h_rec.alloc(slab_bytes);
        std::ofstream f = open_topdown_file(path, region, x0, z0);
        finish();
        OutSlot& o = out[0];
        Work& W = work[0];
        cudaStream_t s = stream;
        for (int r0 = 0; r0 < region; r0 += rows_per_slab) {
            const int rows = std::min(rows_per_slab, region - r0);
            const int n = rows * region;
            for (int r = 0; r < rows; ++r)
                for (int i = 0; i < region; ++i) chunks[static_cast<size_t>(r) * region + i] = tg_chunk_xz{x0 + i, z0 + r0 + r};
            check_chunks(chunks.data(), n);
            ck(cudaMemcpyAsync(d_chunks.p, chunks.data(), sizeof(tg_chunk_xz) * n, cudaMemcpyHostToDevice, s), "h2d");
            for (int first = 0; first < n; first += piece_max) {
                const int cnt = std::min(piece_max, n - first);
                launch(k_split_chunks, s, cnt, d_chunks.as<tg_chunk_xz>() + first, cnt, static_cast<int32_t>(current_slot), W.d_cx.as<int32_t>(),
                       W.d_cz.as<int32_t>(), W.d_cs.as<int32_t>(), W.d_n.as<int32_t>());
                enqueue_batch(W, batch_view(W, &o), s, max_batch, nullptr, false);
                launch(k_topdown, s, 256L * cnt, o.blocks.as<const uint16_t>(), model.block_flags, cnt, first, region, d_rec.as<uint2>());
                ck(cudaGetLastError(), "kernel launch");
            }
            const size_t bytes = static_cast<size_t>(rows) * 16 * side * 8;
            ck(cudaMemcpyAsync(h_rec.p, d_rec.p, bytes, cudaMemcpyDeviceToHost, s), "d2h");
            ck(cudaStreamSynchronize(s), "sync");
            write_topdown_rows(f, path, h_rec.as<uint8_t>(), bytes);
        }
        check_device_errors();
        f.close();
        if (f.fail()) throw Error(TG_ERR_IO, std::string("cannot write the top-down map ") + path);
    }

    static std::ofstream open_topdown_file(const char* path, int region, int x0, int z0) {
        std::ofstream f(path, std::ios::binary);
        const int32_t head[5] = {1, region, x0, z0, tbm::kMinY};
        f.write("MCTD", 4);
        f.write(reinterpret_cast<const char*>(head), sizeof head);
        if (!f) throw Error(TG_ERR_IO, std::string("cannot write the top-down map ") + path);
        return f;
    }

    static void write_topdown_rows(std::ofstream& f, const char* path, const uint8_t* rec, size_t bytes) {
        f.write(reinterpret_cast<const char*>(rec), static_cast<std::streamsize>(bytes));
        if (!f) throw Error(TG_ERR_IO, std::string("cannot write the top-down map ") + path);
    }

    // Top-down records of `rows` chunk rows of u8 blocks (row-major, region chunks per row)
    // into rec: the rows' block rows, side records each.
    static void topdown_records(const uint8_t* blocks, int rows, int region, size_t side, uint8_t* rec) {
        auto air = [](int st) { return (tbm::kBlockFlags[st] & 1) != 0; };
        auto fluid = [](int st) { return (tbm::kBlockFlags[st] & 8) != 0; };
        for (int r = 0; r < rows; ++r)
            for (int i = 0; i < region; ++i) {
                const uint8_t* b = blocks + (static_cast<size_t>(r) * region + i) * kBlocksPerChunk;
                const size_t rx = static_cast<size_t>(i) * 16, rz = static_cast<size_t>(r) * 16;
                for (int z = 0; z < 16; ++z)
                    for (int x = 0; x < 16; ++x) {
                        int y = tbm::kHeight - 1;
                        while (y > 0 && air(b[(y * 16 + z) * 16 + x])) --y;
                        const int top = b[(y * 16 + z) * 16 + x], top_y = y;
                        while (y > 0 && fluid(b[(y * 16 + z) * 16 + x])) --y;
                        uint8_t* o = rec + ((rz + z) * side + rx + x) * 8;
                        o[0] = static_cast<uint8_t>(top);
                        o[1] = b[(y * 16 + z) * 16 + x];
                        o[2] = static_cast<uint8_t>(std::min(255, top_y - y));
                        o[3] = 0;
                        const int16_t ty = static_cast<int16_t>(tbm::kMinY + top_y), fy = static_cast<int16_t>(tbm::kMinY + y);
                        std::memcpy(o + 4, &ty, 2);
                        std::memcpy(o + 6, &fy, 2);
                    }
            }
    }

    void generate_device(const tg_chunk_xz* chunks_dev, int count, uint16_t* blocks_dev, uint8_t* biomes_dev, tg_timing* t) {
        if (current_slot < 0) throw Error(TG_ERR_NO_SEED, "tg_set_seed has not been called");
        if (count > max_batch) throw Error(TG_ERR_INVALID_ARGUMENT, "count exceeds max_batch_chunks");
        finish();
        OutSlot& o = out[0];
        Work& W = work[0];
        cudaStream_t s = stream;
        launch(k_split_chunks, s, count, chunks_dev, count, static_cast<int32_t>(current_slot), W.d_cx.as<int32_t>(), W.d_cz.as<int32_t>(),
               W.d_cs.as<int32_t>(), W.d_n.as<int32_t>());
        // The kernels write the caller's buffers directly when they are 16-byte aligned (the
        // pipeline reads and writes them only within the count chunks); otherwise the
        // output slot's buffers and a device-to-device copy.
        const bool direct = reinterpret_cast<uintptr_t>(blocks_dev) % 16 == 0 && reinterpret_cast<uintptr_t>(biomes_dev) % 16 == 0;
        Batch B = batch_view(W, &o);
        if (direct) {
            B.blocks = blocks_dev;
            if (biomes_dev) B.biomes_out = biomes_dev;
        }
        enqueue_batch(W, B, s, max_batch, nullptr, t != nullptr);
        if (t) add_stage_times(t);
        if (!direct) {
            ck(cudaMemcpyAsync(blocks_dev, o.blocks.p, sizeof(uint16_t) * count * kBlocksPerChunk, cudaMemcpyDeviceToDevice, s), "d2d");
            if (biomes_dev) ck(cudaMemcpyAsync(biomes_dev, o.biomes.p, static_cast<size_t>(count) * kQuartsPerChunk, cudaMemcpyDeviceToDevice, s), "d2d");
        }
        ck(cudaGetLastError(), "kernel launch");
        ck(cudaStreamSynchronize(s), "sync");
        check_device_errors();
    }

    // Final density of every block (the value the fill tests with the aquifer), written by
    // the fill kernel into an extra buffer while the whole TERRAIN step runs as usual. The
    // chunks go in batches of at most min(max_batch, 1024); out is host memory of
    // count * kBlocksPerChunk floats in the block layout.
    DevBuf d_density;
    void generate_density(const tg_chunk_xz* chunks, int count, float* out_host) {
        if (current_slot < 0) throw Error(TG_ERR_NO_SEED, "tg_set_seed has not been called");
        check_chunks(chunks, count);
        if (count == 0) return;
        finish();
        const int piece = std::min(max_batch, 1024);
        const size_t bytes = sizeof(float) * static_cast<size_t>(piece) * kBlocksPerChunk;
        if (d_density.bytes < bytes) d_density.alloc(bytes);
        OutSlot& o = out[0];
        Work& W = work[0];
        cudaStream_t s = stream;
        std::vector<int32_t> cx(piece), cz(piece), cs(piece, current_slot);
        for (int off = 0; off < count; off += piece) {
            const int n = std::min(piece, count - off);
            for (int i = 0; i < n; ++i) {
                cx[i] = chunks[off + i].x;
                cz[i] = chunks[off + i].z;
            }
            stage(o, n, cx.data(), cz.data(), cs.data());
            upload_coords(W, o, n, s);
            Batch B = batch_view(W, &o);
            B.density = d_density.as<float>();
            enqueue_batch(W, B, s, max_batch, nullptr, false);
            ck(cudaGetLastError(), "kernel launch");
            ck(cudaMemcpyAsync(out_host + static_cast<size_t>(off) * kBlocksPerChunk, d_density.p, sizeof(float) * static_cast<size_t>(n) * kBlocksPerChunk,
                               cudaMemcpyDeviceToHost, s),
               "d2h");
            ck(cudaStreamSynchronize(s), "sync");
        }
        check_device_errors();
    }

    // Biome lookups at independent positions: one thread per position computes the zoomed
    // quart and its exact chain result on its own (biome_point), so scattered positions cost
    // one quart each instead of the 3x3 chunk neighbourhood. Positions go in sub-batches of
    // up to 2^20 whose distinct seeds fit the resident seed slots.
    void biome_lookup(const int64_t* seeds, const int32_t* xyz, int n, uint8_t* res) {
        const int cap = std::min(n, 1 << 20);
        if (cap <= 0) return;
        finish();
        // Two sub-batches in flight: while one runs on the GPU the host prepares the next
        // (positions checked and staged, slots assigned, new seeds built and installed).
        struct Sub {
            DevBuf xyz, slot, res, tied, ntied;
            PinBuf hxyz, hslot, hres;
            cudaEvent_t done = nullptr;
            std::vector<int> used;   // seed slots its kernels read
            int off = 0, m = 0;
            bool busy = false;
            ~Sub() {
                if (done) cudaEventDestroy(done);
            }
        };
        Sub sub[2];
        for (Sub& S : sub) {
            S.tied.alloc(sizeof(TiedLookup) * static_cast<size_t>(cap));
            S.ntied.alloc(sizeof(int32_t));
            S.xyz.alloc(sizeof(int32_t) * 3 * static_cast<size_t>(cap));
            S.slot.alloc(sizeof(int32_t) * static_cast<size_t>(cap));
            S.res.alloc(static_cast<size_t>(cap));
            S.hxyz.alloc(sizeof(int32_t) * 3 * static_cast<size_t>(cap));
            S.hslot.alloc(sizeof(int32_t) * static_cast<size_t>(cap));
            S.hres.alloc(static_cast<size_t>(cap));
            ck(cudaEventCreateWithFlags(&S.done, cudaEventDisableTiming), "event");
        }
        cudaStream_t s = stream;
        auto collect = [&](Sub& S) {
            ck(cudaEventSynchronize(S.done), "sync");
            std::memcpy(res + S.off, S.hres.p, static_cast<size_t>(S.m));
            S.busy = false;
        };
        try {
            int k = 0;
            for (int off = 0; off < n; k ^= 1) {
                Sub& S = sub[k];
                const Sub& P = sub[k ^ 1];   // in flight, if busy
                if (S.busy) collect(S);
                // The sub-batch: positions up to cap whose seeds fit the slots. Resident seeds
                // keep their slots; the new ones' host tables are built side by side on host
                // threads, then installed into slots neither this sub-batch nor the one in
                // flight reads (so no device sync is needed).
                std::vector<int> used;
                std::unordered_map<int64_t, int> seen;   // seed -> slot, or -1 - index into fresh
                std::vector<int64_t> fresh;
                int m = 0;
                bool have_prev = false;
                int64_t prev = 0;
                for (; m < cap && off + m < n; ++m) {
                    const int32_t* p = xyz + 3 * static_cast<size_t>(off + m);
                    const int32_t cx = p[0] >> 4, cz = p[2] >> 4;
                    if (cx <= -(1 << 23) || cx >= (1 << 23) || cz <= -(1 << 23) || cz >= (1 << 23)) throw Error(TG_ERR_RANGE, "position out of range");
                    const int64_t sd = seeds[off + m];
                    if (have_prev && sd == prev) continue;   // runs of one seed: no map lookup
                    have_prev = true;
                    prev = sd;
                    if (seen.count(sd)) continue;
                    if (static_cast<int>(seen.size()) == kMaxSlots / 2) break;   // the two sub-batches' slots stay disjoint
                    const int sl = resident_slot(sd);
                    if (sl >= 0) {
                        used.push_back(sl);
                        seen.emplace(sd, sl);
                    } else {
                        seen.emplace(sd, -1 - static_cast<int>(fresh.size()));
                        fresh.push_back(sd);
                    }
                }
                if (!fresh.empty()) {
                    std::vector<SeedHost> built(fresh.size());
                    const int nt = static_cast<int>(std::min<size_t>(fresh.size(), std::max(1u, std::min(16u, std::thread::hardware_concurrency()))));
                    std::vector<std::thread> pool;
                    for (int w = 0; w < nt; ++w)
                        pool.emplace_back([&, w] {
                            for (size_t i = w; i < fresh.size(); i += nt) build_seed_host(fresh[i], built[i]);
                        });
                    for (auto& th : pool) th.join();
                    std::vector<int> keep = used;
                    if (P.busy) keep.insert(keep.end(), P.used.begin(), P.used.end());
                    for (size_t i = 0; i < fresh.size(); ++i) {
                        const int sl = install_seed(fresh[i], built[i], keep, /*sync=*/false);
                        keep.push_back(sl);
                        used.push_back(sl);
                        seen[fresh[i]] = sl;
                    }
                }
                int32_t* slot_of = S.hslot.as<int32_t>();
                for (int i = 0; i < m; ++i) {
                    const int64_t sd = seeds[off + i];
                    slot_of[i] = (i > 0 && sd == seeds[off + i - 1]) ? slot_of[i - 1] : seen[sd];
                }
                std::memcpy(S.hxyz.p, xyz + 3 * static_cast<size_t>(off), sizeof(int32_t) * 3 * static_cast<size_t>(m));
                ck(cudaMemcpyAsync(S.xyz.p, S.hxyz.p, sizeof(int32_t) * 3 * static_cast<size_t>(m), cudaMemcpyHostToDevice, s), "h2d");
                ck(cudaMemcpyAsync(S.slot.p, S.hslot.p, sizeof(int32_t) * static_cast<size_t>(m), cudaMemcpyHostToDevice, s), "h2d");
                ck(cudaMemsetAsync(S.ntied.p, 0, sizeof(int32_t), s), "memset");
                launch(k_biome_point1, s, m, model, d_seeds.as<DevSeed>(), S.slot.as<int32_t>(), S.xyz.as<int32_t>(), m, S.res.as<uint8_t>(),
                       S.tied.as<TiedLookup>(), S.ntied.as<int32_t>());
                launch(k_biome_tied, s, 32L * m, model, d_seeds.as<DevSeed>(), S.slot.as<int32_t>(), S.tied.as<TiedLookup>(), S.ntied.as<int32_t>(),
                       S.res.as<uint8_t>());
                ck(cudaGetLastError(), "kernel launch");
                ck(cudaMemcpyAsync(S.hres.p, S.res.p, static_cast<size_t>(m), cudaMemcpyDeviceToHost, s), "d2h");
                ck(cudaEventRecord(S.done, s), "event");
                S.used = std::move(used);
                S.off = off;
                S.m = m;
                S.busy = true;
                off += m;
            }
            for (Sub& S : sub)
                if (S.busy) collect(S);   // the last two sub-batches
        } catch (...) {
            cudaStreamSynchronize(s);   // nothing in flight may outlive the buffers
            throw;
        }
    }

    // Biome lookups for the current seed that allocate nothing: positions and results pass
    // through the fixed scratch array (g_noalloc_scratch), the chunk list through the
    // generator's own pinned staging and batch buffers, built at tg_create.
    void biome_lookup_noalloc(const int32_t* xyz, int n, uint8_t* res) {
        if (current_slot < 0) throw Error(TG_ERR_NO_SEED, "tg_set_seed has not been called");
        const int cap = std::min(kNoAllocMaxLookups, max_batch);
        if (n > cap)
            throw Error(TG_ERR_INVALID_ARGUMENT, "n = " + std::to_string(n) + " exceeds the no-allocation lookup limit of " + std::to_string(cap) +
                                                     " positions (4,096 per call, and at most max_batch_chunks)");
        for (int i = 0; i < n; ++i) {
            const int32_t cx = xyz[3 * i] >> 4, cz = xyz[3 * i + 2] >> 4;
            if (cx <= -(1 << 23) || cx >= (1 << 23) || cz <= -(1 << 23) || cz >= (1 << 23)) throw Error(TG_ERR_RANGE, "position out of range");
        }
        if (n == 0) return;
        unsigned char* scratch = noalloc_scratch(device);
        finish();
        int32_t* h = out[0].coords.as<int32_t>();
        for (int i = 0; i < n; ++i) {
            h[i] = xyz[3 * i] >> 4;
            h[max_batch + i] = xyz[3 * i + 2] >> 4;
            h[2 * max_batch + i] = current_slot;
        }
        h[3 * max_batch] = n;
        cudaStream_t s = stream;
        Work& W = work[0];
        ck(cudaMemsetAsync(scratch, 0, sizeof(unsigned int), s), "memset");   // the finished count starts at zero
        ck(cudaMemcpyAsync(W.d_cx.p, h, 4 * static_cast<size_t>(n), cudaMemcpyHostToDevice, s), "h2d");
        ck(cudaMemcpyAsync(W.d_cz.p, h + max_batch, 4 * static_cast<size_t>(n), cudaMemcpyHostToDevice, s), "h2d");
        ck(cudaMemcpyAsync(W.d_cs.p, h + 2 * max_batch, 4 * static_cast<size_t>(n), cudaMemcpyHostToDevice, s), "h2d");
        ck(cudaMemcpyAsync(W.d_n.p, h + 3 * max_batch, 4, cudaMemcpyHostToDevice, s), "h2d");
        ck(cudaMemcpyAsync(scratch + kNoAllocXyzOff, xyz, sizeof(int32_t) * 3 * static_cast<size_t>(n), cudaMemcpyHostToDevice, s), "h2d");
        const Batch B = batch_view(W, nullptr);
        enqueue_biomes(W, B, s, n);
        launch(k_biome_lookup_scratch, s, n, B, scratch);
        ck(cudaGetLastError(), "kernel launch");
        unsigned int finished = 0;
        ck(cudaMemcpyAsync(res, scratch + kNoAllocOutOff, static_cast<size_t>(n), cudaMemcpyDeviceToHost, s), "d2h");
        ck(cudaMemcpyAsync(&finished, scratch, sizeof finished, cudaMemcpyDeviceToHost, s), "d2h");
        ck(cudaStreamSynchronize(s), "sync");
        if (finished != static_cast<unsigned int>(n))
            throw Error(TG_ERR_INTERNAL, "no-allocation lookup finished " + std::to_string(finished) + " of " + std::to_string(n) + " positions");
    }

    // ---- device-resident multi-seed batch from a device work queue --------------------------------
    DevBuf q_req, q_cx, q_cz, q_cs, q_rq, q_ix, q_state;
    size_t q_item_cap = 0, q_req_cap = 0;
    PinBuf q_req_host;
    cudaGraphExec_t q_loop = nullptr, q_iter = nullptr;   // the WHILE-loop graph, one iteration's graph
    cudaStream_t q_stream = nullptr;

    QueueView queue_view(int n_req) const {
        return QueueView{q_req.as<QueueReq>(), q_cx.as<int32_t>(), q_cz.as<int32_t>(), q_cs.as<int32_t>(), q_rq.as<int32_t>(), q_ix.as<int32_t>(),
                         q_state.as<int32_t>(), n_req};
    }

    // one queue iteration: take, TERRAIN step on lane 0 into out[0], scatter, advance
    void enqueue_queue_iteration(cudaStream_t s, cudaGraphConditionalHandle h, bool looped) {
        Work& W = work[0];
        const QueueView Q = queue_view(0);
        launch(k_queue_take, s, max_batch, Q, max_batch, W.d_cx.as<int32_t>(), W.d_cz.as<int32_t>(), W.d_cs.as<int32_t>(), W.d_n.as<int32_t>());
        const Batch B = batch_view(W, &out[0]);
        // one stream: the iteration is captured into a conditional node's body graph
        enqueue_batch(W, B, s, max_batch, nullptr, false, true, false);
        launch(k_queue_scatter, s, static_cast<long>(max_batch) * (kScatterBlockVecs + kScatterBiomeVecs), Q, out[0].blocks.as<const uint4>(),
               out[0].biomes.as<const uint4>());
        k_queue_advance<<<1, 1, 0, s>>>(Q, h, looped ? 1 : 0);
        ++g_launches;
    }

    void destroy_queue_graphs() {
        if (q_loop) cudaGraphExecDestroy(q_loop);
        if (q_iter) cudaGraphExecDestroy(q_iter);
        q_loop = q_iter = nullptr;
    }

    // Builds the graphs of the queue form once per set of queue buffers and stream: a WHILE
    // node whose body is one iteration (device loop), and one iteration alone (host loop).
    void build_queue_graphs(cudaStream_t s) {
        if (q_loop && q_iter && q_stream == s) return;
        destroy_queue_graphs();
        const int before = g_launches;
        cudaGraph_t g;
        ck(cudaGraphCreate(&g, 0), "graph create");
        cudaGraphConditionalHandle h;
        ck(cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault), "conditional handle");
        cudaGraphNodeParams p{};
        p.type = cudaGraphNodeTypeConditional;
        p.conditional.handle = h;
        p.conditional.type = cudaGraphCondTypeWhile;
        p.conditional.size = 1;
        cudaGraphNode_t node;
        ck(cudaGraphAddNode(&node, g, nullptr, 0, &p), "conditional node");
        cudaGraph_t body = p.conditional.phGraph_out[0];
        ck(cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal), "capture");
        enqueue_queue_iteration(s, h, true);
        ck(cudaStreamEndCapture(s, &body), "capture");
        ck(cudaGraphInstantiate(&q_loop, g, 0), "graph instantiate");
        cudaGraphDestroy(g);
        cudaGraph_t gi;
        ck(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "capture");
        enqueue_queue_iteration(s, cudaGraphConditionalHandle{}, false);
        ck(cudaStreamEndCapture(s, &gi), "capture");
        ck(cudaGraphInstantiate(&q_iter, gi, 0), "graph instantiate");
        cudaGraphDestroy(gi);
        g_launches = before;
        q_stream = s;
    }

    // The multi-seed TERRAIN step with every request's chunks and outputs in HBM. The requests
    // go into a device work queue; with host_loop false one graph launch runs batch after
    // batch on the device until the queue is empty, with host_loop true the host launches one
    // graph per batch (the same kernels). Requests whose distinct seeds exceed the resident
    // slots go in groups, one launch per group.
    void generate_batch_device(const tg_request_device* req, int n, bool host_loop, tg_timing* t) {
        for (int r = 0; r < n; ++r) {
            const tg_request_device& q = req[r];
            if (q.count < 0 || (q.count > 0 && (!q.chunks || !q.blocks_out))) throw Error(TG_ERR_INVALID_ARGUMENT, "bad request");
            if ((reinterpret_cast<uintptr_t>(q.blocks_out) | reinterpret_cast<uintptr_t>(q.biomes_out)) & 15u)
                throw Error(TG_ERR_INVALID_ARGUMENT, "request outputs must be 16-byte aligned");
        }
        finish();
        cudaStream_t s = stream;
        for (int r0 = 0; r0 < n;) {
            // a group: consecutive requests with at most kMaxSlots / 2 distinct seeds
            std::vector<int64_t> seeds;
            int r1 = r0;
            for (; r1 < n; ++r1) {
                if (std::find(seeds.begin(), seeds.end(), req[r1].seed) == seeds.end()) {
                    if (static_cast<int>(seeds.size()) == kMaxSlots / 2) break;
                    seeds.push_back(req[r1].seed);
                }
            }
            std::vector<int> keep;
            std::vector<QueueReq> qr;
            int64_t total = 0;
            for (int r = r0; r < r1; ++r) {
                if (req[r].count == 0) continue;
                const int slot = seed_slot(req[r].seed, keep);
                if (std::find(keep.begin(), keep.end(), slot) == keep.end()) keep.push_back(slot);
                qr.push_back(QueueReq{req[r].chunks, req[r].blocks_out, req[r].biomes_out, static_cast<int32_t>(total), req[r].count, slot, 0});
                total += req[r].count;
            }
            r0 = r1;
            if (total == 0) continue;
            if (total > INT32_MAX / 2) throw Error(TG_ERR_INVALID_ARGUMENT, "too many chunks in one batch call");
            // queue buffers (graphs hold their addresses: rebuilt when they grow)
            if (static_cast<size_t>(total) > q_item_cap || qr.size() > q_req_cap) {
                destroy_queue_graphs();
                q_item_cap = std::max<size_t>(static_cast<size_t>(total), q_item_cap);
                q_req_cap = std::max<size_t>(qr.size(), q_req_cap);
                for (DevBuf* b : {&q_cx, &q_cz, &q_cs, &q_rq, &q_ix}) b->alloc(sizeof(int32_t) * q_item_cap);
                q_req.alloc(sizeof(QueueReq) * q_req_cap);
                q_req_host.alloc(sizeof(QueueReq) * q_req_cap + 64);
            }
            if (!q_state.p) q_state.alloc(sizeof(int32_t) * 8);
            const int iters = static_cast<int>((total + max_batch - 1) / max_batch);
            int32_t* hs = reinterpret_cast<int32_t*>(q_req_host.as<uint8_t>() + sizeof(QueueReq) * q_req_cap);
            hs[0] = 0;
            hs[1] = static_cast<int32_t>(total);
            hs[2] = 0;
            hs[3] = iters + 1;
            hs[4] = 0;
            std::memcpy(q_req_host.p, qr.data(), sizeof(QueueReq) * qr.size());
            ck(cudaMemcpyAsync(q_req.p, q_req_host.p, sizeof(QueueReq) * qr.size(), cudaMemcpyHostToDevice, s), "h2d");
            ck(cudaMemcpyAsync(q_state.p, hs, sizeof(int32_t) * 5, cudaMemcpyHostToDevice, s), "h2d");
            launch(k_queue_fill, s, total, queue_view(static_cast<int>(qr.size())));
            if (t) {
                // timed: the host loop with stage events between the kernels
                for (int k = 0; k < iters; ++k) {
                    Work& W = work[0];
                    const QueueView Q = queue_view(0);
                    launch(k_queue_take, s, max_batch, Q, max_batch, W.d_cx.as<int32_t>(), W.d_cz.as<int32_t>(), W.d_cs.as<int32_t>(),
                           W.d_n.as<int32_t>());
                    enqueue_batch(W, batch_view(W, &out[0]), s, max_batch, nullptr, true);
                    add_stage_times(t);
                    launch(k_queue_scatter, s, static_cast<long>(max_batch) * (kScatterBlockVecs + kScatterBiomeVecs), Q,
                           out[0].blocks.as<const uint4>(), out[0].biomes.as<const uint4>());
                    k_queue_advance<<<1, 1, 0, s>>>(Q, cudaGraphConditionalHandle{}, 0);
                    ++g_launches;
                }
            } else {
                build_queue_graphs(s);
                if (host_loop) {
                    for (int k = 0; k < iters; ++k) ck(cudaGraphLaunch(q_iter, s), "graph launch");
                } else {
                    ck(cudaGraphLaunch(q_loop, s), "graph launch");
                }
                g_launches += iters * (graph_launches_per_batch() + 3);
            }
            ck(cudaGetLastError(), "kernel launch");
            int32_t done[5];
            ck(cudaMemcpyAsync(done, q_state.p, sizeof done, cudaMemcpyDeviceToHost, s), "d2h");
            ck(cudaStreamSynchronize(s), "sync");
            check_device_errors();
            if (done[0] != total) throw Error(TG_ERR_INTERNAL, "device work queue ended at item " + std::to_string(done[0]) + " of " + std::to_string(total));
        }
    }

    // kernels of one batch (as enqueued by enqueue_batch without the aquifer copy)
    int graph_launches_per_batch() {
        if (!graph_launches) {
            const int before = g_launches;
            g_launches = 0;
            // count by enqueueing into a throwaway capture
            cudaGraph_t g;
            ck(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "capture");
            enqueue_batch(work[0], batch_view(work[0], &out[0]), stream, max_batch, nullptr, false);
            ck(cudaStreamEndCapture(stream, &g), "capture");
            cudaGraphDestroy(g);
            graph_launches = g_launches;
            g_launches = before;
        }
        return graph_launches;
    }

    // Multi-seed batch: requests are cut into device batches; a batch mixes seeds.
    void generate_batch(const tg_request* req, int n, tg_timing* t) {
        order_lanes();
        for (int r = 0; r < n; ++r) {
            if (req[r].count < 0 || (req[r].count > 0 && (!req[r].chunks || !req[r].blocks_out))) throw Error(TG_ERR_INVALID_ARGUMENT, "bad request");
            check_chunks(req[r].chunks, req[r].count);
        }
        std::vector<int32_t> cx, cz, cs;
        std::vector<Piece> pieces;
        std::vector<int> used;
        auto flush = [&]() {
            const int m = static_cast<int>(cx.size());
            if (!m) return;
            OutSlot& o = out[next_out];
            next_out ^= 1;
            stage(o, m, cx.data(), cz.data(), cs.data());
            run_batch(o, m, t, false);
            drain(o, pieces);
            cx.clear();
            cz.clear();
            cs.clear();
            pieces.clear();
            used.clear();
        };
        for (int r = 0; r < n; ++r) {
            int done = 0;
            while (done < req[r].count) {
                if (static_cast<int>(cx.size()) == max_batch) flush();
                const int slot = seed_slot(req[r].seed, used);
                if (std::find(used.begin(), used.end(), slot) == used.end()) used.push_back(slot);
                const int take = std::min(req[r].count - done, max_batch - static_cast<int>(cx.size()));
                pieces.push_back(Piece{req[r].blocks_out + static_cast<size_t>(done) * kBlocksPerChunk,
                                       req[r].biomes_out ? req[r].biomes_out + static_cast<size_t>(done) * kQuartsPerChunk : nullptr, nullptr,
                                       static_cast<int>(cx.size()), take});
                for (int i = 0; i < take; ++i) {
                    cx.push_back(req[r].chunks[done + i].x);
                    cz.push_back(req[r].chunks[done + i].z);
                    cs.push_back(slot);
                }
                done += take;
            }
        }
        flush();
        finish();
    }
};

// ---- continuous-batching server ---------------------------------------------------------------------
// A worker thread owns the generator. Requests (seed, chunk list, host output buffers in the
// u16 or the u8 form) queue on submit; the worker admits them into an active set while the
// chunks in flight, priced at the device memory a chunk of batch capacity takes, stay within
// the HBM budget; it cuts device batches across all active requests (mixing seeds, request
// sizes and output forms) and drains each batch's outputs on the copy stream while the next
// batch computes. A request completes when its last chunk is copied out; a cancelled one
// when its chunks already in flight are (its remaining chunks are never issued).
struct Server {
    struct Req {
        uint64_t id = 0;
        int64_t seed = 0;
        std::vector<tg_chunk_xz> chunks;
        uint16_t* blocks = nullptr;
        uint8_t* blocks8 = nullptr;    // u8 form
        uint8_t* biomes = nullptr;
        int issued = 0, finished = 0;
        double t_submit = 0, t_done = 0;
        bool complete = false, cancelled = false;
        int slot = -1;
    };
    struct InFlight {
        int out = 0;
        std::vector<std::pair<Req*, int>> parts;   // request, chunks
    };

    Generator* g;
    int batch_chunks;
    long max_active_chunks;
    double device_bytes_per_chunk;
    std::thread worker;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Req*> queue;
    std::vector<Req*> active;
    std::unordered_map<uint64_t, std::unique_ptr<Req>> reqs;
    uint64_t next_id = 1;
    bool stop = false;
    tg_status failure = TG_OK;
    std::string failure_msg;
    // statistics
    std::vector<double> lat;
    long chunks_done = 0;
    double t_first = -1, t_last = 0;
    int batches = 0;
    int64_t cancelled = 0;
    bool unchecked = false;   // batches completed since the device error word was last read

    Server(Generator* gen, const tg_server_config* cfg) : g(gen) {
        batch_chunks = cfg && cfg->batch_chunks > 0 ? std::min(cfg->batch_chunks, g->max_batch) : g->max_batch;
        device_bytes_per_chunk = g->device_bytes_per_chunk();
        const long budget_chunks =
            cfg && cfg->hbm_budget_bytes > 0 ? static_cast<long>(static_cast<double>(cfg->hbm_budget_bytes) / device_bytes_per_chunk) : 8L * g->max_batch;
        max_active_chunks = std::max<long>(batch_chunks, budget_chunks);
        g->served = true;
        worker = std::thread([this] { run(); });
    }
    ~Server() {
        {
            std::lock_guard<std::mutex> l(mu);
            stop = true;
        }
        cv_work.notify_all();
        if (worker.joinable()) worker.join();
        g->served = false;
    }

    uint64_t submit(int64_t seed, const tg_chunk_xz* chunks, int count, uint16_t* blocks, uint8_t* blocks8, uint8_t* biomes) {
        g->check_chunks(chunks, count);
        auto r = std::make_unique<Req>();
        r->seed = seed;
        r->chunks.assign(chunks, chunks + count);
        r->blocks = blocks;
        r->blocks8 = blocks8;
        r->biomes = biomes;
        r->t_submit = now_ms();
        std::lock_guard<std::mutex> l(mu);
        if (failure != TG_OK) throw Error(failure, failure_msg);
        r->id = next_id++;
        const uint64_t id = r->id;
        if (t_first < 0) t_first = r->t_submit;
        if (count == 0) {
            r->complete = true;
            r->t_done = r->t_submit;
        } else {
            queue.push_back(r.get());
        }
        reqs.emplace(id, std::move(r));
        cv_work.notify_one();
        return id;
    }

    // A queued request is dropped at once; an active one issues no more chunks and completes
    // when its chunks in flight are copied out (its outputs then hold only those chunks).
    // Returns false when the request had already completed (its result stands).
    bool cancel(uint64_t id) {
        std::lock_guard<std::mutex> l(mu);
        auto it = reqs.find(id);
        if (it == reqs.end()) throw Error(TG_ERR_INVALID_ARGUMENT, "unknown ticket");
        Req* r = it->second.get();
        if (r->complete) return false;
        r->cancelled = true;
        ++cancelled;
        auto q = std::find(queue.begin(), queue.end(), r);
        if (q != queue.end()) {
            queue.erase(q);
            r->complete = true;
            r->t_done = now_ms();
            cv_done.notify_all();
        } else if (r->finished == r->issued) {
            // active with nothing in flight: done now
            auto a = std::find(active.begin(), active.end(), r);
            if (a != active.end()) active.erase(a);
            r->complete = true;
            r->t_done = now_ms();
            cv_done.notify_all();
        }
        cv_work.notify_one();
        return true;
    }

    // 1 = done (the ticket is released), 0 = pending; a cancelled request throws
    // TG_ERR_CANCELLED once done (and is released).
    int poll(uint64_t id, int wait_ms) {
        std::unique_lock<std::mutex> l(mu);
        auto it = reqs.find(id);
        if (it == reqs.end()) throw Error(TG_ERR_INVALID_ARGUMENT, "unknown ticket");
        Req* r = it->second.get();
        auto pred = [&] { return r->complete || failure != TG_OK; };
        if (wait_ms < 0) cv_done.wait(l, pred);
        else if (wait_ms > 0) cv_done.wait_for(l, std::chrono::milliseconds(wait_ms), pred);
        if (failure != TG_OK && !r->complete) throw Error(failure, failure_msg);
        if (!r->complete) return 0;
        const bool was_cancelled = r->cancelled;
        reqs.erase(it);
        if (was_cancelled) throw Error(TG_ERR_CANCELLED, "the request was cancelled");
        return 1;
    }

    void stats(tg_server_stats* s) {
        std::lock_guard<std::mutex> l(mu);
        std::memset(s, 0, sizeof *s);
        s->completed_requests = static_cast<int64_t>(lat.size());
        s->completed_chunks = chunks_done;
        s->batches = batches;
        if (!lat.empty()) {
            std::vector<double> v = lat;
            std::sort(v.begin(), v.end());
            auto pct = [&](double q) { return v[std::min(v.size() - 1, static_cast<size_t>(q * static_cast<double>(v.size() - 1) + 0.5))]; };
            s->p50_ms = pct(0.50);
            s->p99_ms = pct(0.99);
            s->max_ms = v.back();
            double sum = 0;
            for (double x : v) sum += x;
            s->mean_ms = sum / static_cast<double>(v.size());
        }
        if (t_first >= 0 && t_last > t_first) s->chunks_per_s = static_cast<double>(chunks_done) / ((t_last - t_first) / 1000.0);
        s->queued_requests = static_cast<int32_t>(queue.size());
        s->active_requests = static_cast<int32_t>(active.size());
        s->cancelled_requests = cancelled;
        s->device_bytes_per_chunk = device_bytes_per_chunk;
        s->max_active_chunks = max_active_chunks;
    }

    // latencies (submit -> last byte on the host) of the requests completed since the last
    // reset, in completion order
    int latencies(double* out, int cap) {
        std::lock_guard<std::mutex> l(mu);
        const int n = static_cast<int>(std::min<size_t>(lat.size(), static_cast<size_t>(cap)));
        if (out) std::copy(lat.begin(), lat.begin() + n, out);
        return static_cast<int>(lat.size());
    }

    void reset_stats() {
        std::lock_guard<std::mutex> l(mu);
        lat.clear();
        chunks_done = 0;
        t_first = -1;
        t_last = 0;
        batches = 0;
        cancelled = 0;
    }

    void complete_batch(InFlight& f) {
        ck(cudaEventSynchronize(g->out[f.out].drained), "sync");
        g->out[f.out].busy = false;
        unchecked = true;
        const double t = now_ms();
        std::lock_guard<std::mutex> l(mu);
        for (auto& part : f.parts) {
            Req* r = part.first;
            r->finished += part.second;
            chunks_done += part.second;
            const bool all = r->finished == static_cast<int>(r->chunks.size());
            if (all || (r->cancelled && r->finished == r->issued)) {
                r->complete = true;
                r->t_done = t;
                if (!r->cancelled) lat.push_back(t - r->t_submit);
                auto a = std::find(active.begin(), active.end(), r);
                if (a != active.end()) active.erase(a);
            }
        }
        t_last = t;
        ++batches;
        cv_done.notify_all();
    }

    void run() {
        try {
            ck(cudaSetDevice(g->device), "cudaSetDevice");
            std::deque<InFlight> flight;
            std::vector<int32_t> cx(g->max_batch), cz(g->max_batch), cs(g->max_batch);
            auto unissued = [&] {
                for (Req* r : active)
                    if (!r->cancelled && r->issued < static_cast<int>(r->chunks.size())) return true;
                return false;
            };
            for (;;) {
                // retire the batches whose copies have landed, without blocking
                while (!flight.empty()) {
                    const cudaError_t q = cudaEventQuery(g->out[flight.front().out].drained);
                    if (q == cudaErrorNotReady) break;
                    ck(q, "event query");
                    complete_batch(flight.front());
                    flight.pop_front();
                }
                // The device error word is read once the work in flight is done (a copy
                // beside the output copies would stall the worker behind them).
                if (flight.empty() && unchecked) {
                    g->check_device_errors();
                    unchecked = false;
                }
                std::vector<Req*> admitted;
                {
                    std::unique_lock<std::mutex> l(mu);
                    // idle until a request arrives; with batches in flight, wake every 100 us to
                    // retire them (a new request wakes the worker at once)
                    if (!stop && queue.empty() && !unissued()) {
                        if (flight.empty()) cv_work.wait(l, [&] { return stop || !queue.empty(); });
                        else cv_work.wait_for(l, std::chrono::microseconds(100), [&] { return stop || !queue.empty(); });
                    }
                    if (stop && flight.empty()) break;
                    // admission: chunks still to issue across the active set stay within the
                    // device-memory budget
                    long pending = 0;
                    for (Req* r : active)
                        if (!r->cancelled) pending += static_cast<long>(r->chunks.size()) - r->issued;
                    while (!queue.empty() && (active.empty() || pending + static_cast<long>(queue.front()->chunks.size()) <= max_active_chunks)) {
                        Req* r = queue.front();
                        queue.pop_front();
                        active.push_back(r);
                        admitted.push_back(r);
                        pending += static_cast<long>(r->chunks.size());
                    }
                }
                // per-seed tables stay resident; none is evicted while an active request uses it
                if (!admitted.empty()) {
                    std::vector<int> keep;
                    {
                        std::lock_guard<std::mutex> l(mu);
                        for (Req* r : active)
                            if (r->slot >= 0) keep.push_back(r->slot);
                    }
                    for (Req* r : admitted) {
                        const int slot = g->seed_slot(r->seed, keep);
                        keep.push_back(slot);
                        std::lock_guard<std::mutex> l(mu);
                        r->slot = slot;
                    }
                }
                // cut one batch across the active requests, oldest first
                InFlight f;
                int n = 0;
                bool narrow = false;
                std::vector<Generator::Piece> pieces;
                {
                    std::lock_guard<std::mutex> l(mu);
                    for (Req* r : active) {
                        if (n == batch_chunks) break;
                        const int left = static_cast<int>(r->chunks.size()) - r->issued;
                        if (left <= 0 || r->slot < 0 || r->cancelled) continue;
                        const int take = std::min(left, batch_chunks - n);
                        for (int i = 0; i < take; ++i) {
                            cx[n + i] = r->chunks[r->issued + i].x;
                            cz[n + i] = r->chunks[r->issued + i].z;
                            cs[n + i] = r->slot;
                        }
                        const size_t at = static_cast<size_t>(r->issued) * kBlocksPerChunk;
                        Generator::Piece pc{r->blocks ? r->blocks + at : nullptr, r->biomes ? r->biomes + static_cast<size_t>(r->issued) * kQuartsPerChunk : nullptr,
                                            nullptr, n, take};
                        if (r->blocks8) {
                            pc.blocks8 = r->blocks8 + at;
                            narrow = true;
                        }
                        pieces.push_back(pc);
                        f.parts.push_back({r, take});
                        r->issued += take;
                        n += take;
                    }
                }
                if (n > 0) {
                    const int oi = g->next_out;
                    g->next_out ^= 1;
                    OutSlot& o = g->out[oi];
                    if (o.busy) {
                        // the slot's previous batch completes before its buffers are reused
                        complete_batch(flight.front());
                        flight.pop_front();
                    }
                    g->stage(o, n, cx.data(), cz.data(), cs.data());
                    g->run_batch(o, n, nullptr, false, narrow);
                    g->drain(o, pieces);
                    f.out = oi;
                    flight.push_back(std::move(f));
                }
            }
        } catch (const Error& e) {
            std::lock_guard<std::mutex> l(mu);
            failure = e.code;
            failure_msg = e.what();
            cv_done.notify_all();
        } catch (const std::exception& e) {
            std::lock_guard<std::mutex> l(mu);
            failure = TG_ERR_INTERNAL;
            failure_msg = e.what();
            cv_done.notify_all();
        }
    }
};

// ---- live flythrough renderer -----------------------------------------------------------------------
// Flat block colours by name (sRGB), this renderer's own choice; palette entries match by
// the name before any state properties. Grass, podzol and mycelium show dirt on their sides
// under a capped top.
struct BlockColour {
    const char* name;
    uint8_t r, g, b;
};
const BlockColour kBlockColours[] = {
    {"minecraft:stone", 125, 125, 125},          {"minecraft:water", 40, 86, 170},            {"minecraft:lava", 220, 96, 20},
    {"minecraft:terracotta", 150, 93, 66},       {"minecraft:white_terracotta", 208, 176, 160}, {"minecraft:orange_terracotta", 160, 84, 38},
    {"minecraft:yellow_terracotta", 185, 131, 36}, {"minecraft:brown_terracotta", 77, 52, 36}, {"minecraft:red_terracotta", 142, 60, 46},
    {"minecraft:light_gray_terracotta", 134, 106, 97}, {"minecraft:packed_ice", 140, 178, 248}, {"minecraft:snow_block", 240, 245, 248},
    {"minecraft:bedrock", 58, 58, 58},           {"minecraft:deepslate", 78, 78, 82},         {"minecraft:grass_block", 90, 128, 56},
    {"minecraft:dirt", 133, 95, 66},             {"minecraft:sand", 218, 206, 160},           {"minecraft:sandstone", 214, 201, 152},
    {"minecraft:gravel", 130, 126, 125},         {"minecraft:red_sand", 189, 101, 34},        {"minecraft:coarse_dirt", 118, 84, 58},
    {"minecraft:podzol", 90, 62, 25},            {"minecraft:mycelium", 110, 98, 104},        {"minecraft:calcite", 222, 223, 219},
    {"minecraft:ice", 146, 182, 252},            {"minecraft:powder_snow", 247, 252, 252},    {"minecraft:mud", 61, 57, 60},
    {"minecraft:tuff", 107, 108, 101},           {"minecraft:granite", 148, 102, 85},         {"minecraft:copper_ore", 124, 124, 118},
    {"minecraft:raw_copper_block", 153, 104, 78}, {"minecraft:iron_ore", 136, 129, 122},     {"minecraft:raw_iron_block", 165, 135, 106},
    {"minecraft:moss_block", 89, 110, 45},       {"minecraft:clay", 160, 166, 179},           {"minecraft:smooth_basalt", 72, 72, 78},
    {"minecraft:dripstone_block", 134, 107, 92}, {"minecraft:red_sandstone", 180, 97, 32},    {"minecraft:air", 0, 0, 0},
};

// The linear colour table of the compiled palette (a name missing from kBlockColours is grey).
ViewColours palette_colours() {
    static_assert(tbm::kPaletteSize <= kViewPalette, "palette larger than the renderer's colour table");
    ViewColours c{};
    auto lin = [](uint8_t v) { return std::pow(static_cast<float>(v) / 255.0f, 2.2f); };
    auto find = [&](const std::string& n, float* out) {
        for (const BlockColour& b : kBlockColours)
            if (n == b.name) {
                out[0] = lin(b.r);
                out[1] = lin(b.g);
                out[2] = lin(b.b);
                return;
            }
        out[0] = out[1] = out[2] = lin(128);
    };
    for (int i = 0; i < tbm::kPaletteSize; ++i) {
        const std::string full = tbm::kPaletteNames[i];
        const std::string n = full.substr(0, full.find('['));
        find(n, c.top[i]);
        find(n, c.side[i]);
        if (n == "minecraft:grass_block" || n == "minecraft:podzol" || n == "minecraft:mycelium") {
            find("minecraft:dirt", c.side[i]);
            c.cap[i] = n == "minecraft:grass_block" ? 3 : 2;
        }
    }
    return c;
}

struct Viewer {
    Generator* g;
    int W, WB, WC, width, height;
    DevBuf vox, cells, d_slot, d_born, d_coords, d_chunks, d_frame, d_hits, d_colours;
    PinBuf h_frame;
    std::vector<int2> slot;
    std::vector<int32_t> born;
    cudaEvent_t e0 = nullptr, e1 = nullptr, e2 = nullptr;

    Viewer(Generator* gen, const tg_viewer_config* cfg) : g(gen) {
        W = cfg && cfg->window_chunks > 0 ? cfg->window_chunks : 64;
        width = cfg && cfg->width > 0 ? cfg->width : 1280;
        height = cfg && cfg->height > 0 ? cfg->height : 720;
        if (W < 4 || W > 256 || W % 4) throw Error(TG_ERR_INVALID_ARGUMENT, "window_chunks must be a multiple of 4 in 4..256");
        if (width > 8192 || height > 8192) throw Error(TG_ERR_INVALID_ARGUMENT, "frame larger than 8192 pixels on a side");
        WB = W * 16;
        WC = WB / kViewCell;
        const size_t plane = static_cast<size_t>(WB) * WB;
        vox.alloc(plane * tbm::kHeight);
        ck(cudaMemset(vox.p, tbm::kAir, vox.bytes), "memset");
        cells.alloc(sizeof(uint32_t) * WC * WC);
        ck(cudaMemset(cells.p, 0, cells.bytes), "memset");
        slot.assign(static_cast<size_t>(W) * W, make_int2(INT32_MIN, INT32_MIN));
        born.assign(static_cast<size_t>(W) * W, -1000000);
        d_slot.alloc(sizeof(int2) * slot.size());
        d_born.alloc(sizeof(int32_t) * born.size());
        ck(cudaMemcpy(d_slot.p, slot.data(), d_slot.bytes, cudaMemcpyHostToDevice), "h2d");
        ck(cudaMemcpy(d_born.p, born.data(), d_born.bytes, cudaMemcpyHostToDevice), "h2d");
        d_coords.alloc(sizeof(int2) * g->max_batch);
        d_chunks.alloc(sizeof(tg_chunk_xz) * g->max_batch);
        d_frame.alloc(static_cast<size_t>(width) * height * 3);
        d_hits.alloc(sizeof(int4) * static_cast<size_t>(width) * height);
        const ViewColours col = palette_colours();
        d_colours.alloc(sizeof col);
        ck(cudaMemcpy(d_colours.p, &col, sizeof col, cudaMemcpyHostToDevice), "h2d");
        for (cudaEvent_t* e : {&e0, &e1, &e2}) ck(cudaEventCreate(e), "event");
    }
    ~Viewer() {
        for (cudaEvent_t e : {e0, e1, e2})
            if (e) cudaEventDestroy(e);
    }

    ViewWorld world() const {
        return ViewWorld{vox.as<uint8_t>(), cells.as<uint32_t>(), d_slot.as<int2>(), d_born.as<int32_t>(), W, WB, WC, tbm::kAir, tbm::kWater, tbm::kLava,
                         tbm::kBedrock >= 0 ? tbm::kBedrock : tbm::kDefaultBlock};
    }
    int slot_of(int cx, int cz) const { return ((cz % W + W) % W) * W + ((cx % W + W) % W); }

    // The chunks within radius of chunk (ccx, ccz) that the window does not hold, nearest
    // first, at most cap (and max_batch) of them, generated on the device straight into the
    // window (the generator's batch, narrowed to u8 voxels at their slots, then the cells).
    int update(int ccx, int ccz, int radius, int cap, int frame, float* ms) {
        if (radius < 0 || 2 * radius + 2 > W) throw Error(TG_ERR_INVALID_ARGUMENT, "radius must be in 0 .. window_chunks / 2 - 1");
        if (g->current_slot < 0) throw Error(TG_ERR_NO_SEED, "tg_set_seed has not been called");
        std::vector<std::pair<int, tg_chunk_xz>> need;
        for (int dz = -radius; dz <= radius; ++dz)
            for (int dx = -radius; dx <= radius; ++dx) {
                if (dx * dx + dz * dz > radius * radius) continue;
                const int cx = ccx + dx, cz = ccz + dz;
                const int2 s = slot[slot_of(cx, cz)];
                if (s.x != cx || s.y != cz) need.push_back({dx * dx + dz * dz, tg_chunk_xz{cx, cz}});
            }
        std::stable_sort(need.begin(), need.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
        const int n = std::min<int>({static_cast<int>(need.size()), cap > 0 ? cap : g->max_batch, g->max_batch});
        if (ms) *ms = 0.0f;
        if (n == 0) return 0;
        std::vector<tg_chunk_xz> list(static_cast<size_t>(n));
        for (int i = 0; i < n; ++i) list[i] = need[i].second;
        g->check_chunks(list.data(), n);
        g->finish();
        cudaStream_t s = g->stream;
        Work& Wk = g->work[0];
        OutSlot& o = g->out[0];
        ck(cudaEventRecord(e0, s), "event");
        ck(cudaMemcpyAsync(d_chunks.p, list.data(), sizeof(tg_chunk_xz) * n, cudaMemcpyHostToDevice, s), "h2d");
        ck(cudaMemcpyAsync(d_coords.p, list.data(), sizeof(tg_chunk_xz) * n, cudaMemcpyHostToDevice, s), "h2d");
        launch(k_split_chunks, s, n, d_chunks.as<tg_chunk_xz>(), n, static_cast<int32_t>(g->current_slot), Wk.d_cx.as<int32_t>(), Wk.d_cz.as<int32_t>(),
               Wk.d_cs.as<int32_t>(), Wk.d_n.as<int32_t>());
        g->enqueue_batch(Wk, g->batch_view(Wk, &o), s, g->max_batch, nullptr, false);
        const ViewWorld w = world();
        launch(k_view_scatter, s, static_cast<long>(n) * tbm::kHeight * 32, w, o.blocks.as<const uint4>(), d_coords.as<const int2>(), n);
        launch(k_view_cells_clear, s, static_cast<long>(n) * 16, w, d_coords.as<const int2>(), n);
        launch(k_view_cells, s, static_cast<long>(n) * 256, w, d_coords.as<const int2>(), n);
        for (int i = 0; i < n; ++i) {
            const int k = slot_of(list[i].x, list[i].z);
            slot[k] = make_int2(list[i].x, list[i].z);
            born[k] = frame;
        }
        ck(cudaMemcpyAsync(d_slot.p, slot.data(), d_slot.bytes, cudaMemcpyHostToDevice, s), "h2d");
        ck(cudaMemcpyAsync(d_born.p, born.data(), d_born.bytes, cudaMemcpyHostToDevice, s), "h2d");
        ck(cudaEventRecord(e1, s), "event");
        ck(cudaGetLastError(), "kernel launch");
        ck(cudaStreamSynchronize(s), "sync");
        g->check_device_errors();
        if (ms) ck(cudaEventElapsedTime(ms, e0, e1), "elapsed");
        return n;
    }

    ViewCam camera(const tg_camera& c) const {
        ViewCam cam{};
        const double kPi = 3.14159265358979323846;
        const double yaw = c.yaw_deg * kPi / 180.0, pitch = c.pitch_deg * kPi / 180.0;
        cam.px = c.x;
        cam.py = c.y;
        cam.pz = c.z;
        cam.fx = static_cast<float>(std::sin(yaw) * std::cos(pitch));
        cam.fy = static_cast<float>(std::sin(pitch));
        cam.fz = static_cast<float>(std::cos(yaw) * std::cos(pitch));
        // right = forward x up, horizontal; up = right x forward
        const float rn = std::sqrt(cam.fz * cam.fz + cam.fx * cam.fx);
        cam.rx = -cam.fz / rn;
        cam.ry = 0.0f;
        cam.rz = cam.fx / rn;
        cam.ux = cam.ry * cam.fz - cam.rz * cam.fy;
        cam.uy = cam.rz * cam.fx - cam.rx * cam.fz;
        cam.uz = cam.rx * cam.fy - cam.ry * cam.fx;
        cam.tan_half = static_cast<float>(std::tan((c.fov_deg > 0.0f ? c.fov_deg : 70.0f) * kPi / 360.0));
        cam.aspect = static_cast<float>(width) / static_cast<float>(height);
        const float ln = std::sqrt(c.sun_x * c.sun_x + c.sun_y * c.sun_y + c.sun_z * c.sun_z);
        if (!(ln > 0.0f)) throw Error(TG_ERR_INVALID_ARGUMENT, "sun direction is zero");
        cam.lx = c.sun_x / ln;
        cam.ly = c.sun_y / ln;
        cam.lz = c.sun_z / ln;
        cam.fog = c.fog > 0.0f ? c.fog : static_cast<float>((W / 2 - 1) * 16);
        return cam;
    }

    void render(const tg_camera& c, int frame, uint8_t* rgb, int32_t* hits, float* ms) {
        const ViewCam cam = camera(c);
        g->finish();
        cudaStream_t s = g->stream;
        const dim3 blk(16, 8), grd((width + 15) / 16, (height + 7) / 8);
        ck(cudaEventRecord(e1, s), "event");
        k_view_render<<<grd, blk, 0, s>>>(world(), cam, d_colours.as<ViewColours>(), width, height, frame, d_frame.as<uint8_t>(), hits ? d_hits.as<int4>() : nullptr);
        ck(cudaEventRecord(e2, s), "event");
        ck(cudaGetLastError(), "kernel launch");
        if (rgb) ck(cudaMemcpyAsync(rgb, d_frame.p, static_cast<size_t>(width) * height * 3, cudaMemcpyDeviceToHost, s), "d2h");
        if (hits) ck(cudaMemcpyAsync(hits, d_hits.p, sizeof(int4) * static_cast<size_t>(width) * height, cudaMemcpyDeviceToHost, s), "d2h");
        ck(cudaStreamSynchronize(s), "sync");
        if (ms) ck(cudaEventElapsedTime(ms, e1, e2), "elapsed");
    }

    // The window's state for checks: voxels [y][z][x], cells, slots (x, z pairs), born frames.
    void state(uint8_t* v, uint32_t* cl, int32_t* sl, int32_t* bn) {
        g->finish();
        if (v) ck(cudaMemcpy(v, vox.p, vox.bytes, cudaMemcpyDeviceToHost), "d2h");
        if (cl) ck(cudaMemcpy(cl, cells.p, cells.bytes, cudaMemcpyDeviceToHost), "d2h");
        if (sl) std::memcpy(sl, slot.data(), sizeof(int2) * slot.size());
        if (bn) std::memcpy(bn, born.data(), sizeof(int32_t) * born.size());
    }
};

namespace {

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

}  // namespace
}  // namespace tb

struct tg_generator {
    std::unique_ptr<tb::Generator> g;
};

struct tg_server {
    std::unique_ptr<tb::Server> s;
};

struct tg_viewer {
    std::unique_ptr<tb::Viewer> v;
    tg_generator* gen;
};

namespace {
void usable(tg_generator* gen) {
    if (!gen) throw tb::Error(TG_ERR_INVALID_ARGUMENT, "gen is null");
    if (gen->g->served) throw tb::Error(TG_ERR_INVALID_ARGUMENT, "the generator is owned by a server");
    tb::ck(cudaSetDevice(gen->g->device), "cudaSetDevice");
}
}  // namespace

extern "C" {

tg_status tg_create(const char* ir_json_path, const char* terrain_json_path, const tg_config* config, tg_generator** out) {
    return tb::guarded([&] {
        if (!out) throw tb::Error(TG_ERR_INVALID_ARGUMENT, "out is null");
        *out = nullptr;
        if (ir_json_path && tb::sha256_hex(tb::read_file(ir_json_path)) != tbm::kModelIrSha256)
            throw tb::Error(TG_ERR_MODEL_MISMATCH, "IR file differs from the compiled model");
        if (terrain_json_path && tb::sha256_hex(tb::read_file(terrain_json_path)) != tbm::kModelTerrainSha256)
            throw tb::Error(TG_ERR_MODEL_MISMATCH, "terrain model file differs from the compiled model");
        const int batch = config && config->max_batch_chunks > 0 ? config->max_batch_chunks : 2048;
        if (batch > (1 << 16)) throw tb::Error(TG_ERR_INVALID_ARGUMENT, "max_batch_chunks too large");
        if (config && (config->pipeline_slots < 0 || config->pipeline_slots > 2)) throw tb::Error(TG_ERR_INVALID_ARGUMENT, "pipeline_slots must be 0, 1 or 2");
        const int dev = config ? config->device : 0;
        auto h = std::make_unique<tg_generator>();
        h->g = std::make_unique<tb::Generator>(dev, batch, config ? config->pipeline_slots : 0);
        *out = h.release();
    });
}

tg_status tg_destroy(tg_generator* gen) {
    return tb::guarded([&] {
        if (gen && gen->g->served) throw tb::Error(TG_ERR_INVALID_ARGUMENT, "destroy the server first");
        delete gen;
    });
}

tg_status tg_set_stream(tg_generator* gen, void* cuda_stream) {
    return tb::guarded([&] {
        usable(gen);
        gen->g->finish();
        gen->g->stream = cuda_stream ? static_cast<cudaStream_t>(cuda_stream) : gen->g->own_stream;
    });
}

tg_status tg_set_seed(tg_generator* gen, int64_t seed) {
    return tb::guarded([&] {
        usable(gen);
        gen->g->current_slot = gen->g->seed_slot(seed);
    });
}

tg_status tg_generate_u8(tg_generator* gen, const tg_chunk_xz* chunks, int32_t count, uint8_t* terrain_out, uint8_t* biomes_out, uint8_t* aquifer_out,
                         tg_timing* timing) {
    return tb::guarded([&] {
        usable(gen);
        if ((count > 0 && (!chunks || !terrain_out)) || count < 0) throw tb::Error(TG_ERR_INVALID_ARGUMENT, "bad argument");
        const auto t0 = std::chrono::steady_clock::now();
        if (timing) std::memset(timing, 0, sizeof *timing);
        tb::g_launches = 0;
        gen->g->generate(chunks, count, nullptr, biomes_out, nullptr, timing, terrain_out, aquifer_out);
        if (timing) {
            timing->launches = tb::g_launches;
            timing->wall_ms = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
        }
    });
}

tg_status tg_generate(tg_generator* gen, const tg_chunk_xz* chunks, int32_t count, uint16_t* blocks_out, uint8_t* biomes_out, uint16_t* aquifer_out,
                      tg_timing* timing) {
    return tb::guarded([&] {
        usable(gen);
        if ((count > 0 && (!chunks || !blocks_out)) || count < 0) throw tb::Error(TG_ERR_INVALID_ARGUMENT, "bad argument");
        const auto t0 = std::chrono::steady_clock::now();
        if (timing) std::memset(timing, 0, sizeof *timing);
        tb::g_launches = 0;
        gen->g->generate(chunks, count, blocks_out, biomes_out, aquifer_out, timing);
        if (timing) {
            timing->launches = tb::g_launches;
            timing->wall_ms = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
        }
    });
}

tg_status tg_generate_device(tg_generator* gen, const tg_chunk_xz* chunks_dev, int32_t count, uint16_t* blocks_dev, uint8_t* biomes_dev, tg_timing* timing) {
    return tb::guarded([&] {
        usable(gen);
        if (count <= 0 || !chunks_dev || !blocks_dev) throw tb::Error(TG_ERR_INVALID_ARGUMENT, "bad argument");
        if (timing) std::memset(timing, 0, sizeof *timing);
        tb::g_launches = 0;
        gen->g->generate_device(chunks_dev, count, blocks_dev, biomes_dev, timing);
        if (timing) timing->launches = tb::g_launches;
    });
}

tg_status tg_generate_density(tg_generator* gen, const tg_chunk_xz* chunks, int32_t count, float* density_out) {
    return tb::guarded([&] {
        usable(gen);
        if (count < 0 || (count > 0 && (!chunks || !density_out))) throw tb::Error(TG_ERR_INVALID_ARGUMENT, "bad argument");
        gen->g->generate_density(chunks, count, density_out);
    });
}

tg_status tg_generate_batch(tg_generator* gen, const tg_request* requests, int32_t n, tg_timing* timing) {
    return tb::guarded([&] {
        usable(gen);
        if (n < 0 || (n > 0 && !requests)) throw tb::Error(TG_ERR_INVALID_ARGUMENT, "bad argument");
        const auto t0 = std::chrono::steady_clock::now();
        if (timing) std::memset(timing, 0, sizeof *timing);
        tb::g_launches = 0;
        gen->g->generate_batch(requests, n, timing);
        if (timing) {
            timing->launches = tb::g_launches;
            timing->wall_ms = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
        }
    });
}

tg_status tg_generate_batch_device(tg_generator* gen, const tg_request_device* requests, int32_t n, int32_t flags, tg_timing* timing) {
    return tb::guarded([&] {
        usable(gen);
        if (n < 0 || (n > 0 && !requests) || (flags & ~TG_BATCH_HOST_LOOP)) throw tb::Error(TG_ERR_INVALID_ARGUMENT, "bad argument");
        const auto t0 = std::chrono::steady_clock::now();
        if (timing) std::memset(timing, 0, sizeof *timing);
        tb::g_launches = 0;
        gen->g->generate_batch_device(requests, n, (flags & TG_BATCH_HOST_LOOP) != 0, timing);
        if (timing) {
            timing->launches = tb::g_launches;
            timing->wall_ms = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
        }
    });
}

tg_status tg_biome_lookup(tg_generator* gen, const int64_t* seeds, const int32_t* xyz, int32_t n, uint8_t* out) {
    return tb::guarded([&] {
        usable(gen);
        if (n < 0 || (n > 0 && (!seeds || !xyz || !out))) throw tb::Error(TG_ERR_INVALID_ARGUMENT, "bad argument");
        gen->g->biome_lookup(seeds, xyz, n, out);
    });
}

tg_status tg_write_region(tg_generator* gen, int64_t seed, int32_t x0, int32_t z0, int32_t region, const char* dump_dir, const char* topdown_path) {
    return tb::guarded([&] {
        usable(gen);
        if (!dump_dir && !topdown_path) throw tb::Error(TG_ERR_INVALID_ARGUMENT, "nothing to write: dump_dir and topdown_path are both null");
        gen->g->write_region(seed, x0, z0, region, dump_dir, topdown_path);
    });
}

tg_status tg_biome_lookup_noalloc(tg_generator* gen, const int32_t* xyz, int32_t n, uint8_t* out) {
    return tb::guarded([&] {
        usable(gen);
        if (n < 0 || (n > 0 && (!xyz || !out))) throw tb::Error(TG_ERR_INVALID_ARGUMENT, "bad argument");
        gen->g->biome_lookup_noalloc(xyz, n, out);
    });
}

tg_status tg_viewer_create(tg_generator* gen, const tg_viewer_config* config, tg_viewer** out) {
    return tb::guarded([&] {
        usable(gen);
        if (!out) throw tb::Error(TG_ERR_INVALID_ARGUMENT, "out is null");
        *out = nullptr;
        auto h = std::make_unique<tg_viewer>();
        h->v = std::make_unique<tb::Viewer>(gen->g.get(), config);
        h->gen = gen;
        *out = h.release();
    });
}

tg_status tg_viewer_update(tg_viewer* viewer, int32_t cx, int32_t cz, int32_t radius, int32_t cap, int32_t frame, int32_t* generated, float* ms) {
    return tb::guarded([&] {
        if (!viewer) throw tb::Error(TG_ERR_INVALID_ARGUMENT, "viewer is null");
        usable(viewer->gen);
        const int n = viewer->v->update(cx, cz, radius, cap, frame, ms);
        if (generated) *generated = n;
    });
}

tg_status tg_viewer_render(tg_viewer* viewer, const tg_camera* camera, int32_t frame, uint8_t* rgb_out, int32_t* hits_out, float* ms) {
    return tb::guarded([&] {
        if (!viewer || !camera) throw tb::Error(TG_ERR_INVALID_ARGUMENT, "bad argument");
        usable(viewer->gen);
        viewer->v->render(*camera, frame, rgb_out, hits_out, ms);
    });
}

tg_status tg_viewer_state(tg_viewer* viewer, uint8_t* voxels, uint32_t* cells, int32_t* slots, int32_t* born) {
    return tb::guarded([&] {
        if (!viewer) throw tb::Error(TG_ERR_INVALID_ARGUMENT, "viewer is null");
        usable(viewer->gen);
        viewer->v->state(voxels, cells, slots, born);
    });
}

tg_status tg_viewer_params(tg_viewer* viewer, const tg_camera* camera, float* cam_out, float* top, float* side, int32_t* caps, int32_t* ids) {
    return tb::guarded([&] {
        if (!viewer || !camera) throw tb::Error(TG_ERR_INVALID_ARGUMENT, "bad argument");
        const tb::ViewCam c = viewer->v->camera(*camera);
        static_assert(sizeof(tb::ViewCam) == 18 * sizeof(float), "camera record of 18 floats");
        if (cam_out) std::memcpy(cam_out, &c, sizeof c);
        const tb::ViewColours col = tb::palette_colours();
        if (top) std::memcpy(top, col.top, sizeof col.top);
        if (side) std::memcpy(side, col.side, sizeof col.side);
        if (caps) std::memcpy(caps, col.cap, sizeof col.cap);
        if (ids) {
            const tb::ViewWorld w = viewer->v->world();
            const int32_t v[7] = {w.W, w.air, w.water, w.lava, w.bedrock, tbm::kMinY, tbm::kHeight};
            std::memcpy(ids, v, sizeof v);
        }
    });
}

tg_status tg_viewer_destroy(tg_viewer* viewer) {
    return tb::guarded([&] { delete viewer; });
}

tg_status tg_set_launch_table(tg_generator* gen, const char* text) {
    return tb::guarded([&] {
        usable(gen);
        gen->g->set_launch_table(tb::parse_launch_table(text ? std::string(text) : std::string(tb::kLaunchTableText)));
    });
}

tg_status tg_get_launch_table(tg_generator* gen, char* buf, size_t cap, size_t* needed) {
    return tb::guarded([&] {
        if (!gen) throw tb::Error(TG_ERR_INVALID_ARGUMENT, "gen is null");
        const std::string t = tb::format_launch_table(gen->g->lt);
        if (needed) *needed = t.size() + 1;
        if (buf && cap) {
            const size_t n = std::min(cap - 1, t.size());
            std::memcpy(buf, t.data(), n);
            buf[n] = 0;
        }
    });
}

tg_status tg_host_schedule(const char* text, int32_t u8, int32_t count, int32_t max_batch_chunks, int32_t* sizes, int32_t cap, int32_t* n) {
    return tb::guarded([&] {
        if (count < 0 || max_batch_chunks <= 0 || cap < 0 || (cap > 0 && !sizes)) throw tb::Error(TG_ERR_INVALID_ARGUMENT, "bad count, max_batch_chunks or buffer");
        const tb::LaunchTable t = tb::parse_launch_table(text ? std::string(text) : std::string(tb::kLaunchTableText));
        const tb::HostSchedule& hs = t.host[u8 ? 1 : 0];
        const int hb = hs.batch > 0 ? std::min(max_batch_chunks, hs.batch) : max_batch_chunks;
        const std::vector<int> v = tb::host_schedule(count, hb, hs);
        if (n) *n = static_cast<int32_t>(v.size());
        for (size_t i = 0; i < v.size() && static_cast<int32_t>(i) < cap; ++i) sizes[i] = v[i];
    });
}

tg_status tg_kernel_times(tg_generator* gen, int32_t enable, float* ms, int32_t* calls, int32_t cap) {
    return tb::guarded([&] {
        usable(gen);
        tb::Generator& g = *gen->g;
        for (int i = 0; i < std::min<int>(cap, tb::K_COUNT); ++i) {
            if (ms) ms[i] = static_cast<float>(g.prof_ms[i]);
            if (calls) calls[i] = g.prof_calls[i];
        }
        for (int i = 0; i < tb::K_COUNT; ++i) {
            g.prof_ms[i] = 0.0;
            g.prof_calls[i] = 0;
        }
        g.prof = enable != 0;
    });
}

tg_status tg_server_create(tg_generator* gen, const tg_server_config* config, tg_server** out) {
    return tb::guarded([&] {
        usable(gen);
        if (!out) throw tb::Error(TG_ERR_INVALID_ARGUMENT, "out is null");
        gen->g->finish();
        auto h = std::make_unique<tg_server>();
        h->s = std::make_unique<tb::Server>(gen->g.get(), config);
        *out = h.release();
    });
}

tg_status tg_server_submit(tg_server* srv, int64_t seed, const tg_chunk_xz* chunks, int32_t count, uint16_t* blocks_out, uint8_t* biomes_out,
                           uint64_t* ticket) {
    return tb::guarded([&] {
        if (!srv || !ticket || count < 0 || (count > 0 && (!chunks || !blocks_out))) throw tb::Error(TG_ERR_INVALID_ARGUMENT, "bad argument");
        *ticket = srv->s->submit(seed, chunks, count, blocks_out, nullptr, biomes_out);
    });
}

tg_status tg_server_submit_u8(tg_server* srv, int64_t seed, const tg_chunk_xz* chunks, int32_t count, uint8_t* terrain_out, uint8_t* biomes_out,
                              uint64_t* ticket) {
    return tb::guarded([&] {
        if (!srv || !ticket || count < 0 || (count > 0 && (!chunks || !terrain_out))) throw tb::Error(TG_ERR_INVALID_ARGUMENT, "bad argument");
        *ticket = srv->s->submit(seed, chunks, count, nullptr, terrain_out, biomes_out);
    });
}

tg_status tg_server_cancel(tg_server* srv, uint64_t ticket, int32_t* was_pending) {
    return tb::guarded([&] {
        if (!srv) throw tb::Error(TG_ERR_INVALID_ARGUMENT, "bad argument");
        const bool p = srv->s->cancel(ticket);
        if (was_pending) *was_pending = p ? 1 : 0;
    });
}

tg_status tg_server_latencies(tg_server* srv, double* ms, int32_t cap, int32_t* n) {
    return tb::guarded([&] {
        if (!srv || cap < 0 || (cap > 0 && !ms)) throw tb::Error(TG_ERR_INVALID_ARGUMENT, "bad argument");
        const int k = srv->s->latencies(ms, cap);
        if (n) *n = k;
    });
}

tg_status tg_server_wait(tg_server* srv, uint64_t ticket, int32_t timeout_ms, int32_t* done) {
    return tb::guarded([&] {
        if (!srv || !done) throw tb::Error(TG_ERR_INVALID_ARGUMENT, "bad argument");
        *done = 0;
        try {
            *done = srv->s->poll(ticket, timeout_ms);
        } catch (const tb::Error& e) {
            if (e.code == TG_ERR_CANCELLED) *done = 1;
            throw;
        }
    });
}

tg_status tg_server_get_stats(tg_server* srv, tg_server_stats* stats) {
    return tb::guarded([&] {
        if (!srv || !stats) throw tb::Error(TG_ERR_INVALID_ARGUMENT, "bad argument");
        srv->s->stats(stats);
    });
}

tg_status tg_server_reset_stats(tg_server* srv) {
    return tb::guarded([&] {
        if (!srv) throw tb::Error(TG_ERR_INVALID_ARGUMENT, "bad argument");
        srv->s->reset_stats();
    });
}

tg_status tg_server_destroy(tg_server* srv) {
    return tb::guarded([&] { delete srv; });
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
