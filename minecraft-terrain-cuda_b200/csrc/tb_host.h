// Host-side per-model and per-seed setup of the TERRAIN step.
//
// Per model (seed independent): the climate R-tree over the biome parameter list
// (reference cpu/src/biome.cpp:95-199) flattened with depth-first leaf ranks, and the
// legacy simplex permutations of biome temperature (cpu/src/terrain.cpp:70-80).
// Per seed: noise octave tables (cpu/src/seed_tables.cpp:159-184), positional random
// factories and clay bands (cpu/src/terrain.cpp:112-149), BiomeManager zoom seed
// (cpu/src/biome.cpp:61-70).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "tb_noise.cuh"
#include "tb_rng.cuh"

namespace tb {

void md5(const uint8_t* data, size_t len, uint8_t out[16]);
void sha256(const uint8_t* data, size_t len, uint8_t out[32]);
std::string sha256_hex(const std::string& text);

// XoroshiroPositionalRandomFactory seeded from MD5 of a name (fromHashOf).
Xoro xoro_from_hash(const Positional& p, const std::string& name);
// fork_positional: two longs from the stream.
Positional xoro_fork(Xoro& r);

// java.util.stream.DoubleStream.sum (compensated summation)
double java_stream_sum(const std::vector<double>& v);

struct RNode {                 // flattened R-tree node (device layout)
    int64_t mn[7], mx[7];
    int32_t first_child, child_count;
    int32_t leaf;              // parameter index for leaves, -1 otherwise
    int32_t rank;              // depth-first rank of the first leaf in the subtree
};

// The same node as 16 int32 (64 bytes), used when every box bound fits in +/-2^29. The
// boxes are stored breadth first from the root (box 0), the children of a node
// consecutive: info = ~leaf for leaves, (first child box << 5) | child_count otherwise.
struct alignas(16) RBox {
    int32_t mn[7], mx[7];
    int32_t info, rank;
};
constexpr int32_t kBox32Limit = 1 << 29;

struct ModelHost {
    std::vector<RNode> nodes;
    std::vector<RBox> boxes;       // empty unless every bound fits the 32-bit search
    std::vector<int32_t> box_leaf; // parameter index -> box index
    std::vector<int32_t> children;
    std::vector<int32_t> leaf_biome;   // per parameter index
    std::vector<int32_t> leaf_node;    // parameter index -> node index
    std::vector<int32_t> leaf_rank;    // parameter index -> depth-first rank
    int32_t root = -1;
    int32_t depth = 0;
    Simplex2 temp, frozen[3], info;
    float frozen_amp[3];
    double f2 = 0, g2 = 0;
};

struct SeedHost {
    int64_t seed = 0;
    std::vector<OctaveOff> off;
    std::vector<uint8_t> perm;
    std::vector<uint16_t> perm2;   // perm[i] | perm[(i + 1) & 255] << 8, per octave
    std::vector<Layer> layers;
    Positional random{}, aquifer{}, ore{};
    std::vector<Positional> gradient;
    int64_t zoom_seed = 0;
    uint16_t clay[192];
    // per corner row, the y coordinate record of every volume-stack layer of the corner
    // context (kYRows x tbm::kYLayers, row-major)
    std::vector<AxisRec> ytab;
};

// corner rows of a chunk column (one per 8 heights, both ends included)
extern const int kYRows;

void build_model_host(ModelHost& m);
void build_seed_host(int64_t seed, SeedHost& s);

}  // namespace tb
