// Counting build of the reference's C++ port (TEST AND MEASUREMENT INFRASTRUCTURE).
//
// oracle/Makefile compiles the reference's cpu/ sources a second time with GCC's
// -finstrument-functions, which calls __cyg_profile_func_enter / _exit around every
// function, inlined ones included, with that function's address. This file supplies
// those hooks and counts, per pipeline phase, how often the algorithm's units of work run:
//   units   perlin_volume, smeared_volume (one volume-path octave sample,
//           cpu/include/mccuda/noise_eval.h:163-178, :203-220), perlin_get, smeared_get (one
//           point-path octave sample, :115-124, :190), Simplex2D::get (cpu/src/terrain.cpp:46-68),
//           BiomeTree::distance (one R-tree node distance, cpu/src/biome.cpp:201-209),
//           fiddled_distance (one BiomeManager zoom corner, cpu/src/biome.cpp:255-268);
//   phases  biome (inside cpu_chunk_biomes), aquifer (inside the Aquifer class), surface
//           (inside the Surface class), corners (inside
//           VolumeEvaluator::sample_interpolated_block_step and none of the former: the
//           interpolated channels' cell corners of the final density), fill (the rest of
//           cpu_terrain_from_biomes: per-block density work outside the interpolation).
// The caller (oracle/count_ops.py) resolves the functions' offsets in the built library
// from its symbol table and passes them to ref_count_setup; counting runs only between
// ref_count_enable(1) and ref_count_enable(0). Nothing in the product links this.
#include <dlfcn.h>

#include <cstdint>
#include <cstring>
#include <mutex>
#include <vector>

namespace {

constexpr int kUnits = 7;
constexpr int kPhases = 5;           // 0 fill, 1 corners, 2 biome, 3 aquifer, 4 surface
constexpr int kMaxPhaseFns = 256;

uintptr_t g_base = 0;
uintptr_t g_unit[kUnits] = {};
uintptr_t g_phase_fn[kMaxPhaseFns] = {};
int g_phase_of[kMaxPhaseFns] = {};
int g_n_phase_fns = 0;
volatile int g_enabled = 0;

struct ThreadCounts {
    uint64_t n[kPhases][kUnits];
    int active[kPhases];
};
std::mutex g_mu;
std::vector<ThreadCounts*> g_threads;

__attribute__((no_instrument_function)) ThreadCounts* mine() {
    thread_local ThreadCounts* t = nullptr;
    if (!t) {
        t = new ThreadCounts();
        std::memset(t, 0, sizeof *t);
        std::lock_guard<std::mutex> l(g_mu);
        g_threads.push_back(t);
    }
    return t;
}

__attribute__((no_instrument_function)) int phase_now(const ThreadCounts* t) {
    if (t->active[2]) return 2;
    if (t->active[3]) return 3;
    if (t->active[4]) return 4;
    if (t->active[1]) return 1;
    return 0;
}

}  // namespace

extern "C" {

__attribute__((no_instrument_function)) void __cyg_profile_func_enter(void* fn, void*) {
    if (!g_enabled) return;
    const uintptr_t off = reinterpret_cast<uintptr_t>(fn) - g_base;
    ThreadCounts* t = mine();
    for (int i = 0; i < g_n_phase_fns; ++i)
        if (g_phase_fn[i] == off) ++t->active[g_phase_of[i]];
    for (int u = 0; u < kUnits; ++u)
        if (g_unit[u] == off) {
            ++t->n[phase_now(t)][u];
            break;
        }
}

__attribute__((no_instrument_function)) void __cyg_profile_func_exit(void* fn, void*) {
    if (!g_enabled) return;
    const uintptr_t off = reinterpret_cast<uintptr_t>(fn) - g_base;
    ThreadCounts* t = mine();
    for (int i = 0; i < g_n_phase_fns; ++i)
        if (g_phase_fn[i] == off && t->active[g_phase_of[i]] > 0) --t->active[g_phase_of[i]];
}

// unit_off: kUnits symbol offsets in this library (0 = not present); phase_off / phase_id:
// n functions whose activity defines a phase.
__attribute__((no_instrument_function)) int ref_count_setup(const uint64_t* unit_off, const uint64_t* phase_off, const int32_t* phase_id, int32_t n) {
    if (n > kMaxPhaseFns) return -1;
    Dl_info info{};
    if (!dladdr(reinterpret_cast<void*>(&ref_count_setup), &info)) return -2;
    g_base = reinterpret_cast<uintptr_t>(info.dli_fbase);
    for (int u = 0; u < kUnits; ++u) g_unit[u] = unit_off[u] ? static_cast<uintptr_t>(unit_off[u]) : ~static_cast<uintptr_t>(0);
    for (int i = 0; i < n; ++i) {
        g_phase_fn[i] = static_cast<uintptr_t>(phase_off[i]);
        g_phase_of[i] = phase_id[i];
    }
    g_n_phase_fns = n;
    return 0;
}

__attribute__((no_instrument_function)) void ref_count_enable(int32_t on) { g_enabled = on; }

// counts: kPhases * kUnits totals over every thread since the last reset
__attribute__((no_instrument_function)) void ref_count_read(uint64_t* counts, int32_t reset) {
    std::lock_guard<std::mutex> l(g_mu);
    std::memset(counts, 0, sizeof(uint64_t) * kPhases * kUnits);
    for (ThreadCounts* t : g_threads) {
        for (int p = 0; p < kPhases; ++p)
            for (int u = 0; u < kUnits; ++u) counts[p * kUnits + u] += t->n[p][u];
        if (reset) std::memset(t->n, 0, sizeof t->n);
    }
}

}  // extern "C"
