// Host-side per-model and per-seed setup; see tb_host.h for the reference mapping.
#include "tb_host.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <functional>
#include <limits>
#include <stdexcept>

#include "model_gen.cuh"

namespace tb {

const int kYRows = tbm::kHeight / 8 + 1;

// ---- hashes -------------------------------------------------------------------------------
namespace {

uint32_t rol32(uint32_t v, int s) { return (v << s) | (v >> (32 - s)); }
uint32_t ror32(uint32_t v, int s) { return (v >> s) | (v << (32 - s)); }

// Padded message: data, 0x80, zeros, 64-bit length (little endian for MD5, big for SHA-2).
std::vector<uint8_t> md_pad(const uint8_t* data, size_t len, bool big_endian_length) {
    std::vector<uint8_t> m(data, data + len);
    m.push_back(0x80);
    while (m.size() % 64 != 56) m.push_back(0);
    const uint64_t bits = static_cast<uint64_t>(len) * 8u;
    for (int i = 0; i < 8; ++i) m.push_back(static_cast<uint8_t>(bits >> (big_endian_length ? 56 - 8 * i : 8 * i)));
    return m;
}

}  // namespace

void md5(const uint8_t* data, size_t len, uint8_t out[16]) {
    // RFC 1321: per-round shift amounts and the sine-derived constants floor(|sin(i+1)| * 2^32)
    static const int S[4][4] = {{7, 12, 17, 22}, {5, 9, 14, 20}, {4, 11, 16, 23}, {6, 10, 15, 21}};
    // a function-local static is built once even when seed tables are built on several threads
    struct Table {
        uint32_t v[64];
        Table() {
            for (int i = 0; i < 64; ++i) v[i] = static_cast<uint32_t>(std::floor(std::fabs(std::sin(static_cast<double>(i + 1))) * 4294967296.0));
        }
    };
    static const Table T;
    const uint32_t* K = T.v;
    uint32_t h[4] = {0x67452301u, 0xefcdab89u, 0x98badcfeu, 0x10325476u};
    const std::vector<uint8_t> m = md_pad(data, len, false);
    for (size_t blk = 0; blk < m.size(); blk += 64) {
        uint32_t w[16];
        for (int i = 0; i < 16; ++i) {
            const uint8_t* p = &m[blk + 4 * i];
            w[i] = p[0] | (p[1] << 8) | (p[2] << 16) | (static_cast<uint32_t>(p[3]) << 24);
        }
        uint32_t a = h[0], b = h[1], c = h[2], d = h[3];
        for (int i = 0; i < 64; ++i) {
            const int round = i / 16;
            uint32_t f;
            int g;
            switch (round) {
                case 0: f = (b & c) | (~b & d); g = i; break;
                case 1: f = (d & b) | (~d & c); g = (5 * i + 1) & 15; break;
                case 2: f = b ^ c ^ d; g = (3 * i + 5) & 15; break;
                default: f = c ^ (b | ~d); g = (7 * i) & 15; break;
            }
            const uint32_t nb = b + rol32(a + f + K[i] + w[g], S[round][i & 3]);
            a = d;
            d = c;
            c = b;
            b = nb;
        }
        h[0] += a;
        h[1] += b;
        h[2] += c;
        h[3] += d;
    }
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) out[4 * i + j] = static_cast<uint8_t>(h[i] >> (8 * j));
}

void sha256(const uint8_t* data, size_t len, uint8_t out[32]) {
    // FIPS 180-4: K = first 32 bits of the fractional parts of the cube roots of the
    // first 64 primes, H0 = the same for the square roots of the first 8 primes.
    struct Table {
        uint32_t K[64], H0[8];
        Table() {
            int primes[64], n = 0;
            for (int c = 2; n < 64; ++c) {
                bool p = true;
                for (int d = 2; d * d <= c; ++d)
                    if (c % d == 0) p = false;
                if (p) primes[n++] = c;
            }
            auto frac32 = [](long double v) {
                long double f = v - std::floor(v);
                return static_cast<uint32_t>(static_cast<uint64_t>(std::floor(f * 4294967296.0L)));
            };
            for (int i = 0; i < 64; ++i) {
                // long double cube root: 61 fraction bits, far more than the 32 kept; the MD5 /
                // SHA-256 known-answer tests pin every constant
                long double r = std::cbrt(static_cast<long double>(primes[i]));
                K[i] = frac32(r);
            }
            for (int i = 0; i < 8; ++i) H0[i] = frac32(std::sqrt(static_cast<long double>(primes[i])));
        }
    };
    static const Table T;   // built once, also when seed tables are built on several threads
    const uint32_t* K = T.K;
    uint32_t h[8];
    std::memcpy(h, T.H0, sizeof h);
    const std::vector<uint8_t> m = md_pad(data, len, true);
    for (size_t blk = 0; blk < m.size(); blk += 64) {
        uint32_t w[64];
        for (int i = 0; i < 16; ++i) {
            const uint8_t* p = &m[blk + 4 * i];
            w[i] = (static_cast<uint32_t>(p[0]) << 24) | (p[1] << 16) | (p[2] << 8) | p[3];
        }
        for (int i = 16; i < 64; ++i) {
            const uint32_t s0 = ror32(w[i - 15], 7) ^ ror32(w[i - 15], 18) ^ (w[i - 15] >> 3);
            const uint32_t s1 = ror32(w[i - 2], 17) ^ ror32(w[i - 2], 19) ^ (w[i - 2] >> 10);
            w[i] = w[i - 16] + s0 + w[i - 7] + s1;
        }
        uint32_t v[8];
        std::memcpy(v, h, sizeof v);
        for (int i = 0; i < 64; ++i) {
            const uint32_t S1 = ror32(v[4], 6) ^ ror32(v[4], 11) ^ ror32(v[4], 25);
            const uint32_t ch = (v[4] & v[5]) ^ (~v[4] & v[6]);
            const uint32_t t1 = v[7] + S1 + ch + K[i] + w[i];
            const uint32_t S0 = ror32(v[0], 2) ^ ror32(v[0], 13) ^ ror32(v[0], 22);
            const uint32_t mj = (v[0] & v[1]) ^ (v[0] & v[2]) ^ (v[1] & v[2]);
            for (int k = 7; k > 0; --k) v[k] = v[k - 1];
            v[4] += t1;
            v[0] = t1 + S0 + mj;
        }
        for (int k = 0; k < 8; ++k) h[k] += v[k];
    }
    for (int i = 0; i < 8; ++i)
        for (int j = 0; j < 4; ++j) out[4 * i + j] = static_cast<uint8_t>(h[i] >> (24 - 8 * j));
}

std::string sha256_hex(const std::string& text) {
    uint8_t d[32];
    sha256(reinterpret_cast<const uint8_t*>(text.data()), text.size(), d);
    static const char* hx = "0123456789abcdef";
    std::string s;
    for (uint8_t b : d) {
        s += hx[b >> 4];
        s += hx[b & 15];
    }
    return s;
}

// ---- random factories ----------------------------------------------------------------------
Xoro xoro_from_hash(const Positional& p, const std::string& name) {
    uint8_t h[16];
    md5(reinterpret_cast<const uint8_t*>(name.data()), name.size(), h);
    uint64_t lo = 0, hi = 0;
    for (int i = 0; i < 8; ++i) lo = (lo << 8) | h[i];
    for (int i = 8; i < 16; ++i) hi = (hi << 8) | h[i];
    return Xoro::raw(lo ^ p.lo, hi ^ p.hi);
}

Positional xoro_fork(Xoro& r) {
    const uint64_t lo = r.next();
    const uint64_t hi = r.next();
    return Positional{lo, hi};
}

double java_stream_sum(const std::vector<double>& v) {
    double sum = 0.0, comp = 0.0, plain = 0.0;
    for (double x : v) {
        const double y = x - comp;
        const double t = sum + y;
        comp = (t - sum) - y;
        sum = t;
        plain += x;
    }
    const double r = sum - comp;
    if (std::isnan(r) && std::isinf(plain)) return plain;
    return r;
}

// ---- java.util.Random (48-bit LCG) -----------------------------------------------------------
namespace {

struct Lcg {
    uint64_t s;
    explicit Lcg(int64_t seed) : s((static_cast<uint64_t>(seed) ^ 0x5DEECE66Dull) & ((1ull << 48) - 1)) {}
    int32_t bits(int n) {
        s = (s * 0x5DEECE66Dull + 0xBull) & ((1ull << 48) - 1);
        return static_cast<int32_t>(static_cast<int64_t>(s) >> (48 - n));
    }
    int32_t next_int(int32_t bound) {
        if ((bound & -bound) == bound) return static_cast<int32_t>((static_cast<int64_t>(bound) * bits(31)) >> 31);
        int32_t r, m;
        do {
            r = bits(31);
            m = r % bound;
        } while (static_cast<int32_t>(static_cast<uint32_t>(r) - static_cast<uint32_t>(m) + static_cast<uint32_t>(bound - 1)) < 0);
        return m;
    }
    double next_double() {
        const int64_t hi = bits(26), lo = bits(27);
        return static_cast<double>((hi << 27) + lo) * 0x1p-53;
    }
};

// SimplexNoise(random): three offset draws scaled by zero, then a Fisher-Yates permutation.
Simplex2 make_simplex(Lcg& r) {
    Simplex2 s{};
    s.ox = r.next_double() * 0.0;
    s.oy = r.next_double() * 0.0;
    (void)(r.next_double() * 0.0);
    for (int i = 0; i < 256; ++i) s.perm[i] = static_cast<uint8_t>(i);
    for (int i = 0; i < 256; ++i) {
        const int j = i + r.next_int(256 - i);
        std::swap(s.perm[i], s.perm[j]);
    }
    return s;
}

// GradientNoise(random, 256): offsets in [0, 256), then the shuffled permutation.
void make_octave(Xoro& r, double smear, SeedHost& s) {
    OctaveOff o;
    o.ox = r.next_double() * 256.0;
    o.oy = r.next_double() * 256.0;
    o.oz = r.next_double() * 256.0;
    o.smear = smear;
    uint8_t p[256];
    for (int i = 0; i < 256; ++i) p[i] = static_cast<uint8_t>(i);
    for (int i = 0; i < 256; ++i) {
        const int j = i + r.next_int(256 - i);
        std::swap(p[i], p[j]);
    }
    s.off.push_back(o);
    s.perm.insert(s.perm.end(), p, p + 256);
    for (int i = 0; i < 256; ++i) s.perm2.push_back(static_cast<uint16_t>(p[i] | (p[(i + 1) & 255] << 8)));
}

// NormalNoise(parameters).create(random): octave list, normalisation, two positional forks.
void normal_noise(const tbm::NoiseDef& d, Xoro random, SeedHost& s) {
    const bool normalize = d.normalize != 1;
    struct Oct {
        int index;
        double freq, amp;
    };
    std::vector<Oct> octs;
    double freq = std::ldexp(1.0, d.base_octave);
    double amp = d.base_amplitude;
    if (normalize) amp *= std::ldexp(1.0, d.octave_count - 1) / (std::ldexp(1.0, d.octave_count) - 1.0);
    for (int i = 0; i < d.octave_count; ++i) {
        const double mod = d.num_mods ? tbm::kNoiseMods[d.first_mod + i] : 1.0;
        if (mod != 0.0) octs.push_back({d.base_octave + i, freq, amp * mod});
        freq *= 2.0;
        amp *= 0.5;
    }
    std::vector<double> mags;
    double var = 0.0;
    for (const Oct& o : octs) {
        mags.push_back(std::fabs(o.amp));
        const double l = 0.2702247831245211 * std::fabs(o.amp);
        var += l * l;
    }
    const double target = java_stream_sum(mags);
    const double dev = std::sqrt(var);
    double norm = dev == 0.0 ? 0.0 : (target * 0.3333333333333333) / (dev * std::sqrt(2.0));
    if (d.normalize == 2 && norm != 0.0) {
        int lo = INT32_MAX, hi = INT32_MIN;
        for (int i = 0; i < d.octave_count; ++i) {
            const double mod = d.num_mods ? tbm::kNoiseMods[d.first_mod + i] : 1.0;
            if (mod != 0.0) {
                lo = std::min(lo, i);
                hi = std::max(hi, i);
            }
        }
        const double expected = 0.1 * (1.0 + 1.0 / (hi - lo + 1));
        norm = d.base_amplitude * 0.5 * 0.3333333333333333 / expected;
    }
    Positional first = xoro_fork(random);
    Positional second = xoro_fork(random);
    for (const Oct& o : octs) {
        const std::string key = "octave_" + std::to_string(o.index);
        Xoro r1 = xoro_from_hash(first, key);
        Xoro r2 = xoro_from_hash(second, key);
        const int32_t i1 = static_cast<int32_t>(s.off.size());
        make_octave(r1, 0.0, s);
        const int32_t i2 = static_cast<int32_t>(s.off.size());
        make_octave(r2, 0.0, s);
        const float vf = static_cast<float>(norm * o.amp);
        s.layers.push_back({o.freq, vf, i1});
        s.layers.push_back({o.freq * 1.0181268882175227, vf, i2});
    }
}

// BlendedNoise.createFbm: octaves from the coarsest layer, frequency halving and
// amplitude doubling per layer, value factor normalised by 2^n - 1.
void fbm(Xoro& r, int first_octave, double smear_y, double value_factor, SeedHost& s) {
    const int n = -first_octave + 1;
    double f = 1.0;
    value_factor /= std::ldexp(1.0, n) - 1.0;
    for (int i = n - 1; i >= 0; --i) {
        const int32_t idx = static_cast<int32_t>(s.off.size());
        make_octave(r, smear_y * f, s);
        s.layers.push_back({f, static_cast<float>(value_factor), idx});
        f /= 2.0;
        value_factor *= 2.0;
    }
}

}  // namespace

void build_seed_host(int64_t seed, SeedHost& s) {
    s = SeedHost{};
    s.seed = seed;
    Xoro base = Xoro::from_seed(seed);
    const Positional rnd = xoro_fork(base);
    s.random = rnd;
    for (int k = 0; k < tbm::kNumNoises; ++k) normal_noise(tbm::kNoiseDefs[k], xoro_from_hash(rnd, tbm::kNoiseKeys[k]), s);
    for (int b = 0; b < tbm::kNumBlended; ++b) {
        const tbm::BlendedDef& d = tbm::kBlended[b];
        Xoro r = xoro_from_hash(rnd, "minecraft:terrain");
        const double ymul = 684.412 * d.y_scale;
        const double limit_smear = ymul * d.smear_mult;
        const double main_smear = limit_smear / d.y_factor;
        const double limit_factor = static_cast<double>(0.99998474f);
        fbm(r, -15, limit_smear, limit_factor, s);
        fbm(r, -15, limit_smear, limit_factor, s);
        fbm(r, -7, main_smear, 12.75, s);
    }
    if (static_cast<int>(s.layers.size()) != tbm::kNumLayers || static_cast<int>(s.off.size()) != tbm::kNumOctaves)
        throw std::runtime_error("seed table layout differs from the generated layout");
    Xoro aq = xoro_from_hash(rnd, "minecraft:aquifer");
    s.aquifer = xoro_fork(aq);
    Xoro ore = xoro_from_hash(rnd, "minecraft:ore");
    s.ore = xoro_fork(ore);
    for (int k = 0; k < tbm::kNumGradientRandoms; ++k) {
        Xoro g = xoro_from_hash(rnd, tbm::kGradientRandomNames[k]);
        s.gradient.push_back(xoro_fork(g));
    }
    // BiomeManager.obfuscateSeed: SHA-256 of the seed's 8 little-endian bytes, first 8 bytes little endian.
    uint8_t in[8], d[32];
    for (int i = 0; i < 8; ++i) in[i] = static_cast<uint8_t>(static_cast<uint64_t>(seed) >> (8 * i));
    sha256(in, 8, d);
    uint64_t z = 0;
    for (int i = 7; i >= 0; --i) z = (z << 8) | d[i];
    s.zoom_seed = static_cast<int64_t>(z);
    // MaterialSystem clay bands
    Xoro r = xoro_from_hash(rnd, "minecraft:clay_bands");
    const int* T = tbm::kTerracotta;   // terracotta, white, orange, yellow, brown, red, light gray
    int bands[192];
    std::fill(bands, bands + 192, T[0]);
    for (int i = 0; i < 192; ++i) {
        i += r.next_int(5) + 1;
        if (i < 192) bands[i] = T[2];
    }
    auto layer = [&](int width, int state) {
        const int count = r.next_int(15 - 6 + 1) + 6;
        for (int i = 0; i < count; ++i) {
            const int w = width + r.next_int(3);
            const int start = r.next_int(192);
            for (int p = 0; start + p < 192 && p < w; ++p) bands[start + p] = state;
        }
    };
    layer(1, T[3]);
    layer(2, T[4]);
    layer(1, T[5]);
    const int whites = r.next_int(15 - 9 + 1) + 9;
    int placed = 0;
    for (int start = 0; placed < whites && start < 192; start += r.next_int(16) + 4) {
        bands[start] = T[1];
        if (start - 1 > 0 && r.next_bool()) bands[start - 1] = T[6];
        if (start + 1 < 192 && r.next_bool()) bands[start + 1] = T[6];
        ++placed;
    }
    for (int i = 0; i < 192; ++i) s.clay[i] = static_cast<uint16_t>(bands[i]);
    // the corner context's y records: row r (height min_y + 8 r) holds the record of each
    // entry of tbm::kYLayer, with the device's arithmetic (y_record)
    const NoiseTables nt{s.off.data(), s.perm.data(), s.layers.data(), s.perm2.data()};
    s.ytab.resize(static_cast<size_t>(kYRows) * tbm::kYLayers);
    for (int r = 0; r < kYRows; ++r)
        for (int e = 0; e < tbm::kYLayers; ++e)
            s.ytab[static_cast<size_t>(r) * tbm::kYLayers + e] = y_record(nt, tbm::kYLayer[e], tbm::kYScale[e], tbm::kYSmeared[e], tbm::kMinY + 8 * r);
}

// ---- climate R-tree (Climate.RTree build order) ------------------------------------------------
namespace {

struct TreeBuild {
    struct N {
        int64_t mn[7], mx[7];
        std::vector<int> kids;
        int leaf = -1;
    };
    std::vector<N> n;
    static int64_t center(int64_t a, int64_t b) { return (a + b) / 2; }
    static int64_t absl(int64_t v) { return v < 0 ? -v : v; }

    int subtree(const std::vector<int>& kids) {
        N t;
        for (int d = 0; d < 7; ++d) {
            t.mn[d] = n[kids[0]].mn[d];
            t.mx[d] = n[kids[0]].mx[d];
            for (size_t k = 1; k < kids.size(); ++k) {
                t.mn[d] = std::min(t.mn[d], n[kids[k]].mn[d]);
                t.mx[d] = std::max(t.mx[d], n[kids[k]].mx[d]);
            }
        }
        t.kids = kids;
        n.push_back(t);
        return static_cast<int>(n.size()) - 1;
    }

    // order by the center of dimension `dim`, ties broken by the following dimensions cyclically
    void sort_dim(std::vector<int>& v, int dim, bool absolute) {
        std::stable_sort(v.begin(), v.end(), [&](int a, int b) {
            for (int k = 0; k < 7; ++k) {
                const int d = (dim + k) % 7;
                int64_t ca = center(n[a].mn[d], n[a].mx[d]), cb = center(n[b].mn[d], n[b].mx[d]);
                if (absolute) {
                    ca = absl(ca);
                    cb = absl(cb);
                }
                if (ca != cb) return ca < cb;
            }
            return false;
        });
    }

    int build(std::vector<int> kids) {
        const int per = 19;
        if (kids.size() == 1) return kids[0];
        if (static_cast<int>(kids.size()) <= per) {
            std::stable_sort(kids.begin(), kids.end(), [&](int a, int b) {
                int64_t sa = 0, sb = 0;
                for (int d = 0; d < 7; ++d) {
                    sa += absl(center(n[a].mn[d], n[a].mx[d]));
                    sb += absl(center(n[b].mn[d], n[b].mx[d]));
                }
                return sa < sb;
            });
            return subtree(kids);
        }
        const double lg = std::floor(std::log(static_cast<double>(kids.size()) - 0.01) / std::log(static_cast<double>(per)));
        const int group = static_cast<int>(std::pow(static_cast<double>(per), lg));
        int64_t best_cost = INT64_MAX;
        int best_dim = -1;
        std::vector<std::vector<int>> best;
        for (int d = 0; d < 7; ++d) {
            sort_dim(kids, d, false);
            std::vector<std::vector<int>> buckets;
            for (size_t i = 0; i < kids.size(); i += static_cast<size_t>(group))
                buckets.emplace_back(kids.begin() + static_cast<long>(i), kids.begin() + static_cast<long>(std::min(kids.size(), i + group)));
            int64_t cost = 0;
            for (const auto& b : buckets)
                for (int dd = 0; dd < 7; ++dd) {
                    int64_t lo = n[b[0]].mn[dd], hi = n[b[0]].mx[dd];
                    for (size_t k = 1; k < b.size(); ++k) {
                        lo = std::min(lo, n[b[k]].mn[dd]);
                        hi = std::max(hi, n[b[k]].mx[dd]);
                    }
                    cost += absl(hi - lo);
                }
            if (cost < best_cost) {
                best_cost = cost;
                best_dim = d;
                best = buckets;
            }
        }
        std::vector<int> bnodes;
        for (const auto& b : best) bnodes.push_back(subtree(b));
        sort_dim(bnodes, best_dim, true);
        std::vector<int> built;
        for (int bn : bnodes) {
            std::vector<int> sub = n[bn].kids;
            built.push_back(build(sub));
        }
        return subtree(built);
    }
};

}  // namespace

void build_model_host(ModelHost& m) {
    m = ModelHost{};
    TreeBuild tb;
    std::vector<int> leaves;
    for (int i = 0; i < tbm::kNumParams; ++i) {
        TreeBuild::N leaf;
        for (int d = 0; d < 6; ++d) {
            leaf.mn[d] = tbm::kParams[i].p[2 * d];
            leaf.mx[d] = tbm::kParams[i].p[2 * d + 1];
        }
        leaf.mn[6] = leaf.mx[6] = tbm::kParams[i].offset;
        leaf.leaf = i;
        tb.n.push_back(leaf);
        leaves.push_back(i);
        m.leaf_biome.push_back(tbm::kParams[i].biome);
    }
    m.root = tb.build(leaves);
    // flatten, assigning each leaf its depth-first rank
    m.nodes.resize(tb.n.size());
    m.leaf_node.assign(tbm::kNumParams, -1);
    m.leaf_rank.assign(tbm::kNumParams, -1);
    for (size_t i = 0; i < tb.n.size(); ++i) {
        RNode& r = m.nodes[i];
        std::memcpy(r.mn, tb.n[i].mn, sizeof r.mn);
        std::memcpy(r.mx, tb.n[i].mx, sizeof r.mx);
        r.leaf = tb.n[i].leaf;
        r.first_child = static_cast<int32_t>(m.children.size());
        r.child_count = static_cast<int32_t>(tb.n[i].kids.size());
        for (int c : tb.n[i].kids) m.children.push_back(c);
        if (r.leaf >= 0) m.leaf_node[r.leaf] = static_cast<int32_t>(i);
    }
    int rank = 0;
    std::vector<char> reachable(m.nodes.size(), 0);
    std::function<int(int, int)> dfs = [&](int node, int depth) -> int {
        m.depth = std::max(m.depth, depth);
        reachable[node] = 1;
        RNode& r = m.nodes[node];
        r.rank = rank;
        if (r.leaf >= 0) {
            m.leaf_rank[r.leaf] = rank++;
            return r.rank;
        }
        for (int k = 0; k < r.child_count; ++k) dfs(m.children[r.first_child + k], depth + 1);
        return r.rank;
    };
    dfs(m.root, 1);
    if (rank != tbm::kNumParams) throw std::runtime_error("climate tree does not cover every parameter box");
    // (nodes the build made only to order its buckets are not part of the tree)
    bool fits = true;
    for (size_t i = 0; i < m.nodes.size(); ++i) {
        if (!reachable[i]) continue;
        const RNode& r = m.nodes[i];
        if (r.child_count >= 32) fits = false;
        for (int d = 0; d < 7; ++d)
            if (r.mn[d] > r.mx[d] || r.mn[d] < -kBox32Limit || r.mx[d] > kBox32Limit) fits = false;
    }
    if (fits) {
        // breadth first from the root, so that the children of a node are consecutive boxes
        std::vector<int> order{m.root};
        std::vector<int32_t> box_of(m.nodes.size(), -1);
        box_of[m.root] = 0;
        for (size_t h = 0; h < order.size(); ++h) {
            const RNode& r = m.nodes[order[h]];
            if (r.leaf >= 0) continue;
            for (int k = 0; k < r.child_count; ++k) {
                const int ch = m.children[r.first_child + k];
                box_of[ch] = static_cast<int32_t>(order.size());
                order.push_back(ch);
            }
        }
        m.boxes.resize(order.size());
        m.box_leaf.assign(tbm::kNumParams, -1);
        for (size_t i = 0; i < order.size(); ++i) {
            const RNode& r = m.nodes[order[i]];
            RBox& b = m.boxes[i];
            for (int d = 0; d < 7; ++d) {
                b.mn[d] = static_cast<int32_t>(r.mn[d]);
                b.mx[d] = static_cast<int32_t>(r.mx[d]);
            }
            if (r.leaf >= 0) {
                b.info = ~r.leaf;
                m.box_leaf[r.leaf] = static_cast<int32_t>(i);
            } else {
                b.info = (box_of[m.children[r.first_child]] << 5) | r.child_count;
            }
            b.rank = r.rank;
        }
    }
    // biome temperature simplex noises
    Lcg r1(1234);
    m.temp = make_simplex(r1);
    Lcg r3(3456);
    for (int i = 0; i < 3; ++i) m.frozen[i] = make_simplex(r3);
    m.frozen_amp[0] = 0.14285715f;
    m.frozen_amp[1] = 0.2857143f;
    m.frozen_amp[2] = 0.5714286f;
    Lcg r2(2345);
    m.info = make_simplex(r2);
    const double s3 = std::sqrt(3.0);
    m.f2 = 0.5 * (s3 - 1.0);
    m.g2 = (3.0 - s3) / 6.0;
}

}  // namespace tb
