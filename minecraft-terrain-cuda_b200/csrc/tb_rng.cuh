// Random sources of the TERRAIN step (host + device):
//   Xoroshiro128++ with the positional factory (XoroshiroRandomSource,
//   cpu/src/rng.cpp:42-103), Mth.getSeed (cpu/src/rng.cpp:105-113), the
//   java.util.Random LCG (cpu/src/rng.cpp:115-156) and the BiomeManager fiddle LCG
//   (cpu/src/biome.cpp:241-268).
#pragma once

#include "tb_math.cuh"

namespace tb {

constexpr uint64_t kGolden64 = 0x9E3779B97F4A7C15ull;
constexpr uint64_t kSilver64 = 0x6A09E667F3BCC909ull;

TB_HD TB_FI uint64_t rotl64(uint64_t v, int k) { return (v << k) | (v >> (64 - k)); }

TB_HD TB_FI uint64_t stafford13(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// XoroshiroRandomSource; the all-zero state is replaced as the reference does.
struct Xoro {
    uint64_t lo, hi;
    TB_HD TB_FI static Xoro raw(uint64_t lo, uint64_t hi) {
        Xoro x{lo, hi};
        if ((lo | hi) == 0) {
            x.lo = kGolden64;
            x.hi = kSilver64;
        }
        return x;
    }
    // RandomSupport.upgradeSeedTo128bit
    TB_HD TB_FI static Xoro from_seed(int64_t seed) {
        uint64_t l = static_cast<uint64_t>(seed) ^ kSilver64;
        return raw(stafford13(l), stafford13(l + kGolden64));
    }
    TB_HD TB_FI uint64_t next() {
        const uint64_t s0 = lo;
        uint64_t s1 = hi;
        const uint64_t r = rotl64(s0 + s1, 17) + s0;
        s1 ^= s0;
        lo = rotl64(s0, 49) ^ s1 ^ (s1 << 21);
        hi = rotl64(s1, 28);
        return r;
    }
    // nextInt(bound): Lemire multiply-shift with rejection of the biased low part.
    TB_HD TB_FI int32_t next_int(int32_t bound) {
        const uint64_t ub = static_cast<uint32_t>(bound);
        uint64_t m = static_cast<uint64_t>(static_cast<uint32_t>(next())) * ub;
        if ((m & 0xFFFFFFFFull) < ub) {
            const uint32_t thresh = static_cast<uint32_t>(0u - static_cast<uint32_t>(bound)) % static_cast<uint32_t>(bound);
            while ((m & 0xFFFFFFFFull) < thresh) m = static_cast<uint64_t>(static_cast<uint32_t>(next())) * ub;
        }
        return static_cast<int32_t>(m >> 32);
    }
    // nextFloat: top 24 bits times 2^-24; nextDouble: top 53 bits times 2^-53.
    TB_HD TB_FI float next_float() { return static_cast<float>(static_cast<int64_t>(next() >> 40)) * 0x1p-24f; }
    TB_HD TB_FI double next_double() { return static_cast<double>(static_cast<int64_t>(next() >> 11)) * 0x1p-53; }
    TB_HD TB_FI bool next_bool() { return (next() & 1ull) != 0; }
};

// Mth.getSeed(x, y, z): (x * 3129871 as int) ^ z * 116129781L ^ y, then the
// quadratic scramble, arithmetic shift by 16.
TB_HD TB_FI int64_t pos_seed(int32_t x, int32_t y, int32_t z) {
    const int64_t xm = static_cast<int32_t>(static_cast<uint32_t>(x) * 3129871u);
    uint64_t s = static_cast<uint64_t>(xm) ^ (static_cast<uint64_t>(static_cast<int64_t>(z)) * 116129781ull) ^
                 static_cast<uint64_t>(static_cast<int64_t>(y));
    s = s * s * 42317861ull + s * 11ull;
    return static_cast<int64_t>(s) >> 16;
}

// XoroshiroPositionalRandomFactory: at(x, y, z) seeds (getSeed ^ lo, hi).
struct Positional {
    uint64_t lo, hi;
    TB_HD TB_FI Xoro at(int32_t x, int32_t y, int32_t z) const { return Xoro::raw(static_cast<uint64_t>(pos_seed(x, y, z)) ^ lo, hi); }
};

// BiomeManager's LCG step: r * (r * A + B) + c.
TB_HD TB_FI int64_t zoom_lcg(int64_t r, int64_t c) {
    const uint64_t u = static_cast<uint64_t>(r);
    return static_cast<int64_t>(u * (u * 6364136223846793005ull + 1442695040888963407ull) + static_cast<uint64_t>(c));
}

// The fiddle draw as its integer part m = floorMod(r >> 24, 1024); the offset is
// (m / 1024 - 0.5) * 0.9.
TB_HD TB_FI int32_t zoom_fiddle_m(int64_t r) { return static_cast<int32_t>((r >> 24) & 1023); }
TB_HD TB_FI double zoom_fiddle(int32_t m) { return (static_cast<double>(m) / 1024.0 - 0.5) * 0.9; }

}  // namespace tb
