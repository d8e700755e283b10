// Improved-Perlin gradient noise in the two association orders the TERRAIN step
// uses, octave stacks over per-seed layer tables, and the legacy 2-D simplex noise
// of biome temperature (host + device).
//
// Reference semantics (cpu/include/mccuda/noise_eval.h):
//   point path   PerlinNoise.get            noise_eval.h:115-124 (dot (gx x + gy y) + gz z)
//   volume path  PerlinNoise.addToVolume    noise_eval.h:163-178 (dot (gx x + gz z) + gy y,
//                                           coordinate block * (scale * frequency))
//   smeared      SmearedPerlinNoise         noise_eval.h:181-220
//   stacks       NoiseStack.get / addToVolume  noise_eval.h:267-304
//   wrap         GradientNoise.wrap         noise_eval.h:56-70
//   simplex      SimplexNoise (2-D)         cpu/src/terrain.cpp:35-68
#pragma once

#include "tb_math.cuh"

namespace tb {

struct OctaveOff {       // random lattice offsets of one octave (and the BlendedNoise y smear)
    double ox, oy, oz, smear;
};
struct Layer {           // one NoiseStack layer: frequency, float amplitude, octave index
    double freq;
    float amp;
    int32_t oct;
};
struct NoiseTables {
    const OctaveOff* off;
    const uint8_t* perm;     // 256 bytes per octave
    const Layer* layer;
    const uint16_t* perm2;   // per octave, entry i = perm[i] | perm[(i + 1) & 255] << 8
};

// GradientNoise.GRADIENT[h & 15], one component, as a float in {-1, 0, 1}.
// Packed as two 16-bit masks per axis: which vectors have a non-zero component and
// which of those are negative.
TB_HD TB_FI float grad_axis(uint32_t h, uint32_t nz, uint32_t neg) {
    const uint32_t b = 1u << (h & 15u);
    return (nz & b) ? ((neg & b) ? -1.0f : 1.0f) : 0.0f;
}
//                                    vector:  fedcba9876543210
constexpr uint32_t kGxNz = 0x50FFu;   // x != 0: 0..7, 12, 14
constexpr uint32_t kGxNeg = 0x40AAu;  // x < 0 : 1, 3, 5, 7, 14
constexpr uint32_t kGyNz = 0xFF0Fu;   // y != 0: 0..3, 8..15
constexpr uint32_t kGyNeg = 0xAA0Cu;  // y < 0 : 2, 3, 9, 11, 13, 15
constexpr uint32_t kGzNz = 0xAFF0u;   // z != 0: 4..11, 13, 15
constexpr uint32_t kGzNeg = 0x8CC0u;  // z < 0 : 6, 7, 10, 11, 15
TB_HD TB_FI float gx_of(uint32_t h) { return grad_axis(h, kGxNz, kGxNeg); }
TB_HD TB_FI float gy_of(uint32_t h) { return grad_axis(h, kGyNz, kGyNeg); }
TB_HD TB_FI float gz_of(uint32_t h) { return grad_axis(h, kGzNz, kGzNeg); }

// GRADIENT[h & 15] . (dx, dy, dz) as the sum of its two non-zero terms. Each of the 16
// vectors has exactly two components of +-1 and one of 0: the first term is dx for h < 8
// and dy otherwise, the second dy for h < 4, dx for h = 12 and 14, dz otherwise; bits 0 and
// 1 of h negate them. The zero component's product is a signed zero, and adding it to the
// other two (in either association order, IEEE addition being commutative) changes at
// most the sign of a zero sum. Through the trilinear lerps a zero's sign reaches only the
// sign of a zero result, and every octave value is accumulated onto a stack sum that
// starts at +0 (x + -0 = x, +0 + -0 = +0), so stack values are bit-identical to the
// three-product forms of the reference.
TB_HD TB_FI float grad_pair(uint32_t h, float dx, float dy, float dz) {
    h &= 15u;
    const float u = h < 8u ? dx : dy;
    const float v = h < 4u ? dy : ((h == 12u || h == 14u) ? dx : dz);
    return bitsf(fbits(u) ^ ((h & 1u) << 31)) + bitsf(fbits(v) ^ ((h & 2u) << 30));
}
#ifndef TB_GRAD_PAIR
#define TB_GRAD_PAIR 1
#endif

constexpr double kWrapLimit = 0x1.fffffffffffffp+23;   // largest double below 2^24

// GradientNoise.wrap: values inside [-L, L) pass unchanged; the rest fold by 2^25. One
// compare on |v|: at v = -L the fold gives v back (floor(-L / 2^25 + 0.5) = 0), and NaN,
// the infinities and L take the fold as before.
TB_HD TB_FI double nwrap(double v) {
    if (dabs(v) < kWrapLimit) return v;
    return v - dfloor(v / 33554432.0 + 0.5) * 33554432.0;
}

// The eight corner hashes of lattice cell (fx, fy, fz), ordered x + 2y + 4z.
struct CellHash {
    uint32_t h[8];
};
TB_HD TB_FI CellHash cell_hash(const uint8_t* P, int32_t fx, int32_t fy, int32_t fz) {
    const uint32_t X = static_cast<uint32_t>(fx), Y = static_cast<uint32_t>(fy), Z = static_cast<uint32_t>(fz);
    const uint32_t a0 = P[X & 255u], a1 = P[(X + 1u) & 255u];
    const uint32_t b00 = P[(a0 + Y) & 255u], b01 = P[(a0 + Y + 1u) & 255u];
    const uint32_t b10 = P[(a1 + Y) & 255u], b11 = P[(a1 + Y + 1u) & 255u];
    CellHash c;
    c.h[0] = P[(b00 + Z) & 255u];
    c.h[1] = P[(b10 + Z) & 255u];
    c.h[2] = P[(b01 + Z) & 255u];
    c.h[3] = P[(b11 + Z) & 255u];
    c.h[4] = P[(b00 + Z + 1u) & 255u];
    c.h[5] = P[(b10 + Z + 1u) & 255u];
    c.h[6] = P[(b01 + Z + 1u) & 255u];
    c.h[7] = P[(b11 + Z + 1u) & 255u];
    return c;
}

// The same eight hashes from the paired table: each 16-bit entry holds perm[i] and
// perm[i + 1], the two values every lattice step reads together, so 7 loads replace 14.
// From the first lookup's entry a = P2[fx & 255] on.
TB_HD TB_FI CellHash cell_hash2_from(const uint16_t* P2, uint32_t a, int32_t fy, int32_t fz) {
    const uint32_t Y = static_cast<uint32_t>(fy), Z = static_cast<uint32_t>(fz);
    const uint32_t b0 = P2[((a & 255u) + Y) & 255u], b1 = P2[((a >> 8) + Y) & 255u];
    const uint32_t c00 = P2[((b0 & 255u) + Z) & 255u], c01 = P2[((b0 >> 8) + Z) & 255u];
    const uint32_t c10 = P2[((b1 & 255u) + Z) & 255u], c11 = P2[((b1 >> 8) + Z) & 255u];
    CellHash c;
    c.h[0] = c00 & 255u;
    c.h[1] = c10 & 255u;
    c.h[2] = c01 & 255u;
    c.h[3] = c11 & 255u;
    c.h[4] = c00 >> 8;
    c.h[5] = c10 >> 8;
    c.h[6] = c01 >> 8;
    c.h[7] = c11 >> 8;
    return c;
}
TB_HD TB_FI CellHash cell_hash2(const uint16_t* P2, int32_t fx, int32_t fy, int32_t fz) {
    return cell_hash2_from(P2, P2[static_cast<uint32_t>(fx) & 255u], fy, fz);
}
#ifndef TB_PERM_PAIRS
#define TB_PERM_PAIRS 1
#endif
TB_HD TB_FI CellHash octave_hash(const NoiseTables& T, int32_t oct, int32_t fx, int32_t fy, int32_t fz) {
#if TB_PERM_PAIRS
    return cell_hash2(T.perm2 + 256 * oct, fx, fy, fz);
#else
    return cell_hash(T.perm + 256 * oct, fx, fy, fz);
#endif
}

// Point-path cell value: dot products (gx*dx + gy*dy) + gz*dz, weights from
// smoothstep of (rx, wy, rz); ry is the y offset fed to the dot products.
TB_HD TB_FI float cell_point(const CellHash& c, float rx, float ry, float rz, float wy) {
    float d[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const float dx = (k & 1) ? rx - 1.0f : rx;
        const float dy = (k & 2) ? ry - 1.0f : ry;
        const float dz = (k & 4) ? rz - 1.0f : rz;
#if TB_GRAD_PAIR
        d[k] = grad_pair(c.h[k], dx, dy, dz);
#else
        const float xy = gx_of(c.h[k]) * dx + gy_of(c.h[k]) * dy;
        d[k] = xy + gz_of(c.h[k]) * dz;
#endif
    }
    return lerp3f(smoothf(rx), smoothf(wy), smoothf(rz), d[0], d[1], d[2], d[3], d[4], d[5], d[6], d[7]);
}

// Volume-path cell value: (gx*dx + gz*dz) + gy*dy with precomputed weights.
TB_HD TB_FI float cell_volume(const CellHash& c, float rx, float rz, float ry, float ax, float ay, float az) {
    float d[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const float dx = (k & 1) ? rx - 1.0f : rx;
        const float dz = (k & 4) ? rz - 1.0f : rz;
        const float dy = (k & 2) ? ry - 1.0f : ry;
#if TB_GRAD_PAIR
        d[k] = grad_pair(c.h[k], dx, dy, dz);
#else
        const float xz = gx_of(c.h[k]) * dx + gz_of(c.h[k]) * dz;
        d[k] = xz + gy_of(c.h[k]) * dy;
#endif
    }
    return lerp3f(ax, ay, az, d[0], d[1], d[2], d[3], d[4], d[5], d[6], d[7]);
}

// One axis of the volume coordinate setup: lattice cell, offset, weight.
struct AxisSetup {
    int32_t f;
    float r, a;
};
TB_HD TB_FI AxisSetup axis_setup(int32_t b, double scale, double off) {
    const double v = nwrap(static_cast<double>(b) * scale) + off;
    const int32_t f = jfloor_finite(v);
    const float r = static_cast<float>(v - static_cast<double>(f));
    return {f, r, smoothf(r)};
}

// SmearedPerlinNoise.computeFudgeY
TB_HD TB_FI double smear_fudge(double orig_y, double rel_y, double smear) {
    const double lim = (orig_y >= 0.0 && orig_y < rel_y) ? orig_y : rel_y;
    return static_cast<double>(jfloor(lim / smear + static_cast<double>(1.0E-7f))) * smear;
}

// One octave, volume path (PerlinNoise.addToVolume, one sample).
TB_HD TB_FI float octave_volume(const NoiseTables& T, int32_t oct, int32_t bx, int32_t by, int32_t bz, double xs, double ys) {
    const OctaveOff o = T.off[oct];
    const AxisSetup Z = axis_setup(bz, xs, o.oz);
    const AxisSetup X = axis_setup(bx, xs, o.ox);
    const AxisSetup Y = axis_setup(by, ys, o.oy);
    const CellHash c = octave_hash(T, oct, X.f, Y.f, Z.f);
    return cell_volume(c, X.r, Z.r, Y.r, X.a, Y.a, Z.a);
}

// One octave, smeared volume path (SmearedPerlinNoise.addToVolume, one sample).
TB_HD TB_FI float octave_volume_smeared(const NoiseTables& T, int32_t oct, int32_t bx, int32_t by, int32_t bz, double xs, double ys) {
    const OctaveOff o = T.off[oct];
    const AxisSetup Z = axis_setup(bz, xs, o.oz);
    const AxisSetup X = axis_setup(bx, xs, o.ox);
    const double oy = static_cast<double>(by) * ys;
    const double y = nwrap(oy) + o.oy;
    const int32_t fy = jfloor_finite(y);
    const double rel = y - static_cast<double>(fy);
    const float ay = smoothf(static_cast<float>(rel));
    const CellHash c = octave_hash(T, oct, X.f, fy, Z.f);
    const float fudged = static_cast<float>(rel - smear_fudge(oy, rel, o.smear));
    return cell_volume(c, X.r, Z.r, fudged, X.a, ay, Z.a);
}

// One octave, point path (PerlinNoise.get).
TB_HD TB_FI float octave_point(const NoiseTables& T, int32_t oct, double px, double py, double pz) {
    const OctaveOff o = T.off[oct];
    const double x = nwrap(px) + o.ox, y = nwrap(py) + o.oy, z = nwrap(pz) + o.oz;
    const int32_t fx = jfloor(x), fy = jfloor(y), fz = jfloor(z);
    const float rx = static_cast<float>(x - static_cast<double>(fx));
    const float ry = static_cast<float>(y - static_cast<double>(fy));
    const float rz = static_cast<float>(z - static_cast<double>(fz));
    return cell_point(octave_hash(T, oct, fx, fy, fz), rx, ry, rz, ry);
}

// One octave, smeared point path (SmearedPerlinNoise.get).
TB_HD TB_FI float octave_point_smeared(const NoiseTables& T, int32_t oct, double px, double py, double pz) {
    const OctaveOff o = T.off[oct];
    const double x = nwrap(px) + o.ox, y = nwrap(py) + o.oy, z = nwrap(pz) + o.oz;
    const int32_t fx = jfloor(x), fy = jfloor(y), fz = jfloor(z);
    const float rx = static_cast<float>(x - static_cast<double>(fx));
    const double rel = y - static_cast<double>(fy);
    const float rz = static_cast<float>(z - static_cast<double>(fz));
    const float fudged = static_cast<float>(rel - smear_fudge(py, rel, o.smear));
    return cell_point(octave_hash(T, oct, fx, fy, fz), rx, fudged, rz, static_cast<float>(rel));
}

// NoiseStack.addToVolume / NoiseStack.get over a run of layers. One out-of-line copy
// per variant serves every noise of the evaluators, so the octave code stays resident
// in the instruction cache; the layer loop is not unrolled for the same reason.
#if defined(__CUDA_ARCH__)
#define TB_NOINLINE __noinline__
#else
#define TB_NOINLINE
#endif

// Work counting, in the host build of the test suite only (TB_COUNT_OPS): one count per
// octave sample (volume, smeared volume, point, smeared point) and per simplex sample,
// into the array the host twin points tb_op_counts at for the stage it runs. The device
// build never counts.
#if defined(TB_COUNT_OPS) && !defined(__CUDA_ARCH__)
extern thread_local long long* tb_op_counts;
#define TB_COUNT(kind) (++tb_op_counts[kind])
#else
#define TB_COUNT(kind) ((void)0)
#endif
enum OpKind { kOpVolume, kOpVolumeSmeared, kOpPoint, kOpPointSmeared, kOpSimplex, kOpKinds };

TB_HD TB_NOINLINE inline float stack_volume_rt(const NoiseTables& T, int first, int count, int32_t bx, int32_t by, int32_t bz, double xzs, double yss,
                                                float amplitude) {
    float acc = 0.0f;
#pragma unroll 1
    for (int i = first; i < first + count; ++i) {
        TB_COUNT(kOpVolume);
        const Layer L = T.layer[i];
        const double xs = xzs * L.freq, ys = yss * L.freq;
        const float amp = amplitude * L.amp;
        acc = acc + amp * octave_volume(T, L.oct, bx, by, bz, xs, ys);
    }
    return acc;
}

TB_HD TB_NOINLINE inline float stack_volume_smeared_rt(const NoiseTables& T, int first, int count, int32_t bx, int32_t by, int32_t bz, double xzs,
                                                        double yss, float amplitude) {
    float acc = 0.0f;
#pragma unroll 1
    for (int i = first; i < first + count; ++i) {
        TB_COUNT(kOpVolumeSmeared);
        const Layer L = T.layer[i];
        const double xs = xzs * L.freq, ys = yss * L.freq;
        const float amp = amplitude * L.amp;
        acc = acc + amp * octave_volume_smeared(T, L.oct, bx, by, bz, xs, ys);
    }
    return acc;
}

TB_HD TB_NOINLINE inline float stack_point_rt(const NoiseTables& T, int first, int count, double x, double y, double z) {
    float acc = 0.0f;
#pragma unroll 1
    for (int i = first; i < first + count; ++i) {
        TB_COUNT(kOpPoint);
        const Layer L = T.layer[i];
        const double f = L.freq;
        acc = acc + L.amp * octave_point(T, L.oct, x * f, y * f, z * f);
    }
    return acc;
}

TB_HD TB_NOINLINE inline float stack_point_smeared_rt(const NoiseTables& T, int first, int count, double x, double y, double z) {
    float acc = 0.0f;
#pragma unroll 1
    for (int i = first; i < first + count; ++i) {
        TB_COUNT(kOpPointSmeared);
        const Layer L = T.layer[i];
        const double f = L.freq;
        acc = acc + L.amp * octave_point_smeared(T, L.oct, x * f, y * f, z * f);
    }
    return acc;
}

// The x or z coordinate record of one octave layer at one coordinate, precomputed per batch
// (axis_setup of the coordinate, the stack's xz scale times the layer frequency, and the
// octave's x or z offset): the corner kernel's columns share x and z across their 49 rows
// and across neighbouring columns, so the tables replace most of an octave's FP64 work by
// two 16-byte loads.
struct AxisRec {
    int32_t f;
    float r, a;
    int32_t hx;   // x records: the paired-permutation entry of the lattice x (the hash's first lookup); else 0
};
#ifndef TB_AXIS_TABLE
#define TB_AXIS_TABLE 1
#endif
#if TB_AXIS_TABLE
#define TB_AXIS_SEL(table, plain) (table)
#else
#define TB_AXIS_SEL(table, plain) (plain)
#endif

// The y coordinate record of one octave layer at corner height by, for a stack of y scale
// yss: the volume path's y setup (floor, fraction, smoothstep), or for a smeared stack
// (SmearedPerlinNoise) the floor, the fudged fraction the gradients read and the smoothstep of
// the plain fraction. It depends only on the seed, the layer and the height, so it is built
// once per seed for every corner row (on the host) instead of once per sample.
TB_HD TB_FI AxisRec y_record(const NoiseTables& T, int layer, double yss, bool smeared, int32_t by) {
    const Layer L = T.layer[layer];
    const double ys = yss * L.freq;
    const OctaveOff o = T.off[L.oct];
    if (!smeared) {
        const AxisSetup Y = axis_setup(by, ys, o.oy);
        return {Y.f, Y.r, Y.a, 0};
    }
    const double oy = static_cast<double>(by) * ys;
    const double y = nwrap(oy) + o.oy;
    const int32_t fy = jfloor_finite(y);
    const double rel = y - static_cast<double>(fy);
    const float ay = smoothf(static_cast<float>(rel));
    const float fudged = static_cast<float>(rel - smear_fudge(oy, rel, o.smear));
    return {fy, fudged, ay, 0};
}

// A volume stack (plain or smeared) with the x / z / y records of layer first + k at ax[k],
// az[k], ay[k]
template <bool SMEARED>
TB_HD TB_NOINLINE inline float stack_volume_axy_rt(const NoiseTables& T, int first, int count, const AxisRec* ax, const AxisRec* az, const AxisRec* ay,
                                                    float amplitude) {
    float acc = 0.0f;
#pragma unroll 1
    for (int k = 0; k < count; ++k) {
        TB_COUNT(SMEARED ? kOpVolumeSmeared : kOpVolume);
        const Layer L = T.layer[first + k];
        const float amp = amplitude * L.amp;
        const AxisRec X = ax[k], Z = az[k], Y = ay[k];
#if TB_PERM_PAIRS
        const CellHash c = cell_hash2_from(T.perm2 + 256 * L.oct, static_cast<uint32_t>(X.hx), Y.f, Z.f);
#else
        const CellHash c = octave_hash(T, L.oct, X.f, Y.f, Z.f);
#endif
        acc = acc + amp * cell_volume(c, X.r, Z.r, Y.r, X.a, Y.a, Z.a);
    }
    return acc;
}

template <int FIRST, int COUNT, bool SMEARED>
TB_HD TB_FI float stack_volume_ax(const NoiseTables& T, const AxisRec* ax, const AxisRec* az, const AxisRec* ay, float amplitude) {
    return stack_volume_axy_rt<SMEARED>(T, FIRST, COUNT, ax, az, ay, amplitude);
}

// The same stacks with the layer run chosen per thread: threads of a warp that evaluate
// different stacks of one noise (a blended noise's lower or upper limit) share one call.
template <bool SMEARED>
TB_HD TB_FI float stack_volume_ax_dyn(const NoiseTables& T, int first, int count, const AxisRec* ax, const AxisRec* az, const AxisRec* ay,
                                      float amplitude) {
    return stack_volume_axy_rt<SMEARED>(T, first, count, ax, az, ay, amplitude);
}
template <bool SMEARED>
TB_HD TB_FI float stack_volume_dyn(const NoiseTables& T, int first, int count, int32_t bx, int32_t by, int32_t bz, double xzs, double yss, float amplitude) {
    return SMEARED ? stack_volume_smeared_rt(T, first, count, bx, by, bz, xzs, yss, amplitude) : stack_volume_rt(T, first, count, bx, by, bz, xzs, yss, amplitude);
}
template <bool SMEARED>
TB_HD TB_FI float stack_point_dyn(const NoiseTables& T, int first, int count, double x, double y, double z) {
    return SMEARED ? stack_point_smeared_rt(T, first, count, x, y, z) : stack_point_rt(T, first, count, x, y, z);
}

template <int FIRST, int COUNT, bool SMEARED>
TB_HD TB_FI float stack_volume(const NoiseTables& T, int32_t bx, int32_t by, int32_t bz, double xzs, double yss, float amplitude) {
    return SMEARED ? stack_volume_smeared_rt(T, FIRST, COUNT, bx, by, bz, xzs, yss, amplitude) : stack_volume_rt(T, FIRST, COUNT, bx, by, bz, xzs, yss, amplitude);
}

template <int FIRST, int COUNT, bool SMEARED>
TB_HD TB_FI float stack_point(const NoiseTables& T, double x, double y, double z) {
    return SMEARED ? stack_point_smeared_rt(T, FIRST, COUNT, x, y, z) : stack_point_rt(T, FIRST, COUNT, x, y, z);
}

// ---- legacy 2-D simplex (SimplexNoise with zero offsets) -----------------------------
struct Simplex2 {
    uint8_t perm[256];
    double ox, oy;
};

TB_HD TB_FI double simplex_corner(int g, double x, double y) {
    // gradient g of the first twelve cube-edge vectors; z = 0
    double t = 0.5 - x * x - y * y - 0.0 * 0.0;
    if (t < 0.0) return 0.0;
    t *= t;
    const double gx = static_cast<double>(gx_of(static_cast<uint32_t>(g)));
    const double gy = static_cast<double>(gy_of(static_cast<uint32_t>(g)));
    const double gz = static_cast<double>(gz_of(static_cast<uint32_t>(g)));
    const double dot = (gx * x + gy * y) + gz * 0.0;
    return t * t * dot;
}

// f2 = (sqrt(3) - 1) / 2, g2 = (3 - sqrt(3)) / 6 as computed in double.
TB_HD TB_FI float simplex2(const Simplex2& s, double px, double py, double f2, double g2) {
    TB_COUNT(kOpSimplex);
    const double xin = px + s.ox, yin = py + s.oy;
    const double sk = (xin + yin) * f2;
    const int32_t i = jfloor(xin + sk), j = jfloor(yin + sk);
    const double t = static_cast<double>(iadd(i, j)) * g2;
    const double x0 = xin - (static_cast<double>(i) - t), y0 = yin - (static_cast<double>(j) - t);
    const int i1 = x0 > y0 ? 1 : 0, j1 = 1 - i1;
    const double x1 = x0 - static_cast<double>(i1) + g2, y1 = y0 - static_cast<double>(j1) + g2;
    const double x2 = x0 - 1.0 + 2.0 * g2, y2 = y0 - 1.0 + 2.0 * g2;
    const int ii = i & 255, jj = j & 255;
    const uint8_t* P = s.perm;
    const int g0 = P[(ii + P[jj]) & 255] % 12;
    const int g1 = P[(ii + i1 + P[(jj + j1) & 255]) & 255] % 12;
    const int gg2 = P[(ii + 1 + P[(jj + 1) & 255]) & 255] % 12;
    const double n0 = simplex_corner(g0, x0, y0), n1 = simplex_corner(g1, x1, y1), n2 = simplex_corner(gg2, x2, y2);
    return static_cast<float>(70.0 * (n0 + n1 + n2));
}

}  // namespace tb
