// Java-language arithmetic used by the TERRAIN step (JLS casts, java.lang.Math,
// Mojang's Mth helpers), written for sm_100a device code and, for the test-only
// host build, for the host. Every function must give the bits the reference port
// gives (cpu/include/mccuda/javamath.h); that relies on IEEE binary32/64 with
// round-to-nearest, no contraction (-fmad=false / -ffp-contract=off), no FTZ and
// correctly rounded division and square root.
#pragma once

#include <cstdint>
#include <cstring>
#include <cmath>

#if defined(__CUDACC__)
#define TB_HD __host__ __device__
#define TB_FI __forceinline__
#else
#define TB_HD
#define TB_FI inline __attribute__((always_inline))
#endif

namespace tb {

TB_HD TB_FI uint32_t fbits(float f) {
#if defined(__CUDA_ARCH__)
    return __float_as_uint(f);
#else
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return u;
#endif
}
TB_HD TB_FI float bitsf(uint32_t u) {
#if defined(__CUDA_ARCH__)
    return __uint_as_float(u);
#else
    float f;
    std::memcpy(&f, &u, 4);
    return f;
#endif
}
TB_HD TB_FI uint64_t dbits(double d) {
#if defined(__CUDA_ARCH__)
    return static_cast<uint64_t>(__double_as_longlong(d));
#else
    uint64_t u;
    std::memcpy(&u, &d, 8);
    return u;
#endif
}
TB_HD TB_FI double bitsd(uint64_t u) {
#if defined(__CUDA_ARCH__)
    return __longlong_as_double(static_cast<long long>(u));
#else
    double d;
    std::memcpy(&d, &u, 8);
    return d;
#endif
}

// (int) d per JLS 5.1.3: NaN -> 0, out of range -> the nearer bound, else toward zero.
TB_HD TB_FI int32_t d2i(double v) {
    if (!(v == v)) return 0;
    if (v >= 2147483647.0) return 2147483647;
    if (v <= -2147483648.0) return INT32_MIN;
    return static_cast<int32_t>(v);
}

// Mth.floor(double): (int) Math.floor(v). The device form is one cvt.rmi.s32.f64,
// which saturates like the Java cast; NaN is decided on the bits.
#ifndef TB_FLOOR_FINITE
#define TB_FLOOR_FINITE 1
#endif
TB_HD TB_FI int32_t jfloor(double v) {
#if defined(__CUDA_ARCH__)
    if ((dbits(v) << 1) > 0xFFE0000000000000ull) return 0;
    return __double2int_rd(v);
#else
    return d2i(std::floor(v));
#endif
}

// Mth.floor for a value known to be finite (an integer block coordinate times a finite
// scale plus a finite offset): the NaN test of jfloor is not needed.
TB_HD TB_FI int32_t jfloor_finite(double v) {
#if defined(__CUDA_ARCH__) && TB_FLOOR_FINITE
    return __double2int_rd(v);
#else
    return jfloor(v);
#endif
}

TB_HD TB_FI double dfloor(double v) {
#if defined(__CUDA_ARCH__)
    return ::floor(v);
#else
    return std::floor(v);
#endif
}

TB_HD TB_FI double dsqrt(double v) {
#if defined(__CUDA_ARCH__)
    return __dsqrt_rn(v);
#else
    return std::sqrt(v);
#endif
}

TB_HD TB_FI double dabs(double v) { return bitsd(dbits(v) & 0x7FFFFFFFFFFFFFFFull); }
TB_HD TB_FI float fabs_j(float v) { return bitsf(fbits(v) & 0x7FFFFFFFu); }

// wrapping int32 arithmetic (Java int overflow semantics)
TB_HD TB_FI int32_t iadd(int32_t a, int32_t b) { return static_cast<int32_t>(static_cast<uint32_t>(a) + static_cast<uint32_t>(b)); }
TB_HD TB_FI int32_t isub(int32_t a, int32_t b) { return static_cast<int32_t>(static_cast<uint32_t>(a) - static_cast<uint32_t>(b)); }
TB_HD TB_FI int32_t imul(int32_t a, int32_t b) { return static_cast<int32_t>(static_cast<uint32_t>(a) * static_cast<uint32_t>(b)); }

// Math.floorDiv / floorMod (int)
TB_HD TB_FI int32_t fdiv(int32_t a, int32_t b) {
    int32_t q = a / b;
    return (q * b != a && ((a ^ b) < 0)) ? q - 1 : q;
}
TB_HD TB_FI int32_t fmod_i(int32_t a, int32_t b) { return a - fdiv(a, b) * b; }
TB_HD TB_FI int32_t imin(int32_t a, int32_t b) { return a < b ? a : b; }
// index of the highest set bit of m != 0
TB_HD TB_FI int hibit(uint32_t m) {
#if defined(__CUDA_ARCH__)
    return 31 - __clz(m);
#else
    return 31 - __builtin_clz(m);
#endif
}
TB_HD TB_FI int32_t imax(int32_t a, int32_t b) { return a < b ? b : a; }

// Math.min / Math.max (float and double): NaN propagates from either side, and
// -0.0 orders below +0.0.
TB_HD TB_FI float jmin(float a, float b) {
    if (!(a == a)) return a;
    if (a == 0.0f && b == 0.0f) return (fbits(b) == 0x80000000u) ? b : a;
    return a <= b ? a : b;
}
TB_HD TB_FI float jmax(float a, float b) {
    if (!(a == a)) return a;
    if (a == 0.0f && b == 0.0f) return (fbits(a) == 0x80000000u) ? b : a;
    return a >= b ? a : b;
}
TB_HD TB_FI double jmind(double a, double b) {
    if (!(a == a)) return a;
    if (a == 0.0 && b == 0.0) return (dbits(b) == 0x8000000000000000ull) ? b : a;
    return a <= b ? a : b;
}

// Mth.clamp(float): v < lo ? lo : Math.min(v, hi); Mth.clamp(double) likewise.
TB_HD TB_FI float jclamp(float v, float lo, float hi) { return v < lo ? lo : jmin(v, hi); }
TB_HD TB_FI double jclampd(double v, double lo, double hi) { return v < lo ? lo : jmind(v, hi); }

// Mth.lerp(alpha, a, b) = a + alpha * (b - a)
TB_HD TB_FI float lerpf(float t, float a, float b) { return a + t * (b - a); }
TB_HD TB_FI float lerp2f(float t1, float t2, float a00, float a10, float a01, float a11) {
    return lerpf(t2, lerpf(t1, a00, a10), lerpf(t1, a01, a11));
}
TB_HD TB_FI float lerp3f(float t1, float t2, float t3, float a000, float a100, float a010, float a110, float a001, float a101, float a011,
                         float a111) {
    return lerpf(t3, lerp2f(t1, t2, a000, a100, a010, a110), lerp2f(t1, t2, a001, a101, a011, a111));
}

// Mth.smoothstep(x) = x^3 (x (6x - 15) + 10), evaluated left to right as in Java.
TB_HD TB_FI float smoothf(float x) {
    float inner = x * (x * 6.0f - 15.0f) + 10.0f;
    return x * x * x * inner;
}

// Math.round(float) = floor(a + 0.5) on the exact double sum, then the int cast.
TB_HD TB_FI int32_t jround(float a) { return d2i(dfloor(static_cast<double>(a) + 0.5)); }

// Math.signum(float)
TB_HD TB_FI float jsignum(float x) {
    if (!(x == x) || x == 0.0f) return x;
    return x > 0.0f ? 1.0f : -1.0f;
}

// (long) f per JLS: NaN -> 0, saturating.
TB_HD TB_FI int64_t f2l(float v) {
    if (!(v == v)) return 0;
    if (v >= 9.2233720368547758e18f) return INT64_MAX;
    if (v <= -9.2233720368547758e18f) return INT64_MIN;
    return static_cast<int64_t>(v);
}

}  // namespace tb
