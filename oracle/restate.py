"""TEST INFRASTRUCTURE: a numpy restatement of the reference's TERRAIN-step arithmetic.

An independent second implementation of the reference C++ port (cpu/ of
bonquifo/minecraft-terrain-cuda), written from its algorithm in array form and used only by
tests/ as a checker. It covers RNGs and seed setup (cpu/src/rng.cpp, cpu/src/seed_tables.cpp,
cpu/src/terrain.cpp:112-149), gradient noise (cpu/include/mccuda/noise_eval.h), the
density-function interpreter in volume and point semantics (cpu/src/volume_eval.cpp), climate
quantisation, the climate R-tree with its last-result candidate and chunk biomes
(cpu/src/biome.cpp:95-236, cpu/src/terrain.cpp:152-176) and the BiomeManager zoom
(cpu/src/biome.cpp:241-289). The aquifer and the material rules are not restated: the
compiled reference port (oracle/_ref) checks those.

Pinned by tests/test_restate.py against the golden fixtures and the compiled port.
Exactness: float32 / float64 element-wise numpy arithmetic is IEEE round-to-nearest with
no contraction; 64-bit integer arithmetic uses Python ints with explicit wrapping.
"""
import hashlib
import json
import math
import struct

import numpy as np

F32 = np.float32
F64 = np.float64
M64 = (1 << 64) - 1


def f32(bits):
    return F32(struct.unpack('<f', struct.pack('<I', bits & 0xFFFFFFFF))[0])


def f64(hexbits):
    return struct.unpack('<d', struct.pack('<Q', int(hexbits, 16)))[0]


def s64(v):
    v &= M64
    return v - (1 << 64) if v >> 63 else v


# ---- Java semantics (cpu/include/mccuda/javamath.h:61-173) -------------------------------
def d2i(v):
    """(int) double per JLS 5.1.3, elementwise."""
    v = np.asarray(v, F64)
    with np.errstate(invalid='ignore'):
        out = np.where(np.isnan(v), 0, np.clip(np.trunc(np.nan_to_num(v, nan=0.0)), -2147483648.0, 2147483647.0))
    return out.astype(np.int64)


def jfloor(v):
    """Mth.floor: (int) Math.floor(v)."""
    v = np.asarray(v, F64)
    with np.errstate(invalid='ignore'):
        return d2i(np.floor(v))


def jmin(a, b):
    a, b = F32(a) if np.isscalar(a) else a, F32(b) if np.isscalar(b) else b
    a, b = np.broadcast_arrays(np.asarray(a, F32), np.asarray(b, F32))
    neg0b = (a == 0) & (b == 0) & np.signbit(b)
    return np.where(np.isnan(a), a, np.where(neg0b, b, np.where(a <= b, a, b))).astype(F32)


def jmax(a, b):
    a, b = np.broadcast_arrays(np.asarray(a, F32), np.asarray(b, F32))
    neg0a = (a == 0) & (b == 0) & np.signbit(a)
    return np.where(np.isnan(a), a, np.where(neg0a, b, np.where(a >= b, a, b))).astype(F32)


def jclamp(v, lo, hi):
    v = np.asarray(v, F32)
    return np.where(v < F32(lo), F32(lo), jmin(v, F32(hi))).astype(F32)


def lerp(t, a, b):
    return (a + t * (b - a)).astype(F32)


def lerp2(t1, t2, a00, a10, a01, a11):
    return lerp(t2, lerp(t1, a00, a10), lerp(t1, a01, a11))


def lerp3(t1, t2, t3, a000, a100, a010, a110, a001, a101, a011, a111):
    return lerp(t3, lerp2(t1, t2, a000, a100, a010, a110), lerp2(t1, t2, a001, a101, a011, a111))


def smooth(x):
    x = np.asarray(x, F32)
    return (x * x * x * (x * (x * F32(6) - F32(15)) + F32(10))).astype(F32)


def floor_div(a, b):
    return np.floor_divide(np.asarray(a, np.int64), b)


# ---- random sources (cpu/src/rng.cpp) -------------------------------------------------
def stafford(z):
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
    return z ^ (z >> 31)


# vanilla scales random bits by float literals (cpu/src/rng.cpp:16-17); they round to
# 2^-53 and 2^-24.
DOUBLE_UNIT = float(F32(1.110223e-16))
FLOAT_UNIT = F32(5.9604645e-8)


def rotl(x, k):
    return ((x << k) | (x >> (64 - k))) & M64


class Xoroshiro:
    def __init__(self, lo, hi):
        lo, hi = lo & M64, hi & M64
        if lo == 0 and hi == 0:
            lo, hi = 0x9E3779B97F4A7C15, 0x6A09E667F3BCC909
        self.lo, self.hi = lo, hi

    @staticmethod
    def from_seed(seed):
        lo = (seed & M64) ^ 0x6A09E667F3BCC909
        return Xoroshiro(stafford(lo), stafford((lo + 0x9E3779B97F4A7C15) & M64))

    def next(self):
        s0, s1 = self.lo, self.hi
        r = (rotl((s0 + s1) & M64, 17) + s0) & M64
        s1 ^= s0
        self.lo = rotl(s0, 49) ^ s1 ^ ((s1 << 21) & M64)
        self.hi = rotl(s1, 28)
        return r

    def next_int(self, bound):
        m = (self.next() & 0xFFFFFFFF) * bound
        if (m & 0xFFFFFFFF) < bound:
            t = ((-bound) & 0xFFFFFFFF) % bound
            while (m & 0xFFFFFFFF) < t:
                m = (self.next() & 0xFFFFFFFF) * bound
        return m >> 32

    def next_double(self):
        return float(self.next() >> 11) * DOUBLE_UNIT

    def next_float(self):
        return F32(F32(self.next() >> 40) * FLOAT_UNIT)

    def next_bool(self):
        return (self.next() & 1) != 0

    def fork(self):
        return (self.next(), self.next())


def from_hash(pos, name):
    h = hashlib.md5(name.encode()).digest()
    return Xoroshiro(int.from_bytes(h[:8], 'big') ^ pos[0], int.from_bytes(h[8:], 'big') ^ pos[1])


def mth_get_seed(x, y, z):
    xm = ((x * 3129871) & 0xFFFFFFFF)
    xm = xm - (1 << 32) if xm >> 31 else xm
    s = (xm & M64) ^ ((z * 116129781) & M64) ^ (y & M64)
    s = (s * s * 42317861 + s * 11) & M64
    return s64(s) >> 16


def at(pos, x, y, z):
    return Xoroshiro(mth_get_seed(x, y, z) ^ pos[0], pos[1])


class Lcg:
    def __init__(self, seed):
        self.s = (seed ^ 0x5DEECE66D) & ((1 << 48) - 1)

    def bits(self, n):
        self.s = (self.s * 0x5DEECE66D + 0xB) & ((1 << 48) - 1)
        v = self.s >> (48 - n)
        return v - (1 << n) if n == 32 and v >> 31 else v

    def next_int(self, bound):
        if bound & -bound == bound:
            return (bound * self.bits(31)) >> 31
        while True:
            r = self.bits(31)
            m = r % bound
            if ((r - m + bound - 1) & 0xFFFFFFFF) >> 31 == 0:
                return m

    def next_double(self):
        return float((self.bits(26) << 27) + self.bits(27)) * DOUBLE_UNIT


# ---- per-seed noise tables (cpu/src/seed_tables.cpp:23-184) -------------------------
def stream_sum(vals):
    s0 = s1 = simple = 0.0
    for v in vals:
        tmp = v - s1
        velvel = s0 + tmp
        s1 = (velvel - s0) - tmp
        s0 = velvel
        simple += v
    r = s0 - s1
    return simple if math.isnan(r) and math.isinf(simple) else r


def make_octave(r, smear):
    ox, oy, oz = r.next_double() * 256.0, r.next_double() * 256.0, r.next_double() * 256.0
    p = list(range(256))
    for i in range(256):
        j = i + r.next_int(256 - i)
        p[i], p[j] = p[j], p[i]
    return (ox, oy, oz, smear, np.array(p, np.int64))


class Seed:
    def __init__(self, model, seed):
        self.m = model
        self.seed = seed
        self.octaves, self.layers = [], []
        self.noise, self.blended = {}, {}
        base = Xoroshiro.from_seed(seed)
        self.random = base.fork()
        for key in sorted(model.ir['noises']):
            self.noise[key] = self.normal_noise(model.ir['noises'][key], from_hash(self.random, key))
        for n in model.nodes:
            if n['t'] == 'blended_noise':
                r = from_hash(self.random, 'minecraft:terrain')
                ymul = 684.412 * f64(n['y_scale'])
                limit = ymul * f64(n['smear_scale_multiplier'])
                main = limit / f64(n['y_factor'])
                lf = float(F32(0.99998474))
                self.blended[n['id']] = (self.fbm(r, -15, limit, lf), self.fbm(r, -15, limit, lf), self.fbm(r, -7, main, 12.75))
        z = hashlib.sha256((seed & M64).to_bytes(8, 'little')).digest()
        self.zoom_seed = s64(int.from_bytes(z[:8], 'little'))
        # TerrainSeed (cpu/src/terrain.cpp:112-149)
        self.aquifer = from_hash(self.random, 'minecraft:aquifer').fork()
        self.ore = from_hash(self.random, 'minecraft:ore').fork()
        self.clay = self.clay_bands(model)

    def clay_bands(self, model):
        """MaterialSystem.generateBands (cpu/src/terrain.cpp:119-149)."""
        pal = model.tm['palette']
        T, WHITE, ORANGE, YELLOW, BROWN, RED, LIGHT_GRAY = (pal.index('minecraft:' + c + 'terracotta') if ('minecraft:' + c + 'terracotta') in pal else -1
                                                           for c in ('', 'white_', 'orange_', 'yellow_', 'brown_', 'red_', 'light_gray_'))
        r = from_hash(self.random, 'minecraft:clay_bands')
        b = [T] * 192
        i = 0
        while i < 192:
            i += r.next_int(5) + 1
            if i < 192:
                b[i] = ORANGE
            i += 1
        for base, state in ((1, YELLOW), (2, BROWN), (1, RED)):
            for _ in range(r.next_int(15 - 6 + 1) + 6):
                width = base + r.next_int(3)
                start = r.next_int(192)
                for p in range(width):
                    if start + p >= 192:
                        break
                    b[start + p] = state
        white = r.next_int(15 - 9 + 1) + 9
        i, start = 0, 0
        while i < white and start < 192:
            b[start] = WHITE
            if start - 1 > 0 and r.next_bool():
                b[start - 1] = LIGHT_GRAY
            if start + 1 < 192 and r.next_bool():
                b[start + 1] = LIGHT_GRAY
            i += 1
            start += r.next_int(16) + 4
        return np.array(b, np.int32)

    def normal_noise(self, d, random):
        mods = [f64(m) for m in d['amplitude_modifiers']]
        n = d['octave_count']
        mod = lambda i: mods[i] if mods else 1.0
        freq = math.ldexp(1.0, d['base_octave'])
        amp = f64(d['base_amplitude'])
        if d['normalize'] != 'disabled':
            amp *= math.ldexp(1.0, n - 1) / (math.ldexp(1.0, n) - 1.0)
        octs = []
        for i in range(n):
            if mod(i) != 0.0:
                octs.append((d['base_octave'] + i, freq, amp * mod(i)))
            freq *= 2.0
            amp *= 0.5
        var = 0.0
        for o in octs:
            l = 0.2702247831245211 * abs(o[2])
            var += l * l
        dev = math.sqrt(var)
        target = stream_sum([abs(o[2]) for o in octs])
        norm = 0.0 if dev == 0.0 else (target * 0.3333333333333333) / (dev * math.sqrt(2.0))
        if d['normalize'] == 'legacy' and norm != 0.0:
            idx = [i for i in range(n) if mod(i) != 0.0]
            span = max(idx) - min(idx)
            norm = f64(d['base_amplitude']) * 0.5 * 0.3333333333333333 / (0.1 * (1.0 + 1.0 / (span + 1)))
        first, second = random.fork(), random.fork()
        start = len(self.layers)
        for index, fr, a in octs:
            key = 'octave_%d' % index
            vf = float(F32(norm * a))
            self.octaves.append(make_octave(from_hash(first, key), 0.0))
            self.layers.append((fr, vf, len(self.octaves) - 1))
            self.octaves.append(make_octave(from_hash(second, key), 0.0))
            self.layers.append((fr * 1.0181268882175227, vf, len(self.octaves) - 1))
        return (start, len(self.layers) - start)

    def fbm(self, r, first_octave, smear_y, vf):
        n = -first_octave + 1
        f = 1.0
        vf /= math.ldexp(1.0, n) - 1.0
        start = len(self.layers)
        for _ in range(n):
            self.octaves.append(make_octave(r, smear_y * f))
            self.layers.append((f, float(F32(vf)), len(self.octaves) - 1))
            f /= 2.0
            vf *= 2.0
        return (start, n)


# ---- noise (cpu/include/mccuda/noise_eval.h) --------------------------------------------
GRAD = np.array([(1, 1, 0), (-1, 1, 0), (1, -1, 0), (-1, -1, 0), (1, 0, 1), (-1, 0, 1), (1, 0, -1), (-1, 0, -1), (0, 1, 1), (0, -1, 1), (0, 1, -1),
                 (0, -1, -1), (1, 1, 0), (0, -1, 1), (-1, 1, 0), (0, -1, -1)], np.float32)
HALF = float.fromhex('0x1.fffffffffffffp+23')


def wrap(x):
    x = np.asarray(x, F64)
    inside = (x >= -HALF) & (x < HALF)
    return np.where(inside, x, x - np.floor(x / 33554432.0 + 0.5) * 33554432.0)


def hashes(p, fx, fy, fz):
    P = lambda v: p[np.asarray(v, np.int64) & 255]
    x0, x1 = P(fx), P(fx + 1)
    b00, b01, b10, b11 = P(x0 + fy), P(x0 + fy + 1), P(x1 + fy), P(x1 + fy + 1)
    return [P(b00 + fz), P(b10 + fz), P(b01 + fz), P(b11 + fz), P(b00 + fz + 1), P(b10 + fz + 1), P(b01 + fz + 1), P(b11 + fz + 1)]


def octave_point(o, px, py, pz, smeared=False, orig_y=None):
    ox, oy, oz, smear, p = o
    x, y, z = wrap(px) + ox, wrap(py) + oy, wrap(pz) + oz
    fx, fy, fz = jfloor(x), jfloor(y), jfloor(z)
    rx = (x - fx).astype(F32)
    rel = y - fy
    rz = (z - fz).astype(F32)
    if smeared:
        ry = (rel - fudge(py, rel, smear)).astype(F32)
        wy = rel.astype(F32)
    else:
        ry = rel.astype(F32)
        wy = ry
    h = hashes(p, fx, fy, fz)
    d = []
    for k in range(8):
        dx = rx - F32(1) if k & 1 else rx
        dy = ry - F32(1) if k & 2 else ry
        dz = rz - F32(1) if k & 4 else rz
        g = GRAD[h[k] & 15]
        d.append(((g[..., 0] * dx + g[..., 1] * dy) + g[..., 2] * dz).astype(F32))
    return lerp3(smooth(rx), smooth(wy), smooth(rz), *d)


def fudge(orig_y, rel, smear):
    lim = np.where((orig_y >= 0.0) & (orig_y < rel), orig_y, rel)
    return jfloor(lim / smear + float(F32(1.0e-7))).astype(F64) * smear


def octave_volume(o, bx, by, bz, xs, ys, smeared):
    ox, oy, oz, smear, p = o
    z = wrap(np.asarray(bz, F64) * xs) + oz
    fz = jfloor(z)
    rz = (z - fz).astype(F32)
    x = wrap(np.asarray(bx, F64) * xs) + ox
    fx = jfloor(x)
    rx = (x - fx).astype(F32)
    orig = np.asarray(by, F64) * ys
    y = wrap(orig) + oy
    fy = jfloor(y)
    rel = y - fy
    if smeared:
        ay = smooth(rel.astype(F32))
        ry = (rel - fudge(orig, rel, smear)).astype(F32)
    else:
        ry = rel.astype(F32)
        ay = smooth(ry)
    h = hashes(p, fx, fy, fz)
    d = []
    for k in range(8):
        dx = rx - F32(1) if k & 1 else rx
        dz = rz - F32(1) if k & 4 else rz
        dy = ry - F32(1) if k & 2 else ry
        g = GRAD[h[k] & 15]
        d.append(((g[..., 0] * dx + g[..., 2] * dz) + g[..., 1] * dy).astype(F32))
    return lerp3(smooth(rx), ay, smooth(rz), *d)


def stack_volume(S, ref, bx, by, bz, xzs, ys, amplitude, smeared):
    first, count = ref
    acc = np.zeros(np.broadcast(bx, by, bz).shape, F32)
    for fr, amp, oi in S.layers[first:first + count]:
        a = F32(F32(amplitude) * F32(amp))
        acc = (acc + a * octave_volume(S.octaves[oi], bx, by, bz, xzs * fr, ys * fr, smeared)).astype(F32)
    return acc


def stack_point(S, ref, x, y, z, smeared=False):
    first, count = ref
    acc = np.zeros(np.broadcast(x, y, z).shape, F32)
    for fr, amp, oi in S.layers[first:first + count]:
        acc = (acc + F32(amp) * octave_point(S.octaves[oi], np.asarray(x, F64) * fr, np.asarray(y, F64) * fr, np.asarray(z, F64) * fr,
                                             smeared)).astype(F32)
    return acc


# ---- model ---------------------------------------------------------------------------
class Model:
    def __init__(self, ir_path, tm_path):
        self.ir = json.load(open(ir_path))
        self.tm = json.load(open(tm_path))
        self.nodes = self.ir['nodes']
        self.roots = self.ir['roots']
        self.min_y, self.height = self.ir['min_y'], self.ir['height']
        self.tree = ClimateTree(self.tm['biome_parameters'])

    def node(self, i):
        return self.nodes[i]


# ---- density-function interpreter (cpu/src/volume_eval.cpp) -------------------------
class Volume:
    """sx, sy, sz cells from (minx, miny, minz) with strides (stx, sty, stz); element
    arrays are ordered y + (x + z * sx) * sy, as DensityVolume."""

    def __init__(self, sx, sy, sz, minx, miny, minz, stx=1, sty=1, stz=1):
        self.s = (sx, sy, sz)
        self.min = (minx, miny, minz)
        self.st = (stx, sty, stz)
        iz, ix, iy = np.meshgrid(np.arange(sz), np.arange(sx), np.arange(sy), indexing='ij')
        self.x = (minx + ix * stx).ravel().astype(np.int64)
        self.y = (miny + iy * sty).ravel().astype(np.int64)
        self.z = (minz + iz * stz).ravel().astype(np.int64)

    def key(self):
        return self.s + self.min + self.st


def plan(M, n):
    """BinaryFunction compile-time decision (volume_eval.cpp:38-71)."""
    L, R = M.node(n['l']), M.node(n['r'])
    lc, rc = L['t'] == 'constant', R['t'] == 'constant'
    op = n['op']
    if op == 'div' and not lc and rc:
        return 'divc', n['l'], n['r']
    if op in ('add', 'sub', 'mul', 'div'):
        return op, n['l'], n['r']
    lmin, lmax, rmin, rmax = f32(L['range'][0]), f32(L['range'][1]), f32(R['range'][0]), f32(R['range'][1])
    if op == 'min':
        if lmax < rmin:
            return 'pass', n['l'], None
        if rmax < lmin:
            return 'pass', n['r'], None
    else:
        if lmin > rmax:
            return 'pass', n['l'], None
        if rmin > lmax:
            return 'pass', n['r'], None
    return (op, n['r'], n['l']) if lc else (op, n['l'], n['r'])


def gradient(n, c):
    frm, to = n['from'], n['to']
    rng = to - frm
    fv, tv = f32(n['from_value']), f32(n['to_value'])
    factor = F32((tv - fv) / F32(rng))
    c = np.asarray(c, np.int64)
    if n['tiling'] == 'clamp_to_edge':
        rel = np.clip(c, min(frm, to), max(frm, to)) - frm
        return (fv + rel.astype(F32) * factor).astype(F32)
    rel = c - frm
    if n['tiling'] == 'repeat':
        return (fv + np.mod(rel, rng).astype(F32) * factor).astype(F32)
    tile = np.floor_divide(rel, rng)
    local = rel - tile * rng
    return np.where(tile & 1 == 0, fv + local.astype(F32) * factor, fv + (rng - local).astype(F32) * factor).astype(F32)


def squeeze(x):
    c = jclamp(x, -1.0, 1.0)
    return (c / F32(2) - ((c * c) * c) / F32(24)).astype(F32)


UNARY = {
    'abs': lambda x: np.abs(x).astype(F32),
    'square': lambda x: (x * x).astype(F32),
    'cube': lambda x: (x * x * x).astype(F32),
    'sqrt': lambda x: np.sqrt(x.astype(F64)).astype(F32),
    'half_negative': lambda x: np.where(x > 0, x, x * F32(0.5)).astype(F32),
    'quarter_negative': lambda x: np.where(x > 0, x, x * F32(0.25)).astype(F32),
    'reciprocal': lambda x: (F32(1) / x).astype(F32),
    'negate': lambda x: (-x).astype(F32),
    'squeeze': lambda x: squeeze(x),
    'sign': lambda x: np.where(np.isnan(x) | (x == 0), x, np.where(x > 0, F32(1), F32(-1))).astype(F32),
}


def spline_eval(s, coord_value):
    """CubicSpline.Multipoint.sample (volume_eval.cpp:339-355, :511-541), elementwise."""
    if 'k' in s:
        return None, f32(s['k'])
    x = coord_value(s['coord'])
    loc = np.array([f32(b) for b in s['loc']], F32)
    der = np.array([f32(b) for b in s['der']], F32)
    n = len(loc)
    start = np.sum(~(x[:, None] < loc[None, :]), axis=1) - 1
    out = np.zeros(x.shape, F32)
    for st in range(-1, n):
        sel = start == st
        if not sel.any():
            continue
        xi = x[sel]
        if st < 0 or st == n - 1:
            j = 0 if st < 0 else n - 1
            v = value_of(s['val'][j], coord_value, sel)
            out[sel] = v if der[j] == 0 else (v + der[j] * (xi - loc[j])).astype(F32)
        else:
            x1, x2, d1, d2 = loc[st], loc[st + 1], der[st], der[st + 1]
            y1 = value_of(s['val'][st], coord_value, sel)
            y2 = value_of(s['val'][st + 1], coord_value, sel)
            dx = F32(x2 - x1)
            t = ((xi - x1) / dx).astype(F32)
            dy = (y2 - y1).astype(F32)
            a = (d1 * dx - dy).astype(F32)
            b = ((-d2) * dx + dy).astype(F32)
            out[sel] = (lerp(t, y1, y2) + t * (F32(1) - t) * lerp(t, a, b)).astype(F32)
    return x, out


def value_of(s, coord_value, sel):
    if 'k' in s:
        return np.full(int(sel.sum()), f32(s['k']), F32)
    sub = lambda c: coord_value(c)[sel]
    return spline_eval(s, sub)[1]


class Evaluator:
    def __init__(self, model, seed):
        self.M = model
        self.S = seed
        self.cache = {}

    # VolumeEvaluator::sample (volume_eval.cpp:111-328)
    def sample(self, i, v):
        k = (i, v.key())
        if k in self.cache:
            return self.cache[k]
        out = self._sample(i, v)
        self.cache[k] = out
        return out

    def _sample(self, i, v):
        M, S = self.M, self.S
        n = M.node(i)
        t = n['t']
        size = v.x.size
        if t in ('cache', 'blend_density'):
            return self.sample(n['in'], v)
        if t == 'constant':
            return np.full(size, f32(n['v']), F32)
        if t == 'simple':
            return np.full(size, F32(1) if n['kind'] == 'blend_alpha' else F32(0), F32)
        if t == 'gradient':
            return gradient(n, {'x': v.x, 'y': v.y, 'z': v.z}[n['axis']])
        if t == 'noise':
            ref = S.noise[n['noise']]
            xz, ys = f64(n['xz_scale']), f64(n['y_scale'])
            if n['shift_x_zero'] and n['shift_y_zero'] and n['shift_z_zero']:
                return stack_volume(S, ref, v.x, v.y, v.z, xz, ys, 1.0, False)
            sx = self.sample(n['shift_x'], v).astype(F64)
            sz = self.sample(n['shift_z'], v).astype(F64)
            ny = v.y.astype(F64) * ys
            if not n['shift_y_zero']:
                ny = ny + self.sample(n['shift_y'], v).astype(F64)
            return stack_point(S, ref, v.x.astype(F64) * xz + sx, ny, v.z.astype(F64) * xz + sz)
        if t in ('shift_a', 'shift'):
            ref = S.noise[n['noise']]
            return (stack_volume(S, ref, v.x, v.y, v.z, 0.25, 0.0 if t == 'shift_a' else 0.25, 1.0, False) * F32(4)).astype(F32)
        if t == 'shift_b':
            ref = S.noise[n['noise']]
            return stack_volume(S, ref, v.z, v.x, np.zeros_like(v.x), 0.25, 0.25, 4.0, False)
        if t == 'blended_noise':
            mn, mx, main = S.blended[i]
            xzm, ym = 684.412 * f64(n['xz_scale']), 684.412 * f64(n['y_scale'])
            a = stack_volume(S, main, v.x, v.y, v.z, xzm / f64(n['xz_factor']), ym / f64(n['y_factor']), 1.0, True)
            a = jclamp((a + F32(0.5)).astype(F32), 0.0, 1.0)
            lo = stack_volume(S, mn, v.x, v.y, v.z, xzm, ym, 1.0, True)
            hi = stack_volume(S, mx, v.x, v.y, v.z, xzm, ym, 1.0, True)
            return np.where(a == 0, lo, np.where(a == 1, hi, lerp(a, lo, hi))).astype(F32)
        if t == 'binary':
            kind, a, b = plan(M, n)
            if kind == 'pass':
                return self.sample(a, v)
            A = self.sample(a, v)
            if kind == 'divc':
                return (A * (F32(1) / f32(M.node(b)['v']))).astype(F32)
            B = self.sample(b, v)
            return {'add': lambda: A + B, 'sub': lambda: A - B, 'mul': lambda: A * B, 'div': lambda: A / B,
                    'min': lambda: np.where(B < A, B, A), 'max': lambda: np.where(B > A, B, A)}[kind]().astype(F32)
        if t == 'unary':
            with np.errstate(all='ignore'):
                return UNARY[n['op']](self.sample(n['in'], v))
        if t == 'clamp':
            return jclamp(self.sample(n['in'], v), f32(n['min']), f32(n['max']))
        if t == 'lerp':
            a = self.sample(n['alpha'], v)
            f, s = self.sample(n['first'], v), self.sample(n['second'], v)
            return np.where(a == 0, f, np.where(a == 1, s, lerp(a, f, s))).astype(F32)
        if t == 'range_choice':
            c = self.sample(n['in'], v)
            ins = (c >= f32(n['min_inclusive'])) & (c < f32(n['max_exclusive']))
            return np.where(ins, self.sample(n['when_in'], v), self.sample(n['when_out'], v)).astype(F32)
        if t == 'interval_select':
            c = self.sample(n['in'], v)
            ths = [f32(b) for b in n['thresholds']]
            sel = np.full(size, len(ths), np.int64)
            for k in reversed(range(len(ths))):
                sel = np.where(c < ths[k], k, sel)
            out = np.zeros(size, F32)
            for k, fn in enumerate(n['functions']):
                if (sel == k).any():
                    out = np.where(sel == k, self.sample(fn, v), out)
            return out.astype(F32)
        if t == 'spline':
            return np.broadcast_to(spline_eval(n['spline'], lambda c: self.sample(c, v))[1], (size,)).astype(F32)
        if t == 'interpolated':
            return self.interpolated(n, v)
        if t == 'slice':
            return self.slice(n, v)
        if t == 'find_top_surface':
            v0 = Volume(v.s[0], 1, v.s[2], v.min[0], 0, v.min[2], *v.st) if not (v.s[1] == 1 and v.min[1] == 0) else v
            ub = self.sample(n['upper_bound'], v0)
            col = self.surface(n, v0.x, v0.z, ub)
            return np.repeat(col, v.s[1])
        raise ValueError(t)

    def slice(self, n, v):
        inner = self.M.node(n['in'])
        sx, sy, sz = v.s
        if inner['t'] == 'slice' and {n['axis'], inner['axis']} == {'x', 'z'}:
            x = n['coord'] if n['axis'] == 'x' else inner['coord']
            z = inner['coord'] if n['axis'] == 'x' else n['coord']
            iv = Volume(1, sy, 1, x, v.min[1], z, *v.st)
            col = self.sample(inner['in'], iv)
            return np.tile(col, sx * sz)
        ax = 'xyz'.index(n['axis'])
        s = list(v.s)
        mn = list(v.min)
        s[ax] = 1
        mn[ax] = n['coord']
        iv = Volume(*s, *mn, *v.st)
        buf = self.sample(n['in'], iv).reshape(s[2], s[0], s[1])
        rep = np.broadcast_to(buf, (sz, sx, sy))
        return np.ascontiguousarray(rep).ravel()

    def interpolated(self, n, v):
        cxz, cy = n['cell_xz'], n['cell_y']
        (sx, sy, sz), (mnx, mny, mnz), (stx, sty, stz) = v.s, v.min, v.st
        if ((stx == cxz or sx == 1) and (sty == cy or sy == 1) and (stz == cxz or sz == 1) and mnx % cxz == 0 and mny % cy == 0
                and mnz % cxz == 0):
            return self.sample(n['in'], v)
        if not (stx == sty == stz == 1):
            bv = Volume(sx * stx, sy * sty, sz * stz, mnx, mny, mnz)
            bb = self.interpolated(n, bv).reshape(sz * stz, sx * stx, sy * sty)
            return bb[::stz, ::stx, ::sty][:sz, :sx, :sy].ravel()
        return self.block_step(n, v)

    def block_step(self, n, v):
        """InterpolatedFunction over a unit-stride volume: corners, then z, x, y steps."""
        cxz, cy = n['cell_xz'], n['cell_y']
        (sx, sy, sz), (mnx, mny, mnz) = v.s, v.min
        mx, my, mz = mnx + sx - 1, mny + sy - 1, mnz + sz - 1
        c0 = (mnx // cxz, mny // cy, mnz // cxz)
        cnt = (mx // cxz - c0[0] + 1, my // cy - c0[1] + 1, mz // cxz - c0[2] + 1)
        cs = (cnt[0] + (mx % cxz != 0), cnt[1] + (my % cy != 0), cnt[2] + (mz % cxz != 0))
        cv = Volume(cs[0], cs[1], cs[2], c0[0] * cxz, c0[1] * cy, c0[2] * cxz, cxz, cy, cxz)
        cb = self.sample(n['in'], cv).reshape(cs[2], cs[0], cs[1])
        out = np.zeros((sz, sx, sy), F32)
        inv_xz, inv_y = F32(1) / F32(cxz), F32(1) / F32(cy)
        for cz in range(cnt[2]):
            nz = min(cz + 1, cs[2] - 1)
            for cx in range(cnt[0]):
                nx = min(cx + 1, cs[0] - 1)
                for cyy in range(cnt[1]):
                    ny = min(cyy + 1, cs[1] - 1)
                    v000, v100, v001, v101 = cb[cz, cx, cyy], cb[cz, nx, cyy], cb[nz, cx, cyy], cb[nz, nx, cyy]
                    v010, v110, v011, v111 = cb[cz, cx, ny], cb[cz, nx, ny], cb[nz, cx, ny], cb[nz, nx, ny]
                    ox, oy, oz = c0[0] * cxz + cx * cxz - mnx, c0[1] * cy + cyy * cy - mny, c0[2] * cxz + cz * cxz - mnz
                    x0, y0, z0 = max(0, -ox), max(0, -oy), max(0, -oz)
                    x1, y1, z1 = min(cxz, sx - ox) - 1, min(cy, sy - oy) - 1, min(cxz, sz - oz) - 1
                    for z in range(z0, z1 + 1):
                        az = F32(F32(z) * inv_xz)
                        v00, v01 = lerp(az, v000, v001), lerp(az, v010, v011)
                        v10, v11 = lerp(az, v100, v101), lerp(az, v110, v111)
                        for x in range(x0, x1 + 1):
                            ax = F32(F32(x) * inv_xz)
                            a0, a1 = lerp(ax, v00, v10), lerp(ax, v01, v11)
                            step = F32((a1 - a0) * inv_y)
                            val = F32(a0 + step * F32(y0))
                            for y in range(y0, y1 + 1):
                                out[oz + z, ox + x, oy + y] = val
                                val = F32(val + step)
        return out.ravel()

    def surface(self, n, x, z, ub):
        """find_top_surface probes (volume_eval.cpp:330-337), point path."""
        cell, lower = n['cell_height'], n['lower_bound']
        top = jfloor((ub / F32(cell)).astype(F64)) * cell
        res = np.full(x.shape, F32(lower), F32)
        active = top > lower
        probe = np.where(active, top, lower)
        while active.any():
            idx = np.nonzero(active)[0]
            d = self.point(n['density'], x[idx], probe[idx], z[idx])
            hit = d > 0
            res[idx[hit]] = probe[idx[hit]].astype(F32)
            active[idx[hit]] = False
            probe[idx] -= cell
            active &= probe >= lower
        return res

    # VolumeEvaluator::point (volume_eval.cpp:357-509), elementwise over positions
    def point(self, i, x, y, z):
        M, S = self.M, self.S
        n = M.node(i)
        t = n['t']
        x, y, z = (np.asarray(a, np.int64) for a in (x, y, z))
        x, y, z = np.broadcast_arrays(x, y, z)
        P = lambda j, xx=x, yy=y, zz=z: self.point(j, xx, yy, zz)
        if t in ('cache', 'blend_density'):
            return P(n['in'])
        if t == 'constant':
            return np.full(x.shape, f32(n['v']), F32)
        if t == 'simple':
            return np.full(x.shape, F32(1) if n['kind'] == 'blend_alpha' else F32(0), F32)
        if t == 'gradient':
            return gradient(n, {'x': x, 'y': y, 'z': z}[n['axis']])
        if t == 'noise':
            ref = S.noise[n['noise']]
            xz, ys = f64(n['xz_scale']), f64(n['y_scale'])
            if n['shift_x_zero'] and n['shift_y_zero'] and n['shift_z_zero']:
                return stack_point(S, ref, x.astype(F64) * xz, y.astype(F64) * ys, z.astype(F64) * xz)
            nx = x.astype(F64) * xz + P(n['shift_x']).astype(F64)
            ny = y.astype(F64) * ys
            if not n['shift_y_zero']:
                ny = ny + P(n['shift_y']).astype(F64)
            nz = z.astype(F64) * xz + P(n['shift_z']).astype(F64)
            return stack_point(S, ref, nx, ny, nz)
        if t in ('shift_a', 'shift', 'shift_b'):
            ref = S.noise[n['noise']]
            if t == 'shift_b':
                v = stack_point(S, ref, z.astype(F64) * 0.25, x.astype(F64) * 0.25, np.zeros(x.shape))
            else:
                v = stack_point(S, ref, x.astype(F64) * 0.25, y.astype(F64) * (0.0 if t == 'shift_a' else 0.25), z.astype(F64) * 0.25)
            return (v * F32(4)).astype(F32)
        if t == 'blended_noise':
            mn, mx, main = S.blended[i]
            xzm, ym = 684.412 * f64(n['xz_scale']), 684.412 * f64(n['y_scale'])
            mxz, my = xzm / f64(n['xz_factor']), ym / f64(n['y_factor'])
            a = stack_point(S, main, x * mxz, y * my, z * mxz, True)
            a = jclamp((a + F32(0.5)).astype(F32), 0.0, 1.0)
            lo = stack_point(S, mn, x * xzm, y * ym, z * xzm, True)
            hi = stack_point(S, mx, x * xzm, y * ym, z * xzm, True)
            return np.where(a == 0, lo, np.where(a == 1, hi, lerp(a, lo, hi))).astype(F32)
        if t == 'binary':
            L, R = M.node(n['l']), M.node(n['r'])
            lc, rc = L['t'] == 'constant', R['t'] == 'constant'
            op = n['op']
            with np.errstate(all='ignore'):
                if op == 'add':
                    return (P(n['l']) + P(n['r'])).astype(F32)
                if op == 'sub':
                    return (P(n['l']) - P(n['r'])).astype(F32)
                if op == 'mul':
                    a = P(n['l'])
                    if lc or rc:
                        return (a * P(n['r'])).astype(F32)
                    return np.where(a == 0, F32(0), a * P(n['r'])).astype(F32)
                if op == 'div':
                    if lc:
                        return (f32(L['v']) / P(n['r'])).astype(F32)
                    if rc:
                        return (P(n['l']) * (F32(1) / f32(R['v']))).astype(F32)
                    a = P(n['l'])
                    return np.where(a == 0, F32(0), a / P(n['r'])).astype(F32)
            kind, a_id, b_id = plan(M, n)
            if kind == 'pass':
                return P(a_id)
            fn = jmin if op == 'min' else jmax
            if lc or rc:
                return fn(P(a_id), f32(M.node(b_id)['v']))
            a = P(n['l'])
            if op == 'min':
                return np.where(a <= f32(R['range'][0]), a, jmin(a, P(n['r']))).astype(F32)
            return np.where(a >= f32(R['range'][1]), a, jmax(a, P(n['r']))).astype(F32)
        if t == 'unary':
            with np.errstate(all='ignore'):
                return UNARY[n['op']](P(n['in']))
        if t == 'clamp':
            return jclamp(P(n['in']), f32(n['min']), f32(n['max']))
        if t == 'lerp':
            a = P(n['alpha'])
            f, s = P(n['first']), P(n['second'])
            return np.where(a == 0, f, np.where(a == 1, s, lerp(a, f, s))).astype(F32)
        if t == 'range_choice':
            c = P(n['in'])
            ins = (c >= f32(n['min_inclusive'])) & (c < f32(n['max_exclusive']))
            return np.where(ins, P(n['when_in']), P(n['when_out'])).astype(F32)
        if t == 'interval_select':
            c = P(n['in'])
            ths = [f32(b) for b in n['thresholds']]
            out = P(n['functions'][-1])
            for k in reversed(range(len(ths))):
                out = np.where(c < ths[k], P(n['functions'][k]), out)
            return out.astype(F32)
        if t == 'spline':
            return np.broadcast_to(spline_eval(n['spline'], lambda c: P(c))[1], x.shape).astype(F32)
        if t == 'interpolated':
            cxz, cy = n['cell_xz'], n['cell_y']
            out = np.empty(x.shape, F32)
            for k in range(x.size):
                px, py, pz = int(x.flat[k]), int(y.flat[k]), int(z.flat[k])
                xi, yi, zi = px % cxz, py % cy, pz % cxz
                if xi == 0 and yi == 0 and zi == 0:
                    out.flat[k] = self.point(n['in'], [px], [py], [pz])[0]
                    continue
                c = self.sample(n['in'], Volume(2, 2, 2, px - xi, py - yi, pz - zi, cxz, cy, cxz)).reshape(2, 2, 2)   # [z][x][y]
                out.flat[k] = lerp3(F32(F32(xi) / F32(cxz)), F32(F32(yi) / F32(cy)), F32(F32(zi) / F32(cxz)), c[0, 0, 0], c[0, 1, 0], c[0, 0, 1], c[0, 1, 1],
                                    c[1, 0, 0], c[1, 1, 0], c[1, 0, 1], c[1, 1, 1])
            return out
        if t == 'slice':
            c = {'x': x, 'y': y, 'z': z}
            c[n['axis']] = np.full(x.shape, n['coord'], np.int64)
            return self.point(n['in'], c['x'], c['y'], c['z'])
        if t == 'find_top_surface':
            ub = self.point(n['upper_bound'], x, np.zeros_like(y), z)
            return self.surface(n, x, z, ub)
        raise ValueError('point path: %s' % t)


# ---- climate R-tree (cpu/src/biome.cpp:95-236) --------------------------------------------
class ClimateTree:
    def __init__(self, params):
        self.mn, self.mx, self.kids, self.leaf = [], [], [], []
        self.biome = []
        for i, p in enumerate(params):
            self.mn.append([p['p'][2 * d] for d in range(6)] + [p['offset']])
            self.mx.append([p['p'][2 * d + 1] for d in range(6)] + [p['offset']])
            self.kids.append([])
            self.leaf.append(i)
            self.biome.append(p['biome'])
        self.root = self.build(list(range(len(params))))
        self.leaf_node = {l: i for i, l in enumerate(self.leaf) if l >= 0}

    def subtree(self, kids):
        self.mn.append([min(self.mn[k][d] for k in kids) for d in range(7)])
        self.mx.append([max(self.mx[k][d] for k in kids) for d in range(7)])
        self.kids.append(list(kids))
        self.leaf.append(-1)
        return len(self.kids) - 1

    def cent(self, k, d):
        s = self.mn[k][d] + self.mx[k][d]
        return s // 2 if s >= 0 else -((-s) // 2)     # Java long division truncates

    def build(self, kids):
        if len(kids) == 1:
            return kids[0]
        if len(kids) <= 19:
            kids = sorted(kids, key=lambda k: sum(abs(self.cent(k, d)) for d in range(7)))
            return self.subtree(kids)
        group = int(19 ** math.floor(math.log(len(kids) - 0.01) / math.log(19)))
        best = None
        for dim in range(7):
            kids = sorted(kids, key=lambda k: tuple(self.cent(k, (dim + j) % 7) for j in range(7)))
            buckets = [kids[i:i + group] for i in range(0, len(kids), group)]
            cost = sum(abs(max(self.mx[k][d] for k in b) - min(self.mn[k][d] for k in b)) for b in buckets for d in range(7))
            if best is None or cost < best[0]:
                best = (cost, dim, buckets)
        _, dim, buckets = best
        bnodes = [self.subtree(b) for b in buckets]
        bnodes = sorted(bnodes, key=lambda k: tuple(abs(self.cent(k, (dim + j) % 7)) for j in range(7)))
        return self.subtree([self.build(self.kids[b]) for b in bnodes])

    def dist(self, k, t):
        d = 0
        for i in range(7):
            p = t[i] - self.mx[k][i]
            q = self.mn[k][i] - t[i]
            d += (p if p > 0 else max(q, 0)) ** 2
        return d

    def search(self, t, cand_leaf):
        cand = -1 if cand_leaf < 0 else self.leaf_node[cand_leaf]

        def rec(node, cand):
            if self.leaf[node] >= 0:
                return node
            md = (1 << 63) - 1 if cand < 0 else self.dist(cand, t)
            closest = cand
            for c in self.kids[node]:
                cd = self.dist(c, t)
                if md > cd:
                    leaf = rec(c, closest)
                    ld = cd if c == leaf else self.dist(leaf, t)
                    if md > ld:
                        md, closest = ld, leaf
            return closest
        return self.leaf[rec(self.root, cand)]


def quantize(v):
    with np.errstate(over='ignore'):
        v = np.asarray(v, F32) * F32(10000)
    with np.errstate(invalid='ignore'):
        out = np.where(np.isnan(v), 0, np.clip(v.astype(F64), -9.2233720368547758e18, 9.2233720368547758e18))
    r = [int(a) if abs(a) < 9.2233720368547758e18 else ((1 << 63) - 1 if a > 0 else -(1 << 63)) for a in out]
    return r


def chunk_biomes(model, seed, ev, cx, cz):
    """cpu_chunk_biomes (cpu/src/terrain.cpp:152-176)."""
    qh = model.height // 4
    v = Volume(4, qh, 4, cx * 16, model.min_y, cz * 16, 4, 4, 4)
    names = ('temperature', 'vegetation', 'continents', 'erosion', 'depth', 'ridges')
    bufs = [quantize(ev.sample(model.roots['climate/' + k], v)) for k in names]
    out = np.zeros(16 * qh, np.uint8)
    last = -1
    T = model.tree
    for sy in range(qh // 4):
        for x in range(4):
            for y in range(4):
                for z in range(4):
                    qy = sy * 4 + y
                    idx = qy + (x + z * 4) * qh
                    t = [bufs[k][idx] for k in range(6)] + [0]
                    last = T.search(t, last)
                    out[(qy * 4 + z) * 4 + x] = T.biome[last]
    return out


def zoom(zoom_seed, x, y, z, quart_biome):
    """BiomeManager.getBiome (cpu/src/biome.cpp:241-289)."""
    def lcg(r, c):
        return s64(r * (r * 6364136223846793005 + 1442695040888963407) + c)

    def fid(r):
        return ((r >> 24) % 1024 / 1024.0 - 0.5) * 0.9
    ax, ay, az = x - 2, y - 2, z - 2
    px, py, pz = ax >> 2, ay >> 2, az >> 2
    fx, fy, fz = (ax & 3) / 4.0, (ay & 3) / 4.0, (az & 3) / 4.0
    best, bd = 0, math.inf
    for i in range(8):
        xe, ye, ze = (i & 4) == 0, (i & 2) == 0, (i & 1) == 0
        qx, qy, qz = (px if xe else px + 1), (py if ye else py + 1), (pz if ze else pz + 1)
        r = zoom_seed
        for c in (qx, qy, qz, qx, qy, qz):
            r = lcg(r, c)
        ox = fid(r)
        r = lcg(r, zoom_seed)
        oy = fid(r)
        r = lcg(r, zoom_seed)
        oz = fid(r)
        dx, dy, dz = (fx if xe else fx - 1.0), (fy if ye else fy - 1.0), (fz if ze else fz - 1.0)
        d = (dz + oz) * (dz + oz) + (dy + oy) * (dy + oy) + (dx + ox) * (dx + ox)
        if bd > d:
            best, bd = i, d
    return quart_biome((px if best & 4 == 0 else px + 1), (py if best & 2 == 0 else py + 1), (pz if best & 1 == 0 else pz + 1))
