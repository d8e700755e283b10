"""The numpy restatement (oracle/restate.py), pinned two ways: against the committed golden
fixtures (known-answer vectors and the per-chunk biome digests the reference's port wrote)
and, where oracle/_ref is built, against the reference's own C++ port on the same inputs:
per-seed noise tables, every named density root through both the volume path and the
point path, chunk biomes and the zoomed biome lookup. All comparisons are bit-exact."""
import ctypes
import hashlib
import json
import math
import os

import numpy as np
import pytest

import restate

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
MODEL_DIR = os.path.join(REPO, 'minecraft-terrain-cuda_b200', 'model')
KAT = json.load(open(os.path.join(REPO, 'tests', 'golden', 'kat.json')))
GOLDEN = json.load(open(os.path.join(REPO, 'tests', 'golden', 'terrain_digests.json')))
SEEDS = (123456789, -4172144997902289642)


@pytest.fixture(scope='module')
def model():
    return restate.Model(os.path.join(MODEL_DIR, 'overworld_ir.json'), os.path.join(MODEL_DIR, 'overworld_terrain.json'))


def bits(a):
    return np.ascontiguousarray(np.asarray(a, np.float32)).view(np.uint32)


def test_kat_rng_and_hash_vectors():
    for seed, longs in KAT['xoroshiro_longs'].items():
        r = restate.Xoroshiro.from_seed(int(seed))
        assert [restate.s64(r.next()) for _ in longs] == longs
    for x, y, z, want in KAT['mth_get_seed']:
        assert restate.mth_get_seed(x, y, z) == want
    for v, want in KAT['quantize']:
        assert restate.quantize([v])[0] == want
    for vals, want in KAT['stream_sum']:
        got = restate.stream_sum(vals)
        assert got == want or (math.isnan(got) and math.isnan(want))
    for seed, want in KAT['zoom_seed'].items():
        z = hashlib.sha256((int(seed) & restate.M64).to_bytes(8, 'little')).digest()
        assert restate.s64(int.from_bytes(z[:8], 'little')) == want


def test_java_semantics():
    assert restate.d2i(float('nan')) == 0 and restate.d2i(3e9) == 2147483647 and restate.d2i(-3e9) == -2147483648
    assert restate.jfloor(-0.5) == -1 and restate.jfloor(2.999) == 2
    assert np.signbit(restate.jmin(np.float32(0.0), np.float32(-0.0)))
    assert not np.signbit(restate.jmax(np.float32(-0.0), np.float32(0.0)))
    assert np.isnan(restate.jmin(np.float32('nan'), np.float32(1)))
    # the Java float literals 1.110223E-16F and 5.9604645E-8F round to 2^-53 and 2^-24
    assert restate.DOUBLE_UNIT == 2.0 ** -53 and restate.FLOAT_UNIT == np.float32(2.0 ** -24)
    # GradientNoise.wrap leaves |x| < 2^24 alone and folds larger values by 2^25
    assert restate.wrap(1.0e6) == 1.0e6 and restate.wrap(3.0e7) == 3.0e7 - 33554432.0


@pytest.mark.parametrize('seed_key', ['0', '-1', '-4172144997902289642'])
def test_chunk_biomes_match_golden_digests(model, seed_key):
    """Quart biomes of the restatement hash to the fixture digests (no reference needed)."""
    S = restate.Seed(model, int(seed_key))
    ev = restate.Evaluator(model, S)
    pick = [0, 4, 9, 13, 16]          # (-1,-1), (0,0), (6250,6250), (1874999,1874999), (-6129,0)
    for i in pick:
        cx, cz = GOLDEN['chunks'][i]
        b = restate.chunk_biomes(model, S, ev, cx, cz)
        assert hashlib.sha256(b.tobytes()).hexdigest() == GOLDEN['seeds'][seed_key][i][1], (seed_key, cx, cz)
        ev.cache.clear()


@pytest.mark.parametrize('seed', SEEDS)
def test_seed_tables_match_reference(model, ref_model, seed):
    S = restate.Seed(model, seed)
    rs = ref_model.seed(seed)
    for key, (first, count) in S.noise.items():
        f, amp, offs, perms = rs.noise_layers(key)
        assert len(f) == count, key
        for i in range(count):
            fr, a, oi = S.layers[first + i]
            ox, oy, oz, _, perm = S.octaves[oi]
            assert fr == f[i] and np.float32(a) == amp[i], (key, i)
            assert (ox, oy, oz) == tuple(offs[i]) and np.array_equal(perm, perms[i]), (key, i)
    sc, clay = rs.scalars()
    assert S.zoom_seed == sc[0]
    assert [restate.s64(v) for v in (*S.random, *S.aquifer, *S.ore)] == list(sc[1:7])
    assert np.array_equal(S.clay, clay)


@pytest.mark.parametrize('seed', SEEDS)
def test_density_roots_match_reference(model, ref_model, seed):
    """Every named root, volume path (quart grid and an off-grid unit-stride box that takes
    the interpolated block-step path) and point path, bit for bit."""
    S = restate.Seed(model, seed)
    rs = ref_model.seed(seed)
    ev = restate.Evaluator(model, S)
    rng = np.random.default_rng(seed & 0xFFFF)
    vols = ([4, 12, 4, 48, -64, -112, 4, 4, 4], [3, 10, 2, 5, 37, -3, 1, 1, 1], [2, 6, 2, 29999980, 90, -29999990, 4, 8, 4])
    for name, node in model.roots.items():
        for vol in vols:
            a = ev.sample(node, restate.Volume(*vol))
            assert np.array_equal(bits(a), bits(rs.sample(node, vol))), (name, vol)
        xyz = np.stack([rng.integers(-3000, 3000, 16), rng.integers(-64, 320, 16), rng.integers(-3000, 3000, 16)], 1)
        a = ev.point(node, xyz[:, 0], xyz[:, 1], xyz[:, 2])
        assert np.array_equal(bits(a), bits(rs.point(node, xyz))), name


def test_chunk_biomes_and_lookup_match_reference(model, ref_model):
    seed = SEEDS[0]
    S = restate.Seed(model, seed)
    rs = ref_model.seed(seed)
    ev = restate.Evaluator(model, S)
    qh = model.height // 4
    cache = {}

    def chunk(cx, cz):
        if (cx, cz) not in cache:
            cache[(cx, cz)] = restate.chunk_biomes(model, S, ev, cx, cz)
        return cache[(cx, cz)]

    for cx, cz in ((0, 0), (-7, 3), (117124, -62500)):
        want = np.empty(16 * qh, np.uint8)
        rs.L.ref_chunk_biomes(ctypes.c_void_p(rs.h), cx, cz, want.ctypes.data)
        assert np.array_equal(chunk(cx, cz), want), (cx, cz)
    qmin = model.min_y >> 2

    def quart(qx, qy, qz):
        cqy = min(max(qy, qmin), qmin + qh - 1) - qmin
        return chunk(qx >> 2, qz >> 2)[(cqy * 4 + (qz & 3)) * 4 + (qx & 3)]

    rng = np.random.default_rng(1)
    xyz = np.stack([rng.integers(-20, 20, 40), rng.integers(-70, 330, 40), rng.integers(-20, 20, 40)], 1).astype(np.int32)
    mine = np.array([restate.zoom(S.zoom_seed, int(x), int(y), int(z), quart) for x, y, z in xyz], np.uint8)
    assert np.array_equal(mine, rs.biome_lookup(xyz))


def test_planted_mistake_is_caught(model, ref_model):
    """A one-ulp change planted in the restatement's output fails the bit comparison."""
    S = restate.Seed(model, SEEDS[0])
    node = model.roots['final_density']
    vol = [3, 10, 2, 5, 37, -3, 1, 1, 1]
    a = restate.Evaluator(model, S).sample(node, restate.Volume(*vol)).copy()
    want = ref_model.seed(SEEDS[0]).sample(node, vol)
    assert np.array_equal(bits(a), bits(want))
    a[4] = np.nextafter(a[4], np.float32(1e9))
    assert not np.array_equal(bits(a), bits(want))
