"""tg_biome_lookup_noalloc, the lookup that allocates nothing (for callers that cannot
allocate device memory after start-up), called through the C ABI: compared with
tg_biome_lookup on the same positions over two calls in a row (the largest allowed call,
then a smaller one, so stale scratch contents cannot pass), with the reference port's
zoomed_biome over cpu_chunk_biomes (cpu/src/biome.cpp:272-289, cpu/src/terrain.cpp:152-176)
on positions at chunk edges and above and below the world, and the size limit. Integer
results, zero tolerance. Collected last; passes alone in a fresh process and after the
other tests."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SEED = 20240607
LIMIT = 4096


def positions(rng, n):
    return np.ascontiguousarray(np.stack([rng.integers(-3000, 3000, n), rng.integers(-80, 330, n), rng.integers(-3000, 3000, n)], 1), np.int32)


@pytest.fixture(scope='module')
def gen():
    import terrain_b200
    g = terrain_b200.TerrainGenerator(max_batch_chunks=LIMIT)
    g.set_seed(SEED)
    yield g
    g.close()


def test_noalloc_equals_lookup_on_two_calls_in_a_row(gen):
    L, h = gen.L, gen.h
    rng = np.random.default_rng(7)
    for xyz in (positions(rng, LIMIT), positions(rng, 777)):
        n = xyz.shape[0]
        got = np.full(n, 0xEE, np.uint8)
        st = L.tg_biome_lookup_noalloc(h, ctypes.c_void_p(xyz.ctypes.data), n, ctypes.c_void_p(got.ctypes.data))
        assert st == 0, L.tg_last_error_string().decode()
        seeds = np.full(n, SEED, np.int64)
        want = np.full(n, 0xDD, np.uint8)
        st = L.tg_biome_lookup(h, ctypes.c_void_p(seeds.ctypes.data), ctypes.c_void_p(xyz.ctypes.data), n, ctypes.c_void_p(want.ctypes.data))
        assert st == 0, L.tg_last_error_string().decode()
        assert np.unique(want).size > 1
        assert np.array_equal(got, want)


def test_noalloc_rejects_sizes_beyond_the_limit(gen):
    L, h = gen.L, gen.h
    xyz = np.zeros((LIMIT + 1, 3), np.int32)
    out = np.zeros(LIMIT + 1, np.uint8)
    st = L.tg_biome_lookup_noalloc(h, ctypes.c_void_p(xyz.ctypes.data), LIMIT + 1, ctypes.c_void_p(out.ctypes.data))
    assert st == 1                                            # TG_ERR_INVALID_ARGUMENT
    assert b'4,096' in L.tg_last_error_string()
    # the generator stays usable after the rejection
    ok = positions(np.random.default_rng(3), 64)
    st = L.tg_biome_lookup_noalloc(h, ctypes.c_void_p(ok.ctypes.data), 64, ctypes.c_void_p(out.ctypes.data))
    assert st == 0, L.tg_last_error_string().decode()


def test_noalloc_equals_reference_port(gen, ref_model):
    """Chunk-edge x / z (block 0 and 15 of a chunk, where the zoom reaches the neighbour
    chunk) and y below and above the world (the quart y is clamped) against the port."""
    rng = np.random.default_rng(11)
    n = 1024
    edge = rng.choice(np.array([0, 1, 14, 15]), (n, 2))
    cx, cz = rng.integers(-3000, 3000, n), rng.integers(-3000, 3000, n)
    y = np.concatenate([rng.integers(-200, -64, n // 4), rng.integers(-64, 320, n // 2), rng.integers(320, 500, n - n // 4 - n // 2)])
    xyz = np.ascontiguousarray(np.stack([cx * 16 + edge[:, 0], y, cz * 16 + edge[:, 1]], 1), np.int32)
    got = gen.biome_lookup_noalloc(xyz)
    want = ref_model.seed(SEED).biome_lookup(xyz)
    assert np.unique(want).size > 1
    bad = np.nonzero(got != want)[0]
    assert bad.size == 0, 'positions differing from the reference: %s' % xyz[bad[:10]].tolist()
