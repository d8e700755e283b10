"""tg_biome_lookup_noalloc, the lookup that allocates nothing, called through the C ABI and
compared with tg_biome_lookup on the same positions: two calls in a row (the largest
allowed call, then a smaller one, so stale scratch contents cannot pass), and the size
limit. Collected last; passes alone in a fresh process and after the other tests."""
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
