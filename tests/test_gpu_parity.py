"""GPU parity: the sm_100a TERRAIN step through the C ABI against the reference port.

Bar: bit-exact for every block state (u16) and every quart biome (u8), zero tolerance
(integer outputs). Reference: cpu_generate_terrain / cpu_terrain_from_biomes
(cpu/src/terrain.cpp:750-810) compiled from the reference's own sources (oracle/_ref).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SEEDS = [0, 1, -1, 12345, -9223372036854775808, 9223372036854775807, 2147483648, -2147483648, -4172144997902289642]

# chunk sets: origin block, near / far / world border (reference corpus positions),
# the 32-bit noise-lattice wrap chunks, the literal +/-117,187 border reading, and
# chunks whose surface biomes trigger the eroded-badlands and frozen-ocean extensions, and
# chunks past the BlockPos wrap of the aquifer cell locations (|c| from 2^21 - 1 to the
# accepted 2^23 - 1)
CHUNKS = [(0, 0), (1, 0), (0, 1), (-1, -1), (6250, -6250), (-625000, 625000), (1874999, -1874999), (-1874999, 1874999), (6128, -6129),
          (-6129, 6128), (117187, -117187), (-4000, -3360), (-4000, -1440), (-4000, 1600), (2097148, -2097149), (3000000, -5000000),
          (-8388607, 8388607)]


def compare(got_blocks, got_biomes, ref_blocks, ref_biomes, chunks):
    for i, c in enumerate(chunks):
        nb = int((got_blocks[i] != ref_blocks[i]).sum())
        nq = int((got_biomes[i] != ref_biomes[i]).sum())
        assert nb == 0 and nq == 0, 'chunk %s: %d block and %d biome mismatches' % (c, nb, nq)


@pytest.mark.parametrize('seed', SEEDS[:5])
def test_chunks_match_reference(gpu_gen, ref_model, seed):
    gpu_gen.set_seed(seed)
    blocks, biomes = gpu_gen.generate(CHUNKS)
    rb, rq = ref_model.seed(seed).generate(CHUNKS)
    compare(blocks, biomes, rb, rq, CHUNKS)


def test_region_8x8_matches_reference(gpu_gen, ref_model):
    seed = 7
    chunks = [(x, z) for z in range(-4, 4) for x in range(-4, 4)]
    gpu_gen.set_seed(seed)
    blocks, biomes = gpu_gen.generate(chunks)
    rb, rq = ref_model.seed(seed).generate(chunks)
    compare(blocks, biomes, rb, rq, chunks)


def test_extreme_seeds(gpu_gen, ref_model):
    chunks = [(0, 0), (3, -2), (1874999, 1874999)]
    for seed in SEEDS[4:]:
        gpu_gen.set_seed(seed)
        blocks, biomes = gpu_gen.generate(chunks)
        rb, rq = ref_model.seed(seed).generate(chunks)
        compare(blocks, biomes, rb, rq, chunks)


def test_random_seeds_scattered_and_far_chunks(ref_model):
    """Random seeds, chunks scattered over +/-2M and across the whole accepted range (past
    the BlockPos wrap of the aquifer locations), and a small square, through tg_generate on
    a 4,096-chunk generator (host-output batches): every block and biome equals the
    reference."""
    import terrain_b200
    g = terrain_b200.TerrainGenerator(max_batch_chunks=4096)
    try:
        rng = np.random.default_rng(2026)
        for seed in [int(v) for v in rng.integers(-(1 << 63), (1 << 63) - 1, 4, dtype=np.int64)]:
            near = rng.integers(-2000000, 2000000, (160, 2))
            far = rng.integers(-8388607, 8388608, (24, 2))
            square = np.array([(x, z) for z in range(4) for x in range(4)]) + rng.integers(-100000, 100000, 2)
            chunks = np.concatenate([near, far, square]).astype(np.int32)
            g.set_seed(seed)
            b, q = g.generate(chunks)
            rb, rq = ref_model.seed(seed).generate([tuple(int(v) for v in c) for c in chunks])
            compare(b, q, rb, rq, [tuple(c) for c in chunks])
    finally:
        g.close()
