"""The device code's arithmetic on the CPU: the host twin of the kernel bodies (the same
generated evaluators and per-element bodies, built for the host) against the reference
port, stage by stage and for whole chunks. Integer outputs and float evaluator values
are compared bit for bit."""
import json
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, 'hostcheck'))
import hostcheck  # noqa: E402

pytestmark = pytest.mark.skipif(not hostcheck.available(), reason='host twin not built')

SEEDS = [0, -(1 << 63), 4172144997902289642, 12345]


@pytest.fixture(scope='module')
def ir():
    import ref_oracle
    return json.load(open(ref_oracle.IR_PATH))


@pytest.mark.parametrize('seed', SEEDS)
def test_seed_tables(ref_model, ir, seed):
    rs = ref_model.seed(seed)
    a, clay = rs.scalars()
    b, clay2 = hostcheck.seed_scalars(seed)
    assert (a == b).all() and (clay == clay2).all()
    for k, key in enumerate(sorted(ir['noises'])):
        f1, a1, o1, p1 = rs.noise_layers(key)
        f2, a2, o2, p2 = hostcheck.noise_layers(seed, k)
        assert (f1 == f2).all() and (a1.view(np.uint32) == a2.view(np.uint32)).all() and (o1 == o2).all() and (p1 == p2).all(), key


@pytest.mark.parametrize('seed', SEEDS[:2])
def test_climate_and_corner_evaluators(ref_model, ir, seed):
    rs = ref_model.seed(seed)
    roots = [ir['roots']['climate/' + k] for k in ('temperature', 'vegetation', 'continents', 'erosion', 'depth', 'ridges')]
    sys.path.insert(0, os.path.join(os.path.dirname(HERE), 'minecraft-terrain-cuda_b200', 'codegen'))
    import gen_eval
    import ref_oracle
    G = gen_eval.Gen(gen_eval.Model(ref_oracle.IR_PATH, ref_oracle.TERRAIN_PATH))
    cin = [G.M.nodes[c]['in'] for c in G.chans]
    for cx, cz in [(0, 0), (6128, -6129), (-1874999, 1874999)]:
        vol = [4, 96, 4, cx * 16, -64, cz * 16, 4, 4, 4]
        want = np.stack([rs.sample(r, vol) for r in roots], 1)
        xyz = [(cx * 16 + 4 * x, -64 + 4 * y, cz * 16 + 4 * z) for z in range(4) for x in range(4) for y in range(96)]
        assert (hostcheck.climate(seed, xyz).view(np.uint32) == want.view(np.uint32)).all()
        vol = [5, 49, 5, cx * 16, -64, cz * 16, 4, 8, 4]
        want = np.stack([rs.sample(r, vol) for r in cin], 1)
        xyz = [(cx * 16 + 4 * x, -64 + 8 * y, cz * 16 + 4 * z) for z in range(5) for x in range(5) for y in range(49)]
        assert (hostcheck.corners(seed, xyz).view(np.uint32) == want.view(np.uint32)).all()


def test_point_path_roots(ref_model, ir):
    rng = np.random.default_rng(11)
    xyz = np.stack([rng.integers(-30000000, 30000000, 300), rng.integers(-64, 320, 300), rng.integers(-30000000, 30000000, 300)], 1)
    rs = ref_model.seed(77)
    for k, name in enumerate(['barrier', 'fluid_level_floodedness', 'fluid_level_spread', 'lava', 'exclusion']):
        want = rs.point(ir['roots']['aquifer/' + name], xyz)
        assert (hostcheck.point(77, k, xyz).view(np.uint32) == want.view(np.uint32)).all(), name


CHUNKS = [(0, 0), (-1, -1), (6128, -6129), (1874999, -1874999), (117187, -117187), (-4000, -3360), (-4000, -1440), (-4000, 1600),
          (2097148, -2097149), (3000000, -5000000), (-2097152, 4194303), (8388607, -8388607)]


@pytest.mark.parametrize('seed', [12345, -1])
def test_whole_chunks(ref_model, seed):
    b, q, aq = hostcheck.generate(seed, CHUNKS, aquifer=True)
    rb, rq, raq = ref_model.seed(seed).generate(CHUNKS, aquifer=True)
    for i, c in enumerate(CHUNKS):
        assert (q[i] == rq[i]).all(), c
        assert (aq[i] == raq[i]).all(), c
        assert (b[i] == rb[i]).all(), c


def test_random_chunks(ref_model):
    """Scattered chunks of random seeds: every aquifer decision (the nearest-cell scan and
    the per-query shortcuts) on terrain of all kinds, blocks after the fill and final."""
    rng = np.random.default_rng(5)
    for seed in [int(v) for v in rng.integers(-(1 << 62), 1 << 62, 3)]:
        chunks = [(int(a), int(b)) for a, b in zip(rng.integers(-200000, 200000, 24), rng.integers(-200000, 200000, 24))]
        b, q, aq = hostcheck.generate(seed, chunks, aquifer=True)
        rb, rq, raq = ref_model.seed(seed).generate(chunks, aquifer=True)
        assert (aq == raq).all() and (b == rb).all() and (q == rq).all(), seed


@pytest.mark.parametrize('per_chunk', [0, 1, 64])
def test_walk_deferred_list_sizes(ref_model, per_chunk):
    """The column walk leaves blocks whose rules need a per-block noise or an ore vein past
    its bit to a deferred pass; with no list, or one that fills after a few blocks (the
    rest run in the walk), the blocks are the same."""
    seed = 4172144997902289642
    chunks = CHUNKS[:6] + [(-62500, -62500), (-62499, -62500)]
    try:
        hostcheck.set_defer(per_chunk)
        b, q = hostcheck.generate(seed, chunks)
    finally:
        hostcheck.set_defer(8192)
    rb, rq = ref_model.seed(seed).generate(chunks)
    assert (b == rb).all() and (q == rq).all()
    per, meta = hostcheck.count_ops(seed, chunks)
    assert meta['deferred_blocks'] > 100 * len(chunks)


@pytest.mark.parametrize('seed', [123456789, -4172144997902289642])
def test_biome_point_lookups(ref_model, seed):
    """The single-position lookup path (zoom corner, the quart's minimum and tie test, the
    chunk chain replayed from the nearest earlier fixed quart) against the reference's
    zoomed_biome over whole-chunk quart biomes: scattered positions up to the world border,
    dense ones (tied quarts replay the chain), and y outside the world (clamped rows)."""
    rng = np.random.default_rng(seed & 0xFFFF)
    far = np.stack([rng.integers(-1874999, 1875000, 300), rng.integers(-64, 320, 300), rng.integers(-1874999, 1875000, 300)], 1)
    near = np.stack([rng.integers(-40, 40, 300), rng.integers(-90, 345, 300), rng.integers(-40, 40, 300)], 1)
    xyz = np.ascontiguousarray(np.concatenate([far, near]).astype(np.int32))
    assert (hostcheck.biome_point(seed, xyz) == ref_model.seed(seed).biome_lookup(xyz)).all()


def test_dedupe_table_errors_are_reported():
    """The dedupe tables' invariant checks on the host build of the same code: keys within
    the capacity number 0..n-1 with no error bit; more keys than slots set the full bit
    (an insert found no slot) and the missing-key bit (their resolves give index 0, in
    bounds), which the library turns into TG_ERR_INTERNAL instead of a silent wrong index."""
    e, idx = hostcheck.table_errors(600, 1024)
    assert e == 0 and sorted(idx.tolist()) == list(range(600))
    e, idx = hostcheck.table_errors(1500, 1024)
    assert e == 3                                   # kErrTableFull | kErrKeyMissing
    assert idx.min() >= 0 and idx.max() < 1024
