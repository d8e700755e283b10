"""GPU parity on the workloads the bench times, byte for byte against the reference port
(oracle/_ref, cpu_terrain_from_biomes over cpu_chunk_biomes, cpu/src/terrain.cpp:152-176,
765-810), through the same calls the bench makes:

  - the 32x32-chunk region at the origin (the plain 1,024-chunk configuration);
  - the three 64x64-chunk ladder regions (origin, block -1,000,000, the +1,874,999-block
    border reading), through tg_generate_device on all 12,288 chunks as one batch (the
    bench's device-resident figure), and all 12,288 chunks in one tg_generate_u8 call and
    one tg_generate call (its end-to-end figures);
  - the reference's true world-border region, 64x64 chunks ending at chunk 1,874,999
    (block 29,999,984; oracle/src/main/java/mccuda/oracle/Corpus.java:185-186);
  - the 256-seed batched workload (bench.batched_lists) in one tg_generate_batch call,
    with the first, middle and last chunk of every request compared.

Integer outputs: zero tolerance.
"""
import concurrent.futures as cf

import numpy as np
import pytest

import bench
import terrain_b200

pytestmark = pytest.mark.gpu

SIDE = 64
TRUE_BORDER = ('true border', 1874936, 1874936)


@pytest.fixture(scope='module')
def big_gen():
    g = terrain_b200.TerrainGenerator(max_batch_chunks=3 * SIDE * SIDE)
    g.set_seed(bench.SEED)
    yield g
    g.close()


@pytest.fixture(scope='module')
def ref_seed(ref_model):
    return ref_model.seed(bench.SEED)


def bad_chunks(blocks, biomes, rb, rq):
    n = rb.shape[0]
    return np.nonzero((blocks.reshape(n, -1) != rb.reshape(n, -1)).any(1) | (biomes.reshape(n, -1) != rq.reshape(n, -1)).any(1))[0]


def test_region_32x32_at_origin(big_gen, ref_seed):
    chunks = bench.region_chunks(0, 0, 32)
    b, q = big_gen.generate(chunks)
    rb, rq = ref_seed.generate(chunks)
    bad = bad_chunks(b, q, rb, rq)
    assert bad.size == 0, 'chunks differing from the reference: %s' % chunks[bad[:10]].tolist()


def test_ladder_regions_through_the_benched_calls(big_gen, ref_seed):
    """Every chunk of the three ladder regions, through the three calls the bench times."""
    import torch
    n = SIDE * SIDE
    regions = [bench.region_chunks(x0, z0) for _, x0, z0 in bench.REGIONS]
    all_chunks = np.concatenate(regions)
    u8_blocks, u8_biomes = big_gen.generate_u8(all_chunks)
    u16_blocks, u16_biomes = big_gen.generate(all_chunks)
    dev_b = torch.empty((len(all_chunks), big_gen.height, 16, 16), dtype=torch.int16, device='cuda')
    dev_q = torch.empty((len(all_chunks), big_gen.qper), dtype=torch.uint8, device='cuda')
    d_chunks = torch.from_numpy(all_chunks).cuda()
    big_gen.generate_device(d_chunks.data_ptr(), len(all_chunks), dev_b.data_ptr(), dev_q.data_ptr(), timing=False)
    torch.cuda.synchronize()
    all_db, all_dq = dev_b.cpu().numpy().view(np.uint16), dev_q.cpu().numpy()
    for r, ((name, _, _), chunks) in enumerate(zip(bench.REGIONS, regions)):
        rb, rq = ref_seed.generate(chunks)
        sl = slice(r * n, (r + 1) * n)
        db, dq = all_db[sl], all_dq[sl]
        for form, (b, q) in (('device', (db, dq)), ('u16', (u16_blocks[sl], u16_biomes[sl])),
                             ('u8', (u8_blocks[sl].astype(np.uint16), u8_biomes[sl]))):
            bad = bad_chunks(b, q, rb, rq)
            assert bad.size == 0, '%s region, %s form: chunks differing from the reference: %s' % (name, form, chunks[bad[:10]].tolist())


def test_true_world_border_region(big_gen, ref_seed):
    name, x0, z0 = TRUE_BORDER
    chunks = bench.region_chunks(x0, z0)
    assert chunks[:, 0].max() == 1874999 and chunks[:, 1].max() == 1874999
    b, q = big_gen.generate_u8(chunks)
    rb, rq = ref_seed.generate(chunks)
    bad = bad_chunks(b.astype(np.uint16), q, rb, rq)
    assert bad.size == 0, 'chunks differing from the reference: %s' % chunks[bad[:10]].tolist()


def test_batched_workload_sample(ref_model):
    """The bench's 256-seed batched workload in one tg_generate_batch call (37,490 chunks in
    mixed-seed device batches); the first, middle and last chunk of every request equal the
    reference port for that request's seed."""
    seeds, lists = bench.batched_lists()
    g = terrain_b200.TerrainGenerator(max_batch_chunks=SIDE * SIDE)
    try:
        outs = g.generate_batch(list(zip(seeds, lists)))
    finally:
        g.close()

    def check(i):
        c = lists[i]
        pick = sorted({0, len(c) // 2, len(c) - 1})
        rb, rq = ref_model.seed(seeds[i]).generate(c[pick], threads=2)
        b, q = outs[i]
        bad = bad_chunks(b[pick], q[pick], rb, rq)
        return i, c[pick][bad].tolist()

    with cf.ThreadPoolExecutor(8) as ex:
        results = list(ex.map(check, range(len(seeds))))
    failed = [(i, c) for i, c in results if c]
    assert not failed, 'requests with chunks differing from the reference: %s' % failed[:10]
    assert sum(len(c) for c in lists) == 37490
