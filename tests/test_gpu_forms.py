"""GPU: the batched multi-seed form, the continuous-batching server, biome lookups,
the aquifer-fill output and argument errors, each checked against the reference port
or against the plain form. Integer outputs, zero tolerance.
"""
import numpy as np
import pytest

import terrain_b200

pytestmark = pytest.mark.gpu


def test_aquifer_output_matches_reference(gpu_gen, ref_model):
    chunks = [(0, 0), (5, -3), (1874999, 1874999), (-4000, 1600)]
    gpu_gen.set_seed(99)
    blocks, biomes, aq = gpu_gen.generate(chunks, aquifer=True)
    rb, rq, raq = ref_model.seed(99).generate(chunks, aquifer=True)
    assert (aq == raq).all() and (blocks == rb).all() and (biomes == rq).all()


def test_batch_mixes_seeds_and_sizes(gpu_gen, ref_model):
    rng = np.random.default_rng(3)
    reqs = []
    for seed, n in [(11, 1), (-5, 7), (11, 3), (2 ** 40, 20), (-5, 2)]:
        base = rng.integers(-50000, 50000, 2)
        reqs.append((seed, [(int(base[0] + i % 5), int(base[1] + i // 5)) for i in range(n)]))
    outs = gpu_gen.generate_batch(reqs)
    for (seed, chunks), (b, q) in zip(reqs, outs):
        rb, rq = ref_model.seed(seed).generate(chunks)
        assert (b == rb).all() and (q == rq).all(), 'seed %d' % seed


def test_batch_larger_than_one_device_batch(ref_model):
    g = terrain_b200.TerrainGenerator(max_batch_chunks=8)
    try:
        chunks = [(x, z) for z in range(3) for x in range(5)]
        outs = g.generate_batch([(1234, chunks), (4321, chunks[:4])])
        rb, rq = ref_model.seed(1234).generate(chunks)
        assert (outs[0][0] == rb).all() and (outs[0][1] == rq).all()
        rb, rq = ref_model.seed(4321).generate(chunks[:4])
        assert (outs[1][0] == rb).all() and (outs[1][1] == rq).all()
        g.set_seed(1234)
        b2, q2 = g.generate(chunks)            # the plain form splits the list the same way
        assert (b2 == outs[0][0]).all() and (q2 == outs[0][1]).all()
    finally:
        g.close()


def test_host_batches_equal_whole_device_batches(ref_model):
    """tg_generate cuts host-output work into the batches of the launch table's host_u16
    schedule; on a generator of capacity 4,096 its result for 5,100 chunks equals the
    device-resident form run on whole 4,096-chunk batches (written in place into aligned
    buffers; through the generator's buffers and a copy into unaligned ones, and with no
    biome buffer), and its last chunks equal the reference."""
    import torch
    g = terrain_b200.TerrainGenerator(max_batch_chunks=4096)
    try:
        g.set_seed(777)
        chunks = np.array([(x, z) for z in range(-30, 30) for x in range(-43, 42)], np.int32)[:5100]
        b, q = g.generate(chunks)
        dev_b = torch.empty((4096, g.height, 16, 16), dtype=torch.int16, device='cuda')
        dev_q = torch.empty((4096, g.qper), dtype=torch.uint8, device='cuda')
        for off in (0, 4096):
            part = torch.from_numpy(np.ascontiguousarray(chunks[off:off + 4096])).cuda()
            n = part.shape[0]
            g.generate_device(part.data_ptr(), n, dev_b.data_ptr(), dev_q.data_ptr(), timing=False)
            torch.cuda.synchronize()
            assert (dev_b[:n].cpu().numpy().view(np.uint16) == b[off:off + n]).all(), off
            assert (dev_q[:n].cpu().numpy() == q[off:off + n]).all(), off
        # unaligned outputs (2 and 1 bytes past a 16-byte boundary), then no biome buffer
        n = 70
        part = torch.from_numpy(np.ascontiguousarray(chunks[:n])).cuda()
        flat_b = torch.zeros(n * g.height * 256 + 16, dtype=torch.int16, device='cuda')
        flat_q = torch.zeros(n * g.qper + 16, dtype=torch.uint8, device='cuda')
        g.generate_device(part.data_ptr(), n, flat_b.data_ptr() + 2, flat_q.data_ptr() + 1, timing=False)
        torch.cuda.synchronize()
        got_b = flat_b[1:1 + n * g.height * 256].cpu().numpy().view(np.uint16).reshape(b[:n].shape)
        assert (got_b == b[:n]).all() and (flat_q[1:1 + n * g.qper].cpu().numpy().reshape(q[:n].shape) == q[:n]).all()
        assert int(flat_b[0]) == 0 and int(flat_q[0]) == 0
        dev_b.zero_()
        g.generate_device(part.data_ptr(), n, dev_b.data_ptr(), None, timing=False)
        torch.cuda.synchronize()
        assert (dev_b[:n].cpu().numpy().view(np.uint16) == b[:n]).all()
        tail = [tuple(int(v) for v in c) for c in chunks[-6:]]
        rb, rq = ref_model.seed(777).generate(tail)
        assert (b[-6:] == rb).all() and (q[-6:] == rq).all()
    finally:
        g.close()


def test_u8_form_equals_narrowed_u16(ref_model):
    """tg_generate_u8 (the reference generator's output type) gives every u16 state of
    tg_generate as one byte, for blocks and the aquifer fill, over several batches and the
    halving tail, with graphs and with stage timing, alternating with the u16 form; some of
    its chunks also equal the reference directly."""
    g = terrain_b200.TerrainGenerator(max_batch_chunks=256)
    try:
        g.set_seed(-4242)
        chunks = np.array([(x, z) for z in range(-12, 13) for x in range(-14, 14)], np.int32)[:700]
        chunks[-3:] = [(2097148, -2097149), (-2097152, 4194303), (8388607, -8388607)]
        b16, q16, a16 = g.generate(chunks, aquifer=True)
        assert int(b16.max()) < 256 and int(a16.max()) < 256
        b8, q8, a8 = g.generate_u8(chunks, aquifer=True)
        assert b8.dtype == np.uint8 and (b8 == b16.astype(np.uint8)).all() and (b8.astype(np.uint16) == b16).all()
        assert (a8.astype(np.uint16) == a16).all() and (q8 == q16).all()
        b8t, q8t, t = g.generate_u8(chunks[:300], timing=True)
        assert (b8t.astype(np.uint16) == b16[:300]).all() and (q8t == q16[:300]).all() and t['launches'] > 0
        b16b, _ = g.generate(chunks[:40])
        assert (b16b == b16[:40]).all()
        part = [tuple(int(v) for v in c) for c in chunks[-4:]]
        rb, rq = ref_model.seed(-4242).generate(part)
        assert (b8[-4:].astype(np.uint16) == rb).all() and (q8[-4:] == rq).all()
    finally:
        g.close()


def test_server_alone_equals_mixed(ref_model):
    """Each served result is byte-identical alone and in a mix of concurrent requests."""
    g = terrain_b200.TerrainGenerator(max_batch_chunks=64)
    try:
        rng = np.random.default_rng(7)
        reqs = []
        for k in range(12):
            r = int(rng.integers(0, 3))
            cx, cz = (int(v) for v in rng.integers(-100000, 100000, 2))
            reqs.append((int(rng.choice([1, 2, 3])), [(cx + dx, cz + dz) for dz in range(-r, r + 1) for dx in range(-r, r + 1)]))
        alone = []
        for seed, chunks in reqs:
            g.set_seed(seed)
            alone.append(g.generate(chunks))
        with terrain_b200.TerrainServer(g, batch_chunks=40) as srv:
            tickets = [srv.submit(seed, chunks) for seed, chunks in reqs]
            mixed = [srv.wait(t) for t in tickets]
            st = srv.stats()
        assert st['completed_requests'] == len(reqs)
        for (a_b, a_q), (m_b, m_q) in zip(alone, mixed):
            assert (a_b == m_b).all() and (a_q == m_q).all()
        seed, chunks = reqs[0]
        rb, rq = ref_model.seed(seed).generate(chunks)
        assert (mixed[0][0] == rb).all() and (mixed[0][1] == rq).all()
    finally:
        g.close()


def test_biome_lookup_matches_reference(gpu_gen, ref_model):
    rng = np.random.default_rng(5)
    n = 3000
    xyz = np.stack([rng.integers(-1874999, 1874999, n), rng.integers(-64, 320, n), rng.integers(-1874999, 1874999, n)], 1).astype(np.int32)
    seeds = rng.choice(np.array([0, 77, -3, 2 ** 62], np.int64), n)
    got = gpu_gen.biome_lookup(seeds, xyz)
    for s in np.unique(seeds):
        sel = seeds == s
        want = ref_model.seed(int(s)).biome_lookup(xyz[sel])
        assert (got[sel] == want).all(), 'seed %d' % s


def test_biome_lookup_dense_and_many_seeds(gpu_gen, ref_model):
    """Lookups packed into a few chunks (so chain ties are replayed from earlier quarts), y
    outside the world (clamped quart rows), and 40 seeds interleaved position by position."""
    rng = np.random.default_rng(17)
    n = 4000
    xyz = np.stack([rng.integers(-48, 48, n), rng.integers(-90, 345, n), rng.integers(-48, 48, n)], 1).astype(np.int32)
    pool = np.array([int(v) for v in rng.integers(-(1 << 62), 1 << 62, 40)], np.int64)
    seeds = pool[rng.integers(0, 40, n)]
    got = gpu_gen.biome_lookup(seeds, xyz)
    for s in np.unique(seeds):
        sel = seeds == s
        want = ref_model.seed(int(s)).biome_lookup(xyz[sel])
        assert (got[sel] == want).all(), 'seed %d' % s


def test_biome_lookup_many_seeds_across_sub_batches(gpu_gen, ref_model):
    """700 seeds interleaved position by position: each sub-batch holds at most 256 distinct
    seeds (11 sub-batches, two in flight at a time), and there are more seeds than resident
    slots, so slots are recycled while the previous sub-batch runs. Every position equals
    the lookup of its seed alone, 24 seeds equal the reference, and a second call in reverse
    order (some seeds resident, others rebuilt) gives the same bytes."""
    rng = np.random.default_rng(12)
    pool = np.array([int(v) for v in rng.integers(-(1 << 62), 1 << 62, 700)], np.int64)
    n = 2800
    seeds = pool[np.arange(n) % 700]
    xyz = np.stack([rng.integers(-1874999, 1875000, n), rng.integers(-64, 320, n), rng.integers(-1874999, 1875000, n)], 1).astype(np.int32)
    got = gpu_gen.biome_lookup(seeds, xyz)
    assert (gpu_gen.biome_lookup(seeds[::-1], xyz[::-1]) == got[::-1]).all()
    for s in pool:
        sel = seeds == s
        assert (gpu_gen.biome_lookup(np.full(int(sel.sum()), s), xyz[sel]) == got[sel]).all(), int(s)
    for s in pool[:24]:
        sel = seeds == s
        assert (ref_model.seed(int(s)).biome_lookup(xyz[sel]) == got[sel]).all(), int(s)


def test_biome_lookup_beyond_one_sub_batch(gpu_gen):
    """2^20 + 70,000 positions of 3 seeds (two sub-batches by size): the tail equals the same
    positions looked up alone."""
    rng = np.random.default_rng(13)
    n = (1 << 20) + 70000
    pool = np.array([5, -77, 1 << 40], np.int64)
    seeds = pool[rng.integers(0, 3, n)]
    xyz = np.stack([rng.integers(-300000, 300000, n), rng.integers(-64, 320, n), rng.integers(-300000, 300000, n)], 1).astype(np.int32)
    got = gpu_gen.biome_lookup(seeds, xyz)
    k = (1 << 20) - 30000
    assert (gpu_gen.biome_lookup(seeds[k:], xyz[k:]) == got[k:]).all()
    assert (gpu_gen.biome_lookup(seeds[:50000], xyz[:50000]) == got[:50000]).all()


def test_errors_are_status_codes(gpu_gen):
    with pytest.raises(terrain_b200.TerrainError) as e:
        gpu_gen.generate([(1 << 23, 0)])
    assert e.value.status == 5
    g = terrain_b200.TerrainGenerator(max_batch_chunks=4)
    try:
        with pytest.raises(terrain_b200.TerrainError) as e:
            g.generate([(0, 0)])
        assert e.value.status == 6
    finally:
        g.close()
    with pytest.raises(terrain_b200.TerrainError) as e:
        terrain_b200.TerrainGenerator(max_batch_chunks=4, ir_path=__file__)
    assert e.value.status == 2


def test_repeatable(gpu_gen):
    gpu_gen.set_seed(31337)
    chunks = [(x, 0) for x in range(6)]
    a = gpu_gen.generate(chunks)
    b = gpu_gen.generate(chunks[::-1])
    assert (a[0] == b[0][::-1]).all() and (a[1] == b[1][::-1]).all()
