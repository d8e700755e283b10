"""GPU: the device-resident multi-seed batch (tg_generate_batch_device), whose requests run
from a device work queue -- one CUDA-graph launch looping on the device (a WHILE node), or
one graph per batch from the host -- against the reference port and the host-output batched
form; argument checks; and the launch table (shapes, work-queue kernels, hash-table load),
whose setting changes no output. Integer outputs, zero tolerance."""
import numpy as np
import pytest

import terrain_b200

pytestmark = pytest.mark.gpu


def device_requests(reqs, height, qper):
    """Device chunk lists and output buffers for (seed, chunks) requests."""
    import torch
    out = []
    for seed, chunks in reqs:
        c = torch.from_numpy(np.ascontiguousarray(np.asarray(chunks, np.int32).reshape(-1, 2))).cuda()
        n = c.shape[0]
        b = torch.empty((max(n, 1), height, 16, 16), dtype=torch.int16, device='cuda')
        q = torch.empty((max(n, 1), qper), dtype=torch.uint8, device='cuda')
        out.append((seed, c, n, b, q))
    return out


def run_device(g, dreqs, host_loop=False, timing=False):
    import torch
    g.generate_batch_device([(sd, c.data_ptr(), n, b.data_ptr(), q.data_ptr()) for sd, c, n, b, q in dreqs], host_loop=host_loop, timing=timing)
    torch.cuda.synchronize()
    return [(b[:n].cpu().numpy().view(np.uint16), q[:n].cpu().numpy()) for _, _, n, b, q in dreqs]


@pytest.fixture(scope='module')
def small_gen():
    g = terrain_b200.TerrainGenerator(max_batch_chunks=8)
    yield g
    g.close()


def test_device_queue_equals_reference_and_host_batches(small_gen, ref_model):
    rng = np.random.default_rng(41)
    reqs = []
    for seed, n in [(11, 1), (-5, 7), (11, 3), (2 ** 40, 20), (-5, 0), (77, 9)]:
        base = rng.integers(-50000, 50000, 2)
        reqs.append((seed, [(int(base[0] + i % 5), int(base[1] + i // 5)) for i in range(n)]))
    reqs.append((-5, [(6128, -6129), (1874999, -1874999), (-2097150, 3)]))
    dreqs = device_requests(reqs, small_gen.height, small_gen.qper)
    loop = run_device(small_gen, dreqs)                      # one graph launch, 6 device iterations
    host = run_device(small_gen, dreqs, host_loop=True)
    timed = run_device(small_gen, dreqs, timing=True)
    ref_host = small_gen.generate_batch([r for r in reqs if len(r[1])])
    k = 0
    for (seed, chunks), a, b, c in zip(reqs, loop, host, timed):
        assert (a[0] == b[0]).all() and (a[1] == b[1]).all() and (a[0] == c[0]).all() and (a[1] == c[1]).all()
        if not chunks:
            continue
        rb, rq = ref_model.seed(seed).generate(chunks)
        assert (a[0] == rb).all() and (a[1] == rq).all(), 'seed %d' % seed
        assert (ref_host[k][0] == a[0]).all() and (ref_host[k][1] == a[1]).all()
        k += 1


def test_device_queue_groups_beyond_the_seed_slots(ref_model):
    """More distinct seeds than one launch keeps resident (300 > 256): two groups."""
    g = terrain_b200.TerrainGenerator(max_batch_chunks=64)
    try:
        seeds = [1000 + 7 * i for i in range(300)]
        reqs = [(sd, [(i % 17 - 8, i // 17 - 8)]) for i, sd in enumerate(seeds)]
        dreqs = device_requests(reqs, g.height, g.qper)
        outs = run_device(g, dreqs)
        for i in (0, 1, 255, 256, 299):
            rb, rq = ref_model.seed(seeds[i]).generate(reqs[i][1])
            assert (outs[i][0] == rb).all() and (outs[i][1] == rq).all(), i
    finally:
        g.close()


def test_device_queue_rejects_unaligned_outputs(small_gen):
    import torch
    c = torch.zeros((1, 2), dtype=torch.int32, device='cuda')
    b = torch.empty(98304 * 2 + 16, dtype=torch.int16, device='cuda')
    with pytest.raises(terrain_b200.TerrainError) as e:
        small_gen.generate_batch_device([(1, c.data_ptr(), 1, b.data_ptr() + 2, 0)])
    assert e.value.status == 1


def test_launch_tables_change_no_output(ref_model):
    """Work-queue forms, other block sizes and grids, a larger hash-table load, host-output
    schedules and deferred-list sizes of the column walk (none; one block per chunk, so
    that it fills): the same blocks and biomes as the compiled-in table; per-kernel times
    are gathered."""
    g = terrain_b200.TerrainGenerator(max_batch_chunks=64)
    try:
        g.set_seed(4242)
        chunks = [(x, z) for z in range(-4, 4) for x in range(-4, 4)] + [(6128, 33), (-117187, 117187)]
        base = g.generate(chunks)
        default = g.launch_table()
        names = terrain_b200.KERNELS
        variants = ['table_load 4\n' + ''.join('%s 128 12 %d\n' % (k, 0 if k == 'chain' else 2) for k in names),
                    ''.join('%s %d %d %d\n' % (k, 64 * (1 + i % 4), 1 + i % 16, 0 if k == 'chain' else i % 3) for i, k in enumerate(names))]
        for text in variants:
            g.set_launch_table(text)
            g.kernel_times(enable=True)
            b, q, t = g.generate(chunks, timing=True)
            times = g.kernel_times(enable=False)
            assert (b == base[0]).all() and (q == base[1]).all()
            assert all(times[k][1] >= 1 for k in names) and times['corner'][0] > 0
            b, q = g.generate(chunks)                       # graphs of the new shapes
            assert (b == base[0]).all() and (q == base[1]).all()
        # host-output batch schedules: tails, heads and small batches cut the same chunks
        base8 = g.generate_u8(chunks)
        for text in ['host_u8 16 4 50 4 200\nhost_u16 24 8 75 0 0\n', 'host_u8 0 0 0 0 0\nhost_u16 7 0 0 3 300\nwalk_defer 1\n',
                     'walk_defer 0\n']:
            g.set_launch_table(text)
            if 'host_u16' in text:
                assert len(terrain_b200.host_schedule(len(chunks), 64, u8=False, table=text)) > 2
            b, q = g.generate(chunks)
            assert (b == base[0]).all() and (q == base[1]).all()
            b8, q8 = g.generate_u8(chunks)
            assert (b8 == base8[0]).all() and (q8 == base8[1]).all()
        g.set_launch_table(None)
        assert g.launch_table() == default
        with pytest.raises(terrain_b200.TerrainError):
            g.set_launch_table('corner 300 8 0\n')
        with pytest.raises(terrain_b200.TerrainError):
            g.set_launch_table('chain 256 8 1\n')
        rb, rq = ref_model.seed(4242).generate(chunks)
        assert (base[0] == rb).all() and (base[1] == rq).all()
    finally:
        g.close()
