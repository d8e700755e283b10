"""Host logic: the batch schedule of calls with host outputs (tg_host_schedule, the launch
table's host_u8 / host_u16 lines), and the launch-table parser's errors. No GPU: both run on
the host."""
import numpy as np
import pytest

import terrain_b200


def table(u8=None, u16=None):
    lines = []
    if u8 is not None:
        lines.append('host_u8 %d %d %d %d %d' % u8)
    if u16 is not None:
        lines.append('host_u16 %d %d %d %d %d' % u16)
    return '\n'.join(lines) + '\n'


def test_compiled_in_table_covers_every_chunk():
    for u8 in (True, False):
        for count in (0, 1, 100, 511, 512, 513, 4095, 4096, 4097, 12288, 37490, 100000):
            s = terrain_b200.host_schedule(count, 4096, u8=u8)
            assert sum(s) == count and all(0 < n <= 4096 for n in s), (u8, count, s)


def test_halving_tail():
    s = terrain_b200.host_schedule(12288, 4096, table=table(u8=(4096, 512, 50, 0, 0)))
    assert s == [512, 4096, 4096, 2048, 1024, 512]
    assert terrain_b200.host_schedule(12288, 4096, table=table(u8=(4096, 0, 0, 0, 0))) == [4096] * 3
    assert terrain_b200.host_schedule(300, 4096, table=table(u8=(4096, 512, 50, 0, 0))) == [300]
    assert terrain_b200.host_schedule(1000, 4096, table=table(u8=(4096, 512, 50, 0, 0))) == [488, 512]


def test_batch_bound_by_the_generator():
    # the form's batch above max_batch_chunks: max_batch_chunks bounds it; 0: max_batch_chunks
    assert terrain_b200.host_schedule(8192, 2048, table=table(u8=(4096, 0, 0, 0, 0))) == [2048] * 4
    assert terrain_b200.host_schedule(5000, 1024, table=table(u16=(0, 0, 0, 0, 0)), u8=False) == [904] + [1024] * 4


def test_head_and_tail():
    s = terrain_b200.host_schedule(12288, 4096, table=table(u8=(4096, 512, 50, 512, 200)))
    assert s[:3] == [512, 1024, 2048] and s[-3:] == [2048, 1024, 512] and sum(s) == 12288
    s = terrain_b200.host_schedule(12288, 4096, table=table(u8=(4096, 512, 67, 0, 0)))
    assert s[-1] == 512 and sum(s) == 12288
    tail = s[-6:]
    assert all(a >= b for a, b in zip(tail, tail[1:]))                # shrinking to the end


def test_forms_are_separate():
    t = table(u8=(4096, 0, 0, 0, 0), u16=(1024, 0, 0, 0, 0))
    assert terrain_b200.host_schedule(4096, 4096, u8=True, table=t) == [4096]
    assert terrain_b200.host_schedule(4096, 4096, u8=False, table=t) == [1024] * 4


def test_random_counts_and_tables():
    rng = np.random.default_rng(7)
    for _ in range(200):
        mb = int(rng.integers(1, 8193))
        sched = (int(rng.integers(0, 9000)), int(rng.integers(0, 3000)), int(rng.integers(0, 100)),
                 int(rng.integers(0, 3000)), int(rng.choice([0, 150, 200, 400])))
        count = int(rng.integers(0, 50000))
        s = terrain_b200.host_schedule(count, mb, table=table(u8=sched))
        hb = min(mb, sched[0]) if sched[0] > 0 else mb
        assert sum(s) == count and all(0 < n <= hb for n in s), (mb, sched, count)


@pytest.mark.parametrize('bad', ['host_u8 4096 512 100 0 0', 'host_u8 4096 512 50 512 100', 'host_u16 -1 0 0 0 0',
                                 'host_u8 4096 512', 'host_u16 2048 512 50 0 1001', 'walk_defer -1', 'walk_defer 70000',
                                 'table_load 9', 'corner 300 8 0', 'no_such_kernel 128 8 0'])
def test_bad_lines_are_errors(bad):
    with pytest.raises(terrain_b200.TerrainError) as e:
        terrain_b200.host_schedule(100, 4096, table=bad + '\n')
    assert e.value.status == 1
