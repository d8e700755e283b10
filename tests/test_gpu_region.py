"""Region outputs for consumers (tg_write_region): the dump a game-side reader maps
(terrain.u8, biomes.u8, meta.json; reference bench/bench_main.cpp:170-187, read by the
client's GpuDump.java:88-104) and the top-down map (bench_main.cpp:134-165). The files must
hold the u8 form of the same chunks in row-major order, and the top-down records the
reference's column rule, restated here over numpy arrays, whether computed on the host from
the dumped blocks or on the device when the map is asked for alone."""
import json
import os
import struct

import numpy as np
import pytest

import terrain_b200

pytestmark = pytest.mark.gpu

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def palette_flags():
    """air / fluid per palette state by the reference's rule (cpu/src/terrain_model.cpp:120-127)."""
    pal = json.load(open(os.path.join(REPO, 'minecraft-terrain-cuda_b200', 'model', 'overworld_terrain.json')))['palette']
    air = np.array([p == 'minecraft:air' for p in pal])
    fluid = np.array([p.startswith('minecraft:water') or p.startswith('minecraft:lava') for p in pal])
    return air, fluid


def topdown_records(blocks, region, min_y):
    """blocks: (region * region, height, 16, 16) u8, row-major chunks. Per block column: the
    highest non-air y (0 when the column is all air), then down while fluid and y > 0."""
    air, fluid = palette_flags()
    n, height = blocks.shape[0], blocks.shape[1]
    b = blocks.reshape(region, region, height, 16, 16).transpose(0, 3, 1, 4, 2).reshape(region * 16, region * 16, height)   # [z][x][y]
    solid = ~air[b]
    any_solid = solid.any(axis=2)
    top_y = np.where(any_solid, height - 1 - np.argmax(solid[:, :, ::-1], axis=2), 0)
    y = top_y.copy()
    for _ in range(height):
        cur = np.take_along_axis(b, y[:, :, None], axis=2)[:, :, 0]
        step = (y > 0) & fluid[cur]
        if not step.any():
            break
        y = np.where(step, y - 1, y)
    top = np.take_along_axis(b, top_y[:, :, None], axis=2)[:, :, 0]
    floor = np.take_along_axis(b, y[:, :, None], axis=2)[:, :, 0]
    rec = np.zeros((region * 16, region * 16, 8), np.uint8)
    rec[:, :, 0] = top
    rec[:, :, 1] = floor
    rec[:, :, 2] = np.minimum(255, top_y - y)
    rec[:, :, 4:6] = (min_y + top_y).astype('<i2').view(np.uint8).reshape(region * 16, region * 16, 2)
    rec[:, :, 6:8] = (min_y + y).astype('<i2').view(np.uint8).reshape(region * 16, region * 16, 2)
    return rec.reshape(-1)


@pytest.mark.parametrize('x0,z0,region', [(-3, 2, 5), (117184, 117184, 4), (2097148, -2097150, 3)])
def test_region_dump_and_topdown(tmp_path, ref_model, x0, z0, region):
    seed = 0x5EED0 + region
    g = terrain_b200.TerrainGenerator(max_batch_chunks=8)
    try:
        dump, td = tmp_path / 'dump', tmp_path / 'top.mctd'
        g.write_region(seed, x0, z0, region, dump_dir=str(dump), topdown_path=str(td))
        meta = json.load(open(dump / 'meta.json'))
        assert meta == {'seed': seed, 'x0': x0, 'z0': z0, 'region': region, 'height': g.height, 'min_y': g.min_y, 'chunk_bytes': g.height * 256,
                        'biome_bytes': g.qper}
        n = region * region
        terrain = np.fromfile(dump / 'terrain.u8', np.uint8)
        biomes = np.fromfile(dump / 'biomes.u8', np.uint8)
        assert terrain.size == n * g.height * 256 and biomes.size == n * g.qper
        chunks = [(x0 + i, z0 + r) for r in range(region) for i in range(region)]
        b8, q8 = g.generate_u8(chunks)          # write_region left the seed set
        assert (terrain == b8.reshape(-1)).all() and (biomes == q8.reshape(-1)).all()
        raw = open(td, 'rb').read()
        assert raw[:4] == b'MCTD' and struct.unpack('<5i', raw[4:24]) == (1, region, x0, z0, g.min_y)
        rec = np.frombuffer(raw[24:], np.uint8)
        assert (rec == topdown_records(b8, region, g.min_y)).all()
        # the map alone is computed on the device (k_topdown over the u16 states in HBM, in
        # pieces of at most max_batch_chunks that cross chunk-row boundaries): same bytes
        td2 = tmp_path / 'top_device.mctd'
        g.write_region(seed, x0, z0, region, topdown_path=str(td2))
        assert open(td2, 'rb').read() == raw
        # one chunk of the dump against the reference port directly
        k = n // 2
        rb, rq = ref_model.seed(seed).generate([chunks[k]])
        assert (b8[k].astype(np.uint16) == rb[0]).all() and (q8[k] == rq[0]).all()
    finally:
        g.close()


def test_region_arguments(tmp_path):
    g = terrain_b200.TerrainGenerator(max_batch_chunks=8)
    try:
        with pytest.raises(terrain_b200.TerrainError, match='INVALID_ARGUMENT'):
            g.write_region(1, 0, 0, 0, dump_dir=str(tmp_path / 'a'))
        with pytest.raises(terrain_b200.TerrainError, match='INVALID_ARGUMENT'):
            g.write_region(1, 0, 0, 2)
        with pytest.raises(terrain_b200.TerrainError, match='RANGE'):
            g.write_region(1, 8388606, 0, 4, dump_dir=str(tmp_path / 'b'))
        with pytest.raises(terrain_b200.TerrainError, match='TG_ERR_IO'):
            g.write_region(1, 0, 0, 1, topdown_path=str(tmp_path / 'missing' / 'dir' / 'top.mctd'))
    finally:
        g.close()
