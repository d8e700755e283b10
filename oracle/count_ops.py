"""Per-chunk counts of the TERRAIN step's units of work, from the counting build of the
reference's own C++ port (TEST AND MEASUREMENT INFRASTRUCTURE).

oracle/_ref/libref_count.so is the reference's cpu/ sources compiled with
-finstrument-functions plus the hooks of oracle/count_driver.cpp (make -C oracle count).
This script resolves the counted functions in that library's symbol table, runs the
reference's region form (ref_generate: biomes of the region plus a one-chunk border, then
fill and surface per chunk, as bench/bench_main.cpp:253-304 does) over a sample of the
ladder workload, and writes the per-chunk counts per phase:

    python oracle/count_ops.py [--side 8] [--threads 8] [--out minecraft-terrain-cuda_b200/model/op_counts.json]

Units (one count = one call): vol_octave (perlin_volume + smeared_volume), point_octave
(perlin_get + smeared_get), simplex (Simplex2D::get), rtree_distance (BiomeTree::distance),
zoom_corner (fiddled_distance). Phases: biome, corners, fill, aquifer, surface (see
count_driver.cpp). The counts are the reference algorithm's work per chunk, each chunk
computing its own cell corners; a deduplicating pipeline does the corner work once per
distinct corner column.
"""
import argparse
import ctypes
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
LIB = os.path.join(HERE, '_ref', 'libref_count.so')
SYMS = os.path.join(HERE, '_ref', 'libref_count.syms')
MODEL = os.path.join(REPO, 'minecraft-terrain-cuda_b200', 'model')
UNITS = ['perlin_volume', 'smeared_volume', 'perlin_get', 'smeared_get', 'simplex', 'rtree_distance', 'zoom_corner']
UNIT_SYMS = ['mcc::perlin_volume(', 'mcc::smeared_volume(', 'mcc::perlin_get(', 'mcc::smeared_get(', 'mcc::Simplex2D::get(',
             'mcc::BiomeTree::distance(', 'mcc::(anonymous namespace)::fiddled_distance(']
PHASES = ['fill', 'corners', 'biome', 'aquifer', 'surface']

# the ladder workload's seed and regions (bench.py)
SEED = 0x5445525241494E31
REGIONS = [('origin', 0, 0), ('negative', -62500, -62500), ('border', 117124, 117124)]


def available():
    return os.path.exists(LIB) and os.path.exists(SYMS)


def symbols():
    """(unit offsets, phase function offsets, phase ids) from the library's symbol table."""
    unit = [0] * len(UNITS)
    phase = {}
    with open(SYMS) as f:
        for line in f:
            parts = line.rstrip('\n').split(' ', 2)
            if len(parts) < 3 or parts[1] not in 'TtWw' or '[clone' in parts[2]:
                continue
            off, name = int(parts[0], 16), parts[2]
            for i, s in enumerate(UNIT_SYMS):
                if name.startswith(s):
                    unit[i] = off
            if name.startswith('mcc::VolumeEvaluator::sample_interpolated_block_step('):
                phase[off] = 1
            elif name.startswith('mcc::cpu_chunk_biomes('):
                phase[off] = 2
            elif '::Aquifer::' in name:
                phase[off] = 3
            elif '::Surface::' in name:
                phase[off] = 4
    return unit, sorted(phase.items())


class Counter:
    def __init__(self):
        L = ctypes.CDLL(LIB)
        vp = ctypes.c_void_p
        L.ref_open.restype = vp
        L.ref_open.argtypes = [ctypes.c_char_p, ctypes.c_char_p]
        L.ref_seed.restype = vp
        L.ref_seed.argtypes = [vp, ctypes.c_int64]
        L.ref_seed_free.argtypes = [vp]
        L.ref_generate.argtypes = [vp, vp, vp, ctypes.c_int32, ctypes.c_int32, vp, vp, vp, vp]
        L.ref_count_setup.argtypes = [vp, vp, vp, ctypes.c_int32]
        L.ref_count_enable.argtypes = [ctypes.c_int32]
        L.ref_count_read.argtypes = [vp, ctypes.c_int32]
        L.ref_last_error.restype = ctypes.c_char_p
        self.L = L
        unit, phase = symbols()
        if not all(unit):
            missing = [UNITS[i] for i, u in enumerate(unit) if not u]
            raise RuntimeError('counted functions missing from the symbol table: %s' % missing)
        uo = np.array(unit, np.uint64)
        po = np.array([p[0] for p in phase], np.uint64)
        pi = np.array([p[1] for p in phase], np.int32)
        if L.ref_count_setup(uo.ctypes.data, po.ctypes.data, pi.ctypes.data, len(phase)) != 0:
            raise RuntimeError('ref_count_setup failed')
        self.model = L.ref_open(os.path.join(MODEL, 'overworld_ir.json').encode(), os.path.join(MODEL, 'overworld_terrain.json').encode())
        if not self.model:
            raise RuntimeError(L.ref_last_error().decode())

    def count(self, seed, chunks, threads=8):
        """Counts per phase x unit over one region-form run of chunks: a (5, 7) uint64 array."""
        L = self.L
        s = L.ref_seed(self.model, int(seed))
        a = np.ascontiguousarray(np.asarray(chunks, np.int32).reshape(-1, 2))
        cx, cz = np.ascontiguousarray(a[:, 0]), np.ascontiguousarray(a[:, 1])
        n = a.shape[0]
        blocks = np.empty(n * 98304, np.uint16)
        c = np.zeros(len(PHASES) * len(UNITS), np.uint64)
        L.ref_count_read(c.ctypes.data, 1)
        L.ref_count_enable(1)
        st = L.ref_generate(s, cx.ctypes.data, cz.ctypes.data, n, threads, blocks.ctypes.data, None, None, None)
        L.ref_count_enable(0)
        L.ref_count_read(c.ctypes.data, 1)
        L.ref_seed_free(s)
        if st != 0:
            raise RuntimeError(L.ref_last_error().decode())
        return c.reshape(len(PHASES), len(UNITS))


def summarize(counts, n_chunks):
    per = {}
    for p, name in enumerate(PHASES):
        row = {u: counts[p, i] / n_chunks for i, u in enumerate(UNITS)}
        per[name] = {'vol_octave': row['perlin_volume'] + row['smeared_volume'], 'point_octave': row['perlin_get'] + row['smeared_get'],
                     'simplex': row['simplex'], 'rtree_distance': row['rtree_distance'], 'zoom_corner': row['zoom_corner']}
    return per


def sha256(path):
    with open(path, 'rb') as f:
        return hashlib.sha256(f.read()).hexdigest()


def main(argv):
    ap = argparse.ArgumentParser()
    ap.add_argument('--side', type=int, default=8, help='chunks per side of the square sampled at the corner of each ladder region')
    ap.add_argument('--threads', type=int, default=8)
    ap.add_argument('--out', default=os.path.join(MODEL, 'op_counts.json'))
    args = ap.parse_args(argv)
    if not available():
        sys.exit('counting build missing: make -C oracle count')
    ctr = Counter()
    side = args.side
    total = np.zeros((len(PHASES), len(UNITS)), np.uint64)
    regions = {}
    for name, x0, z0 in REGIONS:
        chunks = [(x0 + x, z0 + z) for z in range(side) for x in range(side)]
        c = ctr.count(SEED, chunks, args.threads)
        total += c
        regions[name] = summarize(c, len(chunks))
    out = {'what': 'reference port (cpu/), counting build: calls per chunk of each unit of work, per phase, region form '
                   '(biomes of the square plus a one-chunk border computed once per chunk, then fill and surface per chunk)',
           'model': {'overworld_ir.json': sha256(os.path.join(MODEL, 'overworld_ir.json')),
                     'overworld_terrain.json': sha256(os.path.join(MODEL, 'overworld_terrain.json'))},
           'seed': SEED, 'sample': '%dx%d chunks at the corner of each ladder region (origin, -62,500, 117,124)' % (side, side),
           'chunks': 3 * side * side, 'per_chunk': summarize(total, 3 * side * side), 'per_region': regions}
    with open(args.out, 'w') as f:
        json.dump(out, f, indent=1, sort_keys=True)
        f.write('\n')
    print(json.dumps(out['per_chunk'], indent=1))


if __name__ == '__main__':
    main(sys.argv[1:])
