"""Writes tests/golden/terrain_digests.json and tests/golden/kat.json from the reference's
own C++ port (oracle/_ref, built from the reference sources by oracle/Makefile).

Corpus, shaped like the reference's oracle corpus (oracle/.../Corpus.java:185-234):
fixed seeds (0, +-1, Long.MIN/MAX, +-2^31, one negative 64-bit seed) plus four drawn from
a fixed SplitMix64 stream; per seed the origin 3x3, near (+-6,250), far (+-625,000),
world border (+-1,874,999), the 32-bit noise-wrap chunks 6128 / -6129, and the
+-117,187 border reading. Per chunk: SHA-256 of the u16 block states (little endian) and
of the u8 quart biomes, both in the layouts of cpu/include/mccuda/terrain.h:55-60.

Run in the repository root:  python tests/golden/make_golden.py
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, 'oracle'))
import ref_oracle  # noqa: E402

FIXED = [0, 1, -1, -(1 << 63), (1 << 63) - 1, 1 << 31, -(1 << 31), -4172144997902289642]
CHUNKS = [(x, z) for z in (-1, 0, 1) for x in (-1, 0, 1)] + [(6250, 6250), (-6250, -6250), (625000, -625000), (-625000, 625000),
                                                            (1874999, 1874999), (-1874999, -1874999), (6128, 0), (-6129, 0), (117187, -117187)]


def splitmix64(state, n):
    out = []
    for _ in range(n):
        state = (state + 0x9E3779B97F4A7C15) & ((1 << 64) - 1)
        z = state
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & ((1 << 64) - 1)
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & ((1 << 64) - 1)
        z ^= z >> 31
        out.append(z - (1 << 64) if z >= (1 << 63) else z)
    return out


SEEDS = FIXED + splitmix64(0x7465727261696E, 4)


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def main():
    m = ref_oracle.RefModel()
    L = ref_oracle.lib()
    out = {'format': 'terrain-digests/1', 'model_ir_sha256': hashlib.sha256(open(ref_oracle.IR_PATH, 'rb').read()).hexdigest(),
           'model_terrain_sha256': hashlib.sha256(open(ref_oracle.TERRAIN_PATH, 'rb').read()).hexdigest(), 'chunks': CHUNKS, 'seeds': {}}
    for sd in SEEDS:
        b, q = m.seed(sd).generate(CHUNKS)
        out['seeds'][str(sd)] = [[digest(b[i].astype('<u2')), digest(q[i])] for i in range(len(CHUNKS))]
        print('seed', sd, 'done', flush=True)
    with open(os.path.join(HERE, 'terrain_digests.json'), 'w') as f:
        json.dump(out, f, indent=1)
    # known answers of the reference's hashes and random sources
    kat = {'md5': {}, 'xoroshiro_longs': {}, 'mth_get_seed': [], 'quantize': [], 'stream_sum': [], 'zoom_seed': {}}
    for s in ['', 'The quick brown fox jumps over the lazy dog', 'a' * 1000, 'octave_-7', 'minecraft:terrain']:
        h = (np.zeros(16, np.uint8))
        L.ref_md5(s.encode(), len(s), h.ctypes.data_as(__import__('ctypes').c_void_p))
        kat['md5'][s] = h.tobytes().hex()
    import ctypes
    for sd in SEEDS:
        a = np.zeros(8, np.int64)
        L.ref_xoroshiro_longs(sd, 8, a.ctypes.data_as(ctypes.c_void_p))
        kat['xoroshiro_longs'][str(sd)] = [int(v) for v in a]
        kat['zoom_seed'][str(sd)] = int(L.ref_zoom_seed(sd))
    for x, y, z in [(0, 0, 0), (1, 2, 3), (-1, -64, 5), (2147483647, 319, -2147483648), (30000000, 100, -30000000)]:
        kat['mth_get_seed'].append([x, y, z, int(L.ref_mth_get_seed(x, y, z))])
    for v in [0.0, -0.0, 1.0, -1.5, 0.12345, 1e30, -1e30, float('inf'), float('-inf'), float('nan'), 3.4e38]:
        kat['quantize'].append([float(np.float32(v)) if v == v else 'nan', int(L.ref_quantize(ctypes.c_float(v)))])
    for vals in [[1.0, 1e100, 1.0, -1e100], [0.1] * 10, [0.5, 0.25, 0.125], [1e308, 1e308]]:
        arr = np.array(vals, np.float64)
        kat['stream_sum'].append([vals, float(L.ref_stream_sum(arr.ctypes.data_as(ctypes.c_void_p), len(vals)))])
    with open(os.path.join(HERE, 'kat.json'), 'w') as f:
        json.dump(kat, f, indent=1)
    print('wrote terrain_digests.json and kat.json')


if __name__ == '__main__':
    main()
