"""Chunk sets the parity tests share (test infrastructure).

fold_chunks() derives from the world model the chunks where a noise octave's input
coordinate wraps: GradientNoise.wrap folds a coordinate v once |v| >= 2^24
(cpu/include/mccuda/noise_eval.h:56-70), and v = block * scale * frequency, so octave
(scale, frequency) folds at block 2^24 / (scale * frequency). The scale of each noise is
read from the model:
  - noise nodes: their xz_scale (cpu/src/ir.cpp:99-104);
  - shift_a / shift_b / shift nodes: 0.25 (cpu/src/volume_eval.cpp:175-186);
  - blended noise: 684.412 * xz_scale for the limit stacks and that divided by xz_factor for
    the main stack, octave frequencies 2^-k (cpu/src/volume_eval.cpp:195-209,
    cpu/src/seed_tables.cpp:123-140);
  - every named noise also at scale 1 (the material rules sample at block coordinates).
The octave frequencies come from the reference port's seed tables (both stacks of a
NormalNoise, the second at 1.0181268882175227 times the first: cpu/src/seed_tables.cpp:90-120).
The reference's own corpus uses the first of these, chunks 6128 / -6129
(oracle/src/main/java/mccuda/oracle/Corpus.java:213-214).
"""
import json
import math
import os
import struct

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
IR_PATH = os.path.join(REPO, 'minecraft-terrain-cuda_b200', 'model', 'overworld_ir.json')
LIMIT = 1 << 23          # the library accepts |chunk| < 2^23


def _hexd(h):
    return struct.unpack('>d', bytes.fromhex(h[2:]))[0]


def octave_scales(ref_seed, ir_path=IR_PATH):
    """(scale * frequency, noise) for every octave layer of every noise the model samples."""
    with open(ir_path) as f:
        ir = json.load(f)
    out = []
    for n in ir['nodes']:
        t = n['t']
        if t == 'noise':
            for fr in ref_seed.noise_layers(n['noise'])[0]:
                out.append((_hexd(n['xz_scale']) * fr, n['noise']))
        elif t in ('shift_a', 'shift_b', 'shift'):
            for fr in ref_seed.noise_layers(n['noise'])[0]:
                out.append((0.25 * fr, n['noise']))
        elif t == 'blended_noise':
            xm = 684.412 * _hexd(n['xz_scale'])
            out += [(xm * 2.0 ** -k, 'blended limit') for k in range(16)]
            out += [(xm / _hexd(n['xz_factor']) * 2.0 ** -k, 'blended main') for k in range(8)]
    for key in ir['noises']:
        for fr in ref_seed.noise_layers(key)[0]:
            out.append((fr, key))
    return out


def fold_chunks(ref_seed, ir_path=IR_PATH):
    """Sorted distinct chunk coordinates c >= 0 in range whose 16 blocks hold an octave's
    wrap point 2^24 / (scale * frequency)."""
    folds = set()
    for sc, _ in octave_scales(ref_seed, ir_path):
        if sc > 0:
            c = math.floor(2.0 ** 24 / sc / 16)
            if c + 1 < LIMIT:
                folds.add(c)
    return sorted(folds)


def fold_chunk_list(ref_seed, ir_path=IR_PATH):
    """Chunks straddling every fold, on both signs of x and z: for fold chunk f, (f - 1 .. f + 1)
    and (-f - 2 .. -f) paired with the mirrored fold coordinate on the other axis."""
    out = []
    for f in fold_chunks(ref_seed, ir_path):
        for d in (-1, 0, 1):
            out.append((f + d, -f - 1 - d))
            out.append((-f - 1 - d, f + d))
    seen, uniq = set(), []
    for c in out:
        if c not in seen and all(-LIMIT < v < LIMIT for v in c):
            seen.add(c)
            uniq.append(c)
    return uniq


# Reference corpus positions (Corpus.java:185-234): origin, near / far / world border,
# the wrap chunks, chunks at +/-117,187 (the world border read as a chunk coordinate), eroded-badlands and frozen-ocean chunks
# of the model, and chunks past the BlockPos wrap of the aquifer cell locations.
CORPUS = [(0, 0), (1, 0), (0, 1), (-1, -1), (6250, -6250), (-625000, 625000), (1874999, -1874999), (-1874999, 1874999), (6128, -6129),
          (-6129, 6128), (117187, -117187), (-4000, -3360), (-4000, -1440), (-4000, 1600), (2097148, -2097149), (3000000, -5000000),
          (-8388607, 8388607)]
