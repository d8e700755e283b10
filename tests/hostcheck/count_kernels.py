"""Samples each kernel of the TERRAIN step evaluates, counted on the host twin of the kernel
bodies (TEST AND MEASUREMENT INFRASTRUCTURE; the device build never counts).

The twin runs the same per-element bodies as the sm_100a kernels, stage by stage, with a
count per octave sample (volume, smeared volume, point, smeared point) and per simplex
sample in the noise primitives. Unlike the reference port's volume path, which evaluates
both branches of every choice node over a whole volume, the bodies evaluate density
functions lazily per point (the same values: the functions are pure), so these are the
samples the kernels actually do. Per stage the counts are normalised by the stage's work
items (corner points for the corner kernels, distinct quarts for surface levels, chunks
otherwise) so that the bench can scale them to any launch.

    python tests/hostcheck/count_kernels.py [--side 16]    # updates op_counts.json['kernels']
"""
import argparse
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [HERE, REPO]
import bench  # noqa: E402
import hostcheck  # noqa: E402

OUT = os.path.join(REPO, 'minecraft-terrain-cuda_b200', 'model', 'op_counts.json')
ROWS = 49   # corner rows per corner column


def main(argv):
    ap = argparse.ArgumentParser()
    ap.add_argument('--side', type=int, default=16)
    args = ap.parse_args(argv)
    side = args.side
    total = {s: {k: 0 for k in hostcheck.OP_KINDS} for s in hostcheck.STAGES}
    meta_t = {'corner_columns': 0, 'surface_quarts': 0, 'biome_chunks': 0, 'deferred_blocks': 0}
    for _, x0, z0 in bench.REGIONS:
        per, meta = hostcheck.count_ops(bench.SEED, bench.region_chunks(x0, z0, side))
        for s in per:
            for k in per[s]:
                total[s][k] += per[s][k]
        for k in meta:
            meta_t[k] += meta[k]
    n = 3 * side * side
    unit = {'corner_col': ('corner column', meta_t['corner_columns']), 'corner': ('corner point', meta_t['corner_columns'] * ROWS),
            'surface_level': ('distinct surface-level quart', meta_t['surface_quarts']),
            'climate_col': ('biome chunk', meta_t['biome_chunks']), 'climate_quart': ('biome chunk', meta_t['biome_chunks'])}
    kernels = {}
    for s, c in total.items():
        if not any(c.values()):
            continue
        name, count = unit.get(s, ('chunk', n))
        kernels[s] = {'per': name, 'samples_per_unit': {k: round(v / count, 4) for k, v in c.items() if v}}
    with open(OUT) as f:
        doc = json.load(f)
    doc['kernels'] = {'what': 'samples each kernel evaluates (lazy per-point evaluation), counted on the host twin of the kernel bodies, '
                              'per work unit of the kernel', 'sample': '%dx%d chunks at the corner of each ladder region, one batch per region' % (side, side),
                      'seed': bench.SEED, 'per_kernel': kernels,
                      'units_in_sample': {'chunks': n, 'corner_columns': meta_t['corner_columns'], 'surface_quarts': meta_t['surface_quarts'],
                                          'biome_chunks': meta_t['biome_chunks'], 'walk_deferred_blocks': meta_t['deferred_blocks']}}
    with open(OUT, 'w') as f:
        json.dump(doc, f, indent=1, sort_keys=True)
        f.write('\n')
    print(json.dumps(kernels, indent=1))


if __name__ == '__main__':
    main(sys.argv[1:])
