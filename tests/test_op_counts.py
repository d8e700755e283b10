"""The per-chunk work counts behind the bench's compute roofline: the committed
op_counts.json belongs to the compiled model (its SHA-256 of the model files), the counting
build of the reference port reproduces its corner-phase count, and the kernel bodies'
lazy per-point evaluation never samples more octaves per corner point than the port's
eager volume path does. CPU only."""
import hashlib
import json
import os
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
MODEL = os.path.join(REPO, 'minecraft-terrain-cuda_b200', 'model')
sys.path.insert(0, os.path.join(HERE, 'hostcheck'))


@pytest.fixture(scope='module')
def counts():
    with open(os.path.join(MODEL, 'op_counts.json')) as f:
        return json.load(f)


def test_counts_are_for_the_compiled_model(counts):
    for name, sha in counts['model'].items():
        with open(os.path.join(MODEL, name), 'rb') as f:
            assert hashlib.sha256(f.read()).hexdigest() == sha, name


def test_port_counting_build_reproduces_the_corner_phase(counts):
    import count_ops
    if not count_ops.available():
        pytest.skip('counting build not made (make -C oracle count)')
    c = count_ops.Counter()
    per = count_ops.summarize(c.count(count_ops.SEED, [(x, z) for z in range(2) for x in range(2)], threads=4), 4)
    assert per['corners']['vol_octave'] == counts['per_chunk']['corners']['vol_octave']   # eager: the same for every chunk
    assert per['biome']['rtree_distance'] > 0 and per['surface']['zoom_corner'] > 0


def test_lazy_kernel_samples_do_not_exceed_the_port(counts):
    import hostcheck
    if not hostcheck.available():
        pytest.skip('host twin not built')
    import bench
    per, meta = hostcheck.count_ops(bench.SEED, bench.region_chunks(0, 0, 4))
    points = meta['corner_columns'] * 49
    lazy = sum(per['corner'].values()) / points
    port = (counts['per_chunk']['corners']['vol_octave'] + counts['per_chunk']['corners']['point_octave']) / (25 * 49)
    assert 0 < lazy <= port
    committed = sum(counts['kernels']['per_kernel']['corner']['samples_per_unit'].values())
    assert abs(lazy - committed) / committed < 0.25          # a different sample of the same terrain
