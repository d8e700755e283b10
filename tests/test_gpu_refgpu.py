"""The bench's side arm, the reference's own GPU generator (mcc::cuda::FullTerrainGenerator,
cuda/src/terrain.cu) built for sm_100a from the same model files (baseline/), computes the
same bytes as the reference port and as this library on the benched workload: a 32x32-chunk
region of the ladder's origin region and the reference corpus chunks inside the world
border (|chunk| <= 1,874,999). Far chunks past the BlockPos wrap of the aquifer cell
locations (|chunk| >= 2^21 - 1, outside the world border) are left out: there the
reference's GPU generator differs from its own port, and this library follows the port.
Integer outputs, zero tolerance.
"""
import os
import sys

import numpy as np
import pytest

import bench
import corpus

pytestmark = pytest.mark.gpu

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), 'baseline'))
import refgpu  # noqa: E402


@pytest.fixture(scope='module')
def ref_gpu():
    if not refgpu.available():
        pytest.skip('reference GPU generator not built (make -C baseline)')
    g = refgpu.RefGpuGenerator(max_batch_chunks=1024, pipeline_slots=2)
    yield g
    g.close()


def test_reference_gpu_equals_port_and_ours_on_the_benched_region(ref_gpu, gpu_gen, ref_model):
    chunks = bench.region_chunks(0, 0, 32)
    ref_gpu.set_seed(bench.SEED)
    t8, b8 = ref_gpu.generate(chunks)
    gpu_gen.set_seed(bench.SEED)
    o8, ob = gpu_gen.generate_u8(chunks)
    rb, rq = ref_model.seed(bench.SEED).generate(chunks)
    assert (t8.astype(np.uint16) == rb).all() and (b8 == rq).all()
    assert (o8 == t8).all() and (ob == b8).all()


@pytest.mark.parametrize('seed', [0, bench.SEED])
def test_reference_gpu_equals_port_inside_the_world_border(ref_gpu, ref_model, seed):
    chunks = [c for c in corpus.CORPUS if max(abs(c[0]), abs(c[1])) <= 1874999]
    ref_gpu.set_seed(seed)
    t8, b8 = ref_gpu.generate(chunks)
    rb, rq = ref_model.seed(seed).generate(chunks)
    bad = [c for i, c in enumerate(chunks) if (t8[i].astype(np.uint16) != rb[i]).any() or (b8[i] != rq[i]).any()]
    assert not bad, bad
