"""GPU against the golden digests (no oracle needed on the box): every seed and chunk of
the reference-shaped corpus in tests/golden/terrain_digests.json."""
import hashlib
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GOLDEN = json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden', 'terrain_digests.json')))


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.mark.parametrize('seed', list(GOLDEN['seeds']))
def test_gpu_reproduces_golden(gpu_gen, seed):
    chunks = GOLDEN['chunks']
    gpu_gen.set_seed(int(seed))
    b, q = gpu_gen.generate(chunks)
    for i, c in enumerate(chunks):
        assert [digest(b[i].astype('<u2')), digest(q[i])] == GOLDEN['seeds'][seed][i], c
