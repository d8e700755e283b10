"""Golden fixtures (tests/golden/, written by tests/golden/make_golden.py from the
reference's own C++ port): the reference build and the product's host twin reproduce
every digest. The GPU counterpart lives in tests/test_gpu_golden.py."""
import hashlib
import json
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = json.load(open(os.path.join(HERE, 'golden', 'terrain_digests.json')))


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def test_golden_matches_the_compiled_model():
    import ref_oracle
    assert GOLDEN['model_ir_sha256'] == hashlib.sha256(open(ref_oracle.IR_PATH, 'rb').read()).hexdigest()
    assert GOLDEN['model_terrain_sha256'] == hashlib.sha256(open(ref_oracle.TERRAIN_PATH, 'rb').read()).hexdigest()


@pytest.mark.parametrize('seed', list(GOLDEN['seeds'])[:6])
def test_reference_port_reproduces_golden(ref_model, seed):
    chunks = GOLDEN['chunks']
    b, q = ref_model.seed(int(seed)).generate(chunks)
    for i, c in enumerate(chunks):
        assert [digest(b[i].astype('<u2')), digest(q[i])] == GOLDEN['seeds'][seed][i], c


@pytest.mark.parametrize('seed', list(GOLDEN['seeds'])[6:9])
def test_host_twin_reproduces_golden(seed):
    sys.path.insert(0, os.path.join(HERE, 'hostcheck'))
    import hostcheck
    if not hostcheck.available():
        pytest.skip('host twin not built')
    chunks = GOLDEN['chunks'][7:]
    b, q = hostcheck.generate(int(seed), chunks)
    for i, c in enumerate(chunks):
        assert [digest(b[i].astype('<u2')), digest(q[i])] == GOLDEN['seeds'][seed][7 + i], c
