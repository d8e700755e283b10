"""Shared test setup: markers, import paths and lazily built handles.

Tests marked gpu need a B200 (sm_100a) and call the product through its C ABI
(include/terrain_b200.h). Everything else runs on the CPU: the oracle against
known-answer vectors and golden fixtures, the host-built kernel bodies against the
oracle, and the C-ABI library's symbol table.
"""
import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, 'minecraft-terrain-cuda_b200')
for p in (REPO, PKG, os.path.join(REPO, 'oracle')):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line('markers', 'gpu: needs a B200 GPU; calls the sm_100a library through its C ABI')


@pytest.fixture(scope='session')
def ref_model():
    import ref_oracle
    if not ref_oracle.available():
        pytest.skip('reference oracle not built (make -C oracle)')
    return ref_oracle.RefModel()


@pytest.fixture(scope='session')
def gpu_gen():
    import terrain_b200
    g = terrain_b200.TerrainGenerator(max_batch_chunks=1024)
    yield g
    g.close()
