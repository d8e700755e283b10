"""GPU parity at the density level: tg_generate_density (the final density the fill kernel
evaluates for every block) against the reference port's per-block final density
(ChunkTerrain::density, cpu/src/terrain.cpp:787-795), compared as raw f32 bits; this is
the reference's own level L2 check (tests/test_chunks.cpp:28-70, raw-bit compares).

Chunks: the reference corpus positions, and the fold chunks of every noise octave of the
model (tests/corpus.py), where the blocks, biomes and densities are all compared.
Bar: bit-exact, zero tolerance (the f32 values must have identical bits).
"""
import numpy as np
import pytest

import corpus

pytestmark = pytest.mark.gpu


def mismatches(got, want):
    g = got.reshape(got.shape[0], -1).view(np.uint32)
    w = want.reshape(want.shape[0], -1).view(np.uint32)
    return (g != w).sum(1)


@pytest.mark.parametrize('seed', [0, -1, 12345, -4172144997902289642])
def test_density_matches_reference_on_corpus(gpu_gen, ref_model, seed):
    gpu_gen.set_seed(seed)
    d = gpu_gen.generate_density(corpus.CORPUS)
    _, _, rd = ref_model.seed(seed).generate(corpus.CORPUS, density=True)
    bad = mismatches(d, rd)
    assert not bad.any(), 'seed %d: density bit mismatches per chunk %s' % (seed, dict(zip(map(tuple, corpus.CORPUS), bad.tolist())))
    assert np.isfinite(d).all()


def test_density_blocks_and_biomes_at_fold_chunks(gpu_gen, ref_model):
    """Every chunk that straddles an octave's wrap point (both signs, each with its
    neighbours): density bits, block states and quart biomes equal the reference."""
    seed = 20260607
    ref = ref_model.seed(seed)
    chunks = corpus.fold_chunk_list(ref)
    assert len(chunks) >= 300 and (6128, -6129) in chunks
    gpu_gen.set_seed(seed)
    d = gpu_gen.generate_density(chunks)
    b, q = gpu_gen.generate(chunks)
    rb, rq, rd = ref.generate(chunks, density=True)
    bad_d = mismatches(d, rd)
    bad_b = (b != rb).reshape(len(chunks), -1).sum(1) + (q != rq).sum(1)
    assert not bad_d.any(), 'density mismatches at %s' % [chunks[i] for i in np.nonzero(bad_d)[0][:10]]
    assert not bad_b.any(), 'block / biome mismatches at %s' % [chunks[i] for i in np.nonzero(bad_b)[0][:10]]


def test_density_output_leaves_blocks_unchanged(gpu_gen):
    """The density pass runs the same TERRAIN step: the blocks of the plain call are unchanged
    by a density call in between, on the same generator."""
    gpu_gen.set_seed(77)
    chunks = [(3, 4), (-9, 2), (6128, 6128)]
    b1, q1 = gpu_gen.generate(chunks)
    gpu_gen.generate_density(chunks)
    b2, q2 = gpu_gen.generate(chunks)
    assert (b1 == b2).all() and (q1 == q2).all()
