"""ctypes access to the host twin of the kernel bodies (lib/libterrain_b200_hostcheck.so).

The twin compiles csrc/tb_pipeline.cuh and the generated evaluators for the host, so the
CPU test suite can compare the device code's arithmetic with the reference port without
a GPU. It is test infrastructure; the product never loads it.
"""
import ctypes
import os

import numpy as np

REPO = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
PATH = os.path.join(REPO, 'minecraft-terrain-cuda_b200', 'lib', 'libterrain_b200_hostcheck.so')
_L = None


def available():
    return os.path.exists(PATH)


def lib():
    global _L
    if _L is None:
        L = ctypes.CDLL(PATH)
        vp = ctypes.c_void_p
        L.hc_generate.argtypes = [ctypes.c_int64, vp, vp, ctypes.c_int32, vp, vp, vp]
        L.hc_point.argtypes = [ctypes.c_int64, ctypes.c_int32, vp, ctypes.c_int32, vp]
        L.hc_climate.argtypes = [ctypes.c_int64, vp, ctypes.c_int32, vp]
        L.hc_corners.argtypes = [ctypes.c_int64, vp, ctypes.c_int32, vp]
        L.hc_seed_scalars.argtypes = [ctypes.c_int64, vp, vp]
        L.hc_noise_layers.argtypes = [ctypes.c_int64, ctypes.c_int32, vp, vp, vp, vp]
        L.hc_biome_point.argtypes = [ctypes.c_int64, vp, ctypes.c_int32, vp]
        L.hc_table_errors.argtypes = [ctypes.c_int32, ctypes.c_uint32, vp]
        L.hc_count_ops.argtypes = [ctypes.c_int64, vp, vp, ctypes.c_int32, vp, vp]
        L.hc_set_defer.argtypes = [ctypes.c_int32]
        L.hc_table_errors.restype = ctypes.c_uint32
        _L = L
    return _L


def _p(a):
    return ctypes.c_void_p(a.ctypes.data)


def generate(seed, chunks, aquifer=False):
    a = np.ascontiguousarray(np.asarray(chunks, np.int32).reshape(-1, 2))
    n = a.shape[0]
    cx, cz = np.ascontiguousarray(a[:, 0]), np.ascontiguousarray(a[:, 1])
    b = np.empty((n, 384, 16, 16), np.uint16)
    q = np.empty((n, 1536), np.uint8)
    aq = np.empty((n, 384, 16, 16), np.uint16) if aquifer else None
    lib().hc_generate(int(seed), _p(cx), _p(cz), n, _p(b), _p(q), _p(aq) if aquifer else None)
    return (b, q, aq) if aquifer else (b, q)


def biome_point(seed, xyz):
    """Biome lookups through the single-position path (zoom corner, quart leaf, tie replay)."""
    xyz = np.ascontiguousarray(np.asarray(xyz, np.int32).reshape(-1, 3))
    out = np.empty(xyz.shape[0], np.uint8)
    assert lib().hc_biome_point(int(seed), _p(xyz), xyz.shape[0], _p(out)) == 0
    return out


def point(seed, root, xyz):
    xyz = np.ascontiguousarray(np.asarray(xyz, np.int32).reshape(-1, 3))
    out = np.empty(xyz.shape[0], np.float32)
    assert lib().hc_point(int(seed), root, _p(xyz), xyz.shape[0], _p(out)) == 0
    return out


def climate(seed, xyz):
    xyz = np.ascontiguousarray(np.asarray(xyz, np.int32).reshape(-1, 3))
    out = np.empty((xyz.shape[0], 6), np.float32)
    lib().hc_climate(int(seed), _p(xyz), xyz.shape[0], _p(out))
    return out


def corners(seed, xyz):
    xyz = np.ascontiguousarray(np.asarray(xyz, np.int32).reshape(-1, 3))
    nch = lib().hc_num_channels()
    out = np.empty((xyz.shape[0], nch), np.float32)
    lib().hc_corners(int(seed), _p(xyz), xyz.shape[0], _p(out))
    return out


def seed_scalars(seed):
    a = np.zeros(7, np.int64)
    clay = np.zeros(192, np.int32)
    lib().hc_seed_scalars(int(seed), _p(a), _p(clay))
    return a, clay


def noise_layers(seed, key_index):
    f = np.zeros(128)
    amp = np.zeros(128, np.float32)
    offs = np.zeros(384)
    perms = np.zeros(128 * 256, np.uint8)
    n = lib().hc_noise_layers(int(seed), key_index, _p(f), _p(amp), _p(offs), _p(perms))
    return f[:n], amp[:n], offs[:3 * n].reshape(-1, 3), perms[:256 * n].reshape(-1, 256)


def table_errors(n, cap):
    """(error bits, resolved indices) of n keys through a cap-slot dedupe table (host build)."""
    idx = np.zeros(n, np.int32)
    e = lib().hc_table_errors(n, cap, _p(idx))
    return int(e), idx


STAGES = ['nb_insert', 'nb_resolve', 'climate_col', 'climate_quart', 'chain', 'cc_insert', 'cc_resolve', 'corner_col', 'corner', 'zoom_table',
          'zoom_uniform', 'sg_insert', 'sg_resolve', 'surface_level', 'aquifer_cell', 'aquifer_query', 'aquifer_skip', 'init_heights', 'fill',
          'surface1', 'block_biome', 'walk_rules', 'surface_frozen', 'gather', 'axis_insert', 'axis_number', 'axis_fill', 'walk_deferred']
OP_KINDS = ['vol_octave', 'vol_octave_smeared', 'point_octave', 'point_octave_smeared', 'simplex']


def count_ops(seed, chunks):
    """Samples per stage of one batch of chunks through the host twin: ({stage: {kind: count}},
    {'corner_columns', 'surface_quarts', 'biome_chunks'})."""
    a = np.ascontiguousarray(np.asarray(chunks, np.int32).reshape(-1, 2))
    cx, cz = np.ascontiguousarray(a[:, 0]), np.ascontiguousarray(a[:, 1])
    counts = np.zeros((len(STAGES), len(OP_KINDS)), np.int64)
    meta = np.zeros(4, np.int32)
    if lib().hc_count_ops(int(seed), _p(cx), _p(cz), a.shape[0], _p(counts), _p(meta)) != 0:
        raise RuntimeError('hc_count_ops failed')
    per = {s: {k: int(counts[i, j]) for j, k in enumerate(OP_KINDS)} for i, s in enumerate(STAGES)}
    return per, {'corner_columns': int(meta[0]), 'surface_quarts': int(meta[1]), 'biome_chunks': int(meta[2]), 'deferred_blocks': int(meta[3])}


def set_defer(per_chunk):
    """Blocks per chunk the twin's deferred list holds from now on (0: the walk keeps all)."""
    lib().hc_set_defer(int(per_chunk))
