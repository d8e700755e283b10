"""The reference's own GPU TERRAIN generator (bonquifo/minecraft-terrain-cuda,
mcc::cuda::FullTerrainGenerator, cuda/src/terrain.cu), built unchanged for sm_100a by
baseline/Makefile from the same model files as this repository's library.

A timed side arm of bench.py (the reference pipeline on the same B200 and model); the
product never imports it.

    g = RefGpuGenerator(max_batch_chunks=4096, pipeline_slots=2)
    g.set_seed(seed)
    terrain_u8, biomes = g.generate(chunks, terrain_out, biomes_out)
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, '_refgpu', 'librefgpu.so')
MODEL = os.path.join(os.path.dirname(HERE), 'minecraft-terrain-cuda_b200', 'model')

_lib = None


def available():
    return os.path.exists(LIB)


def lib():
    global _lib
    if _lib is None:
        L = ctypes.CDLL(LIB)
        vp = ctypes.c_void_p
        L.refgpu_open.restype = vp
        L.refgpu_open.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int32, ctypes.c_int32]
        L.refgpu_close.argtypes = [vp]
        L.refgpu_set_seed.argtypes = [vp, ctypes.c_int64]
        L.refgpu_generate.argtypes = [vp, vp, ctypes.c_int32, vp, vp, vp, vp]
        L.refgpu_last_error.restype = ctypes.c_char_p
        L.refgpu_alloc_pinned.restype = vp
        L.refgpu_alloc_pinned.argtypes = [ctypes.c_size_t]
        L.refgpu_free_pinned.argtypes = [vp]
        _lib = L
    return _lib


def _p(a):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


class RefGpuGenerator:
    STAGES = ('h2d_ms', 'biome_ms', 'noise_ms', 'aquifer_ms', 'fill_ms', 'surface_ms', 'd2h_ms', 'wall_ms')

    def __init__(self, max_batch_chunks=256, pipeline_slots=2):
        self.L = lib()
        self.h = self.L.refgpu_open(os.path.join(MODEL, 'overworld_ir.json').encode(), os.path.join(MODEL, 'overworld_terrain.json').encode(),
                                    int(max_batch_chunks), int(pipeline_slots))
        if not self.h:
            raise RuntimeError('reference GPU generator: ' + self.L.refgpu_last_error().decode())

    def close(self):
        if self.h:
            self.L.refgpu_close(ctypes.c_void_p(self.h))
            self.h = None

    def set_seed(self, seed):
        if self.L.refgpu_set_seed(ctypes.c_void_p(self.h), int(seed)) != 0:
            raise RuntimeError(self.L.refgpu_last_error().decode())

    def generate(self, chunks, terrain_out=None, biomes_out=None, timing=False):
        """u8 palette index per block (n, 384, 16, 16) and u8 quart biomes (n, 1536); with
        timing, also the reference's TerrainTiming stage times (ms)."""
        a = np.ascontiguousarray(np.asarray(chunks, np.int32).reshape(-1, 2))
        n = a.shape[0]
        t8 = terrain_out if terrain_out is not None else np.empty((n, 384, 16, 16), np.uint8)
        b8 = biomes_out if biomes_out is not None else np.empty((n, 1536), np.uint8)
        st = np.zeros(8) if timing else None
        if self.L.refgpu_generate(ctypes.c_void_p(self.h), _p(a), n, _p(t8), _p(b8), None, _p(st)) != 0:
            raise RuntimeError(self.L.refgpu_last_error().decode())
        return (t8, b8, dict(zip(self.STAGES, st.tolist()))) if timing else (t8, b8)
