"""TEST INFRASTRUCTURE: Python access to the reference's own C++ port.

oracle/_ref/libref_terrain.so is the reference's cpu/ sources (bonquifo/minecraft-terrain-cuda)
compiled in place by oracle/Makefile, plus the thin C binding oracle/ref_driver.cpp.
Only tests/, bench.py's CPU-baseline leg and __graft_entry__.smoke() use this module, as
the checker; the product never imports it.

The reference port is the correctness bar of the TERRAIN step: cpu_generate_terrain /
cpu_terrain_from_biomes (cpu/src/terrain.cpp:750-810).
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, '_ref', 'libref_terrain.so')
REPO = os.path.dirname(HERE)
MODEL_DIR = os.path.join(REPO, 'minecraft-terrain-cuda_b200', 'model')
IR_PATH = os.path.join(MODEL_DIR, 'overworld_ir.json')
TERRAIN_PATH = os.path.join(MODEL_DIR, 'overworld_terrain.json')

_lib = None


def available():
    return os.path.exists(REF_LIB)


def reference_root():
    """Where the reference's sources lie: $TERRAIN_REFERENCE_ROOT, else /root/reference."""
    return os.environ.get('TERRAIN_REFERENCE_ROOT', '/root/reference')


def build(ref_root=None):
    """Compiles oracle/_ref from the reference sources (only where they exist)."""
    import subprocess
    subprocess.check_call(['make', '-s', '-C', HERE, 'REF=%s' % (ref_root or reference_root()), '-j8'])


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise FileNotFoundError('reference oracle not built: %s' % REF_LIB)
        L = ctypes.CDLL(REF_LIB)
        vp = ctypes.c_void_p
        L.ref_open.restype = vp
        L.ref_open.argtypes = [ctypes.c_char_p, ctypes.c_char_p]
        L.ref_seed.restype = vp
        L.ref_seed.argtypes = [vp, ctypes.c_int64]
        L.ref_seed_free.argtypes = [vp]
        L.ref_last_error.restype = ctypes.c_char_p
        L.ref_generate.argtypes = [vp, vp, vp, ctypes.c_int32, ctypes.c_int32, vp, vp, vp, vp]
        L.ref_chunk_biomes.argtypes = [vp, ctypes.c_int32, ctypes.c_int32, vp]
        L.ref_biome_lookup.argtypes = [vp, vp, ctypes.c_int32, ctypes.c_int32, vp]
        L.ref_sample.argtypes = [vp, ctypes.c_int32, vp, vp]
        L.ref_point.argtypes = [vp, ctypes.c_int32, vp, ctypes.c_int32, vp]
        L.ref_seed_scalars.argtypes = [vp, vp, vp]
        L.ref_noise_layers.argtypes = [vp, ctypes.c_char_p, ctypes.c_int32, vp, vp, vp, vp]
        L.ref_md5.argtypes = [ctypes.c_char_p, ctypes.c_int64, vp]
        L.ref_zoom_seed.restype = ctypes.c_int64
        L.ref_zoom_seed.argtypes = [ctypes.c_int64]
        L.ref_xoroshiro_longs.restype = ctypes.c_int64
        L.ref_xoroshiro_longs.argtypes = [ctypes.c_int64, ctypes.c_int32, vp]
        L.ref_mth_get_seed.restype = ctypes.c_int64
        L.ref_mth_get_seed.argtypes = [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32]
        L.ref_quantize.restype = ctypes.c_int64
        L.ref_quantize.argtypes = [ctypes.c_float]
        L.ref_stream_sum.restype = ctypes.c_double
        L.ref_stream_sum.argtypes = [vp, ctypes.c_int32]
        _lib = L
    return _lib


def _p(a):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


class RefModel:
    def __init__(self, ir_path=IR_PATH, terrain_path=TERRAIN_PATH):
        L = lib()
        self.L = L
        self.h = L.ref_open(ir_path.encode(), terrain_path.encode())
        if not self.h:
            raise RuntimeError(L.ref_last_error().decode())
        info = (ctypes.c_int32 * 9)()
        L.ref_model_info(ctypes.c_void_p(self.h), info)
        self.min_y, self.height, self.sea_level = info[0], info[1], info[2]

    def seed(self, seed):
        return RefSeed(self, seed)


class RefSeed:
    def __init__(self, model, seed):
        self.m = model
        self.L = model.L
        self.h = self.L.ref_seed(ctypes.c_void_p(model.h), int(seed))
        if not self.h:
            raise RuntimeError(self.L.ref_last_error().decode())

    def __del__(self):
        try:
            self.L.ref_seed_free(ctypes.c_void_p(self.h))
        except Exception:
            pass

    def generate(self, chunks, threads=None, aquifer=False, density=False):
        """TERRAIN step for a chunk list: (blocks u16 (n, h, 16, 16), biomes u8 (n, 1536)[, aquifer u16][, density f32]),
        density being the final density per block (ChunkTerrain::density, cpu/src/terrain.cpp:787-795)."""
        a = np.ascontiguousarray(np.asarray(chunks, np.int32).reshape(-1, 2))
        n = a.shape[0]
        cx = np.ascontiguousarray(a[:, 0])
        cz = np.ascontiguousarray(a[:, 1])
        h = self.m.height
        blocks = np.empty((n, h, 16, 16), np.uint16)
        biomes = np.empty((n, 16 * (h // 4)), np.uint8)
        aq = np.empty((n, h, 16, 16), np.uint16) if aquifer else None
        dens = np.empty((n, h, 16, 16), np.float32) if density else None
        st = self.L.ref_generate(ctypes.c_void_p(self.h), _p(cx), _p(cz), n, threads or os.cpu_count(), _p(blocks), _p(biomes), _p(aq), _p(dens))
        if st != 0:
            raise RuntimeError(self.L.ref_last_error().decode())
        return (blocks, biomes) + ((aq,) if aquifer else ()) + ((dens,) if density else ())

    def biome_lookup(self, xyz, threads=None):
        xyz = np.ascontiguousarray(np.asarray(xyz, np.int32).reshape(-1, 3))
        out = np.empty(xyz.shape[0], np.uint8)
        st = self.L.ref_biome_lookup(ctypes.c_void_p(self.h), _p(xyz), xyz.shape[0], threads or os.cpu_count(), _p(out))
        if st != 0:
            raise RuntimeError(self.L.ref_last_error().decode())
        return out

    def sample(self, node, vol):
        v = np.asarray(vol, np.int32)
        out = np.empty(int(v[0] * v[1] * v[2]), np.float32)
        if self.L.ref_sample(ctypes.c_void_p(self.h), int(node), _p(v), _p(out)) != 0:
            raise RuntimeError(self.L.ref_last_error().decode())
        return out

    def point(self, node, xyz):
        xyz = np.ascontiguousarray(np.asarray(xyz, np.int32).reshape(-1, 3))
        out = np.empty(xyz.shape[0], np.float32)
        if self.L.ref_point(ctypes.c_void_p(self.h), int(node), _p(xyz), xyz.shape[0], _p(out)) != 0:
            raise RuntimeError(self.L.ref_last_error().decode())
        return out

    def scalars(self):
        a = np.zeros(7, np.int64)
        clay = np.zeros(192, np.int32)
        self.L.ref_seed_scalars(ctypes.c_void_p(self.h), _p(a), _p(clay))
        return a, clay

    def noise_layers(self, key, max_layers=128):
        f = np.zeros(max_layers)
        amp = np.zeros(max_layers, np.float32)
        offs = np.zeros(3 * max_layers)
        perms = np.zeros(256 * max_layers, np.uint8)
        n = self.L.ref_noise_layers(ctypes.c_void_p(self.h), key.encode(), max_layers, _p(f), _p(amp), _p(offs), _p(perms))
        return f[:n], amp[:n], offs[:3 * n].reshape(-1, 3), perms[:256 * n].reshape(-1, 256)
