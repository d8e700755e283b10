"""Known-answer tests: the reference's own unit vectors (tests/test_l0.cpp:36-85 of the
reference: Java casts, floor, floorDiv/Mod, min/max with signed zeros, MD5 vectors, RNG
units) and the golden RNG / hash vectors of tests/golden/kat.json, checked against the
product's host code (built into the host twin) and, where present, the reference port."""
import ctypes
import hashlib
import json
import math
import os
import struct

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HOSTLIB = os.path.join(REPO, 'minecraft-terrain-cuda_b200', 'lib', 'libterrain_b200_hostcheck.so')
KAT = json.load(open(os.path.join(REPO, 'tests', 'golden', 'kat.json')))


@pytest.fixture(scope='module')
def H():
    if not os.path.exists(HOSTLIB):
        pytest.skip('host twin not built (python minecraft-terrain-cuda_b200/build.py --host)')
    L = ctypes.CDLL(HOSTLIB)
    L.hc_d2i.argtypes = [ctypes.c_double]
    L.hc_jfloor.argtypes = [ctypes.c_double]
    L.hc_jmin.argtypes = L.hc_jmax.argtypes = [ctypes.c_float, ctypes.c_float]
    L.hc_jmin.restype = L.hc_jmax.restype = ctypes.c_float
    L.hc_fabs.argtypes = [ctypes.c_float]
    L.hc_fabs.restype = ctypes.c_float
    L.hc_f2l.argtypes = [ctypes.c_float]
    L.hc_f2l.restype = ctypes.c_int64
    L.hc_nwrap.argtypes = [ctypes.c_double]
    L.hc_nwrap.restype = ctypes.c_double
    L.hc_grad.restype = ctypes.c_float
    L.hc_pos_seed.restype = ctypes.c_int64
    L.hc_xoroshiro_longs.argtypes = [ctypes.c_int64, ctypes.c_int32, ctypes.c_void_p]
    L.hc_stream_sum.argtypes = [ctypes.c_void_p, ctypes.c_int32]
    L.hc_stream_sum.restype = ctypes.c_double
    L.hc_zoom_seed.argtypes = [ctypes.c_int64]
    L.hc_zoom_seed.restype = ctypes.c_int64
    L.hc_md5.argtypes = L.hc_sha256.argtypes = [ctypes.c_char_p, ctypes.c_int64, ctypes.c_void_p]
    return L


def fbits(v):
    return struct.unpack('<I', struct.pack('<f', v))[0]


def test_java_casts_and_floor(H):
    assert H.hc_d2i(float('nan')) == 0
    assert H.hc_d2i(1e10) == 2147483647 and H.hc_d2i(-1e10) == -2147483648
    assert H.hc_d2i(-0.5) == 0 and H.hc_d2i(2147483647.5) == 2147483647
    assert H.hc_jfloor(-0.5) == -1 and H.hc_jfloor(-1e-300) == -1 and H.hc_jfloor(3e9) == 2147483647
    assert H.hc_jfloor(float('nan')) == 0
    assert H.hc_fdiv(-1, 4) == -1 and H.hc_fmod(-1, 4) == 3 and H.hc_fdiv(-8, 8) == -1 and H.hc_fmod(7, 4) == 3
    assert H.hc_f2l(float('nan')) == 0 and H.hc_f2l(3.4e38) == (1 << 63) - 1 and H.hc_f2l(-3.4e38) == -(1 << 63)


def test_java_min_max_signed_zero_and_nan(H):
    assert fbits(H.hc_jmin(0.0, -0.0)) == 0x80000000 and fbits(H.hc_jmin(-0.0, 0.0)) == 0x80000000
    assert fbits(H.hc_jmax(-0.0, 0.0)) == 0 and fbits(H.hc_jmax(0.0, -0.0)) == 0
    assert math.isnan(H.hc_jmin(float('nan'), 1.0)) and math.isnan(H.hc_jmin(1.0, float('nan')))
    assert fbits(H.hc_fabs(-0.0)) == 0


def test_gradient_table(H):
    table = [(1, 1, 0), (-1, 1, 0), (1, -1, 0), (-1, -1, 0), (1, 0, 1), (-1, 0, 1), (1, 0, -1), (-1, 0, -1), (0, 1, 1), (0, -1, 1), (0, 1, -1),
             (0, -1, -1), (1, 1, 0), (0, -1, 1), (-1, 1, 0), (0, -1, -1)]
    for h in range(32):
        for c in range(3):
            assert H.hc_grad(h, c) == table[h & 15][c]


def test_wrap_limit(H):
    lim = float.fromhex('0x1.fffffffffffffp+23')
    assert H.hc_nwrap(lim) != lim and H.hc_nwrap(-lim) == -lim and H.hc_nwrap(1e7) == 1e7
    assert H.hc_nwrap(2.0 ** 24) == 2.0 ** 24 - 33554432.0


def test_md5_and_sha256(H):
    for s, want in KAT['md5'].items():
        out = np.zeros(16, np.uint8)
        H.hc_md5(s.encode(), len(s), out.ctypes.data)
        assert out.tobytes().hex() == want == hashlib.md5(s.encode()).hexdigest()
    for s in [b'', b'abc', b'a' * 1000, bytes(range(256)) * 3]:
        out = np.zeros(32, np.uint8)
        H.hc_sha256(s, len(s), out.ctypes.data)
        assert out.tobytes().hex() == hashlib.sha256(s).hexdigest()


def test_xoroshiro_streams_and_zoom_seeds(H):
    for sd, want in KAT['xoroshiro_longs'].items():
        out = np.zeros(8, np.int64)
        H.hc_xoroshiro_longs(int(sd), 8, out.ctypes.data)
        assert [int(v) for v in out] == want
        assert H.hc_zoom_seed(int(sd)) == KAT['zoom_seed'][sd]


def test_positional_seed(H):
    for x, y, z, want in KAT['mth_get_seed']:
        assert H.hc_pos_seed(x, y, z) == want


def test_stream_sum(H):
    for vals, want in KAT['stream_sum']:
        a = np.array(vals, np.float64)
        got = H.hc_stream_sum(a.ctypes.data, len(vals))
        assert got == want or (math.isnan(got) and math.isnan(want))


def test_quantize(H):
    for v, want in KAT['quantize']:
        f = float('nan') if v == 'nan' else v
        with np.errstate(over='ignore', invalid='ignore'):
            q = np.float32(np.float32(f) * np.float32(10000.0))
        assert H.hc_f2l(q) == want
