"""TEST INFRASTRUCTURE: the CPU restatement of the flythrough renderer's ray march
(oracle/render_restate.cpp, built into oracle/_ref/librender_restate.so by make -C oracle
render). Only tests/ and the bench's checks use it; the product never loads it."""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, '_ref', 'librender_restate.so')
_lib = None


def available():
    return os.path.exists(LIB)


def render(vox, cells, slots, born, ids, cam, top, side, caps, width, height, frame, threads=None):
    """(rgb (h, w, 3) u8, hits (h, w, 4) int32) of one frame traced on the CPU from a window
    state and the frame's parameters (TerrainViewer.state / .params)."""
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(LIB)
        _lib.rr_render.argtypes = [ctypes.c_void_p] * 9 + [ctypes.c_int32] * 4 + [ctypes.c_void_p] * 2
    rgb = np.empty((height, width, 3), np.uint8)
    hits = np.empty((height, width, 4), np.int32)
    arrs = [np.ascontiguousarray(a) for a in (vox, cells, slots, born, ids, cam, top, side, caps)]
    _lib.rr_render(*[ctypes.c_void_p(a.ctypes.data) for a in arrs], int(width), int(height), int(frame), int(threads or os.cpu_count()),
                   ctypes.c_void_p(rgb.ctypes.data), ctypes.c_void_p(hits.ctypes.data))
    return rgb, hits
