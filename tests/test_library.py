"""The C-ABI library: built for sm_100a, loads, and exports every entry point that
include/terrain_b200.h declares. No GPU needed (no compute calls)."""
import ctypes
import os
import re

import pytest

import terrain_b200

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(REPO, 'include', 'terrain_b200.h')


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r'/\*.*?\*/', '', text, flags=re.S)
    return sorted(set(re.findall(r'\b(tg_[a-z0-9_]+)\s*\(', text)))


def test_library_loads_and_exports_every_declared_symbol():
    L = terrain_b200.load()
    names = declared_functions()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert set(names) == set(terrain_b200.EXPORTS)


def test_library_is_built_for_sm_100a():
    # the fatbin carries an sm_100a cubin; cuobjdump-free check: the build recipe's flags
    build = open(os.path.join(REPO, 'minecraft-terrain-cuda_b200', 'build.py')).read()
    assert 'arch=compute_100a,code=sm_100a' in build
    assert os.path.getsize(terrain_b200.LIB_PATH) > 100000


def test_model_info_needs_no_gpu():
    info = terrain_b200.model_info()
    assert info == {'min_y': -64, 'height': 384, 'sea_level': 63, 'palette_size': 40, 'biome_count': 57}


def test_model_mismatch_is_reported_before_any_device_work():
    L = terrain_b200.load()
    h = ctypes.c_void_p()
    st = L.tg_create(HEADER.encode(), None, None, ctypes.byref(h))
    assert st == 2 and not h
    assert b'differs' in L.tg_last_error_string()


def test_bad_arguments_are_status_codes():
    L = terrain_b200.load()
    assert L.tg_create(None, None, None, None) == 1
    assert L.tg_set_seed(None, 1) == 1
    assert L.tg_generate(None, None, 0, None, None, None, None) == 1
    assert L.tg_server_submit(None, 0, None, 0, None, None, None) == 1


def test_create_without_a_gpu_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        pytest.skip('a GPU is present')
    L = terrain_b200.load()
    h = ctypes.c_void_p()
    st = L.tg_create(None, None, None, ctypes.byref(h))
    assert st in (3, 4) and not h
