"""The project-authored world model: it exercises everything the reference's loaders
accept (minus 'log', which the reference rejects), loads in the reference port, and the
code generator enforces the structure the TERRAIN step relies on."""
import collections
import copy
import json
import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
MODEL = os.path.join(REPO, 'minecraft-terrain-cuda_b200', 'model')
sys.path.insert(0, os.path.join(REPO, 'minecraft-terrain-cuda_b200', 'codegen'))
import gen_eval  # noqa: E402

IR = json.load(open(os.path.join(MODEL, 'overworld_ir.json')))
TM = json.load(open(os.path.join(MODEL, 'overworld_terrain.json')))


def test_every_node_type_op_and_tiling():
    types = collections.Counter(n['t'] for n in IR['nodes'])
    for t in ('cache', 'constant', 'simple', 'gradient', 'noise', 'shift_a', 'shift_b', 'shift', 'blended_noise', 'binary', 'unary', 'clamp', 'lerp',
              'range_choice', 'interval_select', 'spline', 'interpolated', 'slice', 'blend_density', 'find_top_surface'):
        assert types[t] > 0, t
    ops = {n['op'] for n in IR['nodes'] if n['t'] == 'binary'}
    assert ops == {'add', 'sub', 'mul', 'div', 'min', 'max'}
    un = {n['op'] for n in IR['nodes'] if n['t'] == 'unary'}
    assert un == {'abs', 'square', 'cube', 'sqrt', 'half_negative', 'quarter_negative', 'reciprocal', 'negate', 'squeeze', 'sign'}
    assert {n['tiling'] for n in IR['nodes'] if n['t'] == 'gradient'} == {'clamp_to_edge', 'repeat', 'mirrored_repeat'}
    assert {n['kind'] for n in IR['nodes'] if n['t'] == 'simple'} == {'blend_alpha', 'blend_offset', 'beardifier'}
    assert {d['normalize'] for d in IR['noises'].values()} == {'enabled', 'disabled', 'legacy'}


def test_compile_time_plans_are_exercised():
    M = gen_eval.Model(os.path.join(MODEL, 'overworld_ir.json'), os.path.join(MODEL, 'overworld_terrain.json'))
    kinds = collections.Counter(gen_eval.binary_plan(M, n)[0] for n in M.nodes if n['t'] == 'binary')
    for k in ('add', 'sub', 'mul', 'div', 'divc', 'min', 'max', 'pass'):
        assert kinds[k] > 0, k
    shifted = [n for n in IR['nodes'] if n['t'] == 'noise' and not n['shift_x_zero']]
    assert any(not n['shift_y_zero'] for n in shifted) and any(n['shift_y_zero'] for n in shifted)


def test_every_rule_and_condition_type():
    rules, conds = collections.Counter(), collections.Counter()

    def walk_c(c):
        conds[c['t']] += 1
        if c['t'] in ('not', 'ref'):
            walk_c(c['cond'])

    def walk(r):
        rules[r['t']] += 1
        if r['t'] == 'sequence':
            for x in r['rules']:
                walk(x)
        elif r['t'] == 'condition':
            walk_c(r['if'])
            walk(r['then'])
        elif r['t'] == 'ref':
            walk(r['rule'])
    walk(TM['material_rule'])
    for t in ('block', 'sequence', 'condition', 'bandlands', 'ore_vein', 'ref'):
        assert rules[t] > 0, t
    for t in ('biome', 'noise_threshold', 'vertical_gradient', 'y_above', 'water', 'temperature', 'steep', 'not', 'hole', 'above_preliminary_surface',
              'stone_depth', 'ref'):
        assert conds[t] > 0, t


def test_reference_loaders_accept_the_model(ref_model):
    assert (ref_model.min_y, ref_model.height, ref_model.sea_level) == (-64, 384, 63)


def test_biome_list_shape():
    names = TM['biome_names']
    assert names == sorted(names) and len(names) < 128
    for n in ('minecraft:eroded_badlands', 'minecraft:frozen_ocean', 'minecraft:deep_frozen_ocean'):
        assert n in names
    assert 5000 < len(TM['biome_parameters']) < 10000


def _generate(tmp_path, ir, tm):
    pi, pt = tmp_path / 'ir.json', tmp_path / 'tm.json'
    pi.write_text(json.dumps(ir))
    pt.write_text(json.dumps(tm))
    return gen_eval.generate(str(pi), str(pt), str(tmp_path / 'out.cuh'))


def test_codegen_rejects_air_rule_results(tmp_path):
    tm = copy.deepcopy(TM)
    tm['material_rule']['rules'].insert(0, {'t': 'block', 'state': 0})
    with pytest.raises(SystemExit, match='air or a fluid'):
        _generate(tmp_path, IR, tm)


def test_codegen_requires_one_find_top_surface(tmp_path):
    ir = copy.deepcopy(IR)
    for n in ir['nodes']:
        if n['t'] == 'find_top_surface':
            n['t'] = 'constant'
            n['v'] = 0
    with pytest.raises(SystemExit, match='find_top_surface'):
        _generate(tmp_path, ir, TM)


def test_codegen_is_deterministic(tmp_path):
    a = open(gen_eval.generate(os.path.join(MODEL, 'overworld_ir.json'), os.path.join(MODEL, 'overworld_terrain.json'), str(tmp_path / 'g.cuh'))).read()
    b = open(os.path.join(REPO, 'minecraft-terrain-cuda_b200', '_gen', 'model_gen.cuh')).read()
    assert a == b


def test_guard_algebra():
    T = gen_eval.TRUE
    a = gen_eval.g_and(T, 'g1')
    b = gen_eval.g_and(a, 'g2')
    assert gen_eval.g_or(a, b) == a              # absorption
    assert gen_eval.g_or(a, T) == T
    c = gen_eval.g_and(T, 'g3')
    assert gen_eval.g_or(a, c) == frozenset([frozenset(['g1']), frozenset(['g3'])])


def test_float_literals_are_exact():
    import numpy as np
    for v in [0.1, -1.5e-7, 3.4e38, 1e-45, 0.0, -0.0]:
        f = np.float32(v)
        lit = gen_eval.flit(f)
        assert np.float32(float.fromhex(lit[:-1])) == f


def _live_table():
    """kOreLiveCells as compiled into the library (the generated header)."""
    import re
    text = open(os.path.join(REPO, 'minecraft-terrain-cuda_b200', '_gen', 'model_gen.cuh')).read()
    m = re.search(r'constexpr uint32_t kOreLiveCells\[(\d+)\] = \{([^}]*)\}', text)
    return [int(v.strip().rstrip('u'), 16) for v in m.group(2).split(',')]


def test_ore_live_cells_against_the_port(ref_model):
    """The fill evaluates an ore vein's density only in the cell rows whose bit is set in
    kOreLiveCells. Where a bit is clear the port's density of that vein (ref_point on the
    vein's density root) must be <= 0 at every height of the row, on every sampled column."""
    M = gen_eval.Model(os.path.join(MODEL, 'overworld_ir.json'), os.path.join(MODEL, 'overworld_terrain.json'))
    ores = gen_eval.Gen(M).ores
    live = _live_table()
    assert len(live) == M.height // 8
    assert any(v != (1 << len(ores)) - 1 for v in live), 'no cell row skips a vein in this model'
    rs = ref_model.seed(0x5445525241494E31)
    import numpy as np
    rng = np.random.default_rng(7)
    cols = np.concatenate([rng.integers(-2000, 2000, size=(24, 2)), [[0, 0], [-1000000, 1874999], [6128 * 16, -6129 * 16]]])
    ys = np.arange(M.min_y, M.min_y + M.height)
    xyz = np.array([(x, y, z) for x, z in cols for y in ys], np.int32)
    for k, o in enumerate(ores):
        v = rs.point(M.roots[o['density']], xyz).reshape(len(cols), len(ys))
        for cell in range(M.height // 8):
            if (live[cell] >> k) & 1:
                continue
            block = v[:, 8 * cell:8 * cell + 8]
            assert (block <= 0).all(), 'vein %d density above zero in skipped cell row %d' % (k, cell)
