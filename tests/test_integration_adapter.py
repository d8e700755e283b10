"""The drop-in C++ adapter include/terrain_b200_adapter.hpp (the reference's
FullTerrainGenerator over the C ABI) compiles against include/terrain_b200.h, and both
generate overloads -- the reference's u8 palette-index form and the u16 form -- resolve.
No GPU, no link."""
import os
import shutil
import subprocess

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(shutil.which('g++') is None, reason='needs g++')
def test_adapter_compiles_and_keeps_the_reference_signature(tmp_path):
    src = open(os.path.join(REPO, 'include', 'terrain_b200_adapter.hpp')).read()
    assert 'tg_generate_u8' in src
    use = '''
#include "terrain_b200_adapter.hpp"
void use(mcc::cuda::FullTerrainGenerator& g, const mcc::cuda::ChunkXZ* c, uint8_t* t8, uint8_t* b8, uint16_t* t16) {
    g.generate(c, 1, t8, b8, nullptr);            // terrain_gpu.h:43
    g.generate(c, 1, t8, b8, t8, nullptr);
    g.generate(c, 1, t16);                        // u16 overload
    mcc::cuda::TerrainTiming t;
    g.generate(c, 1, t8, nullptr, nullptr, &t);
}
'''
    f = tmp_path / 'adapter_check.cpp'
    f.write_text(use)
    r = subprocess.run(['g++', '-std=c++17', '-fsyntax-only', '-Wall', '-I', os.path.join(REPO, 'include'), str(f)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
