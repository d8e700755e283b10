"""GPU: the live flythrough renderer (tg_viewer_*). The chunks a viewer generates land in its
voxel window exactly as the TERRAIN step's u8 form gives them, its column cells hold each
cell's highest non-air height, and a traced frame equals the CPU restatement of the ray
march (oracle/render_restate.cpp) on the same window and camera: every pixel's first-ray
hit (block, x, y, z) exactly, and the colours within 3 u8 steps per channel (the shading
calls exp / pow / sqrt, whose last bits differ between the GPU and the host library)."""
import numpy as np
import pytest

import terrain_b200

pytestmark = pytest.mark.gpu

SEED = 123456789
W, WIDTH, HEIGHT = 16, 240, 136


@pytest.fixture(scope='module')
def viewer():
    g = terrain_b200.TerrainGenerator(max_batch_chunks=512)
    g.set_seed(SEED)
    v = terrain_b200.TerrainViewer(g, window_chunks=W, width=WIDTH, height=HEIGHT)
    yield g, v
    v.close()
    g.close()


def check_frame(v, cam, frame):
    import render_oracle
    rgb, hits, ms = v.render(cam, frame, hits=True)
    vox, cells, slots, born = v.state()
    c, top, side, caps, ids = v.params(cam)
    ref_rgb, ref_hits = render_oracle.render(vox, cells, slots, born, ids, c, top, side, caps, WIDTH, HEIGHT, frame)
    bad = np.nonzero((hits != ref_hits).any(2))
    assert bad[0].size == 0, 'pixels whose hit differs: %s' % list(zip(bad[0][:5].tolist(), bad[1][:5].tolist()))
    diff = np.abs(rgb.astype(np.int32) - ref_rgb.astype(np.int32))
    assert diff.max() <= 3 and diff.mean() < 0.05, (diff.max(), diff.mean())
    assert ms > 0
    return rgb, hits


def test_window_holds_the_generated_chunks(viewer):
    g, v = viewer
    n, ms = v.update(0, 0, 6, frame=0)
    assert n > 100 and ms > 0
    assert v.update(0, 0, 6, frame=1)[0] == 0                     # nothing left to generate
    vox, cells, slots, born = v.state()
    probe = [(0, 0), (-3, 4), (5, -2), (-6, 0)]
    blocks, _ = g.generate_u8(probe)
    for (cx, cz), b in zip(probe, blocks):
        k = (cz % W) * W + (cx % W)
        assert tuple(slots[k]) == (cx, cz) and born[k] == 0
        wx, wz = (cx % W) * 16, (cz % W) * 16
        assert (vox[:, wz:wz + 16, wx:wx + 16] == b).all(), (cx, cz)
    # cells: 1 + highest non-air height index of each held 4 x 4 column cell
    air = int(v.params(terrain_b200.camera(0.0, 100.0, 0.0))[4][1])
    nonair = vox != air
    top = np.where(nonair.any(0), vox.shape[0] - np.argmax(nonair[::-1], axis=0), 0)      # per column (z, x)
    want = top.reshape(W * 4, 4, W * 4, 4).max(axis=(1, 3))
    held = np.zeros((W, W), bool)
    for k, (sx, sz) in enumerate(slots):
        if sx != np.iinfo(np.int32).min:
            held[k // W, k % W] = True
    mask = np.repeat(np.repeat(held, 4, 0), 4, 1)
    assert (cells[mask] == want[mask]).all()


def test_frames_match_the_cpu_ray_march(viewer):
    g, v = viewer
    v.update(0, 0, 6, frame=0)
    for frame, cam in enumerate([terrain_b200.camera(8.0, 120.0, 8.0, yaw_deg=30.0, pitch_deg=-20.0),
                                 terrain_b200.camera(-20.5, 90.0, 33.25, yaw_deg=200.0, pitch_deg=-8.0, fov_deg=80.0),
                                 terrain_b200.camera(3.0, 40.0, -5.0, yaw_deg=95.0, pitch_deg=-45.0, sun=(0.3, 0.9, 0.1))]):
        rgb, hits = check_frame(v, cam, frame)
        assert (hits[..., 0] >= 0).mean() > 0.3                   # the terrain is in view
        assert rgb.std() > 5


def test_moving_window_replaces_slots(viewer):
    """The camera moves 20 chunks: the new chunks take the slots of those that left the
    window, and a frame there still matches the CPU ray march."""
    g, v = viewer
    v.update(0, 0, 6, frame=0)
    n, _ = v.update(20, -3, 6, cap=50, frame=5)
    assert n == 50                                                  # capped, nearest first
    n2, _ = v.update(20, -3, 6, frame=6)
    assert n2 > 0
    vox, cells, slots, born = v.state()
    k = ((-3) % W) * W + (20 % W)
    assert tuple(slots[k]) == (20, -3) and born[k] == 5
    check_frame(v, terrain_b200.camera(20 * 16 + 8.0, 110.0, -3 * 16 + 8.0, yaw_deg=-60.0, pitch_deg=-25.0), 7)
    with pytest.raises(terrain_b200.TerrainError):
        v.update(0, 0, W // 2, frame=8)                            # radius beyond the window
