"""Hi-Z pyramid: CUDA (one fused launch) vs the oracle's per-level restatement of
hiz_depth_copy.wgsl + hiz_build.wgsl, bit for bit, on every level."""
import numpy as np
import pytest

from helpers import gpu_hiz
from oracle import oracle as O

pytestmark = pytest.mark.gpu

SIZES = [(1, 1), (2, 1), (1, 2), (3, 3), (5, 3), (17, 13), (63, 65), (64, 64), (65, 64), (130, 70), (257, 1),
         (1, 300), (200, 3), (1000, 999), (1024, 1024), (1920, 1080), (2048, 2048), (3840, 2160)]


def _levels_equal(a, b):
    assert len(a) == len(b), (len(a), len(b))
    for l, (x, y) in enumerate(zip(a, b)):
        assert x.shape == y.shape, (l, x.shape, y.shape)
        np.testing.assert_array_equal(x.view(np.uint32), y.view(np.uint32), err_msg=f"level {l}")


@pytest.mark.parametrize("w,h", SIZES)
def test_hiz_matches_oracle(cuda, w, h):
    rng = np.random.default_rng(w * 7919 + h)
    depth = rng.random((h, w), dtype=np.float32)
    _, g = gpu_hiz(depth)
    _levels_equal(g, O.hiz_build(depth))


@pytest.mark.parametrize("w,h", [(37, 19), (1921, 1081), (4096, 4096)])
def test_hiz_alias_and_pitch(cuda, w, h):
    rng = np.random.default_rng(w + h)
    depth = rng.random((h, w), dtype=np.float32)
    ref = O.hiz_build(depth)
    _, g = gpu_hiz(depth, alias=True)
    _levels_equal(g, ref)
    _, g2 = gpu_hiz(depth, pitch=w + 3)  # unaligned pitch -> scalar path
    _levels_equal(g2, ref)
    assert len(ref) == min(O.mip_levels(w, h), 12)


@pytest.mark.parametrize("w,h", [(64, 64), (1000, 999), (1920, 1080), (3840, 2160), (256, 4096), (8192, 8),
                                 (4, 1), (4, 4096), (68, 3), (32768, 2), (4100, 130)])
def test_hiz_tma_and_plain_loads_agree(cuda, w, h):
    """The TMA tile-load path (persistent grid, several tiles in flight per CTA) and the
    128-bit-load path give the oracle's pyramid, with and without the level-0 copy."""
    rng = np.random.default_rng(w * 31 + h)
    depth = rng.random((h, w), dtype=np.float32)
    ref = O.hiz_build(depth)
    for alias in (False, True):
        for tma in (True, False):
            hz, g = gpu_hiz(depth, alias=alias, tma=tma)
            _levels_equal(g, ref)


def test_hiz_tma_repeated_launches_and_pitch(cuda):
    """Many TMA launches over a depth with a longer (16-byte multiple) row pitch: the
    ticket resets itself and rows past the width are never read into the pyramid."""
    import torch
    from helio_b200.passes import HiZBuildPass

    rng = np.random.default_rng(4)
    depth = rng.random((517, 1030), dtype=np.float32)
    buf = torch.full((517, 1036), 5.0, dtype=torch.float32, device="cuda")
    buf[:, :1030] = torch.from_numpy(depth).cuda()
    hz = HiZBuildPass(1030, 517)
    hz.prepare(buf[:, :1030])
    for _ in range(20):
        hz.execute()
    torch.cuda.synchronize()
    hz.device_status()
    got = [hz.level(l).cpu().numpy() for l in range(hz.publish().mip_count)]
    _levels_equal(got, O.hiz_build(depth))


def test_hiz_workload_depth(cuda):
    from helio_b200 import scene as S

    v = S.config(0).views[0]
    _, g = gpu_hiz(v.depth)
    _levels_equal(g, O.hiz_build(v.depth))


def test_hiz_camera_generation_reuse(cuda):
    """Unchanged camera generation reuses the previous pyramid (reference lib.rs:472-478)."""
    import torch
    from helio_b200.passes import HiZBuildPass

    d = torch.rand(64, 96, device="cuda")
    hz = HiZBuildPass(96, 64)
    hz.prepare(d, camera_generation=5)
    hz.execute()
    first = hz.level(3).cpu().clone()
    d.mul_(0.5)
    hz.prepare(d, camera_generation=5)
    hz.execute()
    assert torch.equal(hz.level(3).cpu(), first)
    hz.prepare(d, camera_generation=6)
    hz.execute()
    assert not torch.equal(hz.level(3).cpu(), first)


def test_hiz_repeated_launches_stable(cuda):
    """The per-view tail ticket resets itself: many launches give identical pyramids."""
    import torch
    from helio_b200.passes import HiZBuildPass

    rng = np.random.default_rng(3)
    depth = rng.random((517, 1031), dtype=np.float32)
    d = torch.from_numpy(depth).cuda()
    hz = HiZBuildPass(1031, 517)
    hz.prepare(d)
    for _ in range(20):
        hz.execute()
    torch.cuda.synchronize()
    got = [hz.level(l).cpu().numpy() for l in range(hz.publish().mip_count)]
    _levels_equal(got, O.hiz_build(depth))
