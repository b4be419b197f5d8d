"""helio_hiz_build_noalloc: the Hi-Z build for callers that cannot allocate device
memory (its scratch lives in a fixed device array inside the library). Called through
the C-ABI and checked bit for bit against HiZBuildPass (the allocating entry point),
on two calls in a row that reuse the shared array. This file is collected last."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SIZES = [(1920, 1080, 0), (1031, 517, 0), (64, 64, 0), (300, 1, 0), (513, 257, 1)]
# 32 views, the most one call takes: small probe-like views, a third of them read
# from depth rows longer than the view (pitch > width), some with level 0 aliased.
SIZES_32 = [(128 + 9 * i, 64 + 5 * i, i % 4 == 3, 7 * (i % 3)) for i in range(32)]


def _views(seed, sizes=SIZES):
    """(depth view, width, height, alias) per size; a size with a fourth entry k > 0
    reads its depth from rows of width + k floats."""
    import torch

    rng = np.random.default_rng(seed)
    out = []
    for size in sizes:
        w, h, alias = size[:3]
        extra = size[3] if len(size) > 3 else 0
        full = torch.from_numpy(rng.random((h, w + extra), dtype=np.float32)).cuda()
        out.append((full[:, :w], w, h, alias))
    return out


def _reference_levels(depth, w, h, alias):
    from helio_b200.passes import HiZBuildPass

    hz = HiZBuildPass(w, h, alias_mip0=bool(alias))
    hz.prepare(depth)
    hz.execute()
    return [hz.level(l).cpu().numpy().copy() for l in range(hz.publish().mip_count)]


def _noalloc(views, levels_floats=None):
    import torch
    from helio_b200 import native as N
    from helio_b200.passes import device_view

    lib = N.cull_lib()
    n = len(views)
    inp = (N.HizViewInput * n)(*[N.HizViewInput(d.data_ptr(), w, h, d.stride(0), N.HELIO_HIZ_ALIAS_MIP0 if a else 0)
                                 for d, w, h, a in views])
    need = 0
    for _, w, h, a in views:
        need = (need + 3) & ~3
        m = min(max(w, h).bit_length(), 12)
        for l in range(0 if not a else 1, m):
            lw, lh = max(w >> l, 1), max(h >> l, 1)
            need += ((lw + 3) & ~3) * lh
    buf = torch.full((levels_floats or need,), -1.0, dtype=torch.float32, device="cuda")
    pyr = (N.HizPyramid * n)()
    st = lib.helio_hiz_build_noalloc(n, inp, C.c_void_p(buf.data_ptr()), buf.numel(), pyr,
                                     C.c_void_p(torch.cuda.current_stream().cuda_stream))
    if st != N.HELIO_OK:
        return st, lib.helio_last_error(), None
    torch.cuda.synchronize()
    out = []
    for v in range(n):
        p = pyr[v]
        out.append([device_view(p.levels[l], (p.height[l], p.width[l]), "<f4", (p.pitch[l] * 4, 4)).cpu().numpy()
                    for l in range(p.mip_count)])
    return st, b"", out


def test_noalloc_matches_allocating_pass_on_two_calls(cuda):
    for call, seed in enumerate((1, 2)):  # the second call reuses the shared scratch array
        views = _views(seed)
        st, msg, got = _noalloc(views)
        assert st == 0, msg
        for (d, w, h, a), levels in zip(views, got):
            ref = _reference_levels(d, w, h, a)
            assert len(levels) == len(ref)
            for l, (x, y) in enumerate(zip(levels, ref)):
                np.testing.assert_array_equal(x.view(np.uint32), y.view(np.uint32),
                                              err_msg=f"call {call} view {w}x{h} level {l}")


def test_noalloc_32_views_with_pitched_depth_matches_allocating_pass(cuda):
    """The whole fixed array in use (32 views, the largest job search), with depth rows
    longer than the views, on two calls in a row."""
    for call, seed in enumerate((5, 6)):
        views = _views(seed, SIZES_32)
        st, msg, got = _noalloc(views)
        assert st == 0, msg
        for (d, w, h, a), levels in zip(views, got):
            ref = _reference_levels(d, w, h, a)
            assert len(levels) == len(ref)
            for l, (x, y) in enumerate(zip(levels, ref)):
                np.testing.assert_array_equal(x.view(np.uint32), y.view(np.uint32),
                                              err_msg=f"call {call} view {w}x{h} pitch {d.stride(0)} level {l}")


def test_noalloc_rejects_sizes_beyond_its_limits(cuda):
    from helio_b200 import native as N

    views = _views(3)[:1] * 33
    st, msg, _ = _noalloc(views)
    assert st == N.HELIO_ERR_INVALID_ARG and b"32 views" in msg
    st, msg, _ = _noalloc(_views(4)[:1], levels_floats=16)
    assert st == N.HELIO_ERR_INVALID_ARG and b"too small" in msg
