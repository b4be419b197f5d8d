"""LOD selection on the rounding boundary of the pixel-error threshold.

The select kernels decide `RN(err * max_scale * focal / closest) <= threshold`
from an approximate quotient when it is clearly on one side and fall back to the
correctly rounded division otherwise (the reference computes the division at
crates/helio-pass-virtual-geometry/shaders/vg_cull.wgsl:329-331).
Here every visible object's level-1 error is placed a few ulps around the exact
value at which the oracle's choice flips, and around the edges of the fast path's
margin; the single-view pass and the batched launch must pick the oracle's level
for each one."""
import numpy as np
import pytest

from helpers import cull_dtype, gpu_hiz, gpu_vg_view, u32
from oracle import oracle as O

pytestmark = pytest.mark.gpu

# ulp offsets from the last error that still keeps level 1: around the flip point
# and around the fast path's margin (|threshold| * 2^-18, i.e. 16 ulps of 2.0).
OFFSETS = np.array([-40, -17, -16, -15, -3, -2, -1, 0, 1, 2, 3, 4, 15, 16, 17, 40], np.int64)


def _selected(scene, view, levels):
    return O.run_view(scene, view.camera, view.width, view.height, levels, view.lod_threshold_px, None, 11, 4,
                      cull_dtype())["selected"]


def boundary_workload():
    from helio_b200 import scene as S

    w = S.config(1, scale=0.05)
    scene, view = w.scene, w.views[0]
    objs = scene.objects
    assert (objs["lod_count"] >= 2).all()
    objs["lod_errors"][:, 2:] = np.inf  # only the level-1 decision matters
    levels = O.hiz_build(view.depth)
    # Bisection over the bit patterns of positive floats, all objects at once:
    # lo keeps level 1 (selected == 2), hi does not.
    n = len(objs)
    lo = np.zeros(n, np.int64)
    hi = np.full(n, 0x7F800000, np.int64)
    visible = _selected(scene, view, levels) > 0
    while (hi - lo > 1).any():
        mid = (lo + hi) // 2
        objs["lod_errors"][:, 1] = mid.astype(np.uint32).view(np.float32)
        keep = _selected(scene, view, levels) == 2
        lo = np.where(keep, mid, lo)
        hi = np.where(keep, hi, mid)
    bits = lo + OFFSETS[np.arange(n) % len(OFFSETS)]
    objs["lod_errors"][:, 1] = np.clip(bits, 0, 0x7F7FFFFF).astype(np.uint32).view(np.float32)
    ref = _selected(scene, view, levels)
    return w, levels, ref, visible


def test_threshold_boundary_single_view_and_batched():
    from helpers import gather, run_batch

    w, levels, ref, visible = boundary_workload()
    scene, view = w.scene, w.views[0]
    assert visible.sum() >= 32, "the view must see enough objects to matter"
    vis_sel = ref[visible]
    assert (vis_sel == 1).any() and (vis_sel == 2).any(), "both sides of the threshold are exercised"

    hz, _ = gpu_hiz(view.depth)
    g = gpu_vg_view(scene, view, hz=hz)
    np.testing.assert_array_equal(g["selected"], ref, err_msg="single-view pass: selected LOD + 1")

    b, _, _ = run_batch(scene, [view, view])
    for v in range(2):
        got = gather(b, v, len(scene.objects))
        np.testing.assert_array_equal(got["lod"], ref, err_msg=f"batched view {v}: selected LOD + 1")
    np.testing.assert_array_equal(u32(b.view_outputs(0)["counters"]), u32(b.view_outputs(1)["counters"]))
