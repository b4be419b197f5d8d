"""Normal-cone decisions on the rounding boundary.

The meshlet test decides dot(normalize(apex - camera), normalize(N * axis)) >= cutoff
from approximate arithmetic when it is clearly on one side and falls back to the
reference's own sequence (crates/helio-pass-virtual-geometry/shaders/vg_cull.wgsl:172-180)
otherwise. Here every meshlet's cutoff is set a few ulps around the exact value of
that dot product for the view's camera (computed in binary32 with the reference's
operation order), and the single-view pass and the batched launch must keep exactly
the oracle's meshlets."""
import numpy as np
import pytest

from helpers import cull_dtype, gpu_hiz, gpu_vg_view, u32
from oracle import oracle as O

pytestmark = pytest.mark.gpu

OFFSETS = np.array([-3, -2, -1, 0, 1, 2, 3, 40, -40], np.int64)


def _f(x):
    return np.asarray(x, np.float32)


def exact_cone_dot(scene, cam_pos):
    """Per meshlet (with its instance), the reference's binary32 value of
    dot(normalize(apex_ws - cam), normalize(N * axis))."""
    objs, inst, m = scene.objects, scene.instances, scene.meshlets
    owner = np.zeros(len(m), np.int64)
    for o in range(len(objs)):
        for l in range(int(objs["lod_count"][o])):
            f, n = int(objs["lod_first_meshlets"][o][l]), int(objs["lod_meshlet_counts"][o][l])
            owner[f:f + n] = objs["instance_index"][o]
    M = inst["model"].reshape(-1, 4, 4)[owner].astype(np.float32)       # [k][column][row]
    N = inst["normal_mat"].reshape(-1, 3, 4)[owner].astype(np.float32)  # [k][column][row]
    ax, ap = m["cone_axis"].astype(np.float32), m["cone_apex"].astype(np.float32)
    a = [(N[:, 0, r] * ax[:, 0] + N[:, 1, r] * ax[:, 1]) + N[:, 2, r] * ax[:, 2] for r in range(3)]
    la = np.sqrt((a[0] * a[0] + a[1] * a[1]) + a[2] * a[2])
    an = [a[r] / la for r in range(3)]
    apex = [((M[:, 0, r] * ap[:, 0] + M[:, 1, r] * ap[:, 1]) + M[:, 2, r] * ap[:, 2]) + M[:, 3, r] for r in range(3)]
    c = [apex[r] - _f(cam_pos[r]) for r in range(3)]
    lc = np.sqrt((c[0] * c[0] + c[1] * c[1]) + c[2] * c[2])
    cn = [c[r] / lc for r in range(3)]
    return ((cn[0] * an[0] + cn[1] * an[1]) + cn[2] * an[2]).astype(np.float32)


def test_cone_cutoff_on_the_boundary():
    from helio_b200 import scene as S
    from helpers import gather, run_batch

    w = S.config(1, scale=0.05)
    sc, view = w.scene, w.views[0]
    e = exact_cone_dot(sc, np.array(view.camera.position_near[:3], np.float32))
    ok = np.isfinite(e) & (e <= 1.0)
    bits = e.view(np.int32).astype(np.int64)
    k = OFFSETS[np.arange(len(e)) % len(OFFSETS)]
    # Adjacent binary32 values: step the integer image (towards +inf for positive values).
    step = np.where(e >= 0, k, -k)
    cut = np.clip(bits + step, np.iinfo(np.int32).min, np.iinfo(np.int32).max).astype(np.int32).view(np.float32)
    sc.meshlets["cone_cutoff"] = np.where(ok, np.minimum(cut, np.float32(1.0)), sc.meshlets["cone_cutoff"])
    levels = O.hiz_build(view.depth)
    ref = O.run_view(sc, view.camera, view.width, view.height, levels, view.lod_threshold_px, None, 11, 4,
                     cull_dtype())
    assert int(ref["counters"][0]) > 100

    hz, _ = gpu_hiz(view.depth)
    g = gpu_vg_view(sc, view, hz=hz)
    np.testing.assert_array_equal(g["counters"][:11], ref["counters"][:11], err_msg="single view: counters")
    np.testing.assert_array_equal(g["visibility"], ref["visibility"], err_msg="single view: visibility")

    b, _, _ = run_batch(sc, [view])
    got = gather(b, 0, len(sc.objects))
    np.testing.assert_array_equal(got["counters"], ref["counters"], err_msg="batched: counters")
    np.testing.assert_array_equal(got["indirect"], ref["indirect"], err_msg="batched: indirect")
    np.testing.assert_array_equal(got["draws"], ref["draws"], err_msg="batched: draws")
