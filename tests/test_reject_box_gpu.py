"""The batched select's reject boxes never reject an (object, view) pair that the
exact sphere test keeps.

Object centres are placed around the corners, edges and faces of several views'
frusta, at distances within a few radii of the sphere test's boundary, where the
axis-aligned reject box (the bound of the frustum widened by the largest radius)
is tightest; the selected LOD of every (view, object) must equal the oracle's."""
import numpy as np
import pytest

from helpers import cull_dtype
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def frustum_points(view_proj: np.ndarray) -> np.ndarray:
    """The 8 corners, 12 edge midpoints, 6 face centres (and the centre) of the view
    volume (NDC x, y in [-1, 1], z in [0, 1]) in world space."""
    inv = np.linalg.inv(view_proj.astype(np.float64))
    pts = []
    for x in (-1.0, 0.0, 1.0):
        for y in (-1.0, 0.0, 1.0):
            for z in (0.0, 0.5, 1.0):
                p = inv @ np.array([x, y, z, 1.0])
                pts.append(p[:3] / p[3])
    return np.array(pts)


def boundary_scene(views, seed=7):
    from helio_b200 import scene as S

    w = S.config(1, scale=0.2)  # 2000 instances
    sc = w.scene
    rng = np.random.default_rng(seed)
    n = len(sc.objects)
    model = sc.instances["model"].reshape(n, 4, 4).astype(np.float64)  # model[i][column][row]
    lb = sc.objects["local_bounds"].astype(np.float64)
    scale = np.sqrt((model[:, :3, :3] ** 2).sum(axis=2)).max(axis=1)
    radius = lb[:, 3] * scale
    targets = np.empty((n, 3))
    for i in range(n):
        v = views[i % len(views)]
        vp = np.array(v.camera.view_proj, dtype=np.float64).reshape(4, 4).T  # row-major
        pts = frustum_points(vp)
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        targets[i] = pts[rng.integers(len(pts))] + d * radius[i] * rng.uniform(0.0, 3.0)
    # world centre c = M[:3, :3] lb + t, so t = target - M[:3, :3] lb
    lin = np.einsum("ncr,nc->nr", model[:, :3, :3], lb[:, :3])
    model[:, 3, :3] = targets - lin
    sc.instances["model"] = model.reshape(n, 16).astype(np.float32)
    return sc


def test_reject_box_keeps_every_visible_pair():
    from helio_b200 import scene as S
    from helpers import gather, run_batch

    mv = S.multiview_set(11, depth=True, scale=0.05)
    views = [mv[0], mv[1], mv[5], mv[6], mv[21], mv[30]]  # main, a cascade, two spots, two probes
    sc = boundary_scene(views)
    b, _, _ = run_batch(sc, views)
    kept = 0
    for i, v in enumerate(views):
        got = gather(b, i, len(sc.objects))
        levels = O.hiz_build(v.depth)
        ref = O.run_view(sc, v.camera, v.width, v.height, levels, v.lod_threshold_px, None, 11, 4, cull_dtype())
        np.testing.assert_array_equal(got["lod"], ref["selected"], err_msg=f"view {i}: selected LOD + 1")
        np.testing.assert_array_equal(got["counters"], ref["counters"], err_msg=f"view {i}: counters")
        kept += int((ref["selected"] > 0).sum())
    assert kept > 100, "enough objects straddle the frusta to exercise the boundary"
