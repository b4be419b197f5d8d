"""Batched multi-view cull (one cooperative launch) vs the oracle, view by view:
pyramid levels, selected LOD per object, counters, indirect args and draw metadata in
the canonical (object, span, lane) order, and the per-span visibility words."""
import numpy as np
import pytest

from helpers import benchmark_scene, check_batch as _check_batch, check_view, gather, run_batch, u32

pytestmark = pytest.mark.gpu


def test_batch_85_views_matches_oracle(cuda):
    from helio_b200 import scene as S

    w = S.config(3, scale=0.02)
    assert len(w.views) == 85
    _check_batch(w, w.views)


@pytest.mark.parametrize("cfg,scale,nviews", [(0, 1.0, 1), (1, 0.2, 1), (2, 0.05, 1)])
def test_batch_single_view_equals_plain_pipeline(cuda, cfg, scale, nviews):
    from helio_b200 import scene as S

    w = S.config(cfg, scale=scale)
    _check_batch(w, w.views[:nviews])


def test_batch_mixed_views_alias_and_capacity(cuda):
    """A cfg2-shaped scene seen by the 85-view mix at a small scale, level 0 aliased
    to the depth, and a small per-view capacity that overflows."""
    from helio_b200 import scene as S

    w = S.config(2, scale=0.03)
    views = S.multiview_set(S.SEED_BASE + 2, True, 0.04)[:24]
    b, vs, _ = run_batch(w.scene, views, alias=True, capacities=[50] * len(views))
    for i, v in enumerate(views):
        got = gather(b, i, len(w.scene.objects))
        check_view(w.scene, v, got, None, None, 50)


def test_batch_repeat_and_camera_update(cuda):
    import torch
    from helio_b200 import scene as S

    w = S.config(3, scale=0.02)
    views = w.views[:10]
    b, vs, depths = run_batch(w.scene, views, repeats=3)
    for i, v in enumerate(views):
        check_view(w.scene, v, gather(b, i, len(w.scene.objects)), None, None, gather(b, i, 1)["capacity"])
    # Move every camera and re-run without re-preparing.
    moved = []
    for v in views:
        cam = S.perspective(tuple(np.array(v.camera.position_near[:3]) + 7.0), (0, 0, -300), (0, 1, 0), 70.0,
                            v.width / v.height)
        moved.append(S.View(cam, v.width, v.height, v.depth, v.kind, v.lod_threshold_px))
    b.set_cameras([m.camera for m in moved])
    b.execute()
    torch.cuda.synchronize()
    b.status()
    for i, v in enumerate(moved):
        check_view(w.scene, v, gather(b, i, len(w.scene.objects)), None, None, gather(b, i, 1)["capacity"])


def test_batch_benchmark_scene(cuda):
    """Every meshlet of the constant benchmark scene is emitted (meshlet_cull_benchmark.rs:284-294)."""
    sc, v = benchmark_scene(64, 1024)
    b, vs, _ = run_batch(sc, [v], span_visibility=False, capacities=[64 * 1024])
    got = gather(b, 0, len(sc.objects))
    assert got["counters"][0] == 64 * 1024 and got["counters"][1] == 0
    np.testing.assert_array_equal(got["indirect"][:, 4], np.arange(64 * 1024))


def test_autotune_keeps_results(cuda):
    """The launch-shape autotuner only changes how work is split, never the results."""
    from helio_b200 import scene as S

    w = S.config(3, scale=0.05)
    views = w.views[:24]
    b, vs, _ = run_batch(w.scene, views, span_visibility=False)
    before = [gather(b, i, len(w.scene.objects)) for i in range(len(views))]
    t = b.autotune(repeats=2)
    # 12 first-launch shapes, then at least one CTA per SM of the meshlet-test launch.
    assert t["candidates"] >= 13 and 8 <= t["select_views"] <= 32 and t["ctas"] >= 1 and t["cull_ctas"] >= 1
    assert t["best_ms"] <= t["default_ms"] * 1.5
    after = [gather(b, i, len(w.scene.objects)) for i in range(len(views))]
    for x, y in zip(before, after):
        for k in ("counters", "indirect", "draws", "lod"):
            np.testing.assert_array_equal(x[k], y[k])


def test_pack_draws_matches_per_view_outputs(cuda):
    """helio_batch_pack_draws lays every view's published draws end to end."""
    import torch
    from helio_b200 import scene as S

    w = S.config(3, scale=0.05)
    views = w.views[:16]
    b, vs, _ = run_batch(w.scene, views, span_visibility=False)
    per = [gather(b, i, len(w.scene.objects)) for i in range(len(views))]
    total = sum(len(p["indirect"]) for p in per)
    cap = total + 7
    ind = torch.full((cap, 5), -1, dtype=torch.int32, device="cuda")
    drw = torch.full((cap, 4), -1, dtype=torch.int32, device="cuda")
    off = torch.zeros(len(views) + 1, dtype=torch.int32, device="cuda")
    b.pack_draws(ind, drw, off)
    torch.cuda.synchronize()
    o = off.cpu().numpy()
    assert o[-1] == total
    for i, p in enumerate(per):
        np.testing.assert_array_equal(u32(ind[o[i]:o[i + 1]]), p["indirect"], err_msg=f"view {i} indirect")
        np.testing.assert_array_equal(u32(drw[o[i]:o[i + 1]]), p["draws"], err_msg=f"view {i} draws")
    assert (ind[total:].cpu().numpy() == -1).all()
    # A capacity below the total writes only what fits.
    small = max(1, total // 3)
    ind2 = torch.zeros((small, 5), dtype=torch.int32, device="cuda")
    drw2 = torch.zeros((small, 4), dtype=torch.int32, device="cuda")
    b.pack_draws(ind2, drw2, off)
    torch.cuda.synchronize()
    assert off.cpu().numpy()[-1] == small
    np.testing.assert_array_equal(u32(ind2), np.concatenate([p["indirect"] for p in per])[:small])


@pytest.mark.parametrize("cull_ctas", [1, 19, 100000])
def test_batch_cull_grid_matches_oracle(cuda, cull_ctas):
    """The meshlet-test launch's grid, set apart from the first launch's (one CTA, an
    odd count, more than fit: capped), changes only how the work is split."""
    from helio_b200 import scene as S

    w = S.config(3, scale=0.05)
    views = w.views[:1] + w.views[5:9] + w.views[21:26]
    _check_batch(w, views, cull_ctas=cull_ctas)


@pytest.mark.parametrize("ctas", [1, 7])
def test_batch_small_grid_matches_oracle(cuda, ctas):
    """A grid of a few CTAs gives every warp many units in every phase (multi-round
    span expansion over 32 chunks at a time, many Hi-Z and select units per CTA)."""
    from helio_b200 import scene as S

    w = S.config(3, scale=0.05)
    views = w.views[:1] + w.views[1:5] + w.views[5:9] + w.views[21:30]
    _check_batch(w, views, max_ctas=ctas)

