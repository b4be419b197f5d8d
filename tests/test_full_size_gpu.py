"""Bit-exact parity at the full sizes the benchmark times, against the oracle.

* The 85-view batch over one scene of 200,000 instances x 50 LOD0 meshlets (10M): one
  main view of 3840x2160, 4 orthographic cascades of 2048^2, 16 spot views of 512^2 and
  64 probe views of 128^2, each with its own depth, level 0 aliased to the depth as the
  benchmark runs it. Every view: every pyramid level, the selected LOD of every object,
  the counters, the indirect args and draw records in canonical order, the active spans
  and their visibility words (vg_cull.wgsl:135-405).
* The plain single-view passes over 100,000 instances x 100 LOD0 meshlets (10M) at
  3840x2160 with 20,000 occluders, the same outputs plus the per-work-item bitmask.

The oracle's count of decisions inside the 1e-6 relative margin band is reported
(printed); no GPU / oracle difference is tolerated, marginal or not."""
import numpy as np
import pytest

from helpers import assert_vg_equal, check_batch, gpu_vg_view, oracle_vg_view

pytestmark = pytest.mark.gpu


def test_batched_85_views_10M_full_size_matches_oracle(cuda):
    from helio_b200 import scene as S

    w = S.config(3)
    assert len(w.views) == 85 and w.scene.lod0_total == 10_000_000
    assert (w.views[0].width, w.views[0].height) == (3840, 2160)
    b = check_batch(w, w.views, alias=True)
    st = b._parity_stats
    print(f"85 views: {st['marginal_decisions']} marginal decisions over {st['meshlets_tested']} meshlet tests")


def test_single_view_10M_full_size_matches_oracle(cuda):
    from helio_b200 import scene as S
    from oracle import oracle as O

    w = S.config(2)
    v = w.views[0]
    assert w.scene.lod0_total == 10_000_000 and (v.width, v.height) == (3840, 2160)
    g = gpu_vg_view(w.scene, v)
    levels = O.hiz_build(v.depth)
    for l, ref in enumerate(levels):
        np.testing.assert_array_equal(g["hz"].level(l).cpu().numpy().view(np.uint32), ref.view(np.uint32),
                                      err_msg=f"Hi-Z level {l}")
    o = oracle_vg_view(w.scene, v, levels, v.lod_threshold_px)
    assert_vg_equal(g, o)  # includes counters[1], the draws past the publication budget
    print(f"config 2: {int(o['counters'][0])} visible meshlets ({len(o['indirect'])} published), "
          f"{o['stats'].marginal_decisions} marginal decisions")
