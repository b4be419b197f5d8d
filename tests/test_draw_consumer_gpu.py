"""The draw side of the VG pass's outputs, as the reference's render pass consumes them
(crates/helio-pass-virtual-geometry/src/rendering.rs:1194-1208; the benchmark's draw,
crates/examples/meshlet_cull_benchmark.rs:770-777): multi_draw_indexed_indirect_count
reads the draw count from byte 0 of the counter buffer and draws
min(count, max_draw_count) 20-byte DrawIndexedIndirect records; a device without the
count feature draws all max_draw_count records of an indirect buffer cleared every
frame (rendering.rs:1127-1130), here HELIO_VG_CLEAR_INDIRECT. Both consumers are
emulated on the host and must execute exactly the oracle's visible meshlets."""
import numpy as np
import pytest

from helpers import gpu_vg_view, oracle_vg_view, u32

pytestmark = pytest.mark.gpu


def count_form(out: dict) -> np.ndarray:
    """multi_draw_indexed_indirect_count(indirect, 0, counters, 0, max_draw_count = capacity)."""
    raw = out["pass"].outputs()["counters"].cpu().numpy().view(np.uint8)
    count = int.from_bytes(raw[0:4].tobytes(), "little")  # the count buffer's byte 0
    assert count == int(out["counters"][0])
    n = min(count, out["pass"].publish().capacity)
    return u32(out["pass"].outputs()["indirect"])[:n]


def plain_form(out: dict) -> np.ndarray:
    """multi_draw_indexed_indirect(indirect, 0, max_draw_count = capacity): every record;
    the ones with no instances or no indices draw nothing."""
    rec = u32(out["pass"].outputs()["indirect"])
    return rec[(rec[:, 1] > 0) & (rec[:, 0] > 0)]


def expected_commands(scene, ref: dict) -> np.ndarray:
    """DrawIndexedIndirect of each oracle draw (vg_cull.wgsl:241-254): the meshlet's
    index_count, one instance, its first_index and vertex_offset, first_instance = slot."""
    m = scene.meshlets[ref["draws"][:, 1]]
    n = len(ref["draws"])
    return np.stack([m["index_count"], np.ones(n, np.uint32), m["first_index"],
                     m["vertex_offset"].view(np.uint32), np.arange(n, dtype=np.uint32)], axis=1)


def _cascade_views(w):
    """The orthographic cascades of the 85-view set: one size, nested coverage."""
    return [v for v in w.views if (v.width, v.height) == (w.views[1].width, w.views[1].height)][:4]


def test_count_form_draws_the_visible_meshlets(cuda):
    from helio_b200 import scene as S
    from oracle import oracle as O

    w = S.config(1, scale=0.25)
    v = w.views[0]
    g = gpu_vg_view(w.scene, v)
    ref = oracle_vg_view(w.scene, v, O.hiz_build(v.depth))
    got = count_form(g)
    assert len(got) == int(ref["counters"][0]) > 0
    np.testing.assert_array_equal(got, expected_commands(w.scene, ref))
    np.testing.assert_array_equal(u32(g["pass"].outputs()["draws"])[:len(got)], ref["draws"])


def test_count_form_clamps_an_overflowing_count(cuda):
    from helio_b200 import scene as S
    from oracle import oracle as O

    w = S.config(0, scale=1.0)
    v = w.views[0]
    cap = 777
    g = gpu_vg_view(w.scene, v, publication_limit=cap)
    ref = oracle_vg_view(w.scene, v, O.hiz_build(v.depth), capacity=cap)
    assert int(g["counters"][0]) > cap  # the count at byte 0 counts every visible meshlet
    got = count_form(g)
    assert len(got) == cap
    np.testing.assert_array_equal(got, expected_commands(w.scene, ref))


def test_cleared_buffer_serves_a_consumer_without_the_count(cuda):
    """Two frames on one pass, the second with fewer visible meshlets: with the clear,
    drawing every record executes exactly the second frame's draws; without it, records
    of the first frame stay behind the count."""
    from helio_b200 import scene as S
    from helio_b200.passes import VirtualGeometryPass
    from oracle import oracle as O

    w = S.config(3, scale=0.02)
    views = _cascade_views(w)
    refs = [oracle_vg_view(w.scene, v, O.hiz_build(v.depth)) for v in views]
    counts = [int(r["counters"][0]) for r in refs]
    a, b = int(np.argmax(counts)), int(np.argmin(counts))
    assert counts[a] > counts[b]
    frame = S.frame_data(w.scene)
    for clear in (True, False):
        vg = VirtualGeometryPass(views[a].width, views[a].height, clear_indirect=clear)
        gpu_vg_view(w.scene, views[a], vg_pass=vg, frame=frame)
        g = gpu_vg_view(w.scene, views[b], vg_pass=vg, frame=frame)
        want = expected_commands(w.scene, refs[b])
        np.testing.assert_array_equal(count_form(g), want)
        if clear:
            np.testing.assert_array_equal(plain_form(g), want)
            rest = u32(vg.outputs()["indirect"])[len(want):]
            assert not rest.any()
        else:
            assert len(plain_form(g)) > len(want)  # stale records: this consumer needs the flag
