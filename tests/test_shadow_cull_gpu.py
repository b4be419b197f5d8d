"""Per-face shadow cull (helio_shadow_cull_*: ShadowCullPass, shadow_cull.wgsl) against
the oracle's restatement: every dirty face's visible draws in draw order, the counts of
all 256 faces, records of clean faces kept from earlier frames, more than 4096 visible
draws on a face, the pass's early return, and skipped draws (r <= 0, instance index
past the array; a NaN radius passes every plane, as in the reference)."""
import numpy as np
import pytest

from helpers import u32
from oracle import oracle as O


def shadow_faces(seed):
    from helio_b200 import scene as S

    return S.shadow_faces(seed)


def shadow_scene(seed, instances, draws, spread=200.0):
    from helio_b200 import scene as S

    return S.shadow_draws(seed, instances, draws, spread)

pytestmark = pytest.mark.gpu


class Gpu:
    def __init__(self):
        from helio_b200.passes import ShadowCullPass

        self.p = ShadowCullPass()

    def run(self, mats, inst, src, dirty, face_count):
        import torch

        def dev(a, dt=None):
            return torch.from_numpy(np.ascontiguousarray(a if dt is None else a.astype(dt))).cuda()

        self.p.prepare(dev(mats), dev(inst.view(np.uint8)), dev(src.view(np.int32)), dev(dirty.view(np.int32)),
                       face_count)
        self.p.execute()
        torch.cuda.synchronize()
        o = self.p.outputs()
        return u32(o["face_indirect"]), u32(o["face_counts"])


def check_frame(dst, counts, ref_dst, ref_counts, faces):
    np.testing.assert_array_equal(counts, ref_counts, err_msg="face counts")
    for f in faces:
        n = min(int(ref_counts[f]), 4096)
        np.testing.assert_array_equal(dst[f * 4096:f * 4096 + n], ref_dst[f * 4096:f * 4096 + n],
                                      err_msg=f"face {f}")


@pytest.mark.parametrize("seed,draws", [(1, 3000), (2, 20000)])
def test_shadow_cull_matches_oracle(cuda, seed, draws):
    mats, nf = shadow_faces(seed)
    inst, src = shadow_scene(seed, 5000, draws)
    rng = np.random.default_rng(seed + 100)
    dirty = np.zeros(256, np.uint32)
    dirty[:nf] = rng.random(nf) < 0.8
    dirty[0] = 1
    g = Gpu()
    dst, counts = g.run(mats, inst, src, dirty, nf)
    ref_dst, ref_counts, ran = O.shadow_cull(mats, inst, src, dirty, nf)
    assert ran and ref_counts[np.nonzero(dirty)[0]].sum() > 0
    check_frame(dst, counts, ref_dst, ref_counts, np.nonzero(dirty)[0])


def test_clean_faces_keep_their_records_and_full_faces_count_on(cuda):
    mats, nf = shadow_faces(3)
    # The widest cascade sees everything: more than 4096 visible draws on face 3.
    inst, src = shadow_scene(3, 8000, 30000, spread=150.0)
    g = Gpu()
    a = np.zeros(256, np.uint32)
    a[:nf] = 1
    dst, counts = g.run(mats, inst, src, a, nf)
    ref_dst, ref_counts, _ = O.shadow_cull(mats, inst, src, a, nf)
    assert ref_counts[3] > 4096
    check_frame(dst, counts, ref_dst, ref_counts, range(nf))
    # Frame 2: other draws, only the even faces dirty; the odd faces keep frame 1's records.
    inst2, src2 = shadow_scene(4, 8000, 9000, spread=150.0)
    b = np.zeros(256, np.uint32)
    b[:nf:2] = 7
    dst2, counts2 = g.run(mats, inst2, src2, b, nf)
    ref_dst2, ref_counts2, _ = O.shadow_cull(mats, inst2, src2, b, nf, dst=ref_dst, counts=ref_counts)
    check_frame(dst2, counts2, ref_dst2, ref_counts2, range(nf))
    assert (counts2[1:nf:2] == 0).all()  # clean faces' counts are cleared, their records kept
    for f in range(1, nf, 2):
        n = min(int(ref_counts[f]), 4096)
        np.testing.assert_array_equal(dst2[f * 4096:f * 4096 + n], dst[f * 4096:f * 4096 + n])
    # Frame 3: no faces in use: nothing runs and the counts stay as they were.
    dst3, counts3 = g.run(mats, inst2, src2, b, 0)
    np.testing.assert_array_equal(counts3, counts2)
    _, ref_counts3, ran = O.shadow_cull(mats, inst2, src2, b, 0, dst=ref_dst2, counts=ref_counts2)
    assert not ran
    np.testing.assert_array_equal(counts3, ref_counts3)


@pytest.mark.parametrize("max_ctas", [0, 37])
def test_shadow_cull_folded_into_a_batch(cuda, max_ctas):
    """helio_batch_attach_shadow: the pass's stages run as units of the batch's phases.
    Two frames (the second with other draws and only the even faces dirty): the pass's
    outputs equal the oracle's and the standalone pass's, the batch's own outputs equal
    those of the same batch without the pass, and detaching restores the plain batch.
    With 37 CTAs every CTA scans several faces and places several blocks."""
    import torch
    from helio_b200 import scene as S
    from helio_b200.passes import BatchedCull, ShadowCullPass, VgScene

    def dev(a):
        return torch.from_numpy(np.ascontiguousarray(a)).cuda()

    w = S.config(3, scale=0.03)
    views = w.views[:6]
    vs = VgScene()
    vs.upload(S.frame_data(w.scene))
    depths = [dev(v.depth) for v in views]
    specs = [{"camera": v.camera, "depth": d, "alias_mip0": True, "lod_threshold_px": v.lod_threshold_px}
             for v, d in zip(views, depths)]

    def batch_outputs(b):
        out = []
        for i in range(len(views)):
            o = b.view_outputs(i)
            c = u32(o["counters"])
            n = int(min(c[0], o["capacity"]))
            out.append((c, u32(o["indirect"])[:n], u32(o["draws"])[:n]))
        return out

    plain = BatchedCull(len(views), max_ctas=max_ctas)
    plain.prepare(vs, specs)
    plain.execute()
    torch.cuda.synchronize()
    want = batch_outputs(plain)

    mats, nf = shadow_faces(5)
    frames = [(shadow_scene(5, 6000, 20000, spread=150.0), np.arange(256) < nf),
              (shadow_scene(6, 6000, 9000, spread=150.0), (np.arange(256) < nf) & (np.arange(256) % 2 == 0))]
    folded, alone = ShadowCullPass(), Gpu()
    b = BatchedCull(len(views), max_ctas=max_ctas)
    b.prepare(vs, specs)
    b.attach_shadow(folded)
    ref_dst = ref_counts = None
    for (inst, src), dirty_b in frames:
        dirty = dirty_b.astype(np.uint32)
        keep = (dev(mats), dev(inst.view(np.uint8)), dev(src.view(np.int32)), dev(dirty.view(np.int32)))
        folded.prepare(*keep, nf)
        b.execute()
        torch.cuda.synchronize()
        b.status()
        o = folded.outputs()
        dst, counts = u32(o["face_indirect"]), u32(o["face_counts"])
        ref_dst, ref_counts, ran = O.shadow_cull(mats, inst, src, dirty, nf, dst=ref_dst, counts=ref_counts)
        assert ran and ref_counts[:nf].sum() > 0
        check_frame(dst, counts, ref_dst, ref_counts, range(nf))
        a_dst, a_counts = alone.run(mats, inst, src, dirty, nf)
        np.testing.assert_array_equal(counts, a_counts)
        for f in range(nf):
            n = min(int(counts[f]), 4096)
            np.testing.assert_array_equal(dst[f * 4096:f * 4096 + n], a_dst[f * 4096:f * 4096 + n])
        for (c, ind, dr), (wc, wind, wdr) in zip(batch_outputs(b), want):
            np.testing.assert_array_equal(c, wc)
            np.testing.assert_array_equal(ind, wind)
            np.testing.assert_array_equal(dr, wdr)
    # No face in use: the attached pass does nothing (its counts stay as they were).
    inst, src = frames[1][0]
    folded.prepare(dev(mats), dev(inst.view(np.uint8)), dev(src.view(np.int32)),
                   dev(np.ones(256, np.uint32).view(np.int32)), 0)
    before = u32(folded.outputs()["face_counts"]).copy()
    b.execute()
    torch.cuda.synchronize()
    np.testing.assert_array_equal(u32(folded.outputs()["face_counts"]), before)
    b.attach_shadow(None)
    b.execute()
    torch.cuda.synchronize()
    np.testing.assert_array_equal(u32(folded.outputs()["face_counts"]), before)
    for (c, ind, dr), (wc, wind, wdr) in zip(batch_outputs(b), want):
        np.testing.assert_array_equal(c, wc)
        np.testing.assert_array_equal(ind, wind)
        np.testing.assert_array_equal(dr, wdr)
