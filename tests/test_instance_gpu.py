"""IndirectDispatchPass / OcclusionCullPass (and their fused launch): CUDA vs oracle,
exact indirect words and statistics."""
import numpy as np
import pytest

from helpers import gpu_hiz, u32
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _scene(cfg=0, scale=1.0, edge_cases=True):
    from helio_b200 import scene as S

    w = S.config(cfg, scale=scale)
    sc = w.scene
    inst, aabbs, draws = sc.instances.copy(), sc.aabbs.copy(), sc.draw_calls.copy()
    if edge_cases:
        rng = np.random.default_rng(11)
        n = len(draws)
        # degenerate AABBs fall back to the sphere test
        k = rng.choice(n, n // 16, replace=False)
        aabbs["max"][k] = aabbs["min"][k]
        # non-positive radii are skipped by the occlusion pass
        k = rng.choice(n, n // 32, replace=False)
        inst["bounds"][k, 3] = 0.0
        # batched draws: representative instance elsewhere, several instances
        perm = rng.permutation(n)
        draws["first_instance"] = perm.astype(np.uint32)
        draws["instance_count"] = rng.integers(0, 4, n).astype(np.uint32)
    return w, inst, aabbs, draws


def _gpu_instance(w, inst, aabbs, draws, levels_gpu=None, hz=None, mode="separate", frame=1, static_hiz=None):
    import torch
    from helio_b200 import passes as P

    view = w.views[0]
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.uint8)).cuda()
    cam = dev(P.camera_bytes(view.camera))
    ti, ta, td = dev(inst), dev(aabbs), dev(draws)
    indirect = torch.zeros(len(draws) * 5, dtype=torch.int32, device="cuda")
    stats = torch.zeros(8, dtype=torch.int32, device="cuda")
    sb = P.scene_buffers(cam, ti, td, ta, indirect)
    sb.instance_count = len(inst)
    sb.draw_count = len(draws)
    fr = P.IndirectDispatchPass(stats)
    oc = P.OcclusionCullPass(view.width, view.height, stats)
    fr.prepare(view.camera, len(draws))
    oc.prepare(len(draws))
    if static_hiz is not None:
        oc.set_static_hiz(torch.from_numpy(static_hiz["texels"]).cuda(), static_hiz["grid"], static_hiz["min"],
                          static_hiz["max"])
    if mode == "separate":
        fr.execute(sb)
        oc.execute(sb, hz.publish(), frame)
    elif mode == "fused":
        P.fused_instance_cull(fr, oc, sb, hz.publish(), frame)
    elif mode == "frustum":
        fr.execute(sb)
    torch.cuda.synchronize()
    return u32(indirect).reshape(-1, 5), u32(stats)


@pytest.mark.parametrize("mode", ["frustum", "separate", "fused"])
def test_instance_cull_matches_oracle(cuda, mode):
    w, inst, aabbs, draws = _scene()
    view = w.views[0]
    hz, levels = gpu_hiz(view.depth)
    g_ind, g_st = _gpu_instance(w, inst, aabbs, draws, hz=hz, mode=mode)
    o_ind, o_st = O.indirect_dispatch(view.camera, inst, draws, aabbs)
    if mode != "frustum":
        O.occlusion_cull(view.camera, view.width, view.height, O.hiz_build(view.depth), inst, draws, o_ind, o_st)
    np.testing.assert_array_equal(g_ind, o_ind)
    np.testing.assert_array_equal(g_st, o_st)
    assert o_st[0] == len(draws)
    if mode != "frustum":
        assert o_st[4] > 0, "workload should exercise the occlusion test"


def test_occlusion_frame_zero_is_skipped(cuda):
    w, inst, aabbs, draws = _scene(edge_cases=False)
    hz, _ = gpu_hiz(w.views[0].depth)
    g_sep, s_sep = _gpu_instance(w, inst, aabbs, draws, hz=hz, mode="separate", frame=0)
    g_fr, s_fr = _gpu_instance(w, inst, aabbs, draws, hz=hz, mode="frustum")
    np.testing.assert_array_equal(g_sep, g_fr)
    np.testing.assert_array_equal(s_sep, s_fr)
    assert s_sep[4] == 0


def test_instance_cull_larger_scene(cuda):
    w, inst, aabbs, draws = _scene(cfg=1, scale=1.0)
    view = w.views[0]
    hz, _ = gpu_hiz(view.depth)
    g_ind, g_st = _gpu_instance(w, inst, aabbs, draws, hz=hz, mode="fused")
    o_ind, o_st = O.indirect_dispatch(view.camera, inst, draws, aabbs)
    O.occlusion_cull(view.camera, view.width, view.height, O.hiz_build(view.depth), inst, draws, o_ind, o_st)
    np.testing.assert_array_equal(g_ind, o_ind)
    np.testing.assert_array_equal(g_st, o_st)


def static_grid(seed, grid=(12, 10, 8), lo=(-100.0, -100.0, -100.0), hi=(100.0, 100.0, 100.0), far=400.0):
    """A baked static Hi-Z: per voxel and direction layer, the distance past which an
    object counts as hidden (uniform in [0, far])."""
    rng = np.random.default_rng(seed)
    tex = rng.uniform(0.0, far, grid[0] * grid[1] * grid[2] * 6).astype(np.float32)
    return {"texels": tex, "grid": grid, "min": lo, "max": hi}


@pytest.mark.parametrize("mode", ["separate", "fused"])
def test_static_hiz_matches_oracle(cuda, mode):
    """occlusion_cull.wgsl:222-259: the static test after the dynamic one keeps a draw."""
    w, inst, aabbs, draws = _scene()
    view = w.views[0]
    hz, _ = gpu_hiz(view.depth)
    sh = static_grid(5, far=150.0)
    g_ind, g_st = _gpu_instance(w, inst, aabbs, draws, hz=hz, mode=mode, static_hiz=sh)
    levels = O.hiz_build(view.depth)
    o_ind, o_st = O.indirect_dispatch(view.camera, inst, draws, aabbs)
    O.occlusion_cull(view.camera, view.width, view.height, levels, inst, draws, o_ind, o_st, static_hiz=sh)
    np.testing.assert_array_equal(g_ind, o_ind)
    np.testing.assert_array_equal(g_st, o_st)
    d_ind, d_st = O.indirect_dispatch(view.camera, inst, draws, aabbs)
    O.occlusion_cull(view.camera, view.width, view.height, levels, inst, draws, d_ind, d_st)
    assert o_st[4] > d_st[4], "the static grid should hide draws the dynamic pyramid keeps"


def test_static_hiz_edge_cases_and_switch_off(cuda):
    """A flat world box (division by zero: clamped), a one-voxel grid, then the branch off."""
    w, inst, aabbs, draws = _scene()
    view = w.views[0]
    hz, _ = gpu_hiz(view.depth)
    levels = O.hiz_build(view.depth)
    for sh in (static_grid(6, grid=(5, 7, 3), lo=(-100.0, 0.0, -100.0), hi=(100.0, 0.0, 100.0)),
               static_grid(7, grid=(1, 1, 1), far=150.0)):
        g_ind, g_st = _gpu_instance(w, inst, aabbs, draws, hz=hz, mode="fused", static_hiz=sh)
        o_ind, o_st = O.indirect_dispatch(view.camera, inst, draws, aabbs)
        O.occlusion_cull(view.camera, view.width, view.height, levels, inst, draws, o_ind, o_st, static_hiz=sh)
        np.testing.assert_array_equal(g_ind, o_ind)
        np.testing.assert_array_equal(g_st, o_st)
    import torch
    from helio_b200 import passes as P

    st = torch.zeros(8, dtype=torch.int32, device="cuda")
    oc = P.OcclusionCullPass(view.width, view.height, st)
    oc.set_static_hiz(torch.from_numpy(static_grid(8)["texels"]).cuda(), (12, 10, 8), (-100.0,) * 3, (100.0,) * 3)
    oc.set_static_hiz(None)
    g_ind, g_st = _gpu_instance(w, inst, aabbs, draws, hz=hz, mode="separate")
    o_ind, o_st = O.indirect_dispatch(view.camera, inst, draws, aabbs)
    O.occlusion_cull(view.camera, view.width, view.height, levels, inst, draws, o_ind, o_st)
    np.testing.assert_array_equal(g_ind, o_ind)
