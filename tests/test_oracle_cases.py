"""The oracle's restatements of the shadow cull (shadow_cull.wgsl) and of the static Hi-Z
branch (occlusion_cull.wgsl:222-259) on hand-built cases whose answers follow from the
shaders' text, on the CPU: these pin the oracle that the GPU parity tests compare with."""
import numpy as np

from oracle import oracle as O


def _instances(spheres):
    from helio_b200 import scene as S

    inst = np.zeros(len(spheres), S.DT_INSTANCE)
    for i, (x, y, z, r) in enumerate(spheres):
        inst[i]["bounds"] = (x, y, z, r)
        inst[i]["model"] = np.eye(4, dtype=np.float32).reshape(16)
    return inst


def _draws(first_instances):
    src = np.zeros((len(first_instances), 5), np.uint32)
    src[:, 0] = 3
    src[:, 1] = 1
    src[:, 2] = np.arange(len(first_instances)) * 3
    src[:, 4] = first_instances
    return src


def _box_face(half: float) -> np.ndarray:
    """Column-major matrix whose column-built planes are the box |x|, |y| <= half,
    0 <= z <= half (vp = scale(1/half, 1/half, 1/half))."""
    m = np.zeros(16, np.float32)
    m[0] = m[5] = m[10] = 1.0 / half
    m[15] = 1.0
    return m


def test_shadow_cull_cases():
    mats = np.zeros((256, 16), np.float32)
    mats[0] = _box_face(10.0)
    mats[5] = _box_face(1.0)
    dirty = np.zeros(256, np.uint32)
    dirty[[0, 5]] = 1
    inst = _instances([
        (0.0, 0.0, 5.0, 1.0),      # 0: inside face 0, outside face 5 (z beyond 1 + r)
        (12.0, 0.0, 5.0, 1.0),     # 1: 1 past face 0's x plane: outside
        (10.5, 0.0, 5.0, 1.0),     # 2: crosses face 0's x plane: visible
        (0.0, 0.0, 5.0, 0.0),      # 3: radius 0: skipped
        (0.0, 0.0, 5.0, -2.0),     # 4: negative radius: skipped
        (0.0, 0.0, 5.0, np.nan),   # 5: NaN radius: passes every plane
        (0.0, 0.0, -0.5, 1.0),     # 6: behind z = 0 by less than r: visible in both faces
    ])
    src = _draws([0, 1, 2, 3, 4, 5, 6, 99])  # draw 7 names an instance past the array
    dst, counts, ran = O.shadow_cull(mats, inst, src, dirty, 2, max_per_face=4)
    assert ran
    assert counts[0] == 4 and counts[5] == 2 and counts.sum() == 6
    np.testing.assert_array_equal(dst[0:4], src[[0, 2, 5, 6]])  # draw order
    np.testing.assert_array_equal(dst[5 * 4:5 * 4 + 2], src[[5, 6]])
    # More visible draws than the face holds: the count goes on, the first 4 are stored.
    src2 = _draws([0, 2, 5, 6, 0, 2])
    dst2, counts2, _ = O.shadow_cull(mats, inst, src2, dirty, 2, max_per_face=4)
    assert counts2[0] == 6
    np.testing.assert_array_equal(dst2[0:4], src2[:4])
    # No face in use: nothing changes, the previous counts stay.
    _, counts3, ran3 = O.shadow_cull(mats, inst, src2, dirty, 0, max_per_face=4, dst=dst2, counts=counts2)
    assert not ran3 and (counts3 == counts2).all()


def _static_case(value: float):
    grid = (3, 2, 2)
    return {"texels": np.full(grid[0] * grid[1] * grid[2] * 6, value, np.float32), "grid": grid,
            "min": (-50.0, -50.0, -50.0), "max": (50.0, 50.0, 50.0)}


def test_static_hiz_constant_grid():
    """A constant grid filters to the constant exactly (weights are multiples of 1/256 and
    100 * k / 256 is exact), so a kept draw is culled iff its distance > 100 + 0.1."""
    from helio_b200 import scene as S

    cam = S.perspective((0.0, 0.0, 0.0), (0.0, 0.0, -1.0), (0.0, 1.0, 0.0), 60.0, 1.0, 0.1, 1000.0)
    inst = _instances([(0.0, 0.0, -50.0, 1.0), (0.0, 0.0, -100.05, 1.0), (0.0, 0.0, -100.2, 1.0),
                       (3.0, 2.0, -140.0, 1.0)])
    from helio_b200 import native as N

    dc = np.zeros(len(inst), np.dtype(N.GpuDrawCall))
    dc["first_instance"] = np.arange(len(inst))
    dc["instance_count"] = 1
    dc["index_count"] = 3
    far = [np.ones((64, 64), np.float32)]  # the dynamic pyramid hides nothing
    levels = O.hiz_build(far[0])
    ind = np.zeros((len(inst), 5), np.uint32)
    ind[:, 1] = 1
    stats = np.zeros(8, np.uint32)
    O.occlusion_cull(cam, 64, 64, levels, inst, dc, ind, stats, static_hiz=_static_case(100.0))
    assert ind[:, 1].tolist() == [1, 1, 0, 0]
    assert stats[4] == 2
    # Without the static grid nothing is culled.
    ind[:, 1] = 1
    stats[:] = 0
    O.occlusion_cull(cam, 64, 64, levels, inst, dc, ind, stats)
    assert ind[:, 1].tolist() == [1, 1, 1, 1] and stats[4] == 0
