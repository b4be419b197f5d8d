"""InstanceCullData::from_instance on the GPU (helio_instance_cull_data, the kernel the
scene upload runs) against the oracle, field for field as raw bytes, on the reference's
own known-answer matrices (crates/helio-pass-virtual-geometry/src/lib.rs:315-372) and on
random, reflected, sheared, non-uniformly scaled, singular, tiny, non-finite and
non-affine matrices (lib.rs:132-167 decides each of those cases)."""
import ctypes as C
import json
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

KATS = json.loads((Path(__file__).parent / "golden" / "reference_kats.json").read_text())


def _quat_matrix(q):
    w, x, y, z = q / np.linalg.norm(q)
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)],
                     [2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)],
                     [2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)]])


def _matrices(rng, n):
    """n column-major 4x4 models covering every branch of from_instance."""
    out = []
    for i in range(n):
        kind = i % 10
        r = _quat_matrix(rng.normal(size=4))
        s = rng.uniform(0.5, 4.0)
        m = np.eye(4)
        if kind == 0:    # rotation + uniform scale (cone culling enabled)
            m[:3, :3] = r * s
        elif kind == 1:  # reflection (det < 0: cone culling off)
            m[:3, :3] = r * s @ np.diag([1.0, 1.0, -1.0])
        elif kind == 2:  # non-uniform scale
            m[:3, :3] = r @ np.diag(rng.uniform(0.2, 5.0, 3))
        elif kind == 3:  # shear (not orthogonal)
            sh = np.eye(3)
            sh[0, 1] = rng.uniform(-0.5, 0.5)
            m[:3, :3] = r @ sh * s
        elif kind == 4:  # nearly uniform: scale differences around the 1e-4 relative limit
            m[:3, :3] = r @ np.diag(s * (1.0 + rng.choice([-1.0, 1.0], 3) * rng.uniform(0.5e-4, 2e-4, 3)))
        elif kind == 5:  # singular / tiny columns
            m[:3, :3] = r * s
            m[:3, rng.integers(0, 3)] *= rng.choice([0.0, 1e-9, 1e-7])
        elif kind == 6:  # non-finite entries
            m[:3, :3] = r * s
            m[rng.integers(0, 4), rng.integers(0, 4)] = rng.choice([np.nan, np.inf, -np.inf])
        elif kind == 7:  # affine row perturbed around its 1e-6 / 1e-4 tolerances
            m[:3, :3] = r * s
            m[3, rng.integers(0, 4)] += rng.choice([1e-7, 5e-6, 5e-5, 2e-4]) * rng.choice([-1.0, 1.0])
        elif kind == 8:  # arbitrary floats
            m = rng.normal(size=(4, 4)) * 10 ** rng.uniform(-3, 3)
        else:            # translation only, large offsets
            m[:3, :3] = r
        m[:3, 3] = rng.uniform(-1e3, 1e3, 3)
        out.append(m.T.astype(np.float32).reshape(16))  # column-major
    return out


def _gpu_cull_data(inst):
    import torch
    from helio_b200 import native as N

    dt = np.dtype(N.InstanceCullData)
    src = torch.from_numpy(inst.view(np.uint8).copy()).cuda()
    dst = torch.zeros(len(inst) * dt.itemsize, dtype=torch.uint8, device="cuda")
    st = N.cull_lib().helio_instance_cull_data(C.c_void_p(src.data_ptr()), len(inst), C.c_void_p(dst.data_ptr()),
                                               C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == N.HELIO_OK
    torch.cuda.synchronize()
    return dst.cpu().numpy().view(dt)


def _check(models):
    from helio_b200 import native as N

    inst = np.zeros(len(models), np.dtype(N.GpuInstanceData))
    for i, m in enumerate(models):
        inst["model"][i] = m
    got = _gpu_cull_data(inst)
    ref = O.instance_cull_data(inst, np.dtype(N.InstanceCullData))
    bad = np.nonzero(got.view(np.uint32).reshape(len(models), -1) != ref.view(np.uint32).reshape(len(models), -1))[0]
    assert len(bad) == 0, f"{len(bad)} instances differ, first {bad[:5]}: {got[bad[:2]]} vs {ref[bad[:2]]}"
    return ref


def test_reference_known_answer_matrices(cuda):
    models = [np.array([float(x) for x in k["model"]], np.float32) for k in KATS["instance_cull"]]
    ref = _check(models)
    for k, r in zip(KATS["instance_cull"], ref):  # the oracle itself against the KATs
        if "valid" in k:
            assert r["valid_transform"] == k["valid"]
        if "cone" in k:
            assert r["cone_cull_enabled"] == k["cone"]


def test_random_and_degenerate_matrices(cuda):
    rng = np.random.default_rng(20261204)
    ref = _check(_matrices(rng, 20_000))
    # every branch was exercised
    assert ref["valid_transform"].min() == 0 and ref["valid_transform"].max() == 1
    assert ref["cone_cull_enabled"].min() == 0 and ref["cone_cull_enabled"].max() == 1
