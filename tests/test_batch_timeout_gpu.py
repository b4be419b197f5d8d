"""Failure detection of the batched launch without a GPU fault: every device wait of
the batch is bounded. A batch whose grid barriers wait for CTAs that never arrive (a
count nothing reaches) gives up after a short poll limit, ends its CTAs, and the host
reads HELIO_ERR_TIMEOUT; the context stays usable and the next execute is bit-exact
against the oracle."""
import time

import numpy as np
import pytest

from helpers import check_view, gather, run_batch

pytestmark = pytest.mark.gpu


def test_barrier_timeout_is_reported_and_the_next_batch_is_exact(cuda):
    import torch
    from helio_b200 import native as N
    from helio_b200 import scene as S

    w = S.config(3, scale=0.02)
    views = w.views[:12]
    b, vs, depths = run_batch(w.scene, views)
    lib = N.cull_lib()

    # ~4k polls of 64..256 ns: each CTA gives up after about a millisecond.
    b.set_wait_limit(4096, 1)
    t0 = time.perf_counter()
    b.execute()
    torch.cuda.synchronize()
    elapsed = time.perf_counter() - t0
    assert lib.helio_batch_status(b._h, None) == N.HELIO_ERR_TIMEOUT
    assert b"timed out" in lib.helio_last_error()
    assert elapsed < 10.0, elapsed

    # The same context, normal limits: exact again (the cleared region is reset per execute).
    b.set_wait_limit(0, 0)
    b.execute()
    torch.cuda.synchronize()
    b.status()
    for i, v in enumerate(views):
        got = gather(b, i, len(w.scene.objects))
        check_view(w.scene, v, got, None, None, got["capacity"])


def test_short_wait_limit_alone_changes_nothing(cuda):
    """A short but sufficient limit with every CTA arriving: no timeout, same results."""
    import torch
    from helio_b200 import scene as S

    w = S.config(3, scale=0.02)
    views = w.views[:6]
    b, vs, depths = run_batch(w.scene, views)
    ref = [gather(b, i, len(w.scene.objects)) for i in range(len(views))]
    b.set_wait_limit(1 << 20, 0)
    b.execute()
    torch.cuda.synchronize()
    b.status()
    for i in range(len(views)):
        got = gather(b, i, len(w.scene.objects))
        for k in ("counters", "indirect", "draws", "lod"):
            np.testing.assert_array_equal(got[k], ref[i][k])
