"""The serving loop's batch rule (helio_serve_plan_batch), on the host: the oldest
pending request always leads; later requests join only if they name the same scene
and the batch stays within max_views (and max_requests); arrival order is kept."""
import pytest

from helio_b200 import native as N
from helio_b200.passes import plan_batch


def test_oldest_leads_and_same_scene_joins_in_order(native_built):
    q = [(0, 5), (1, 3), (0, 100), (0, 7), (2, 1), (0, 120)]
    assert plan_batch(q, 128) == [0, 2, 3]  # 5 + 100 + 7 = 112 views; 120 more would not fit


def test_other_scenes_wait_for_their_own_batch(native_built):
    q = [(3, 10), (1, 1), (3, 10), (1, 1)]
    assert plan_batch(q, 128) == [0, 2]
    assert plan_batch(q[1:], 128) == [0, 2]


def test_later_smaller_request_fills_the_gap(native_built):
    q = [(0, 60), (0, 70), (0, 68), (0, 1)]
    assert plan_batch(q, 128) == [0, 2]  # 60 + 68 = 128 exactly; the 1-view request no longer fits


def test_request_limit(native_built):
    q = [(0, 1)] * 10
    assert plan_batch(q, 128, max_requests=4) == [0, 1, 2, 3]
    assert plan_batch(q, 3) == [0, 1, 2]


def test_empty_queue_and_invalid_head(native_built):
    assert plan_batch([], 128) == []
    with pytest.raises(N.HelioError):
        plan_batch([(0, 129)], 128)
    with pytest.raises(N.HelioError):
        plan_batch([(0, 0)], 128)


def test_device_occupancy_is_the_union_of_batch_intervals():
    """The serving bench line's `device` figures: overlapping batches (two slots) count once,
    gaps count as idle, and requests of one batch (same interval) count once."""
    import sys
    from pathlib import Path

    sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
    from bench import device_occupancy

    comps = [{"status": 0, "device_start_ms": 0.0, "device_end_ms": 2.0},
             {"status": 0, "device_start_ms": 1.0, "device_end_ms": 3.0},  # overlaps the first
             {"status": 0, "device_start_ms": 5.0, "device_end_ms": 6.0},
             {"status": 0, "device_start_ms": 5.0, "device_end_ms": 6.0},  # same batch
             {"status": 7, "device_start_ms": 6.0, "device_end_ms": 9.0}]  # failed: not counted
    d = device_occupancy(comps)
    assert d["batches"] == 3
    assert d["span_ms"] == 6.0
    assert abs(d["busy_fraction"] - 4.0 / 6.0) < 1e-12
    assert abs(d["batch_device_ms_mean"] - 5.0 / 3.0) < 1e-12
    assert device_occupancy([{"status": 7, "device_start_ms": 0.0, "device_end_ms": 1.0}]) is None
