"""The 32-bit contribution order keys of the accumulation (fdg_kernels.cu:
the key spaces above `expand`) sort exactly like the reference CPU's
accumulation order, restated as (stage, index) pairs: scanline events in
(triangle, axis, 1-dy, 1-dx) order, then faces in triangle order, then
boundary edges in list order (flexible_dual_grid.cpp:173-283, :298-414,
:741-757).  With F triangles: events (3t + axis) * 4 + (1-dy) * 2 + (1-dx)
in [0, 12F), faces 12F + t, boundary edges 13F + e with e < 3F, so every key
is below 16F, which fits 32 bits for F up to 2^28 - 1 (the library's limit).
"""
import numpy as np
import pytest

MAX_TRIANGLES = (1 << 28) - 1


def key32(stage, idx, F):
    if stage == 0:
        return idx
    if stage == 1:
        return 12 * F + idx
    return 13 * F + idx


def event_index(t, axis, dx, dy):
    return (3 * t + axis) * 4 + (1 - dy) * 2 + (1 - dx)


@pytest.mark.parametrize("F", [1, 7, 1000, 2_000_003, MAX_TRIANGLES])
def test_keys_sort_like_stage_then_index(F):
    rng = np.random.default_rng(F % 1000)
    items = []
    for _ in range(3000):
        stage = int(rng.integers(0, 3))
        if stage == 0:
            idx = event_index(int(rng.integers(0, F)), int(rng.integers(0, 3)), int(rng.integers(0, 2)), int(rng.integers(0, 2)))
        elif stage == 1:
            idx = int(rng.integers(0, F))
        else:
            idx = int(rng.integers(0, 3 * F))
        items.append((stage, idx))
    # the extremes of every key space
    items += [(0, 0), (0, 12 * F - 1), (1, 0), (1, F - 1), (2, 0), (2, 3 * F - 1)]
    items = sorted(set(items))
    keys = [key32(s, i, F) for s, i in items]
    assert keys == sorted(keys)                     # same order as (stage, index)
    assert len(set(keys)) == len(keys)              # unique
    assert max(keys) < (1 << 32) and max(keys) < 16 * F


def test_event_index_is_the_reference_order():
    """Within one triangle: axis first, then (1-dy), then (1-dx)."""
    order = sorted(((a, 1 - dy, 1 - dx), event_index(5, a, dx, dy)) for a in range(3) for dx in (0, 1) for dy in (0, 1))
    idx = [k for _, k in order]
    assert idx == sorted(idx) and idx[0] == event_index(5, 0, 1, 1) and idx[-1] == event_index(5, 2, 0, 0)
    assert event_index(5, 2, 0, 0) < event_index(6, 0, 1, 1)


def test_limit_is_the_largest_that_fits():
    assert 16 * MAX_TRIANGLES < (1 << 32) <= 16 * (MAX_TRIANGLES + 1)
