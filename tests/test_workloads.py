"""Seeded synthetic workloads are deterministic and sized as the configs state."""
import numpy as np

import fdg_workloads as W


def test_deterministic():
    a, b = W.ico_cap(3), W.ico_cap(3)
    assert np.array_equal(a.vertices, b.vertices) and np.array_equal(a.faces, b.faces)
    c, d = W.primitives(1, faces_total=20_000), W.primitives(1, faces_total=20_000)
    assert np.array_equal(c.vertices, d.vertices) and np.array_equal(c.faces, d.faces)


def test_sizes_and_types():
    w = W.ico_cap(0)
    assert w.vertices.dtype == np.float32 and w.faces.dtype == np.int64
    assert w.vertices.shape == (2562, 3) and 4800 < w.num_faces < 5120 and w.grid_size == 64
    p = W.primitives(1)
    assert 275_000 <= p.num_faces <= 290_000 and p.grid_size == 512
    assert np.all(p.vertices >= -0.5) and np.all(p.vertices <= 0.5)
    assert p.faces.min() >= 0 and p.faces.max() < p.vertices.shape[0]
