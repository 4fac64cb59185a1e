"""The work-shape table lookup of the o_voxel wrapper (o_voxel/convert/_tuning.py)."""
import json

from o_voxel.convert import _tuning as T


def test_values_by_grid_bucket(tmp_path, monkeypatch):
    table = {"buckets": [
        {"max_grid": 128, "tuning": {"unit_cells": 32, "warp_scan_cells": 128, "inline_face_bricks": 4,
                                     "dense_candidates": 16, "long_walk": 32}},
        {"max_grid": 512, "tuning": {"unit_cells": 128, "warp_scan_cells": 512, "inline_face_bricks": 16,
                                     "dense_candidates": 64, "long_walk": 128}},
    ]}
    p = tmp_path / "tuning.json"
    p.write_text(json.dumps(table))
    monkeypatch.setattr(T, "PATH", str(p))
    monkeypatch.setattr(T, "_TABLE", None)
    assert T.values_for(64) == (32, 128, 4, 16, 32)
    assert T.values_for(128) == (32, 128, 4, 16, 32)
    assert T.values_for(300) == (128, 512, 16, 64, 128)
    assert T.values_for(2048) == (128, 512, 16, 64, 128)  # beyond the last bucket: the last bucket's shapes
    calls = []

    class Ext:
        def set_tuning_cuda(self, device, values):
            calls.append((device, tuple(values)))

    monkeypatch.setattr(T, "_APPLIED", {})
    T.apply(Ext(), 0, 64)
    T.apply(Ext(), 0, 100)  # same bucket: not set again
    T.apply(Ext(), 0, 512)
    assert calls == [(0, (32, 128, 4, 16, 32)), (0, (128, 512, 16, 64, 128))]


def test_no_table_means_defaults(tmp_path, monkeypatch):
    monkeypatch.setattr(T, "PATH", str(tmp_path / "missing.json"))
    monkeypatch.setattr(T, "_TABLE", None)
    assert T.values_for(512) == ()
