"""Snapshot PNGs as Compute::drawSnapshot writes them (Compute.cpp:413-446):
the colour map, a PNG that an independent decoder reads back to the same
pixels, and the every-1000-s schedule with its file names."""
from __future__ import annotations

import numpy as np
import pytest


def test_colour_map(pkg):
    img = np.zeros((1024, 1024), np.int32)
    img[0, 0], img[0, 1], img[5, 7] = 402, 400, 401
    rgba = pkg.snapshot.colourise(img)
    assert tuple(rgba[0, 0]) == (160, 160, 160, 255)
    assert tuple(rgba[0, 1]) == (255, 100, 0, 255)
    assert tuple(rgba[5, 7]) == (255, 255, 255, 255)
    assert tuple(rgba[100, 100]) == (255, 255, 255, 255)


def test_png_decodes_to_the_same_pixels(pkg, tmp_path):
    Image = pytest.importorskip("PIL.Image")
    rng = np.random.default_rng(0)
    img = rng.choice(np.array([0, 400, 401, 402], np.int32), size=(1024, 1024))
    path = pkg.snapshot.write_png(str(tmp_path / "s.png"), img)
    with Image.open(path) as im:
        assert im.size == (1024, 1024) and im.mode == "RGBA"
        got = np.asarray(im)
    assert np.array_equal(got, pkg.snapshot.colourise(img))


def test_schedule_and_names(pkg, tmp_path):
    class Fake:
        def __init__(self):
            self.ticks = 0

        def download(self, field):
            assert field == "global_time"
            return np.array([self.ticks], np.int32)

        def drawSnapshot(self, stream=None):
            return np.zeros((1024, 1024), np.int32)

    w = pkg.snapshot.SnapshotWriter(str(tmp_path))
    c = Fake()
    assert w(c) is None                     # t = 0 is not past 0
    c.ticks = 1                             # 2^-11 s
    assert w(c).endswith("snapshot_0.png")
    c.ticks = 2048 * 999                    # 999 s
    assert w(c) is None
    c.ticks = 2048 * 1000 + 1               # just past 1000 s
    assert w(c).endswith("snapshot_1.png")
    assert sorted(p.name for p in tmp_path.iterdir()) == ["snapshot_0.png", "snapshot_1.png"]
