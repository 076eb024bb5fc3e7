"""The HDF5 initial-conditions reader (readHDFFile, hdfHandler.cpp:12-136).

With the reference checkout present (SPH_REFERENCE_ROOT), the reader's output
for the reference's own input file must equal, bit for bit, the initial
conditions stored in tests/golden/demo_impact_n40.npz (made from the same
file by tests/golden/make_golden.py); the fixture itself is checked for the
file's shape and contents everywhere."""
from __future__ import annotations

import hashlib
import os

import numpy as np
import pytest

from conftest import golden

FIELDS = ("pos", "vel", "rho", "u", "mass", "pressure", "h", "material")


def _demo_path(O):
    return os.path.join(O.reference_root(), "SPH", "demo_impact_n40.hdf5")


def test_reader_reproduces_the_fixture_from_the_reference_file(pkg, O):
    path = _demo_path(O)
    if not os.path.exists(path):
        pytest.skip("reference checkout not present")
    g = golden("demo_impact_n40.npz")
    with open(path, "rb") as f:
        assert hashlib.sha256(f.read()).digest() == g["file_sha256"].tobytes()
    ic = pkg.hdf5io.read_ic(path)
    for k in FIELDS:
        assert ic[k].dtype == g[f"ic_{k}"].dtype, k
        assert np.array_equal(ic[k], g[f"ic_{k}"]), k
    grp = pkg.hdf5io.read_group(path)
    # coordinates are stored in FP64 and rounded to nearest, as H5Dread to float does
    assert grp["Coordinates"].dtype == np.float64
    assert np.array_equal(grp["Coordinates"].astype(np.float32), ic["pos"])
    # hard links to one object read the same data
    assert np.array_equal(grp["Density"], grp["Densities"])
    assert np.array_equal(grp["SmoothingLength"], grp["SmoothingLengths"])


def test_fixture_holds_the_demo_impact():
    g = golden("demo_impact_n40.npz")
    n = g["ic_pos"].shape[0]
    assert n == 10766 and g["ic_pos"].shape == (n, 3) and g["ic_vel"].shape == (n, 3)
    assert set(np.unique(g["ic_material"]).tolist()) == {400, 402}
    assert (g["ic_h"] > 0).all() and (g["ic_mass"] > 0).all() and (g["ic_rho"] > 0).all()
    # two bodies near (318, 318, 318) Mm, the reference's coordinate origin
    assert 300 < g["ic_pos"].min() and g["ic_pos"].max() < 350


def test_reader_rejects_other_files(pkg, tmp_path):
    p = tmp_path / "not.hdf5"
    p.write_bytes(b"plain text, not HDF5" * 10)
    with pytest.raises(pkg.hdf5io.UnsupportedHDF5):
        pkg.hdf5io.read_ic(str(p))
    q = tmp_path / "sb2.hdf5"
    q.write_bytes(pkg.hdf5io.SIGNATURE + bytes([2]) + bytes(200))
    with pytest.raises(pkg.hdf5io.UnsupportedHDF5, match="superblock version 2"):
        pkg.hdf5io.read_ic(str(q))
