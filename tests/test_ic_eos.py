"""Host-side input generators: the seeded impact initial conditions and the
stand-in EOS tables in the reference's ANEOS text format."""
from __future__ import annotations

import math

import numpy as np


def test_impact_ic_counts_masses_and_layers(pkg):
    ic = pkg.ic.make_impact(16384, 4096, seed=0)
    assert ic["n"] == 20480
    assert ic["pos"].shape == (20480, 3) and ic["pos"].dtype == np.float32
    t, b = slice(0, 16384), slice(16384, None)
    assert math.isclose(float(ic["mass"][t].sum()), 5.97, rel_tol=1e-5)
    assert math.isclose(float(ic["mass"][b].sum()), 0.13 * 5.97, rel_tol=1e-5)
    # equal-mass particles within each body, 30% of them in the iron core
    assert np.allclose(ic["mass"][t], ic["mass"][t][0])
    core = ic["material"][t] == 402
    assert abs(core.mean() - 0.3) < 1e-3
    assert np.all(ic["u"][t][core] == np.float32(1.5e-6)) and np.all(ic["u"][t][~core] == np.float32(1e-6))
    # the core sits inside the mantle
    c = ic["pos"][t].astype(np.float64).mean(axis=0)
    r = np.linalg.norm(ic["pos"][t] - c, axis=1)
    assert r[core].max() < np.percentile(r[~core], 5) + 0.5


def test_impact_ic_is_seeded_and_in_com_frame(pkg):
    a = pkg.ic.make_impact(2048, 512, seed=4)
    b = pkg.ic.make_impact(2048, 512, seed=4)
    c = pkg.ic.make_impact(2048, 512, seed=5)
    assert np.array_equal(a["pos"], b["pos"]) and not np.array_equal(a["pos"], c["pos"])
    p = (a["mass"][:, None].astype(np.float64) * a["vel"]).sum(axis=0)
    assert np.abs(p).max() < 1e-9
    # straight-line approach along -x in the relative frame
    vrel = a["vel"][2048].astype(np.float64) - a["vel"][0]
    assert vrel[0] < 0 and abs(vrel[1]) < 1e-12


def test_stand_in_tables_follow_reference_layout(pkg, tmp_path):
    path = pkg.eos_tables.write_table(str(tmp_path / "t.txt"), "forsterite", n_rho=8, n_t=6)
    lines = open(path).read().splitlines()
    assert lines[13].split() == ["8", "6"]          # ANEOS.cpp:36-40 (line 14)
    rho = [float(x) for x in " ".join(lines[14:16]).split()]
    assert len(rho) == 8
    rows = lines[14 + 2 + 2:]
    assert len(rows) == 8 * 6
    assert all(len(r.split()) == 4 for r in rows)


def test_stand_in_energy_is_monotone_for_the_resampler(pkg):
    """u must be non-decreasing in density at fixed T and strictly increasing
    in T (float32): the reference's resampler walks both directions."""
    for mat in ("forsterite", "Fe85Si15"):
        rho, temp, u, p, c, s = pkg.eos_tables.table_values(mat)
        u32 = u.astype(np.float32)
        assert np.all(np.diff(u32, axis=1) > 0), mat
        assert np.all(np.diff(u32, axis=0) >= 0), mat
        assert np.all(p >= 0) and np.all(c > 0)


def test_resampled_tables_are_finite(O, eos_grids):
    for g in eos_grids:
        assert np.all(np.isfinite(g))
        assert np.all(g[..., 1] > 0)
