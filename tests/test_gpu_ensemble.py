"""Batched ensemble on the GPU: instances stepped together through one graph
launch per step match the same impacts stepped alone, bit for bit, and the
tuner's choices are valid and meet their accuracy bound."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELDS = ("pos", "vel", "acc", "rho", "u", "h", "pressure", "sound_speed", "du", "dhdt", "balsara",
          "next_active_time", "global_time", "dt")


def _ics(pkg, count, seed, n_min, n_max):
    specs = pkg.ensemble.make_specs(count, seed=seed, n_min=n_min, n_max=n_max)
    return specs, [pkg.ensemble.make_ic(s) for s in specs]


def test_ensemble_matches_instances_stepped_alone(cuda, pkg):
    specs, ics = _ics(pkg, 3, 4, 3000, 12000)
    forms = [None, {"gravity": "theta", "theta": 0.6}, {"gravity": "theta", "theta": 0.6, "precision": "mixed"}]
    steps = 3
    with pkg.Ensemble(ics, forms, max_children_in_leaf=32, max_tree_depth=7) as ens:
        assert len(ens) == 3 and ens.sizes == [s["n"] for s in specs]
        ens.step(steps)
        ens.synchronize()
        got = [{k: c.download(k) for k in FIELDS} for c in ens.instances]
        assert all(c.health() == 0 for c in ens.instances)
    for ic, form, g in zip(ics, forms, got):
        with pkg.Compute(ic, max_children_in_leaf=32, max_tree_depth=7) as c:
            if form:
                c.set_form(**form)
            c.step_all(steps)
            c.synchronize()
            for k in FIELDS:
                want = c.download(k)
                assert np.array_equal(g[k], want), f"{k} differs from the instance stepped alone"
        assert int(g["global_time"][0]) > 0


def test_ensemble_autotune_choices(cuda, pkg):
    specs, ics = _ics(pkg, 3, 6, 20000, 40000)
    forms = [{"gravity": "theta", "theta": 0.6}, {"gravity": "theta", "theta": 0.6}, None]
    with pkg.Ensemble(ics, forms, autotune=True, max_children_in_leaf=16, max_tree_depth=7) as ens:
        tun = ens.tuning()
        for t, f in zip(tun, forms):
            assert t["tile_block_max"] in (128, 320, 640)
            assert t["ms_per_step"] > 0.0
            if f:  # theta gravity: leaf capacity tuned under the accuracy bound
                assert t["max_children_in_leaf"] in (16, 32, 64)
                assert 0.0 <= t["gravity_median_error"] <= 1e-3
            else:  # the reference's gravity keeps the requested capacity
                assert t["max_children_in_leaf"] == 16
                assert t["gravity_median_error"] == -1.0
        ens.step(2)
        ens.synchronize()
        for c in ens.instances:
            assert np.isfinite(c.download("pos")).all()
            assert c.health() == 0
