"""Individual timesteps (SPH_TIMESTEP_INDIVIDUAL, README.md:60-64): on an
impact whose impactor is 100x hotter than the target (so sound speeds, and
with them the CFL timesteps, differ), every step must
  * make active every particle that is due (next active time reached),
  * leave inactive particles' acceleration, du/dt, dh/dt and next active time
    untouched (they are only integrated),
  * give active particles a next active time after the current time,
  * advance the global time without passing any particle's next active time,
and the run must do less work than the global-timestep form's
every-particle-every-step (the reference's test as shipped, Q1)."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _hot_impact(pkg):
    ic = pkg.ic.make_impact(16384, 4096, seed=5)
    u = np.asarray(ic["u"], np.float32).copy()
    u[16384:] *= 100.0  # the impactor's particles come last
    ic = dict(ic, u=u)
    return ic


@pytest.mark.parametrize("gravity", ["reference", "theta"])
def test_individual_timesteps(cuda, pkg, gravity):
    ic = _hot_impact(pkg)
    n = ic["pos"].shape[0]
    active_total = 0
    steps = 16
    with pkg.Compute(ic, max_children_in_leaf=32, max_tree_depth=7) as c:
        c.set_form(gravity=gravity, theta=0.6, timestep="individual")
        assert c.get_form()["timestep"] == "individual"
        for s in range(steps):
            gt0 = int(c.download("global_time")[0])
            nat0 = c.download("next_active_time")
            acc0, du0, dh0 = c.download("acc"), c.download("du"), c.download("dhdt")
            c.step()
            c.synchronize()
            assert c.health() == 0
            act = c.download("active").astype(bool)
            nat1 = c.download("next_active_time")
            gt1 = int(c.download("global_time")[0])
            dt = int(c.download("dt")[0])
            assert act[nat0 <= gt0].all(), f"step {s}: a due particle stayed inactive"
            ina = ~act
            assert np.array_equal(nat1[ina], nat0[ina]), f"step {s}: an inactive particle's next time moved"
            assert np.array_equal(c.download("acc")[ina], acc0[ina])
            assert np.array_equal(c.download("du")[ina], du0[ina])
            assert np.array_equal(c.download("dhdt")[ina], dh0[ina])
            assert (nat1[act] > gt0).all()
            assert dt > 0 and gt1 == gt0 + dt
            assert gt1 <= nat1.min(), f"step {s}: the global time passed a next active time"
            assert np.isfinite(c.download("pos")).all()
            active_total += int(act.sum())
    frac = active_total / (steps * n)
    print(f"\n  {gravity}: mean active fraction {frac:.3f} over {steps} steps")
    assert frac < 0.9  # the hot impactor sets the step; most of the target sits out some steps
