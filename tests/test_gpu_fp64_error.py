"""Error of each form against an all-FP64 run of the same seed (oracle/fp64.cpp:
FP64 direct-sum gravity and the reference's SPH passes in double), after 40
steps of a 8192 + 2048 impact:

  plain   the reference's logic (its FMM, float positions);
  theta   opening-angle gravity (theta 0.6), float positions;
  mixed   opening-angle gravity + FP64 master positions and time + Kahan sums.

Every GPU run takes the FP64 run's timestep each step (its CFL tick count is
set before the step pass), so all runs integrate over the same steps.
Positions are compared in units of the mean smoothing length, velocities
relative to their rms, u, rho and h relative to each value; the forms with
the opening-angle gravity must sit closer to the FP64 run than the plain
form."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

STEPS = 40


def _errors(c, ref, mixed: bool) -> dict:
    pos = c.download("pos64") if mixed else c.download("pos").astype(np.float64)
    out = {}
    hbar = float(np.mean(ref.field("h")))
    dx = np.linalg.norm(pos - ref.field("pos"), axis=1) / hbar
    out["pos/h"] = dx
    v = c.download("vel").astype(np.float64)
    vr = ref.field("vel")
    out["vel"] = np.linalg.norm(v - vr, axis=1) / np.sqrt(np.mean(np.sum(vr * vr, axis=1)))
    for f in ("u", "rho", "h"):
        g = c.download(f).astype(np.float64)
        r = ref.field(f)
        out[f] = np.abs(g - r) / np.abs(r)
    return out


def test_forms_against_an_all_fp64_run(cuda, pkg, O, eos_grids):
    ic = pkg.ic.make_impact(8192, 2048, seed=2)
    ref = O.F64Run(ic, *eos_grids)
    forms = (("plain", None), ("theta", dict(gravity="theta", theta=0.6)),
             ("mixed", dict(gravity="theta", theta=0.6, precision="mixed")))
    ctxs = {}
    for name, form in forms:
        c = pkg.Compute(ic, max_children_in_leaf=32, max_tree_depth=7)
        if form:
            c.set_form(**form)
        ctxs[name] = c
    try:
        # every run takes the FP64 run's step: its CFL tick count is set after
        # the acceleration pass, so all runs integrate over the same steps
        for _ in range(STEPS):
            ref.steps(1)
            dt = np.array([int(ref.dt[0])], np.int32)
            for c in ctxs.values():
                c.updateOctreeBuffer()
                c.sort()
                c.gravitationalPass()
                c.densityPass()
                c.accelerationPass()
                c.upload("dt", dt)
                c.stepPass()
        e_ref = ref.energy()["total"]
        rows = {}
        for name, c in ctxs.items():
            c.synchronize()
            assert int(c.download("global_time")[0]) == int(ref.gt[0])
            err = _errors(c, ref, name == "mixed")
            rows[name] = {k: (float(np.median(v)), float(np.percentile(v, 99))) for k, v in err.items()}
            rows[name]["energy"] = abs(c.diagnostics()["total"] - e_ref) / abs(e_ref)
    finally:
        for c in ctxs.values():
            c.close()
    print(f"\n  after {STEPS} steps ({ref.t[0]:.0f} s), median / p99 against the all-FP64 run:")
    for name, r in rows.items():
        cols = "  ".join(f"{k} {m:.2e}/{p:.2e}" for k, (m, p) in ((k, r[k]) for k in ("pos/h", "vel", "u", "rho", "h")))
        print(f"  {name:6s} {cols}  |dE|/|E| {r['energy']:.2e}")
    # the opening-angle forms follow the FP64 run more closely than the
    # reference's gravity does, in positions and velocities
    for k in ("pos/h", "vel"):
        assert rows["mixed"][k][0] < rows["plain"][k][0], (k, rows)
        assert rows["theta"][k][0] < rows["plain"][k][0], (k, rows)
    # and stay close to it: sub-percent of a smoothing length, 1e-2 of the rms velocity
    assert rows["mixed"]["pos/h"][1] < 1e-2 and rows["mixed"]["vel"][1] < 1e-2, rows["mixed"]
    assert rows["mixed"]["rho"][1] < 1e-2 and rows["mixed"]["u"][1] < 1e-2, rows["mixed"]
