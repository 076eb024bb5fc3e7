"""The mixed-precision form and the FP64 conservation diagnostics.

The reference keeps positions in float and drifts them in float
(step.metal:45): at ~318 Mm from the origin one ulp is 3e-5 Mm, a few percent
of a step's displacement.  The mixed-precision form keeps FP64 master
positions and global time, float working copies, and Kahan-compensated
acceleration sums.  sph_diagnostics sums mass, energies, momentum and angular
momentum in FP64; the reference has no such reduction (and no potential).
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def host_sums(c):
    m = c.download("mass").astype(np.float64)
    v = c.download("vel").astype(np.float64)
    x = c.download("pos").astype(np.float64)
    u = c.download("u").astype(np.float64)
    mv, lx = m[:, None] * v, m[:, None] * np.cross(x, v)
    return dict(mass=m.sum(), kinetic=0.5 * (m * (v * v).sum(1)).sum(), internal=(m * u).sum(),
                momentum=mv.sum(0), angular_momentum=lx.sum(0),
                momentum_abs=np.abs(mv).sum(0), angular_momentum_abs=np.abs(lx).sum(0))


def test_diagnostics_match_host_sums_and_direct_potential(cuda, pkg):
    ic = pkg.ic.make_impact(4096, 1024, seed=3)
    with pkg.Compute(ic, max_children_in_leaf=16) as c:
        for _ in range(3):
            c.step()
        c.synchronize()
        d = c.diagnostics(theta_potential=0.3)
        h = host_sums(c)
        for k in ("mass", "kinetic", "internal"):
            assert abs(d[k] - h[k]) <= 1e-12 * abs(h[k]), (k, d[k], h[k])
        for k in ("momentum", "angular_momentum"):
            # the totals cancel to near zero: compare against the sum of magnitudes
            assert np.all(np.abs(np.asarray(d[k]) - h[k]) <= 1e-12 * h[k + "_abs"]), (k, d[k], h[k])
        # potential energy against the FP64 direct sum over every particle
        n = int(ic["n"])
        ref = c.gravity_direct_f64(np.arange(n, dtype=np.int32))
        m = c.download("mass").astype(np.float64)
        epot = 0.5 * float((m * ref[:, 3]).sum())
        assert d["potential_valid"]
        assert abs(d["potential"] - epot) <= 1e-4 * abs(epot), (d["potential"], epot)
        assert d["health"] == 0


def energy_drift(pkg, ic, steps, form):
    with pkg.Compute(ic, max_children_in_leaf=32) as c:
        if form != "plain":
            c.set_form(gravity="theta", theta=0.5, precision="mixed" if form == "chosen" else "reference")
        e0 = c.diagnostics()["total"]
        worst = 0.0
        done = 0
        while done < steps:
            k = min(100, steps - done)
            c.step_all(k)
            done += k
            e = c.diagnostics()["total"]
            worst = max(worst, abs(e - e0) / abs(e0))
        c.synchronize()
        return worst


def test_energy_drift_over_1000_steps_plain_and_mixed(cuda, pkg):
    """Config 0 (16 384 + 4 096 particles, leaf capacity 32), 1000 steps:
    largest relative change of the total energy in each form.  The chosen
    forms must not drift more than 1.2x the plain form."""
    ic = pkg.ic.make_impact(16384, 4096, seed=0)
    drifts = {form: energy_drift(pkg, ic, 1000, form) for form in ("plain", "theta", "chosen")}
    print()
    for form, dr in drifts.items():
        print(f"  {form:7s} max |E - E0| / |E0| over 1000 steps: {dr:.3e}")
    assert drifts["chosen"] <= 1.2 * drifts["plain"], drifts
