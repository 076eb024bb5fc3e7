"""The opening-angle gravity form against FP64 direct sums.

The reference's own gravity (its adaptive acceptance test with forced leaf
interactions) is what the parity tests pin; this form has no counterpart in
the reference.  It is judged on accuracy instead, as the configuration
"Gravity-only FMM check" states it: a Plummer sphere and a uniform cube of
2^20 equal-mass float32 particles, opening angles 0.3 / 0.5 / 0.7, relative
acceleration error against an FP64 direct sum on 16 384 random targets,
median and 99th percentile.

The FP64 direct sum itself (sph_gravity_direct_f64, on the GPU) is first
checked against the oracle's CPU direct sum.
"""
from __future__ import annotations

import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N_C1 = 1 << 20
N_TARGETS = 16384
# median relative acceleration error allowed per opening angle (the metric's
# bound is 1e-3; the looser angle is reported, not gated)
MEDIAN_BOUND = {0.3: 1e-3, 0.5: 1e-3}


def rel_acc_err(got, want):
    d = np.linalg.norm(got - want, axis=1)
    return d / np.linalg.norm(want, axis=1)


def test_direct_f64_matches_oracle(cuda, pkg, O):
    ic = pkg.ic.make_impact(16384, 4096, seed=0)
    rng = np.random.default_rng(1)
    targets = rng.choice(ic["n"], 1000, replace=False).astype(np.int32)
    with pkg.Compute(ic, max_children_in_leaf=32) as c:
        got = c.gravity_direct_f64(targets)
    want = O.gravity_direct_f64(ic["pos"], ic["mass"], targets)
    err = np.abs(got - want) / np.maximum(np.abs(want), 1e-300)
    assert err.max() < 1e-10, err.max()


@pytest.mark.parametrize("body", ["plummer", "cube"])
def test_theta_form_error_against_fp64_direct_sum(cuda, pkg, body):
    make = pkg.ic.make_plummer if body == "plummer" else pkg.ic.make_cube
    ic = make(N_C1, seed=7)
    rng = np.random.default_rng(11)
    targets = rng.choice(N_C1, N_TARGETS, replace=False).astype(np.int32)
    print()
    with pkg.Compute(ic, max_children_in_leaf=16, max_tree_depth=10) as c:
        ref = c.gravity_direct_f64(targets)
        for theta in (0.3, 0.5, 0.7):
            c.set_form(gravity="theta", theta=theta)
            c.updateOctreeBuffer()
            c.gravitationalPass()
            c.synchronize()
            t0 = time.perf_counter()
            for _ in range(3):
                c.gravitationalPass()
            c.synchronize()
            ms = (time.perf_counter() - t0) / 3 * 1e3
            acc = c.download("acc")[targets].astype(np.float64)
            phi = c.download("potential")[targets].astype(np.float64)
            e = rel_acc_err(acc, ref[:, :3])
            ep = np.abs(phi - ref[:, 3]) / np.abs(ref[:, 3])
            med, p99 = float(np.median(e)), float(np.percentile(e, 99))
            print(f"  {body:8s} theta {theta:.1f}: acc rel err median {med:.2e} p99 {p99:.2e} max {e.max():.2e}; "
                  f"phi median {np.median(ep):.2e}; pass {ms:.2f} ms (host-timed)")
            assert c.health() == 0, hex(c.health())
            if theta in MEDIAN_BOUND:
                assert med <= MEDIAN_BOUND[theta], (body, theta, med)
            assert p99 < 0.05, (body, theta, p99)
