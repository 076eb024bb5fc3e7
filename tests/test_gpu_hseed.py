"""The learned smoothing-length seed: tensor-core MLP training and its use.

1. Gradients of the tcgen05 training kernel against the CPU oracle
   (oracle/mlp.py), which restates the same arithmetic with the same BF16
   rounding points in FP64.
2. Online training on pairs recorded from the solver's own density passes
   lowers the loss.
3. On an impact, the density pass started from the learned seed against the
   plain initial guess (the particle's own h): sweeps of the h iteration per
   particle, the fallback rate and the pass time; and, iterated to a tight
   tolerance, both starts converge to the same h within 1e-6 relative.
"""
from __future__ import annotations

import numpy as np
import pytest

import mlp

pytestmark = pytest.mark.gpu


def recorded(pkg, ic, steps=2, leaf=32):
    c = pkg.Compute(ic, max_children_in_leaf=leaf)
    c.hseed_capture(True)
    for _ in range(steps):
        c.step()
    c.synchronize()
    return c


def test_tensor_core_gradient_matches_cpu_oracle(cuda, pkg):
    ic = pkg.ic.make_impact(16384, 4096, seed=0)
    with recorded(pkg, ic) as c:
        c.hseed_train(20, 4096, 1e-3)  # weights away from their start, standardisation fixed
        X, y, norm = c.hseed_dataset()
        p = c.hseed_params()
        for batch, salt in ((512, 99), (1000, 12345)):  # 1000: a partial last tile
            g, loss = c.hseed_gradient(batch, salt)
            rows = mlp.sample_rows(batch, salt, X.shape[0])
            loss_ref, g_ref = mlp.forward_backward(p, X, y, norm, rows)
            assert abs(loss - loss_ref) <= 1e-3 * loss_ref, (loss, loss_ref)
            o = 0
            for name, shape in mlp.SIZES:
                k = int(np.prod(shape))
                a, b = g[o:o + k].astype(np.float64), g_ref[o:o + k]
                err = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)
                print(f"  batch {batch} grad {name:2s}: relative error {err:.2e} (|g| {np.linalg.norm(b):.2e})")
                assert err < 1e-2, (batch, name, err)
                o += k


def test_online_training_lowers_the_loss(cuda, pkg):
    ic = pkg.ic.make_impact(16384, 4096, seed=1)
    with recorded(pkg, ic) as c:
        first = c.hseed_train(1, 8192, 1e-3)
        last = c.hseed_train(300, 8192, 1e-3)
        print(f"\n  loss {first:.4f} -> {last:.4f} after 300 Adam steps")
        assert last < 0.98 * first


def test_learned_seed_against_plain_guess(cuda, pkg):
    import torch

    ic = pkg.ic.make_impact(80000, 20000, seed=2)
    fields = ("pos", "vel", "u", "h", "rho", "pressure", "grad_term", "sound_speed", "balsara", "dhdt", "acc")
    with recorded(pkg, ic, steps=1) as c:
        # online training: a few steps, each recording its density pass
        for _ in range(4):
            c.step()
            c.hseed_train(100, 16384, 1e-3)
        c.updateOctreeBuffer()
        c.sort()
        c.gravitationalPass()
        c.synchronize()
        state = {f: c.download(f) for f in fields}
        gt, dt = c.download("global_time"), c.download("dt")
        s = torch.cuda.Stream()
        res = {}
        for tol in (0.0, 1e-7):
            for seed in ("plain", "learned"):
                def restore():
                    for f, v in state.items():
                        c.upload(f, v)
                    c.upload("global_time", gt)
                    c.upload("dt", dt)

                restore()
                c.set_form(h_seed=seed, h_tolerance=tol)
                c.densityPass(s)  # warm
                s.synchronize()
                restore()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(s)
                c.densityPass(s)
                e1.record(s)
                s.synchronize()
                st = c.hseed_stats()
                res[(tol, seed)] = dict(ms=e0.elapsed_time(e1), h=c.download("h"),
                                        sweeps=st["sweeps"] / st["particles"], max=st["max_sweeps"],
                                        fallback=st["fallbacks"] / st["particles"])
        print()
        for (tol, seed), r in res.items():
            print(f"  tol {tol or 0.005:.0e} {seed:7s}: {r['sweeps']:.3f} sweeps/particle (max {r['max']}), "
                  f"fallback {r['fallback']:.4f}, density pass {r['ms']:.2f} ms")
        # the seed must save iterations, and rarely fall back
        assert res[(0.0, "learned")]["sweeps"] < res[(0.0, "plain")]["sweeps"]
        assert res[(0.0, "learned")]["fallback"] < 0.05
        # iterated tightly, both starts converge to the same h
        a, b = res[(1e-7, "learned")]["h"].astype(np.float64), res[(1e-7, "plain")]["h"].astype(np.float64)
        rel = np.abs(a - b) / b
        print(f"  tight tolerance: converged h max relative difference {rel.max():.2e}")
        assert rel.max() <= 1e-6


def test_online_refresh_keeps_the_seed_fresh(cuda, pkg):
    """Graph-replayed steps with the online refresh (sph_hseed_online): the
    weights keep changing from replay to replay (the Adam step counter and the
    minibatches live on the device), and after 12 steps the seeded density
    passes still take fewer sweeps than the plain start at the same point."""
    ic = pkg.ic.make_impact(80000, 20000, seed=2)
    res = {}
    for online in (False, True):
        with recorded(pkg, ic, steps=1) as c:
            for _ in range(2):
                c.step()
                c.hseed_train(200, 16384, 1e-3)
            c.hseed_capture(False)
            c.set_form(h_seed="learned")
            if online:
                c.hseed_online(16, 16384, 1e-3)
            c.step_all(2)
            c.synchronize()
            p0 = c.hseed_params()
            c.step_all(12)
            c.synchronize()
            assert c.health() == 0
            st = c.hseed_stats()
            res[online] = (st["sweeps"] / st["particles"], st["fallbacks"] / st["particles"])
            changed = not np.array_equal(p0, c.hseed_params())
            assert changed == online
    with recorded(pkg, ic, steps=1) as c:
        c.hseed_capture(False)
        c.step_all(2 + 2 + 12)
        c.synchronize()
        st = c.hseed_stats()
        plain = st["sweeps"] / st["particles"]
    print(f"\n  sweeps/particle after 16 steps: plain start {plain:.2f}, seed trained once {res[False][0]:.2f} "
          f"(fallback {res[False][1]:.4f}), refreshed online {res[True][0]:.2f} (fallback {res[True][1]:.4f})")
    assert res[True][0] < plain
    assert res[True][1] < 0.02
