"""Checkpoint and resume: a context written with Compute.checkpoint and
rebuilt with Compute.resume continues exactly (bit for bit) as the original
context does, in the plain form, the chosen form (theta gravity + mixed
precision) and with the learned h seed."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELDS = ("pos", "vel", "acc", "rho", "u", "h", "pressure", "grad_term", "sound_speed", "du", "dhdt", "balsara",
          "grav_norm", "active", "next_active_time", "global_time", "dt")


def _state(c, mixed):
    out = {f: c.download(f) for f in FIELDS}
    if mixed:
        out["pos64"] = c.download("pos64")
    return out


@pytest.mark.parametrize("form", ["plain", "chosen", "learned"])
def test_resume_continues_bit_for_bit(cuda, pkg, tmp_path, form):
    ic = pkg.ic.make_impact(6144, 2048, seed=21)
    path = str(tmp_path / "ck.npz")
    mixed = form != "plain"
    with pkg.Compute(ic, max_children_in_leaf=32, max_tree_depth=7) as c:
        if form == "learned":
            c.hseed_capture(True)
            c.step()
            c.hseed_train(40, 4096, 1e-3)
            c.hseed_capture(False)
        if mixed:
            c.set_form(gravity="theta", theta=0.6, precision="mixed",
                       h_seed="learned" if form == "learned" else "plain")
        c.step_all(2)
        c.checkpoint(path)
        c.step_all(3)
        c.synchronize()
        want = _state(c, mixed)
    with pkg.Compute.resume(path) as r:
        assert r.get_form()["precision"] == ("mixed" if mixed else "reference")
        r.step_all(3)
        r.synchronize()
        got = _state(r, mixed)
    for k, v in want.items():
        assert np.array_equal(got[k], v), f"{form}: {k} differs after resuming"
