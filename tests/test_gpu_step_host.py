"""sph_step_host: one full step whose state travels through page-locked host
memory, with the non-position inputs copied on a second stream while the
tree, sort and gravity passes run.  It must give bit-identical results to
the same step written as sph_upload_async of each field, sph_step_all(1) and
sph_download_async of each field (the eager first call and the replayed
graph alike); an h outside (0, 10] raises SPH_HEALTH_BAD_INPUT; pageable
buffers and positions of the wrong precision are refused."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SPH_HEALTH_BAD_INPUT = 0x0080


def _pinned(a):
    import torch

    t = torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
    return t, t.numpy()


@pytest.mark.parametrize("mixed", [False, True])
def test_step_host_matches_per_field_copies(cuda, pkg, mixed):
    ic = pkg.ic.make_impact(8192, 2048, seed=4)
    fields = ["pos64" if mixed else "pos", "vel", "u", "h", "rho"]
    with pkg.Compute(ic, max_children_in_leaf=32) as a, pkg.Compute(ic, max_children_in_leaf=32) as b:
        for c in (a, b):
            c.set_form(gravity="theta", theta=0.6, precision="mixed" if mixed else "reference")
        keep, host_a, host_b = [], {}, {}
        for f in fields:
            x = a.download(f)
            ta, xa = _pinned(x)
            tb, xb = _pinned(x)
            keep += [ta, tb]
            host_a[f], host_b[f] = xa, xb
        for _ in range(3):  # eager first call, then two graph replays
            for f, x in host_a.items():
                a.upload_async(f, x)
            a.step_all(1)
            for f, x in host_a.items():
                a.download_async(f, x)
            a.synchronize()
            b.step_host(host_b, host_b)
            b.synchronize()
            for f in fields:
                assert np.array_equal(host_a[f], host_b[f]), f
        assert int(a.download("global_time")[0]) == int(b.download("global_time")[0])
        assert a.health() == 0 and b.health() == 0


def test_step_host_checks(cuda, pkg):
    ic = pkg.ic.make_impact(4096, 1024, seed=6)
    with pkg.Compute(ic, max_children_in_leaf=32) as c:
        h_t, h = _pinned(c.download("h"))
        u_t, u = _pinned(c.download("u"))
        # pageable memory is refused
        with pytest.raises(Exception):
            c.step_host({"h": np.array(h)}, {})
        # FP64 positions exist in the mixed-precision form only
        p_t, p64 = _pinned(c.download("pos").astype(np.float64))
        with pytest.raises(Exception):
            c.step_host({"pos64": p64}, {})
        # an out-of-range h is replaced and reported on the device
        h[7] = 0.0
        h[9] = 50.0
        c.step_host({"h": h, "u": u}, {"h": h})
        with pytest.raises(Exception):
            c.synchronize()
        w = c.health()
        assert w & SPH_HEALTH_BAD_INPUT, hex(w)
        assert np.isfinite(h).all() and float(h.max()) <= 10.0
        c.clear_health()
        # outputs only: the state stays on the device between steps
        c.step_host({}, {"u": u})
        c.synchronize()
        assert c.health() == 0
        assert np.array_equal(u, c.download("u"))
