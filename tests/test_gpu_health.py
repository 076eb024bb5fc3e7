"""Failure detection on the GPU without faulting it.

Kernels never trap: bounded waits and capacity or finiteness checks raise bits
in a device health word, which sph_synchronize turns into an error status.
Each case below makes one such failure happen on purpose from the host (a
withheld predecessor with a short spin limit, a non-finite input) and checks
that the error comes back and that the context stays usable afterwards.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SPH_ERR_DEVICE_HEALTH = 5
SPH_ERR_TIMEOUT = 6


def test_lookback_timeout_is_reported_and_context_recovers(cuda, pkg):
    lib = pkg._lib.load()
    ic = pkg.ic.make_impact(2048, 512, seed=4)
    with pkg.Compute(ic, max_children_in_leaf=16) as c:
        c.step()
        c.synchronize()
        assert lib.sph_selftest_lookback_timeout(c._h, 1000, None) == 0
        rc = lib.sph_synchronize(c._h, None)
        assert rc == SPH_ERR_TIMEOUT, rc
        assert c.health() & pkg._lib.HEALTH["sort_timeout"]
        c.clear_health()
        c.step()
        c.synchronize()  # raises on any error
        assert np.all(np.isfinite(c.download("pos")))


def test_non_finite_density_is_reported(cuda, pkg):
    lib = pkg._lib.load()
    ic = pkg.ic.make_impact(2048, 512, seed=4)
    with pkg.Compute(ic, max_children_in_leaf=16) as c:
        u = ic["u"].copy()
        u[17] = np.float32("nan")
        c.upload("u", u)
        c.updateOctreeBuffer()
        c.sort()
        c.gravitationalPass()
        c.densityPass()
        rc = lib.sph_synchronize(c._h, None)
        assert rc == SPH_ERR_DEVICE_HEALTH, rc
        assert c.health() & pkg._lib.HEALTH["nan_density"]
        c.clear_health()
        c.upload("u", ic["u"])
        c.step()
        c.synchronize()


def test_tree_capacity_is_reported_and_context_recovers(cuda, pkg):
    lib = pkg._lib.load()
    ic = pkg.ic.make_impact(2048, 512, seed=4)
    with pkg.Compute(ic, max_children_in_leaf=16) as c:
        c.step()
        c.synchronize()
        want_ok = c.download("pos")
        assert lib.sph_selftest_tree_capacity(c._h, None) == 0
        rc = lib.sph_synchronize(c._h, None)
        assert rc == SPH_ERR_DEVICE_HEALTH, rc
        assert c.health() & pkg._lib.HEALTH["tree_capacity"]
        c.clear_health()
        c.step()  # rebuilds a whole tree
        c.synchronize()
        assert np.all(np.isfinite(c.download("pos")))
        assert not np.array_equal(c.download("pos"), want_ok)  # it stepped


def test_async_transfers_round_trip_on_a_stream(cuda, pkg):
    import torch

    ic = pkg.ic.make_impact(2048, 512, seed=6)
    n = int(ic["n"])
    with pkg.Compute(ic, max_children_in_leaf=16) as c:
        s = torch.cuda.Stream()
        pos = torch.from_numpy(ic["pos"].reshape(-1).copy()).pin_memory().numpy()
        u = torch.from_numpy(ic["u"].copy()).pin_memory().numpy()
        out_pos = torch.empty(3 * n, dtype=torch.float32).pin_memory().numpy()
        out_u = torch.empty(n, dtype=torch.float32).pin_memory().numpy()
        pos2 = pos + np.float32(0.25)
        c.upload_async("pos", pos2, s)
        c.upload_async("u", u * np.float32(2.0), s)
        c.download_async("pos", out_pos, s)
        c.download_async("u", out_u, s)
        s.synchronize()
        assert np.array_equal(out_pos, pos2)
        assert np.array_equal(out_u, u * np.float32(2.0))
        # the mass rides in the position records and must survive the upload
        assert np.array_equal(c.download("mass"), ic["mass"])
