"""Coarse tiles (sph_set_tiling coarse = 1, the default) against the
per-particle walk (coarse = 0) for particles whose neighbour boxes reach more
than 3 cells past their own: the same step from the same state, density and
acceleration outputs compared particle by particle.

Small impacts have smoothing lengths of 2-3 cell widths, so nearly all their
particles take the coarse tiles; a larger one mixes both kinds of tile.  The
two schedules sum each particle's neighbours in different orders, so the
comparison allows float rounding: as in the parity tests, a particle that
sits on the h iteration's stopping threshold (|dh| / h <= 0.005) may stop one
iteration earlier or later; such particles are counted and bounded, and they
and their neighbours are left out of the acceleration comparison."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# relative tolerances: rounding of reordered float sums (the EOS table's
# steep parts amplify a density difference on pressure and sound speed)
TOL = {"h": 1e-5, "rho": 1e-5, "grad_term": 1e-5, "pressure": 5e-4, "sound_speed": 5e-4, "balsara": 1e-3,
       "acc": 1e-4, "du": 3e-3, "dhdt": 1e-3}


def _rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    floor = max(1e-3 * float(np.sqrt(np.mean(b * b))), 1e-30)
    if a.ndim == 2:
        return np.linalg.norm(a - b, axis=1) / np.maximum(np.linalg.norm(b, axis=1), floor)
    return np.abs(a - b) / np.maximum(np.abs(b), floor)


def _passes_to_density(c):
    c.updateOctreeBuffer()
    c.sort()
    c.gravitationalPass()
    c.densityPass()
    c.synchronize()


@pytest.mark.parametrize("n_target,n_imp,min_coarse_frac", [(16384, 4096, 0.5), (160000, 40000, 0.0)])
def test_coarse_tiles_match_the_per_particle_walk(cuda, pkg, n_target, n_imp, min_coarse_frac):
    from scipy.spatial import cKDTree

    ic = pkg.ic.make_impact(n_target, n_imp, seed=3)
    n = int(ic["n"])
    with pkg.Compute(ic, max_children_in_leaf=32) as on, pkg.Compute(ic, max_children_in_leaf=32) as off:
        assert on.get_tiling()["coarse"] is True
        off.set_tiling(coarse=False)
        assert off.get_tiling()["coarse"] is False
        for c in (on, off):
            _passes_to_density(c)
        st_on, st_off = on.hseed_stats(), off.hseed_stats()
        # the coarse tiles take what the cell tiles cannot: with them, few
        # particles are left for the per-particle walk
        assert st_off["coarse_tiles"] == 0
        assert st_on["deferred"] <= st_off["deferred"]
        if min_coarse_frac:
            assert st_off["deferred"] >= min_coarse_frac * n, st_off
            assert st_on["coarse_tiles"] > 0
            assert st_on["deferred"] <= 0.05 * n, st_on
        print(f"\n  n {n}: deferred {st_off['deferred']} -> {st_on['deferred']} with "
              f"{st_on['coarse_tiles']} coarse tiles")
        h_on = on.download("h").astype(np.float64)
        h_off = off.download("h").astype(np.float64)
        flip = np.abs(h_on - h_off) / h_off > TOL["h"]
        nf = int(flip.sum())
        assert nf <= max(5, int(1e-3 * n)), f"{nf} h-threshold flips"
        keep = ~flip
        for f in ("h", "rho", "grad_term", "pressure", "sound_speed", "balsara"):
            e = _rel(on.download(f)[keep], off.download(f)[keep])
            print(f"  density {f:12s} max rel {e.max():.2e}")
            assert e.max() <= TOL[f], (f, float(e.max()))
        on.accelerationPass()
        off.accelerationPass()
        on.synchronize()
        off.synchronize()
        assert on.health() == 0 and off.health() == 0
        after = np.ones(n, bool)
        if nf:
            pos = on.download("pos").astype(np.float64)
            near = cKDTree(pos).query_ball_point(pos[flip], r=2.0 * float(h_off.max()))
            after[np.unique(np.concatenate([np.asarray(q, np.int64) for q in near]))] = False
        for f in ("acc", "du", "dhdt"):
            e = _rel(on.download(f)[after], off.download(f)[after])
            print(f"  acceleration {f:7s} max rel {e.max():.2e}")
            assert e.max() <= TOL[f], (f, float(e.max()))
        if not nf:
            assert int(on.download("dt")[0]) == int(off.download("dt")[0])
            assert np.array_equal(on.download("next_active_time"), off.download("next_active_time"))


def test_tiling_arguments_are_checked(cuda, pkg):
    ic = pkg.ic.make_impact(2048, 512, seed=1)
    with pkg.Compute(ic) as c:
        t = c.get_tiling()
        assert t == dict(big_max=0, block_max=320, half_max=256, coarse=True)
        with pytest.raises(Exception):
            c.set_tiling(block_max=0)
        assert c.get_tiling() == t
        c.set_tiling(block_max=128, half_max=128)
        assert c.get_tiling()["block_max"] == 128
        c.step()
        c.synchronize()
        assert c.health() == 0
