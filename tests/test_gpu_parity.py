"""Parity of the CUDA path (through the C ABI) with the reference's logic.

Integer outputs (cell keys, sorted order, cell ranges, active flags, next
active times, dt, global time, the GPU-built tree) must be bit-identical.
Float outputs are compared per particle as
    err = |gpu - ref| / max(|ref|, 1e-3 * rms(ref))
against the tolerances below.  SPH fields differ only by FMA contraction
(<= 1e-5).  Gravity is ill-conditioned in the reference's coordinates: bodies
sit ~318 Mm from the origin, so float32 centres of mass carry ~3e-5 Mm of
rounding and near-field M2L forces move by ~1e-3 relative when only the
rounding changes.  The reference's own kernels compiled with FMA contraction
differ from the uncontracted build by max 1.46e-3 / p99 3.3e-4 on the golden
case (tests/test_fp_sensitivity.py); gravity tolerances are set at twice that.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu

PASS_OUTPUTS = {
    "sort": ("cell_key", "cell_index"),
    "gravity": ("acc", "grav_norm", "active"),
    "density": ("h", "rho", "grad_term", "pressure", "sound_speed", "balsara", "dt"),
    "acceleration": ("acc", "du", "dhdt", "next_active_time", "dt"),
    "step": ("pos", "vel", "u", "h", "rho", "global_time"),
}
INT_FIELDS = {"cell_key", "cell_index", "active", "next_active_time", "dt", "global_time"}
# max relative tolerances (see module docstring); p99 of gravity fields <= 1e-3
# pressure and sound speed come from the EOS table at coordinates log(u)/log(1e10)
# and log(rho)/log(1e6) scaled by 2048 texels: one ulp of logf (CUDA vs glibc)
# moves the sample by ~1e-4 texel, up to a few 1e-5 of the value where the table is steep
TOL = {"acc": 3e-3, "grav_norm": 3e-3, "h": 1e-5, "rho": 1e-5, "grad_term": 1e-5, "pressure": 1e-4,
       "sound_speed": 1e-4, "balsara": 1e-4, "du": 1e-4, "dhdt": 1e-4, "pos": 1e-6, "vel": 3e-3, "u": 1e-5}
P99_TOL = {"acc": 1e-3, "grav_norm": 1e-3, "vel": 1e-4}
# The product build sums each particle's neighbours in 8 interleaved slices
# (one per lane of its group) and adds the slices at the end, so its float sums
# differ from the reference's sequential ones by rounding: ~5e-7 relative on
# density, which the steep EOS table turns into up to ~1e-4 on pressure.
TOL_PRODUCT = dict(TOL, pressure=5e-4, sound_speed=5e-4, balsara=1e-3, du=3e-3, dhdt=1e-3,
                   acc=5e-3, grav_norm=5e-3, vel=5e-3)
# The parity build (-fmad=false, sequential sums) rounds like the reference:
# gravity bit-identical; h, density, the grad-h term, positions, velocities
# and u within 1e-5; the EOS outputs differ by one ulp of logf/powf (CUDA
# against glibc) in the table coordinate, which moves pressure by up to
# 1.4e-4 and sound speed by up to 2.4e-5 on the steep parts of the table
# (measured over config 0's ten steps).  What is computed from them carries
# that: the Balsara switch (5e-5), the acceleration pass's acc (3e-5), dh/dt
# (4e-5, a sum with cancellation) and du/dt (3.5e-4, where its pressure and
# viscous terms cancel).
TOL_PARITY = {"acc": 1e-4, "grav_norm": 1e-5, "h": 1e-5, "rho": 1e-5, "grad_term": 1e-5, "pressure": 2e-4,
              "sound_speed": 1e-4, "balsara": 1e-4, "du": 1e-3, "dhdt": 1e-4, "pos": 1e-6, "vel": 1e-5, "u": 1e-5}

P99_TOL_PARITY = {}
PASS_METHOD = {"sort": "sort", "gravity": "gravitationalPass", "density": "densityPass",
               "acceleration": "accelerationPass", "step": "stepPass"}


def rel_err(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    scale = np.sqrt(np.mean(b * b)) if b.size else 1.0
    floor = max(1e-3 * scale, 1e-30)
    if a.ndim == 2:
        d = np.linalg.norm(a - b, axis=1)
        m = np.linalg.norm(b, axis=1)
    else:
        d = np.abs(a - b)
        m = np.abs(b)
    return d / np.maximum(m, floor)


def compare(field, got, want, where, tol=None, p99=None):
    tol = TOL if tol is None else tol
    p99 = P99_TOL if p99 is None else p99
    if field in INT_FIELDS:
        bad = np.nonzero(np.asarray(got).reshape(-1) != np.asarray(want).reshape(-1))[0]
        assert bad.size == 0, f"{where} {field}: {bad.size} mismatches, first at {bad[:5]}"
        return 0.0
    e = rel_err(got, want)
    worst = float(e.max()) if e.size else 0.0
    print(f"  {where:28s} {field:12s} max rel err {worst:.3e}  p99 {np.percentile(e, 99):.3e}")
    assert np.all(np.isfinite(np.asarray(got))), f"{where} {field}: non-finite values"
    assert worst <= tol[field], f"{where} {field}: max rel err {worst:.3e} > {tol[field]:.1e}"
    if field in p99 and e.size:
        q = float(np.percentile(e, 99))
        assert q <= p99[field], f"{where} {field}: p99 rel err {q:.3e} > {p99[field]:.1e}"
    return worst


def tree_of(g, s):
    return dict(tree=g[f"s{s}_tree_tree"], level_offsets=g[f"s{s}_tree_level_offsets"],
                level_nodes=g[f"s{s}_tree_level_nodes"], n_levels=int(g[f"s{s}_tree_meta"][0]),
                n_nodes=int(g[f"s{s}_tree_meta"][1]))


def test_sort_and_cells_bit_exact(cuda, pkg, O, eos_grids):
    g = golden("sort_impact_20480.npz")
    ic = pkg.ic.make_impact(16384, 4096, seed=0)
    assert np.array_equal(ic["pos"], g["pos"])
    with pkg.Compute(ic, tree_source="host") as c:
        for rep in range(2):  # the second sort clears the first sort's cells
            c.sort()
            c.synchronize()
            assert np.array_equal(c.download("cell_key"), g["cell_key"])
            assert np.array_equal(c.download("cell_index"), g["cell_index"])
            start, end = c.download("cell_start"), c.download("cell_end")
            want_s = np.full(1 << 24, 0xFFFFFFFF, np.uint32)
            want_e = np.zeros(1 << 24, np.uint32)
            want_s[g["cells"][:, 0]] = g["cells"][:, 1]
            want_e[g["cells"][:, 0]] = g["cells"][:, 2]
            assert np.array_equal(start, want_s)
            assert np.array_equal(end, want_e)
        # move every particle: stale cells must be cleared
        pos2 = ic["pos"] + np.float32(0.37)
        c.upload("pos", pos2)
        c.sort()
        c.synchronize()
        st = O.OracleState(dict(ic, pos=pos2), *eos_grids)
        st.sort()
        assert np.array_equal(c.download("cell_key"), st.cell_key)
        assert np.array_equal(c.download("cell_index"), st.cell_index)
        assert np.array_equal(c.download("cell_start"), st.cell_start)
        assert np.array_equal(c.download("cell_end"), st.cell_end)


@pytest.mark.parametrize("build", ["parity", "product"])
def test_every_pass_matches_reference_two_steps(cuda, pkg, build):
    """Each pass against the reference's own outputs (golden), with the
    reference's CPU octree; each step starts from the reference's state."""
    g = golden("steps_impact_2560.npz")
    ic = {k[3:]: v for k, v in g.items() if k.startswith("ic_")}
    print()
    parity = build == "parity"
    if parity:
        pkg.build(parity=True)
    tol = TOL_PARITY if parity else TOL_PRODUCT
    p99 = P99_TOL_PARITY if parity else P99_TOL
    with pkg.Compute(ic, tree_source="host", max_children_in_leaf=8, parity=parity) as c:
        for s in range(2):
            if s == 1:
                # restart from the reference's state after step 0
                for f in ("pos", "vel", "u", "h", "rho"):
                    c.upload(f, g[f"s0_step_{f}"])
                c.upload("global_time", g["s0_step_global_time"])
                c.upload("next_active_time", g["s0_acceleration_next_active_time"])
                c.upload("grav_norm", g["s0_gravity_grav_norm"])
                c.upload("active", g["s0_gravity_active"])
                for f in ("pressure", "grad_term", "balsara", "sound_speed"):
                    c.upload(f, g[f"s0_density_{f}"])
            c.set_tree(tree_of(g, s))
            for p, fields in PASS_OUTPUTS.items():
                getattr(c, PASS_METHOD[p])()
                c.synchronize()
                for f in fields:
                    compare(f, c.download(f), g[f"s{s}_{p}_{f}"], f"{build} step {s} {p}", tol, p99)


@pytest.mark.parametrize("build", ["product", "parity"])
def test_demo_file_steps_match_reference(cuda, pkg, build):
    """The reference's own input (SPH/demo_impact_n40.hdf5, 10 766 particles,
    read by hdf5io as readHDFFile does): every pass of step 0 and the state
    after step 1 against the reference's kernels on the same input and the
    same CPU octree (leaf capacity 4, the reference's default); step 1 restarts
    from the reference's state after step 0."""
    g = golden("demo_impact_n40.npz")
    ic = {k[3:]: v for k, v in g.items() if k.startswith("ic_")}
    parity = build == "parity"
    if parity:
        pkg.build(parity=True)
    # On this input FMA contraction alone moves the reference's own gravity by
    # max 5.7e-3 (p99 1.4e-4; tests/test_fp_sensitivity.py); the product
    # build's gravity-derived fields get twice that, the p99 bounds unchanged.
    # In the parity build gravity is bit-identical; the acceleration pass's acc
    # carries one ulp of logf/powf in the EOS table coordinate (5.9e-5 here,
    # inside its 1e-4 bound), and v += dt a carries that into the velocity
    # (1.3e-5 after two steps): 5e-5 for this input.
    tol = dict(TOL_PARITY, vel=5e-5) if parity else dict(TOL_PRODUCT, acc=1.2e-2, grav_norm=1.2e-2, vel=1.2e-2)
    p99 = P99_TOL_PARITY if parity else P99_TOL
    print()
    with pkg.Compute(ic, tree_source="host", max_children_in_leaf=4, parity=parity) as c:
        for s in range(2):
            if s == 1:
                for f in ("pos", "vel", "u", "h", "rho"):
                    c.upload(f, g[f"s0_step_{f}"])
                c.upload("global_time", g["s0_step_global_time"])
                c.upload("next_active_time", g["s0_acceleration_next_active_time"])
                c.upload("grav_norm", g["s0_gravity_grav_norm"])
                c.upload("active", g["s0_gravity_active"])
                for f in ("pressure", "grad_term", "balsara", "sound_speed"):
                    c.upload(f, g[f"s0_density_{f}"])
            c.set_tree(tree_of(g, s))
            for p, fields in PASS_OUTPUTS.items():
                getattr(c, PASS_METHOD[p])()
                c.synchronize()
                if s == 0 or p == "step":
                    for f in fields:
                        compare(f, c.download(f), g[f"s{s}_{p}_{f}"], f"demo {build} step {s} {p}", tol, p99)


def test_gpu_tree_matches_oracle_morton_tree(cuda, pkg, O):
    ic = pkg.ic.make_impact(16384, 4096, seed=0)
    for leaf, depth in ((4, 7), (32, 7), (32, 10)):
        with pkg.Compute(ic, tree_source="gpu", max_children_in_leaf=leaf, max_tree_depth=depth) as c:
            c.updateOctreeBuffer()
            t = c.get_tree()
            w = O.tree_morton(ic["pos"], leaf, depth)
            assert t["n_levels"] == w["n_levels"] and t["n_nodes"] == w["n_nodes"], (leaf, depth)
            for k in ("tree", "level_offsets", "level_nodes"):
                assert np.array_equal(t[k], w[k]), (leaf, depth, k)


def test_gravity_on_gpu_tree_matches_oracle(cuda, pkg, O, eos_grids):
    ic = pkg.ic.make_impact(16384, 4096, seed=0)
    print()
    with pkg.Compute(ic, tree_source="gpu", max_children_in_leaf=32) as c:
        st = O.OracleState(ic, *eos_grids)
        st.set_tree(O.tree_morton(ic["pos"], 32, 7))
        for rep in range(2):  # second pass: minGrav from the first pass's |a|
            c.updateOctreeBuffer()
            c.sort()
            c.gravitationalPass()
            c.synchronize()
            st.sort()
            st.gravity()
            compare("acc", c.download("acc"), st.acc, f"gpu tree gravity {rep}")
            compare("grav_norm", c.download("grav_norm"), st.grav_norm, f"gpu tree gravity {rep}")
            compare("active", c.download("active"), st.active, f"gpu tree gravity {rep}")


def test_full_steps_match_oracle(cuda, pkg, O, eos_grids):
    """Three complete steps (GPU tree) against the oracle with the same tree
    definition; trajectories may drift by rounding, so tolerances are looser."""
    ic = pkg.ic.make_impact(4096, 1024, seed=5)
    print()
    with pkg.Compute(ic, tree_source="gpu", max_children_in_leaf=16) as c:
        st = O.OracleState(ic, *eos_grids)
        for s in range(3):
            c.step()
            c.synchronize()
            st.full_step(lambda p: O.tree_morton(p, 16, 7))
            assert c.download("dt")[0] == st.dt[0]
            assert c.download("global_time")[0] == st.global_time[0]
            for f in ("pos", "vel", "u", "h", "rho"):
                e = rel_err(c.download(f), getattr(st, f))
                print(f"  full step {s} {f:6s} max rel err {e.max():.3e}")
                assert e.max() < 1e-3 * (s + 1), (s, f)


def test_step_all_graph_equals_eager(cuda, pkg):
    ic = pkg.ic.make_impact(4096, 1024, seed=7)
    with pkg.Compute(ic, max_children_in_leaf=16) as a, pkg.Compute(ic, max_children_in_leaf=16) as b:
        for _ in range(4):
            a.step()
        b.step_all(4)
        a.synchronize()
        b.synchronize()
        for f in ("pos", "vel", "u", "h", "rho", "acc", "global_time", "next_active_time"):
            assert np.array_equal(a.download(f).view(np.uint8), b.download(f).view(np.uint8)), f


def test_snapshot_splat(cuda, pkg, O):
    """Compute::drawSnapshot (render.metal:49-66): the GPU splat equals the
    oracle's restatement (pinned to the reference's kernel in
    test_oracle_golden) on a synthetic impact, and the reference's own splat
    of its demo input (golden fixture)."""
    ic = pkg.ic.make_impact(4096, 1024, seed=0)
    with pkg.Compute(ic) as c:
        img = c.drawSnapshot()
    assert np.array_equal(img.reshape(1024, 1024), O.draw_snapshot(ic["pos"], ic["material"]))
    g = golden("demo_impact_n40.npz")
    ic = {k[3:]: v for k, v in g.items() if k.startswith("ic_")}
    want = np.zeros(1024 * 1024, np.int32)
    want[g["snapshot_pixel"]] = g["snapshot_material"]
    with pkg.Compute(ic, max_children_in_leaf=4) as c:
        img = c.drawSnapshot()
    assert np.array_equal(img.reshape(-1), want)


STATE = ("pos", "vel", "u", "h", "rho", "pressure", "grad_term", "sound_speed", "balsara", "grav_norm", "active",
         "next_active_time", "global_time")


def upload_state(c, st):
    for f in STATE:
        c.upload(f, getattr(st, f))


@pytest.mark.parametrize("build", ["parity", "product"])
def test_config0_ten_steps_every_pass(cuda, pkg, O, eos_grids, build):
    """Config 0 as stated (16384 + 4096 particles, leaf capacity 32), ten
    steps: every pass of the CUDA path against the oracle (pinned bit-exact to
    the reference's own kernels over these ten steps by
    test_oracle_golden.py), on the reference's octree; each step restarts
    the GPU from the oracle's state so that differences do not compound.

    The h iteration stops at a threshold (|dh| / h <= 0.005): a particle that
    sits on it can take one iteration more or less under any rounding change,
    which moves its h by up to 0.5%.  Such particles ("flips", found from h
    after the density pass) are counted and bounded; they and every particle
    within 2 max(h) of them (whose pair sums include them) are left out of
    the later passes' comparisons of that step.  Everything else meets the
    tolerances."""
    from scipy.spatial import cKDTree

    parity = build == "parity"
    if parity:
        pkg.build(parity=True)
    tol = TOL_PARITY if parity else TOL_PRODUCT
    p99 = P99_TOL_PARITY if parity else P99_TOL
    ic = pkg.ic.make_impact(16384, 4096, seed=0)
    n = int(ic["n"])
    st = O.OracleState(ic, *eos_grids)
    worst, flips_total, failures = {}, 0, []
    print()
    with pkg.Compute(ic, tree_source="host", max_children_in_leaf=32, parity=parity) as c:
        for s in range(10):
            t = O.tree_reference(st.pos, 32)
            st.set_tree(t)
            upload_state(c, st)
            c.set_tree(t)
            keep = np.ones(n, bool)
            pos0 = np.asarray(st.pos, np.float64).reshape(-1, 3).copy()
            for p, fields in PASS_OUTPUTS.items():
                getattr(st, p)()
                getattr(c, PASS_METHOD[p])()
                c.synchronize()
                if p == "density":
                    h_ref = np.asarray(st.h, np.float64)
                    flip = np.abs(c.download("h").astype(np.float64) - h_ref) / h_ref > tol["h"]
                    nf = int(flip.sum())
                    flips_total += nf
                    assert nf <= max(5, int(1e-3 * n)), f"{build} step {s}: {nf} h-threshold flips"
                    keep = ~flip
                    if nf:
                        near = cKDTree(pos0).query_ball_point(pos0[flip], r=2.0 * float(h_ref.max()))
                        affected = np.unique(np.concatenate([np.asarray(q, np.int64) for q in near]))
                        after = np.ones(n, bool)
                        after[affected] = False
                    else:
                        after = keep
                for f in fields:
                    got, want = c.download(f), getattr(st, f)
                    m = None if p in ("sort", "gravity") else (keep if p == "density" else after)
                    if m is not None and f not in ("dt", "global_time"):
                        got, want = np.asarray(got)[m], np.asarray(want)[m]
                    try:
                        e = compare(f, got, want, f"{build} c0 step {s} {p}", tol, p99)
                        worst[f] = max(worst.get(f, 0.0), e)
                    except AssertionError as exc:
                        failures.append(str(exc))
    print(f"  h-threshold flips over ten steps: {flips_total}")
    print("  worst over ten steps (flips and their neighbours excluded):", {k: f"{v:.1e}" for k, v in worst.items()})
    assert not failures, "\n".join(failures)


def test_sort_cells_and_tree_structure_at_1e6(cuda, pkg):
    """Size-independent checks at N = 10^6 (the benchmark impact): the sort
    is a stable permutation with non-decreasing keys that equal the hash of
    each particle's position; the cell table covers [0, N) exactly, one range
    per occupied key; the GPU tree's leaves hold every particle exactly once."""
    ic = pkg.ic.make_impact(800000, 200000, seed=0)
    n = int(ic["n"])
    with pkg.Compute(ic, max_children_in_leaf=32, max_tree_depth=7) as c:
        c.step()
        c.updateOctreeBuffer()
        c.sort()
        c.synchronize()
        pos = c.download("pos")
        key, idx = c.download("cell_key"), c.download("cell_index")
        # permutation, sorted keys, stability
        assert np.array_equal(np.sort(idx), np.arange(n, dtype=np.uint32))
        assert np.all(np.diff(key.astype(np.int64)) >= 0)
        same = np.diff(key.astype(np.int64)) == 0
        assert np.all(np.diff(idx.astype(np.int64))[same] > 0)
        # keys are the hash of the positions (sort.metal:15-44)
        cell = np.floor(pos / np.float32(0.18)).astype(np.int64) & 255

        def spread(v):
            v = v & 0x3FF
            v = (v | (v << 16)) & 0x030000FF
            v = (v | (v << 8)) & 0x0300F00F
            v = (v | (v << 4)) & 0x030C30C3
            return (v | (v << 2)) & 0x09249249

        want = spread(cell[:, 0]) | (spread(cell[:, 1]) << 1) | (spread(cell[:, 2]) << 2)
        assert np.array_equal(key.astype(np.int64), want[idx])
        # cell ranges: one (first, last) per run of equal keys, empty elsewhere
        start, end = c.download("cell_start"), c.download("cell_end")
        first = np.concatenate([[True], np.diff(key.astype(np.int64)) != 0])
        last = np.concatenate([np.diff(key.astype(np.int64)) != 0, [True]])
        occ = key[first]
        assert np.array_equal(start[occ], np.nonzero(first)[0].astype(np.uint32))
        assert np.array_equal(end[occ], np.nonzero(last)[0].astype(np.uint32))
        assert int((end[occ].astype(np.int64) - start[occ] + 1).sum()) == n
        empty = np.ones(1 << 24, bool)
        empty[occ] = False
        assert np.all(start[empty] == 0xFFFFFFFF) and np.all(end[empty] == 0)
        # tree: leaf membership is a permutation
        t = c.get_tree()
        T = t["tree"]
        members = []
        for off in t["level_nodes"]:
            cnt = T[off]
            if cnt > 0:
                members.append(T[off + 2:off + 2 + cnt])
        members = np.concatenate(members)
        assert members.size == n
        assert np.array_equal(np.sort(members), np.arange(n, dtype=np.int32))
