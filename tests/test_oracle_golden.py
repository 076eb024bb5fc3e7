"""The oracle restatement against the golden fixtures made by the reference's
own code (tests/golden/make_golden.py): every integer and float output must be
bit-identical, since both are single-precision host builds without FP
contraction."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import golden

PASS_OUTPUTS = {
    "sort": ("cell_key", "cell_index"),
    "gravity": ("acc", "grav_norm", "active"),
    "density": ("h", "rho", "grad_term", "pressure", "sound_speed", "balsara", "dt"),
    "acceleration": ("acc", "du", "dhdt", "next_active_time", "dt"),
    "step": ("pos", "vel", "u", "h", "rho", "global_time"),
}


def bits(a):
    a = np.ascontiguousarray(a)
    return a.view(np.uint8)


def test_aneos_loader_matches_reference(O, eos_paths):
    g = golden("aneos_res128.npz")
    assert np.array_equal(bits(O.aneos_load(eos_paths["forsterite"], 128)), bits(g["forsterite"]))
    assert np.array_equal(bits(O.aneos_load(eos_paths["Fe85Si15"], 128)), bits(g["fe85si15"]))


def test_aneos_missing_file_is_an_error(O, tmp_path):
    with pytest.raises(RuntimeError):
        O.aneos_load(str(tmp_path / "absent.txt"), 16)


def test_sort_and_cells_match_reference(O, eos_grids):
    g = golden("sort_impact_20480.npz")
    ic = dict(pos=g["pos"], vel=np.zeros_like(g["pos"]), rho=np.ones(len(g["pos"])), u=np.ones(len(g["pos"])),
              mass=np.ones(len(g["pos"])), h=np.ones(len(g["pos"])), material=np.zeros(len(g["pos"]), np.int32))
    st = O.OracleState(ic, *eos_grids)
    st.sort()
    assert np.array_equal(st.cell_key, g["cell_key"])
    assert np.array_equal(st.cell_index, g["cell_index"])
    occ = np.nonzero(st.cell_start != 0xFFFFFFFF)[0]
    assert np.array_equal(occ, g["cells"][:, 0])
    assert np.array_equal(st.cell_start[occ], g["cells"][:, 1])
    assert np.array_equal(st.cell_end[occ], g["cells"][:, 2])
    # empty cells: start UINT_MAX, end 0 (sort.metal:131-138)
    assert np.all(st.cell_end[st.cell_start == 0xFFFFFFFF] == 0)


def test_cell_key_wraps_negative_coordinates(O):
    # floor(x/0.18) % 256 is negative for x < 0 and wraps (sort.metal:24-34)
    k_neg = O.load().ora_cell_key(-0.01, 0.0, 0.0)
    k_pos = O.load().ora_cell_key(255 * 0.18 + 0.01, 0.0, 0.0)
    assert k_neg == k_pos


@pytest.mark.parametrize("leaf", [4, 32])
def test_octree_matches_reference(O, leaf):
    g = golden("octree_impact_20480.npz")
    t = O.tree_reference(g["pos"], leaf, 7)
    for k in ("tree", "level_offsets", "level_nodes"):
        assert np.array_equal(t[k], g[f"leaf{leaf}_{k}"]), k
    assert [t["n_levels"], t["n_nodes"]] == list(g[f"leaf{leaf}_meta"])


def test_two_steps_of_every_pass_match_reference(O, eos_grids):
    g = golden("steps_impact_2560.npz")
    ic = {k[3:]: v for k, v in g.items() if k.startswith("ic_")}
    st = O.OracleState(ic, *eos_grids)
    for s in range(2):
        tree = dict(tree=g[f"s{s}_tree_tree"], level_offsets=g[f"s{s}_tree_level_offsets"],
                    level_nodes=g[f"s{s}_tree_level_nodes"], n_levels=int(g[f"s{s}_tree_meta"][0]),
                    n_nodes=int(g[f"s{s}_tree_meta"][1]))
        st.set_tree(tree)
        for p, fields in PASS_OUTPUTS.items():
            getattr(st, p)()
            for f in fields:
                assert np.array_equal(bits(getattr(st, f)), bits(g[f"s{s}_{p}_{f}"])), f"step {s} {p} {f}"


def test_morton_tree_properties(O):
    """The GPU builder's tree, restated: every particle in exactly one leaf,
    leaves within capacity unless at the depth cap, children in octant order."""
    g = golden("sort_impact_20480.npz")
    pos = g["pos"]
    for leaf, depth in ((4, 7), (32, 7), (32, 10)):
        t = O.tree_morton(pos, leaf, depth)
        T = t["tree"]
        seen = np.zeros(len(pos), np.int32)
        off = t["level_offsets"]
        for lvl in range(t["n_levels"]):
            for tp in t["level_nodes"][off[lvl]:off[lvl + 1]]:
                n = T[tp]
                if n > 0:
                    assert n <= leaf or lvl == depth
                    seen[T[tp + 2:tp + 2 + n]] += 1
        assert np.all(seen == 1)
        # data pointers are the DFS preorder index
        dps = np.sort(T[t["level_nodes"] + 1])
        assert np.array_equal(dps, np.arange(t["n_nodes"]))


def test_config0_ten_steps_match_reference_digests(O, eos_grids, pkg):
    """Config 0 as stated (16384 + 4096 particles, leaf capacity 32): ten full
    steps with the reference's octree rebuilt each step; every output of every
    pass is bit-identical to the reference's own kernels (SHA-256 per array)."""
    import hashlib

    g = golden("config0_digests.npz")
    want = dict(zip([str(x) for x in g["names"]], g["digests"]))
    ic = pkg.ic.make_impact(16384, 4096, seed=0)
    st = O.OracleState(ic, *eos_grids)
    for s in range(10):
        st.set_tree(O.tree_reference(st.pos, 32))
        for p, fields in PASS_OUTPUTS.items():
            getattr(st, p)()
            for f in fields:
                d = np.frombuffer(hashlib.sha256(np.ascontiguousarray(getattr(st, f)).tobytes()).digest(), np.uint8)
                assert np.array_equal(d, want[f"s{s}_{p}_{f}"]), f"step {s} {p} {f}"
    for f in ("pos", "vel", "u", "h", "rho"):
        assert np.array_equal(bits(getattr(st, f)), bits(g[f"final_{f}"])), f


def test_snapshot_splat_matches_reference_kernel(O, pkg):
    """The oracle's splat equals the reference's drawToSnapshot
    (render.metal:49-66, built into oracle/_ref when the reference tree is
    present) and the reference's splat of its demo input (golden fixture)."""
    import os
    g = golden("demo_impact_n40.npz")
    want = np.zeros(1024 * 1024, np.int32)
    want[g["snapshot_pixel"]] = g["snapshot_material"]
    assert np.array_equal(O.draw_snapshot(g["ic_pos"], g["ic_material"]).reshape(-1), want)
    if not os.path.exists(O.REF_PATH):
        pytest.skip("reference build (oracle/_ref) not present")
    ic = pkg.ic.make_impact(4096, 1024, seed=0)
    assert np.array_equal(O.draw_snapshot(ic["pos"], ic["material"]), O.draw_snapshot_ref(ic["pos"], ic["material"]))
    # splats on the edges: x exactly 250 Mm and just inside the far side
    p = np.array([[250.0, 250.0, 0.0], [250.0 + 127.42 * 0.999, 300.0, 0.0], [249.99, 300.0, 0.0]], np.float32)
    m = np.array([400, 402, 400], np.int32)
    assert np.array_equal(O.draw_snapshot(p, m), O.draw_snapshot_ref(p, m))
