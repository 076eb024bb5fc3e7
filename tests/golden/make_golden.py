"""Generate the golden fixtures under tests/golden/ from the reference itself.

The reference ships no tests, golden vectors or known-answer data for its hot
path, so the fixtures come from the reference's own code run here:
oracle/ref_build.sh compiles its Metal kernels (SPH/Shaders/*.metal, through a
host shim), its CPU octree (SPH/octree/octree.cpp) and its ANEOS loader
(SPH/ANEOS/ANEOS.cpp) unchanged into oracle/_ref/libref.so, and this script
drives them in the dispatch order of SPH/Compute/Compute.cpp on seeded
synthetic inputs.  Needs the reference tree ($SPH_REFERENCE_ROOT, default the recipe's path); the
fixtures are committed so the tests run without it.

    python tests/golden/make_golden.py [reference_root]
"""
from __future__ import annotations

import hashlib
import importlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle as O  # noqa: E402

pkg_ic = importlib.import_module("real-time-planetary-impacts-mps_b200.ic")
pkg_h5 = importlib.import_module("real-time-planetary-impacts-mps_b200.hdf5io")
pkg_eos = importlib.import_module("real-time-planetary-impacts-mps_b200.eos_tables")

PASS_OUTPUTS = {
    "sort": ("cell_key", "cell_index"),
    "gravity": ("acc", "grav_norm", "active"),
    "density": ("h", "rho", "grad_term", "pressure", "sound_speed", "balsara", "dt"),
    "acceleration": ("acc", "du", "dhdt", "next_active_time", "dt"),
    "step": ("pos", "vel", "u", "h", "rho", "global_time"),
}


C0_STEPS = 10


def occupied_cells(st) -> np.ndarray:
    occ = np.nonzero(st.cell_start != 0xFFFFFFFF)[0].astype(np.uint32)
    return np.stack([occ, st.cell_start[occ], st.cell_end[occ]], axis=1)


def main(ref_root: str | None = None):
    ref_root = ref_root or O.reference_root()
    if O.build_ref(ref_root) is None:
        raise SystemExit(f"reference sources not found under {ref_root}")
    O.build()
    tabs = pkg_eos.ensure_tables()
    # 1. ANEOS loader (ANEOS.cpp) at a reduced resolution
    np.savez_compressed(os.path.join(HERE, "aneos_res128.npz"),
                        forsterite=O.aneos_load(tabs["forsterite"], 128, kind="ref"),
                        fe85si15=O.aneos_load(tabs["Fe85Si15"], 128, kind="ref"))
    ef = O.aneos_load(tabs["forsterite"], 2048, kind="ref")
    ee = O.aneos_load(tabs["Fe85Si15"], 2048, kind="ref")
    # 2. hash + sort + cell ranges on the 16384 + 4096 two-body impact
    ic = pkg_ic.make_impact(16384, 4096, seed=0)
    st = O.OracleState(ic, ef, ee, kind="ref")
    st.sort()
    np.savez_compressed(os.path.join(HERE, "sort_impact_20480.npz"), pos=ic["pos"], cell_key=st.cell_key,
                        cell_index=st.cell_index, cells=occupied_cells(st))
    # 3. the reference's CPU octree at leaf capacities 4 and 32
    trees = {}
    for leaf in (4, 32):
        t = O.tree_reference(ic["pos"], leaf, kind="ref")
        for k in ("tree", "level_offsets", "level_nodes"):
            trees[f"leaf{leaf}_{k}"] = t[k]
        trees[f"leaf{leaf}_meta"] = np.array([t["n_levels"], t["n_nodes"]], np.int32)
    np.savez_compressed(os.path.join(HERE, "octree_impact_20480.npz"), pos=ic["pos"], **trees)
    # 4. two full steps of every pass on a 2048 + 512 impact, reference tree (leaf 8)
    ic = pkg_ic.make_impact(2048, 512, seed=3)
    st = O.OracleState(ic, ef, ee, kind="ref")
    out = {f"ic_{k}": np.asarray(v) for k, v in ic.items() if isinstance(v, np.ndarray)}
    for s in range(2):
        t = O.tree_reference(st.pos, 8, kind="ref")
        st.set_tree(t)
        for k in ("tree", "level_offsets", "level_nodes"):
            out[f"s{s}_tree_{k}"] = t[k]
        out[f"s{s}_tree_meta"] = np.array([t["n_levels"], t["n_nodes"]], np.int32)
        for p, fields in PASS_OUTPUTS.items():
            getattr(st, p)()
            for f in fields:
                out[f"s{s}_{p}_{f}"] = getattr(st, f).copy()
    np.savez_compressed(os.path.join(HERE, "steps_impact_2560.npz"), **out)
    # 5. config 0 as stated (16384 + 4096, leaf capacity 32): ten full steps,
    # every pass, the reference's CPU octree rebuilt from the current
    # positions each step; SHA-256 of every output array per pass per step
    ic = pkg_ic.make_impact(16384, 4096, seed=0)
    st = O.OracleState(ic, ef, ee, kind="ref")
    digests, names = [], []
    for s in range(C0_STEPS):
        st.set_tree(O.tree_reference(st.pos, 32, kind="ref"))
        for p, fields in PASS_OUTPUTS.items():
            getattr(st, p)()
            for f in fields:
                digests.append(np.frombuffer(hashlib.sha256(np.ascontiguousarray(getattr(st, f)).tobytes()).digest(),
                                             np.uint8))
                names.append(f"s{s}_{p}_{f}")
    np.savez_compressed(os.path.join(HERE, "config0_digests.npz"), names=np.array(names), digests=np.stack(digests),
                        final_pos=st.pos, final_vel=st.vel, final_u=st.u, final_h=st.h, final_rho=st.rho)
    # 6. the reference's own input file, SPH/demo_impact_n40.hdf5, read as
    # readHDFFile does (hdfHandler.cpp:12-136); two full steps at the
    # reference's default leaf capacity (4) on its CPU octree.  Kept: the
    # initial conditions, both steps' trees, every pass output of step 0 and
    # the step-pass outputs of step 1.
    demo = os.path.join(ref_root, "SPH", "demo_impact_n40.hdf5")
    ic = pkg_h5.read_ic(demo)
    with open(demo, "rb") as f:
        file_digest = np.frombuffer(hashlib.sha256(f.read()).digest(), np.uint8)
    st = O.OracleState(ic, ef, ee, kind="ref")
    out = {f"ic_{k}": np.asarray(v) for k, v in ic.items() if isinstance(v, np.ndarray)}
    out["file_sha256"] = file_digest
    # Compute::drawSnapshot of the initial state, the reference's kernel
    # (render.metal:49-66); stored as the set pixels
    img = O.draw_snapshot_ref(ic["pos"], ic["material"]).reshape(-1)
    out["snapshot_pixel"] = np.nonzero(img)[0].astype(np.int32)
    out["snapshot_material"] = img[out["snapshot_pixel"]]
    for s in range(2):
        t = O.tree_reference(st.pos, 4, kind="ref")
        st.set_tree(t)
        for k in ("tree", "level_offsets", "level_nodes"):
            out[f"s{s}_tree_{k}"] = t[k]
        out[f"s{s}_tree_meta"] = np.array([t["n_levels"], t["n_nodes"]], np.int32)
        for p, fields in PASS_OUTPUTS.items():
            getattr(st, p)()
            if s == 0 or p == "step":
                for f in fields:
                    out[f"s{s}_{p}_{f}"] = getattr(st, f).copy()
    np.savez_compressed(os.path.join(HERE, "demo_impact_n40.npz"), **out)
    print("fixtures written to", HERE)


if __name__ == "__main__":
    main(*sys.argv[1:])
