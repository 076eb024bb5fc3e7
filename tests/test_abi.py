"""The C ABI on the CPU: the library loads, exports every function that
include/sph.h declares, and its host-only entry points (parameter defaults,
status strings, argument checks that fail before any device work, the ANEOS
table resampler) behave.  No kernel is launched here."""
from __future__ import annotations

import ctypes as C
import subprocess

import numpy as np
import pytest


def test_library_exports_every_declared_symbol(pkg):
    pkg.build()
    lib_path = pkg._lib.LIB_PATH
    out = subprocess.run(["nm", "-D", "--defined-only", lib_path], capture_output=True, text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    declared = set(pkg._lib.declared_symbols())
    assert declared, "no declarations parsed from include/sph.h"
    missing = declared - exported
    assert not missing, f"declared but not exported: {sorted(missing)}"
    lib = pkg._lib.load()  # binds every signature; loads without a GPU
    for name in declared:
        assert hasattr(lib, name)


def test_params_default_matches_reference_parameters(pkg):
    lib = pkg._lib.load()
    p = pkg._lib.SphParams()
    lib.sph_params_default(C.byref(p))
    # SPH/Parameters.h:20, 39, 42, 43
    assert p.aneos_resolution == 2048
    assert p.max_tree_depth == 7
    assert p.max_unchecked_pointers == 1024
    assert p.max_children_in_leaf == 4
    assert p.tree_source == pkg._lib.SPH_TREE_GPU
    assert p.forsterite_table == b"ANEOS_forsterite_S19.txt"
    assert p.fe85si15_table == b"ANEOS_Fe85Si15_S20.txt"


def test_status_strings(pkg):
    lib = pkg._lib.load()
    for code, text in pkg._lib.STATUS.items():
        assert lib.sph_status_string(code).decode() == text


def test_create_rejects_bad_initial_conditions_before_device_work(pkg, eos_paths):
    lib = pkg._lib.load()
    p = pkg._lib.SphParams()
    lib.sph_params_default(C.byref(p))
    p.forsterite_table = eos_paths["forsterite"].encode()
    p.fe85si15_table = eos_paths["Fe85Si15"].encode()
    n = 8
    arrays = dict(pos=np.zeros(3 * n, np.float32), vel=np.zeros(3 * n, np.float32), rho=np.ones(n, np.float32),
                  u=np.ones(n, np.float32), mass=np.ones(n, np.float32), pressure=np.zeros(n, np.float32),
                  h=np.ones(n, np.float32), material=np.full(n, 400, np.int32))
    fp, ip = C.POINTER(C.c_float), C.POINTER(C.c_int32)

    def create(**over):
        a = {k: v.copy() for k, v in arrays.items()}
        a.update(over)
        ic = pkg._lib.SphIC()
        ic.n = n
        for k in ("pos", "vel", "rho", "u", "mass", "pressure", "h"):
            setattr(ic, k, a[k].ctypes.data_as(fp))
        ic.material = a["material"].ctypes.data_as(ip)
        h = C.c_void_p()
        return lib.sph_create(C.byref(p), C.byref(ic), C.byref(h))

    bad_pos = arrays["pos"].copy()
    bad_pos[4] = np.nan
    assert create(pos=bad_pos) == 1
    assert b"non-finite" in lib.sph_last_error()
    assert create(h=np.full(n, -1.0, np.float32)) == 1
    assert create(h=np.full(n, 50.0, np.float32)) == 1
    assert create(mass=np.zeros(n, np.float32)) == 1
    # missing table -> i/o error, before any allocation
    p.forsterite_table = b"/nonexistent/ANEOS_forsterite_S19.txt"
    assert create() == 3
    # null initial conditions
    assert lib.sph_create(C.byref(p), None, C.byref(C.c_void_p())) == 1


def test_host_resampler_matches_oracle_bit_for_bit(pkg, O, eos_paths):
    for mat in ("forsterite", "Fe85Si15"):
        a = pkg.eos_resample(eos_paths[mat], 256)
        b = O.aneos_load(eos_paths[mat], 256)
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), mat


def test_resampler_rejects_missing_and_truncated_tables(pkg, eos_paths, tmp_path):
    with pytest.raises(pkg.SphError) as e:
        pkg.eos_resample(str(tmp_path / "missing.txt"), 16)
    assert e.value.status == 3
    text = open(eos_paths["forsterite"]).read().splitlines()
    short = tmp_path / "short.txt"
    short.write_text("\n".join(text[: len(text) // 2]) + "\n")
    with pytest.raises(pkg.SphError) as e:
        pkg.eos_resample(str(short), 16)
    assert e.value.status == 3
