"""ctypes binding of libsph_b200.so (include/sph.h) and its in-tree build.

The library is built in place (nvcc, sm_100a) next to this file so that it
travels with the repository; `load()` fails loudly when it is missing or when
no CUDA device is visible -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB_PATH = os.path.join(HERE, "libsph_b200.so")
# The parity build: the same sources with FMA contraction off (-fmad=false)
# and SPH_PARITY, under which every float sum runs in the reference's
# sequential order.  Only the parity tests load it; it is not the product.
PARITY_LIB_PATH = os.path.join(HERE, "libsph_b200_parity.so")
PARITY_FLAGS = ["-fmad=false", "-DSPH_PARITY"]
SOURCES = ["sph_api.cu", "sph_sort.cu", "sph_hydro.cu", "sph_gravity.cu", "sph_gravity_theta.cu", "sph_tree.cu",
           "sph_hseed.cu", "sph_ensemble.cu"]
HEADERS = ["sph_common.cuh", "sph_internal.h", "sph_tc.cuh"]
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
              "-Xcompiler", "-fPIC,-ffp-contract=off", "-shared"]

SPH_OK = 0
STATUS = {0: "ok", 1: "invalid argument", 2: "out of device memory", 3: "i/o error", 4: "cuda error",
          5: "device health bit raised", 6: "bounded device wait timed out", 7: "unsupported"}

SPH_TREE_GPU = 0
SPH_TREE_HOST = 1

SPH_GRAVITY_REFERENCE = 0
SPH_GRAVITY_THETA = 1

FIELDS = {
    "pos": 0, "vel": 1, "acc": 2, "rho": 3, "u": 4, "mass": 5, "pressure": 6, "h": 7,
    "grad_term": 8, "sound_speed": 9, "du": 10, "balsara": 11, "dhdt": 12, "grav_norm": 13,
    "material": 14, "active": 15, "next_active_time": 16, "global_time": 17, "dt": 18,
    "cell_key": 19, "cell_index": 20, "cell_start": 21, "cell_end": 22, "potential": 23, "pos64": 24,
    "neighbours": 25,
}
VECTOR_FIELDS = ("pos", "vel", "acc")

HEALTH = {"sort_timeout": 0x1, "list_capacity": 0x2, "tree_capacity": 0x4, "nan_density": 0x8,
          "scan_timeout": 0x10, "root_leaf": 0x20, "mlp_timeout": 0x40}


class SphParams(C.Structure):
    _fields_ = [
        ("max_children_in_leaf", C.c_int32),
        ("max_tree_depth", C.c_int32),
        ("max_unchecked_pointers", C.c_int32),
        ("aneos_resolution", C.c_int32),
        ("tree_source", C.c_int32),
        ("forsterite_table", C.c_char_p),
        ("fe85si15_table", C.c_char_p),
    ]


_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int32)


class SphIC(C.Structure):
    _fields_ = [
        ("n", C.c_int32),
        ("pos", _fp), ("vel", _fp), ("rho", _fp), ("u", _fp), ("mass", _fp), ("pressure", _fp), ("h", _fp),
        ("material", _ip),
    ]


class SphForm(C.Structure):
    _fields_ = [("gravity", C.c_int32), ("theta", C.c_float), ("h_seed", C.c_int32), ("precision", C.c_int32),
                ("h_tolerance", C.c_float), ("timestep", C.c_int32)]


class SphHostState(C.Structure):
    _fields_ = [("pos64", C.c_void_p), ("pos", C.c_void_p), ("vel", C.c_void_p), ("u", C.c_void_p),
                ("h", C.c_void_p), ("rho", C.c_void_p)]


class SphTiling(C.Structure):
    _fields_ = [("big_max", C.c_uint32), ("block_max", C.c_uint32), ("half_max", C.c_uint32), ("coarse", C.c_int32)]


class SphEnsembleTuning(C.Structure):
    _fields_ = [("max_children_in_leaf", C.c_int32), ("tile_block_max", C.c_uint32), ("ms_per_step", C.c_float),
                ("gravity_median_error", C.c_float)]


class SphHSeedStats(C.Structure):
    _fields_ = [("sweeps", C.c_uint32), ("fallbacks", C.c_uint32), ("max_sweeps", C.c_uint32),
                ("particles", C.c_uint32), ("tiles", C.c_uint32), ("deferred", C.c_uint32),
                ("accel_deferred", C.c_uint32), ("coarse_tiles", C.c_uint32),
                ("accel_coarse_tiles", C.c_uint32)]


SPH_HSEED_PLAIN = 0
SPH_HSEED_LEARNED = 1


SPH_PRECISION_REFERENCE = 0
SPH_PRECISION_MIXED = 1


class SphDiag(C.Structure):
    _fields_ = [("mass", C.c_double), ("kinetic", C.c_double), ("internal", C.c_double),
                ("potential", C.c_double), ("total", C.c_double), ("momentum", C.c_double * 3),
                ("angular_momentum", C.c_double * 3), ("time", C.c_double), ("potential_valid", C.c_int32),
                ("health", C.c_uint32)]


class SphError(RuntimeError):
    def __init__(self, status: int, what: str, detail: str = ""):
        self.status = status
        super().__init__(f"{what}: {STATUS.get(status, status)}" + (f" ({detail})" if detail else ""))


def build(force: bool = False, verbose: bool = False, parity: bool = False) -> str:
    """Compile libsph_b200.so (or, with parity=True, libsph_b200_parity.so)
    for sm_100a in place (cross-compiles without a GPU).  The sources are
    compiled in parallel and linked into one shared library."""
    from concurrent.futures import ThreadPoolExecutor
    out = PARITY_LIB_PATH if parity else LIB_PATH
    csrc = os.path.join(HERE, "csrc")
    srcs = [os.path.join(csrc, s) for s in SOURCES]
    deps = srcs + [os.path.join(csrc, h) for h in HEADERS] + [os.path.join(ROOT, "include", "sph.h")]
    if not force and os.path.exists(out):
        t = os.path.getmtime(out)
        if all(os.path.getmtime(d) <= t for d in deps):
            return out
    nvcc = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
    if not os.path.exists(nvcc):
        nvcc = "nvcc"
    flags = NVCC_FLAGS[:-1] + (PARITY_FLAGS if parity else [])  # without -shared for the objects
    tag = f"{os.getpid()}{'p' if parity else ''}"
    objs = [out + f".{os.path.basename(s)}.{tag}.o" for s in srcs]

    def compile_one(pair):
        src, obj = pair
        return subprocess.run([nvcc] + flags + ["-c", "-o", obj, src], capture_output=not verbose, text=True)

    with ThreadPoolExecutor(max_workers=len(srcs)) as ex:
        results = list(ex.map(compile_one, zip(srcs, objs)))
    try:
        for r in results:
            if r.returncode != 0:
                raise RuntimeError("nvcc failed:\n" + (r.stderr or "") + (r.stdout or ""))
        tmp = out + f".{tag}.tmp"
        r = subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", tmp] + objs,
                           capture_output=not verbose, text=True)
        if r.returncode != 0:
            raise RuntimeError("nvcc link failed:\n" + (r.stderr or "") + (r.stdout or ""))
        os.replace(tmp, out)
    finally:
        for o in objs:
            if os.path.exists(o):
                os.remove(o)
    return out


_LIBS: dict = {}


def load(parity: bool = False) -> C.CDLL:
    """Load the CUDA library (built in place), or its parity build.  Raises if
    it is missing."""
    if parity in _LIBS:
        return _LIBS[parity]
    path = PARITY_LIB_PATH if parity else LIB_PATH
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is not built; run __graft_entry__.build()")
    lib = C.CDLL(path)
    vp = C.c_void_p
    st = C.c_int
    sig = {
        "sph_params_default": (None, [C.POINTER(SphParams)]),
        "sph_create": (st, [C.POINTER(SphParams), C.POINTER(SphIC), C.POINTER(vp)]),
        "sph_destroy": (st, [vp]),
        "sph_num_particles": (C.c_int32, [vp]),
        "sph_update_tree": (st, [vp, vp]),
        "sph_get_tree": (st, [vp, _ip, C.c_int64, _ip, _ip, _ip, C.c_int64, _ip, _ip]),
        "sph_get_tree_nodes": (st, [vp, _fp, _fp, C.c_int32]),
        "sph_set_tree": (st, [vp, _ip, C.c_int32, _ip, _ip, C.c_int32, C.c_int32]),
        "sph_sort": (st, [vp, vp]),
        "sph_gravity": (st, [vp, vp]),
        "sph_density": (st, [vp, vp]),
        "sph_acceleration": (st, [vp, vp]),
        "sph_step": (st, [vp, vp]),
        "sph_step_all": (st, [vp, vp, C.c_int32]),
        "sph_step_host": (st, [vp, C.POINTER(SphHostState), C.POINTER(SphHostState), vp]),
        "sph_sort_cells_noalloc": (st, [vp, C.c_int32, vp, vp, vp]),
        "sph_sort_cells_noalloc_health": (st, [vp, C.POINTER(C.c_uint32)]),
        "sph_selftest_lookback_timeout": (st, [vp, C.c_int32, vp]),
        "sph_selftest_tree_capacity": (st, [vp, vp]),
        "sph_upload_async": (st, [vp, C.c_int, vp, C.c_size_t, vp]),
        "sph_download_async": (st, [vp, C.c_int, vp, C.c_size_t, vp]),
        "sph_form_default": (None, [C.POINTER(SphForm)]),
        "sph_set_form": (st, [vp, C.POINTER(SphForm)]),
        "sph_get_form": (st, [vp, C.POINTER(SphForm)]),
        "sph_set_tiling": (st, [vp, C.POINTER(SphTiling)]),
        "sph_get_tiling": (st, [vp, C.POINTER(SphTiling)]),
        "sph_gravity_direct_f64": (st, [vp, _ip, C.c_int32, C.POINTER(C.c_double), vp]),
        "sph_diagnostics": (st, [vp, vp, C.c_float, C.POINTER(SphDiag)]),
        "sph_hseed_num_params": (C.c_int32, []),
        "sph_hseed_capture": (st, [vp, C.c_int32]),
        "sph_hseed_train": (st, [vp, C.c_int32, C.c_int32, C.c_float, _fp, vp]),
        "sph_hseed_gradient": (st, [vp, C.c_int32, C.c_uint32, _fp, _fp, vp]),
        "sph_hseed_online": (st, [vp, C.c_int32, C.c_int32, C.c_float]),
        "sph_hseed_params": (st, [vp, _fp, _fp]),
        "sph_hseed_dataset": (st, [vp, _fp, _fp, _fp]),
        "sph_hseed_norm": (st, [vp, _fp, _fp]),
        "sph_hseed_get_stats": (st, [vp, C.POINTER(SphHSeedStats)]),
        "sph_draw_snapshot": (st, [vp, vp, _ip]),
        "sph_probe_fp32_fma": (st, [C.c_int32, C.c_int32, vp, vp]),
        "sph_upload": (st, [vp, C.c_int, vp, C.c_size_t]),
        "sph_download": (st, [vp, C.c_int, vp, C.c_size_t]),
        "sph_get_buffer": (st, [vp, C.c_int, C.POINTER(vp), C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)]),
        "sph_synchronize": (st, [vp, vp]),
        "sph_get_health": (st, [vp, C.POINTER(C.c_uint32)]),
        "sph_clear_health": (st, [vp]),
        "sph_eos_resample": (st, [C.c_char_p, C.c_int32, _fp]),
        "sph_ensemble_create": (st, [C.POINTER(SphParams), C.c_int32, C.POINTER(SphIC), C.POINTER(SphForm), C.c_int32,
                                     C.POINTER(vp)]),
        "sph_ensemble_destroy": (st, [vp]),
        "sph_ensemble_size": (C.c_int32, [vp]),
        "sph_ensemble_instance": (st, [vp, C.c_int32, C.POINTER(vp)]),
        "sph_ensemble_get_tuning": (st, [vp, C.c_int32, C.POINTER(SphEnsembleTuning)]),
        "sph_ensemble_step": (st, [vp, vp, C.c_int32]),
        "sph_ensemble_synchronize": (st, [vp, vp]),
        "sph_status_string": (C.c_char_p, [st]),
        "sph_last_error": (C.c_char_p, []),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _LIBS[parity] = lib
    return lib


def check(status: int, what: str, lib: C.CDLL | None = None):
    if status != SPH_OK:
        detail = (lib or load()).sph_last_error().decode(errors="replace")
        raise SphError(status, what, detail)


def declared_symbols() -> list[str]:
    """Function names declared in include/sph.h (for the export check)."""
    import re
    with open(os.path.join(ROOT, "include", "sph.h")) as f:
        text = f.read()
    return sorted(set(re.findall(r"\b(sph_[a-z0-9_]+)\s*\(", text)))
