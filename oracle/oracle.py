"""ctypes harness for the CPU oracle (liboracle.so) and, when built, the
reference's own kernels compiled on the host (_ref/libref.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, never by the product package.

Both libraries take the same `ora_state` (oracle.h): SoA arrays in original
particle order, xyz-interleaved vectors.  `OracleState` owns the numpy arrays
and exposes the pass API in the reference's order (sort, gravity, density,
acceleration, step).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_PATH = os.path.join(HERE, "_ref", "libref.so")
NCELLS = 1 << 24

_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int32)
_up = C.POINTER(C.c_uint32)
_bp = C.POINTER(C.c_uint8)


class OraState(C.Structure):
    _fields_ = [
        ("n", C.c_int32),
        ("pos", _fp), ("vel", _fp), ("acc", _fp),
        ("rho", _fp), ("u", _fp), ("mass", _fp), ("pressure", _fp), ("h", _fp),
        ("grad_term", _fp), ("sound_speed", _fp), ("du", _fp), ("balsara", _fp), ("dhdt", _fp),
        ("grav_norm", _fp),
        ("material", _ip), ("active", _bp), ("next_active_time", _ip),
        ("global_time", _ip), ("dt", _ip),
        ("cell_key", _up), ("cell_index", _up), ("cell_start", _up), ("cell_end", _up),
        ("eos_forsterite", _fp), ("eos_fe", _fp), ("eos_res", C.c_int32),
        ("tree", _ip), ("tree_len", C.c_int32), ("level_offsets", _ip), ("level_nodes", _ip),
        ("n_levels", C.c_int32), ("n_nodes", C.c_int32), ("max_unchecked", C.c_int32),
    ]


def build(force: bool = False) -> str:
    """Compile liboracle.so with the system g++ (OpenMP, no FP contraction)."""
    srcs = [os.path.join(HERE, f) for f in ("oracle.cpp", "fp64.cpp", "oracle.h")]
    if force or not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < max(map(os.path.getmtime, srcs)):
        cxx = os.environ.get("SPH_HOST_CXX", "g++")
        cmd = [cxx, "-O3", "-std=c++17", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off",
               "-fno-fast-math", "-o", LIB_PATH + ".tmp"] + srcs[:2]
        subprocess.run(cmd, check=True)
        os.replace(LIB_PATH + ".tmp", LIB_PATH)
    return LIB_PATH


def reference_root() -> str:
    """Root of the reference checkout: $SPH_REFERENCE_ROOT, else the path the
    build recipe (ref_build.sh) defaults to."""
    return os.environ.get("SPH_REFERENCE_ROOT", "/root/reference")


def build_ref(reference_root_dir: str | None = None) -> str | None:
    """Build _ref/libref.so from the reference's sources when they are present."""
    reference_root = reference_root_dir or globals()["reference_root"]()
    if not os.path.isdir(os.path.join(reference_root, "SPH", "Shaders")):
        return None
    subprocess.run([os.path.join(HERE, "ref_build.sh"), reference_root], check=True,
                   stdout=subprocess.DEVNULL)
    return REF_PATH


def _bind(lib: C.CDLL, prefix: str) -> C.CDLL:
    st = C.POINTER(OraState)
    for name in ("sort", "gravity", "density", "acceleration", "step"):
        f = getattr(lib, f"{prefix}_{name}")
        f.argtypes = [st]
        f.restype = None
    return lib


_LIBS: dict = {}


def load(kind: str = "oracle") -> C.CDLL:
    """kind 'oracle' (restatement) or 'ref' (reference kernels via the shim)."""
    if kind in _LIBS:
        return _LIBS[kind]
    if kind == "oracle":
        lib = C.CDLL(build())
        _bind(lib, "ora")
        vp = C.c_void_p
        for fn in ("ora_tree_build_reference", "ora_tree_build_morton"):
            getattr(lib, fn).argtypes = [C.c_int, _fp, C.c_int, C.c_int]
            getattr(lib, fn).restype = vp
        lib.ora_tree_sizes.argtypes = [vp, _ip, _ip, _ip]
        lib.ora_tree_export.argtypes = [vp, _ip, _ip, _ip]
        lib.ora_tree_free.argtypes = [vp]
        lib.ora_aneos_load.argtypes = [C.c_char_p, C.c_int, _fp]
        lib.ora_aneos_load.restype = C.c_int
        lib.ora_cell_key.argtypes = [C.c_float, C.c_float, C.c_float]
        lib.ora_cell_key.restype = C.c_uint32
        lib.ora_gravity_direct_f64.argtypes = [C.c_int, _fp, _fp, _ip, C.c_int, C.POINTER(C.c_double)]
        lib.ora_gravity_direct_f64.restype = None
        lib.ora_set_threads.argtypes = [C.c_int]
        lib.ora_get_threads.restype = C.c_int
    elif kind == "ref":
        if not os.path.exists(REF_PATH):
            raise FileNotFoundError(REF_PATH)
        lib = C.CDLL(REF_PATH)
        _bind(lib, "ref")
        vp = C.c_void_p
        lib.ref_tree_build.argtypes = [C.c_int, _fp, C.c_int]
        lib.ref_tree_build.restype = vp
        lib.ref_tree_sizes.argtypes = [vp, _ip, _ip, _ip]
        lib.ref_tree_export.argtypes = [vp, _ip, _ip, _ip]
        lib.ref_tree_free.argtypes = [vp]
        lib.ref_aneos_load.argtypes = [C.c_char_p, C.c_int, _fp]
        lib.ref_aneos_load.restype = C.c_int
        lib.ref_draw_snapshot.argtypes = [C.c_int, _fp, _ip, _ip]
    else:
        raise ValueError(kind)
    _LIBS[kind] = lib
    return lib


def gravity_direct_f64(pos: np.ndarray, mass: np.ndarray, targets) -> np.ndarray:
    """FP64 direct-sum (ax, ay, az, phi) at the target particles, G included."""
    lib = load("oracle")
    p = np.ascontiguousarray(np.asarray(pos, np.float32).reshape(-1))
    m = np.ascontiguousarray(np.asarray(mass, np.float32).reshape(-1))
    t = np.ascontiguousarray(np.asarray(targets, np.int32).reshape(-1))
    out = np.zeros((t.size, 4), np.float64)
    lib.ora_gravity_direct_f64(int(m.size), p.ctypes.data_as(_fp), m.ctypes.data_as(_fp), t.ctypes.data_as(_ip),
                               int(t.size), out.ctypes.data_as(C.POINTER(C.c_double)))
    return out


def ptr(a: np.ndarray, t):
    return a.ctypes.data_as(t)


def _export_tree(lib, prefix: str, handle) -> dict:
    ln, nl, nn = C.c_int32(), C.c_int32(), C.c_int32()
    getattr(lib, f"{prefix}_tree_sizes")(handle, C.byref(ln), C.byref(nl), C.byref(nn))
    tree = np.zeros(max(ln.value, 1), np.int32)
    off = np.zeros(nl.value + 1, np.int32)
    nodes = np.zeros(max(ln.value, 1), np.int32)
    getattr(lib, f"{prefix}_tree_export")(handle, ptr(tree, _ip), ptr(off, _ip), ptr(nodes, _ip))
    getattr(lib, f"{prefix}_tree_free")(handle)
    return dict(tree=tree[:ln.value], level_offsets=off, level_nodes=nodes[:off[-1]],
                n_levels=nl.value, n_nodes=nn.value)


def tree_reference(pos: np.ndarray, max_leaf: int, max_depth: int = 7, kind: str = "oracle") -> dict:
    """The reference's mean-split CPU octree (octree.cpp), from the oracle
    restatement or from the reference file itself (kind='ref', depth fixed 7)."""
    pos = np.ascontiguousarray(pos, np.float32)
    lib = load(kind)
    if kind == "ref":
        h = lib.ref_tree_build(pos.shape[0], ptr(pos, _fp), max_leaf)
        return _export_tree(lib, "ref", h)
    h = lib.ora_tree_build_reference(pos.shape[0], ptr(pos, _fp), max_leaf, max_depth)
    return _export_tree(lib, "ora", h)


def tree_morton(pos: np.ndarray, max_leaf: int, max_depth: int = 7) -> dict:
    """The GPU builder's Morton octree, restated on the CPU."""
    pos = np.ascontiguousarray(pos, np.float32)
    lib = load("oracle")
    h = lib.ora_tree_build_morton(pos.shape[0], ptr(pos, _fp), max_leaf, max_depth)
    return _export_tree(lib, "ora", h)


def aneos_load(path: str, res: int = 2048, kind: str = "oracle") -> np.ndarray:
    out = np.zeros((res, res, 2), np.float32)
    lib = load(kind)
    fn = lib.ora_aneos_load if kind == "oracle" else lib.ref_aneos_load
    rc = fn(path.encode(), res, ptr(out, _fp))
    if rc != 0:
        raise RuntimeError(f"ANEOS load failed ({rc}) for {path}")
    return out


FLOAT_FIELDS = ("rho", "u", "mass", "pressure", "h", "grad_term", "sound_speed", "du", "balsara",
                "dhdt", "grav_norm")


class OracleState:
    """Owns one simulation's arrays; passes run through liboracle or libref."""

    def __init__(self, ic: dict, eos_forsterite: np.ndarray, eos_fe: np.ndarray, kind: str = "oracle",
                 max_unchecked: int = 1024):
        n = int(ic["pos"].shape[0])
        self.n = n
        self.kind = kind
        self.lib = load(kind)
        self.prefix = "ora" if kind == "oracle" else "ref"
        f32 = lambda a: np.ascontiguousarray(a, dtype=np.float32)  # noqa: E731
        self.pos = f32(ic["pos"]).reshape(n, 3).copy()
        self.vel = f32(ic["vel"]).reshape(n, 3).copy()
        self.acc = np.zeros((n, 3), np.float32)
        self.rho = f32(ic["rho"]).copy()
        self.u = f32(ic["u"]).copy()
        self.mass = f32(ic["mass"]).copy()
        self.pressure = f32(ic.get("pressure", np.zeros(n))).copy()
        self.h = f32(ic["h"]).copy()
        for name in ("grad_term", "sound_speed", "du", "balsara", "dhdt", "grav_norm"):
            setattr(self, name, np.zeros(n, np.float32))
        self.material = np.ascontiguousarray(ic["material"], dtype=np.int32).copy()
        self.active = np.ones(n, np.uint8)                 # Compute.cpp:66-70
        self.next_active_time = np.zeros(n, np.int32)      # Compute.cpp:73-77
        self.global_time = np.zeros(1, np.int32)
        self.dt = np.zeros(1, np.int32)
        self.cell_key = np.zeros(n, np.uint32)
        self.cell_index = np.zeros(n, np.uint32)
        self.cell_start = np.zeros(NCELLS, np.uint32)
        self.cell_end = np.zeros(NCELLS, np.uint32)
        self.eos_forsterite = f32(eos_forsterite)
        self.eos_fe = f32(eos_fe)
        self.eos_res = int(eos_forsterite.shape[0])
        self.max_unchecked = max_unchecked
        self.tree = None
        self._st = OraState()
        self._fill()

    def _fill(self):
        s = self._st
        s.n = self.n
        for name in ("pos", "vel", "acc") + FLOAT_FIELDS:
            setattr(s, name, ptr(getattr(self, name), _fp))
        s.material = ptr(self.material, _ip)
        s.active = ptr(self.active, _bp)
        s.next_active_time = ptr(self.next_active_time, _ip)
        s.global_time = ptr(self.global_time, _ip)
        s.dt = ptr(self.dt, _ip)
        for name in ("cell_key", "cell_index", "cell_start", "cell_end"):
            setattr(s, name, ptr(getattr(self, name), _up))
        s.eos_forsterite = ptr(self.eos_forsterite, _fp)
        s.eos_fe = ptr(self.eos_fe, _fp)
        s.eos_res = self.eos_res
        s.max_unchecked = self.max_unchecked
        if self.tree is not None:
            t = self.tree
            s.tree = ptr(t["tree"], _ip)
            s.tree_len = int(t["tree"].shape[0])
            s.level_offsets = ptr(t["level_offsets"], _ip)
            s.level_nodes = ptr(t["level_nodes"], _ip)
            s.n_levels = int(t["n_levels"])
            s.n_nodes = int(t["n_nodes"])
        else:
            s.n_levels = 0
            s.tree_len = 0
            s.n_nodes = 0

    def set_tree(self, tree: dict):
        self.tree = {k: (np.ascontiguousarray(v, np.int32) if isinstance(v, np.ndarray) else v)
                     for k, v in tree.items()}
        self._fill()

    def _call(self, name):
        getattr(self.lib, f"{self.prefix}_{name}")(C.byref(self._st))

    def sort(self):
        self._call("sort")

    def gravity(self):
        self._call("gravity")

    def density(self):
        self._call("density")

    def acceleration(self):
        self._call("acceleration")

    def step(self):
        self._call("step")

    def full_step(self, tree_fn=None):
        """One global step in the reference's order (Headless.cpp:43-51), with
        the tree rebuilt from the current positions by `tree_fn` first."""
        if tree_fn is not None:
            self.set_tree(tree_fn(self.pos))
        self.sort()
        self.gravity()
        self.density()
        self.acceleration()
        self.step()

    def snapshot(self) -> dict:
        out = {k: getattr(self, k).copy() for k in ("pos", "vel", "acc") + FLOAT_FIELDS}
        for k in ("material", "active", "next_active_time", "global_time", "dt", "cell_key", "cell_index"):
            out[k] = getattr(self, k).copy()
        return out


def draw_snapshot(pos: np.ndarray, material: np.ndarray) -> np.ndarray:
    """render.metal:49-66 restated in numpy: each particle's (x, y) shifted
    by -250 Mm and scaled by 1024 / (20 R_E) in float32; inside [0, 1024] it
    takes pixel int(u) + (1023 - int(v)) * 1024 and the image keeps the
    largest material id per pixel.  Splats at exactly 1024 (one past the
    image in the reference) are dropped."""
    p = np.asarray(pos, np.float32).reshape(-1, 3)
    R_E = np.float32(6.3710)
    s = np.float32(1024) / (np.float32(20) * R_E)
    ux = (p[:, 0] - np.float32(250)) * s
    uy = (p[:, 1] - np.float32(250)) * s
    ok = (ux >= 0) & (uy >= 0) & (ux < 1024) & (uy < 1024)
    px = ux[ok].astype(np.int64) + (1023 - uy[ok].astype(np.int64)) * 1024
    img = np.zeros(1024 * 1024, np.int64)
    np.maximum.at(img, px, np.asarray(material).reshape(-1)[ok].astype(np.int64))
    return img.astype(np.int32).reshape(1024, 1024)


def draw_snapshot_ref(pos: np.ndarray, material: np.ndarray) -> np.ndarray:
    """The reference's drawToSnapshot (render.metal:49-66) over all
    particles into a cleared 1024 x 1024 int image (oracle/_ref)."""
    lib = load("ref")
    pos = np.ascontiguousarray(pos, np.float32).reshape(-1, 3)
    mat = np.ascontiguousarray(material, np.int32).reshape(-1)
    img = np.zeros((1024, 1024), np.int32)
    lib.ref_draw_snapshot(pos.shape[0], ptr(pos, _fp), ptr(mat, _ip), ptr(img, _ip))
    return img


def last_tree_nodes(n_nodes: int):
    """(poles [n, 24], locals [n, 16]) of the last oracle gravity pass."""
    lib = load("oracle")
    lib.ora_last_tree_nodes.argtypes = [_fp, _fp, C.c_int]
    lib.ora_last_tree_nodes.restype = C.c_int
    poles = np.zeros((n_nodes, 24), np.float32)
    locs = np.zeros((n_nodes, 16), np.float32)
    if lib.ora_last_tree_nodes(ptr(poles, _fp), ptr(locs, _fp), n_nodes) < 0:
        raise RuntimeError("no gravity pass with that many nodes")
    return poles, locs


class _F64(C.Structure):
    _dp = C.POINTER(C.c_double)
    _fields_ = [("n", C.c_int32)] + [(k, C.POINTER(C.c_double)) for k in (
        "pos", "vel", "acc", "rho", "u", "mass", "pressure", "h", "grad_term", "sound_speed", "du", "balsara",
        "dhdt")] + [("material", _ip), ("next_active_time", _ip), ("global_time", _ip), ("dt", _ip),
                    ("time_s", C.POINTER(C.c_double)), ("eos_forsterite", _fp), ("eos_fe", _fp),
                    ("eos_res", C.c_int32)]


class F64Run:
    """An all-FP64 run of the step from float initial conditions (fp64.cpp):
    FP64 direct-sum gravity and the reference's SPH passes in double."""

    FIELDS = ("pos", "vel", "acc", "rho", "u", "mass", "pressure", "h", "grad_term", "sound_speed", "du",
              "balsara", "dhdt")

    def __init__(self, ic: dict, eos_forsterite: np.ndarray, eos_fe: np.ndarray):
        lib = load("oracle")
        lib.ora_f64_steps.argtypes = [C.POINTER(_F64), C.c_int]
        lib.ora_f64_energy.argtypes = [C.POINTER(_F64), C.POINTER(C.c_double)]
        self.lib = lib
        n = int(np.asarray(ic["pos"]).reshape(-1, 3).shape[0])
        self.n = n
        d = lambda a, k=1: np.ascontiguousarray(np.asarray(a, np.float64).reshape(-1))  # noqa: E731
        self.a = {f: np.zeros(3 * n if f in ("pos", "vel", "acc") else n, np.float64) for f in self.FIELDS}
        for f in ("pos", "vel", "rho", "u", "mass", "pressure", "h"):
            self.a[f][:] = d(ic[f])
        self.material = np.ascontiguousarray(np.asarray(ic["material"], np.int32).reshape(-1))
        self.nat = np.zeros(n, np.int32)
        self.gt = np.zeros(1, np.int32)
        self.dt = np.zeros(1, np.int32)
        self.t = np.zeros(1, np.float64)
        self.eos = (np.ascontiguousarray(eos_forsterite, np.float32), np.ascontiguousarray(eos_fe, np.float32))
        s = _F64()
        s.n = n
        for f in self.FIELDS:
            setattr(s, f, self.a[f].ctypes.data_as(C.POINTER(C.c_double)))
        s.material = ptr(self.material, _ip)
        s.next_active_time = ptr(self.nat, _ip)
        s.global_time = ptr(self.gt, _ip)
        s.dt = ptr(self.dt, _ip)
        s.time_s = self.t.ctypes.data_as(C.POINTER(C.c_double))
        s.eos_forsterite = ptr(self.eos[0], _fp)
        s.eos_fe = ptr(self.eos[1], _fp)
        s.eos_res = int(round((self.eos[0].size // 2) ** 0.5))
        self.s = s

    def steps(self, k: int):
        self.lib.ora_f64_steps(C.byref(self.s), int(k))

    def energy(self) -> dict:
        out = (C.c_double * 4)()
        self.lib.ora_f64_energy(C.byref(self.s), out)
        return dict(kinetic=out[0], internal=out[1], potential=out[2], total=out[3])

    def field(self, f: str) -> np.ndarray:
        a = self.a[f]
        return a.reshape(-1, 3) if f in ("pos", "vel", "acc") else a

