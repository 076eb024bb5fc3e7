"""Host-side mirror of the reference's pass API, class Compute
(SPH/Compute/Compute.hpp:40-59), over the C ABI of libsph_b200.so.

    Compute(ic, ...)        Compute::Compute (Compute.cpp:22-36)
    updateOctreeBuffer()    Compute::updateOctreeBuffer (:456-508), GPU build
    sort()                  Compute::sort (:265-326)
    gravitationalPass()     Compute::gravitationalPass (:328-377)
    densityPass()           Compute::densityPass (:179-208)
    accelerationPass()      Compute::accelerationPass (:210-240)
    stepPass()              Compute::stepPass (:242-263)
    drawSnapshot()          Compute::drawSnapshot (:396-448)
    positionBuffer, materialIdBuffer, densityBuffer, nParticles  (public members)

Each pass takes an optional CUDA stream (an int cudaStream_t, or an object with
a `cuda_stream` attribute such as torch.cuda.Stream) in place of the
reference's MTL::CommandBuffer; passes are asynchronous until synchronize().
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import _lib
from . import eos_tables

_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int32)


def _stream(s) -> C.c_void_p:
    if s is None:
        return C.c_void_p(0)
    if hasattr(s, "cuda_stream"):
        return C.c_void_p(int(s.cuda_stream))
    return C.c_void_p(int(s))


def _ptr(a: np.ndarray, t):
    return a.ctypes.data_as(t)


def _tables(forsterite_table, fe85si15_table):
    if forsterite_table is None or fe85si15_table is None:
        tabs = eos_tables.ensure_tables()
        forsterite_table = forsterite_table or tabs["forsterite"]
        fe85si15_table = fe85si15_table or tabs["Fe85Si15"]
    if not os.path.exists(forsterite_table) or not os.path.exists(fe85si15_table):
        raise FileNotFoundError("ANEOS tables not found")
    return forsterite_table.encode(), fe85si15_table.encode()


def _params(lib, paths, max_children_in_leaf, max_tree_depth, max_unchecked_pointers, aneos_resolution,
            tree_source) -> "_lib.SphParams":
    p = _lib.SphParams()
    lib.sph_params_default(C.byref(p))
    p.max_children_in_leaf = max_children_in_leaf
    p.max_tree_depth = max_tree_depth
    p.max_unchecked_pointers = max_unchecked_pointers
    p.aneos_resolution = aneos_resolution
    p.tree_source = _lib.SPH_TREE_GPU if tree_source == "gpu" else _lib.SPH_TREE_HOST
    p.forsterite_table = paths[0]
    p.fe85si15_table = paths[1]
    return p


def _ic_struct(ic: dict):
    """(SphIC, the arrays it points into -- keep them alive while it is used)."""
    n = int(np.asarray(ic["pos"]).reshape(-1, 3).shape[0])
    f32 = lambda a: np.ascontiguousarray(np.asarray(a, dtype=np.float32).reshape(-1))  # noqa: E731
    keep = dict(pos=f32(ic["pos"]), vel=f32(ic["vel"]), rho=f32(ic["rho"]), u=f32(ic["u"]),
                mass=f32(ic["mass"]), pressure=f32(ic.get("pressure", np.zeros(n))), h=f32(ic["h"]),
                material=np.ascontiguousarray(np.asarray(ic["material"], dtype=np.int32).reshape(-1)))
    s = _lib.SphIC()
    s.n = n
    for k in ("pos", "vel", "rho", "u", "mass", "pressure", "h"):
        setattr(s, k, _ptr(keep[k], _fp))
    s.material = _ptr(keep["material"], _ip)
    return s, keep


def _form(lib, gravity: str = "reference", theta: float = 0.5, precision: str = "reference",
          h_seed: str = "plain", h_tolerance: float = 0.0, timestep: str = "global") -> "_lib.SphForm":
    f = _lib.SphForm()
    lib.sph_form_default(C.byref(f))
    f.gravity = _lib.SPH_GRAVITY_THETA if gravity == "theta" else _lib.SPH_GRAVITY_REFERENCE
    f.theta = float(theta)
    f.precision = _lib.SPH_PRECISION_MIXED if precision == "mixed" else _lib.SPH_PRECISION_REFERENCE
    f.h_seed = _lib.SPH_HSEED_LEARNED if h_seed == "learned" else _lib.SPH_HSEED_PLAIN
    f.h_tolerance = float(h_tolerance)
    if timestep not in ("global", "individual"):
        raise ValueError(f"timestep must be 'global' or 'individual', not {timestep!r}")
    f.timestep = 1 if timestep == "individual" else 0
    return f


class Compute:
    """One simulation on the current CUDA device."""

    def __init__(self, ic: dict, *, max_children_in_leaf: int = 4, max_tree_depth: int = 7,
                 max_unchecked_pointers: int = 1024, aneos_resolution: int = 2048,
                 tree_source: str = "gpu", forsterite_table: str | None = None,
                 fe85si15_table: str | None = None, parity: bool = False):
        # parity=True runs the parity build (no FMA contraction, sums in the
        # reference's sequential order); only tests use it
        lib = _lib.load(parity)
        self._lib = lib
        self._paths = _tables(forsterite_table, fe85si15_table)
        p = _params(lib, self._paths, max_children_in_leaf, max_tree_depth, max_unchecked_pointers,
                    aneos_resolution, tree_source)
        s, keep = _ic_struct(ic)
        n = s.n
        self._params_tuple = (max_children_in_leaf, max_tree_depth, max_unchecked_pointers, aneos_resolution)
        h = C.c_void_p()
        _lib.check(lib.sph_create(C.byref(p), C.byref(s), C.byref(h)), "sph_create", lib)
        self._lib = lib
        self._h = h
        self._owned = True
        self.nParticles = n
        self.tree_source = tree_source

    @classmethod
    def _borrow(cls, lib, handle: C.c_void_p, tree_source: str = "gpu") -> "Compute":
        """A Compute over a context another object owns (an ensemble
        instance); closing it does not destroy the context."""
        c = cls.__new__(cls)
        c._lib = lib
        c._h = handle
        c._owned = False
        c.nParticles = int(lib.sph_num_particles(handle))
        c.tree_source = tree_source
        return c

    def _check(self, status: int, what: str):
        _lib.check(status, what, self._lib)

    # ---- lifetime ------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            if getattr(self, "_owned", True):
                self._lib.sph_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---- passes (Headless.cpp:43-51 order) -----------------------------
    def updateOctreeBuffer(self, stream=None):
        self._check(self._lib.sph_update_tree(self._h, _stream(stream)), "sph_update_tree")

    def sort(self, stream=None):
        self._check(self._lib.sph_sort(self._h, _stream(stream)), "sph_sort")

    def gravitationalPass(self, stream=None):
        self._check(self._lib.sph_gravity(self._h, _stream(stream)), "sph_gravity")

    def densityPass(self, stream=None):
        self._check(self._lib.sph_density(self._h, _stream(stream)), "sph_density")

    def accelerationPass(self, stream=None):
        self._check(self._lib.sph_acceleration(self._h, _stream(stream)), "sph_acceleration")

    def stepPass(self, stream=None):
        self._check(self._lib.sph_step(self._h, _stream(stream)), "sph_step")

    def drawSnapshot(self, stream=None, download: bool = True):
        if not download:
            self._check(self._lib.sph_draw_snapshot(self._h, _stream(stream), None), "sph_draw_snapshot")
            return None
        img = np.zeros((1024, 1024), np.int32)
        self._check(self._lib.sph_draw_snapshot(self._h, _stream(stream), _ptr(img, _ip)), "sph_draw_snapshot")
        return img

    def step(self, stream=None):
        """One Headless::step without the snapshot: tree, sort, gravity,
        density, acceleration, step."""
        self.updateOctreeBuffer(stream)
        self.sort(stream)
        self.gravitationalPass(stream)
        self.densityPass(stream)
        self.accelerationPass(stream)
        self.stepPass(stream)

    def step_all(self, n_steps: int, stream=None):
        """n_steps full steps replayed from a captured CUDA graph."""
        self._check(self._lib.sph_step_all(self._h, _stream(stream), int(n_steps)), "sph_step_all")

    def synchronize(self, stream=None):
        self._check(self._lib.sph_synchronize(self._h, _stream(stream)), "sph_synchronize")

    # ---- trees ---------------------------------------------------------
    def set_tree(self, tree: dict):
        """Give a host-built tree in the reference format (see oracle/oracle.py
        tree_reference); later gravity passes use it until the next call."""
        t = np.ascontiguousarray(tree["tree"], np.int32)
        off = np.ascontiguousarray(tree["level_offsets"], np.int32)
        nodes = np.ascontiguousarray(tree["level_nodes"], np.int32)
        self._check(self._lib.sph_set_tree(self._h, _ptr(t, _ip), int(t.shape[0]), _ptr(off, _ip),
                                          _ptr(nodes, _ip), int(tree["n_levels"]), int(tree["n_nodes"])),
                   "sph_set_tree")
        self.tree_source = "host"

    def get_tree(self) -> dict:
        """The current tree in the reference format (synchronous)."""
        ln, nl, nn = C.c_int32(), C.c_int32(), C.c_int32()
        self._check(self._lib.sph_get_tree(self._h, None, 0, C.byref(ln), None, None, 0, C.byref(nl), C.byref(nn)),
                   "sph_get_tree")
        tree = np.zeros(max(ln.value, 1), np.int32)
        off = np.zeros(17, np.int32)
        nodes = np.zeros(max(nn.value, 1), np.int32)
        self._check(self._lib.sph_get_tree(self._h, _ptr(tree, _ip), tree.size, C.byref(ln), _ptr(off, _ip),
                                          _ptr(nodes, _ip), nodes.size, C.byref(nl), C.byref(nn)), "sph_get_tree")
        return dict(tree=tree[:ln.value], level_offsets=off[:nl.value + 1], level_nodes=nodes[:off[nl.value]],
                    n_levels=nl.value, n_nodes=nn.value)

    # ---- numerical forms (no reference counterpart) --------------------
    def set_form(self, gravity: str = "reference", theta: float = 0.5, precision: str = "reference",
                 h_seed: str = "plain", h_tolerance: float = 0.0, timestep: str = "global"):
        """Select the numerical form: gravity "reference" (the reference's
        logic) or "theta" (opening-angle group walk with exact near field);
        precision "reference" (float positions) or "mixed" (FP64 master
        positions and time, Kahan-compensated sums); h_seed "plain" or
        "learned" (the trained MLP starts the density iteration);
        h_tolerance of the density iteration (0 = the reference's 0.005);
        timestep "global" (the reference's active test as shipped: every
        particle every step) or "individual" (particles active only when their
        next active time is reached, README.md:60-64)."""
        f = _form(self._lib, gravity, theta, precision, h_seed, h_tolerance, timestep)
        self._check(self._lib.sph_set_form(self._h, C.byref(f)), "sph_set_form")

    def get_form(self) -> dict:
        f = _lib.SphForm()
        self._check(self._lib.sph_get_form(self._h, C.byref(f)), "sph_get_form")
        return dict(gravity="theta" if f.gravity == _lib.SPH_GRAVITY_THETA else "reference", theta=f.theta,
                    precision="mixed" if f.precision == _lib.SPH_PRECISION_MIXED else "reference",
                    h_seed="learned" if f.h_seed == _lib.SPH_HSEED_LEARNED else "plain", h_tolerance=f.h_tolerance,
                    timestep="individual" if f.timestep == 1 else "global")

    def set_tiling(self, big_max: int | None = None, block_max: int | None = None, half_max: int | None = None,
                   coarse: bool | None = None):
        """Scheduling of the density and acceleration passes (sph_set_tiling):
        tile sizes in particles, and whether particles whose neighbour boxes
        reach past 3 cells run in coarse tiles (True) or in the per-particle
        walk (False).  Arguments left at None keep their current value."""
        t = _lib.SphTiling()
        self._check(self._lib.sph_get_tiling(self._h, C.byref(t)), "sph_get_tiling")
        if big_max is not None:
            t.big_max = int(big_max)
        if block_max is not None:
            t.block_max = int(block_max)
        if half_max is not None:
            t.half_max = int(half_max)
        if coarse is not None:
            t.coarse = 1 if coarse else 0
        self._check(self._lib.sph_set_tiling(self._h, C.byref(t)), "sph_set_tiling")

    def get_tiling(self) -> dict:
        t = _lib.SphTiling()
        self._check(self._lib.sph_get_tiling(self._h, C.byref(t)), "sph_get_tiling")
        return dict(big_max=t.big_max, block_max=t.block_max, half_max=t.half_max, coarse=bool(t.coarse))

    # ---- learned smoothing-length seed (no reference counterpart) ------
    def hseed_capture(self, on: bool = True):
        """Record (features, converged h) of every following density pass."""
        self._check(self._lib.sph_hseed_capture(self._h, 1 if on else 0), "sph_hseed_capture")

    def hseed_train(self, iterations: int, batch: int = 16384, lr: float = 1e-3, stream=None) -> float:
        """Adam steps on the recorded pass; returns the last minibatch loss."""
        loss = C.c_float()
        self._check(self._lib.sph_hseed_train(self._h, int(iterations), int(batch), float(lr), C.byref(loss),
                                              _stream(stream)), "sph_hseed_train")
        return loss.value

    def hseed_online(self, iterations: int, batch: int = 16384, lr: float = 1e-3):
        """Online refresh of the learned seed (sph_hseed_online): every
        density pass records its pairs and each step first takes `iterations`
        Adam steps on the previous pass's (beside the tree, sort and gravity
        passes in graph-replayed steps).  0 turns it off."""
        self._check(self._lib.sph_hseed_online(self._h, int(iterations), int(batch), float(lr)), "sph_hseed_online")

    def hseed_gradient(self, batch: int, salt: int, stream=None):
        """(gradient, loss) of one minibatch, weights unchanged."""
        g = np.zeros(self._lib.sph_hseed_num_params(), np.float32)
        loss = C.c_float()
        self._check(self._lib.sph_hseed_gradient(self._h, int(batch), int(salt) & 0xFFFFFFFF, _ptr(g, _fp),
                                                 C.byref(loss), _stream(stream)), "sph_hseed_gradient")
        return g, loss.value

    def hseed_params(self, set_to=None) -> np.ndarray:
        """The FP32 weights (after setting them to `set_to` when given)."""
        if set_to is not None:
            w = np.ascontiguousarray(np.asarray(set_to, np.float32))
            self._check(self._lib.sph_hseed_params(self._h, None, _ptr(w, _fp)), "sph_hseed_params")
        out = np.zeros(self._lib.sph_hseed_num_params(), np.float32)
        self._check(self._lib.sph_hseed_params(self._h, _ptr(out, _fp), None), "sph_hseed_params")
        return out

    def hseed_norm(self, set_to=None) -> np.ndarray:
        """The network's standardisation (18 floats; after setting it to
        `set_to` when given)."""
        if set_to is not None:
            w = np.ascontiguousarray(np.asarray(set_to, np.float32))
            self._check(self._lib.sph_hseed_norm(self._h, None, _ptr(w, _fp)), "sph_hseed_norm")
        out = np.zeros(18, np.float32)
        self._check(self._lib.sph_hseed_norm(self._h, _ptr(out, _fp), None), "sph_hseed_norm")
        return out

    def hseed_dataset(self):
        """(features [n, 8], targets [n], standardisation [18]) of the recorded pass."""
        n = self.nParticles
        X = np.zeros((n, 8), np.float32)
        y = np.zeros(n, np.float32)
        norm = np.zeros(18, np.float32)
        self._check(self._lib.sph_hseed_dataset(self._h, _ptr(X, _fp), _ptr(y, _fp), _ptr(norm, _fp)),
                    "sph_hseed_dataset")
        return X, y, norm

    def hseed_stats(self) -> dict:
        """Counters of the last density pass's h iteration."""
        st = _lib.SphHSeedStats()
        self._check(self._lib.sph_hseed_get_stats(self._h, C.byref(st)), "sph_hseed_get_stats")
        return dict(sweeps=st.sweeps, fallbacks=st.fallbacks, max_sweeps=st.max_sweeps, particles=st.particles,
                    tiles=st.tiles, deferred=st.deferred, accel_deferred=st.accel_deferred,
                    coarse_tiles=st.coarse_tiles, accel_coarse_tiles=st.accel_coarse_tiles)

    def diagnostics(self, stream=None, theta_potential: float = 0.5) -> dict:
        """FP64 conservation sums (mass, energies, momentum, angular momentum)."""
        d = _lib.SphDiag()
        self._check(self._lib.sph_diagnostics(self._h, _stream(stream), float(theta_potential), C.byref(d)),
                    "sph_diagnostics")
        return dict(mass=d.mass, kinetic=d.kinetic, internal=d.internal, potential=d.potential, total=d.total,
                    momentum=list(d.momentum), angular_momentum=list(d.angular_momentum), time=d.time,
                    potential_valid=bool(d.potential_valid), health=d.health)

    def gravity_direct_f64(self, targets, stream=None) -> np.ndarray:
        """FP64 direct-sum (ax, ay, az, phi) at the given particles, G included."""
        t = np.ascontiguousarray(np.asarray(targets, np.int32).reshape(-1))
        out = np.zeros((t.size, 4), np.float64)
        self._check(self._lib.sph_gravity_direct_f64(self._h, _ptr(t, _ip), int(t.size),
                                                    out.ctypes.data_as(C.POINTER(C.c_double)), _stream(stream)),
                   "sph_gravity_direct_f64")
        return out

    def get_tree_nodes(self, n_nodes: int):
        """(poles [n, 24], locals [n, 16]) of the last gravity pass, by data pointer."""
        poles = np.zeros((n_nodes, 24), np.float32)
        locs = np.zeros((n_nodes, 16), np.float32)
        self._check(self._lib.sph_get_tree_nodes(self._h, _ptr(poles, _fp), _ptr(locs, _fp), int(n_nodes)),
                   "sph_get_tree_nodes")
        return poles, locs

    # ---- buffers (Buffers.hpp:14-59) -------------------------------------
    def download(self, field: str) -> np.ndarray:
        n = self.nParticles
        if field in _lib.VECTOR_FIELDS:
            out = np.zeros((n, 3), np.float32)
        elif field == "pos64":
            out = np.zeros((n, 3), np.float64)
        elif field in ("global_time", "dt"):
            out = np.zeros(1, np.int32)
        elif field in ("material", "next_active_time"):
            out = np.zeros(n, np.int32)
        elif field == "active":
            out = np.zeros(n, np.uint8)
        elif field in ("cell_key", "cell_index"):
            out = np.zeros(n, np.uint32)
        elif field in ("cell_start", "cell_end"):
            out = np.zeros(1 << 24, np.uint32)
        else:
            out = np.zeros(n, np.float32)
        self._check(self._lib.sph_download(self._h, _lib.FIELDS[field], out.ctypes.data_as(C.c_void_p), out.size),
                   f"sph_download({field})")
        return out

    def upload(self, field: str, values) -> None:
        if field in _lib.VECTOR_FIELDS:
            a = np.ascontiguousarray(np.asarray(values, np.float32).reshape(-1))
        elif field == "pos64":
            a = np.ascontiguousarray(np.asarray(values, np.float64).reshape(-1))
        elif field in ("global_time", "dt", "material", "next_active_time"):
            a = np.ascontiguousarray(np.asarray(values, np.int32).reshape(-1))
        elif field == "active":
            a = np.ascontiguousarray(np.asarray(values, np.uint8).reshape(-1))
        else:
            a = np.ascontiguousarray(np.asarray(values, np.float32).reshape(-1))
        self._check(self._lib.sph_upload(self._h, _lib.FIELDS[field], a.ctypes.data_as(C.c_void_p), a.size),
                   f"sph_upload({field})")

    def upload_async(self, field: str, values: np.ndarray, stream=None) -> None:
        """Stream-ordered upload from a caller-held host array (pinned for
        overlap); the array must stay alive until the stream reaches the copy."""
        if not values.flags.c_contiguous:
            raise ValueError("upload_async needs a C-contiguous array")
        self._check(self._lib.sph_upload_async(self._h, _lib.FIELDS[field], values.ctypes.data_as(C.c_void_p),
                                              values.size, _stream(stream)), f"sph_upload_async({field})")

    def download_async(self, field: str, out: np.ndarray, stream=None) -> None:
        """Stream-ordered download into a caller-held host array (pinned for
        overlap); valid once the stream has been synchronised."""
        if not out.flags.c_contiguous:
            raise ValueError("download_async needs a C-contiguous array")
        self._check(self._lib.sph_download_async(self._h, _lib.FIELDS[field], out.ctypes.data_as(C.c_void_p),
                                                out.size, _stream(stream)), f"sph_download_async({field})")

    # the layout each field of step_host takes: (elements per particle, dtype)
    _HOST_STATE = {"pos64": (3, np.float64), "pos": (3, np.float32), "vel": (3, np.float32), "u": (1, np.float32),
                   "h": (1, np.float32), "rho": (1, np.float32)}

    def step_host(self, inputs: dict, outputs: dict, stream=None) -> None:
        """One full step with the state moving through host memory
        (sph_step_host): the arrays of `inputs` are copied in at its start and
        those of `outputs` filled at its end, asynchronously on `stream`.
        Fields: pos64 (mixed-precision form) or pos, vel, u, h, rho, in
        sph_upload's layouts; the arrays must be page-locked (e.g. numpy views
        of pinned torch tensors) and stay alive until the stream passes the
        step.  The first call with a set of arrays runs eagerly and captures
        a graph that later calls with the same arrays replay."""
        structs = []
        for d in (inputs, outputs):
            hs = _lib.SphHostState()
            for name, a in d.items():
                if name not in self._HOST_STATE:
                    raise KeyError(f"step_host: unknown field {name!r}")
                per, dt = self._HOST_STATE[name]
                want = per * self.nParticles
                if a.dtype != dt or not a.flags.c_contiguous or a.size != want:
                    raise ValueError(f"step_host: {name} needs {want} contiguous {np.dtype(dt).name}")
                setattr(hs, name, a.ctypes.data)
            structs.append(hs)
        self._check(self._lib.sph_step_host(self._h, C.byref(structs[0]), C.byref(structs[1]), _stream(stream)),
                    "sph_step_host")

    def device_buffer(self, field: str):
        """(device pointer, bytes, stride) of a field's storage."""
        p, b, s = C.c_void_p(), C.c_size_t(), C.c_size_t()
        self._check(self._lib.sph_get_buffer(self._h, _lib.FIELDS[field], C.byref(p), C.byref(b), C.byref(s)),
                   "sph_get_buffer")
        return p.value, b.value, s.value

    @property
    def positionBuffer(self):
        return self.device_buffer("pos")

    @property
    def materialIdBuffer(self):
        return self.device_buffer("material")

    @property
    def densityBuffer(self):
        return self.device_buffer("rho")

    def health(self) -> int:
        w = C.c_uint32()
        self._check(self._lib.sph_get_health(self._h, C.byref(w)), "sph_get_health")
        return w.value

    def clear_health(self):
        self._check(self._lib.sph_clear_health(self._h), "sph_clear_health")

    # ---- checkpoint / resume (the reference has no resume) --------------
    CHECKPOINT_FIELDS = ("pos", "vel", "acc", "rho", "u", "mass", "pressure", "h", "grad_term", "sound_speed",
                         "du", "balsara", "dhdt", "grav_norm", "material", "active", "next_active_time",
                         "global_time", "dt")

    def checkpoint(self, path: str):
        """Write the whole simulation state to `path` (numpy .npz): every
        per-particle field in the original order, the global time and dt,
        the numerical form, the FP64 positions of the mixed form and the
        learned seed's weights and standardisation (not its Adam moments, so
        further training restarts them).  Synchronous.  resume() continues
        from it with the same results as a run that was never stopped."""
        self.synchronize()
        out = {f: self.download(f) for f in self.CHECKPOINT_FIELDS}
        form = self.get_form()
        out["form"] = np.array([form["gravity"], str(form["theta"]), form["precision"], form["h_seed"],
                                str(form["h_tolerance"]), form["timestep"]])
        out["tree_source"] = np.array([self.tree_source])
        out["params"] = np.array(self._params_tuple, np.int64)
        if form["precision"] == "mixed":
            out["pos64"] = self.download("pos64")
        if form["h_seed"] == "learned":
            out["hseed_params"] = self.hseed_params()
            out["hseed_norm"] = self.hseed_norm()
            out["neighbours"] = self.download("neighbours")
        np.savez(path, **out)

    @classmethod
    def resume(cls, path: str, *, forsterite_table: str | None = None, fe85si15_table: str | None = None,
               parity: bool = False) -> "Compute":
        """A context in the state written by checkpoint(path)."""
        with np.load(path) as z:
            ck = {k: z[k] for k in z.files}
        leaf, depth, unchecked, res = (int(v) for v in ck["params"])
        ic = {k: ck[k] for k in ("pos", "vel", "rho", "u", "mass", "pressure", "h", "material")}
        c = cls(ic, max_children_in_leaf=leaf, max_tree_depth=depth, max_unchecked_pointers=unchecked,
                aneos_resolution=res, tree_source=str(ck["tree_source"][0]), forsterite_table=forsterite_table,
                fe85si15_table=fe85si15_table, parity=parity)
        g, th, prec, seed, tol, ts = (str(v) for v in ck["form"])
        if "hseed_params" in ck:
            c.hseed_params(ck["hseed_params"])
            c.hseed_norm(ck["hseed_norm"])
            c.upload("neighbours", ck["neighbours"])
        c.set_form(gravity=g, theta=float(th), precision=prec, h_seed=seed, h_tolerance=float(tol), timestep=ts)
        for f in cls.CHECKPOINT_FIELDS:
            if f not in ic:
                c.upload(f, ck[f])
        if "pos64" in ck:
            c.upload("pos64", ck["pos64"])
        c.synchronize()
        return c

    def state(self) -> dict:
        names = ("pos", "vel", "acc", "rho", "u", "mass", "pressure", "h", "grad_term", "sound_speed", "du",
                 "balsara", "dhdt", "grav_norm", "material", "active", "next_active_time", "global_time", "dt")
        return {k: self.download(k) for k in names}


class Ensemble:
    """Many independent impacts advanced together on the current device
    (sph_ensemble_*; no counterpart in the reference).  `forms` holds one
    set_form keyword dict per instance (or None: the defaults); autotune picks
    each instance's tile size and, for the theta form, its leaf capacity.
    `instances` are Compute views of the instances' contexts."""

    def __init__(self, ics: list, forms: list | None = None, *, autotune: bool = False,
                 max_children_in_leaf: int = 32, max_tree_depth: int = 7, max_unchecked_pointers: int = 1024,
                 aneos_resolution: int = 2048, tree_source: str = "gpu", forsterite_table: str | None = None,
                 fe85si15_table: str | None = None):
        lib = _lib.load()
        self._lib = lib
        self._paths = _tables(forsterite_table, fe85si15_table)
        p = _params(lib, self._paths, max_children_in_leaf, max_tree_depth, max_unchecked_pointers,
                    aneos_resolution, tree_source)
        k = len(ics)
        structs = (_lib.SphIC * k)()
        keep = []
        for i, ic in enumerate(ics):
            s, arrays = _ic_struct(ic)
            structs[i] = s
            keep.append(arrays)
        fa = None
        if forms is not None:
            fa = (_lib.SphForm * k)()
            for i, f in enumerate(forms):
                fa[i] = _form(lib, **(f or {}))
        h = C.c_void_p()
        _lib.check(lib.sph_ensemble_create(C.byref(p), k, structs, fa, 1 if autotune else 0, C.byref(h)),
                   "sph_ensemble_create", lib)
        self._h = h
        self.instances = []
        for i in range(k):
            c = C.c_void_p()
            _lib.check(lib.sph_ensemble_instance(h, i, C.byref(c)), "sph_ensemble_instance", lib)
            self.instances.append(Compute._borrow(lib, c, tree_source))
        self.sizes = [c.nParticles for c in self.instances]

    def __len__(self):
        return len(self.instances)

    def step(self, n_steps: int = 1, stream=None):
        _lib.check(self._lib.sph_ensemble_step(self._h, _stream(stream), int(n_steps)), "sph_ensemble_step",
                   self._lib)

    def synchronize(self, stream=None):
        _lib.check(self._lib.sph_ensemble_synchronize(self._h, _stream(stream)), "sph_ensemble_synchronize",
                   self._lib)

    def tuning(self) -> list:
        out = []
        for i in range(len(self.instances)):
            t = _lib.SphEnsembleTuning()
            _lib.check(self._lib.sph_ensemble_get_tuning(self._h, i, C.byref(t)), "sph_ensemble_get_tuning",
                       self._lib)
            out.append(dict(max_children_in_leaf=t.max_children_in_leaf, tile_block_max=t.tile_block_max,
                            ms_per_step=t.ms_per_step, gravity_median_error=t.gravity_median_error))
        return out

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            for c in self.instances:
                c.close()
            self._lib.sph_ensemble_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def eos_resample(path: str, res: int = 2048) -> np.ndarray:
    """The library's host-side ANEOS resampler (no GPU work)."""
    out = np.zeros((res, res, 2), np.float32)
    _lib.check(_lib.load().sph_eos_resample(path.encode(), res, _ptr(out, _fp)), "sph_eos_resample")
    return out
