"""Seeded synthetic initial conditions for a two-body planetary impact.

The reference reads a SWIFT-style HDF5 snapshot (SPH/hdfHandler/hdfHandler.cpp:12-136;
datasets Coordinates, Velocities, Densities, InternalEnergies, Masses, MaterialIDs,
Pressures, SmoothingLengths).  No such file ships for the sizes measured here, so this
module builds the same fields from a seeded generator.

Code units follow the reference's constants: length 1 Mm, mass 1e24 kg, time 1 s
(G = 6.67e-5, SPH/Shaders/gravity/poles/poles.h:16), density 1e6 kg/m^3, specific
energy 1e12 J/kg.  Material ids: 400 forsterite (mantle), 402 Fe85Si15 (core)
(density.metal:50 picks the forsterite table for id 400, the iron table otherwise).

Each body is a sphere of equal-mass particles on cubic lattices with uniform +-10%
jitter of the spacing: a 30%-by-mass iron core of density 8000 kg/m^3 (the finer
lattice) inside a forsterite mantle of 3300 kg/m^3.  The target has one Earth mass
(5.97 code units); radii follow from the layer densities.  Specific internal energy
is 1.0e6 J/kg in the mantle and 1.5e6 J/kg in the core, and h = 1.2 x the local
lattice spacing.
"""
from __future__ import annotations

import math

import numpy as np

G = 6.67e-5
RHO_CORE = 8.0e-3
RHO_MANTLE = 3.3e-3
U_CORE = 1.5e-6
U_MANTLE = 1.0e-6
MAT_FORSTERITE = 400
MAT_FE85SI15 = 402
EARTH_MASS = 5.97
BOX_CENTRE = 637.1 / 2.0  # the demo snapshot's box is 637.1 Mm


def _lattice_shell(n: int, spacing: float, r_min: float, rng: np.random.Generator) -> np.ndarray:
    """The n jittered lattice points of the given spacing closest to the origin
    among those at radius >= r_min."""
    r_out = ((r_min ** 3) + 3.0 * n * spacing ** 3 / (4.0 * math.pi)) ** (1.0 / 3.0)
    k = int(math.ceil(r_out / spacing)) + 3
    ax = np.arange(-k, k + 1, dtype=np.float64)
    gx, gy, gz = np.meshgrid(ax, ax, ax, indexing="ij")
    pts = np.stack([gx.ravel(), gy.ravel(), gz.ravel()], axis=1) * spacing
    pts += rng.uniform(-0.1 * spacing, 0.1 * spacing, size=pts.shape)
    r = np.sqrt((pts * pts).sum(axis=1))
    keep = r >= r_min
    pts, r = pts[keep], r[keep]
    return pts[np.argsort(r, kind="stable")[:n]]


def _body(n: int, mass: float, core_frac: float, rng: np.random.Generator):
    """Equal-mass particles: the core lattice is finer than the mantle lattice by
    (rho_mantle / rho_core)^(1/3), so each particle carries mass / n."""
    m = mass / n
    n_core = int(round(core_frac * n))
    n_mantle = n - n_core
    r_core = (3.0 * n_core * m / (4.0 * math.pi * RHO_CORE)) ** (1.0 / 3.0)
    s_core = (m / RHO_CORE) ** (1.0 / 3.0)
    s_mantle = (m / RHO_MANTLE) ** (1.0 / 3.0)
    core = _lattice_shell(n_core, s_core, 0.0, rng)
    core = core[np.sqrt((core * core).sum(axis=1)) < r_core + 0.5 * s_core] if n_core else core
    core = core[:n_core]
    mantle = _lattice_shell(n_mantle, s_mantle, r_core, rng)
    pts = np.concatenate([core, mantle])
    is_core = np.arange(n) < core.shape[0]
    radius = (r_core ** 3 + 3.0 * n_mantle * m / (4.0 * math.pi * RHO_MANTLE)) ** (1.0 / 3.0)
    mat = np.where(is_core, MAT_FE85SI15, MAT_FORSTERITE).astype(np.int32)
    rho = np.where(is_core, RHO_CORE, RHO_MANTLE)
    u = np.where(is_core, U_CORE, U_MANTLE)
    h = np.where(is_core, 1.2 * s_core, 1.2 * s_mantle)
    return dict(pos=pts, mass=np.full(n, m), rho=rho, u=u, h=h, material=mat, radius=radius, spacing=s_mantle)


def make_impact(n_target: int = 16384, n_impactor: int = 4096, seed: int = 0, *,
                target_mass: float = EARTH_MASS, mass_ratio: float = 0.13,
                speed_factor: float = 1.1, angle_deg: float = 45.0,
                separation_radii: float = 2.0, core_frac: float = 0.3) -> dict:
    """Two bodies on a straight-line approach.

    The impactor starts `separation_radii` target radii from the target's centre
    with impact parameter (R_t + R_i) sin(angle) and relative speed
    `speed_factor` x the mutual escape speed sqrt(2 G (M_t + M_i) / (R_t + R_i)),
    in the centre-of-mass frame, shifted to the centre of a 637.1 Mm box.

    Returns float32/int32 arrays: pos (n,3), vel (n,3), mass, rho, u, pressure, h,
    material; plus scalar metadata.
    """
    rng = np.random.default_rng(seed)
    t = _body(n_target, target_mass, core_frac, rng)
    parts = [t]
    if n_impactor > 0:
        rng_i = np.random.default_rng(seed + 1)
        mi = mass_ratio * target_mass
        b = _body(n_impactor, mi, core_frac, rng_i)
        rsum = t["radius"] + b["radius"]
        v_esc = math.sqrt(2.0 * G * (target_mass + mi) / rsum)
        v_imp = speed_factor * v_esc
        d = separation_radii * t["radius"]
        bpar = rsum * math.sin(math.radians(angle_deg))
        x0 = math.sqrt(max(d * d - bpar * bpar, 0.0))
        rel = np.array([x0, bpar, 0.0])
        vrel = np.array([-v_imp, 0.0, 0.0])
        mt, mtot = target_mass, target_mass + mi
        t_pos = t["pos"] - (mi / mtot) * rel
        b_pos = b["pos"] + (mt / mtot) * rel
        t_vel = np.tile(-(mi / mtot) * vrel, (n_target, 1))
        b_vel = np.tile((mt / mtot) * vrel, (n_impactor, 1))
        parts = [dict(t, pos=t_pos, vel=t_vel), dict(b, pos=b_pos, vel=b_vel)]
    else:
        parts = [dict(t, vel=np.zeros_like(t["pos"]))]
    out = {}
    for key in ("pos", "vel", "mass", "rho", "u", "h", "material"):
        out[key] = np.concatenate([p[key] for p in parts])
    out["pos"] = out["pos"] + BOX_CENTRE
    n = out["mass"].shape[0]
    ic = dict(
        pos=np.ascontiguousarray(out["pos"], dtype=np.float32),
        vel=np.ascontiguousarray(out["vel"], dtype=np.float32),
        mass=out["mass"].astype(np.float32),
        rho=out["rho"].astype(np.float32),
        u=out["u"].astype(np.float32),
        pressure=np.zeros(n, dtype=np.float32),
        h=out["h"].astype(np.float32),
        material=out["material"].astype(np.int32),
    )
    ic["n"] = n
    ic["spacing_target"] = t["spacing"]
    return ic


def make_plummer(n: int, seed: int = 0, *, total_mass: float = EARTH_MASS, scale: float = 3.0) -> dict:
    """Plummer sphere of n equal-mass particles (seeded inverse-CDF radii,
    isotropic directions), at rest, centred in the box.  Gravity-only cases."""
    rng = np.random.default_rng(seed)
    x = rng.uniform(1e-6, 0.999, size=n)
    r = scale / np.sqrt(x ** (-2.0 / 3.0) - 1.0)
    cost = rng.uniform(-1.0, 1.0, size=n)
    phi = rng.uniform(0.0, 2.0 * math.pi, size=n)
    sint = np.sqrt(1.0 - cost * cost)
    pos = np.stack([r * sint * np.cos(phi), r * sint * np.sin(phi), r * cost], axis=1) + BOX_CENTRE
    return _equal_mass(pos, total_mass)


def make_cube(n: int, seed: int = 0, *, total_mass: float = EARTH_MASS, side: float = 10.0) -> dict:
    """Uniform-density cube of n equal-mass particles, centred in the box."""
    rng = np.random.default_rng(seed)
    pos = rng.uniform(-0.5 * side, 0.5 * side, size=(n, 3)) + BOX_CENTRE
    return _equal_mass(pos, total_mass)


def _equal_mass(pos: np.ndarray, total_mass: float) -> dict:
    n = pos.shape[0]
    return dict(
        n=n,
        pos=np.ascontiguousarray(pos, dtype=np.float32),
        vel=np.zeros((n, 3), dtype=np.float32),
        mass=np.full(n, total_mass / n, dtype=np.float32),
        rho=np.full(n, RHO_MANTLE, dtype=np.float32),
        u=np.full(n, U_MANTLE, dtype=np.float32),
        pressure=np.zeros(n, dtype=np.float32),
        h=np.full(n, 0.1, dtype=np.float32),
        material=np.full(n, MAT_FORSTERITE, dtype=np.int32),
    )
