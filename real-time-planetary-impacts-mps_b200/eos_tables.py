"""Synthetic equation-of-state tables in the reference's ANEOS text format.

The reference loads `ANEOS_forsterite_S19.txt` and `ANEOS_Fe85Si15_S20.txt`
(SPH/Compute/Compute.cpp:45-46); both files are absent from the reference
repository.  This module writes stand-in tables in the exact layout its loader
parses (SPH/ANEOS/ANEOS.cpp:21-116):

    13 header lines
    "<numRho> <numT>"
    numRho densities [kg/m^3] (several per line)
    numT temperatures [K] (several per line)
    numRho*numT lines "u[J/kg] p[Pa] c[m/s] s[J/kg/K]", density index fastest

The physics is a simple cold-compression + thermal model (not ANEOS):
    x = rho/rho0
    p_cold = K0 x ln(x) above rho0, 0 below     (logarithmic cold curve, no tension)
    e_cold = K0 ln(x)^2 / (2 rho0) above rho0, 0 below rho0
    u = cv T + e_cold,   p = p_cold + (gamma-1) rho cv T
    c^2 = K0 max(ln(x) + 1, 0.05) / rho0 + gamma (gamma-1) cv T
e_cold is non-decreasing in density, so u at fixed T is non-decreasing down each
temperature column; the reference's resampler relies on that to stay inside the
table (see the upper-row index note at ANEOS.cpp:158).  e_cold stays small enough
that u is strictly increasing in temperature even in float32, so no interpolation
denominator of the resampler is zero.
"""
from __future__ import annotations

import os
import tempfile

import numpy as np

MATERIALS = {
    # name: (rho0 kg/m^3, K0 Pa, cv J/kg/K, gamma)
    "forsterite": (3300.0, 1e9, 1000.0, 1.5),
    "Fe85Si15": (8000.0, 1e9, 450.0, 1.6),
}
FILENAMES = {"forsterite": "ANEOS_forsterite_S19.txt", "Fe85Si15": "ANEOS_Fe85Si15_S20.txt"}


def table_values(material: str, n_rho: int = 96, n_t: int = 96):
    rho0, k0, cv, gam = MATERIALS[material]
    rho = np.logspace(np.log10(0.5), np.log10(2.0e6), n_rho)
    temp = np.logspace(1.0, np.log10(3.0e9), n_t)
    x = rho / rho0
    lnx = np.log(x)
    p_cold = np.where(x > 1.0, k0 * x * lnx, 0.0)
    e_cold = np.where(x > 1.0, k0 * lnx * lnx / (2.0 * rho0), 0.0)
    R, T = np.meshgrid(rho, temp, indexing="ij")  # [rho, T]
    X = R / rho0
    PC = np.broadcast_to(p_cold[:, None], R.shape)
    EC = np.broadcast_to(e_cold[:, None], R.shape)
    u = cv * T + EC
    p = PC + (gam - 1.0) * R * cv * T
    c2 = k0 * np.maximum(np.log(X) + 1.0, 0.05) / rho0 + gam * (gam - 1.0) * cv * T
    c = np.sqrt(np.maximum(c2, 1.0))
    s = cv * np.log(np.maximum(T, 1.0))
    return rho, temp, u, p, c, s


def write_table(path: str, material: str, n_rho: int = 96, n_t: int = 96) -> str:
    rho, temp, u, p, c, s = table_values(material, n_rho, n_t)
    lines = [f"# synthetic stand-in table for {material} (logarithmic cold curve, K0 = 1e9 Pa, + thermal ideal gas)"]
    lines += [f"# header line {i}" for i in range(2, 14)]
    lines.append(f"{n_rho} {n_t}")
    for vals in (rho, temp):
        for k in range(0, len(vals), 5):
            lines.append(" ".join(f"{v:.8e}" for v in vals[k:k + 5]))
    for ti in range(n_t):
        for ri in range(n_rho):
            lines.append(f"{u[ri, ti]:.8e} {p[ri, ti]:.8e} {c[ri, ti]:.8e} {s[ri, ti]:.8e}")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")
    return path


def ensure_tables(directory: str | None = None) -> dict:
    """Write both stand-in tables (once) and return {material: path}."""
    if directory is None:
        directory = os.path.join(tempfile.gettempdir(), "sph_b200_eos")
    os.makedirs(directory, exist_ok=True)
    out = {}
    for mat, fname in FILENAMES.items():
        path = os.path.join(directory, fname)
        if not os.path.exists(path):
            tmp = path + f".{os.getpid()}.tmp"
            write_table(tmp, mat)
            os.replace(tmp, path)
        out[mat] = path
    return out
