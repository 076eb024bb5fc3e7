"""B200 (sm_100a) SPH + FMM planetary-impact step behind the reference's
Compute pass API.  The compute lives in libsph_b200.so (csrc/, C ABI in
include/sph.h); this package holds its ctypes binding (_lib), the Compute
mirror (compute), the seeded initial conditions (ic), the stand-in EOS
tables (eos_tables), the HDF5 initial-conditions reader (hdf5io), the
snapshot PNG writer (snapshot) and the ensemble's host side (ensemble)."""
from . import _lib, ensemble, eos_tables, hdf5io, ic, snapshot  # noqa: F401
from ._lib import SphError, build  # noqa: F401
from .compute import Compute, Ensemble, eos_resample  # noqa: F401

__all__ = ["Compute", "Ensemble", "SphError", "build", "eos_resample", "ic", "eos_tables", "ensemble", "hdf5io", "snapshot"]
