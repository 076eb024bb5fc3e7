"""The allocation-free cell sort, sph_sort_cells_noalloc.

It exists for callers that may not allocate device memory themselves: code
running inside a framework that owns every device allocation, or code on a
latency-critical thread that must not call cudaMalloc/cudaFree because those
can synchronise the device.  It must give exactly the sorted (cell key,
particle index) pairs of the context-based sph_sort, call after call, even
though every call reuses the same fixed scratch array inside the library: at
the largest size the scratch allows, at sizes that end in a partial tile, and
for a small call that follows a large one (nothing left over from the large
call may leak into the small call's result).  A look-back wait that gives up
must come back as an error through sph_sort_cells_noalloc_health.

This file is collected last on purpose, so a run that stops at the first
failure has already run every other test; it also passes on its own in a
fresh process.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_N = 262144  # SPH_SORT_NOALLOC_MAX_N in include/sph.h
SPH_ERR_TIMEOUT = 6


def _call(lib, dpos, n, keys, idx, stream):
    return lib.sph_sort_cells_noalloc(C.c_void_p(dpos.data_ptr()), int(n), C.c_void_p(keys.data_ptr()),
                                      C.c_void_p(idx.data_ptr()), C.c_void_p(stream.cuda_stream))


def _health(lib, stream):
    w = C.c_uint32(0)
    rc = lib.sph_sort_cells_noalloc_health(C.c_void_p(stream.cuda_stream), C.byref(w))
    return rc, w.value


def _sph_sort(pkg, ic):
    """The context-based sort (sph_sort) of the same positions."""
    with pkg.Compute(ic, tree_source="host") as c:
        c.sort()
        c.synchronize()
        return c.download("cell_key"), c.download("cell_index")


def _noalloc(lib, pos, n, stream):
    import torch
    dpos = torch.from_numpy(np.ascontiguousarray(pos[:n], dtype=np.float32).reshape(-1)).cuda()
    keys = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    idx = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    assert _call(lib, dpos, n, keys, idx, stream) == 0, lib.sph_last_error()
    rc, w = _health(lib, stream)
    assert rc == 0 and w == 0, (rc, hex(w))
    return keys.cpu().numpy().view(np.uint32), idx.cpu().numpy().view(np.uint32)


def _sub_ic(ic, n):
    out = {k: (v[:n] if isinstance(v, np.ndarray) else v) for k, v in ic.items()}
    out["n"] = n
    return out


def test_noalloc_sort_matches_sph_sort_on_two_calls_in_a_row(cuda, pkg):
    import torch

    lib = pkg._lib.load()
    ic = pkg.ic.make_impact(16384, 4096, seed=0)
    n = int(ic["n"])
    stream = torch.cuda.current_stream()
    # the second call sees other cells
    for p in (ic["pos"], ic["pos"] + np.float32(0.37)):
        wk, wi = _sph_sort(pkg, dict(ic, pos=p))
        gk, gi = _noalloc(lib, p, n, stream)
        # integer outputs: exact, like every integer parity check in these tests
        assert np.array_equal(gk, wk)
        assert np.array_equal(gi, wi)


def test_noalloc_sort_full_size_ragged_and_large_then_small(cuda, pkg):
    """n = MAX_N (every tile of the scratch in use), n ending in a partial
    tile, and a small call right after the largest one."""
    import torch

    lib = pkg._lib.load()
    stream = torch.cuda.current_stream()
    big = pkg.ic.make_cube(MAX_N, seed=3)
    for n in (MAX_N, 100_003, 4_097, MAX_N, 1_000):
        ic = _sub_ic(big, n)
        wk, wi = _sph_sort(pkg, ic)
        gk, gi = _noalloc(lib, big["pos"], n, stream)
        assert np.array_equal(gk, wk), n
        assert np.array_equal(gi, wi), n


def test_noalloc_sort_reports_a_lookback_timeout(cuda, pkg):
    """A look-back wait that gives up (its predecessor's status withheld, a
    short spin limit) is reported by sph_sort_cells_noalloc_health; the next
    call clears it and sorts correctly."""
    import torch

    lib = pkg._lib.load()
    stream = torch.cuda.current_stream()
    assert lib.sph_selftest_lookback_timeout(None, 1000, C.c_void_p(stream.cuda_stream)) == 0
    rc, w = _health(lib, stream)
    assert rc == SPH_ERR_TIMEOUT and (w & 0x1), (rc, hex(w))
    ic = pkg.ic.make_impact(4096, 1024, seed=2)
    wk, wi = _sph_sort(pkg, ic)
    gk, gi = _noalloc(lib, ic["pos"], int(ic["n"]), stream)
    assert np.array_equal(gk, wk) and np.array_equal(gi, wi)


def test_noalloc_sort_rejects_sizes_beyond_its_scratch(cuda, pkg):
    import torch

    lib = pkg._lib.load()
    buf = torch.zeros(3, dtype=torch.float32, device="cuda")
    out = torch.zeros(1, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream()
    assert _call(lib, buf, MAX_N + 1, out, out, stream) == 1
    assert b"outside 0..262144" in lib.sph_last_error()
    assert _call(lib, buf, -1, out, out, stream) == 1
    assert _call(lib, buf, 0, out, out, stream) == 0
