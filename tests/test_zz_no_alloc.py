"""The allocation-free cell sort, sph_sort_cells_noalloc.

It exists for callers that may not allocate device memory themselves: code
running inside a framework that owns every device allocation, or code on a
latency-critical thread that must not call cudaMalloc/cudaFree because those
can synchronise the device.  It must give exactly the sorted (cell key,
particle index) pairs of the context-based sph_sort, call after call, even
though every call reuses the same fixed scratch array inside the library.

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


def _call(lib, dpos, n, keys, idx, stream):
    return lib.sph_sort_cells_noalloc(C.c_void_p(dpos.data_ptr()), int(n), C.c_void_p(keys.data_ptr()),
                                      C.c_void_p(idx.data_ptr()), C.c_void_p(stream.cuda_stream))


def test_noalloc_sort_matches_sph_sort_on_two_calls_in_a_row(cuda, pkg):
    import torch

    lib = pkg._lib.load()
    ic = pkg.ic.make_impact(16384, 4096, seed=0)
    n = int(ic["n"])
    inputs = (ic["pos"], ic["pos"] + np.float32(0.37))  # the second call sees other cells
    want = []
    with pkg.Compute(ic, tree_source="host") as c:
        for p in inputs:
            c.upload("pos", p)
            c.sort()
            c.synchronize()
            want.append((c.download("cell_key"), c.download("cell_index")))
    stream = torch.cuda.current_stream()
    keys = torch.empty(n, dtype=torch.int32, device="cuda")
    idx = torch.empty(n, dtype=torch.int32, device="cuda")
    for p, (wk, wi) in zip(inputs, want):
        dpos = torch.from_numpy(np.ascontiguousarray(p, dtype=np.float32).reshape(-1)).cuda()
        keys.fill_(-1)
        idx.fill_(-1)
        assert _call(lib, dpos, n, keys, idx, stream) == 0, lib.sph_last_error()
        torch.cuda.synchronize()
        # integer outputs: exact, like every integer parity check in these tests
        assert np.array_equal(keys.cpu().numpy().view(np.uint32), wk)
        assert np.array_equal(idx.cpu().numpy().view(np.uint32), wi)


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
